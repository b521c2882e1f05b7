// gr_kernels.cuh -- kernels of the routing hot path (sm_100a).
//
// Per batch:
//   k_qtable      per-net query tables (exact Fenwick prefix queries)
//   k_lpat_batch  L-pattern argmin of every pin pair      (bit_util.hpp:119-191)
//   k_mst         Boruvka spanning tree, one CTA per net   (gmst_util.hpp:164-341)
//   k_mark        GCELLs of every MST edge, batch-deduped   (mst_bit_commit.hpp:81-235)
//   k_fen_update  Fenwick node updates, one owner per node  (bit_util.hpp:75-90)
//   k_finalize    demand += 1 per marked cell, marks cleared
#pragma once
#include "gr_device.cuh"

namespace gr {

// A batch as the kernels see it: per-net arrays, offsets exclusive and local
// to the batch.
struct BatchView {
    int32_t n;                // nets in the batch
    const int32_t *npin;      // [n] pins per net
    const int64_t *pin_base;  // [n] first pin in the design's pin array
    const int64_t *pair_ofs;  // [n] prefix of n(n-1)/2
    const int64_t *node_ofs;  // [n] prefix of n (MST slots)
    const int64_t *tab_ofs;   // [n] prefix of query-table entries
    int64_t n_pairs, n_nodes, n_tab;
    int32_t max_pins;
};

__device__ __forceinline__ float lut_cost(const float *__restrict__ lut, int c) {
    c = c < kLutMin ? kLutMin : (c > kLutMax ? kLutMax : c);
    return __ldg(lut + (c - kLutMin));
}
// bit_util.hpp:16-18: cost(cap - 1) - cost(cap)
__device__ __forceinline__ float lut_inc(const float *__restrict__ lut, int c) {
    float a = lut_cost(lut, c - 1);
    float b = lut_cost(lut, c);
    return a - b;
}

// ---------------------------------------------------------------- Fenwick build
// bit_util.hpp:56-74 builds each node by atomically adding every cell's cost
// along its update path. Here each node is owned by one thread that adds the
// costs of its range (i - lowbit(i), i] in ascending order from 0.
__global__ void k_fen_init(GridC g, int csize, const int32_t *__restrict__ capr, const float *__restrict__ lut,
                           float *__restrict__ fen) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < csize; e += gridDim.x * blockDim.x) {
        int z, x, y;
        dec(g, e, z, x, y);
        int p = (z & 1) ? y : x;
        int32_t base = e - p;
        int i = p + 1;
        int lo = i - (i & -i) + 1;
        float res = 0.0f;
        for (int q = lo; q <= i; q++) res += lut_cost(lut, __ldg(capr + base + q - 1));
        fen[e] = res;
    }
}

// ---------------------------------------------------------------- query table
__global__ void k_qtable(GridC g, BatchView bv, const int32_t *__restrict__ pins, const float *__restrict__ fen,
                         float2 *__restrict__ tab) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < bv.n_tab;
         t += (int64_t)gridDim.x * blockDim.x) {
        int net = ofs_search(bv.tab_ofs, bv.n, t);
        int64_t local = t - bv.tab_ofs[net];
        int n = bv.npin[net];
        int64_t nn = (int64_t)n * n;
        int z = (int)(local / nn);
        int r = (int)(local - z * nn);
        int a = r / n, b = r - a * n;
        const int32_t *np = pins + bv.pin_base[net];
        int za, xa, ya, zb, xb, yb;
        dec(g, __ldg(np + a), za, xa, ya);
        dec(g, __ldg(np + b), zb, xb, yb);
        int32_t base = track_base(g, z, xa, yb);
        int pos = (z & 1) ? yb : xa;
        float2 q;
        q.x = fen_query(fen, base, pos);
        q.y = fen_query(fen, base, pos - 1);
        tab[t] = q;
    }
}

// ---------------------------------------------------------------- L-pattern
__global__ void __launch_bounds__(256) k_lpat_batch(GridC g, BatchView bv, const int32_t *__restrict__ pins,
                                                    const float *__restrict__ fen, const float2 *__restrict__ tab,
                                                    float *__restrict__ cost, int16_t *__restrict__ pat) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < bv.n_pairs;
         p += (int64_t)gridDim.x * blockDim.x) {
        int net = ofs_search(bv.pair_ofs, bv.n, p);
        int n = bv.npin[net];
        int j, k;
        pair_decode(p - bv.pair_ofs[net], j, k);
        const int32_t *np = pins + bv.pin_base[net];
        int z1, x1, y1, z2, x2, y2;
        dec(g, __ldg(np + j), z1, x1, y1);
        dec(g, __ldg(np + k), z2, x2, y2);
        float c;
        int cp;
        if (n <= kTableMaxPins) {
            TableEv ev;
            ev.tab = tab + bv.tab_ofs[net];
            ev.n = n;
            ev.j = j;
            ev.k = k;
            ev.z1 = z1;
            ev.z2 = z2;
            ev.xj = x1;
            ev.yj = y1;
            ev.xk = x2;
            ev.yk = y2;
            ev.bth = (x1 != x2 && y1 != y2);
            lpat_argmin(ev, g, c, cp);
        } else {
            DirectEv ev{fen, g, z1, x1, y1, z2, x2, y2, (x1 != x2 && y1 != y2)};
            lpat_argmin(ev, g, c, cp);
        }
        cost[p] = c;
        pat[p] = (int16_t)cp;
    }
}

// arbitrary pairs (the lpattern boundary)
__global__ void __launch_bounds__(256) k_lpat_pairs(GridC g, int csize, const int32_t *__restrict__ pairs,
                                                    int64_t n_pairs, const float *__restrict__ fen,
                                                    float *__restrict__ cost, int16_t *__restrict__ pat,
                                                    uint32_t *status) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_pairs;
         p += (int64_t)gridDim.x * blockDim.x) {
        int32_t e1 = pairs[2 * p], e2 = pairs[2 * p + 1];
        if (e1 < 0 || e1 >= csize || e2 < 0 || e2 >= csize) {
            atomicOr(status, 0x8u);
            cost[p] = __int_as_float(0x7f800000);
            pat[p] = -1;
            continue;
        }
        int z1, x1, y1, z2, x2, y2;
        dec(g, e1, z1, x1, y1);
        dec(g, e2, z2, x2, y2);
        DirectEv ev{fen, g, z1, x1, y1, z2, x2, y2, (x1 != x2 && y1 != y2)};
        float c;
        int cp;
        lpat_argmin(ev, g, c, cp);
        cost[p] = c;
        pat[p] = (int16_t)cp;
    }
}

// ---------------------------------------------------------------- Boruvka
// Block-wide exclusive scan (blockDim.x multiple of 32, <= 1024).
__device__ __forceinline__ int block_excl_scan(int v, int *warp_sums, int &total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    int pre = wid > 0 ? warp_sums[wid - 1] : 0;
    total = warp_sums[nw - 1];
    __syncthreads();
    return pre + x - v;
}

// One CTA per net. Per round (gmst_util.hpp:518-533):
//   key[r]  = min (cost, pair id) over pairs crossing root r's component
//   sel[r]  = the root on the other side of that pair
// The reference then unions candidates one by one in list order and records
// (r, sel[r]) when r and sel[r] are still apart. With a strict key the
// candidate graph is a forest whose only cycles are mutual pairs, so
// processing roots in ascending order records every candidate except the
// larger root of each mutual pair -- computed here in parallel. A merged
// component's root is its largest pin index (union points the smaller root at
// the larger one), found by pointer jumping to each tree's top.
__global__ void __launch_bounds__(256) k_mst(GridC g, BatchView bv, const float *__restrict__ cost,
                                             int64_t *__restrict__ mst, float *__restrict__ dist,
                                             uint32_t *status) {
    extern __shared__ unsigned long long sm[];
    __shared__ int warp_sums[32];
    __shared__ int s_nrec, s_changed;
    const int maxn = bv.max_pins;
    unsigned long long *key = sm;
    int *comp = (int *)(key + maxn);
    int *sel = comp + maxn;
    int *par = sel + maxn;
    int *mx = par + maxn;
    int *flag = mx + maxn;
    const int B = blockDim.x, tid = threadIdx.x;
    for (int net = blockIdx.x; net < bv.n; net += gridDim.x) {
        const int n = bv.npin[net];
        const int64_t pofs = bv.pair_ofs[net], nofs = bv.node_ofs[net];
        const long long P = (long long)n * (n - 1) / 2;
        const float *w = cost + pofs;
        int64_t *out = mst + nofs;
        if (n == 2) {  // one pair: edge (0,1), the reference's first candidate
            if (tid == 0) {
                out[0] = ((int64_t)net << 30) | 1;
                out[1] = -1;
                if (dist) dist[net] = w[0];
            }
            continue;
        }
        for (int v = tid; v < n; v += B) comp[v] = v;
        if (tid == 0) s_nrec = 0;
        float d = 0.0f;
        int rounds = 0;
        __syncthreads();
        while (s_nrec < n - 1 && rounds < kMstMaxRounds) {
            rounds++;
            for (int v = tid; v < n; v += B) key[v] = ~0ull;
            __syncthreads();
            {
                int j, k;
                pair_decode(tid, j, k);
                for (long long e = tid; e < P; e += B) {
                    int r1 = comp[j], r2 = comp[k];
                    if (r1 != r2) {
                        unsigned long long kk = cost_key(__ldg(w + e), (uint32_t)e);
                        atomicMin(key + r1, kk);
                        atomicMin(key + r2, kk);
                    }
                    k += B;
                    while (k >= j) {
                        k -= j;
                        j++;
                    }
                }
            }
            __syncthreads();
            for (int v = tid; v < n; v += B) {
                int s = -1;
                if (comp[v] == v && key[v] != ~0ull) {
                    int j, k;
                    pair_decode((long long)(uint32_t)key[v], j, k);
                    s = (comp[j] == v) ? comp[k] : comp[j];
                }
                sel[v] = s;
            }
            __syncthreads();
            for (int v = tid; v < n; v += B) {
                int s = sel[v];
                if (s >= 0) {
                    bool mutual_top = (sel[s] == v) && (v > s);
                    flag[v] = mutual_top ? 0 : 1;
                    par[v] = mutual_top ? v : s;
                } else {
                    flag[v] = 0;
                    par[v] = v;
                }
                mx[v] = -1;
            }
            __syncthreads();
            // recorded edges in ascending root order
            {
                const int chunk = (n + B - 1) / B;
                const int c0 = min(n, tid * chunk), c1 = min(n, c0 + chunk);
                int cnt = 0;
                for (int v = c0; v < c1; v++) cnt += flag[v];
                int total;
                int pos = block_excl_scan(cnt, warp_sums, total) + s_nrec;
                for (int v = c0; v < c1; v++)
                    if (flag[v]) out[pos++] = ((int64_t)net << 30) | ((int64_t)v << 15) | (int64_t)sel[v];
                if (tid == 0) {
                    for (int v = 0; v < n; v++)
                        if (flag[v]) d += w[(uint32_t)key[v]];
                }
                __syncthreads();
                if (tid == 0) s_nrec += total;
            }
            // tops of the candidate trees
            while (true) {
                if (tid == 0) s_changed = 0;
                __syncthreads();
                for (int v = tid; v < n; v += B) {
                    int p = par[v], pp = par[p];
                    if (pp != p) {
                        par[v] = pp;
                        s_changed = 1;
                    }
                }
                __syncthreads();
                if (!s_changed) break;
                __syncthreads();
            }
            for (int v = tid; v < n; v += B)
                if (sel[v] >= 0) atomicMax(mx + par[v], v);
            __syncthreads();
            for (int u = tid; u < n; u += B) {
                int r = comp[u];
                if (sel[r] >= 0) comp[u] = mx[par[r]];
            }
            __syncthreads();
        }
        const int nrec = s_nrec;
        for (int v = nrec + tid; v < n; v += B) out[v] = -1;
        if (tid == 0) {
            if (dist) dist[net] = d;
            if (nrec != n - 1) atomicOr(status, 0x4u);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- commit
struct Marker {
    uint32_t *mark;
    int32_t *owned;
    int32_t *owned_count;
    __device__ __forceinline__ void cell(int32_t e) const {
        uint32_t bit = 1u << (e & 31);
        uint32_t old = atomicOr(mark + (e >> 5), bit);
        if (!(old & bit)) owned[atomicAdd(owned_count, 1)] = e;
    }
};

// mst_bit_commit.hpp:36-67: a layer change marks its interior layers, a wire
// marks its inclusive span.
__device__ __forceinline__ void walk_via(const GridC &g, const Marker &m, int za, int zb, int x, int y) {
    int zmin = za < zb ? za : zb, zmax = za < zb ? zb : za;
    for (int i = zmin + 1; i < zmax; i++) m.cell(enc(g, i, x, y));
}
__device__ __forceinline__ void walk_wire(const GridC &g, const Marker &m, int z, int &x, int &y, int x2, int y2) {
    if (z & 1) {
        int lo = min(y, y2), hi = max(y, y2);
        int32_t b = z * g.XY + x * g.Y;
        for (int t = lo; t <= hi; t++) m.cell(b + t);
        y = y2;
    } else {
        int lo = min(x, x2), hi = max(x, x2);
        int32_t b = z * g.XY + y * g.X;
        for (int t = lo; t <= hi; t++) m.cell(b + t);
        x = x2;
    }
}

__global__ void __launch_bounds__(256) k_mark(GridC g, BatchView bv, const int32_t *__restrict__ pins,
                                              const int64_t *__restrict__ mst, const int16_t *__restrict__ ppat,
                                              int32_t *__restrict__ mst_pat, Marker m, uint32_t *status) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < bv.n_nodes;
         s += (int64_t)gridDim.x * blockDim.x) {
        int net = ofs_search(bv.node_ofs, bv.n, s);
        int64_t E = mst[s];
        if (E == -1) {
            if (mst_pat) mst_pat[s] = -1;
            continue;
        }
        const int n = bv.npin[net];
        int n1 = (int)(E & 0x7fff), n2 = (int)((E >> 15) & 0x7fff);
        if ((E >> 30) != net || n1 >= n || n2 >= n || n1 == n2) {
            atomicOr(status, 0x1u);
            if (mst_pat) mst_pat[s] = -1;
            continue;
        }
        if (n1 < n2) {
            int t = n1;
            n1 = n2;
            n2 = t;
        }
        int cpat = ppat[bv.pair_ofs[net] + (int64_t)n1 * (n1 - 1) / 2 + n2];
        if (mst_pat) mst_pat[s] = cpat;
        const int32_t *np = pins + bv.pin_base[net];
        int z1, x1, y1, z2, x2, y2;
        dec(g, __ldg(np + n1), z1, x1, y1);
        dec(g, __ldg(np + n2), z2, x2, y2);
        int via1 = cpat / g.Z2, v = cpat % g.Z2;
        bool bth = (x1 != x2 && y1 != y2);
        int via2 = (via1 & 1) ? 2 * v : 2 * v + 1;
        if (cpat < 0 || via1 < 1 || via1 >= g.Z || (bth && via2 != 0 && via2 >= g.Z)) {
            atomicOr(status, 0x2u);
            continue;
        }
        // mst_bit_commit.hpp:209-231
        if (z1 != via1) {
            walk_via(g, m, z1, via1, x1, y1);
            z1 = via1;
        }
        walk_wire(g, m, z1, x1, y1, x2, y2);
        if (bth && via2 != 0 && z1 != via2) {
            walk_via(g, m, z1, via2, x1, y1);
            z1 = via2;
            walk_wire(g, m, z1, x1, y1, x2, y2);
        }
        if (z1 != z2) walk_via(g, m, z1, z2, x1, y1);
        if (x1 != x2 || y1 != y2) atomicOr(status, 0x2u);
    }
}

__device__ __forceinline__ uint32_t mark_word(const uint32_t *__restrict__ mark, int w, int32_t lo, int32_t hi) {
    uint32_t m = __ldg(mark + w);
    if (w == (lo >> 5)) m &= 0xffffffffu << (lo & 31);
    if (w == (hi >> 5)) m &= 0xffffffffu >> (31 - (hi & 31));
    return m;
}

// For each marked cell at track position p: walk its update path
// (bit_util.hpp:39-55). The cell owns node i while no other marked cell lies
// in (p, i-1]; the owner adds the increments of every marked cell of the
// node's range (i - lowbit(i), i] in ascending cell order. Each node touched
// by the batch thus has exactly one writer and a fixed summation order.
__global__ void __launch_bounds__(256) k_fen_update(GridC g, const int32_t *__restrict__ owned,
                                                    const int32_t *__restrict__ owned_count,
                                                    const uint32_t *__restrict__ mark,
                                                    const int32_t *__restrict__ capr, const float *__restrict__ lut,
                                                    float *__restrict__ fen) {
    const int cnt = *owned_count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int32_t e = owned[t];
        int z, x, y;
        dec(g, e, z, x, y);
        const int p = (z & 1) ? y : x;
        const int L = (z & 1) ? g.Y : g.X;
        const int32_t base = e - p;
        int32_t checked = e;  // no other marked cell in (e, checked]
        for (int i = p + 1; i <= L; i += i & -i) {
            const int32_t top = base + i - 1;
            bool other = false;
            for (int w = (checked + 1) >> 5; w <= (top >> 5) && checked < top; w++)
                if (mark_word(mark, w, checked + 1, top)) {
                    other = true;
                    break;
                }
            if (other) break;
            checked = top;
            const int32_t lo = base + i - (i & -i);
            float v = fen[top];
            for (int w = lo >> 5; w <= (top >> 5); w++) {
                uint32_t mw = mark_word(mark, w, lo, top);
                while (mw) {
                    int bit = __ffs(mw) - 1;
                    mw &= mw - 1;
                    v += lut_inc(lut, __ldg(capr + (w << 5) + bit));
                }
            }
            fen[top] = v;
        }
    }
}

__global__ void k_finalize(const int32_t *__restrict__ owned, const int32_t *__restrict__ owned_count,
                           uint32_t *__restrict__ mark, int32_t *__restrict__ capr) {
    const int cnt = *owned_count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int32_t e = owned[t];
        capr[e] -= 1;
        atomicAnd(mark + (e >> 5), ~(1u << (e & 31)));
    }
}

}  // namespace gr
