// gr_kernels.cuh -- kernels of the routing hot path (sm_100a).
//
// Once per design:
//   k_coords_warp / k_coords_block  sorted distinct x and y of every net's pins
// Once per route (reset):
//   k_fen_init     Fenwick nodes from the capacities      (bit_util.hpp:56-74)
// Per batch:
//   k_qtable       per-net query tables (exact Fenwick prefix queries)
//   k_lpat_z<Z>    L-pattern argmin of every pin pair       (bit_util.hpp:119-191)
//                  (k_lpat_batch for Z > 16, k_lpat_pairs for explicit pair lists)
//   k_mst_pin2     Boruvka of 2-pin nets, one thread each     (gmst_util.hpp:164-341)
//   k_mst_warp     Boruvka of 3..32-pin nets, one warp each
//   k_mst_large    Boruvka of larger nets, one CTA each
//   k_mst_cluster  Boruvka of nets whose cost matrix needs a 4- or 8-CTA cluster
//                  (the L-pattern and tree kernels also mark the GCELLs of
//                  every MST edge they settle, batch-deduped in a bitmap,
//                  mst_bit_commit.hpp:81-235; k_mark does it for trees
//                  built elsewhere)
//   k_track_commit per routing track: demand += 1 per marked cell and the
//                  Fenwick node updates, one owner per node   (bit_util.hpp:75-90)
#pragma once
#include <cooperative_groups.h>

#include "gr_device.cuh"

namespace cg = cooperative_groups;

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
    const int32_t *order;     // [n] net indices: 2-pin nets, then 3..32 pins, then larger
    const int32_t *nxy;       // [n] (distinct x count << 16) | distinct y count; 0: no table
    int64_t n_pairs, n_nodes, n_tab;
    int32_t max_pins;
    int32_t n2, nm, nl;       // sizes of the three classes in `order`
    int32_t nmid;             // of the nl larger nets, the first nmid have at most 128 pins
};

// Per design pin (indexed like the pin array): the pin's index into its net's
// sorted distinct x and y lists, packed (xi << 16) | yi; and the lists
// themselves, stored from the net's first pin slot on.
struct Coords {
    const int32_t *pxy;
    const int32_t *cx;
    const int32_t *cy;
};

// ---------------------------------------------------------------- coordinate tables
// Per net: the sorted distinct x and y coordinates of its pins and each pin's
// index into them (nxy[net] = (nx << 16) | ny, 0 when the table would exceed
// kTableMaxCells). Nets of up to 32 pins: one warp each, pin = lane.
__global__ void __launch_bounds__(256) k_coords_warp(GridC g, int32_t n_nets, const int64_t *__restrict__ pin_ofs,
                                                     const int32_t *__restrict__ pins, int32_t *__restrict__ pxy,
                                                     int32_t *__restrict__ cx, int32_t *__restrict__ cy,
                                                     int32_t *__restrict__ nxy) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= n_nets) return;
    const int64_t o = pin_ofs[warp];
    const int n = (int)(pin_ofs[warp + 1] - o);
    if (n > 32) return;
    int x = 0x7fffffff, y = 0x7fffffff;  // lanes past the net sort last and are never counted
    if (lane < n) {
        int z;
        dec(g, pins[o + lane], z, x, y);
    }
    const bool fx = (__ffs(__match_any_sync(FULL, x)) - 1) == lane && lane < n;
    const bool fy = (__ffs(__match_any_sync(FULL, y)) - 1) == lane && lane < n;
    int xi = 0, yi = 0;
    for (int b = 0; b < n; b++) {
        const int xb = __shfl_sync(FULL, x, b), yb = __shfl_sync(FULL, y, b);
        const bool fxb = __shfl_sync(FULL, fx, b), fyb = __shfl_sync(FULL, fy, b);
        xi += fxb && xb < x;
        yi += fyb && yb < y;
    }
    const int nx = __popc(__ballot_sync(FULL, fx)), ny = __popc(__ballot_sync(FULL, fy));
    if (lane < n) {
        pxy[o + lane] = (xi << 16) | yi;
        if (fx) cx[o + xi] = x;
        if (fy) cy[o + yi] = y;
    }
    if (lane == 0) nxy[warp] = (int64_t)nx * ny <= kTableMaxCells ? (nx << 16) | ny : 0;
}

// Larger nets: one CTA each (listed in ids), O(n^2) rank counting in shared
// memory.
__global__ void __launch_bounds__(256) k_coords_block(GridC g, const int32_t *__restrict__ ids,
                                                      const int64_t *__restrict__ pin_ofs,
                                                      const int32_t *__restrict__ pins, int32_t *__restrict__ pxy,
                                                      int32_t *__restrict__ cx, int32_t *__restrict__ cy,
                                                      int32_t *__restrict__ nxy) {
    extern __shared__ int cs[];
    __shared__ int s_nx, s_ny;
    const int net = ids[blockIdx.x];
    const int64_t o = pin_ofs[net];
    const int n = (int)(pin_ofs[net + 1] - o);
    int *xs = cs, *ys = cs + n, *fxs = cs + 2 * n, *fys = cs + 3 * n;
    if (threadIdx.x == 0) s_nx = s_ny = 0;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        int z, x, y;
        dec(g, pins[o + a], z, x, y);
        xs[a] = x;
        ys[a] = y;
    }
    __syncthreads();
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        bool fx = true, fy = true;
        for (int b = 0; b < a; b++) {
            fx &= xs[b] != xs[a];
            fy &= ys[b] != ys[a];
        }
        fxs[a] = fx;
        fys[a] = fy;
        if (fx) atomicAdd(&s_nx, 1);
        if (fy) atomicAdd(&s_ny, 1);
    }
    __syncthreads();
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        int xi = 0, yi = 0;
        for (int b = 0; b < n; b++) {
            xi += fxs[b] && xs[b] < xs[a];
            yi += fys[b] && ys[b] < ys[a];
        }
        pxy[o + a] = (xi << 16) | yi;
        if (fxs[a]) cx[o + xi] = xs[a];
        if (fys[a]) cy[o + yi] = ys[a];
    }
    if (threadIdx.x == 0)
        nxy[net] = (int64_t)s_nx * s_ny <= kTableMaxCells ? (s_nx << 16) | s_ny : 0;
}

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

// dlut[c - kLutMin] = cost(c-1) - cost(c) for c = kLutMin .. kLutMax+1, once per context
__global__ void k_dlut(const float *__restrict__ lut, float *__restrict__ dlut) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < kLutMax - kLutMin + 2; c += gridDim.x * blockDim.x)
        dlut[c] = lut_inc(lut, c + kLutMin);
}

// Lookahead cost of a GCELL with remaining capacity c and predicted
// further demand p: exp(-0.5 (c - beta p)), the reference's cost with the
// capacity the remaining batches are expected to leave (no counterpart in
// the reference; the plain cost keeps using the exact table)
__device__ __forceinline__ float la_cost(int c, float p, float beta) { return expf(-0.5f * ((float)c - beta * p)); }

// ---------------------------------------------------------------- Fenwick build
// bit_util.hpp:56-74 builds each node by atomically adding every cell's cost
// along its update path. Here each node is owned by one thread that adds the
// costs of its range (i - lowbit(i), i] in ascending order from 0.
// the same with the lookahead cost (pred in cell order)
__global__ void k_fen_init_la(GridC g, int csize, const int32_t *__restrict__ capr, const float *__restrict__ pred,
                              float beta, float *__restrict__ fen) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < csize; e += gridDim.x * blockDim.x) {
        int z, x, y;
        dec(g, e, z, x, y);
        const int p = (z & 1) ? y : x;
        const int32_t base = e - p;
        const int i = p + 1;
        float res = 0.0f;
        for (int q = i - (i & -i) + 1; q <= i; q++)
            res += la_cost(__ldg(capr + base + q - 1), __ldg(pred + base + q - 1), beta);
        fen[e] = res;
    }
}

// pred[enc(z, x, y)] = src[z][y][x] (the network's grid layout), clamped at 0
__global__ void k_pred_to_cells(GridC g, int csize, const float *__restrict__ src, float *__restrict__ pred) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < csize; e += gridDim.x * blockDim.x) {
        int z, x, y;
        dec(g, e, z, x, y);
        pred[e] = fmaxf(src[((int64_t)z * g.Y + y) * g.X + x], 0.0f);
    }
}

// network input: feat[z][y][x] = demand * scale, feat[Z + z][y][x] = capacity * scale
__global__ void k_features(GridC g, int csize, const int32_t *__restrict__ cap0, const int32_t *__restrict__ capr,
                           float scale, float *__restrict__ feat) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < csize; e += gridDim.x * blockDim.x) {
        int z, x, y;
        dec(g, e, z, x, y);
        const int64_t o = ((int64_t)z * g.Y + y) * g.X + x;
        feat[o] = (float)(cap0[e] - capr[e]) * scale;
        feat[(int64_t)csize + o] = (float)cap0[e] * scale;
    }
}

// the network's output (demand / 16) as predicted further demand: x 16, and
// in excess mode only its part beyond the remaining capacity (from the
// input features: demand / 16 then capacity / 16)
__global__ void k_la_pred(int n, const float *__restrict__ out, const float *__restrict__ feat, int excess,
                          float *__restrict__ pred) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float p = out[i] * 16.0f;
        pred[i] = excess ? fmaxf(p - (feat[n + i] - feat[i]) * 16.0f, 0.0f) : p;
    }
}

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

// Routing tracks (a row of an even layer, a column of an odd layer) are
// numbered layer by layer: layer z starts at track_first(z).
__device__ __forceinline__ int track_first(const GridC &g, int z) { return ((z + 1) >> 1) * g.Y + (z >> 1) * g.X; }

// The same, one warp per routing track (a row of an even layer, a column of
// an odd one; tracks numbered layer by layer from track_first): the track's
// cell costs are staged in shared memory, then the nodes are built level by
// level -- node i (lowbit 2^k) is its left half's node i - 2^(k-1) followed
// by the cells of its right half added one by one in ascending order, the
// same left-to-right sequence of FP32 additions as summing its whole range
// from 0, so every node is bit-identical to k_fen_init's. Shared memory per
// warp: 2 * L floats (costs, nodes); la != 0 uses the lookahead cost.
__global__ void __launch_bounds__(128) k_fen_tracks(GridC g, int n_tracks, int la, const int32_t *__restrict__ capr,
                                                    const float *__restrict__ lut, const float *__restrict__ pred,
                                                    float beta, float *__restrict__ fen) {
    extern __shared__ float fsm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int Lmax = g.X > g.Y ? g.X : g.Y;
    float *cst = fsm + (size_t)wib * 2 * Lmax, *node = cst + Lmax;
    const int t = blockIdx.x * (blockDim.x >> 5) + wib;
    if (t >= n_tracks) return;
    int z = 0;
    while (z + 1 < g.Z && track_first(g, z + 1) <= t) z++;
    const int r = t - track_first(g, z);
    const int L = (z & 1) ? g.Y : g.X;
    const int32_t base = z * g.XY + r * L;
    for (int q = lane; q < L; q += 32) {
        const int32_t e = base + q;
        cst[q] = la ? la_cost(__ldg(capr + e), __ldg(pred + e), beta) : lut_cost(lut, __ldg(capr + e));
    }
    __syncwarp();
    for (int i = 1 + 2 * lane; i <= L; i += 64) node[i - 1] = 0.0f + cst[i - 1];  // lowbit 1
    __syncwarp();
    for (int h = 1; 2 * h <= L; h <<= 1) {  // lowbit 2h: i = 2h (2j + 1)
        for (int i = 2 * h * (2 * lane + 1); i <= L; i += 2 * h * 64) {
            float v = node[i - h - 1];
            for (int q = i - h + 1; q <= i; q++) v += cst[q - 1];
            node[i - 1] = v;
        }
        __syncwarp();
    }
    for (int q = lane; q < L; q += 32) fen[base + q] = node[q];
}

// ---------------------------------------------------------------- plan descriptors
// The SoA descriptor of a whole plan, built on the device from the plan's
// net ids: per net its pin count, first pin and table shape (k_plan_nets),
// then per batch (one CTA) the exclusive prefix sums of pairs, MST slots and
// table entries and the nets' order by size class, batch order kept within
// a class (k_plan_batches) -- the layout the host builder writes for one
// batch.
struct PlanBatch {  // per-batch totals for the host's launch shapes
    int64_t n_pairs, n_nodes, n_tab;
    int32_t max_pins, n2, nm, nmid;
};

__global__ void k_plan_nets(int64_t total, const int32_t *__restrict__ ids, int32_t n_nets,
                            const int64_t *__restrict__ pin_ofs, const int32_t *__restrict__ nxy_net,
                            int64_t *__restrict__ pin_base, int32_t *__restrict__ npin, int32_t *__restrict__ nxy,
                            uint32_t *status) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t id = ids[i];
        if (id < 0 || id >= n_nets) {
            atomicOr(status, 1u);
            id = 0;  // keeps the descriptor in bounds; the host rejects the plan
        }
        const int64_t o = pin_ofs[id];
        pin_base[i] = o;
        npin[i] = (int32_t)(pin_ofs[id + 1] - o);
        nxy[i] = nxy_net[id];
    }
}

// exclusive prefix of three int64 values over the block (blockDim.x a
// multiple of 32, at most 1024); totals returned in t0..t2
__device__ __forceinline__ void block_excl_scan3(int64_t &a, int64_t &b, int64_t &c, int64_t &t0, int64_t &t1,
                                                 int64_t &t2, int64_t (*wsum)[3]) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int64_t x = a, y = b, z = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t xo = __shfl_up_sync(FULL, x, o), yo = __shfl_up_sync(FULL, y, o), zo = __shfl_up_sync(FULL, z, o);
        if (lane >= o) x += xo, y += yo, z += zo;
    }
    if (lane == 31) wsum[warp][0] = x, wsum[warp][1] = y, wsum[warp][2] = z;
    __syncthreads();
    if (warp == 0) {
        int64_t u = lane < nw ? wsum[lane][0] : 0, v = lane < nw ? wsum[lane][1] : 0, w = lane < nw ? wsum[lane][2] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t uo = __shfl_up_sync(FULL, u, o), vo = __shfl_up_sync(FULL, v, o), wo = __shfl_up_sync(FULL, w, o);
            if (lane >= o) u += uo, v += vo, w += wo;
        }
        if (lane < nw) wsum[lane][0] = u, wsum[lane][1] = v, wsum[lane][2] = w;  // inclusive over warps
    }
    __syncthreads();
    const int64_t p0 = warp ? wsum[warp - 1][0] : 0, p1 = warp ? wsum[warp - 1][1] : 0, p2 = warp ? wsum[warp - 1][2] : 0;
    t0 = wsum[nw - 1][0];
    t1 = wsum[nw - 1][1];
    t2 = wsum[nw - 1][2];
    a = p0 + x - a;
    b = p1 + y - b;
    c = p2 + z - c;
    __syncthreads();  // wsum free for the next call
}

__global__ void __launch_bounds__(1024) k_plan_batches(const int64_t *__restrict__ bofs, int Z, int warp_pins,
                                                       int mid_pins, const int32_t *__restrict__ npin,
                                                       const int32_t *__restrict__ nxy, int64_t *__restrict__ pair_ofs,
                                                       int64_t *__restrict__ node_ofs, int64_t *__restrict__ tab_ofs,
                                                       int32_t *__restrict__ order, PlanBatch *__restrict__ out) {
    __shared__ int64_t wsum[32][3];
    __shared__ int wcnt[4][32];
    __shared__ int s_max;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int64_t first = bofs[blockIdx.x];
    const int n = (int)(bofs[blockIdx.x + 1] - first);
    auto cls = [&](int k) { return k == 2 ? 0 : (k <= warp_pins ? 1 : (k <= mid_pins ? 2 : 3)); };
    if (tid == 0) s_max = 0;
    __syncthreads();
    // pass 1: offsets, class counts, largest net
    int64_t P = 0, Mn = 0, T = 0;
    int c0 = 0, c1 = 0, c2 = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + tid;
        int64_t a = 0, b = 0, c = 0;
        int k = 0;
        if (i < n) {
            k = npin[first + i];
            const int q = nxy[first + i];
            a = (int64_t)k * (k - 1) / 2;
            b = k;
            c = (int64_t)Z * (q >> 16) * (q & 0xffff);
            atomicMax(&s_max, k);
        }
        int64_t ta, tb, tc;
        block_excl_scan3(a, b, c, ta, tb, tc, wsum);
        if (i < n) {
            pair_ofs[first + i] = P + a;
            node_ofs[first + i] = Mn + b;
            tab_ofs[first + i] = T + c;
        }
        P += ta;
        Mn += tb;
        T += tc;
        const int q = i < n ? cls(k) : -1;
        c0 += __syncthreads_count(q == 0);
        c1 += __syncthreads_count(q == 1);
        c2 += __syncthreads_count(q == 2);
    }
    // pass 2: stable partition by class
    int run[4] = {0, c0, c0 + c1, c0 + c1 + c2};
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + tid;
        const int q = i < n ? cls(npin[first + i]) : -1;
        unsigned m[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            m[r] = __ballot_sync(FULL, q == r);
            if (lane == 0) wcnt[r][warp] = __popc(m[r]);
        }
        __syncthreads();
        if (tid < 4) {  // exclusive prefix over the warps, per class
            int acc = 0;
            for (int w = 0; w < nw; w++) {
                const int v = wcnt[tid][w];
                wcnt[tid][w] = acc;
                acc += v;
            }
        }
        __syncthreads();
        if (q >= 0) order[first + run[q] + wcnt[q][warp] + __popc(m[q] & ((1u << lane) - 1))] = i;
#pragma unroll
        for (int r = 0; r < 4; r++) run[r] += __syncthreads_count(q == r);
    }
    if (tid == 0) {
        PlanBatch pb;
        pb.n_pairs = P;
        pb.n_nodes = Mn;
        pb.n_tab = T;
        pb.max_pins = s_max;
        pb.n2 = c0;
        pb.nm = c1;
        pb.nmid = c2;
        out[blockIdx.x] = pb;
    }
}

// ---------------------------------------------------------------- marking
// The GCELLs of one committed edge (mst_bit_commit.hpp:36-67, 209-231): a
// layer change covers its interior layers, a wire its inclusive span. Each
// cell is visited once: V::span(first id, count) for a wire (ids contiguous
// along the track), V::cell(id) for a via cell. Only stacked pins (same x
// and y) can revisit a cell -- the two layer changes and the one-cell wire
// share a column -- so that case visits the union of their layers.
__device__ __forceinline__ uint64_t layer_interior(int a, int b) {
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi - lo < 2) return 0;
    return ((1ull << hi) - 1) & ~((1ull << (lo + 1)) - 1);
}

template <class V>
__device__ __forceinline__ bool walk_edge(const GridC &g, int z1, int x1, int y1, int z2, int x2, int y2, int cpat,
                                          V &vis) {
    const int via1 = cpat / g.Z2, v = cpat % g.Z2;
    const bool bth = (x1 != x2 && y1 != y2);
    const int via2 = (via1 & 1) ? 2 * v : 2 * v + 1;
    if (cpat < 0 || via1 < 1 || via1 >= g.Z || (bth && via2 != 0 && via2 >= g.Z)) return false;
    // The reference's marking kernel walks the first wire also for the
    // threads of the first layer change's d interior cells, whose local
    // index is then -d..-1 (the one call not guarded by tid >= 0,
    // mst_bit_commit.hpp:216): they mark the d cells below the wire's lower
    // end -- cell ids first-d .. first-1 of the wire's track, or the end of
    // the previous track when that end is at coordinate 0.
    const int d = z1 == via1 ? 0 : (z1 < via1 ? via1 - z1 : z1 - via1) - 1;
    if (x1 == x2 && y1 == y2) {
        uint64_t m = layer_interior(z1, via1) | (1ull << via1) | layer_interior(via1, z2);
        while (m) {
            const int i = __ffsll((long long)m) - 1;
            m &= m - 1;
            vis.cell(enc(g, i, x1, y1));
        }
        if (d > 0) vis.span(enc(g, via1, x1, y1) - d, d);
        return true;
    }
    auto via = [&](int za, int zb) {
        const int lo = za < zb ? za : zb, hi = za < zb ? zb : za;
        for (int i = lo + 1; i < hi; i++) vis.cell(enc(g, i, x1, y1));
    };
    auto wire = [&](int z) {
        if (z & 1) {
            const int lo = min(y1, y2), hi = max(y1, y2);
            vis.span(z * g.XY + x1 * g.Y + lo, hi - lo + 1);
            y1 = y2;
        } else {
            const int lo = min(x1, x2), hi = max(x1, x2);
            vis.span(z * g.XY + y1 * g.X + lo, hi - lo + 1);
            x1 = x2;
        }
    };
    if (z1 != via1) {
        via(z1, via1);
        z1 = via1;
    }
    if (d > 0) vis.span(((z1 & 1) ? z1 * g.XY + x1 * g.Y + min(y1, y2) : z1 * g.XY + y1 * g.X + min(x1, x2)) - d, d);
    wire(z1);
    if (bth && via2 != 0 && z1 != via2) {
        via(z1, via2);
        z1 = via2;
        wire(z1);
    }
    if (z1 != z2) via(z1, z2);
    return x1 == x2 && y1 == y2;
}

// Where the marking of a batch's MST edges goes: one bit per GCELL in `mark`
// (the commit then adds one unit of demand to every marked cell: a GCELL
// gains at most one unit per batch, mst_bit_commit.hpp:36-67, 236-255), and
// each MST slot's pattern in mst_pat (-1 for sentinels; may be null). ppat:
// the batch's pair patterns; pins: the design's pins. mark == null: the
// trees are built without marking (the brvsk_build boundary).
struct MarkOut {
    uint32_t *mark;
    int32_t *mst_pat;
    const int16_t *ppat;
    const int32_t *pins;
};

// walk_edge visitor: ORs the path's GCELL bits into the bitmap. The old
// words are not needed, so the ORs are fire-and-forget reductions.
struct RedMark {
    uint32_t *mark;
    __device__ void cell(int32_t e) { atomicOr(mark + (e >> 5), 1u << (e & 31)); }
    __device__ void span(int32_t e0, int cnt) {
        const int32_t e1 = e0 + cnt - 1, w0 = e0 >> 5, w1 = e1 >> 5;
        for (int32_t w = w0; w <= w1; w++) {
            uint32_t m = 0xffffffffu;
            if (w == w0) m &= 0xffffffffu << (e0 & 31);
            if (w == w1) m &= 0xffffffffu >> (31 - (e1 & 31));
            atomicOr(mark + w, m);
        }
    }
};

// Marks MST slot `slot` of the batch: the edge between pins u and v of batch
// net `net` (v < 0: a sentinel). As in mst_bit_commit.hpp:81-105 the larger
// pin index is the source, the pair's pattern the path (bit_util.hpp:134-180
// walked by mst_bit_commit.hpp:147-235).
__device__ __forceinline__ void mark_edge_slot(const GridC &g, const BatchView &bv, const MarkOut &mo, int net,
                                               int64_t slot, int u, int v, uint32_t *status) {
    if (v < 0) {
        if (mo.mst_pat) mo.mst_pat[slot] = -1;
        return;
    }
    const int n1 = u > v ? u : v, n2 = u > v ? v : u;
    const int cpat = mo.ppat[bv.pair_ofs[net] + (int64_t)n1 * (n1 - 1) / 2 + n2];
    if (mo.mst_pat) mo.mst_pat[slot] = cpat;
    const int32_t *np = mo.pins + bv.pin_base[net];
    int z1, x1, y1, z2, x2, y2;
    dec(g, __ldg(np + n1), z1, x1, y1);
    dec(g, __ldg(np + n2), z2, x2, y2);
    RedMark rm{mo.mark};
    if (!walk_edge(g, z1, x1, y1, z2, x2, y2, cpat, rm)) atomicOr(status, 0x2u);
}

// The recorded slots of one net, read back from `out` (written by the
// calling threads before a barrier), marked by threads t0, t0 + stride, ...
__device__ __forceinline__ void mark_net_slots(const GridC &g, const BatchView &bv, const MarkOut &mo, int net,
                                               const int64_t *out, int n, int t0, int stride, uint32_t *status) {
    const int64_t o = bv.node_ofs[net];
    for (int s = t0; s < n; s += stride) {
        const int64_t E = out[s];
        mark_edge_slot(g, bv, mo, net, o + s, E < 0 ? -1 : (int)((E >> 15) & 0x7fff), E < 0 ? -1 : (int)(E & 0x7fff),
                       status);
    }
}

// ---------------------------------------------------------------- query table
// Entry (z, a, b) of a net's table: the two prefix queries at (x_a, y_b) on
// layer z along the layer's direction (x on even layers, y on odd ones).
__global__ void k_qtable(GridC g, BatchView bv, Coords cd, const float *__restrict__ fen, float2 *__restrict__ tab) {
    const int lane = threadIdx.x & 31;
    for (int64_t t0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); t0 < bv.n_tab;
         t0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = t0 + lane;
        const int net = warp_ofs_window(bv.tab_ofs, bv.n, warp_ofs_search(bv.tab_ofs, bv.n, t0, lane),
                                        t < bv.n_tab ? t : bv.n_tab - 1, lane);
        if (t >= bv.n_tab) continue;
        const int64_t local = t - bv.tab_ofs[net];
        const int nxy = bv.nxy[net], nx = nxy >> 16, ny = nxy & 0xffff;
        const int per = nx * ny;
        const int z = (int)(local / per);
        const int r = (int)(local - (int64_t)z * per);
        const int a = r / ny, b = r - a * ny;
        const int64_t pb = bv.pin_base[net];
        const int x = __ldg(cd.cx + pb + a), y = __ldg(cd.cy + pb + b);
        const int32_t base = track_base(g, z, x, y);
        tab[t] = fen_query_pair(fen, base, (z & 1) ? y : x);
    }
}

// ---------------------------------------------------------------- L-pattern
// A 2-pin net's tree is its single pair: written by the L-pattern kernels in
// the fused route (same slots as k_mst_pin2: root 0 records (0, 1)), and its
// path marked there (pin 1 at (z1, x1, y1) is the source, pattern cp).
__device__ __forceinline__ void pin2_tree(const GridC &g, const BatchView &bv, const MarkOut &mo, int net, float c,
                                          int cp, int z1, int x1, int y1, int z2, int x2, int y2,
                                          int64_t *__restrict__ mst, float *__restrict__ dist, uint32_t *status) {
    if (!mst || bv.npin[net] != 2) return;
    const int64_t o = bv.node_ofs[net];
    mst[o] = ((int64_t)net << 30) | 1;
    mst[o + 1] = -1;
    if (dist) dist[net] = c;
    if (mo.mark) {
        if (mo.mst_pat) {
            mo.mst_pat[o] = cp;
            mo.mst_pat[o + 1] = -1;
        }
        RedMark rm{mo.mark};
        if (!walk_edge(g, z1, x1, y1, z2, x2, y2, cp, rm)) atomicOr(status, 0x2u);
    }
}

__global__ void __launch_bounds__(256) k_lpat_batch(GridC g, BatchView bv, const int32_t *__restrict__ pins,
                                                    Coords cd, const float *__restrict__ fen,
                                                    const float2 *__restrict__ tab,
                                                    float *__restrict__ cost, int16_t *__restrict__ pat,
                                                    int64_t *__restrict__ mst, float *__restrict__ dist, MarkOut mo,
                                                    uint32_t *status) {
    const int lane = threadIdx.x & 31;
    for (int64_t p0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); p0 < bv.n_pairs;
         p0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = p0 + lane;
        const int net = warp_ofs_window(bv.pair_ofs, bv.n, warp_ofs_search(bv.pair_ofs, bv.n, p0, lane),
                                        p < bv.n_pairs ? p : bv.n_pairs - 1, lane);
        if (p >= bv.n_pairs) continue;
        int j, k;
        pair_decode(p - bv.pair_ofs[net], j, k);
        const int32_t *np = pins + bv.pin_base[net];
        int z1, x1, y1, z2, x2, y2;
        dec(g, __ldg(np + j), z1, x1, y1);
        dec(g, __ldg(np + k), z2, x2, y2);
        float c;
        int cp;
        const int nxy = bv.nxy[net];
        if (nxy) {
            const int pj = __ldg(cd.pxy + bv.pin_base[net] + j), pk = __ldg(cd.pxy + bv.pin_base[net] + k);
            TableEv ev;
            ev.tab = tab + bv.tab_ofs[net];
            ev.nx = nxy >> 16;
            ev.ny = nxy & 0xffff;
            ev.xij = pj >> 16;
            ev.yij = pj & 0xffff;
            ev.xik = pk >> 16;
            ev.yik = pk & 0xffff;
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
        pin2_tree(g, bv, mo, net, c, cp, z1, x1, y1, z2, x2, y2, mst, dist, status);
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
// Barrier of the first nt threads of the block (nt a multiple of 32): the
// whole block's barrier when nt is the block size, else named barrier 1.
__device__ __forceinline__ void sync_first(int nt) {
    if (nt == (int)blockDim.x) __syncthreads();
    else asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
}

// Exclusive scan over the first nt threads of the block (nt a multiple of
// 32, <= 1024); only those threads call it.
__device__ __forceinline__ int block_excl_scan(int v, int *warp_sums, int &total, int nt) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = nt >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    sync_first(nt);
    if (wid == 0) {
        int s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    sync_first(nt);
    int pre = wid > 0 ? warp_sums[wid - 1] : 0;
    total = warp_sums[nw - 1];
    sync_first(nt);
    return pre + x - v;
}

// Threads that run a round's tail: one per pin rounded up to a warp, at
// least 64 and at most 256 (or the block); the rest of the block skips the
// tail's barriers and waits at one block barrier after it.
__device__ __forceinline__ int tail_threads(int n) {
    int t = ((n + 31) >> 5) << 5;
    t = t < 64 ? 64 : (t > 256 ? 256 : t);
    return t < (int)blockDim.x ? t : (int)blockDim.x;
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
// Each pin scans its own pairs and posts one atomicMin to its root, so late
// rounds (few components) see no atomic contention.
__device__ __forceinline__ int64_t pair_id(int a, int b) {
    return a > b ? (int64_t)a * (a - 1) / 2 + b : (int64_t)b * (b - 1) / 2 + a;
}

// Per-pin state of a block-level Boruvka, in shared memory. A root's key,
// the minimum (cost bits, pair id) of its crossing pairs, is kept as two
// 32-bit halves (kb, ki) and found in two passes of 32-bit atomicMin: the
// least cost bits first, then the least pair id among the rows that reach
// them -- the same minimum as one 64-bit key, without 64-bit atomics
// (which contend badly when every row of a round posts to one root).
struct MstArrays {
    uint32_t *kb, *ki;  // per root: cost bits and pair id of its minimum
    int *comp, *sel, *par, *mx, *flag;
    float *wrec;        // costs of a round's recorded edges, in order
    __device__ static MstArrays carve(void *base, int maxn) {
        MstArrays a;
        a.kb = (uint32_t *)base;
        a.ki = a.kb + maxn;
        a.comp = (int *)(a.ki + maxn);
        a.sel = a.comp + maxn;
        a.par = a.sel + maxn;
        a.mx = a.par + maxn;
        a.flag = a.mx + maxn;
        a.wrec = (float *)(a.flag + maxn);
        return a;
    }
    __device__ float *end(int maxn) const { return wrec + maxn; }
    __device__ unsigned long long key(int r) const { return ((unsigned long long)kb[r] << 32) | ki[r]; }
    // a scan's per-row result (cost bits, pair id); sel and par are free
    // until the round's tail writes them
    __device__ uint32_t *row_bits() const { return (uint32_t *)sel; }
    __device__ uint32_t *row_id() const { return (uint32_t *)par; }
};

// One pin's scan: min key over its crossing pairs, as a warp (row = the
// pin's cost bits to every other pin); the row's result is stored and its
// cost bits posted to its root (first pass). Within a row the pair id grows
// with u, so the minimum (cost, pair id) is the minimum (cost bits, u); the
// pair id is formed for the winner only.
__device__ __forceinline__ void mst_scan_row(const MstArrays &a, const uint32_t *row, int v, int n, int lane) {
    const unsigned FULL = 0xffffffffu;
    const int cv = a.comp[v];
    uint32_t bb = ~0u;
    int bu = 0x7fffffff;
    int u = lane;
#pragma unroll 1
    for (; u + 96 < n; u += 128) {
        const uint32_t c0 = row[u], c1 = row[u + 32], c2 = row[u + 64], c3 = row[u + 96];
        const int m0 = a.comp[u], m1 = a.comp[u + 32], m2 = a.comp[u + 64], m3 = a.comp[u + 96];
        if (m0 != cv && c0 < bb) { bb = c0; bu = u; }
        if (m1 != cv && c1 < bb) { bb = c1; bu = u + 32; }
        if (m2 != cv && c2 < bb) { bb = c2; bu = u + 64; }
        if (m3 != cv && c3 < bb) { bb = c3; bu = u + 96; }
    }
    for (; u < n; u += 32) {
        const uint32_t c = row[u];
        if (a.comp[u] != cv && c < bb) { bb = c; bu = u; }
    }
    const uint32_t hi = __reduce_min_sync(FULL, bb);
    const uint32_t wu = __reduce_min_sync(FULL, bb == hi ? (uint32_t)bu : 0xffffffffu);
    if (lane == 0) {
        a.row_bits()[v] = wu < (uint32_t)n ? hi : ~0u;
        a.row_id()[v] = wu < (uint32_t)n ? (uint32_t)pair_id(v, (int)wu) : ~0u;
        if (wu < (uint32_t)n) atomicMin(a.kb + cv, hi);
    }
}

// The same scan for matrices in shared memory (rows r0..r1-1 of the net at
// M + (v - r0) * ld, ld odd), by groups of T threads per row: T the largest
// power of two up to 32 with (r1 - r0) * T <= B threads, thread j of a group
// scanning columns j, j + T, ... and the group combining its (cost bits,
// column) minima by shuffles, ties to the lower column -- the row's minimum
// (cost bits, u) as in mst_scan_row, with fewer dependent steps per thread
// when rows are few and short.
__device__ __forceinline__ void mst_scan_rows_group(const MstArrays &a, const uint32_t *M, int ld, int r0, int r1,
                                                    int n, int tid, int B) {
    const unsigned FULL = 0xffffffffu;
    const int rows = r1 - r0;
    int T = 32;
    while (T > 1 && rows * T > B) T >>= 1;
    const int per = B / T, j = tid & (T - 1), gi = tid / T;
    for (int base = r0; base < r1; base += per) {  // uniform over the block: every lane shuffles
        const int v = base + gi;
        uint32_t bb = ~0u;
        int bu = n;
        if (v < r1) {
            const uint32_t *row = M + (int64_t)(v - r0) * ld;
            const int cv = a.comp[v];
            for (int u = j; u < n; u += T) {
                const uint32_t c = row[u];
                if (a.comp[u] != cv && c < bb) {
                    bb = c;
                    bu = u;
                }
            }
        }
        for (int o = T >> 1; o > 0; o >>= 1) {
            const uint32_t ob = __shfl_xor_sync(FULL, bb, o);
            const int ou = __shfl_xor_sync(FULL, bu, o);
            if (ob < bb || (ob == bb && ou < bu)) {
                bb = ob;
                bu = ou;
            }
        }
        if (v < r1 && j == 0) {
            a.row_bits()[v] = bu < n ? bb : ~0u;
            a.row_id()[v] = bu < n ? (uint32_t)pair_id(v, bu) : ~0u;
            if (bu < n) atomicMin(a.kb + a.comp[v], bb);
        }
    }
}

// Second pass, after a barrier that follows every row's scan: the rows
// v0, v0 + step, ... below v1 that reach their root's least cost bits post
// their pair ids.
__device__ __forceinline__ void mst_post_ids(const MstArrays &a, int v0, int v1, int step) {
    for (int v = v0; v < v1; v += step) {
        const uint32_t b = a.row_bits()[v];
        const int cv = a.comp[v];
        if (b != ~0u && b == a.kb[cv]) atomicMin(a.ki + cv, a.row_id()[v]);
    }
}

// The rest of a round once a.key holds every root's minimum (gmst_util.hpp:
// 215-341): select the other side, record every candidate except the larger
// root of each mutual pair in ascending root order (written to out when out
// is not null), sum their costs into d in that order, and merge. A merged
// component's root is its largest pin index (union points the smaller root
// at the larger one), found by following each candidate's chain to its
// tree's top. Returns the number of edges recorded this round. want_d false
// (the caller keeps no per-net sums) skips the sum, a serial step of one
// thread per round. Run by the first nt threads of the block only (their
// own barriers); the caller synchronises the block afterwards.
__device__ __forceinline__ int mst_round_tail(const MstArrays &a, int n, int net, int nrec, int64_t *out, float &d,
                                              int *warp_sums, uint32_t *status, bool want_d, int nt) {
    const int B = nt, tid = threadIdx.x;
    for (int v = tid; v < n; v += B) {
        int s = -1;
        if (a.comp[v] == v && a.kb[v] != ~0u) {
            int j, k;
            pair_decode((long long)a.ki[v], j, k);
            s = (a.comp[j] == v) ? a.comp[k] : a.comp[j];
        }
        a.sel[v] = s;
    }
    sync_first(nt);
    for (int v = tid; v < n; v += B) {
        const int s = a.sel[v];
        if (s >= 0) {
            const bool mutual_top = (a.sel[s] == v) && (v > s);
            a.flag[v] = mutual_top ? 0 : 1;
            a.par[v] = mutual_top ? v : s;
        } else {
            a.flag[v] = 0;
            a.par[v] = v;
        }
        a.mx[v] = -1;
    }
    sync_first(nt);
    const int chunk = (n + B - 1) / B;
    const int c0 = min(n, tid * chunk), c1 = min(n, c0 + chunk);
    int cnt = 0;
    for (int v = c0; v < c1; v++) cnt += a.flag[v];
    int total;
    int pos = block_excl_scan(cnt, warp_sums, total, nt);
    for (int v = c0; v < c1; v++)
        if (a.flag[v]) {
            if (out) out[nrec + pos] = ((int64_t)net << 30) | ((int64_t)v << 15) | (int64_t)a.sel[v];
            if (want_d) a.wrec[pos] = key_cost(a.key(v));
            pos++;
        }
    sync_first(nt);
    if (want_d && tid == 0) {
        float dd = d;
        for (int i = 0; i < total; i++) dd += a.wrec[i];
        d = dd;
    }
    for (int v = tid; v < n; v += B) {
        if (a.sel[v] < 0) continue;
        int p = v, steps = 0;
        while (a.par[p] != p && steps < n) {
            p = a.par[p];
            steps++;
        }
        if (steps >= n) atomicOr(status, 0x4u);
        a.flag[v] = p;  // flag[] is free again: it now holds the top
        atomicMax(a.mx + p, v);
    }
    sync_first(nt);
    for (int u = tid; u < n; u += B) {
        const int r = a.comp[u];
        if (a.sel[r] >= 0) a.comp[u] = a.mx[a.flag[r]];
    }
    sync_first(nt);
    return total;
}

// One net's Boruvka on the whole CTA. The net's pair costs are first spread
// into a full symmetric n x n matrix M (shared memory when it fits, else this
// CTA's global scratch) so that each pin's crossing scan is one coalesced row
// read by a warp.
__device__ __forceinline__ void mst_block_net(const GridC &g, const BatchView &bv, const MarkOut &mo,
                                              const float *__restrict__ cost, int64_t *__restrict__ mst,
                                              float *__restrict__ dist, uint32_t *status, const MstArrays &a,
                                              uint32_t *M, bool m_smem, int net, int *warp_sums, int *s_total) {
    const int B = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = B >> 5;
    const int n = bv.npin[net], ld = mst_ld(n);
    const long long P = (long long)n * (n - 1) / 2;
    const float *w = cost + bv.pair_ofs[net];
    int64_t *out = mst + bv.node_ofs[net];
    {
        // four independent loads in flight per thread, then their stores;
        // (j, k) steps through the pair ids e, e + B, e + 2B, ...
        int j, k;
        pair_decode(tid, j, k);
        for (long long e = tid; e < P; e += 4 * (long long)B) {
            float c[4];
#pragma unroll
            for (int i = 0; i < 4; i++) c[i] = e + i * B < P ? __ldg(w + e + i * B) : 0.0f;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if (e + i * B < P) {
                    const uint32_t b = cost_bits(c[i]);
                    M[j * ld + k] = b;
                    M[k * ld + j] = b;
                }
                k += B;
                while (k >= j) {
                    k -= j;
                    j++;
                }
            }
        }
    }
    for (int v = tid; v < n; v += B) a.comp[v] = v;
    float d = 0.0f;
    int nrec = 0, rounds = 0;
    __syncthreads();
    while (nrec < n - 1 && rounds < kMstMaxRounds) {
        rounds++;
        for (int v = tid; v < n; v += B) a.kb[v] = a.ki[v] = ~0u;
        __syncthreads();
        if (m_smem) mst_scan_rows_group(a, M, ld, 0, n, n, tid, B);
        else
            for (int v = warp; v < n; v += nw) mst_scan_row(a, M + (int64_t)v * ld, v, n, lane);
        __syncthreads();
        mst_post_ids(a, tid, n, B);
        __syncthreads();
        {
            const int nt = tail_threads(n);
            int t = 0;
            if (tid < nt) t = mst_round_tail(a, n, net, nrec, out, d, warp_sums, status, dist != nullptr, nt);
            if (tid == 0) *s_total = t;
            __syncthreads();  // the merge visible to every warp
            nrec += *s_total;
        }
    }
    for (int v = nrec + tid; v < n; v += B) out[v] = -1;
    if (tid == 0) {
        if (dist) dist[net] = d;
        if (nrec != n - 1) atomicOr(status, 0x4u);
    }
    __syncthreads();
    if (mo.mark) mark_net_slots(g, bv, mo, net, out, n, tid, B, status);  // the tree's slots, thread by thread
}

__global__ void __launch_bounds__(1024) k_mst_large(GridC g, BatchView bv, const float *__restrict__ cost,
                                                   int64_t *__restrict__ mst, float *__restrict__ dist,
                                                   uint32_t *status, uint32_t *__restrict__ gmat, int64_t gmat_stride,
                                                   int first, int count, MarkOut mo) {
    extern __shared__ unsigned long long sm[];
    __shared__ int warp_sums[32];
    __shared__ int s_total;
    const int maxn = bv.max_pins;
    const MstArrays a = MstArrays::carve(sm, maxn);
    uint32_t *M = gmat ? gmat + (int64_t)blockIdx.x * gmat_stride : (uint32_t *)a.end(maxn);
    for (int t = blockIdx.x; t < count; t += gridDim.x)
        mst_block_net(g, bv, mo, cost, mst, dist, status, a, M, gmat == nullptr, bv.order[first + t], warp_sums,
                      &s_total);
}

// Nets whose n x n matrix exceeds one CTA's shared memory: a cluster of CS
// CTAs holds it row-distributed. Each CTA scans its own rows into its key[],
// the per-root minima are combined through distributed shared memory, and
// the rest of the round runs identically in every CTA (rank 0 writes).
template <int CS>
__global__ void __launch_bounds__(1024) k_mst_cluster(GridC g, BatchView bv, const float *__restrict__ cost,
                                                     int64_t *__restrict__ mst, float *__restrict__ dist,
                                                     uint32_t *status, int first, int count, MarkOut mo) {
    extern __shared__ unsigned long long sm[];
    __shared__ int warp_sums[32];
    __shared__ int s_total;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int maxn = bv.max_pins;
    unsigned long long *part = sm;  // this CTA's per-root minima over its rows (bits, ids)
    uint32_t *pb = (uint32_t *)part, *pi = pb + maxn;
    const MstArrays a = MstArrays::carve(part + maxn, maxn);
    uint32_t *M = (uint32_t *)a.end(maxn);
    const int B = blockDim.x, tid = threadIdx.x;
    const int ncl = gridDim.x / CS, cid = blockIdx.x / CS;
    for (int t = cid; t < count; t += ncl) {
        const int net = bv.order[first + t];
        const int n = bv.npin[net], ld = mst_ld(n);
        const int rn = (n + CS - 1) / CS, r0 = min(n, rank * rn), r1 = min(n, r0 + rn);
        const float *w = cost + bv.pair_ofs[net];
        // this CTA's rows as cost bits; four independent gathers in flight
        const int cnt = (r1 - r0) * n;
        for (int i0 = tid; i0 < cnt; i0 += 4 * B) {
            float c[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int idx = i0 + i * B;
                const int v = r0 + idx / n, u = idx - (v - r0) * n;
                c[i] = (idx < cnt && u != v) ? __ldg(w + pair_id(v, u)) : 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int idx = i0 + i * B, r = idx / n;
                if (idx < cnt) M[r * ld + (idx - r * n)] = cost_bits(c[i]);
            }
        }
        for (int v = tid; v < n; v += B) a.comp[v] = v;
        float d = 0.0f;
        int nrec = 0, rounds = 0;
        __syncthreads();
        while (nrec < n - 1 && rounds < kMstMaxRounds) {
            rounds++;
            for (int v = tid; v < n; v += B) pb[v] = pi[v] = ~0u;
            __syncthreads();
            const MstArrays ap = {pb, pi, a.comp, a.sel, a.par, a.mx, a.flag, a.wrec};
            mst_scan_rows_group(ap, M, ld, r0, r1, n, tid, B);
            __syncthreads();
            mst_post_ids(ap, r0 + tid, r1, B);
            cl.sync();  // every CTA's partial minima final
            for (int v = tid; v < n; v += B) {
                unsigned long long k = ((unsigned long long)pb[v] << 32) | pi[v];
#pragma unroll
                for (int r = 0; r < CS; r++) {
                    if (r == rank) continue;
                    const unsigned long long o = ((unsigned long long)cl.map_shared_rank(pb, r)[v] << 32) |
                                                 cl.map_shared_rank(pi, r)[v];
                    k = o < k ? o : k;
                }
                a.kb[v] = (uint32_t)(k >> 32);
                a.ki[v] = (uint32_t)k;
            }
            cl.sync();  // remote reads done before the partials are reset
            {
                const int nt = tail_threads(n);
                int tt = 0;
                if (tid < nt)
                    tt = mst_round_tail(a, n, net, nrec, rank == 0 ? mst + bv.node_ofs[net] : nullptr, d, warp_sums,
                                        status, dist != nullptr, nt);
                if (tid == 0) s_total = tt;
                __syncthreads();  // the merge visible to every warp
                nrec += s_total;
            }
        }
        if (rank == 0) {
            int64_t *out = mst + bv.node_ofs[net];
            for (int v = nrec + tid; v < n; v += B) out[v] = -1;
            if (tid == 0) {
                if (dist) dist[net] = d;
                if (nrec != n - 1) atomicOr(status, 0x4u);
            }
        }
        cl.sync();  // rank 0's slots written (cluster-scope release / acquire)
        // the tree's slots marked by every thread of the cluster
        if (mo.mark) mark_net_slots(g, bv, mo, net, mst + bv.node_ofs[net], n, rank * B + tid, CS * B, status);
    }
}

// ---------------------------------------------------------------- L-pattern, per-pair register tables
// A pattern of pair (j -> k) only visits the pins' columns and the two
// corners C1 = (x_k, y_j), C2 = (x_j, y_k). Per layer z the table entries at
// (j,j), (k,k), (k,j), (j,k) give every query it makes:
//   point costs  Pj, Pk, Pc1, Pc2     = Q(pos) - Q(pos-1) at J, K, C1, C2
//   first wire   W1 (from J; even z along row y_j, odd z along column x_j)
//   second wire  W2 (even z: row y_k from C2; odd z: column x_k from C1)
// each the same single FP32 subtraction the reference's range query makes
// (bit_util.hpp:36-38). With Z a compile-time constant the 6Z values stay
// in registers and every pattern is summed in path order from them.
// Patterns of the first-via layers via1 with (via1 - 1) % S == SUB (all of
// them for S = 1): the lowest-cost valid pattern (best, bp; bp = -1 when no
// valid pattern has a finite cost) and the lowest valid pattern id (first).
// Z1F / Z2F >= 0 fix the source / target layer at compile time (the caller
// guarantees z1 == Z1F, z2 == Z2F): every via's layer range is then known to
// the compiler and no addition is predicated on the pins' layers. BTHF >= 0
// fixes whether the pins differ in both x and y (1) or not (0).
template <int ZC, int S, int SUB, int Z1F = -1, int Z2F = -1, int BTHF = -1>
__device__ __forceinline__ void lpat_regs_part(const float2 *__restrict__ T, int nx, int ny, int pj, int pk, int z1_,
                                               int z2_, int xj, int yj, int xk, int yk, float &out_c, int &out_p,
                                               int &out_first) {
    constexpr int Z2 = (ZC + 1) / 2;
    const int z1 = Z1F >= 0 ? Z1F : z1_, z2 = Z2F >= 0 ? Z2F : z2_;
    float Pj[ZC], Pk[ZC], Pc1[ZC], Pc2[ZC], W1[ZC], W2[ZC];
    const int64_t nn = (int64_t)nx * ny;
    const int xij = pj >> 16, yij = pj & 0xffff, xik = pk >> 16, yik = pk & 0xffff;
    const int ojj = xij * ny + yij, okk = xik * ny + yik, okj = xik * ny + yij, ojk = xij * ny + yik;
    const bool xlt = xj < xk, ylt = yj < yk;
    const bool mx = BTHF == 1 ? true : xj != xk, my = BTHF == 1 ? true : yj != yk;
#pragma unroll
    for (int z = 0; z < ZC; z++) {
        const float2 *Tz = T + z * nn;
        const float2 tjj = __ldg(Tz + ojj), tkk = __ldg(Tz + okk), tkj = __ldg(Tz + okj), tjk = __ldg(Tz + ojk);
        Pj[z] = tjj.x - tjj.y;
        Pk[z] = tkk.x - tkk.y;
        Pc1[z] = tkj.x - tkj.y;
        Pc2[z] = tjk.x - tjk.y;
        if (z & 1) {
            W1[z] = ylt ? tjk.x - tjj.y : tjj.x - tjk.y;  // column x_j, y_j -> y_k
            W2[z] = ylt ? tkk.x - tkj.y : tkj.x - tkk.y;  // column x_k from C1
        } else {
            W1[z] = xlt ? tkj.x - tjj.y : tjj.x - tkj.y;  // row y_j, x_j -> x_k
            W2[z] = xlt ? tkk.x - tjk.y : tjk.x - tkk.y;  // row y_k from C2
        }
    }
    const bool bth = BTHF >= 0 ? BTHF == 1 : (mx && my);
    float best = __int_as_float(0x7f800000);
    int bp = -1, first = -1;
#pragma unroll
    for (int via1 = 1; via1 < ZC; via1++) {
        if ((via1 - 1) % S != SUB) continue;
        const bool even1 = (via1 & 1) == 0;
        float c0 = 0.0f;
#pragma unroll
        for (int i = 0; i < ZC; i++) {
            const bool in = z1 < via1 ? (i >= z1 && i < via1) : (i >= via1 && i < z1);
            if (in) c0 += Pj[i];
        }
        if (even1 ? mx : my) c0 += W1[via1];
#pragma unroll
        for (int v = 0; v < Z2; v++) {
            const int cpat = via1 * Z2 + v;
            const int via2 = (via1 & 1) ? 2 * v : 2 * v + 1;
            float c = c0;
            bool valid;
            if (bth && via2 != 0) {
                if (via2 >= ZC) continue;  // odd Z: no layer via2
#pragma unroll
                for (int i = 0; i < ZC; i++) {
                    const bool in = (i >= (via1 < via2 ? via1 : via2)) && (i < (via1 < via2 ? via2 : via1));
                    if (in) c += even1 ? Pc1[i] : Pc2[i];
                }
                c += W2[via2 < ZC ? via2 : 0];
#pragma unroll
                for (int i = 0; i < ZC; i++) {
                    const bool in = via2 < z2 ? (i >= via2 && i < z2) : (i >= z2 && i < via2);
                    if (in) c += Pk[i];
                }
                valid = true;
            } else {
#pragma unroll
                for (int i = 0; i < ZC; i++) {
                    const bool in = via1 < z2 ? (i >= via1 && i < z2) : (i >= z2 && i < via1);
                    if (in) c += even1 ? Pc1[i] : Pc2[i];
                }
                valid = even1 ? !my : !mx;
            }
            if (!valid) continue;
            if (first < 0) first = cpat;
            if (c < best) {
                best = c;
                bp = cpat;
            }
        }
    }
    out_c = best;
    out_p = bp;
    out_first = first;
}

// all patterns of the pair: the cheapest, ties to the lowest id; with no
// finite-cost valid pattern, the lowest valid id at cost +inf
template <int ZC, int Z1F = -1, int Z2F = -1, int BTHF = -1>
__device__ __forceinline__ void lpat_regs(const float2 *__restrict__ T, int nx, int ny, int pj, int pk, int z1,
                                          int z2, int xj, int yj, int xk, int yk, float &out_c, int &out_p) {
    int first;
    lpat_regs_part<ZC, 1, 0, Z1F, Z2F, BTHF>(T, nx, ny, pj, pk, z1, z2, xj, yj, xk, yk, out_c, out_p, first);
    if (out_p < 0) {
        out_p = first;
        out_c = __int_as_float(0x7f800000);
    }
}

// Class of a pair: pins are ascending by cell id within a net, so the source
// (the higher pin) has z1 >= z2. Pairs with both pins on layers 0-1 (where
// pins usually sit) fall in layer classes 0 = (0, 0), 1 = (1, 0), 2 = (1, 1);
// those whose pins differ in both x and y keep it, the others add 3. Class 6
// is every other pair, the pairs of nets without a query table, and every
// pair when Z is not 9 or 10 (the layer counts whose pattern bodies are
// compiled per class).
constexpr int kLpatClasses = 7;
constexpr int kLpatBlock = 256;

template <int ZC>
__device__ __forceinline__ int lpat_class(bool table, int z1, int z2, bool bth) {
    if (!table || (ZC != 9 && ZC != 10)) return 6;
    int l = 3;
    if (z2 == 0 && (z1 == 0 || z1 == 1)) l = z1;
    else if (z1 == 1 && z2 == 1) l = 2;
    return l == 3 ? 6 : l + (bth ? 0 : 3);
}

template <int ZC>
__global__ void __launch_bounds__(kLpatBlock, 3) k_lpat_z(GridC g, BatchView bv, const int32_t *__restrict__ pins,
                                                       Coords cd, const float *__restrict__ fen,
                                                       const float2 *__restrict__ tab, float *__restrict__ cost,
                                                       int16_t *__restrict__ pat, int64_t *__restrict__ mst,
                                                       float *__restrict__ dist, MarkOut mo, uint32_t *status) {
    // Per step a block takes 256 consecutive pairs: each thread decodes one
    // (net by a warp search, pins, layer class), the block regroups them by
    // class in shared memory, and each thread then evaluates the pair at its
    // place in that order -- so a warp mostly holds pairs of one class and
    // runs the pattern body compiled for that class's layers.
    __shared__ int s_wcnt[kLpatBlock / 32][kLpatClasses];  // per warp and class: count, then first place
    __shared__ int32_t s_off[kLpatBlock];                   // place -> pair offset in the step
    __shared__ int32_t s_net[kLpatBlock], s_jk[kLpatBlock];
    __shared__ uint32_t s_xy1[kLpatBlock], s_xy2[kLpatBlock];
    __shared__ int16_t s_zz[kLpatBlock];
    __shared__ int s_valid;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t base = blockIdx.x * (int64_t)kLpatBlock; base < bv.n_pairs;
         base += (int64_t)gridDim.x * kLpatBlock) {
        const int64_t p0 = base + warp * 32, p = p0 + lane;
        int cls = -1, net = 0, j = 0, k = 0, z1 = 0, x1 = 0, y1 = 0, z2 = 0, x2 = 0, y2 = 0;
        if (p0 < bv.n_pairs) {  // warp-uniform
            net = warp_ofs_window(bv.pair_ofs, bv.n, warp_ofs_search(bv.pair_ofs, bv.n, p0, lane),
                                  p < bv.n_pairs ? p : bv.n_pairs - 1, lane);
            if (p < bv.n_pairs) {
                pair_decode(p - bv.pair_ofs[net], j, k);
                const int32_t *np = pins + bv.pin_base[net];
                dec(g, __ldg(np + j), z1, x1, y1);
                dec(g, __ldg(np + k), z2, x2, y2);
                cls = lpat_class<ZC>(bv.nxy[net] != 0, z1, z2, x1 != x2 && y1 != y2);
            }
        }
        unsigned m[kLpatClasses];
#pragma unroll
        for (int q = 0; q < kLpatClasses; q++) {
            m[q] = __ballot_sync(FULL, cls == q);
            if (lane == 0) s_wcnt[warp][q] = __popc(m[q]);
        }
        __syncthreads();
        if (tid == 0) {  // places: class by class, warps in order within a class
            int run = 0;
#pragma unroll
            for (int q = 0; q < kLpatClasses; q++)
                for (int w = 0; w < kLpatBlock / 32; w++) {
                    const int c = s_wcnt[w][q];
                    s_wcnt[w][q] = run;
                    run += c;
                }
            s_valid = run;
        }
        __syncthreads();
        if (cls >= 0) {
            const int at = s_wcnt[warp][cls] + __popc(m[cls] & ((1u << lane) - 1u));
            s_off[at] = warp * 32 + lane;
            s_net[at] = net;
            s_jk[at] = (j << 16) | k;
            s_xy1[at] = ((uint32_t)x1 << 16) | (uint32_t)y1;
            s_xy2[at] = ((uint32_t)x2 << 16) | (uint32_t)y2;
            s_zz[at] = (int16_t)((z1 << 8) | z2);
        }
        __syncthreads();
        if (tid < s_valid) {
            const int64_t q = base + s_off[tid];
            const int n = s_net[tid], jk = s_jk[tid], zz = s_zz[tid];
            const uint32_t a = s_xy1[tid], b = s_xy2[tid];
            const int jj = jk >> 16, kk = jk & 0xffff;
            const int za = zz >> 8, zb = zz & 0xff;
            const int xa = (int)(a >> 16), ya = (int)(a & 0xffff), xb = (int)(b >> 16), yb = (int)(b & 0xffff);
            const int nxy = bv.nxy[n];
            const int c3 = lpat_class<ZC>(nxy != 0, za, zb, xa != xb && ya != yb);
            float c;
            int cp;
            if (!nxy) {
                DirectEv ev{fen, g, za, xa, ya, zb, xb, yb, (xa != xb && ya != yb)};
                lpat_argmin(ev, g, c, cp);
            } else {
                const int64_t pb = bv.pin_base[n];
                const float2 *T = tab + bv.tab_ofs[n];
                const int pj = __ldg(cd.pxy + pb + jj), pk = __ldg(cd.pxy + pb + kk);
                const int nx = nxy >> 16, ny = nxy & 0xffff;
                if constexpr (ZC == 9 || ZC == 10) {
                    switch (c3) {
                        case 0: lpat_regs<ZC, 0, 0, 1>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp); break;
                        case 1: lpat_regs<ZC, 1, 0, 1>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp); break;
                        case 2: lpat_regs<ZC, 1, 1, 1>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp); break;
                        case 3: lpat_regs<ZC, 0, 0, 0>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp); break;
                        case 4: lpat_regs<ZC, 1, 0, 0>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp); break;
                        case 5: lpat_regs<ZC, 1, 1, 0>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp); break;
                        default: lpat_regs<ZC>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp);
                    }
                } else {
                    lpat_regs<ZC>(T, nx, ny, pj, pk, za, zb, xa, ya, xb, yb, c, cp);
                }
            }
            cost[q] = c;
            pat[q] = (int16_t)cp;
            pin2_tree(g, bv, mo, n, c, cp, za, xa, ya, zb, xb, yb, mst, dist, status);
        }
        __syncthreads();  // the shared arrays are refilled by the next step
    }
}

// The same with S warps per group of 32 pairs (for batches too small to fill
// the GPU one thread per pair): warp w evaluates the first-via layers of
// subset w % S for pairs 32 (w / S) .. of the block's share, and the S
// partial results are joined in shared memory -- the cheapest pattern over
// all subsets, ties to the lowest id, else the lowest valid id at +inf.
template <int ZC, int S, int SUB>
__device__ __forceinline__ void lpat_sub(const float2 *T, int nx, int ny, int pj, int pk, int z1, int z2, int xj,
                                         int yj, int xk, int yk, int sub, float &c, int &bp, int &first) {
    if constexpr (SUB < S) {
        if (sub == SUB) lpat_regs_part<ZC, S, SUB>(T, nx, ny, pj, pk, z1, z2, xj, yj, xk, yk, c, bp, first);
        else lpat_sub<ZC, S, SUB + 1>(T, nx, ny, pj, pk, z1, z2, xj, yj, xk, yk, sub, c, bp, first);
    }
}

template <int ZC, int S>
__global__ void __launch_bounds__(256, 2) k_lpat_zs(GridC g, BatchView bv, const int32_t *__restrict__ pins,
                                                 Coords cd, const float *__restrict__ fen,
                                                 const float2 *__restrict__ tab, float *__restrict__ cost,
                                                 int16_t *__restrict__ pat, int64_t *__restrict__ mst,
                                                 float *__restrict__ dist, MarkOut mo, uint32_t *status) {
    static_assert(S == 2 || S == 4 || S == 8, "warps per pair group");
    __shared__ float sc[8][32];
    __shared__ int sp[8][32], sf[8][32];
    const float inf = __int_as_float(0x7f800000);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, sub = w % S, pg = w / S;
    constexpr int PPB = 32 * (8 / S);  // pairs per block and step
    for (int64_t bb = (int64_t)blockIdx.x * PPB; bb < bv.n_pairs; bb += (int64_t)gridDim.x * PPB) {
        const int64_t p0 = bb + (int64_t)pg * 32, p = p0 + lane;
        float c = inf;
        int bp = -1, first = -1;
        int net = 0;
        int z1 = 0, x1 = 0, y1 = 0, z2 = 0, x2 = 0, y2 = 0;
        if (p0 < bv.n_pairs) {  // warp-uniform
            net = warp_ofs_window(bv.pair_ofs, bv.n, warp_ofs_search(bv.pair_ofs, bv.n, p0, lane),
                                  p < bv.n_pairs ? p : bv.n_pairs - 1, lane);
            if (p < bv.n_pairs) {
                int j, k;
                pair_decode(p - bv.pair_ofs[net], j, k);
                const int32_t *np = pins + bv.pin_base[net];
                dec(g, __ldg(np + j), z1, x1, y1);
                dec(g, __ldg(np + k), z2, x2, y2);
                const int nxy = bv.nxy[net];
                if (nxy) {
                    const int64_t pb = bv.pin_base[net];
                    lpat_sub<ZC, S, 0>(tab + bv.tab_ofs[net], nxy >> 16, nxy & 0xffff, __ldg(cd.pxy + pb + j),
                                       __ldg(cd.pxy + pb + k), z1, z2, x1, y1, x2, y2, sub, c, bp, first);
                } else if (sub == 0) {
                    DirectEv ev{fen, g, z1, x1, y1, z2, x2, y2, (x1 != x2 && y1 != y2)};
                    int cp;
                    lpat_argmin(ev, g, c, cp);
                    first = cp;
                    bp = c < inf ? cp : -1;
                }
            }
        }
        sc[w][lane] = c;
        sp[w][lane] = bp;
        sf[w][lane] = first;
        __syncthreads();
        if (sub == 0 && p < bv.n_pairs) {
            float bc = inf;
            int bbp = -1, bf = -1;
#pragma unroll
            for (int q = 0; q < S; q++) {
                const float qc = sc[w + q][lane];
                const int qp = sp[w + q][lane], qf = sf[w + q][lane];
                if (qp >= 0 && (bbp < 0 || qc < bc || (qc == bc && qp < bbp))) {
                    bc = qc;
                    bbp = qp;
                }
                if (qf >= 0 && (bf < 0 || qf < bf)) bf = qf;
            }
            if (bbp < 0) {
                bbp = bf;
                bc = inf;
            }
            cost[p] = bc;
            pat[p] = (int16_t)bbp;
            pin2_tree(g, bv, mo, net, bc, bbp, z1, x1, y1, z2, x2, y2, mst, dist, status);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- Boruvka, small nets
// Nets of 2 pins: one thread each (the single pair is the tree; the
// reference's first candidate root 0 records (0, 1)).
__global__ void k_mst_pin2(GridC g, BatchView bv, const float *__restrict__ cost, int64_t *__restrict__ mst,
                           float *__restrict__ dist, MarkOut mo, uint32_t *status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bv.n2) return;
    const int i = bv.order[t];
    const int64_t o = bv.node_ofs[i];
    mst[o] = ((int64_t)i << 30) | 1;
    mst[o + 1] = -1;
    if (dist) dist[i] = cost[bv.pair_ofs[i]];
    if (mo.mark) {
        mark_edge_slot(g, bv, mo, i, o, 0, 1, status);
        mark_edge_slot(g, bv, mo, i, o + 1, -1, -1, status);
    }
}

// Nets of 3..32 pins: one warp each, pin = lane, the same per-round rule as
// k_mst_large with the candidate forest resolved by shuffles. skey/scomp: 32
// entries, sw: the net's pair costs (kMstWarpPins * (kMstWarpPins - 1) / 2),
// all in this warp's shared memory.
__device__ __forceinline__ void mst_warp_net(const GridC &g, const BatchView &bv, const MarkOut &mo,
                                             const float *__restrict__ cost, int64_t *__restrict__ mst,
                                             float *__restrict__ dist, uint32_t *status, int i,
                                             unsigned long long *skey, int *scomp, float *sw, int lane) {
    const unsigned FULL = 0xffffffffu;
    const int n = bv.npin[i];
    {
        const float *wg = cost + bv.pair_ofs[i];
        for (int e = lane; e < n * (n - 1) / 2; e += 32) sw[e] = __ldg(wg + e);
        __syncwarp();
    }
    const float *w = sw;
    int64_t *out = mst + bv.node_ofs[i];
    // each root's least (cost bits, pair id) in two 32-bit passes (as in
    // MstArrays): cost bits in skb, then the least pair id among the lanes
    // that reach them in ski
    uint32_t *skb = (uint32_t *)skey, *ski = skb + 32;
    scomp[lane] = lane;
    int nrec = 0;
    float d = 0.0f;
    for (int round = 0; nrec < n - 1 && round < kMstMaxRounds; round++) {
        skb[lane] = ~0u;
        ski[lane] = ~0u;
        __syncwarp();
        const int cv = scomp[lane];
        uint32_t bb = ~0u, be = ~0u;
        if (lane < n) {
            // pair ids grow with u along the row: the first least cost bits win
            for (int u = 0; u < n; u++) {
                if (scomp[u] == cv) continue;
                const uint32_t e = (uint32_t)pair_id(lane, u);
                const uint32_t c = cost_bits(w[e]);
                if (c < bb) {
                    bb = c;
                    be = e;
                }
            }
            if (be != ~0u) atomicMin(&skb[cv], bb);
        }
        __syncwarp();
        if (be != ~0u && bb == skb[cv]) atomicMin(&ski[cv], be);
        __syncwarp();
        int sel = -1;
        const unsigned long long mykey = ((unsigned long long)skb[lane] << 32) | ski[lane];
        if (lane < n && scomp[lane] == lane && skb[lane] != ~0u) {
            int pj, pk;
            pair_decode((long long)ski[lane], pj, pk);
            sel = scomp[pj] == lane ? scomp[pk] : scomp[pj];
        }
        const int sel_of_sel = __shfl_sync(FULL, sel, sel < 0 ? 0 : sel);
        const bool mutual_top = sel >= 0 && sel_of_sel == lane && lane > sel;
        const bool rec = sel >= 0 && !mutual_top;
        const unsigned recm = __ballot_sync(FULL, rec);
        if (rec)
            out[nrec + __popc(recm & ((1u << lane) - 1))] = ((int64_t)i << 30) | ((int64_t)lane << 15) | (int64_t)sel;
        if (dist) {  // the round's costs in lane order (uniform branch)
            const float wv = rec ? w[(uint32_t)mykey] : 0.0f;
            for (int v = 0; v < 32; v++) {
                const float x = __shfl_sync(FULL, wv, v);
                if ((recm >> v) & 1u) d += x;
            }
        }
        nrec += __popc(recm);
        // tops of the candidate trees, then each tree's largest root
        int par = sel >= 0 ? (mutual_top ? lane : sel) : lane;
#pragma unroll
        for (int it = 0; it < 5; it++) par = __shfl_sync(FULL, par, par);
        const unsigned grp = __match_any_sync(FULL, sel >= 0 ? par : 64 + lane);
        const int newroot = 31 - __clz(grp);
        const int r_old = scomp[lane];
        const int sel_r = __shfl_sync(FULL, sel, r_old);
        const int nr_r = __shfl_sync(FULL, newroot, r_old);
        __syncwarp();
        if (lane < n && sel_r >= 0) scomp[lane] = nr_r;
        __syncwarp();
    }
    for (int v = nrec + lane; v < n; v += 32) out[v] = -1;
    if (lane == 0) {
        if (dist) dist[i] = d;
        if (nrec != n - 1) atomicOr(status, 0x4u);
    }
    if (mo.mark) {
        __syncwarp();  // the lanes' slot writes ordered before the reads below
        mark_net_slots(g, bv, mo, i, out, n, lane, 32, status);
    }
}

constexpr int kMstWarpCosts = kMstWarpPins * (kMstWarpPins - 1) / 2;

__global__ void __launch_bounds__(256) k_mst_warp(GridC g, BatchView bv, const float *__restrict__ cost,
                                                  int64_t *__restrict__ mst, float *__restrict__ dist,
                                                  uint32_t *status, MarkOut mo) {
    __shared__ unsigned long long skey[8][32];
    __shared__ int scomp[8][32];
    __shared__ float sw[8][kMstWarpCosts];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int t = blockIdx.x * (blockDim.x >> 5) + wib;
    if (t >= bv.nm) return;
    mst_warp_net(g, bv, mo, cost, mst, dist, status, bv.order[bv.n2 + t], skey[wib], scomp[wib], sw[wib], lane);
}

// ---------------------------------------------------------------- Boruvka, one persistent launch
// Every net of 3 or more pins of a batch in one launch: CTAs take work items
// from a queue (an atomic counter) -- first the nets above kMstWarpPins pins,
// the largest class first, one per item on the whole CTA (mst_block_net),
// then groups of kQueueWarps nets of 3..32 pins, one per warp
// (mst_warp_net). The last CTA to find the queue empty resets the counters
// for the next launch. Shared memory: the block arrays and matrix for the
// batch's largest net, or the warps' arrays, whichever is larger.
constexpr int kQueueThreads = 512, kQueueWarps = kQueueThreads / 32;
constexpr size_t kQueueWarpSmem = (size_t)kQueueWarps * (32 * 8 + 32 * 4 + kMstWarpCosts * 4);

__global__ void __launch_bounds__(kQueueThreads) k_mst_queue(GridC g, BatchView bv, const float *__restrict__ cost,
                                                            int64_t *__restrict__ mst, float *__restrict__ dist,
                                                            uint32_t *status, uint32_t *__restrict__ gmat,
                                                            int64_t gmat_stride, int *__restrict__ queue,
                                                            MarkOut mo) {
    extern __shared__ unsigned long long sm[];
    __shared__ int warp_sums[32];
    __shared__ int s_total, s_item;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int maxn = bv.max_pins;
    const MstArrays a = MstArrays::carve(sm, maxn);
    uint32_t *M = gmat ? gmat + (int64_t)blockIdx.x * gmat_stride : (uint32_t *)a.end(maxn);
    unsigned long long *skey = sm + warp * 32;
    int *scomp = (int *)(sm + kQueueWarps * 32) + warp * 32;
    float *sw = (float *)((int *)(sm + kQueueWarps * 32) + kQueueWarps * 32) + warp * kMstWarpCosts;
    const int nbig = bv.nl - bv.nmid, nlarge = bv.nl;
    const int total = nlarge + (bv.nm + kQueueWarps - 1) / kQueueWarps;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        if (item < nlarge) {  // nets above 128 pins first, then 33..128
            const int t = item < nbig ? bv.nmid + item : item - nbig;
            mst_block_net(g, bv, mo, cost, mst, dist, status, a, M, gmat == nullptr, bv.order[bv.n2 + bv.nm + t],
                          warp_sums, &s_total);
        } else {
            const int t = (item - nlarge) * kQueueWarps + warp;
            if (t < bv.nm)
                mst_warp_net(g, bv, mo, cost, mst, dist, status, bv.order[bv.n2 + t], skey, scomp, sw, lane);
            __syncthreads();
        }
    }
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
            queue[0] = 0;
            queue[1] = 0;
            __threadfence();
        }
    }
}

// ---------------------------------------------------------------- commit
// The marking of a caller's MST slots (the mst_bit_commit boundary, whose
// trees were built elsewhere; the route marks inside the tree kernels): one
// thread per slot of the batch -- its net from the slot offsets, the slot
// checked to be an edge of that net (mst_bit_commit.hpp:81-105) and its path
// marked.
__global__ void __launch_bounds__(256) k_mark(GridC g, BatchView bv, const int64_t *__restrict__ mst, MarkOut mo,
                                              uint32_t *status) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < bv.n_nodes;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int net = ofs_search(bv.node_ofs, bv.n, s);
        const int64_t E = mst[s];
        if (E == -1) {
            if (mo.mst_pat) mo.mst_pat[s] = -1;
            continue;
        }
        const int n = bv.npin[net];
        const int u = (int)((E >> 15) & 0x7fff), v = (int)(E & 0x7fff);
        if ((E >> 30) != net || u >= n || v >= n || u == v) {
            atomicOr(status, 0x1u);
            if (mo.mst_pat) mo.mst_pat[s] = -1;
            continue;
        }
        mark_edge_slot(g, bv, mo, net, s, u, v, status);
    }
}

constexpr int kTrackWarpsMax = 8;  // warps per k_track_commit block
constexpr int kTrackWords = 48;    // mark words per track in the node sweep's rank table
constexpr int kTrackSweepMin = 64; // tracks with more marked cells update by node

// One warp per routing track, every track of the grid (bit_util.hpp:75-90
// for the cells the batch marked on it; a track without marks costs one read
// of its mark words): (1) the marked positions of the track and their
// increments cost(cap-1) - cost(cap) are compacted in ascending order (shared
// memory when the track fits, else the track's slice of a CSIZE scratch),
// each cell's capacity drops by one and its mark bit is cleared; (2) every
// marked cell walks its update path and, for each node where it is the
// highest marked cell of the node's range (i - lowbit(i), i], adds the
// increments of that range's marked cells to the node in ascending order --
// the node's updates in cell order, as a sequential commit makes them. Nodes
// thus have one writer each; the track's cells are touched by this warp alone.
__global__ void __launch_bounds__(256) k_track_commit(GridC g, int n_tracks, uint32_t *mark,
                                                      int32_t *__restrict__ capr, const float *__restrict__ dlut,
                                                      float *__restrict__ fen, int32_t *__restrict__ gpos,
                                                      float *__restrict__ gdel, int cap,
                                                      const float *__restrict__ pred, float beta) {
    extern __shared__ int32_t tsm[];  // per warp: cap positions, then cap increments
    // per warp: the track's mark words and the marked cells before each word
    __shared__ uint32_t s_wm[kTrackWarpsMax][kTrackWords];
    __shared__ int s_wk[kTrackWarpsMax][kTrackWords];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    uint32_t *wm = s_wm[wib];
    int *wk = s_wk[wib];
    int32_t *spos = tsm + (size_t)wib * 2 * cap;
    float *sdel = reinterpret_cast<float *>(spos + cap);
    for (int t = blockIdx.x * wpb + wib; t < n_tracks; t += gridDim.x * wpb) {
        int z = 0;
        while (z + 1 < g.Z && track_first(g, z + 1) <= t) z++;
        const int L = (z & 1) ? g.Y : g.X;
        const int32_t base = z * g.XY + (t - track_first(g, z)) * L;
        const int w0 = base >> 5, w1 = (base + L - 1) >> 5;
        // marked count of the track
        int total = 0;
        for (int w = w0 + lane; w <= w1; w += 32) {
            uint32_t m = mark[w];
            if (w == w0) m &= 0xffffffffu << (base & 31);
            if (w == w1) m &= 0xffffffffu >> (31 - ((base + L - 1) & 31));
            total += __popc(m);
        }
        total = __reduce_add_sync(FULL, total);
        if (total == 0) continue;  // warp-uniform
        int32_t *P = total <= cap ? spos : gpos + base;
        float *D = total <= cap ? sdel : gdel + base;
        // heavily marked tracks update by node (the per-cell walks would
        // chain many dependent node loads on a few lanes); the words must fit
        // the rank table
        const bool sweep = total > kTrackSweepMin && w1 - w0 + 2 <= kTrackWords;
        // (1) compaction in position order
        int run = 0;
        for (int c0 = w0; c0 <= w1; c0 += 32) {
            const int w = c0 + lane;
            uint32_t m = 0;
            if (w <= w1) {
                m = mark[w];
                if (w == w0) m &= 0xffffffffu << (base & 31);
                if (w == w1) m &= 0xffffffffu >> (31 - ((base + L - 1) & 31));
            }
            const int pc = __popc(m);
            int incl = pc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += y;
            }
            int k = run + incl - pc;
            run += __shfl_sync(FULL, incl, 31);
            if (sweep && w <= w1) {
                wm[w - w0] = m;
                wk[w - w0] = k;
            }
            if (m) {
                uint32_t b = m;
                while (b) {
                    P[k++] = (w << 5) + __ffs(b) - 1 - base;
                    b &= b - 1;
                }
                atomicAnd(mark + w, ~m);
            }
        }
        if (sweep && lane == 0) {  // one word past the track: rank(L) = total
            wm[w1 - w0 + 1] = 0;
            wk[w1 - w0 + 1] = total;
        }
        __syncwarp();
        // capacities and increments, lane-parallel with four gathers in flight
        for (int k0 = lane; k0 < total; k0 += 128) {
            int cv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + 32 * u;
                cv[u] = k < total ? capr[base + P[k]] : 0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + 32 * u;
                if (k < total) {
                    const int e = base + P[k];
                    if (pred) {
                        const float pe = __ldg(pred + e);
                        D[k] = la_cost(cv[u] - 1, pe, beta) - la_cost(cv[u], pe, beta);
                    } else {
                        const int c = cv[u];
                        D[k] = __ldg(dlut + (c < kLutMin ? 0 : (c > kLutMax + 1 ? kLutMax + 1 - kLutMin : c - kLutMin)));
                    }
                    capr[e] = cv[u] - 1;
                }
            }
        }
        __syncwarp();
        if (sweep) {
            // (2) node updates by node: every node whose range (i - lowbit(i),
            // i] holds marked cells gets those cells' increments added in
            // cell order (the same sum as below). Lanes take the nodes in
            // rows of 32, rotated by the row so that the large nodes (i a
            // multiple of 32) spread over the warp; a node's marked cells are
            // compacted entries rank(lo) .. rank(i) - 1, read from the word
            // table; eight nodes' loads are in flight per lane.
            const int off = base & 31;
            auto rank = [&](int q) {  // marked cells of the track before position q
                const int e = q + off;
                return wk[e >> 5] + __popc(wm[e >> 5] & ((1u << (e & 31)) - 1u));
            };
            const int rows = (L + 31) >> 5;
            for (int r0 = 0; r0 < rows; r0 += 8) {
                float v[8];
                int a8[8], b8[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int r = r0 + u;
                    const int i = 32 * r + ((lane + r) & 31) + 1;
                    a8[u] = 0;
                    b8[u] = -1;
                    v[u] = 0.0f;
                    if (r < rows && i <= L) {
                        const int ra = rank(i - (i & -i)), rb = rank(i);
                        if (rb > ra) {
                            a8[u] = ra;
                            b8[u] = rb - 1;
                            v[u] = fen[base + i - 1];
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    if (b8[u] < a8[u]) continue;
                    const int r = r0 + u;
                    const int i = 32 * r + ((lane + r) & 31) + 1;
                    float x = v[u];
                    int j = a8[u];
                    const int k = b8[u];
                    for (; j + 8 <= k + 1; j += 8) {
                        float d[8];
#pragma unroll
                        for (int t = 0; t < 8; t++) d[t] = D[j + t];
#pragma unroll
                        for (int t = 0; t < 8; t++) x += d[t];
                    }
                    for (; j <= k; j++) x += D[j];
                    fen[base + i - 1] = x;
                }
            }
        } else
        // (2) node updates, one owner per node. Row r of 32 compacted cells
        // goes to the lanes rotated by r: on a densely marked track the owners
        // of the large nodes (cells 32r+31) then fall on different lanes
        // instead of all on lane 31.
        for (int r = 0; 32 * r < total; r++) {
            const int k = 32 * r + ((lane + r) & 31);
            if (k >= total) continue;
            const int p = P[k];
            const int nxt = k + 1 < total ? P[k + 1] : L;  // next marked position (L: none)
            // this cell's nodes are p+1, then + lowbit, ... while <= nxt (and
            // so <= L); their values are loaded eight at a time before any
            // is updated (no other lane writes them)
            int i = p + 1;
            while (i <= nxt) {
                float v[8];
                int node[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    node[u] = i <= nxt ? i : 0;
                    v[u] = node[u] ? fen[base + i - 1] : 0.0f;
                    if (node[u]) i += i & -i;
                }
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    if (!node[u]) continue;
                    const int lo = node[u] - (node[u] & -node[u]);  // range [lo, node-1], 0-based
                    int a = 0, b = k;                               // first index with P >= lo
                    while (a < b) {
                        const int mid = (a + b) >> 1;
                        if (P[mid] < lo) a = mid + 1;
                        else b = mid;
                    }
                    // the range's increments in cell order, eight loads
                    // ahead of their additions
                    float x = v[u];
                    int j = a;
                    for (; j + 8 <= k + 1; j += 8) {
                        float d[8];
#pragma unroll
                        for (int q = 0; q < 8; q++) d[q] = D[j + q];
#pragma unroll
                        for (int q = 0; q < 8; q++) x += d[q];
                    }
                    for (; j <= k; j++) x += D[j];
                    fen[base + node[u] - 1] = x;
                }
            }
        }
        __syncwarp();
    }
}

}  // namespace gr
