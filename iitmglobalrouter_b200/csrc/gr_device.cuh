// gr_device.cuh -- device-side building blocks of the routing hot path.
//
// Grid encoding follows the reference (util.hpp:37-68, WIRE_ENC): every
// routing track (row on even layers, column on odd layers) is contiguous, so
// the Fenwick node i (1-based) of a track lives at cell (track base + i - 1)
// exactly as in bit_util.hpp:19-55.
//
// All floating-point sums are written so that the sequence of IEEE FP32
// additions equals the reference's sequential code (and the CPU oracle):
// prefix queries add nodes from index pos+1 downwards, pattern costs add
// terms in path order. Nothing here may be reassociated.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gr {

constexpr int kLutMin = -256;  // cost LUT covers remaining capacity [-256, 1024]
constexpr int kLutMax = 1024;
constexpr int kTableMaxCells = 1 << 20;  // nx*ny above this: direct Fenwick gathers
constexpr int kMstMaxRounds = 40;
// Row stride of a Boruvka cost matrix: odd, so that one thread per row
// reading column u of consecutive rows hits 32 different shared-memory banks.
__host__ __device__ constexpr int mst_ld(int n) { return n | 1; }
constexpr int kMstWarpPins = 32;   // nets up to this size: one warp each
constexpr int kMaxLayers = 32;     // layer sets are 64-bit masks

struct GridC {
    int X, Y, Z, Z2, npat;
    int XY;
};

__device__ __forceinline__ void dec(const GridC &g, int32_t e, int &z, int &x, int &y) {
    z = e / g.XY;
    int r = e - z * g.XY;
    if (z & 1) {
        x = r / g.Y;
        y = r - x * g.Y;
    } else {
        y = r / g.X;
        x = r - y * g.X;
    }
}

__device__ __forceinline__ int32_t enc(const GridC &g, int z, int x, int y) {
    return (z & 1) ? z * g.XY + x * g.Y + y : z * g.XY + y * g.X + x;
}

// base cell of the track through (z, x, y)
__device__ __forceinline__ int32_t track_base(const GridC &g, int z, int x, int y) {
    return (z & 1) ? z * g.XY + x * g.Y : z * g.XY + y * g.X;
}

// Inclusive prefix query of one track (bit_util.hpp:19-35): nodes from
// index pos+1 down to 1, accumulated in that order starting from 0. The
// node indices depend on pos alone, so up to eight nodes are loaded before
// any is added (the loads overlap instead of each waiting for the previous
// addition); the additions keep the reference's order.
__device__ __forceinline__ float fen_query(const float *__restrict__ fen, int32_t base, int pos) {
    float res = 0.0f;
    int i = pos + 1;
    while (i > 0) {
        float v[8];
        bool on[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            on[k] = i > 0;
            v[k] = on[k] ? __ldg(fen + base + i - 1) : 0.0f;
            i &= i - 1;
        }
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (on[k]) res += v[k];
    }
    return res;
}

// The two prefix queries of one cell's point cost, Q(pos) and Q(pos - 1),
// each summed exactly as fen_query sums it, with their shared nodes loaded
// once. With i = pos + 1 and p = i with its lowest set bit cleared, Q(pos)
// adds node i, then the nodes of p's path; Q(pos - 1) adds the nodes from
// i - 1 down to (not including) p, then the same nodes of p's path.
__device__ __forceinline__ float2 fen_query_pair(const float *__restrict__ fen, int32_t base, int pos) {
    const int i = pos + 1, pre = i & (i - 1);
    float r1 = 0.0f, r2 = 0.0f;
    r1 += __ldg(fen + base + i - 1);
    int k = i - 1;
    while (k > pre) {
        float v[8];
        bool on[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            on[t] = k > pre;
            v[t] = on[t] ? __ldg(fen + base + k - 1) : 0.0f;
            if (on[t]) k &= k - 1;
        }
#pragma unroll
        for (int t = 0; t < 8; t++)
            if (on[t]) r2 += v[t];
    }
    k = pre;
    while (k > 0) {
        float v[8];
        bool on[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            on[t] = k > 0;
            v[t] = on[t] ? __ldg(fen + base + k - 1) : 0.0f;
            k &= k - 1;
        }
#pragma unroll
        for (int t = 0; t < 8; t++)
            if (on[t]) {
                r1 += v[t];
                r2 += v[t];
            }
    }
    return make_float2(r1, r2);
}

// Order-preserving 64-bit key of (cost, pair id): the Boruvka minimum is
// the smallest cost, ties broken by the lowest pair id.
// order-preserving bits of a cost: a < b as floats iff bits(a) < bits(b)
__device__ __forceinline__ uint32_t cost_bits(float w) {
    if (w == 0.0f) w = 0.0f;  // -0 == +0 in the reference's comparisons
    const uint32_t u = __float_as_uint(w);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ unsigned long long cost_key(float w, uint32_t e) {
    return ((unsigned long long)cost_bits(w) << 32) | (unsigned long long)e;
}

// the cost whose key this is (exact inverse of cost_key's order transform)
__device__ __forceinline__ float key_cost(unsigned long long key) {
    uint32_t u = (uint32_t)(key >> 32);
    u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    return __uint_as_float(u);
}

// decode a local pair id e = j(j-1)/2 + k (k < j), gmst_util.hpp:192-194
__device__ __forceinline__ void pair_decode(long long e, int &j, int &k) {
    long long jj = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
    while (jj * (jj - 1) / 2 > e) jj--;
    while ((jj + 1) * jj / 2 <= e) jj++;
    j = (int)jj;
    k = (int)(e - jj * (jj - 1) / 2);
}

// largest i in [0, n) with ofs[i] <= t (ofs ascending, ofs[0] == 0)
__device__ __forceinline__ int ofs_search(const int64_t *__restrict__ ofs, int n, int64_t t) {
    int lo = 0, hi = n;  // invariant: ofs[lo] <= t, answer in [lo, hi)
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(ofs + mid) <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The same search done by a whole warp for a warp-uniform t: each round the
// 32 lanes probe 32 evenly spaced entries and the ballot of "<= t" narrows
// the range 32-fold, so ceil(log32 n) rounds of one load per lane.
__device__ __forceinline__ int warp_ofs_search(const int64_t *__restrict__ ofs, int n, int64_t t, int lane) {
    int lo = 0, hi = n;  // invariant: ofs[lo] <= t, answer in [lo, hi)
    while (hi - lo > 1) {
        const int step = (hi - lo + 31) >> 5;
        const int idx = lo + (lane + 1) * step;
        const unsigned le = __ballot_sync(0xffffffffu, idx < hi && __ldg(ofs + idx) <= t);
        lo += __popc(le) * step;  // probes at or below t form a prefix of the lanes
        hi = min(hi, lo + step);
    }
    return lo;
}

// For lane-varying t >= t0 where i0 answers t0: the answer within the 32
// entries from i0 (one load per lane, then a binary search over the lanes'
// values), or a full search when t lies beyond them. All lanes take part.
__device__ __forceinline__ int warp_ofs_window(const int64_t *__restrict__ ofs, int n, int i0, int64_t t, int lane) {
    const int64_t o = i0 + lane < n ? __ldg(ofs + i0 + lane) : INT64_MAX;
    int lo = 0;
#pragma unroll
    for (int step = 16; step; step >>= 1) {
        const int64_t v = __shfl_sync(0xffffffffu, o, lo + step);
        if (v <= t) lo += step;
    }
    const int i = i0 + lo;
    if (lo == 31 && i + 1 < n && __ldg(ofs + i + 1) <= t) return ofs_search(ofs, n, t);
    return i;
}

// ---------------------------------------------------------------------------
// L-pattern evaluation (bit_util.hpp:134-191), generic over how prefix
// queries are answered. Ev provides:
//   z1, z2, bth                       source layer, target layer, both x and y differ
//   State start()                     position at the source pin
//   void via(za, zb, State, float&)   point costs of layers [min, max) at State
//   void wire(z, State&, float&)      wire on layer z to the target's coordinate
//   bool at_dst(State)
// The pattern loop shares the (via1, first wire) prefix across the ceil(Z/2)
// second-via choices; the prefix value is the same FP32 partial sum the
// reference computes per thread, so costs are unchanged.
template <class Ev>
__device__ __forceinline__ void lpat_argmin(const Ev &ev, const GridC &g, float &out_c, int &out_p) {
    float best = __int_as_float(0x7f800000);
    int bp = -1, first = -1;
    for (int via1 = 1; via1 < g.Z; via1++) {
        typename Ev::State st = ev.start();
        float c0 = 0.0f;
        int zs = ev.z1;
        if (zs != via1) {
            ev.via(zs, via1, st, c0);
            zs = via1;
        }
        ev.wire(zs, st, c0);
        for (int v = 0; v < g.Z2; v++) {
            const int cpat = via1 * g.Z2 + v;
            float c = c0;
            typename Ev::State s2 = st;
            int z = zs;
            const int via2 = (z & 1) ? 2 * v : 2 * v + 1;
            if (ev.bth && via2 != 0) {
                if (via2 >= g.Z) continue;  // odd Z: layer Z does not exist
                if (z != via2) {
                    ev.via(z, via2, s2, c);
                    z = via2;
                    ev.wire(z, s2, c);
                }
            }
            if (z != ev.z2) ev.via(z, ev.z2, s2, c);
            if (!ev.at_dst(s2)) continue;
            if (first < 0) first = cpat;
            if (c < best) {
                best = c;
                bp = cpat;
            }
        }
    }
    if (bp < 0) {
        bp = first;
        best = __int_as_float(0x7f800000);
    }
    out_c = best;
    out_p = bp;
}

// Prefix queries answered straight from the Fenwick array (any pair).
struct DirectEv {
    struct State {
        int x, y;
    };
    const float *fen;
    GridC g;
    int z1, x1, y1, z2, x2, y2;
    bool bth;
    __device__ State start() const { return State{x1, y1}; }
    __device__ float point(int z, int x, int y) const {
        const float2 q = fen_query_pair(fen, track_base(g, z, x, y), (z & 1) ? y : x);
        return q.x - q.y;
    }
    __device__ void via(int za, int zb, State s, float &c) const {
        int zmin = za < zb ? za : zb, zmax = za < zb ? zb : za;
        for (int i = zmin; i < zmax; i++) c += point(i, s.x, s.y);
    }
    __device__ void wire(int z, State &s, float &c) const {
        int32_t b = track_base(g, z, s.x, s.y);
        if (z & 1) {
            if (s.y < y2) {
                float hi = fen_query(fen, b, y2), lo = fen_query(fen, b, s.y - 1);
                c += hi - lo;
            } else if (s.y > y2) {
                float hi = fen_query(fen, b, s.y), lo = fen_query(fen, b, y2 - 1);
                c += hi - lo;
            }
            s.y = y2;
        } else {
            if (s.x < x2) {
                float hi = fen_query(fen, b, x2), lo = fen_query(fen, b, s.x - 1);
                c += hi - lo;
            } else if (s.x > x2) {
                float hi = fen_query(fen, b, s.x), lo = fen_query(fen, b, x2 - 1);
                c += hi - lo;
            }
            s.x = x2;
        }
    }
    __device__ bool at_dst(State s) const { return s.x == x2 && s.y == y2; }
};

// Prefix queries read from a per-net query table. A net's pins have nx
// distinct x and ny distinct y coordinates; for every layer z and indices
// (a, b) into those sorted lists the table holds the pair
//   even z: (Q(z, row y_b, x_a), Q(z, row y_b, x_a - 1))
//   odd  z: (Q(z, col x_a, y_b), Q(z, col x_a, y_b - 1))
// at tab[(z*nx + a)*ny + b]. A pattern of pair (j -> k) only visits the four
// points {x_j, x_k} x {y_j, y_k}, so every query it makes is in the table.
struct TableEv {
    struct State {
        bool ak, bk;  // x taken from pin k (else j), y taken from pin k (else j)
    };
    const float2 *tab;
    int nx, ny, xij, yij, xik, yik;  // coordinate indices of pins j and k
    int z1, z2, xj, yj, xk, yk;
    bool bth;
    __device__ State start() const { return State{false, false}; }
    __device__ float2 t(int z, bool ak, bool bk) const {
        return tab[((int64_t)z * nx + (ak ? xik : xij)) * ny + (bk ? yik : yij)];
    }
    __device__ void via(int za, int zb, State s, float &c) const {
        int zmin = za < zb ? za : zb, zmax = za < zb ? zb : za;
        for (int i = zmin; i < zmax; i++) {
            float2 q = t(i, s.ak, s.bk);
            c += q.x - q.y;
        }
    }
    __device__ void wire(int z, State &s, float &c) const {
        if (z & 1) {
            int yb = s.bk ? yk : yj;
            if (yb < yk) c += t(z, s.ak, true).x - t(z, s.ak, s.bk).y;
            else if (yb > yk) c += t(z, s.ak, s.bk).x - t(z, s.ak, true).y;
            s.bk = true;
        } else {
            int xa = s.ak ? xk : xj;
            if (xa < xk) c += t(z, true, s.bk).x - t(z, s.ak, s.bk).y;
            else if (xa > xk) c += t(z, s.ak, s.bk).x - t(z, true, s.bk).y;
            s.ak = true;
        }
    }
    __device__ bool at_dst(State s) const { return (s.ak ? xk : xj) == xk && (s.bk ? yk : yj) == yk; }
};

}  // namespace gr
