// gr_capi.cu -- host side of the C ABI declared in include/iitmgr_b200.h.
//
// A context owns the grid state on one device and one stream:
//   cap0, capr (int32 remaining capacity), fen (FP32 Fenwick nodes),
//   a one-bit-per-cell mark bitmap and the list of cells marked in a batch.
// Every batch runs as a fixed sequence of kernels on that stream with no
// host synchronisation; batch sizes are known on the host from the design's
// pin offsets, so launches (and captured graphs) need no device readback.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include <omp.h>

#include "../../include/iitmgr_b200.h"
#include "gr_kernels.cuh"

using namespace gr;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// batch descriptor arrays (host or device), SoA
struct DescHost {
    std::vector<int32_t> npin;
    std::vector<int64_t> pin_base, pair_ofs, node_ofs, tab_ofs;
};

struct BatchInfo {  // one batch of a plan
    int64_t first;  // index of its first net in the plan arrays
    int32_t n;
    int64_t n_pairs, n_nodes, n_tab, slot0;
    int32_t max_pins;
    int32_t n2, nm, nl;  // nets of 2 pins, 3..32 pins, more
    int32_t nmid;        // of the nl larger nets, those up to kMstMidPins pins (listed first)
};

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> sig;  // everything the captured launches and copies were built from
    int64_t launches = 0;
};

}  // namespace

struct gr_ctx {
    int device = 0, sm_count = 148;
    GridC g{};
    int64_t csize = 0;
    cudaStream_t stream = nullptr;
    // grid state
    int32_t *d_cap0 = nullptr, *d_capr = nullptr;
    float *d_fen = nullptr, *d_lut = nullptr;
    uint32_t *d_mark = nullptr, *d_status = nullptr;
    DevBuf mat;                            // per-CTA pair-cost matrices of the largest nets
    std::vector<int32_t> h_cap0;
    // design
    int32_t n_nets = 0;
    std::vector<int64_t> h_pin_ofs;
    int32_t *d_pins = nullptr;
    int32_t *d_pxy = nullptr, *d_cx = nullptr, *d_cy = nullptr;  // per-net coordinate indices and lists
    int64_t *d_pin_ofs = nullptr;
    int32_t *d_nxy = nullptr, *d_big = nullptr;
    size_t nets_cap = 0;
    std::vector<int32_t> h_nxy;                                    // per design net: (nx << 16) | ny
    // per-call batch descriptor (device) + pinned staging
    DevBuf desc, pcost, ppat, tab, dist;
    DevBuf out_mst, out_pat;             // results of gr_route_design_host
    DevBuf la_feat, la_out;              // network input and output of the lookahead route
    cudaStream_t copy_stream = nullptr;  // its result copies, overlapping the route
    cudaEvent_t ev_out = nullptr;
    cudaEvent_t ev_copy_done = nullptr;  // result copies joined back to the route's stream
    void *h_stage = nullptr;
    size_t h_stage_bytes = 0;
    cudaEvent_t stage_done = nullptr;
    cudaEvent_t nets_up = nullptr;  // gr_set_nets: the caller's buffers uploaded
    cudaStream_t side[3] = {};       // concurrent Boruvka size classes (graph branches when captured)
    cudaEvent_t ev_fork = nullptr, ev_join[3] = {};
    float *d_dlut = nullptr;  // cost(c-1) - cost(c), c = kLutMin .. kLutMax+1
    // lookahead cost mode: predicted further demand per cell and its weight
    float *d_pred = nullptr;
    float la_beta = 0.0f;
    bool la_on = false;
    int32_t n_tracks = 0;                      // routing tracks: rows of even layers, columns of odd ones
    int track_cap = 0;                         // marked cells per track compacted in shared memory
    int32_t *d_gpos = nullptr;                 // CSIZE scratch for tracks beyond track_cap (long tracks only)
    float *d_gdel = nullptr;
    // plan
    std::vector<BatchInfo> plan;
    DevBuf plan_desc;
    int64_t plan_nets = 0, plan_slots = 0;
    int64_t plan_max_pairs = 0, plan_max_tab = 0, plan_max_nets = 0;
    GraphCache graph;
    GraphCache la_graph;  // the learned route of the plan (route_lookahead_impl)
    int64_t launches = 0;
    int mst_smem_max = 0;
    int32_t plan_max_pins = 0;  // largest net of the uploaded plan
    DevBuf plan_ids, plan_bofs, plan_pb;  // device plan builder: inputs, per-batch totals and an error flag
    bool h_nxy_valid = false;             // h_nxy mirrors d_nxy (copied when a host-built descriptor needs it)
    int *d_queue = nullptr;  // k_mst_queue: next item, CTAs finished (zero between launches)
    int tune[GR_TUNE_PARAMS] = {1024, 1024, 1024, 129, 0, 0};  // GR_TUNE_* values (best measured on B200, Z = 10)
    int levels = 0;  // nodes on the longest Fenwick update path: 1 + floor(log2(max(X, Y)))
    // optional per-kernel timing (CUDA events around every launch)
    bool profiling = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_kind;
    size_t ev_used = 0;
    double prof_ms[GR_PROF_KINDS] = {};
    int64_t prof_n[GR_PROF_KINDS] = {};
    size_t pins_cap = 0;
};

namespace {

constexpr int kThreads = 256;
constexpr int kMstSmemMax = 200 * 1024;  // dynamic shared memory of k_mst_large
constexpr int kFenTrackMaxL = 3072;      // longest track k_fen_tracks stages (4 warps x 2 x L floats = 96 KB)
constexpr int kMstMidPins = 128;         // k_mst_large on 128 threads up to this size
constexpr int kMstClusterSmem = 216 * 1024;  // dynamic shared memory of k_mst_cluster CTAs

#define GR_CK(call)                                                                            \
    do {                                                                                       \
        cudaError_t _e = (call);                                                               \
        if (_e != cudaSuccess) {                                                               \
            fprintf(stderr, "iitmgr_b200: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(_e), \
                    __FILE__, __LINE__);                                                       \
            return GR_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

Coords coords(const gr_ctx *c) { return Coords{c->d_pxy, c->d_cx, c->d_cy}; }

int grid_for(const gr_ctx *c, int64_t items, int per_sm = 8) {
    int64_t b = (items + kThreads - 1) / kThreads;
    int64_t cap = (int64_t)c->sm_count * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Records an event before a launch when profiling (never inside a capture).
int prof_begin(gr_ctx *c, cudaStream_t s) {
    if (!c->profiling) return -1;
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return -1;
    if (c->ev_used + 2 > c->ev.size()) {
        for (int i = 0; i < 256; i++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            c->ev.push_back(e);
        }
        c->ev_kind.resize(c->ev.size() / 2 + 1);
    }
    int i = (int)c->ev_used;
    c->ev_used += 2;
    cudaEventRecord(c->ev[i], s);
    return i;
}
void prof_end(gr_ctx *c, cudaStream_t s, int i, int kind) {
    c->launches++;
    if (i < 0) return;
    cudaEventRecord(c->ev[i + 1], s);
    c->ev_kind[i / 2] = kind;
}

int ensure(DevBuf &b, size_t bytes, cudaStream_t s) {
    if (bytes <= b.bytes) return GR_OK;
    if (b.p) {
        GR_CK(cudaStreamSynchronize(s));
        GR_CK(cudaFree(b.p));
        b.p = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes < 256 ? 256 : bytes;
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
        cudaGetLastError();
        return GR_ERR_NOMEM;
    }
    b.bytes = want;
    return GR_OK;
}

cudaStream_t pick(gr_ctx *c, void *stream) { return stream ? (cudaStream_t)stream : c->stream; }

// query-table entries of design net id (0: the net is costed by direct gathers)
int64_t tab_entries(const gr_ctx *c, int32_t id) {
    const int32_t nxy = c->h_nxy[id];
    return (int64_t)c->g.Z * (nxy >> 16) * (nxy & 0xffff);
}

// bytes of a SoA descriptor of n nets
size_t desc_bytes(int64_t n) { return (size_t)n * (3 * sizeof(int32_t) + 4 * sizeof(int64_t)) + 64; }

// lays the SoA arrays of n nets out in a buffer (int64 arrays first)
BatchView view_of(void *buf, int64_t total_n, int64_t first, int32_t n) {
    char *p = (char *)buf;
    BatchView v{};
    int64_t *pin_base = (int64_t *)p;
    int64_t *pair_ofs = pin_base + total_n;
    int64_t *node_ofs = pair_ofs + total_n;
    int64_t *tab_ofs = node_ofs + total_n;
    int32_t *npin = (int32_t *)(tab_ofs + total_n);
    int32_t *order = npin + total_n;
    int32_t *nxy = order + total_n;
    v.n = n;
    v.order = order + first;
    v.nxy = nxy + first;
    v.npin = npin + first;
    v.pin_base = pin_base + first;
    v.pair_ofs = pair_ofs + first;
    v.node_ofs = node_ofs + first;
    v.tab_ofs = tab_ofs + first;
    return v;
}

// Builds the descriptor of one batch into `dst` (host SoA of total_n nets,
// entries [first, first+n)). Returns GR_OK or GR_ERR_ARG / GR_ERR_STATE.
int fill_desc(const gr_ctx *c, const int32_t *ids, int32_t n, void *dst, int64_t total_n, int64_t first,
              BatchInfo &bi) {
    BatchView v = view_of(dst, total_n, first, n);
    int64_t *pin_base = const_cast<int64_t *>(v.pin_base);
    int64_t *pair_ofs = const_cast<int64_t *>(v.pair_ofs);
    int64_t *node_ofs = const_cast<int64_t *>(v.node_ofs);
    int64_t *tab_ofs = const_cast<int64_t *>(v.tab_ofs);
    int32_t *npin = const_cast<int32_t *>(v.npin);
    int32_t *order = const_cast<int32_t *>(v.order);
    int32_t *nxy = const_cast<int32_t *>(v.nxy);
    int64_t P = 0, M = 0, T = 0;
    int32_t mp = 0, n2 = 0, nm = 0;
    for (int32_t i = 0; i < n; i++) {
        int32_t id = ids[i];
        if (id < 0 || id >= c->n_nets) return GR_ERR_ARG;
        int64_t o = c->h_pin_ofs[id];
        int32_t k = (int32_t)(c->h_pin_ofs[id + 1] - o);
        npin[i] = k;
        pin_base[i] = o;
        pair_ofs[i] = P;
        node_ofs[i] = M;
        tab_ofs[i] = T;
        P += (int64_t)k * (k - 1) / 2;
        M += k;
        T += tab_entries(c, id);
        nxy[i] = c->h_nxy[id];
        if (k > mp) mp = k;
        n2 += k == 2;
        nm += k > 2 && k <= kMstWarpPins;
    }
    // nets by size class (k_mst_pin2 / k_mst_warp / k_mst_large on 128 or 512
    // threads), batch order kept within a class
    int32_t nmid = 0;
    for (int32_t i = 0; i < n; i++) nmid += npin[i] > kMstWarpPins && npin[i] <= kMstMidPins;
    int32_t o2 = 0, om = n2, oi = n2 + nm, ol = n2 + nm + nmid;
    for (int32_t i = 0; i < n; i++) {
        const int32_t k = npin[i];
        order[k == 2 ? o2++ : (k <= kMstWarpPins ? om++ : (k <= kMstMidPins ? oi++ : ol++))] = i;
    }
    bi.n2 = n2;
    bi.nm = nm;
    bi.nl = n - n2 - nm;
    bi.nmid = nmid;
    bi.first = first;
    bi.n = n;
    bi.n_pairs = P;
    bi.n_nodes = M;
    bi.n_tab = T;
    bi.max_pins = mp;
    return GR_OK;
}

BatchView make_view(void *dev, int64_t total_n, const BatchInfo &bi) {
    BatchView v = view_of(dev, total_n, bi.first, bi.n);
    v.n_pairs = bi.n_pairs;
    v.n_nodes = bi.n_nodes;
    v.n_tab = bi.n_tab;
    v.max_pins = bi.max_pins;
    v.n2 = bi.n2;
    v.nm = bi.nm;
    v.nl = bi.nl;
    v.nmid = bi.nmid;
    return v;
}

// k_mst_large shared memory: per pin a 64-bit key, five ints and a float
size_t mst_smem(int max_pins) { return (size_t)max_pins * (sizeof(unsigned long long) + 6 * sizeof(int)); }
// whether a net of n pins keeps its n x n cost matrix in shared memory
bool mst_mat_in_smem(int n) { return mst_smem(n) + (size_t)n * mst_ld(n) * sizeof(float) <= (size_t)kMstSmemMax; }
// k_mst_cluster shared memory per CTA: partial minima, the block arrays and
// its ceil(n/cs) matrix rows
size_t mst_cluster_smem(int n, int cs) {
    return (size_t)n * sizeof(unsigned long long) + mst_smem(n) + (size_t)((n + cs - 1) / cs) * mst_ld(n) * sizeof(float);
}
// cluster size for nets of up to n pins (0: no cluster -- one CTA suffices
// or the matrix needs global memory)
// (from_pins > 0: nets of at least that many pins use a cluster whenever one
// fits, even if one CTA could hold the matrix)
int mst_cluster_size(int n, int from_pins = 0) {
    if (n <= kMstMidPins) return 0;
    if (mst_mat_in_smem(n) && !(from_pins > 0 && n >= from_pins)) return 0;
    if (mst_cluster_smem(n, 4) <= (size_t)kMstClusterSmem) return 4;
    if (mst_cluster_smem(n, 8) <= (size_t)kMstClusterSmem) return 8;
    return 0;
}

// ------------------------------------------------------------------ stages

// mst (may be null): also write the trees of the batch's 2-pin nets (and
// their dist), so that launch_mst can skip k_mst_pin2, and mark their paths
// when mo.mark is set
int launch_lpat_batch(gr_ctx *c, const BatchView &v, float *pcost, int16_t *ppat, float2 *tab, cudaStream_t s,
                      int64_t *mst = nullptr, float *dist = nullptr, MarkOut mo = MarkOut{}) {
    if (v.n_tab > 0) {
        int pi = prof_begin(c, s);
        k_qtable<<<grid_for(c, v.n_tab, 16), kThreads, 0, s>>>(c->g, v, coords(c), c->d_fen, tab);
        prof_end(c, s, pi, GR_K_QTABLE);
    }
    if (v.n_pairs > 0) {
        int pi = prof_begin(c, s);
        const int grid = grid_for(c, v.n_pairs, 16);
        // warps per group of 32 pairs: 4 when one thread per pair would fill
        // fewer than half of the SMs (measured: -3 us per batch there, slower
        // as soon as the batch fills the GPU)
        int split = c->tune[GR_TUNE_LPAT_SPLIT];
        if (split == 0) {
            const int64_t blocks1 = (v.n_pairs + kThreads - 1) / kThreads;
            split = 2 * blocks1 < c->sm_count ? 4 : 1;
        }
        const int64_t gs = (v.n_pairs + kThreads / split - 1) / (kThreads / split);
        const int grid_s = (int)(gs < 16LL * c->sm_count ? gs : 16LL * c->sm_count);
#define GR_LPAT_Z(ZV)                                                                                     \
    case ZV:                                                                                              \
        if (split == 4)                                                                                   \
            k_lpat_zs<ZV, 4><<<grid_s, kThreads, 0, s>>>(c->g, v, c->d_pins, coords(c), c->d_fen, tab, pcost, \
                                                         ppat, mst, dist, mo, c->d_status);               \
        else if (split == 2)                                                                              \
            k_lpat_zs<ZV, 2><<<grid_s, kThreads, 0, s>>>(c->g, v, c->d_pins, coords(c), c->d_fen, tab, pcost, \
                                                         ppat, mst, dist, mo, c->d_status);               \
        else                                                                                              \
            k_lpat_z<ZV><<<grid, kThreads, 0, s>>>(c->g, v, c->d_pins, coords(c), c->d_fen, tab, pcost, ppat, \
                                                   mst, dist, mo, c->d_status);                           \
        break;
        switch (c->g.Z) {
            GR_LPAT_Z(3) GR_LPAT_Z(4) GR_LPAT_Z(5) GR_LPAT_Z(6) GR_LPAT_Z(7) GR_LPAT_Z(8) GR_LPAT_Z(9)
            GR_LPAT_Z(10) GR_LPAT_Z(11) GR_LPAT_Z(12) GR_LPAT_Z(13) GR_LPAT_Z(14) GR_LPAT_Z(15) GR_LPAT_Z(16)
            default:
                k_lpat_batch<<<grid, kThreads, 0, s>>>(c->g, v, c->d_pins, coords(c), c->d_fen, tab, pcost, ppat,
                                                       mst, dist, mo, c->d_status);
        }
#undef GR_LPAT_Z
        prof_end(c, s, pi, GR_K_LPAT);
    }
    GR_CK(cudaGetLastError());
    return GR_OK;
}

// where a batch's marking goes (the context's bitmap), for pair patterns
// ppat and slot patterns mst_pat (may be null)
MarkOut mark_out(const gr_ctx *c, const int16_t *ppat, int32_t *mst_pat) {
    return MarkOut{c->d_mark, mst_pat, ppat, c->d_pins};
}

// k_mark over the batch's slots (trees that did not come from this
// context's tree kernels)
int launch_mark(gr_ctx *c, const BatchView &v, const int64_t *mst, const MarkOut &mo, cudaStream_t s) {
    if (v.n_nodes <= 0) return GR_OK;
    int pi = prof_begin(c, s);
    k_mark<<<grid_for(c, v.n_nodes, 8), kThreads, 0, s>>>(c->g, v, mst, mo, c->d_status);
    prof_end(c, s, pi, GR_K_MARK);
    GR_CK(cudaGetLastError());
    return GR_OK;
}

// mo.mark set: every tree kernel marks the GCELLs of the trees it builds
// (and writes the slots' patterns), right after building each one
int launch_mst(gr_ctx *c, const BatchView &v, const float *pcost, int64_t *mst, float *dist, cudaStream_t s,
               bool pin2_done = false, MarkOut mo = MarkOut{}) {
    if (v.n <= 0) return GR_OK;
    if (c->tune[GR_TUNE_MST_QUEUE]) {
        if (v.n2 > 0 && !pin2_done) {
            int pi = prof_begin(c, s);
            k_mst_pin2<<<(v.n2 + kThreads - 1) / kThreads, kThreads, 0, s>>>(c->g, v, pcost, mst, dist, mo,
                                                                          c->d_status);
            prof_end(c, s, pi, GR_K_MST);
        }
        const int items = v.nl + (v.nm + kQueueWarps - 1) / kQueueWarps;
        if (items <= 0) return GR_OK;
        const int maxn = v.nl > 0 ? v.max_pins : kMstWarpPins;
        const bool in_smem = mst_mat_in_smem(maxn);
        size_t sm = mst_smem(maxn) + (in_smem ? (size_t)maxn * mst_ld(maxn) * sizeof(float) : 0);
        sm = sm > kQueueWarpSmem ? sm : kQueueWarpSmem;
        int blocks = c->sm_count * (sm <= 100 * 1024 ? 2 : 1);
        uint32_t *gmat = nullptr;
        if (!in_smem) {
            blocks = c->sm_count;
            if (c->mat.bytes < (size_t)blocks * maxn * mst_ld(maxn) * sizeof(float)) return GR_ERR_STATE;
            gmat = (uint32_t *)c->mat.p;
        }
        blocks = items < blocks ? items : blocks;
        BatchView vv = v;
        vv.max_pins = maxn;
        int pi = prof_begin(c, s);
        k_mst_queue<<<blocks, kQueueThreads, sm, s>>>(c->g, vv, pcost, mst, dist, c->d_status, gmat,
                                                      (int64_t)maxn * mst_ld(maxn), c->d_queue, mo);
        prof_end(c, s, pi, GR_K_MST_LARGE);
        GR_CK(cudaGetLastError());
        return GR_OK;
    }
    // the size classes are independent: warp and larger-net kernels run on
    // side streams forked from s and joined back (parallel graph branches)
    GR_CK(cudaEventRecord(c->ev_fork, s));
    bool used[3] = {false, false, false};
    auto side = [&](int i) {
        if (!used[i]) cudaStreamWaitEvent(c->side[i], c->ev_fork, 0);
        used[i] = true;
        return c->side[i];
    };
    if (v.n2 > 0 && !pin2_done) {
        int pi = prof_begin(c, s);
        k_mst_pin2<<<(v.n2 + kThreads - 1) / kThreads, kThreads, 0, s>>>(c->g, v, pcost, mst, dist, mo,
                                                                          c->d_status);
        prof_end(c, s, pi, GR_K_MST);
    }
    if (v.nm > 0) {
        cudaStream_t s0 = side(0);
        int pi = prof_begin(c, s0);
        k_mst_warp<<<(v.nm + 7) / 8, 256, 0, s0>>>(c->g, v, pcost, mst, dist, c->d_status, mo);
        prof_end(c, s0, pi, GR_K_MST_WARP);
    }
    // larger nets: 128-thread CTAs up to 128 pins, 512-thread CTAs above. A
    // net's full cost matrix sits in the CTA's shared memory when it fits, is
    // spread over a 4- or 8-CTA cluster when that fits, else goes to a per-CTA
    // global scratch (sized by ensure_mst_scratch).
    const int nmid = v.nmid, nbig = v.nl - v.nmid;
    for (int part = 0; part < 2; part++) {
        const int cnt = part ? nbig : nmid;
        if (cnt <= 0) continue;
        const int maxn = part ? v.max_pins : (v.max_pins < kMstMidPins ? v.max_pins : kMstMidPins);
        const int first = v.n2 + v.nm + (part ? nmid : 0);
        BatchView vv = v;
        vv.max_pins = maxn;
        const int cs = mst_cluster_size(maxn, c->tune[GR_TUNE_MST_CLUSTER_MIN_PINS]);
        cudaStream_t sp = side(1 + part);
        int pi = prof_begin(c, sp);
        if (cs) {
            const int clusters = cnt < c->sm_count / cs ? cnt : c->sm_count / cs;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(clusters * cs);
            cfg.blockDim = dim3(c->tune[GR_TUNE_MST_CLUSTER_THREADS]);
            cfg.dynamicSmemBytes = mst_cluster_smem(maxn, cs);
            cfg.stream = sp;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cs;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            if (cs == 4)
                GR_CK(cudaLaunchKernelEx(&cfg, k_mst_cluster<4>, c->g, vv, (const float *)pcost, mst, dist,
                                         c->d_status, first, cnt, mo));
            else
                GR_CK(cudaLaunchKernelEx(&cfg, k_mst_cluster<8>, c->g, vv, (const float *)pcost, mst, dist,
                                         c->d_status, first, cnt, mo));
        } else {
            const bool in_smem = mst_mat_in_smem(maxn);
            const size_t sm = mst_smem(maxn) + (in_smem ? (size_t)maxn * mst_ld(maxn) * sizeof(float) : 0);
            int blocks = cnt < c->sm_count * 8 ? cnt : c->sm_count * 8;
            uint32_t *gmat = nullptr;
            if (!in_smem) {
                blocks = cnt < c->sm_count ? cnt : c->sm_count;
                if (c->mat.bytes < (size_t)blocks * maxn * mst_ld(maxn) * sizeof(float)) return GR_ERR_STATE;
                gmat = (uint32_t *)c->mat.p;
            }
            k_mst_large<<<blocks, c->tune[part ? GR_TUNE_MST_BIG_THREADS : GR_TUNE_MST_MID_THREADS], sm, sp>>>(
                c->g, vv, pcost, mst, dist, c->d_status, gmat, (int64_t)maxn * mst_ld(maxn), first, cnt, mo);
        }
        prof_end(c, sp, pi, GR_K_MST_LARGE);
    }
    for (int i = 0; i < 3; i++)
        if (used[i]) {
            GR_CK(cudaEventRecord(c->ev_join[i], c->side[i]));
            GR_CK(cudaStreamWaitEvent(s, c->ev_join[i], 0));
        }
    GR_CK(cudaGetLastError());
    return GR_OK;
}

// warps per k_track_commit block: small blocks, so that a block held by one
// heavily marked track keeps few finished warps' slots idle (2 warps: 50.0 ms
// per route of the 1.2M-net design, against 50.1 with 4 and 50.2 with 8)
constexpr int kTrackWarps = 2;
static_assert(kTrackWarps <= kTrackWarpsMax, "k_track_commit's per-warp rank tables");
// marked cells per track kept in shared memory (more go to the track's slice
// of the global scratch): 4 KB per 2-warp block
constexpr int kTrackCapMax = 256;

size_t track_smem(int cap) { return (size_t)kTrackWarps * 2 * cap * sizeof(int32_t); }

// marked: the tree kernels already marked the batch's slots
int launch_commit(gr_ctx *c, const BatchView &v, const int64_t *mst, const int16_t *ppat, int32_t *mst_pat,
                  cudaStream_t s, bool marked = false) {
    if (v.n_nodes <= 0) return GR_OK;
    if (!marked) {
        int rc = launch_mark(c, v, mst, mark_out(c, ppat, mst_pat), s);
        if (rc) return rc;
    }
    int pi = prof_begin(c, s);
    int64_t blocks = ((int64_t)c->n_tracks + kTrackWarps - 1) / kTrackWarps;
    if (blocks > (int64_t)c->sm_count * 32) blocks = (int64_t)c->sm_count * 32;
    k_track_commit<<<(int)blocks, kTrackWarps * 32, track_smem(c->track_cap), s>>>(
        c->g, c->n_tracks, c->d_mark, c->d_capr, c->d_dlut, c->d_fen, c->d_gpos, c->d_gdel, c->track_cap,
        c->la_on ? c->d_pred : nullptr, c->la_beta);
    prof_end(c, s, pi, GR_K_FEN_UPDATE);
    GR_CK(cudaGetLastError());
    return GR_OK;
}

int check_mst_smem(gr_ctx *c, int max_pins) {
    if (max_pins > GR_MAX_PINS) return GR_ERR_NET_TOO_LARGE;
    return GR_OK;
}

// global pair-cost matrices for k_mst_large when a batch's largest net
// does not fit in shared memory (one matrix per CTA, at most one CTA per SM)
int ensure_mst_scratch(gr_ctx *c, int max_pins, cudaStream_t s) {
    if (max_pins <= kMstWarpPins || mst_mat_in_smem(max_pins)) return GR_OK;
    if (!c->tune[GR_TUNE_MST_QUEUE] && (max_pins <= kMstMidPins || mst_cluster_size(max_pins))) return GR_OK;
    return ensure(c->mat, (size_t)c->sm_count * max_pins * mst_ld(max_pins) * sizeof(float), s);
}

// scratch for one batch of the given sizes
int ensure_scratch(gr_ctx *c, int64_t pairs, int64_t tab, int64_t nets, cudaStream_t s) {
    int rc;
    if ((rc = ensure(c->pcost, sizeof(float) * (pairs + 1), s))) return rc;
    if ((rc = ensure(c->ppat, sizeof(int16_t) * (pairs + 1), s))) return rc;
    if ((rc = ensure(c->tab, sizeof(float2) * (tab + 1), s))) return rc;
    if ((rc = ensure(c->dist, sizeof(float) * (nets + 1), s))) return rc;
    return GR_OK;
}

// copies the descriptor of a per-call batch to the device; returns its info
// the host mirror of the per-net table shapes (for descriptors built on the host)
int ensure_h_nxy(gr_ctx *c) {
    if (c->h_nxy_valid) return GR_OK;
    c->h_nxy.resize(c->n_nets);
    if (c->n_nets > 0) {
        GR_CK(cudaMemcpyAsync(c->h_nxy.data(), c->d_nxy, sizeof(int32_t) * c->n_nets, cudaMemcpyDeviceToHost,
                              c->stream));
        GR_CK(cudaStreamSynchronize(c->stream));
    }
    c->h_nxy_valid = true;
    return GR_OK;
}

int upload_batch(gr_ctx *c, const int32_t *ids, int32_t n, BatchInfo &bi, BatchView &v, cudaStream_t s) {
    if (!c->d_pins) return GR_ERR_STATE;
    if (n < 0 || (n > 0 && !ids)) return GR_ERR_ARG;
    int rc0 = ensure_h_nxy(c);
    if (rc0) return rc0;
    size_t bytes = desc_bytes(n > 0 ? n : 1);
    if (bytes > c->h_stage_bytes) {
        if (c->h_stage) {
            GR_CK(cudaEventSynchronize(c->stage_done));
            GR_CK(cudaFreeHost(c->h_stage));
        }
        c->h_stage = nullptr;
        if (cudaMallocHost(&c->h_stage, bytes) != cudaSuccess) {
            cudaGetLastError();
            c->h_stage_bytes = 0;
            return GR_ERR_NOMEM;
        }
        c->h_stage_bytes = bytes;
    } else {
        GR_CK(cudaEventSynchronize(c->stage_done));  // previous copy out of staging done
    }
    int rc = fill_desc(c, ids, n, c->h_stage, n, 0, bi);
    if (rc) return rc;
    if ((rc = check_mst_smem(c, bi.max_pins))) return rc;
    if ((rc = ensure_mst_scratch(c, bi.max_pins, s))) return rc;
    if ((rc = ensure(c->desc, bytes, s))) return rc;
    GR_CK(cudaMemcpyAsync(c->desc.p, c->h_stage, bytes, cudaMemcpyHostToDevice, s));
    GR_CK(cudaEventRecord(c->stage_done, s));
    v = make_view(c->desc.p, n, bi);
    return GR_OK;
}

// One batch: L-pattern (which also settles and marks the 2-pin nets), the
// trees of the other nets (each marked by the kernel that builds it), then
// the commit of every marked GCELL.
int route_one(gr_ctx *c, const BatchView &v, int64_t *mst, int32_t *mst_pat, float *dist, float *pcost,
              int16_t *ppat, cudaStream_t s) {
    int rc;
    const MarkOut mo = mark_out(c, ppat, mst_pat);
    if ((rc = launch_lpat_batch(c, v, pcost, ppat, (float2 *)c->tab.p, s, mst, dist, mo))) return rc;
    if ((rc = launch_mst(c, v, pcost, mst, dist, s, true, mo))) return rc;
    return launch_commit(c, v, mst, ppat, mst_pat, s, true);
}

void free_buf(DevBuf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

void drop_graph(gr_ctx *c) {
    if (c->graph.exec) cudaGraphExecDestroy(c->graph.exec);
    c->graph = GraphCache{};
}

void drop_la_graph(gr_ctx *c) {
    if (c->la_graph.exec) cudaGraphExecDestroy(c->la_graph.exec);
    c->la_graph = GraphCache{};
}

// Fenwick trees from the current capacities, with the plain or the lookahead cost
int rebuild_fenwick(gr_ctx *c, cudaStream_t s) {
    int pi = prof_begin(c, s);
    const int lmax = c->g.X > c->g.Y ? c->g.X : c->g.Y;
    if (lmax <= kFenTrackMaxL)  // a warp per track, the track staged in shared memory
        k_fen_tracks<<<(c->n_tracks + 3) / 4, 128, (size_t)4 * 2 * lmax * sizeof(float), s>>>(
            c->g, (int)c->n_tracks, c->la_on ? 1 : 0, c->d_capr, c->d_lut, c->d_pred, c->la_beta, c->d_fen);
    else if (c->la_on)
        k_fen_init_la<<<grid_for(c, c->csize, 16), kThreads, 0, s>>>(c->g, (int)c->csize, c->d_capr, c->d_pred,
                                                                     c->la_beta, c->d_fen);
    else
        k_fen_init<<<grid_for(c, c->csize, 16), kThreads, 0, s>>>(c->g, (int)c->csize, c->d_capr, c->d_lut, c->d_fen);
    prof_end(c, s, pi, GR_K_FEN_INIT);
    GR_CK(cudaGetLastError());
    return GR_OK;
}

}  // namespace

// ====================================================================== API

extern "C" {

int gr_version(void) { return 1; }

const char *gr_error_string(int code) {
    switch (code) {
        case GR_OK: return "ok";
        case GR_ERR_ARG: return "invalid argument";
        case GR_ERR_CUDA: return "CUDA runtime error";
        case GR_ERR_NOMEM: return "out of memory";
        case GR_ERR_STATE: return "call out of order";
        case GR_ERR_NET_TOO_LARGE: return "net has more pins than supported";
        case GR_ERR_DEVICE: return "a kernel reported invalid data";
        case GR_ERR_IO: return "file could not be read or written";
        case GR_ERR_PARSE: return "malformed input text";
        case GR_ERR_NONINTEGER: return "capacity is not an integer";
        default: return "unknown error";
    }
}

int gr_create(gr_ctx **out, int device, int X, int Y, int Z, const int32_t *h_cap) {
    if (!out || !h_cap || X < 1 || Y < 1 || Z < 3 || Z > kMaxLayers) return GR_ERR_ARG;
    int64_t csize = (int64_t)X * Y * Z;
    if (csize >= 0x7fffff00LL) return GR_ERR_ARG;  // cell ids are int32
    *out = nullptr;
    GR_CK(cudaSetDevice(device));
    gr_ctx *c = new gr_ctx();
    c->device = device;
    c->g.X = X;
    c->g.Y = Y;
    c->g.Z = Z;
    c->g.Z2 = (Z + 1) / 2;
    c->g.npat = Z * c->g.Z2;
    c->g.XY = X * Y;
    c->csize = csize;
    for (int L = X > Y ? X : Y; L > 0; L >>= 1) c->levels++;
    int rc = GR_OK;
    auto fail = [&](int code) {
        const cudaError_t e = cudaGetLastError();
        if (code == GR_ERR_CUDA && e != cudaSuccess)
            fprintf(stderr, "iitmgr_b200: gr_create: %s\n", cudaGetErrorString(e));
        gr_destroy(c);
        return code;
    };
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return fail(GR_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(GR_ERR_CUDA);
    if (cudaEventCreateWithFlags(&c->stage_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->nets_up, cudaEventDisableTiming) != cudaSuccess)
        return fail(GR_ERR_CUDA);
    if (cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess) return fail(GR_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_copy_done, cudaEventDisableTiming) != cudaSuccess)
        return fail(GR_ERR_CUDA);
    for (int i = 0; i < 3; i++)
        if (cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->ev_join[i], cudaEventDisableTiming) != cudaSuccess)
            return fail(GR_ERR_CUDA);
    size_t cell4 = sizeof(int32_t) * csize;
    size_t words = (size_t)(csize / 32 + 2);
    c->n_tracks = ((Z + 1) / 2) * Y + (Z / 2) * X;
    c->track_cap = (X > Y ? X : Y) < kTrackCapMax ? (X > Y ? X : Y) : kTrackCapMax;
    // capr is read in aligned 32-cell words: pad it to a whole last word
    if (cudaMalloc(&c->d_cap0, cell4) || cudaMalloc(&c->d_capr, cell4 + 128) || cudaMalloc(&c->d_fen, cell4) ||
        cudaMalloc(&c->d_mark, words * 4) || cudaMalloc(&c->d_status, 16) ||
        cudaMalloc(&c->d_queue, 16) ||
        cudaMalloc(&c->d_lut, sizeof(float) * (kLutMax - kLutMin + 1)) ||
        cudaMalloc(&c->d_dlut, sizeof(float) * (kLutMax - kLutMin + 2)) ||
        (c->track_cap < (X > Y ? X : Y) &&
         (cudaMalloc(&c->d_gpos, sizeof(int32_t) * (size_t)csize) ||
          cudaMalloc(&c->d_gdel, sizeof(float) * (size_t)csize)))) {
        cudaGetLastError();
        return fail(GR_ERR_NOMEM);
    }
    // cost LUT: (float)exp(-0.5 c) for integer remaining capacity c
    std::vector<float> lut(kLutMax - kLutMin + 1);
    for (int cc = kLutMin; cc <= kLutMax; cc++) lut[cc - kLutMin] = (float)std::exp(-0.5 * (double)cc);
    c->h_cap0.assign(h_cap, h_cap + csize);
    // every upload and clear on the context's own (non-blocking) stream: a
    // legacy-stream cudaMemcpy from pageable memory may return before its DMA
    // lands, and nothing orders the legacy stream before this one
    const cudaStream_t s0 = c->stream;
    if (cudaMemcpyAsync(c->d_lut, lut.data(), sizeof(float) * lut.size(), cudaMemcpyHostToDevice, s0) ||
        cudaMemcpyAsync(c->d_cap0, h_cap, cell4, cudaMemcpyHostToDevice, s0) ||
        cudaMemsetAsync(c->d_mark, 0, words * 4, s0) || cudaMemsetAsync(c->d_status, 0, 16, s0) ||
        cudaMemsetAsync(c->d_queue, 0, 16, s0))
        return fail(GR_ERR_CUDA);
    // A function attribute holds for the whole process, not this context:
    // set it to the most any context launches with, so that a context for a
    // smaller grid created later cannot lower it under a larger one's needs.
    if (cudaFuncSetAttribute(k_track_commit, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)track_smem(kTrackCapMax)) != cudaSuccess)
        return fail(GR_ERR_CUDA);
    k_dlut<<<(kLutMax - kLutMin + 2 + 255) / 256, 256, 0, c->stream>>>(c->d_lut, c->d_dlut);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(GR_ERR_CUDA);
    c->mst_smem_max = kMstSmemMax;
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
        optin < kMstClusterSmem + 1024 || optin < kMstSmemMax + 1024) {
        fprintf(stderr, "iitmgr_b200: device allows %d bytes of shared memory per block\n", optin);
        return fail(GR_ERR_CUDA);
    }
    if (cudaFuncSetAttribute(k_coords_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 16 * GR_MAX_PINS))
        return fail(GR_ERR_CUDA);
    if (cudaFuncSetAttribute(k_mst_cluster<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMstClusterSmem) ||
        cudaFuncSetAttribute(k_mst_cluster<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMstClusterSmem))
        return fail(GR_ERR_CUDA);
    if (cudaFuncSetAttribute(k_mst_large, cudaFuncAttributeMaxDynamicSharedMemorySize, c->mst_smem_max) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mst_queue, cudaFuncAttributeMaxDynamicSharedMemorySize, kMstSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(k_fen_tracks, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             4 * 2 * kFenTrackMaxL * (int)sizeof(float)) != cudaSuccess)
        return fail(GR_ERR_CUDA);
    if ((rc = gr_reset(c, nullptr))) return fail(rc);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(GR_ERR_CUDA);
    *out = c;
    return GR_OK;
}

int gr_destroy(gr_ctx *c) {
    if (!c) return GR_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    drop_la_graph(c);
    cudaFree(c->d_cap0);
    cudaFree(c->d_capr);
    cudaFree(c->d_fen);
    cudaFree(c->d_lut);
    cudaFree(c->d_dlut);
    cudaFree(c->d_pred);
    cudaFree(c->d_gpos);
    cudaFree(c->d_gdel);
    cudaFree(c->d_mark);
    cudaFree(c->d_status);
    cudaFree(c->d_queue);
    free_buf(c->mat);
    cudaFree(c->d_pins);
    cudaFree(c->d_pxy);
    cudaFree(c->d_cx);
    cudaFree(c->d_cy);
    free_buf(c->desc);
    free_buf(c->pcost);
    free_buf(c->ppat);
    free_buf(c->tab);
    free_buf(c->dist);
    free_buf(c->plan_desc);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    if (c->stage_done) cudaEventDestroy(c->stage_done);
    if (c->nets_up) cudaEventDestroy(c->nets_up);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream), cudaStreamDestroy(c->copy_stream);
    if (c->ev_out) cudaEventDestroy(c->ev_out);
    if (c->ev_copy_done) cudaEventDestroy(c->ev_copy_done);
    free_buf(c->out_mst);
    free_buf(c->out_pat);
    free_buf(c->la_feat);
    free_buf(c->la_out);
    free_buf(c->plan_ids);
    free_buf(c->plan_bofs);
    free_buf(c->plan_pb);
    for (int i = 0; i < 3; i++) {
        if (c->side[i]) cudaStreamSynchronize(c->side[i]), cudaStreamDestroy(c->side[i]);
        if (c->ev_join[i]) cudaEventDestroy(c->ev_join[i]);
    }
    cudaFree(c->d_pin_ofs);
    cudaFree(c->d_nxy);
    cudaFree(c->d_big);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GR_OK;
}

int gr_reset(gr_ctx *c, void *stream) {
    if (!c) return GR_ERR_ARG;
    cudaStream_t s = pick(c, stream);
    GR_CK(cudaMemcpyAsync(c->d_capr, c->d_cap0, sizeof(int32_t) * c->csize, cudaMemcpyDeviceToDevice, s));
    GR_CK(cudaMemsetAsync(c->d_mark, 0, sizeof(uint32_t) * (size_t)(c->csize / 32 + 2), s));
    GR_CK(cudaMemsetAsync(c->d_queue, 0, 16, s));
    return rebuild_fenwick(c, s);
}

int gr_set_nets(gr_ctx *c, int32_t n_nets, const int64_t *h_pin_ofs, const int32_t *h_pins) {
    if (!c || n_nets < 0 || !h_pin_ofs || (n_nets > 0 && !h_pins) || h_pin_ofs[0] != 0) return GR_ERR_ARG;
    int short_net = 0, long_net = 0, bad_pin = 0;
#pragma omp parallel for reduction(| : short_net, long_net)
    for (int32_t i = 0; i < n_nets; i++) {
        const int64_t k = h_pin_ofs[i + 1] - h_pin_ofs[i];
        short_net |= k < 2;
        long_net |= k > GR_MAX_PINS;
    }
    if (short_net) return GR_ERR_ARG;
    if (long_net) return GR_ERR_NET_TOO_LARGE;
    const int64_t total = h_pin_ofs[n_nets];
    const int64_t csize = c->csize;
#pragma omp parallel for reduction(| : bad_pin)
    for (int64_t t = 0; t < total; t++) bad_pin |= h_pins[t] < 0 || h_pins[t] >= csize;
    if (bad_pin) return GR_ERR_ARG;
    GR_CK(cudaStreamSynchronize(c->stream));
    // a captured plan stays: it is replayed only if its signature (buffer
    // addresses, batch shapes) still matches (graph_sig)
    if ((size_t)(total + 1) > c->pins_cap) {
        for (int32_t **p : {&c->d_pins, &c->d_pxy, &c->d_cx, &c->d_cy}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        c->pins_cap = 0;
        for (int32_t **p : {&c->d_pins, &c->d_pxy, &c->d_cx, &c->d_cy})
            if (cudaMalloc(p, sizeof(int32_t) * (total + 1)) != cudaSuccess) {
                cudaGetLastError();
                return GR_ERR_NOMEM;
            }
        c->pins_cap = (size_t)(total + 1);
    }
    // per net: sorted distinct x and y coordinates and each pin's index into
    // them (the query tables are laid out over these coordinates), computed
    // on the device; only the per-net table shape comes back
    if ((size_t)(n_nets + 1) > c->nets_cap) {
        for (void **p : {(void **)&c->d_pin_ofs, (void **)&c->d_nxy, (void **)&c->d_big}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        c->nets_cap = 0;
        if (cudaMalloc(&c->d_pin_ofs, sizeof(int64_t) * (n_nets + 1)) != cudaSuccess ||
            cudaMalloc(&c->d_nxy, sizeof(int32_t) * (n_nets + 1)) != cudaSuccess ||
            cudaMalloc(&c->d_big, sizeof(int32_t) * (n_nets + 1)) != cudaSuccess) {
            cudaGetLastError();
            return GR_ERR_NOMEM;
        }
        c->nets_cap = (size_t)(n_nets + 1);
    }
    GR_CK(cudaMemcpyAsync(c->d_pins, h_pins, sizeof(int32_t) * total, cudaMemcpyHostToDevice, c->stream));
    // nets above 32 pins (k_coords_block), in net order, gathered per thread while the pins upload
    std::vector<int32_t> big;
    int32_t big_max = 0;
#pragma omp parallel
    {
        std::vector<int32_t> mine;
        int32_t mx = 0;
#pragma omp for schedule(static) nowait
        for (int32_t i = 0; i < n_nets; i++) {
            const int32_t k = (int32_t)(h_pin_ofs[i + 1] - h_pin_ofs[i]);
            if (k > 32) {
                mine.push_back(i);
                mx = k > mx ? k : mx;
            }
        }
#pragma omp for ordered schedule(static, 1)
        for (int t = 0; t < omp_get_num_threads(); t++) {
#pragma omp ordered
            {
                big.insert(big.end(), mine.begin(), mine.end());
                big_max = mx > big_max ? mx : big_max;
            }
        }
    }
    GR_CK(cudaMemcpyAsync(c->d_pin_ofs, h_pin_ofs, sizeof(int64_t) * (n_nets + 1), cudaMemcpyHostToDevice,
                          c->stream));
    if (!big.empty())
        GR_CK(cudaMemcpyAsync(c->d_big, big.data(), sizeof(int32_t) * big.size(), cudaMemcpyHostToDevice,
                              c->stream));
    GR_CK(cudaEventRecord(c->nets_up, c->stream));
    if (n_nets > 0) {
        k_coords_warp<<<(int)(((int64_t)n_nets * 32 + 255) / 256), 256, 0, c->stream>>>(
            c->g, n_nets, c->d_pin_ofs, c->d_pins, c->d_pxy, c->d_cx, c->d_cy, c->d_nxy);
        c->launches++;
    }
    if (!big.empty()) {
        k_coords_block<<<(int)big.size(), 256, 16 * (size_t)big_max, c->stream>>>(
            c->g, c->d_big, c->d_pin_ofs, c->d_pins, c->d_pxy, c->d_cx, c->d_cy, c->d_nxy);
        c->launches++;
    }
    GR_CK(cudaGetLastError());
    c->h_nxy_valid = false;  // copied back when a host-built descriptor needs it
    c->h_pin_ofs.assign(h_pin_ofs, h_pin_ofs + n_nets + 1);
    c->n_nets = n_nets;
    c->plan.clear();
    // the caller's buffers are free once their uploads are done; the
    // coordinate kernels run on (later work on the stream is ordered after them)
    GR_CK(cudaEventSynchronize(c->nets_up));
    return GR_OK;
}

int gr_lpattern(gr_ctx *c, const int32_t *d_pairs, int64_t n_pairs, float *d_cost, int16_t *d_pat, void *stream) {
    if (!c || n_pairs < 0 || (n_pairs > 0 && (!d_pairs || !d_cost || !d_pat))) return GR_ERR_ARG;
    if (n_pairs == 0) return GR_OK;
    cudaStream_t s = pick(c, stream);
    int pi = prof_begin(c, s);
    k_lpat_pairs<<<grid_for(c, n_pairs, 16), kThreads, 0, s>>>(c->g, (int)c->csize, d_pairs, n_pairs, c->d_fen,
                                                              d_cost, d_pat, c->d_status);
    prof_end(c, s, pi, GR_K_LPAT_PAIRS);
    GR_CK(cudaGetLastError());
    return GR_OK;
}

int gr_brvsk_build(gr_ctx *c, const int32_t *h_net_ids, int32_t n_nets, const float *d_pair_cost,
                   int64_t *d_mst_edges, float *d_net_dist, void *stream) {
    if (!c || !d_pair_cost || !d_mst_edges) return GR_ERR_ARG;
    cudaStream_t s = pick(c, stream);
    BatchInfo bi{};
    BatchView v{};
    int rc = upload_batch(c, h_net_ids, n_nets, bi, v, s);
    if (rc) return rc;
    return launch_mst(c, v, d_pair_cost, d_mst_edges, d_net_dist, s);
}

int gr_mst_bit_commit(gr_ctx *c, const int32_t *h_net_ids, int32_t n_nets, const int64_t *d_mst_edges,
                      const int16_t *d_pair_pat, int32_t *d_mst_pat, void *stream) {
    if (!c || !d_mst_edges || !d_pair_pat) return GR_ERR_ARG;
    cudaStream_t s = pick(c, stream);
    BatchInfo bi{};
    BatchView v{};
    int rc = upload_batch(c, h_net_ids, n_nets, bi, v, s);
    if (rc) return rc;
    return launch_commit(c, v, d_mst_edges, d_pair_pat, d_mst_pat, s);
}

int gr_route_batch(gr_ctx *c, const int32_t *h_net_ids, int32_t n_nets, int64_t *d_mst_edges, int32_t *d_mst_pat,
                   float *d_net_dist, float *d_pair_cost, int16_t *d_pair_pat, void *stream) {
    if (!c || !d_mst_edges) return GR_ERR_ARG;
    cudaStream_t s = pick(c, stream);
    BatchInfo bi{};
    BatchView v{};
    int rc = upload_batch(c, h_net_ids, n_nets, bi, v, s);
    if (rc) return rc;
    if ((rc = ensure_scratch(c, bi.n_pairs, bi.n_tab, n_nets, s))) return rc;
    float *pc = d_pair_cost ? d_pair_cost : (float *)c->pcost.p;
    int16_t *pp = d_pair_pat ? d_pair_pat : (int16_t *)c->ppat.p;
    return route_one(c, v, d_mst_edges, d_mst_pat, d_net_dist, pc, pp, s);
}

int gr_plan_set(gr_ctx *c, int32_t n_batches, const int64_t *h_batch_ofs, const int32_t *h_net_ids) {
    if (!c || n_batches < 0 || !h_batch_ofs || h_batch_ofs[0] != 0) return GR_ERR_ARG;
    if (!c->d_pins) return GR_ERR_STATE;
    int64_t total = h_batch_ofs[n_batches];
    if (total < 0 || (total > 0 && !h_net_ids)) return GR_ERR_ARG;
    for (int32_t b = 0; b < n_batches; b++)
        if (h_batch_ofs[b + 1] < h_batch_ofs[b]) return GR_ERR_ARG;
    GR_CK(cudaStreamSynchronize(c->stream));
    c->plan.clear();  // a captured plan is replayed only if its signature still matches
    // the descriptor is built on the device (k_plan_nets, k_plan_batches);
    // only the per-batch totals come back for the launch shapes
    const size_t bytes = desc_bytes(total > 0 ? total : 1);
    int rc;
    if ((rc = ensure(c->plan_desc, bytes, c->stream)) ||
        (rc = ensure(c->plan_ids, sizeof(int32_t) * (size_t)(total + 1), c->stream)) ||
        (rc = ensure(c->plan_bofs, sizeof(int64_t) * (size_t)(n_batches + 1), c->stream)) ||
        (rc = ensure(c->plan_pb, sizeof(PlanBatch) * (size_t)(n_batches + 1) + 16, c->stream)))
        return rc;
    uint32_t *d_bad = (uint32_t *)((char *)c->plan_pb.p + sizeof(PlanBatch) * (size_t)(n_batches + 1));
    if (total > 0)
        GR_CK(cudaMemcpyAsync(c->plan_ids.p, h_net_ids, sizeof(int32_t) * total, cudaMemcpyHostToDevice, c->stream));
    GR_CK(cudaMemcpyAsync(c->plan_bofs.p, h_batch_ofs, sizeof(int64_t) * (n_batches + 1), cudaMemcpyHostToDevice,
                          c->stream));
    GR_CK(cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), c->stream));
    const BatchView all = view_of(c->plan_desc.p, total, 0, (int32_t)total);
    if (total > 0) {
        k_plan_nets<<<grid_for(c, total), kThreads, 0, c->stream>>>(
            total, (const int32_t *)c->plan_ids.p, c->n_nets, c->d_pin_ofs, c->d_nxy, const_cast<int64_t *>(all.pin_base),
            const_cast<int32_t *>(all.npin), const_cast<int32_t *>(all.nxy), d_bad);
        c->launches++;
    }
    if (n_batches > 0) {
        k_plan_batches<<<n_batches, 1024, 0, c->stream>>>(
            (const int64_t *)c->plan_bofs.p, c->g.Z, kMstWarpPins, kMstMidPins, all.npin, all.nxy,
            const_cast<int64_t *>(all.pair_ofs), const_cast<int64_t *>(all.node_ofs),
            const_cast<int64_t *>(all.tab_ofs), const_cast<int32_t *>(all.order), (PlanBatch *)c->plan_pb.p);
        c->launches++;
    }
    GR_CK(cudaGetLastError());
    std::vector<PlanBatch> pb((size_t)n_batches + 1);
    uint32_t bad_ids = 0;
    GR_CK(cudaMemcpyAsync(pb.data(), c->plan_pb.p, sizeof(PlanBatch) * (size_t)n_batches, cudaMemcpyDeviceToHost,
                          c->stream));
    GR_CK(cudaMemcpyAsync(&bad_ids, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    GR_CK(cudaStreamSynchronize(c->stream));
    if (bad_ids) return GR_ERR_ARG;
    std::vector<BatchInfo> plan(n_batches);
    int64_t slot = 0, mp = 0, mt = 0, mn = 0;
    for (int32_t b = 0; b < n_batches; b++) {
        BatchInfo &bi = plan[b];
        const PlanBatch &q = pb[b];
        bi.first = h_batch_ofs[b];
        bi.n = (int32_t)(h_batch_ofs[b + 1] - h_batch_ofs[b]);
        bi.n_pairs = q.n_pairs;
        bi.n_nodes = q.n_nodes;
        bi.n_tab = q.n_tab;
        bi.max_pins = q.max_pins;
        bi.n2 = q.n2;
        bi.nm = q.nm;
        bi.nmid = q.nmid;
        bi.nl = bi.n - q.n2 - q.nm;
        if ((rc = check_mst_smem(c, bi.max_pins))) return rc;
    }
    for (int32_t b = 0; b < n_batches; b++) {
        plan[b].slot0 = slot;
        slot += plan[b].n_nodes;
        if (plan[b].n_pairs > mp) mp = plan[b].n_pairs;
        if (plan[b].n_tab > mt) mt = plan[b].n_tab;
        if (plan[b].n > mn) mn = plan[b].n;
    }
    int32_t plan_max_pins = 0;
    for (const BatchInfo &bi : plan) plan_max_pins = bi.max_pins > plan_max_pins ? bi.max_pins : plan_max_pins;
    c->plan_max_pins = plan_max_pins;
    if ((rc = ensure_mst_scratch(c, plan_max_pins, c->stream))) return rc;
    if ((rc = ensure_scratch(c, mp, mt, mn, c->stream))) return rc;
    GR_CK(cudaStreamSynchronize(c->stream));
    c->plan = std::move(plan);
    c->plan_nets = total;
    c->plan_slots = slot;
    c->plan_max_pairs = mp;
    c->plan_max_tab = mt;
    c->plan_max_nets = mn;
    return GR_OK;
}

int64_t gr_plan_slots(gr_ctx *c) { return c ? c->plan_slots : -1; }

int gr_plan_check(gr_ctx *c) {
    if (!c) return GR_ERR_ARG;
    if (c->plan.empty()) return GR_ERR_STATE;
    int rc = ensure_h_nxy(c);
    if (rc) return rc;
    const int64_t total = c->plan_nets;
    const size_t bytes = desc_bytes(total > 0 ? total : 1);
    std::vector<int32_t> ids((size_t)total + 1);
    std::vector<char> dev(bytes), host(bytes, 0);
    GR_CK(cudaStreamSynchronize(c->stream));
    if (total > 0)
        GR_CK(cudaMemcpy(ids.data(), c->plan_ids.p, sizeof(int32_t) * total, cudaMemcpyDeviceToHost));
    GR_CK(cudaMemcpy(dev.data(), c->plan_desc.p, bytes, cudaMemcpyDeviceToHost));
    int bad = 0;
    for (const BatchInfo &bi : c->plan) {
        BatchInfo hb{};
        if ((rc = fill_desc(c, ids.data() + bi.first, bi.n, host.data(), total, bi.first, hb))) return rc;
        bad |= hb.n_pairs != bi.n_pairs || hb.n_nodes != bi.n_nodes || hb.n_tab != bi.n_tab ||
               hb.max_pins != bi.max_pins || hb.n2 != bi.n2 || hb.nm != bi.nm || hb.nl != bi.nl || hb.nmid != bi.nmid;
    }
    bad |= memcmp(dev.data(), host.data(), bytes - 64) != 0;
    return bad ? GR_ERR_DEVICE : GR_OK;
}

}  // extern "C"

namespace {

// What a captured plan depends on beyond the contents of device memory: the
// batches' launch shapes and offsets, every buffer address its launches and
// copies use, the launch-shape parameters and the cost mode. A graph is
// replayed only while all of it is unchanged.
std::vector<uint64_t> graph_sig(const gr_ctx *c, int32_t b0, int32_t b1, const void *mst, const void *pat,
                                cudaStream_t s, const void *h_mst, const void *h_pat) {
    std::vector<uint64_t> v;
    auto P = [&](const void *p) { v.push_back((uint64_t)(uintptr_t)p); };
    const void *const ptrs[] = {mst, pat, (const void *)s, h_mst, h_pat, c->plan_desc.p, c->pcost.p,
                          c->ppat.p, c->tab.p, c->dist.p, c->mat.p, (const void *)c->d_pins, (const void *)c->d_pxy,
                          (const void *)c->d_cx, (const void *)c->d_cy, (const void *)c->d_fen, (const void *)c->d_capr,
                          (const void *)c->d_mark, (const void *)c->d_status, (const void *)c->d_dlut,
                          (const void *)c->d_gpos, (const void *)c->d_gdel, (const void *)c->d_pred,
                          (const void *)c->d_queue};
    for (const void *p : ptrs) P(p);
    v.push_back((uint64_t)b0 << 32 | (uint32_t)b1);
    v.push_back((uint64_t)c->plan_nets);
    for (int t = 0; t < GR_TUNE_PARAMS; t++) v.push_back((uint64_t)(uint32_t)c->tune[t]);
    uint32_t beta_bits;
    memcpy(&beta_bits, &c->la_beta, 4);
    v.push_back((uint64_t)c->la_on << 32 | beta_bits);
    for (int32_t b = b0; b < b1; b++) {
        const BatchInfo &bi = c->plan[b];
        const int64_t f[] = {bi.first, (int64_t)bi.n, bi.n_pairs, bi.n_nodes, bi.n_tab, bi.slot0, (int64_t)bi.max_pins,
                             (int64_t)bi.n2, (int64_t)bi.nm, (int64_t)bi.nl, (int64_t)bi.nmid};
        for (int64_t x : f) v.push_back((uint64_t)x);
    }
    return v;
}

// gr_route_plan, optionally with the results copied to page-locked host
// buffers chunk by chunk on the copy stream while later chunks route (the
// copies are part of the graph when one is captured)
int route_plan_impl(gr_ctx *c, int32_t b0, int32_t b1, int64_t *d_mst_edges, int32_t *d_mst_pat, int flags,
                    cudaStream_t s, int64_t *h_mst, int32_t *h_pat) {
    // the Boruvka scratch depends on the launch shapes, which may have changed
    // since gr_plan_set
    int rc0 = ensure_mst_scratch(c, c->plan_max_pins, s);
    if (rc0) return rc0;
    const int32_t chunk = 32;
    auto issue = [&]() -> int {
        for (int32_t b = b0; b < b1; b++) {
            const BatchInfo &bi = c->plan[b];
            const BatchView v = make_view(c->plan_desc.p, c->plan_nets, bi);
            // no per-net tree costs: a plan returns trees and patterns only
            int rc = route_one(c, v, d_mst_edges + bi.slot0, d_mst_pat ? d_mst_pat + bi.slot0 : nullptr, nullptr,
                               (float *)c->pcost.p, (int16_t *)c->ppat.p, s);
            if (rc) return rc;
            if (h_mst && ((b + 1 - b0) % chunk == 0 || b + 1 == b1)) {
                const int32_t c0 = b + 1 - ((b + 1 - b0) % chunk ? (b + 1 - b0) % chunk : chunk);
                const int64_t s0 = c->plan[c0].slot0, s1 = b + 1 < (int32_t)c->plan.size() ? c->plan[b + 1].slot0
                                                                                             : c->plan_slots;
                GR_CK(cudaEventRecord(c->ev_out, s));
                GR_CK(cudaStreamWaitEvent(c->copy_stream, c->ev_out, 0));
                GR_CK(cudaMemcpyAsync(h_mst + s0, d_mst_edges + s0, sizeof(int64_t) * (s1 - s0),
                                      cudaMemcpyDeviceToHost, c->copy_stream));
                if (h_pat)
                    GR_CK(cudaMemcpyAsync(h_pat + s0, d_mst_pat + s0, sizeof(int32_t) * (s1 - s0),
                                          cudaMemcpyDeviceToHost, c->copy_stream));
            }
        }
        if (h_mst) {  // the copy stream joins back
            GR_CK(cudaEventRecord(c->ev_copy_done, c->copy_stream));
            GR_CK(cudaStreamWaitEvent(s, c->ev_copy_done, 0));
        }
        return GR_OK;
    };
    if (!(flags & GR_PLAN_GRAPH)) return issue();
    GraphCache &gc = c->graph;
    std::vector<uint64_t> sig = graph_sig(c, b0, b1, d_mst_edges, d_mst_pat, s, h_mst, h_pat);
    if (!(gc.exec && gc.sig == sig)) {
        drop_graph(c);
        int64_t before = c->launches;
        cudaGraph_t graph = nullptr;
        GR_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int rc = issue();
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return GR_ERR_CUDA;
        cudaError_t ie = cudaGraphInstantiate(&gc.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            gc.exec = nullptr;
            return GR_ERR_CUDA;
        }
        gc.sig = std::move(sig);
        gc.launches = c->launches - before;
        c->launches = before;
    }
    GR_CK(cudaGraphLaunch(gc.exec, s));
    c->launches += gc.launches;
    return GR_OK;
}

// The learned route of the whole plan from reset on stream s: before every
// `every` batches, the network predicts from the current state (features
// x 1/16) the demand still to come (output x 16; in GR_LA_EXCESS mode its
// part beyond the remaining capacity), the GCELL cost becomes
// exp(-0.5 (cap_remaining - beta pred)) and the Fenwick trees are rebuilt;
// at the end the plain cost and its trees are restored. Every step is on the
// device (the network's forward pass included), so with GR_PLAN_GRAPH the
// whole route is one captured CUDA graph, replayed while its signature holds.
int route_lookahead_impl(gr_ctx *c, gr_cnn *cnn, int32_t every, float beta, int mode, int64_t *mst, int32_t *pat,
                         int flags, cudaStream_t s) {
    const int64_t n = c->csize;
    const int32_t nb = (int32_t)c->plan.size();
    int rc;
    if ((rc = ensure(c->la_feat, sizeof(float) * 2 * n, s)) || (rc = ensure(c->la_out, sizeof(float) * 2 * n, s)) ||
        (rc = ensure_mst_scratch(c, c->plan_max_pins, s)))
        return rc;
    if (!c->d_pred && cudaMalloc(&c->d_pred, sizeof(float) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        return GR_ERR_NOMEM;
    }
    // any graph of the plain route holds the cost mode it was captured with
    drop_graph(c);
    float *feat = (float *)c->la_feat.p, *out = (float *)c->la_out.p, *pred = out + n;
    auto issue = [&]() -> int {
        int r;
        c->la_on = false;
        c->la_beta = 0.0f;
        GR_CK(cudaMemcpyAsync(c->d_capr, c->d_cap0, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
        GR_CK(cudaMemsetAsync(c->d_mark, 0, sizeof(uint32_t) * (size_t)(n / 32 + 2), s));
        GR_CK(cudaMemsetAsync(c->d_queue, 0, 16, s));
        if (beta == 0.0f && (r = rebuild_fenwick(c, s))) return r;
        for (int32_t b0 = 0; b0 < nb; b0 += every) {
            const int32_t b1 = b0 + every < nb ? b0 + every : nb;
            if (beta > 0.0f) {
                k_features<<<grid_for(c, n, 16), kThreads, 0, s>>>(c->g, (int)n, c->d_cap0, c->d_capr, 1.0f / 16.0f,
                                                                   feat);
                c->launches++;
                if ((r = gr_cnn_forward_async(cnn, feat, out, s))) return r;
                const int64_t gz = (int64_t)c->g.Z * c->g.X * c->g.Y;
                k_la_pred<<<grid_for(c, gz, 16), kThreads, 0, s>>>((int)gz, out, feat, mode == GR_LA_EXCESS, pred);
                k_pred_to_cells<<<grid_for(c, n, 16), kThreads, 0, s>>>(c->g, (int)n, pred, c->d_pred);
                c->launches += 2;
                GR_CK(cudaGetLastError());
                c->la_on = true;
                c->la_beta = beta;
                if ((r = rebuild_fenwick(c, s))) return r;
            }
            for (int32_t b = b0; b < b1; b++) {
                const BatchInfo &bi = c->plan[b];
                const BatchView v = make_view(c->plan_desc.p, c->plan_nets, bi);
                if ((r = route_one(c, v, mst + bi.slot0, pat ? pat + bi.slot0 : nullptr, nullptr, (float *)c->pcost.p,
                                   (int16_t *)c->ppat.p, s)))
                    return r;
            }
        }
        c->la_on = false;  // the plain cost and its trees back
        c->la_beta = 0.0f;
        return rebuild_fenwick(c, s);
    };
    if (!(flags & GR_PLAN_GRAPH)) return issue();
    GraphCache &gc = c->la_graph;
    std::vector<uint64_t> sig = graph_sig(c, 0, nb, mst, pat, s, nullptr, nullptr);
    uint32_t beta_bits;
    memcpy(&beta_bits, &beta, 4);
    for (uint64_t x : {(uint64_t)(uintptr_t)cnn, (uint64_t)every, (uint64_t)beta_bits, (uint64_t)mode,
                       (uint64_t)(uintptr_t)c->la_feat.p, (uint64_t)(uintptr_t)c->la_out.p})
        sig.push_back(x);
    if (!(gc.exec && gc.sig == sig)) {
        drop_la_graph(c);
        const int64_t before = c->launches;
        cudaGraph_t graph = nullptr;
        GR_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int r = issue();
        const cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (r) {
            if (graph) cudaGraphDestroy(graph);
            return r;
        }
        if (ce != cudaSuccess) return GR_ERR_CUDA;
        const cudaError_t ie = cudaGraphInstantiate(&gc.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            gc.exec = nullptr;
            return GR_ERR_CUDA;
        }
        gc.sig = std::move(sig);
        gc.launches = c->launches - before;
        c->launches = before;
    }
    GR_CK(cudaGraphLaunch(gc.exec, s));
    c->launches += gc.launches;
    c->la_on = false;  // the graph ends with the plain cost restored
    c->la_beta = 0.0f;
    return GR_OK;
}

}  // namespace

extern "C" {

int gr_route_plan(gr_ctx *c, int32_t b0, int32_t b1, int64_t *d_mst_edges, int32_t *d_mst_pat, int flags,
                  void *stream) {
    if (!c || !d_mst_edges || b0 < 0 || b1 < b0 || b1 > (int32_t)c->plan.size()) return GR_ERR_ARG;
    if (c->plan.empty() && b1 > 0) return GR_ERR_STATE;
    return route_plan_impl(c, b0, b1, d_mst_edges, d_mst_pat, flags, pick(c, stream), nullptr, nullptr);
}

int gr_route_design_host(gr_ctx *c, int32_t n_nets, const int64_t *h_pin_ofs, const int32_t *h_pins,
                         int32_t n_batches, const int64_t *h_batch_ofs, const int32_t *h_net_ids,
                         int64_t *h_mst_edges, int32_t *h_mst_pat, int flags) {
    if (!c || !h_mst_edges) return GR_ERR_ARG;
    int rc;
    if ((rc = gr_set_nets(c, n_nets, h_pin_ofs, h_pins))) return rc;
    if ((rc = gr_plan_set(c, n_batches, h_batch_ofs, h_net_ids))) return rc;
    if ((rc = gr_reset(c, nullptr))) return rc;
    const int64_t slots = c->plan_slots;
    if ((rc = ensure(c->out_mst, sizeof(int64_t) * (slots + 1), c->stream)) ||
        (rc = ensure(c->out_pat, sizeof(int32_t) * (slots + 1), c->stream)))
        return rc;
    int64_t *mst = (int64_t *)c->out_mst.p;
    int32_t *pat = (int32_t *)c->out_pat.p;
    // with page-locked results, each chunk of batches is copied back on the
    // copy stream while the next chunks route (inside the graph with GR_PLAN_GRAPH)
    auto pinned = [](const void *h) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    };
    if (pinned(h_mst_edges) && (!h_mst_pat || pinned(h_mst_pat))) {
        rc = route_plan_impl(c, 0, n_batches, mst, pat, flags, c->stream, h_mst_edges, h_mst_pat);
    } else {
        rc = route_plan_impl(c, 0, n_batches, mst, pat, flags, c->stream, nullptr, nullptr);
        if (!rc) {
            GR_CK(cudaMemcpyAsync(h_mst_edges, mst, sizeof(int64_t) * slots, cudaMemcpyDeviceToHost, c->stream));
            if (h_mst_pat)
                GR_CK(cudaMemcpyAsync(h_mst_pat, pat, sizeof(int32_t) * slots, cudaMemcpyDeviceToHost, c->stream));
        }
    }
    const int sr = gr_sync(c);
    return rc ? rc : sr;
}

int gr_sync(gr_ctx *c) {
    if (!c) return GR_ERR_ARG;
    GR_CK(cudaStreamSynchronize(c->stream));
    return gr_status(c) ? GR_ERR_DEVICE : GR_OK;
}

uint32_t gr_status(gr_ctx *c) {
    if (!c) return 0;
    uint32_t st = 0;
    if (cudaMemcpyAsync(&st, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
        return 0xffffffffu;
    cudaStreamSynchronize(c->stream);
    return st;
}

int gr_clear_status(gr_ctx *c) {
    if (!c) return GR_ERR_ARG;
    GR_CK(cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream));
    return GR_OK;
}

int gr_get_capr(gr_ctx *c, int32_t *h_out) {
    if (!c || !h_out) return GR_ERR_ARG;
    GR_CK(cudaStreamSynchronize(c->stream));
    GR_CK(cudaMemcpyAsync(h_out, c->d_capr, sizeof(int32_t) * c->csize, cudaMemcpyDeviceToHost, c->stream));
    GR_CK(cudaStreamSynchronize(c->stream));
    return GR_OK;
}

int gr_get_demand(gr_ctx *c, int32_t *h_out) {
    int rc = gr_get_capr(c, h_out);
    if (rc) return rc;
    for (int64_t i = 0; i < c->csize; i++) h_out[i] = c->h_cap0[i] - h_out[i];
    return GR_OK;
}

int gr_get_fenwick(gr_ctx *c, float *h_out) {
    if (!c || !h_out) return GR_ERR_ARG;
    GR_CK(cudaStreamSynchronize(c->stream));
    GR_CK(cudaMemcpyAsync(h_out, c->d_fen, sizeof(float) * c->csize, cudaMemcpyDeviceToHost, c->stream));
    GR_CK(cudaStreamSynchronize(c->stream));
    return GR_OK;
}

void *gr_stream(gr_ctx *c) { return c ? (void *)c->stream : nullptr; }

int gr_features(gr_ctx *c, float *d_feat, float scale, void *stream) {
    if (!c || !d_feat) return GR_ERR_ARG;
    cudaStream_t s = pick(c, stream);
    k_features<<<grid_for(c, c->csize, 16), kThreads, 0, s>>>(c->g, (int)c->csize, c->d_cap0, c->d_capr, scale,
                                                               d_feat);
    GR_CK(cudaGetLastError());
    return GR_OK;
}

int gr_set_lookahead(gr_ctx *c, const float *d_pred, float beta, void *stream) {
    if (!c || !(beta >= 0.0f)) return GR_ERR_ARG;
    cudaStream_t s = pick(c, stream);
    drop_graph(c);  // a captured plan holds the cost mode it was captured with
    if (!d_pred || beta == 0.0f) {
        c->la_on = false;
        c->la_beta = 0.0f;
    } else {
        if (!c->d_pred && cudaMalloc(&c->d_pred, sizeof(float) * (size_t)c->csize) != cudaSuccess) {
            cudaGetLastError();
            return GR_ERR_NOMEM;
        }
        k_pred_to_cells<<<grid_for(c, c->csize, 16), kThreads, 0, s>>>(c->g, (int)c->csize, d_pred, c->d_pred);
        GR_CK(cudaGetLastError());
        c->la_on = true;
        c->la_beta = beta;
    }
    return rebuild_fenwick(c, s);
}

int gr_route_plan_lookahead(gr_ctx *c, gr_cnn *cnn, int32_t every, float beta, int mode, int64_t *d_mst_edges,
                            int32_t *d_mst_pat, int flags, void *stream) {
    if (!c || !cnn || !d_mst_edges || every < 1 || !(beta >= 0.0f) || (mode != GR_LA_DEMAND && mode != GR_LA_EXCESS))
        return GR_ERR_ARG;
    if (c->plan.empty()) return GR_ERR_STATE;
    int dev = -1, cin = 0, cout = 0, H = 0, W = 0;
    int rc = gr_cnn_info(cnn, &dev, &cin, &cout, &H, &W);
    if (rc) return rc;
    if (dev != c->device || cin != 2 * c->g.Z || cout != c->g.Z || H != c->g.Y || W != c->g.X) return GR_ERR_ARG;
    return route_lookahead_impl(c, cnn, every, beta, mode, d_mst_edges, d_mst_pat, flags, pick(c, stream));
}

int gr_route_design_lookahead_host(gr_ctx *c, gr_cnn *cnn, int32_t every, float beta, int mode,
                                   int64_t *h_mst_edges, int32_t *h_mst_pat) {
    if (!c || !h_mst_edges) return GR_ERR_ARG;
    if (c->plan.empty()) return GR_ERR_STATE;
    const int64_t slots = c->plan_slots;
    int rc;
    if ((rc = ensure(c->out_mst, sizeof(int64_t) * (slots + 1), c->stream)) ||
        (rc = ensure(c->out_pat, sizeof(int32_t) * (slots + 1), c->stream)))
        return rc;
    int64_t *mst = (int64_t *)c->out_mst.p;
    int32_t *pat = (int32_t *)c->out_pat.p;
    rc = gr_route_plan_lookahead(c, cnn, every, beta, mode, mst, pat, GR_PLAN_GRAPH, nullptr);
    if (!rc) {
        GR_CK(cudaMemcpyAsync(h_mst_edges, mst, sizeof(int64_t) * slots, cudaMemcpyDeviceToHost, c->stream));
        if (h_mst_pat)
            GR_CK(cudaMemcpyAsync(h_mst_pat, pat, sizeof(int32_t) * slots, cudaMemcpyDeviceToHost, c->stream));
    }
    const int sr = gr_sync(c);
    const int cr = gr_cnn_check(cnn);
    return rc ? rc : (sr ? sr : cr);
}

int gr_tune_set(gr_ctx *c, int param, int value) {
    if (!c || param < 0 || param >= GR_TUNE_PARAMS) return GR_ERR_ARG;
    if (param == GR_TUNE_MST_CLUSTER_MIN_PINS) {
        if (value != 0 && (value <= kMstMidPins || value > GR_MAX_PINS)) return GR_ERR_ARG;
    } else if (param == GR_TUNE_LPAT_SPLIT) {
        if (value != 0 && value != 1 && value != 2 && value != 4) return GR_ERR_ARG;
    } else if (param == GR_TUNE_MST_QUEUE) {
        if (value != 0 && value != 1) return GR_ERR_ARG;
    } else if (value < 64 || value > 1024 || value % 32) {
        return GR_ERR_ARG;
    }
    if (c->tune[param] != value) {
        GR_CK(cudaStreamSynchronize(c->stream));
        drop_graph(c);  // a captured plan holds the old launch shapes
        drop_la_graph(c);
        c->tune[param] = value;
    }
    return GR_OK;
}

int gr_tune_get(gr_ctx *c, int param, int *value) {
    if (!c || !value || param < 0 || param >= GR_TUNE_PARAMS) return GR_ERR_ARG;
    *value = c->tune[param];
    return GR_OK;
}

int gr_profile_enable(gr_ctx *c, int on) {
    if (!c) return GR_ERR_ARG;
    c->profiling = on != 0;
    return GR_OK;
}

int gr_profile_read(gr_ctx *c, double *ms, int64_t *launches, int reset) {
    if (!c) return GR_ERR_ARG;
    GR_CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i + 1 < c->ev_used; i += 2) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, c->ev[i], c->ev[i + 1]) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        int k = c->ev_kind[i / 2];
        c->prof_ms[k] += t;
        c->prof_n[k] += 1;
    }
    c->ev_used = 0;
    for (int k = 0; k < GR_PROF_KINDS; k++) {
        if (ms) ms[k] = c->prof_ms[k];
        if (launches) launches[k] = c->prof_n[k];
        if (reset) {
            c->prof_ms[k] = 0;
            c->prof_n[k] = 0;
        }
    }
    return GR_OK;
}

const char *gr_kernel_name(int kind) {
    static const char *names[GR_PROF_KINDS] = {"k_fen_init", "k_qtable", "k_lpat",   "k_mst_pin2",  "k_mark",
                                               "k_track_commit", "k_finalize", "k_lpat_pairs", "k_mst_warp",
                                               "k_mst_large"};
    return (kind >= 0 && kind < GR_PROF_KINDS) ? names[kind] : "";
}

int64_t gr_launch_count(gr_ctx *c) { return c ? c->launches : -1; }

}  // extern "C"

// ------------------------------------------------------------------------
// gr_brvsk_build_static: the Boruvka stage with no allocation and no context.
//
// Some callers cannot allocate device memory when they need the spanning
// trees: an engine whose memory pool already holds the device's free memory,
// or a loop that must not pay the device-wide synchronisation that cudaFree
// implies. This entry point keeps everything it needs -- the batch's offset
// tables and, for nets whose pair-cost matrix exceeds shared memory, the
// per-CTA matrices -- in one file-scope device array of fixed size, so a call
// launches kernels and copies pin counts, and allocates nothing.
//
// The array is one per device. Calls on a device share it and leave their
// contents behind; each call rewrites the tables it reads and clears the
// status word before its kernels run. Calls whose work may overlap on the
// device (on streams with no ordering between them) race on the array and
// corrupt each other's results: issue them on one stream.
// ------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr int kStaticMaxNets = GR_STATIC_MAX_NETS;         // nets per call
constexpr int kStaticMaxPins = GR_STATIC_MAX_PINS;         // pins per net
constexpr int kStaticMaxDevices = 64;
// layout of the array (offsets in bytes, each a multiple of 256)
constexpr size_t kSsStatus = 0;                                             // uint32
constexpr size_t kSsNpin = 256;                                             // int32 [nets]
constexpr size_t kSsOrder = kSsNpin + sizeof(int32_t) * kStaticMaxNets;     // int32 [nets]
constexpr size_t kSsPairOfs = kSsOrder + sizeof(int32_t) * kStaticMaxNets;  // int64 [nets]
constexpr size_t kSsNodeOfs = kSsPairOfs + sizeof(int64_t) * kStaticMaxNets;
constexpr size_t kSsMat = kSsNodeOfs + sizeof(int64_t) * kStaticMaxNets;    // float matrices
static_assert(kSsMat % 256 == 0 && kSsMat + sizeof(float) * kStaticMaxPins * mst_ld(kStaticMaxPins) <= kStaticScratchBytes,
              "static Boruvka scratch holds its tables and at least one largest matrix");

}  // namespace

static __device__ __align__(256) unsigned char g_brvsk_scratch[kStaticScratchBytes];

namespace {

// Pair and slot offsets of a batch from its pin counts: one CTA of 1024
// threads, each scanning a contiguous chunk, 64-bit sums throughout. (The
// nets' processing order is uploaded beside the pin counts.)
__global__ void __launch_bounds__(1024) k_static_desc(int32_t n, const int32_t *__restrict__ npin,
                                                      int64_t *__restrict__ pair_ofs, int64_t *__restrict__ node_ofs) {
    const unsigned FULL = 0xffffffffu;
    __shared__ long long wp[32], wn[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int chunk = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int c0 = min(n, tid * chunk), c1 = min(n, c0 + chunk);
    long long sp = 0, sn = 0;
    for (int i = c0; i < c1; i++) {
        const long long k = npin[i];
        sp += k * (k - 1) / 2;
        sn += k;
    }
    long long xp = sp, xn = sn;  // inclusive scans within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long yp = __shfl_up_sync(FULL, xp, o), yn = __shfl_up_sync(FULL, xn, o);
        if (lane >= o) {
            xp += yp;
            xn += yn;
        }
    }
    if (lane == 31) {
        wp[warp] = xp;
        wn[warp] = xn;
    }
    __syncthreads();
    if (warp == 0) {
        const long long a = lane < nw ? wp[lane] : 0, b = lane < nw ? wn[lane] : 0;
        long long ia = a, ib = b;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long ya = __shfl_up_sync(FULL, ia, o), yb = __shfl_up_sync(FULL, ib, o);
            if (lane >= o) {
                ia += ya;
                ib += yb;
            }
        }
        if (lane < nw) {
            wp[lane] = ia - a;
            wn[lane] = ib - b;
        }
    }
    __syncthreads();
    long long P = wp[warp] + xp - sp, N = wn[warp] + xn - sn;
    for (int i = c0; i < c1; i++) {
        const long long k = npin[i];
        pair_ofs[i] = P;
        node_ofs[i] = N;
        P += k * (k - 1) / 2;
        N += k;
    }
}

struct StaticDev {
    unsigned char *base = nullptr;
    int sms = 0;
    bool ready = false;
};
std::mutex g_static_mu;
StaticDev g_static_dev[kStaticMaxDevices];

// Once per device, with that device current: the array's address, the SM
// count, and the kernels' attributes (which also loads them).
int static_setup(int dev, StaticDev &out) {
    if (dev < 0 || dev >= kStaticMaxDevices) return GR_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_static_mu);
    StaticDev &d = g_static_dev[dev];
    if (!d.ready) {
        void *p = nullptr;
        GR_CK(cudaGetSymbolAddress(&p, g_brvsk_scratch));
        int sms = 0, optin = 0;
        GR_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        GR_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        if (optin < kMstSmemMax + 1024) {
            fprintf(stderr, "iitmgr_b200: device allows %d bytes of shared memory per block\n", optin);
            return GR_ERR_CUDA;
        }
        GR_CK(cudaFuncSetAttribute(k_mst_large, cudaFuncAttributeMaxDynamicSharedMemorySize, kMstSmemMax));
        cudaFuncAttributes fa;
        GR_CK(cudaFuncGetAttributes(&fa, k_static_desc));
        d.base = (unsigned char *)p;
        d.sms = sms > 0 ? sms : 1;
        d.ready = true;
    }
    out = d;
    return GR_OK;
}

}  // namespace

extern "C" int gr_brvsk_build_static(const int32_t *h_npin, int32_t n_nets, const float *d_pair_cost,
                                     int64_t *d_mst_edges, float *d_net_dist, uint32_t *d_status, void *stream) {
    if (n_nets < 0 || n_nets > kStaticMaxNets) return GR_ERR_ARG;
    if (n_nets == 0) return GR_OK;
    if (!h_npin || !d_pair_cost || !d_mst_edges) return GR_ERR_ARG;
    // nets whose pair-cost matrix fits in shared memory first, in batch
    // order, then the larger ones: each group gets its own launch, so the
    // small nets never queue behind the few CTAs the array's matrices allow
    int max_small = 0, max_large = 0;
    std::vector<int32_t> order((size_t)n_nets);
    int32_t n_small = 0;
    for (int32_t i = 0; i < n_nets; i++) {
        if (h_npin[i] < 0) return GR_ERR_ARG;
        if (h_npin[i] > kStaticMaxPins) return GR_ERR_NET_TOO_LARGE;
        if (mst_mat_in_smem(h_npin[i])) {
            order[n_small++] = i;
            max_small = h_npin[i] > max_small ? h_npin[i] : max_small;
        } else {
            max_large = h_npin[i] > max_large ? h_npin[i] : max_large;
        }
    }
    for (int32_t i = 0, k = n_small; i < n_nets; i++)
        if (!mst_mat_in_smem(h_npin[i])) order[k++] = i;
    int dev = 0;
    GR_CK(cudaGetDevice(&dev));
    StaticDev sd;
    int rc = static_setup(dev, sd);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t *st = d_status ? d_status : (uint32_t *)(sd.base + kSsStatus);
    int32_t *npin = (int32_t *)(sd.base + kSsNpin), *dorder = (int32_t *)(sd.base + kSsOrder);
    int64_t *pair_ofs = (int64_t *)(sd.base + kSsPairOfs), *node_ofs = (int64_t *)(sd.base + kSsNodeOfs);
    GR_CK(cudaMemsetAsync(sd.base + kSsStatus, 0, sizeof(uint32_t), s));
    GR_CK(cudaMemcpyAsync(npin, h_npin, sizeof(int32_t) * (size_t)n_nets, cudaMemcpyHostToDevice, s));
    GR_CK(cudaMemcpyAsync(dorder, order.data(), sizeof(int32_t) * (size_t)n_nets, cudaMemcpyHostToDevice, s));
    k_static_desc<<<1, 1024, 0, s>>>(n_nets, npin, pair_ofs, node_ofs);
    GR_CK(cudaGetLastError());
    BatchView v{};
    v.n = n_nets;
    v.npin = npin;
    v.pair_ofs = pair_ofs;
    v.node_ofs = node_ofs;
    v.order = dorder;
    // k_mst_large: the small nets with their matrices in shared memory on up
    // to 8 CTAs per SM; the larger ones with one matrix per CTA in the array
    // (as many CTAs as it holds, at most one per SM)
    if (n_small > 0) {
        v.max_pins = max_small;
        const size_t smem = mst_smem(max_small) + (size_t)max_small * mst_ld(max_small) * sizeof(float);
        const int blocks = n_small < sd.sms * 8 ? n_small : sd.sms * 8;
        k_mst_large<<<blocks, max_small <= kMstMidPins ? 128 : 512, smem, s>>>(
            GridC{}, v, d_pair_cost, d_mst_edges, d_net_dist, st, nullptr, 0, 0, n_small, MarkOut{});
        GR_CK(cudaGetLastError());
    }
    if (n_small < n_nets) {
        v.max_pins = max_large;
        const size_t mat = (size_t)max_large * mst_ld(max_large) * sizeof(float);
        const size_t fit = (kStaticScratchBytes - kSsMat) / mat;
        int blocks = (int)(fit < (size_t)sd.sms ? fit : (size_t)sd.sms);
        blocks = n_nets - n_small < blocks ? n_nets - n_small : blocks;
        k_mst_large<<<blocks, 512, mst_smem(max_large), s>>>(GridC{}, v, d_pair_cost, d_mst_edges, d_net_dist, st,
                                                             (uint32_t *)(sd.base + kSsMat), (int64_t)max_large * mst_ld(max_large),
                                                             n_small, n_nets - n_small, MarkOut{});
        GR_CK(cudaGetLastError());
    }
    return GR_OK;
}
