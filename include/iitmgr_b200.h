/*
 * iitmgr_b200.h -- C ABI of the B200-native routing hot path.
 *
 * Replaces the per-batch GPU path of SammithKanur/iitmGlobalRouter in its
 * "-bit_pmodel" mode: 3D L-pattern costing of every pin pair against
 * per-track Fenwick cost trees, per-net Boruvka rectilinear spanning tree,
 * and the Fenwick edge commit. Plain C types only: device pointers are
 * `void*`-compatible CUDA allocations, streams are `cudaStream_t` passed as
 * `void*` (NULL = the context's own stream).
 *
 * Grid encoding (reference util.hpp:37-44, WIRE_ENC):
 *     enc(z,x,y) = z*X*Y + (z odd ? x*Y + y : y*X + x)
 * Even layers route along x, odd layers along y; each track is contiguous.
 *
 * Errors: every entry point returns GR_OK (0) or a negative GR_ERR_* code.
 * Kernels that find invalid data record it in a device status word; calls
 * that synchronise (gr_sync, gr_get_*, *_host entry points) report it as
 * GR_ERR_DEVICE and gr_status() returns the GR_ST_* bits.
 * Threading: a context may be used by one host thread at a time.
 */
#ifndef IITMGR_B200_H
#define IITMGR_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GR_OK 0
#define GR_ERR_ARG (-1)          /* invalid argument                         */
#define GR_ERR_CUDA (-2)         /* a CUDA runtime call failed                */
#define GR_ERR_NOMEM (-3)        /* host or device allocation failed          */
#define GR_ERR_STATE (-4)        /* call out of order (no nets, no plan, ...) */
#define GR_ERR_NET_TOO_LARGE (-5)/* a net has more pins than GR_MAX_PINS      */
#define GR_ERR_DEVICE (-6)       /* a kernel reported invalid data            */
#define GR_ERR_IO (-7)           /* file could not be opened / written        */
#define GR_ERR_PARSE (-8)        /* malformed .cap / .net text                */
#define GR_ERR_NONINTEGER (-9)   /* a capacity is not an integer              */

/* device status bits (gr_status) */
#define GR_ST_BAD_EDGE 0x1u      /* MST slot not an edge of its net           */
#define GR_ST_BAD_PATTERN 0x2u   /* pattern id does not route the pair        */
#define GR_ST_MST_ROUNDS 0x4u    /* Boruvka did not finish in its round bound */
#define GR_ST_BAD_PIN 0x8u       /* pin encoding outside the grid             */

#define GR_MAX_PINS 4096         /* pins per net handled by this library     */

typedef struct gr_ctx gr_ctx;

int gr_version(void);
const char *gr_error_string(int code);

/* ------------------------------------------------------------ context */

/* Grid of X*Y*Z GCELLs with integer capacities h_cap[enc] (host memory).
 * Allocates the remaining-capacity, demand and Fenwick state on `device`
 * and builds the Fenwick trees.
 * Replaces: read_data.hpp:557-562 (d_cube_data_bit upload) and
 * BIT_UTIL_SPACE::init_bit_data (bit_util.hpp:192-200). Z must be >= 3. */
int gr_create(gr_ctx **out, int device, int X, int Y, int Z, const int32_t *h_cap);
int gr_destroy(gr_ctx *ctx);

/* demand := 0, Fenwick trees rebuilt from the capacities (bit_util.hpp:192). */
int gr_reset(gr_ctx *ctx, void *stream);

/* The design's nets: net i holds pins h_pins[h_pin_ofs[i] .. h_pin_ofs[i+1]),
 * each pin a WIRE_ENC cell id, 2 <= pins <= GR_MAX_PINS. Pins are expected
 * deduplicated and ascending (read_data.hpp:413-432); pair order and edge
 * ids follow this order. Copied to device once.
 * Replaces: READ_DATA::add_net_gpu_data (read_data.hpp:486-524). */
int gr_set_nets(gr_ctx *ctx, int32_t n_nets, const int64_t *h_pin_ofs, const int32_t *h_pins);

/* ------------------------------------------------------------ boundaries */

/* lpattern: for each pair i (src = d_pairs[2i], dst = d_pairs[2i+1], cell
 * ids) the cheapest one-bend 3D L pattern under the current cost state:
 * d_cost[i] (FP32 sum of Fenwick range queries) and d_pat[i] (pattern id
 * = via1 * ceil(Z/2) + v). Ties go to the lowest pattern id.
 * Replaces: BIT_UTIL_SPACE::get_gpu_lpat_dist<5>(lpat, pt_prs, lpat_res,
 * MAX_PTS) (bit_util.hpp:118-119, launched at test_lpat.hpp:360). */
int gr_lpattern(gr_ctx *ctx, const int32_t *d_pairs, int64_t n_pairs, float *d_cost, int16_t *d_pat,
                void *stream);

/* brvsk_build: per-net Boruvka spanning tree of a batch. The batch is the
 * list h_net_ids[0..n_nets) of design nets (host memory); d_pair_cost holds
 * the batch's pair costs in reference pair order (net after net; within a
 * net pair (j,k), k<j, at j(j-1)/2+k). Output: for net b of the batch with
 * n pins, n slots at d_mst_edges[sum of earlier n]: n-1 edges packed as
 * (b<<30)|(u<<15)|v (u, v component roots when the edge was chosen) then -1;
 * d_net_dist[b] = sum of the chosen costs.
 * Replaces: MST_BUILD::get_mst_tree<0>(bt_id, num_edges) (mst_build.hpp:16-17,
 * called at test_lpat.hpp:380) up to, not including, its commit step. */
int gr_brvsk_build(gr_ctx *ctx, const int32_t *h_net_ids, int32_t n_nets, const float *d_pair_cost,
                   int64_t *d_mst_edges, float *d_net_dist, void *stream);

/* brvsk_build without a context and without allocating: for callers whose
 * device memory is already spoken for (an engine's pool holds it) or that
 * must not pay the device-wide synchronisation of cudaFree. No counterpart
 * in the reference. Net b of the batch has h_npin[b] pins (host memory);
 * d_pair_cost, d_mst_edges and d_net_dist (may be NULL) are laid out and
 * filled exactly as by gr_brvsk_build. Status bits (GR_ST_MST_ROUNDS) are
 * ORed into *d_status when it is not NULL. Works on the calling thread's
 * current device; stream must belong to it (NULL: the legacy stream).
 * Limits: at most GR_STATIC_MAX_NETS nets, GR_STATIC_MAX_PINS pins per net
 * (GR_ERR_ARG / GR_ERR_NET_TOO_LARGE beyond). Its scratch is one fixed
 * 16 MiB device array per device: the first call on a device does the
 * set-up (finds the array, loads the kernels) and should come before any
 * stream capture; calls that may overlap on the device race on the array,
 * so issue them on one stream. */
#define GR_STATIC_MAX_NETS 65536
#define GR_STATIC_MAX_PINS 1024
int gr_brvsk_build_static(const int32_t *h_npin, int32_t n_nets, const float *d_pair_cost, int64_t *d_mst_edges,
                          float *d_net_dist, uint32_t *d_status, void *stream);

/* mst_bit_commit: mark every GCELL on the chosen L pattern of every MST
 * edge of the batch (deduplicated over the batch), then each marked cell
 * gains one unit of demand and its track's Fenwick tree gains
 * cost(cap-1)-cost(cap). d_pair_pat: the batch's pair patterns; d_mst_pat
 * (may be NULL) receives the pattern of each MST slot (-1 for sentinels).
 * Replaces: MST_BIT_COMMIT::bit_commit_edges(max_nodes_len)
 * (mst_bit_commit.hpp:236-255, via MST_COMMIT::gpu_commit_edges,
 * mst_commit.hpp:342-346). */
int gr_mst_bit_commit(gr_ctx *ctx, const int32_t *h_net_ids, int32_t n_nets, const int64_t *d_mst_edges,
                      const int16_t *d_pair_pat, int32_t *d_mst_pat, void *stream);

/* The three stages fused for one batch (the reference's per-batch body of
 * TEST_LPAT::test_gpu_lpat, test_lpat.hpp:280-450). d_pair_cost /
 * d_pair_pat / d_net_dist may be NULL. */
int gr_route_batch(gr_ctx *ctx, const int32_t *h_net_ids, int32_t n_nets, int64_t *d_mst_edges,
                   int32_t *d_mst_pat, float *d_net_dist, float *d_pair_cost, int16_t *d_pair_pat,
                   void *stream);

/* ------------------------------------------------------------ plans */

/* A routing plan: batch b = h_net_ids[h_batch_ofs[b] .. h_batch_ofs[b+1]).
 * Uploaded once; gr_route_plan then routes a range of batches with no host
 * work per batch. Output slots of batch b start at the plan's slot offset
 * (sum of pins of all nets of earlier batches), as in the reference's
 * td_net_mst_edges / td_mst_lpat_pat (mst_util.hpp:317-318). */
int gr_plan_set(gr_ctx *ctx, int32_t n_batches, const int64_t *h_batch_ofs, const int32_t *h_net_ids);
int64_t gr_plan_slots(gr_ctx *ctx);
/* Self-check of the uploaded plan (no counterpart in the reference): the
 * descriptor gr_plan_set built on the device against one built on the host
 * batch by batch. GR_OK when equal, GR_ERR_DEVICE when not. */
int gr_plan_check(gr_ctx *ctx);
#define GR_PLAN_GRAPH 0x1 /* replay the batches as one captured CUDA graph */
int gr_route_plan(gr_ctx *ctx, int32_t b0, int32_t b1, int64_t *d_mst_edges, int32_t *d_mst_pat, int flags,
                  void *stream);

/* End to end with host buffers: upload nets and plan, reset, route every
 * batch, copy MST slots and patterns back (h_* are host pointers).
 * flags: GR_PLAN_GRAPH routes the plan as one captured CUDA graph. */
int gr_route_design_host(gr_ctx *ctx, int32_t n_nets, const int64_t *h_pin_ofs, const int32_t *h_pins,
                         int32_t n_batches, const int64_t *h_batch_ofs, const int32_t *h_net_ids,
                         int64_t *h_mst_edges, int32_t *h_mst_pat, int flags);

/* ------------------------------------------------------------ state */

int gr_sync(gr_ctx *ctx);                         /* wait; GR_ERR_DEVICE if status set */
uint32_t gr_status(gr_ctx *ctx);                  /* GR_ST_* bits seen so far          */
int gr_clear_status(gr_ctx *ctx);
int gr_get_capr(gr_ctx *ctx, int32_t *h_out);     /* remaining capacity, CSIZE         */
int gr_get_demand(gr_ctx *ctx, int32_t *h_out);   /* committed demand, CSIZE           */
int gr_get_fenwick(gr_ctx *ctx, float *h_out);    /* Fenwick nodes, CSIZE              */
void *gr_stream(gr_ctx *ctx);                     /* the context's cudaStream_t        */
/* kernel launches issued by this context since creation (for accounting) */
int64_t gr_launch_count(gr_ctx *ctx);

/* Per-kernel timing: while enabled, every launch outside a graph capture is
 * bracketed by CUDA events on its stream. gr_profile_read synchronises and
 * returns, per kernel kind, the summed milliseconds and launch counts since
 * the last reset. Costs an event pair per launch; off by default. */
#define GR_K_FEN_INIT 0
#define GR_K_QTABLE 1
#define GR_K_LPAT 2
#define GR_K_MST 3
#define GR_K_MARK 4
#define GR_K_FEN_UPDATE 5
#define GR_K_FINALIZE 6
#define GR_K_LPAT_PAIRS 7
#define GR_K_MST_WARP 8
#define GR_K_MST_LARGE 9
#define GR_PROF_KINDS 10
/* Congestion lookahead (no counterpart in the reference). gr_features
 * writes the network input from the current state: d_feat[z][y][x] =
 * demand * scale, d_feat[Z + z][y][x] = capacity * scale (2Z x Y x X f32,
 * device). gr_set_lookahead switches the GCELL cost to
 * exp(-0.5 (cap_remaining - beta * pred)) with d_pred[z][y][x] the predicted
 * further demand (Z x Y x X f32, device; negative values count as 0) and
 * rebuilds the Fenwick trees from the current capacities; d_pred == NULL or
 * beta == 0 returns to the exact table cost of the reference. */
int gr_features(gr_ctx *ctx, float *d_feat, float scale, void *stream);
int gr_set_lookahead(gr_ctx *ctx, const float *d_pred, float beta, void *stream);

/* The whole lookahead route of the uploaded plan (gr_plan_set) from reset:
 * before every `every` batches the network (gr_cnn, 2Z inputs and Z outputs
 * over the Y x X grid) predicts from the current state (features x 1/16) the
 * further demand (output x 16), in GR_LA_EXCESS mode only its part beyond
 * the remaining capacity, and gr_set_lookahead(prediction, beta) applies
 * it. MST slots and patterns are copied to host memory; the plain cost is
 * restored at the end. beta == 0 routes plainly. */
#define GR_LA_DEMAND 0
#define GR_LA_EXCESS 1
typedef struct gr_cnn gr_cnn;
int gr_route_design_lookahead_host(gr_ctx *ctx, gr_cnn *cnn, int32_t every, float beta, int mode,
                                   int64_t *h_mst_edges, int32_t *h_mst_pat);
/* The same learned route into device buffers laid out as gr_route_plan's,
 * on `stream`, without waiting for it: the features, the network's forward
 * pass, the prediction transform, the Fenwick rebuilds and every batch are
 * device work, so with GR_PLAN_GRAPH the whole route is one captured CUDA
 * graph (kept and replayed while the plan, buffers, network and settings are
 * unchanged). Ends with the plain cost restored; gr_sync and gr_cnn_check
 * report device errors. (The host entry above calls this with
 * GR_PLAN_GRAPH.) */
int gr_route_plan_lookahead(gr_ctx *ctx, gr_cnn *cnn, int32_t every, float beta, int mode, int64_t *d_mst_edges,
                            int32_t *d_mst_pat, int flags, void *stream);

/* Launch shapes of the Boruvka size classes (results do not depend on them;
 * the autotuner in iitmglobalrouter_b200/tune.py picks them per GPU and Z). */
#define GR_TUNE_MST_MID_THREADS 0      /* threads per CTA, nets of 33..128 pins  */
#define GR_TUNE_MST_BIG_THREADS 1      /* threads per CTA, larger single-CTA nets */
#define GR_TUNE_MST_CLUSTER_THREADS 2  /* threads per CTA of a cluster            */
#define GR_TUNE_MST_CLUSTER_MIN_PINS 3 /* nets from this size use a cluster even
                                          when one CTA could hold them (0: never) */
#define GR_TUNE_LPAT_SPLIT 4           /* warps sharing a group of 32 pairs in the
                                          L-pattern kernel: 1, 2, 4 (0: by batch size) */
#define GR_TUNE_MST_QUEUE 5            /* 1: every net of 3+ pins of a batch in one
                                          persistent launch fed by a work queue
                                          (k_mst_queue); 0: one kernel per
                                          pin-count class on parallel streams */
#define GR_TUNE_PARAMS 6
int gr_tune_set(gr_ctx *ctx, int param, int value); /* threads: 64..1024, multiple of 32 */
/* (results do not depend on any of them; the L-pattern split only on latency) */
int gr_tune_get(gr_ctx *ctx, int param, int *value);

int gr_profile_enable(gr_ctx *ctx, int on);
int gr_profile_read(gr_ctx *ctx, double *ms, int64_t *launches, int reset);
const char *gr_kernel_name(int kind);

/* ------------------------------------------------------------ designs
 * Host-side design handling around the hot path (no GPU needed).
 * A gr_design holds the grid capacities and the multi-pin nets exactly as
 * the reference's reader leaves them (pins deduplicated and ascending, one
 * pin nets set aside), plus an optional routing plan. */
typedef struct gr_design gr_design;

/* seeded synthetic design; config 1..5 selects grid, capacities and the
 * pin-count mix (4 and 5 reuse the shapes of 2 and 3); n_nets > 0 overrides
 * the net count */
int gr_design_generate(gr_design **out, int config, uint64_t seed, int64_t n_nets);
int gr_design_generate_custom(gr_design **out, int X, int Y, int Z, int cap_lo, int cap_hi, double hot_frac,
                              int hot_lo, int hot_hi, int64_t n_nets, double tail_frac, int tail_hi,
                              double bbox_median, double bbox_sigma, int pin_layers, uint64_t seed);
/* .cap / .net text (reference read_data.hpp:94-169 and :220-300, 413-432,
 * 534-565); new_fmt selects the -new_fmt grammar */
int gr_design_read(gr_design **out, const char *cap_path, const char *net_path, int new_fmt);
/* writes the -new_fmt grammar */
int gr_design_write(const gr_design *d, const char *cap_path, const char *net_path);
int gr_design_free(gr_design *d);
int gr_design_dims(const gr_design *d, int *X, int *Y, int *Z, int32_t *n_nets, int64_t *n_pins,
                   int32_t *n_one_pin);
int gr_design_caps(const gr_design *d, int32_t *out);                  /* GR_ERR_NONINTEGER */
int gr_design_nets(const gr_design *d, int64_t *pin_ofs, int32_t *pins);
int gr_design_net_name(const gr_design *d, int32_t i, char *buf, int64_t cap);
/* -batch_part -num_xdim_parts k: the x-bucket greedy batcher
 * (NET_PART::part_nets / part_xdim, part_net/net_part.hpp:167-379); the
 * plan is kept in the design */
int gr_design_batch(gr_design *d, int num_xdim_parts, int32_t *n_batches, int64_t *n_ids);
/* the stored plan: sizes (either may be NULL) and contents (either may be
 * NULL; batch_ofs holds n_batches+1 entries) */
int gr_design_plan(const gr_design *d, int64_t *batch_ofs, int32_t *net_ids, int32_t *n_batches, int64_t *n_ids);
int gr_design_set_plan(gr_design *d, int32_t n_batches, const int64_t *batch_ofs, const int32_t *net_ids);
/* route text for the plan's MST slots (ROUTE_WRITER, writer_files/
 * writer_util.hpp:79-364); wl_vias (may be NULL) receives the merged
 * wirelength and via count */
#define GR_WRT_MERGE 0x1  /* -wrt_mrg     */
#define GR_WRT_RSEG 0x2   /* -rseg_fmt    */
#define GR_WRT_PPATCH 0x4 /* -oprd_ppatch */
int gr_design_write_routes(const gr_design *d, const char *path, const int64_t *mst, const int32_t *mst_pat,
                           int flags, int threads, int64_t *wl_vias);
/* out3 = {overflow, overflowed cells, total demand} for a demand grid */
int gr_design_eval(const gr_design *d, const int32_t *demand, double *out3);
/* The secondary measurement figure (no counterpart in the reference): the
 * bytes a direct Fenwick evaluation of every pattern of every pin pair
 * would gather, 4 B x sum over pairs and valid patterns of (2 per wire
 * segment + 1 per via cell), and the number of valid patterns: out2[0..1]. */
int gr_design_gather_bytes(const gr_design *d, int threads, double *out2);

/* ------------------------------------------------------------ congestion lookahead network
 * No counterpart in the reference: a stack of n_layers 3x3 convolutions
 * (hidden channels, ReLU between layers) mapping in_channels grids of H x W
 * (channel-major f32, [c][y][x]) to out_channels grids -- per routing layer
 * the demand still to come, predicted from the current demand and capacity.
 * BF16 tensor-core GEMMs with FP32 accumulation, FP32 master parameters
 * (per layer: weights [cout][cin][3][3], then biases), Adam updates on a
 * mean-squared-error loss. d_* are device pointers; calls synchronise.
 * (gr_cnn is declared above, beside gr_route_design_lookahead_host.) */
int gr_cnn_create(gr_cnn **out, int device, int in_channels, int out_channels, int hidden, int n_layers, int H,
                  int W, uint64_t seed);
int gr_cnn_destroy(gr_cnn *cnn);
int64_t gr_cnn_num_params(gr_cnn *cnn);
/* the CUDA device, input and output channels and grid of a network */
int gr_cnn_info(gr_cnn *cnn, int *device, int *in_channels, int *out_channels, int *H, int *W);
int gr_cnn_get_params(gr_cnn *cnn, float *h_out);
int gr_cnn_set_params(gr_cnn *cnn, const float *h_in);
int gr_cnn_forward(gr_cnn *cnn, const float *d_in, float *d_out);
/* the same forward pass enqueued on `stream` (NULL: the network's own
 * stream) without waiting for it, so that it can be captured in a CUDA graph
 * with other work; gr_cnn_check later waits for the network's stream and
 * reports a convolution that gave up waiting for its tensor-core results
 * (GR_ERR_DEVICE). The network's buffers are shared by every call. */
int gr_cnn_forward_async(gr_cnn *cnn, const float *d_in, float *d_out, void *stream);
int gr_cnn_check(gr_cnn *cnn);
/* loss and gradients (host, parameter layout) without an update */
int gr_cnn_grads(gr_cnn *cnn, const float *d_in, const float *d_target, float *h_grads, float *h_loss);
int gr_cnn_train_step(gr_cnn *cnn, const float *d_in, const float *d_target, float lr, float *h_loss);
/* C = A * B (row-major bf16 A: M x K, B: K x N; f32 C), k range split over `splits` blocks */
int gr_cnn_gemm_test(int M, int N, int K, const void *d_a, const void *d_b, float *d_c, int splits);

#ifdef __cplusplus
}
#endif
#endif
