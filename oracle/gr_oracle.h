/*
 * gr_oracle.h -- CPU oracle for the routing hot path (TEST INFRASTRUCTURE).
 *
 * This is a deterministic plain-C restatement of the reference router's
 * "-bit_pmodel" per-batch path (SammithKanur/iitmGlobalRouter):
 *   L-pattern costing  bit_util.hpp:13-191
 *   Boruvka RMST       gmst_util.hpp:68-82,164-341, mst_util.hpp:283-314
 *   BIT edge commit    mst_bit_commit.hpp:17-255, bit_util.hpp:39-90
 *
 * It exists only to check the CUDA implementation: only tests/, the smoke
 * entry point and the benchmark's cpu_baseline / reference legs may load it.
 * The product never links or calls it.
 *
 * Parity status: parity unpinned. The reference ships no golden vectors or
 * tests for this path, and it cannot be built in this image (it needs the
 * Boost.Geometry headers, an absent external library). The oracle is pinned
 * instead by hand-derived known-answer cases (tests/golden) whose expected
 * values follow from the reference source read line by line.
 *
 * Where the reference is racy or undefined the oracle fixes one outcome, in
 * every case one that some legal execution of the reference can produce:
 *   - L-pattern argmin ties: lowest pattern id wins (bit_util.hpp:182-189).
 *   - odd Z: a second-via layer v2 >= Z is an invalid pattern (the reference
 *     reads out of bounds there, bit_util.hpp:157-164).
 *   - no finite-cost valid pattern: lowest valid pattern id, cost +inf.
 *   - Boruvka: per-root minimum by (cost, pair id); candidates processed in
 *     ascending root order (gmst_util.hpp:250-262, 290-292).
 *   - Fenwick build and update: contributions applied to each node in
 *     ascending cell order (bit_util.hpp:39-55 atomics serialised that way).
 *   - GCELL cost: (float)exp(-0.5*c) rounded from double for integer c,
 *     instead of device expf (bit_util.hpp:13-15).
 */
#ifndef GR_ORACLE_H
#define GR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gro_grid {
    int X, Y, Z;
    int64_t csize;
    int32_t *cap0;  /* capacity as read, WIRE_ENC order               */
    int32_t *capr;  /* remaining capacity = cap0 - demand              */
    float *fen;     /* per-track Fenwick nodes, WIRE_ENC order         */
} gro_grid;

/* cell encoding, util.hpp:37-44 (WIRE_ENC) */
int32_t gro_enc(const gro_grid *g, int z, int x, int y);
void gro_dec(const gro_grid *g, int32_t e, int *z, int *x, int *y);

/* cost of one GCELL with remaining capacity c (bit_util.hpp:13-15) */
float gro_cost_of(int c);
/* increment added when demand grows by one (bit_util.hpp:16-18) */
float gro_cost_inc(int c);

gro_grid *gro_grid_new(int X, int Y, int Z, const int32_t *cap);
void gro_grid_free(gro_grid *g);
/* capr = cap0, Fenwick rebuilt (bit_util.hpp:56-74,192-200) */
void gro_grid_reset(gro_grid *g);

/* inclusive prefix query of one track, bit_util.hpp:19-35 */
float gro_query(const gro_grid *g, int z, int x, int y);

/* cost of one pattern; returns 1 if the pattern reaches dst */
int gro_pattern_cost(const gro_grid *g, int32_t enc_src, int32_t enc_dst, int cpat, float *cost);

/* per pair argmin over patterns, bit_util.hpp:119-191 */
void gro_lpattern_pair(const gro_grid *g, int32_t enc_src, int32_t enc_dst, float *cost, int16_t *pat);
void gro_lpattern(const gro_grid *g, const int32_t *pairs, int64_t n_pairs,
                  float *cost, int16_t *pat, int nthreads);

/* the argmin plus the cheapest cost among each pair's other valid patterns */
void gro_lpattern_top2(const gro_grid *g, const int32_t *pairs, int64_t n_pairs,
                       float *cost, int16_t *pat, float *cost2, int nthreads);

/* pair list of a batch in reference order, test_lpat.hpp:313-333 */
int64_t gro_batch_pairs(const int64_t *pin_ofs, const int32_t *pins,
                        const int32_t *net_ids, int32_t n_nets, int32_t *pairs);

/* pairs (out[0]) and pattern evaluations (out[1]) that the reference's
 * L-pattern kernel makes with a second-via layer v2 == Z (odd Z only;
 * bit_util.hpp:157-164 has no v2 < DZ guard) over the listed nets */
void gro_count_oob_pairs(const gro_grid *g, const int64_t *pin_ofs, const int32_t *pins,
                         const int32_t *net_ids, int32_t n_nets, int64_t out[2]);

/* Boruvka of one net of n pins over w[n(n-1)/2]; writes n slots (edges then
 * -1), returns number of rounds or -1 on failure */
int gro_brvsk_net(int n, const float *w, int64_t local_id, int64_t *slots, float *dist);

/* brvsk_build for a batch: mst slots are laid out net after net (n slots per
 * net), pair costs in batch pair order */
int gro_brvsk_build(const int64_t *pin_ofs, const int32_t *net_ids, int32_t n_nets,
                    const float *pair_cost, int64_t *mst, float *dist, int nthreads);

/* mst_bit_commit for a batch; returns 0 or a negative error code */
int gro_commit(gro_grid *g, const int64_t *pin_ofs, const int32_t *pins,
               const int32_t *net_ids, int32_t n_nets, const int64_t *mst,
               const int16_t *pair_pat, int32_t *mst_pat);

/* whole batch (lpattern -> brvsk_build -> mst_bit_commit). pair_cost and
 * pair_pat may be NULL (scratch is allocated); returns 0 or <0 */
int gro_route_batch(gro_grid *g, const int64_t *pin_ofs, const int32_t *pins,
                    const int32_t *net_ids, int32_t n_nets, float *pair_cost,
                    int16_t *pair_pat, int64_t *mst, int32_t *mst_pat,
                    float *dist, int nthreads);

/* route many batches in sequence: batch b = net_ids[batch_ofs[b] .. batch_ofs[b+1]) */
int gro_route_batches(gro_grid *g, const int64_t *pin_ofs, const int32_t *pins,
                      const int32_t *net_ids, const int64_t *batch_ofs, int32_t n_batches,
                      int64_t *mst, int32_t *mst_pat, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
