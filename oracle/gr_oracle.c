/*
 * gr_oracle.c -- CPU oracle for the routing hot path (TEST INFRASTRUCTURE).
 * See gr_oracle.h for scope, provenance and the fixed tie-break rules.
 * Build: gcc -O2 -fPIC -fopenmp -ffp-contract=off (strict IEEE float order).
 */
#include "gr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GRO_LUT_MIN (-256)
#define GRO_LUT_MAX 1024

/* ---------------------------------------------------------------- encoding */

/* util.hpp:37-44: z*X*Y + (z odd ? x*Y + y : y*X + x) -- each routing track
 * (a row on even layers, a column on odd layers) is contiguous. */
int32_t gro_enc(const gro_grid *g, int z, int x, int y) {
    int64_t XY = (int64_t)g->X * g->Y;
    return (int32_t)((z & 1) ? z * XY + (int64_t)x * g->Y + y : z * XY + (int64_t)y * g->X + x);
}

/* util.hpp:53-60 */
void gro_dec(const gro_grid *g, int32_t e, int *z, int *x, int *y) {
    int64_t XY = (int64_t)g->X * g->Y;
    int zz = (int)(e / XY);
    int64_t r = e - zz * XY;
    *z = zz;
    if (zz & 1) {
        *x = (int)(r / g->Y);
        *y = (int)(r % g->Y);
    } else {
        *y = (int)(r / g->X);
        *x = (int)(r % g->X);
    }
}

/* ---------------------------------------------------------------- cost */

/* bit_util.hpp:13-15 computes expf(-cap * 0.5); capacities are integers, so
 * the oracle evaluates exp in double and rounds once to float. */
float gro_cost_of(int c) {
    if (c < GRO_LUT_MIN) c = GRO_LUT_MIN;
    if (c > GRO_LUT_MAX) c = GRO_LUT_MAX;
    return (float)exp(-0.5 * (double)c);
}

/* bit_util.hpp:16-18 with inc_val = 1 */
float gro_cost_inc(int c) {
    float a = gro_cost_of(c - 1);
    float b = gro_cost_of(c);
    return a - b;
}

/* ---------------------------------------------------------------- grid */

static int track_len(const gro_grid *g, int z) { return (z & 1) ? g->Y : g->X; }

/* Fenwick node i (1-based) of the track holding cell enc e sits at cell
 * (track base + i - 1): bit_util.hpp:24,30,43,50. */

/* bit_util.hpp:39-55 gpu_update_bit_cost: add val along the update path */
static void fen_add(gro_grid *g, int32_t e, float val) {
    int z, x, y;
    gro_dec(g, e, &z, &x, &y);
    int p = (z & 1) ? y : x;
    int L = track_len(g, z);
    int32_t base = e - p;
    for (int i = p + 1; i <= L; i += i & (-i)) g->fen[base + i - 1] += val;
}

gro_grid *gro_grid_new(int X, int Y, int Z, const int32_t *cap) {
    gro_grid *g = (gro_grid *)calloc(1, sizeof(gro_grid));
    if (!g) return NULL;
    g->X = X;
    g->Y = Y;
    g->Z = Z;
    g->csize = (int64_t)X * Y * Z;
    g->cap0 = (int32_t *)malloc(sizeof(int32_t) * g->csize);
    g->capr = (int32_t *)malloc(sizeof(int32_t) * g->csize);
    g->fen = (float *)malloc(sizeof(float) * g->csize);
    if (!g->cap0 || !g->capr || !g->fen) {
        gro_grid_free(g);
        return NULL;
    }
    memcpy(g->cap0, cap, sizeof(int32_t) * g->csize);
    gro_grid_reset(g);
    return g;
}

void gro_grid_free(gro_grid *g) {
    if (!g) return;
    free(g->cap0);
    free(g->capr);
    free(g->fen);
    free(g);
}

/* bit_util.hpp:56-74 (zero, then every cell atomically adds its cost along
 * its update path) with the adds applied in ascending cell order. */
void gro_grid_reset(gro_grid *g) {
    memcpy(g->capr, g->cap0, sizeof(int32_t) * g->csize);
    memset(g->fen, 0, sizeof(float) * g->csize);
    for (int64_t e = 0; e < g->csize; e++) fen_add(g, (int32_t)e, gro_cost_of(g->capr[e]));
}

/* bit_util.hpp:19-35: res accumulates nodes from index pos+1 downwards */
float gro_query(const gro_grid *g, int z, int x, int y) {
    float res = 0.0f;
    if (z & 1) {
        int i = y + 1;
        while (i > 0) {
            res += g->fen[gro_enc(g, z, x, i - 1)];
            i = i - (i & (-i));
        }
    } else {
        int i = x + 1;
        while (i > 0) {
            res += g->fen[gro_enc(g, z, i - 1, y)];
            i = i - (i & (-i));
        }
    }
    return res;
}

/* bit_util.hpp:36-38 */
static float range_q(const gro_grid *g, int z, int x1, int y1, int x2, int y2) {
    return gro_query(g, z, x2, y2) - gro_query(g, z, x1, y1);
}

/* ---------------------------------------------------------------- L-pattern */

/* bit_util.hpp:91-107 gpu_get_bit_wire_cost */
static void wire_cost(const gro_grid *g, float *c, int z1, int *x1, int *y1, int x2, int y2) {
    if (z1 & 1) {
        if (*y1 < y2) *c += range_q(g, z1, *x1, *y1 - 1, *x1, y2);
        else if (*y1 > y2) *c += range_q(g, z1, *x1, y2 - 1, *x1, *y1);
        *y1 = y2;
    } else {
        if (*x1 < x2) *c += range_q(g, z1, *x1 - 1, *y1, x2, *y1);
        else if (*x1 > x2) *c += range_q(g, z1, x2 - 1, *y1, *x1, *y1);
        *x1 = x2;
    }
}

/* bit_util.hpp:108-117 gpu_bit_get_via_cost: point costs of layers
 * [min(z1,z2), max(z1,z2)) at (x1,y1) */
static void via_cost(const gro_grid *g, float *c, int z1, int z2, int x1, int y1) {
    int zmin = z1 < z2 ? z1 : z2, zmax = z1 < z2 ? z2 : z1;
    for (int i = zmin; i < zmax; i++) {
        if (i & 1) *c += range_q(g, i, x1, y1 - 1, x1, y1);
        else *c += range_q(g, i, x1 - 1, y1, x1, y1);
    }
}

/* one thread of bit_util.hpp:134-180 */
int gro_pattern_cost(const gro_grid *g, int32_t enc_src, int32_t enc_dst, int cpat, float *cost) {
    int Z2 = (g->Z + 1) / 2;
    int z1, x1, y1, z2, x2, y2;
    gro_dec(g, enc_src, &z1, &x1, &y1);
    gro_dec(g, enc_dst, &z2, &x2, &y2);
    int via1 = cpat / Z2, v = cpat % Z2;
    if (via1 == 0) return 0;
    int zs = z1, xs = x1, ys = y1;
    float c = 0.0f;
    int bth_diff = (xs != x2 && ys != y2);
    if (zs != via1) {
        via_cost(g, &c, zs, via1, xs, ys);
        zs = via1;
    }
    if (zs) wire_cost(g, &c, zs, &xs, &ys, x2, y2);
    int via2 = (zs & 1) ? 2 * v : 2 * v + 1;
    if (bth_diff && via2 != 0) {
        if (via2 >= g->Z) return 0; /* odd Z: no such layer */
        if (zs != via2) {
            via_cost(g, &c, zs, via2, xs, ys);
            zs = via2;
            wire_cost(g, &c, zs, &xs, &ys, x2, y2);
        }
    }
    if (zs != z2) {
        via_cost(g, &c, zs, z2, xs, ys);
        zs = z2;
    }
    if (xs != x2 || ys != y2 || zs != z2) return 0;
    *cost = c;
    return 1;
}

void gro_lpattern_pair(const gro_grid *g, int32_t enc_src, int32_t enc_dst, float *cost, int16_t *pat) {
    int Z2 = (g->Z + 1) / 2, npat = g->Z * Z2;
    float best = INFINITY;
    int bp = -1, first = -1;
    for (int cpat = 0; cpat < npat; cpat++) {
        float c;
        if (!gro_pattern_cost(g, enc_src, enc_dst, cpat, &c)) continue;
        if (first < 0) first = cpat;
        if (c < best) {
            best = c;
            bp = cpat;
        }
    }
    if (bp < 0) {
        bp = first;
        best = INFINITY;
    }
    *cost = best;
    *pat = (int16_t)bp;
}

/* The same argmin, with the cheapest cost among the pair's other valid
 * patterns (+inf if none): a pair whose two values are equal is a tie, where
 * the reference's kernel may store any of the tied patterns
 * (bit_util.hpp:182-189). */
void gro_lpattern_top2(const gro_grid *g, const int32_t *pairs, int64_t n_pairs, float *cost, int16_t *pat,
                       float *cost2, int nthreads) {
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t i = 0; i < n_pairs; i++) {
        const int Z2 = (g->Z + 1) / 2, npat = g->Z * Z2;
        float best = INFINITY, second = INFINITY;
        int bp = -1, first = -1;
        for (int cpat = 0; cpat < npat; cpat++) {
            float c;
            if (!gro_pattern_cost(g, pairs[2 * i], pairs[2 * i + 1], cpat, &c)) continue;
            if (first < 0) first = cpat;
            if (c < best) {
                second = best;
                best = c;
                bp = cpat;
            } else if (c < second) {
                second = c;
            }
        }
        if (bp < 0) {
            bp = first;
            best = INFINITY;
        }
        cost[i] = best;
        pat[i] = (int16_t)bp;
        cost2[i] = second;
    }
}

void gro_lpattern(const gro_grid *g, const int32_t *pairs, int64_t n_pairs, float *cost, int16_t *pat,
                  int nthreads) {
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t i = 0; i < n_pairs; i++) gro_lpattern_pair(g, pairs[2 * i], pairs[2 * i + 1], cost + i, pat + i);
}

/* test_lpat.hpp:313-333 with NET_ID_ORDER_REV=1: for j, for k < j: (pin j, pin k) */
int64_t gro_batch_pairs(const int64_t *pin_ofs, const int32_t *pins, const int32_t *net_ids, int32_t n_nets,
                        int32_t *pairs) {
    int64_t id = 0;
    for (int32_t i = 0; i < n_nets; i++) {
        int32_t nid = net_ids[i];
        int64_t o = pin_ofs[nid];
        int n = (int)(pin_ofs[nid + 1] - o);
        for (int j = 0; j < n; j++)
            for (int k = 0; k < j; k++) {
                if (pairs) {
                    pairs[2 * id] = pins[o + j];
                    pairs[2 * id + 1] = pins[o + k];
                }
                id++;
            }
    }
    return id;
}

/* Pairs whose L patterns the reference evaluates with a second-via layer
 * v2 == Z, past the top layer: bit_util.hpp:157-164 computes v2 = via1 odd ?
 * 2v : 2v+1 with no v2 < DZ guard, so with odd Z every even via1 >= 2 and
 * v = ceil(Z/2)-1 reach v2 = Z whenever both x and y differ (bth_diff), and
 * the kernel then reads point and wire costs of layer Z out of bounds. The
 * oracle treats those patterns as invalid. out[0] = such pairs, out[1] =
 * such (pair, pattern) evaluations, over the nets listed. */
void gro_count_oob_pairs(const gro_grid *g, const int64_t *pin_ofs, const int32_t *pins, const int32_t *net_ids,
                         int32_t n_nets, int64_t out[2]) {
    const int Z2 = (g->Z + 1) / 2;
    int per_pair = 0;
    for (int via1 = 1; via1 < g->Z; via1++)
        for (int v = 0; v < Z2; v++) {
            const int via2 = (via1 & 1) ? 2 * v : 2 * v + 1;
            per_pair += via2 != 0 && via2 >= g->Z;
        }
    int64_t pairs = 0;
    for (int32_t i = 0; i < n_nets && per_pair > 0; i++) {
        const int64_t o = pin_ofs[net_ids[i]];
        const int n = (int)(pin_ofs[net_ids[i] + 1] - o);
        for (int j = 0; j < n; j++) {
            int zj, xj, yj;
            gro_dec(g, pins[o + j], &zj, &xj, &yj);
            for (int k = 0; k < j; k++) {
                int zk, xk, yk;
                gro_dec(g, pins[o + k], &zk, &xk, &yk);
                pairs += xj != xk && yj != yk;
            }
        }
    }
    out[0] = pairs;
    out[1] = pairs * per_pair;
}

/* ---------------------------------------------------------------- Boruvka */

/* order-preserving key of a float cost: ties on cost fall to the pair id */
static uint64_t cost_key(float w, int64_t e) {
    if (w == 0.0f) w = 0.0f; /* -0 and +0 compare equal in the reference */
    uint32_t u;
    memcpy(&u, &w, 4);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((uint64_t)u << 32) | (uint64_t)(uint32_t)e;
}

/* gmst_util.hpp:68-82 gdsu */
static int dsu_find(int *dsu, int v) {
    int r = v;
    while (dsu[r] != r) r = dsu[r];
    dsu[v] = r;
    return r;
}

/* decode local pair id e = j(j-1)/2 + k, k < j (gmst_util.hpp:192-194) */
static void pair_decode(int64_t e, int *j, int *k) {
    int64_t jj = (int64_t)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
    while (jj * (jj - 1) / 2 > e) jj--;
    while ((jj + 1) * jj / 2 <= e) jj++;
    *j = (int)jj;
    *k = (int)(e - jj * (jj - 1) / 2);
}

/* One net of gpu_brvsk_solve<tp> rounds (gmst_util.hpp:164-341) plus the
 * failed-net feedback loop (mst_util.hpp:289-314): rounds continue until the
 * net holds n-1 edges. Records (root, selected root) pairs as the reference
 * does (gmst_util.hpp:310-333). */
int gro_brvsk_net(int n, const float *w, int64_t local_id, int64_t *slots, float *dist) {
    int *dsu = (int *)malloc(sizeof(int) * n);
    int *sel = (int *)malloc(sizeof(int) * n);
    uint64_t *best = (uint64_t *)malloc(sizeof(uint64_t) * n);
    int *root = (int *)malloc(sizeof(int) * n);
    for (int v = 0; v < n; v++) dsu[v] = v;
    int nrec = 0, rounds = 0;
    float d = 0.0f;
    for (int v = 0; v < n; v++) slots[v] = -1;
    while (nrec < n - 1) {
        if (rounds >= 64) {
            rounds = -1;
            break;
        }
        rounds++;
        for (int v = 0; v < n; v++) {
            root[v] = dsu_find(dsu, v);
            best[v] = UINT64_MAX;
            sel[v] = -1;
        }
        /* get_gpu_brvsk_min_edge: cheapest crossing pair per root */
        int64_t e = 0;
        for (int j = 1; j < n; j++)
            for (int k = 0; k < j; k++, e++) {
                int r1 = root[j], r2 = root[k];
                if (r1 == r2) continue;
                uint64_t key = cost_key(w[e], e);
                if (key < best[r1]) best[r1] = key;
                if (key < best[r2]) best[r2] = key;
            }
        /* get_gpu_brvsk_min_node: the root on the other side */
        for (int v = 0; v < n; v++) {
            if (root[v] != v || best[v] == UINT64_MAX) continue;
            int j, k;
            pair_decode((int64_t)(best[v] & 0xffffffffu), &j, &k);
            sel[v] = (root[j] == v) ? root[k] : root[j];
        }
        /* get_gpu_brvsk_edges + get_gpu_brvsk_edges_conn, ascending roots */
        for (int v = 0; v < n; v++) {
            if (sel[v] < 0) continue;
            int a = dsu_find(dsu, v), b = dsu_find(dsu, sel[v]);
            if (a == b) continue;
            if (a < b) dsu[a] = b;
            else dsu[b] = a;
            int j, k;
            pair_decode((int64_t)(best[v] & 0xffffffffu), &j, &k);
            d += w[(int64_t)j * (j - 1) / 2 + k];
            slots[nrec++] = (local_id << 30) | ((int64_t)v << 15) | (int64_t)sel[v];
        }
    }
    if (nrec < n) slots[nrec] = -1;
    *dist = d;
    free(dsu);
    free(sel);
    free(best);
    free(root);
    return rounds;
}

int gro_brvsk_build(const int64_t *pin_ofs, const int32_t *net_ids, int32_t n_nets, const float *pair_cost,
                    int64_t *mst, float *dist, int nthreads) {
    int64_t *pofs = (int64_t *)malloc(sizeof(int64_t) * (n_nets + 1));
    int64_t *nofs = (int64_t *)malloc(sizeof(int64_t) * (n_nets + 1));
    pofs[0] = nofs[0] = 0;
    for (int32_t i = 0; i < n_nets; i++) {
        int64_t n = pin_ofs[net_ids[i] + 1] - pin_ofs[net_ids[i]];
        pofs[i + 1] = pofs[i] + n * (n - 1) / 2;
        nofs[i + 1] = nofs[i] + n;
    }
    int bad = 0;
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : bad)
    for (int32_t i = 0; i < n_nets; i++) {
        int n = (int)(nofs[i + 1] - nofs[i]);
        if (gro_brvsk_net(n, pair_cost + pofs[i], i, mst + nofs[i], dist + i) < 0) bad = 1;
    }
    free(pofs);
    free(nofs);
    return bad ? -1 : 0;
}

/* ---------------------------------------------------------------- commit */

typedef struct {
    gro_grid *g;
    uint8_t *mark;
    int32_t *list;
    int64_t nlist;
} mark_ctx;

static void mark_id(mark_ctx *m, int32_t e) {
    if (!m->mark[e]) {
        m->mark[e] = 1;
        m->list[m->nlist++] = e;
    }
}

static void mark_cell(mark_ctx *m, int z, int x, int y) { mark_id(m, gro_enc(m->g, z, x, y)); }

/* mst_bit_commit.hpp:36-67 gpu_hash_gcell: a layer change marks the
 * interior layers only; a wire marks every cell of its inclusive span */
static void walk_via(mark_ctx *m, int za, int zb, int x, int y) {
    int zmin = za < zb ? za : zb, zmax = za < zb ? zb : za;
    for (int i = zmin + 1; i < zmax; i++) mark_cell(m, i, x, y);
}
static void walk_wire(mark_ctx *m, int z, int *x, int *y, int x2, int y2) {
    if (z & 1) {
        int lo = *y < y2 ? *y : y2, hi = *y < y2 ? y2 : *y;
        for (int yy = lo; yy <= hi; yy++) mark_cell(m, z, *x, yy);
        *y = y2;
    } else {
        int lo = *x < x2 ? *x : x2, hi = *x < x2 ? x2 : *x;
        for (int xx = lo; xx <= hi; xx++) mark_cell(m, z, xx, *y);
        *x = x2;
    }
}

static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* MST_BIT_COMMIT::bit_commit_edges (mst_bit_commit.hpp:236-255): mark every
 * GCELL on the chosen pattern of each MST edge (gpu_commit_edge, :147-235),
 * then each marked cell loses one unit of capacity and its Fenwick path
 * gains cost(cap-1)-cost(cap) (gpu_upd_bit_cost_cube, bit_util.hpp:75-90). */
int gro_commit(gro_grid *g, const int64_t *pin_ofs, const int32_t *pins, const int32_t *net_ids, int32_t n_nets,
               const int64_t *mst, const int16_t *pair_pat, int32_t *mst_pat) {
    int Z2 = (g->Z + 1) / 2;
    mark_ctx m;
    m.g = g;
    m.mark = (uint8_t *)calloc((size_t)g->csize, 1);
    m.list = (int32_t *)malloc(sizeof(int32_t) * g->csize);
    m.nlist = 0;
    int err = 0;
    int64_t slot = 0, pofs = 0;
    for (int32_t i = 0; i < n_nets; i++) {
        int64_t o = pin_ofs[net_ids[i]];
        int n = (int)(pin_ofs[net_ids[i] + 1] - o);
        for (int s = 0; s < n; s++, slot++) {
            int64_t E = mst[slot];
            if (mst_pat) mst_pat[slot] = -1;
            if (E == -1) continue;
            /* mst_bit_commit.hpp:91-99 */
            int n1 = (int)(E & 0x7fff), n2 = (int)((E >> 15) & 0x7fff);
            if ((E >> 30) != i || n1 >= n || n2 >= n || n1 == n2) {
                err = -2;
                continue;
            }
            if (n1 < n2) {
                int t = n1;
                n1 = n2;
                n2 = t;
            }
            int64_t ed = pofs + (int64_t)n1 * (n1 - 1) / 2 + n2;
            int cpat = pair_pat[ed];
            if (mst_pat) mst_pat[slot] = cpat;
            int z1, x1, y1, z2, x2, y2;
            gro_dec(g, pins[o + n1], &z1, &x1, &y1);
            gro_dec(g, pins[o + n2], &z2, &x2, &y2);
            int via1 = cpat / Z2, v = cpat % Z2;
            if (cpat < 0 || via1 < 1 || via1 >= g->Z) {
                err = -3;
                continue;
            }
            int bth_diff = (x1 != x2 && y1 != y2);
            int via2 = ((via1 & 1) ? 2 * v : 2 * v + 1);
            if (bth_diff && via2 != 0 && via2 >= g->Z) {
                err = -3;
                continue;
            }
            /* mst_bit_commit.hpp:209-231 */
            int d = 0; /* interior cells of the first layer change */
            if (z1 != via1) {
                walk_via(&m, z1, via1, x1, y1);
                d = (z1 < via1 ? via1 - z1 : z1 - via1) - 1;
                z1 = via1;
            }
            if (z1) {
                /* The first wire's cell ids are contiguous from `first`. In
                 * gpu_commit_edge the threads of the first layer change's d
                 * interior cells reach this wire with a negative local index
                 * (-d .. -1), and this one call is not guarded by tid >= 0
                 * (mst_bit_commit.hpp:216, unlike :213, :223-225, :228), so
                 * gpu_hash_gcell (:49-66) also marks the d cells just below
                 * the wire's lower end: cell ids first-d .. first-1, wrapping
                 * into the previous track when that end is at coordinate 0. */
                int32_t first = (z1 & 1) ? gro_enc(g, z1, x1, y1 < y2 ? y1 : y2) : gro_enc(g, z1, x1 < x2 ? x1 : x2, y1);
                for (int k = 1; k <= d; k++) mark_id(&m, first - k);
                walk_wire(&m, z1, &x1, &y1, x2, y2);
            }
            if (bth_diff && via2 != 0) {
                if (z1 != via2) {
                    walk_via(&m, z1, via2, x1, y1);
                    z1 = via2;
                    walk_wire(&m, z1, &x1, &y1, x2, y2);
                }
            }
            if (z1 != z2) {
                walk_via(&m, z1, z2, x1, y1);
                z1 = z2;
            }
            if (x1 != x2 || y1 != y2) err = -3;
        }
        pofs += (int64_t)n * (n - 1) / 2;
    }
    qsort(m.list, (size_t)m.nlist, sizeof(int32_t), cmp_i32);
    for (int64_t t = 0; t < m.nlist; t++) {
        int32_t e = m.list[t];
        float val = gro_cost_inc(g->capr[e]);
        g->capr[e] -= 1;
        fen_add(g, e, val);
    }
    free(m.mark);
    free(m.list);
    return err;
}

/* ---------------------------------------------------------------- driver */

int gro_route_batch(gro_grid *g, const int64_t *pin_ofs, const int32_t *pins, const int32_t *net_ids,
                    int32_t n_nets, float *pair_cost, int16_t *pair_pat, int64_t *mst, int32_t *mst_pat,
                    float *dist, int nthreads) {
    int64_t np = gro_batch_pairs(pin_ofs, pins, net_ids, n_nets, NULL);
    int32_t *pairs = (int32_t *)malloc(sizeof(int32_t) * 2 * (np > 0 ? np : 1));
    float *pc = pair_cost ? pair_cost : (float *)malloc(sizeof(float) * (np > 0 ? np : 1));
    int16_t *pp = pair_pat ? pair_pat : (int16_t *)malloc(sizeof(int16_t) * (np > 0 ? np : 1));
    float *dd = dist ? dist : (float *)malloc(sizeof(float) * (n_nets > 0 ? n_nets : 1));
    gro_batch_pairs(pin_ofs, pins, net_ids, n_nets, pairs);
    gro_lpattern(g, pairs, np, pc, pp, nthreads);
    int rc = gro_brvsk_build(pin_ofs, net_ids, n_nets, pc, mst, dd, nthreads);
    if (rc == 0) rc = gro_commit(g, pin_ofs, pins, net_ids, n_nets, mst, pp, mst_pat);
    free(pairs);
    if (!pair_cost) free(pc);
    if (!pair_pat) free(pp);
    if (!dist) free(dd);
    return rc;
}

int gro_route_batches(gro_grid *g, const int64_t *pin_ofs, const int32_t *pins, const int32_t *net_ids,
                      const int64_t *batch_ofs, int32_t n_batches, int64_t *mst, int32_t *mst_pat,
                      int nthreads) {
    int64_t slot = 0;
    for (int32_t b = 0; b < n_batches; b++) {
        const int32_t *ids = net_ids + batch_ofs[b];
        int32_t nn = (int32_t)(batch_ofs[b + 1] - batch_ofs[b]);
        int rc = gro_route_batch(g, pin_ofs, pins, ids, nn, NULL, NULL, mst + slot, mst_pat ? mst_pat + slot : NULL,
                                 NULL, nthreads);
        if (rc) return rc;
        for (int32_t i = 0; i < nn; i++) slot += pin_ofs[ids[i] + 1] - pin_ofs[ids[i]];
    }
    return 0;
}
