// gr_io_capi.cpp -- C ABI of the host-side design functions (gr_design_*).
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/iitmgr_b200.h"
#include "gr_io.hpp"

struct gr_design {
    grio::Design d;
    grio::Plan plan;
    std::string err;
};

extern "C" {

int gr_design_generate(gr_design **out, int config, uint64_t seed, int64_t n_nets) {
    if (!out || config < 1 || config > 5) return GR_ERR_ARG;
    grio::GenParams p = grio::standard_params(config);
    if (n_nets > 0) p.n_nets = n_nets;
    gr_design *g = new gr_design();
    grio::generate(p, seed, g->d);
    *out = g;
    return GR_OK;
}

int gr_design_generate_custom(gr_design **out, int X, int Y, int Z, int cap_lo, int cap_hi, double hot_frac,
                              int hot_lo, int hot_hi, int64_t n_nets, double tail_frac, int tail_hi,
                              double bbox_median, double bbox_sigma, int pin_layers, uint64_t seed) {
    if (!out || X < 1 || Y < 1 || Z < 1 || cap_hi < cap_lo || hot_hi < hot_lo || n_nets < 0 || pin_layers < 1 ||
        pin_layers > Z || bbox_median <= 0)
        return GR_ERR_ARG;
    grio::GenParams p{X, Y, Z, cap_lo, cap_hi, hot_frac, hot_lo, hot_hi, n_nets, tail_frac, 61,
                      tail_hi < 61 ? 61 : tail_hi, 0.03, bbox_median, bbox_sigma, pin_layers, 4};
    gr_design *g = new gr_design();
    grio::generate(p, seed, g->d);
    *out = g;
    return GR_OK;
}

int gr_design_read(gr_design **out, const char *cap_path, const char *net_path, int new_fmt) {
    if (!out || !cap_path || !net_path) return GR_ERR_ARG;
    gr_design *g = new gr_design();
    int rc = grio::read_cap(cap_path, new_fmt != 0, g->d, &g->err);
    if (!rc) rc = grio::read_net(net_path, new_fmt != 0, g->d, &g->err);
    if (rc) {
        delete g;
        *out = nullptr;
        return rc;
    }
    *out = g;
    return GR_OK;
}

int gr_design_write(const gr_design *g, const char *cap_path, const char *net_path) {
    if (!g || !cap_path || !net_path) return GR_ERR_ARG;
    int rc = grio::write_cap(cap_path, g->d);
    return rc ? rc : grio::write_net(net_path, g->d);
}

int gr_design_free(gr_design *g) {
    delete g;
    return GR_OK;
}

int gr_design_dims(const gr_design *g, int *X, int *Y, int *Z, int32_t *n_nets, int64_t *n_pins,
                   int32_t *n_one_pin) {
    if (!g) return GR_ERR_ARG;
    if (X) *X = g->d.X;
    if (Y) *Y = g->d.Y;
    if (Z) *Z = g->d.Z;
    if (n_nets) *n_nets = g->d.n_nets();
    if (n_pins) *n_pins = (int64_t)g->d.pins.size();
    if (n_one_pin) *n_one_pin = (int32_t)g->d.odeg_names.size();
    return GR_OK;
}

int gr_design_caps(const gr_design *g, int32_t *out) {
    if (!g || !out) return GR_ERR_ARG;
    std::vector<int32_t> c;
    int rc = grio::integer_caps(g->d, c);
    if (rc) return rc;
    memcpy(out, c.data(), sizeof(int32_t) * c.size());
    return GR_OK;
}

int gr_design_nets(const gr_design *g, int64_t *pin_ofs, int32_t *pins) {
    if (!g || !pin_ofs || !pins) return GR_ERR_ARG;
    memcpy(pin_ofs, g->d.pin_ofs.data(), sizeof(int64_t) * g->d.pin_ofs.size());
    memcpy(pins, g->d.pins.data(), sizeof(int32_t) * g->d.pins.size());
    return GR_OK;
}

int gr_design_net_name(const gr_design *g, int32_t i, char *buf, int64_t cap) {
    if (!g || i < 0 || i >= g->d.n_nets() || !buf || cap < 1) return GR_ERR_ARG;
    const std::string &s = g->d.names[i];
    size_t n = s.size() < (size_t)cap - 1 ? s.size() : (size_t)cap - 1;
    memcpy(buf, s.data(), n);
    buf[n] = '\0';
    return GR_OK;
}

int gr_design_batch(gr_design *g, int num_xdim_parts, int32_t *n_batches, int64_t *n_ids) {
    if (!g || num_xdim_parts < 1) return GR_ERR_ARG;
    grio::make_batches(g->d, num_xdim_parts, g->plan);
    if (n_batches) *n_batches = (int32_t)g->plan.batch_ofs.size() - 1;
    if (n_ids) *n_ids = (int64_t)g->plan.net_ids.size();
    return GR_OK;
}

int gr_design_plan(const gr_design *g, int64_t *batch_ofs, int32_t *net_ids, int32_t *n_batches, int64_t *n_ids) {
    if (!g) return GR_ERR_ARG;
    if (n_batches) *n_batches = g->plan.batch_ofs.empty() ? 0 : (int32_t)g->plan.batch_ofs.size() - 1;
    if (n_ids) *n_ids = (int64_t)g->plan.net_ids.size();
    if (batch_ofs && !g->plan.batch_ofs.empty())
        memcpy(batch_ofs, g->plan.batch_ofs.data(), sizeof(int64_t) * g->plan.batch_ofs.size());
    if (net_ids) memcpy(net_ids, g->plan.net_ids.data(), sizeof(int32_t) * g->plan.net_ids.size());
    return GR_OK;
}

int gr_design_set_plan(gr_design *g, int32_t n_batches, const int64_t *batch_ofs, const int32_t *net_ids) {
    if (!g || n_batches < 0 || !batch_ofs || (batch_ofs[n_batches] > 0 && !net_ids)) return GR_ERR_ARG;
    g->plan.batch_ofs.assign(batch_ofs, batch_ofs + n_batches + 1);
    g->plan.net_ids.assign(net_ids, net_ids + batch_ofs[n_batches]);
    return GR_OK;
}

int gr_design_write_routes(const gr_design *g, const char *path, const int64_t *mst, const int32_t *mst_pat,
                           int flags, int threads, int64_t *wl_vias) {
    if (!g || !path || !mst || !mst_pat) return GR_ERR_ARG;
    grio::EvalStats st;
    int rc = grio::write_routes(path, g->d, g->plan, mst, mst_pat, (flags & GR_WRT_MERGE) != 0,
                                (flags & GR_WRT_RSEG) != 0, (flags & GR_WRT_PPATCH) != 0, threads, &st);
    if (wl_vias) {
        wl_vias[0] = st.wirelength;
        wl_vias[1] = st.vias;
    }
    return rc;
}

int gr_design_gather_bytes(const gr_design *g, int threads, double *out2) {
    if (!g || !out2) return GR_ERR_ARG;
    const grio::Design &d = g->d;
    const int Z = d.Z, Z2 = (Z + 1) / 2, np = Z * Z2;
    if (Z < 2 || Z > 64) return GR_ERR_ARG;
    // units (2 per wire segment + 1 per via cell) summed over the valid
    // patterns of a pair, and the valid pattern count, by (z1, z2, kind):
    // kind 0 stacked, 1 x differs only, 2 y differs only, 3 both differ
    // (the validity and cell walk of the commit path's edge walk)
    std::vector<int64_t> units((size_t)Z * Z * 4, 0), npat((size_t)Z * Z * 4, 0);
    auto gap = [](int a, int b) { return a == b ? 0 : std::abs(a - b) - 1; };
    for (int z1 = 0; z1 < Z; z1++)
        for (int z2 = 0; z2 < Z; z2++)
            for (int kind = 0; kind < 4; kind++) {
                int64_t u = 0, n = 0;
                for (int cp = 0; cp < np; cp++) {
                    const int via1 = cp / Z2, v = cp % Z2, via2 = (via1 & 1) ? 2 * v : 2 * v + 1;
                    const bool bth = kind == 3;
                    if (via1 < 1 || via1 >= Z || (bth && via2 != 0 && via2 >= Z)) continue;
                    if (kind == 0) {  // the union of the layers between the pins and via1, via1 included
                        uint64_t m = 1ull << via1;
                        for (int i = std::min(z1, via1) + 1; i < std::max(z1, via1); i++) m |= 1ull << i;
                        for (int i = std::min(via1, z2) + 1; i < std::max(via1, z2); i++) m |= 1ull << i;
                        u += __builtin_popcountll(m);
                        n++;
                        continue;
                    }
                    // first wire on via1: even layers move x, odd ones y
                    const bool moves_x = !(via1 & 1);
                    bool xdone = kind == 2, ydone = kind == 1;
                    if (moves_x) xdone = true;
                    else ydone = true;
                    int64_t cu = gap(z1, via1) + 2;
                    int zl = via1;
                    if (bth && via2 != 0 && via1 != via2) {
                        cu += gap(via1, via2) + 2;
                        if (!(via2 & 1)) xdone = true;
                        else ydone = true;
                        zl = via2;
                    }
                    if (!(xdone && ydone)) continue;  // does not reach the second pin
                    if (kind == 1 && (via1 & 1)) continue;   // the wire moved y, which was already there
                    if (kind == 2 && !(via1 & 1)) continue;  // the wire moved x
                    cu += gap(zl, z2);
                    u += cu;
                    n++;
                }
                units[((size_t)z1 * Z + z2) * 4 + kind] = u;
                npat[((size_t)z1 * Z + z2) * 4 + kind] = n;
            }
    double total = 0.0, pats = 0.0;
    const int32_t nn = d.n_nets();
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : total, pats) num_threads(threads > 0 ? threads : 1)
    for (int32_t i = 0; i < nn; i++) {
        const int64_t o = d.pin_ofs[i], k = d.pin_ofs[i + 1] - o;
        for (int64_t a = 0; a < k; a++) {
            int za, xa, ya;
            d.dec(d.pins[o + a], za, xa, ya);
            for (int64_t b = a + 1; b < k; b++) {
                int zb, xb, yb;
                d.dec(d.pins[o + b], zb, xb, yb);
                const int kind = (xa == xb && ya == yb) ? 0 : (ya == yb ? 1 : (xa == xb ? 2 : 3));
                const size_t t = ((size_t)za * Z + zb) * 4 + kind;
                total += (double)units[t];
                pats += (double)npat[t];
            }
        }
    }
    out2[0] = 4.0 * total;
    out2[1] = pats;
    return GR_OK;
}

int gr_design_eval(const gr_design *g, const int32_t *demand, double *out3) {
    if (!g || !demand || !out3) return GR_ERR_ARG;
    grio::EvalStats st;
    grio::evaluate_demand(g->d, demand, st);
    out3[0] = st.overflow;
    out3[1] = (double)st.overflow_cells;
    out3[2] = (double)st.demand;
    return GR_OK;
}

}  // extern "C"
