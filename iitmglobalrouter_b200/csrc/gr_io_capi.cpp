// gr_io_capi.cpp -- C ABI of the host-side design functions (gr_design_*).
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
