// route_main.cpp -- the `route` command line tool, built on the public C ABI.
//
// Flags follow the reference's main.cpp:16-61 (parse_args):
//   -cap F -net F -gr_out F      inputs and the route file
//   -new_fmt                     .cap/.net grammar of the -new_fmt reader
//   -bit_pmodel                  Fenwick cost model (the only model here)
//   -batch_part                  x-bucket greedy batches (the only batcher here)
//   -num_xdim_parts k            x buckets per batch (default 4)
//   -wrt_mrg -rseg_fmt -oprd_ppatch -writer_threads t   route writer options
//   -mst_cpu_threads t -chip_name s                     accepted, no effect
// plus:
//   -device d                    CUDA device (default 0)
//   -report F                    JSON report: timings, nets/s, overflow, WL, vias
//   -graph                       route the plan as one captured CUDA graph
//   -lookahead F.npy             route with the learned congestion lookahead:
//                                network parameters (float32 .npy); its
//                                settings come from F.json beside it when
//                                present (keys mode, beta, every, hidden,
//                                layers) and from these flags, which win:
//   -la_mode demand|excess  -la_beta b  -la_every k  -la_hidden h  -la_layers l
// Unknown flags are ignored (as the reference does). -rbt_part, -ord_part,
// -upd_ispd24_net_file and running without -bit_pmodel select reference modes
// this tool does not provide; it stops with a message.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "iitmgr_b200.h"

namespace {

struct Args {
    std::string cap, net, out, report, chip;
    bool new_fmt = false, bit_pmodel = false, batch_part = false, wrt_mrg = false, rseg = false, ppatch = false;
    bool graph = false, rbt = false, ord = false, upd24 = false;
    int parts = 4, writer_threads = 4, device = 0;
    // lookahead; empty / negative = from the sidecar JSON, else the default
    std::string la_path, la_mode;
    double la_beta = -1.0;
    int la_every = -1, la_hidden = -1, la_layers = -1;
};

std::string slurp(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return std::string();
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// A one-dimensional little-endian float32 .npy array (format versions 1-3).
bool read_npy_f32(const std::string &path, std::vector<float> &out) {
    const std::string b = slurp(path);
    if (b.size() < 10 || b.compare(0, 6, "\x93NUMPY") != 0) return false;
    const int major = (unsigned char)b[6];
    size_t hlen, h0;
    if (major == 1) {
        hlen = (unsigned char)b[8] | ((size_t)(unsigned char)b[9] << 8);
        h0 = 10;
    } else {
        if (b.size() < 12) return false;
        hlen = 0;
        for (int k = 0; k < 4; k++) hlen |= (size_t)(unsigned char)b[8 + k] << (8 * k);
        h0 = 12;
    }
    if (h0 + hlen > b.size()) return false;
    const std::string h = b.substr(h0, hlen);
    if (h.find("'descr': '<f4'") == std::string::npos || h.find("'fortran_order': False") == std::string::npos)
        return false;
    const size_t sp = h.find("'shape': (");
    if (sp == std::string::npos) return false;
    const size_t close = h.find(')', sp);
    if (close == std::string::npos) return false;
    const std::string dims = h.substr(sp + 10, close - sp - 10);  // "n," for one dimension
    if (dims.empty() || dims.back() != ',' || dims.find(',') != dims.size() - 1) return false;
    const long long n = atoll(dims.c_str());
    if (n < 0) return false;
    if (h0 + hlen + (size_t)n * 4 != b.size()) return false;
    out.resize((size_t)n);
    memcpy(out.data(), b.data() + h0 + hlen, (size_t)n * 4);
    return true;
}

// The value of the first "key": in a flat settings file (numbers or strings).
std::string json_value(const std::string &doc, const char *key) {
    const std::string k = std::string("\"") + key + "\":";
    size_t p = doc.find(k);
    if (p == std::string::npos) return std::string();
    p += k.size();
    while (p < doc.size() && (doc[p] == ' ' || doc[p] == '\n')) p++;
    if (p < doc.size() && doc[p] == '"') {
        const size_t e = doc.find('"', p + 1);
        return e == std::string::npos ? std::string() : doc.substr(p + 1, e - p - 1);
    }
    size_t e = p;
    while (e < doc.size() && (isdigit((unsigned char)doc[e]) || doc[e] == '.' || doc[e] == '-' || doc[e] == 'e' ||
                              doc[e] == 'E' || doc[e] == '+'))
        e++;
    return doc.substr(p, e - p);
}

double now() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int fail(const char *what, int rc) {
    fprintf(stderr, "route: %s: %s (%d)\n", what, gr_error_string(rc), rc);
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    Args a;
    for (int i = 1; i < argc; i++) {
        const std::string s = argv[i];
        auto val = [&](std::string &dst) {
            if (i + 1 < argc) dst = argv[++i];
        };
        auto ival = [&](int &dst) {
            if (i + 1 < argc) dst = atoi(argv[++i]);
        };
        if (s == "-cap") val(a.cap);
        else if (s == "-net") val(a.net);
        else if (s == "-gr_out") val(a.out);
        else if (s == "-chip_name") val(a.chip);
        else if (s == "-report") val(a.report);
        else if (s == "-new_fmt") a.new_fmt = true;
        else if (s == "-bit_pmodel") a.bit_pmodel = true;
        else if (s == "-batch_part") a.batch_part = true;
        else if (s == "-rbt_part") a.rbt = true;
        else if (s == "-ord_part") a.ord = true;
        else if (s == "-num_xdim_parts") ival(a.parts);
        else if (s == "-writer_threads") ival(a.writer_threads);
        else if (s == "-mst_cpu_threads") {
            int t;
            ival(t);
        } else if (s == "-wrt_mrg") a.wrt_mrg = true;
        else if (s == "-rseg_fmt") a.rseg = true;
        else if (s == "-oprd_ppatch") a.ppatch = true;
        else if (s == "-upd_ispd24_net_file") a.upd24 = true;
        else if (s == "-ispd24_new_nf_path") {
            std::string t;
            val(t);
        } else if (s == "-device") ival(a.device);
        else if (s == "-graph") a.graph = true;
        else if (s == "-lookahead") val(a.la_path);
        else if (s == "-la_mode") val(a.la_mode);
        else if (s == "-la_beta") {
            if (i + 1 < argc) a.la_beta = atof(argv[++i]);
        } else if (s == "-la_every") ival(a.la_every);
        else if (s == "-la_hidden") ival(a.la_hidden);
        else if (s == "-la_layers") ival(a.la_layers);
    }
    if (a.cap.empty() || a.net.empty() || a.out.empty()) {
        fprintf(stderr, "usage: route -cap F -net F -gr_out F [-new_fmt] -bit_pmodel -batch_part "
                        "[-num_xdim_parts k] [-wrt_mrg] [-rseg_fmt] [-oprd_ppatch] [-graph] [-report F] "
                        "[-lookahead F.npy [-la_mode demand|excess] [-la_beta b] [-la_every k] [-la_hidden h] "
                        "[-la_layers l]]\n");
        return 2;
    }
    if (!a.bit_pmodel || a.rbt || a.ord || a.upd24) {
        fprintf(stderr, "route: only the -bit_pmodel cost model with -batch_part batching is provided\n");
        return 2;
    }
    if (a.parts < 1) a.parts = 1;

    std::vector<float> la_params;
    if (!a.la_path.empty()) {
        if (!read_npy_f32(a.la_path, la_params)) {
            fprintf(stderr, "route: %s is not a one-dimensional float32 .npy file\n", a.la_path.c_str());
            return 2;
        }
        std::string side = a.la_path;
        if (side.size() > 4 && side.compare(side.size() - 4, 4, ".npy") == 0) side.resize(side.size() - 4);
        const std::string js = slurp(side + ".json");
        auto num = [&](const char *key, double dflt) {
            const std::string v = json_value(js, key);
            return v.empty() ? dflt : atof(v.c_str());
        };
        if (a.la_mode.empty()) a.la_mode = json_value(js, "mode");
        if (a.la_mode.empty()) a.la_mode = "demand";
        if (a.la_beta < 0) a.la_beta = num("beta", 0.5);
        if (a.la_every < 0) a.la_every = (int)num("every", 16);
        if (a.la_hidden < 0) a.la_hidden = (int)num("hidden", 32);
        if (a.la_layers < 0) a.la_layers = (int)num("layers", 4);
        if ((a.la_mode != "demand" && a.la_mode != "excess") || a.la_every < 1 || a.la_hidden < 1 ||
            a.la_layers < 2) {
            fprintf(stderr, "route: bad lookahead settings\n");
            return 2;
        }
    }

    const double t0 = now();
    gr_design *d = nullptr;
    int rc = gr_design_read(&d, a.cap.c_str(), a.net.c_str(), a.new_fmt ? 1 : 0);
    if (rc) return fail("reading the design", rc);
    int X, Y, Z;
    int32_t n_nets, n_one;
    int64_t n_pins;
    gr_design_dims(d, &X, &Y, &Z, &n_nets, &n_pins, &n_one);
    std::vector<int32_t> cap((size_t)X * Y * Z);
    if ((rc = gr_design_caps(d, cap.data()))) return fail("capacities", rc);
    std::vector<int64_t> pin_ofs(n_nets + 1);
    std::vector<int32_t> pins(n_pins > 0 ? n_pins : 1);
    gr_design_nets(d, pin_ofs.data(), pins.data());
    const double t1 = now();

    int32_t n_batches;
    int64_t n_ids;
    gr_design_batch(d, a.parts, &n_batches, &n_ids);
    std::vector<int64_t> bofs(n_batches + 1);
    std::vector<int32_t> ids(n_ids > 0 ? n_ids : 1);
    gr_design_plan(d, bofs.data(), ids.data(), nullptr, nullptr);
    const double t2 = now();

    gr_ctx *ctx = nullptr;
    if ((rc = gr_create(&ctx, a.device, X, Y, Z, cap.data()))) return fail("creating the context", rc);
    if ((rc = gr_set_nets(ctx, n_nets, pin_ofs.data(), pins.data()))) return fail("uploading nets", rc);
    if ((rc = gr_plan_set(ctx, n_batches, bofs.data(), ids.data()))) return fail("uploading the plan", rc);
    const int64_t slots = gr_plan_slots(ctx);
    std::vector<int64_t> mst(slots > 0 ? slots : 1);
    std::vector<int32_t> pat(slots > 0 ? slots : 1);
    gr_cnn *cnn = nullptr;
    if (!a.la_path.empty()) {
        if ((rc = gr_cnn_create(&cnn, a.device, 2 * Z, Z, a.la_hidden, a.la_layers, Y, X, 1)))
            return fail("creating the lookahead network", rc);
        if (gr_cnn_num_params(cnn) != (int64_t)la_params.size()) {
            fprintf(stderr, "route: %s holds %zu parameters, a %d-layer network of %d channels on Z=%d needs %lld\n",
                    a.la_path.c_str(), la_params.size(), a.la_layers, a.la_hidden, Z,
                    (long long)gr_cnn_num_params(cnn));
            return 2;
        }
        if ((rc = gr_cnn_set_params(cnn, la_params.data()))) return fail("loading the lookahead network", rc);
    }
    if ((rc = gr_sync(ctx))) return fail("setup", rc);
    const double t3 = now();
    if (cnn)
        rc = gr_route_design_lookahead_host(ctx, cnn, a.la_every, (float)a.la_beta,
                                            a.la_mode == "excess" ? GR_LA_EXCESS : GR_LA_DEMAND, mst.data(),
                                            pat.data());
    else
        rc = gr_route_design_host(ctx, n_nets, pin_ofs.data(), pins.data(), n_batches, bofs.data(), ids.data(),
                                  mst.data(), pat.data(), a.graph ? GR_PLAN_GRAPH : 0);
    if (rc) return fail("routing", rc);
    const double t4 = now();
    if (cnn) printf("route: lookahead %s, beta %g, every %d batches\n", a.la_mode.c_str(), a.la_beta, a.la_every);

    int64_t wv[2] = {0, 0};
    const int flags = (a.wrt_mrg ? GR_WRT_MERGE : 0) | (a.rseg ? GR_WRT_RSEG : 0) | (a.ppatch ? GR_WRT_PPATCH : 0);
    if ((rc = gr_design_write_routes(d, a.out.c_str(), mst.data(), pat.data(), flags, a.writer_threads, wv)))
        return fail("writing routes", rc);
    const double t5 = now();

    std::vector<int32_t> demand((size_t)X * Y * Z);
    gr_get_demand(ctx, demand.data());
    double ev[3];
    gr_design_eval(d, demand.data(), ev);
    printf("route: %d nets (%lld pins, %d one-pin) in %d batches; route %.3f s = %.0f nets/s\n", n_nets,
           (long long)n_pins, n_one, n_batches, t4 - t3, n_nets / (t4 - t3));
    printf("route: overflow %.0f (%lld cells), demand %.0f, wirelength %lld, vias %lld\n", ev[0],
           (long long)ev[1], ev[2], (long long)wv[0], (long long)wv[1]);
    printf("route: read %.3f s, batch %.3f s, setup %.3f s, write %.3f s\n", t1 - t0, t2 - t1, t3 - t2, t5 - t4);
    if (!a.report.empty()) {
        FILE *f = fopen(a.report.c_str(), "w");
        if (f) {
            fprintf(f,
                    "{\"nets\": %d, \"pins\": %lld, \"one_pin_nets\": %d, \"batches\": %d, \"read_s\": %.6f, "
                    "\"batch_s\": %.6f, \"setup_s\": %.6f, \"route_s\": %.6f, \"write_s\": %.6f, "
                    "\"nets_per_s\": %.1f, \"overflow\": %.1f, \"overflow_cells\": %lld, \"demand\": %.0f, "
                    "\"wirelength\": %lld, \"vias\": %lld, \"launches\": %lld}\n",
                    n_nets, (long long)n_pins, n_one, n_batches, t1 - t0, t2 - t1, t3 - t2, t4 - t3, t5 - t4,
                    n_nets / (t4 - t3), ev[0], (long long)ev[1], ev[2], (long long)wv[0], (long long)wv[1],
                    (long long)gr_launch_count(ctx));
            fclose(f);
        }
    }
    if (cnn) gr_cnn_destroy(cnn);
    gr_destroy(ctx);
    gr_design_free(d);
    return 0;
}
