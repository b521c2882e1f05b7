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
// Unknown flags are ignored (as the reference does). -rbt_part, -ord_part,
// -upd_ispd24_net_file and running without -bit_pmodel select reference modes
// this tool does not provide; it stops with a message.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "iitmgr_b200.h"

namespace {

struct Args {
    std::string cap, net, out, report, chip;
    bool new_fmt = false, bit_pmodel = false, batch_part = false, wrt_mrg = false, rseg = false, ppatch = false;
    bool graph = false, rbt = false, ord = false, upd24 = false;
    int parts = 4, writer_threads = 4, device = 0;
};

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
    }
    if (a.cap.empty() || a.net.empty() || a.out.empty()) {
        fprintf(stderr, "usage: route -cap F -net F -gr_out F [-new_fmt] -bit_pmodel -batch_part "
                        "[-num_xdim_parts k] [-wrt_mrg] [-rseg_fmt] [-oprd_ppatch] [-graph] [-report F]\n");
        return 2;
    }
    if (!a.bit_pmodel || a.rbt || a.ord || a.upd24) {
        fprintf(stderr, "route: only the -bit_pmodel cost model with -batch_part batching is provided\n");
        return 2;
    }
    if (a.parts < 1) a.parts = 1;

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
    if ((rc = gr_sync(ctx))) return fail("setup", rc);
    const double t3 = now();
    rc = gr_route_design_host(ctx, n_nets, pin_ofs.data(), pins.data(), n_batches, bofs.data(), ids.data(),
                              mst.data(), pat.data(), a.graph ? GR_PLAN_GRAPH : 0);
    if (rc) return fail("routing", rc);
    const double t4 = now();

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
    gr_destroy(ctx);
    gr_design_free(d);
    return 0;
}
