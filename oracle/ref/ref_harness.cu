// ref_harness.cu -- runs the reference router's own -bit_pmodel code on a
// design and records what every stage produced (TEST INFRASTRUCTURE ONLY).
//
// Built by oracle/ref/build_ref.py from the reference's sources where they
// lie (its headers are included, nothing is copied), for sm_100a, into
// oracle/_ref/ref_harness. The flow is the reference's main.cpp:60-93 with
// its three threads run one after the other:
//   READ_DATA::read_cap_file / read_net_file        (read_data.hpp:184, 534)
//   NET_PART::part_nets                             (part_net/net_part.hpp:236)
//   per batch, the -bit_pmodel body of TEST_LPAT::test_gpu_lpat
//     (l_pattern_files/test_lpat.hpp:231-455): pair list, then
//     BIT_UTIL_SPACE::get_gpu_lpat_dist<5>, then MST_BUILD::get_mst_tree<0>
//     (Boruvka and its commit, mst_files/mst_util.hpp:152-372)
//   ROUTE_WRITER::write_route                       (writer_files/writer.hpp:12)
// The harness adds only copies of what each stage left in memory, and the
// table of the reference's device cost function get_gpu_of_cost
// (bit_util.hpp:13-15) over the integer capacities -256..1024.
//
// Usage: ref_harness -cap F -net F -out DIR [-new_fmt] [-num_xdim_parts K]
//        [-gr_out F] [-wrt_mrg] [-rseg_fmt] [-oprd_ppatch] [-writer_threads T]
//        [-mst_cpu_threads T] [-fen_at b1,b2,...] [-time_only] [-no_route]
//        [-dump_plan] [-repeat N]
// DIR receives raw little-endian arrays and summary.json. -no_route stops
// after the batcher (any Z; the reference's L-pattern kernel itself runs only
// for Z = 9 or 10, and at Z = 9 it reads a layer past the grid, so routing is
// asked for at Z = 10 only). -time_only records nothing but the times;
// -dump_plan then still records the reader's and the batcher's results
// (capacities, nets, batches). -repeat N (with -time_only) routes every batch
// N times, each time from the initial cost state: capacities copied back
// from the reader's cube, the placement counter of the trees set to zero and
// the reference's own init_bit_data run again (bit_util.hpp:192-200); the
// route time of each pass goes to summary.json.
#include "common.h"
#include "read_data.hpp"
#include "./part_net/net_part.hpp"
#include "l_pattern_files/test_lpat.hpp"
#include "l_pattern_files/lpattern_util.hpp"
#include "mst_files/mst_common.h"
#include "writer_files/writer.hpp"

#include <sys/stat.h>

#include <cstdio>
#include <string>
#include <vector>

namespace RW = ROUTE_WRITER;
namespace RWC = ROUTE_WRITER_COMMON;

namespace {

std::string g_out;

template <class T>
void put(const std::string &name, const T *p, size_t n, bool append = false) {
    FILE *f = fopen((g_out + "/" + name).c_str(), append ? "ab" : "wb");
    if (!f) {
        fprintf(stderr, "ref_harness: cannot write %s\n", name.c_str());
        exit(2);
    }
    if (n) fwrite(p, sizeof(T), n, f);
    fclose(f);
}

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e));
        exit(3);
    }
}

// the reference's device cost function at integer capacities
__global__ void k_ref_cost_table(float *out, int lo, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        gcb_dt c = (gcb_dt)(lo + i);
        out[i] = BIT_UTIL_SPACE::get_gpu_of_cost(c);
    }
}

struct Opts {
    bool time_only = false, no_route = false, dump_plan = false;
    int repeat = 1;
};

void parse(int argc, char **argv, std::vector<int> &fen_at, Opts &o) {
    for (int i = 1; i < argc; i++) {
        std::string s = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) {
                fprintf(stderr, "ref_harness: %s needs a value\n", s.c_str());
                exit(1);
            }
            return argv[++i];
        };
        if (s == "-cap") CAP_FILE = next();
        else if (s == "-net") NET_FILE = next();
        else if (s == "-out") g_out = next();
        else if (s == "-gr_out") OUT_FILE_PATH = next();
        else if (s == "-new_fmt") NEW_FMT = true;
        else if (s == "-num_xdim_parts") NUM_XDIM_PARTS = std::stoi(next());
        else if (s == "-wrt_mrg") WRT_MRG = true;
        else if (s == "-rseg_fmt") RSEG_FMT = true;
        else if (s == "-oprd_ppatch") OPRD_PPATCH = true;
        else if (s == "-writer_threads") RWC::NUM_THREADS = std::stoi(next());
        else if (s == "-mst_cpu_threads") MSC::MST_THREADS = std::stoi(next());
        else if (s == "-time_only") o.time_only = true;
        else if (s == "-no_route") o.no_route = true;
        else if (s == "-dump_plan") o.dump_plan = true;
        else if (s == "-repeat") o.repeat = std::stoi(next());
        else if (s == "-fen_at") {
            std::string v = next();
            size_t p = 0;
            while (p < v.size()) {
                size_t q = v.find(',', p);
                if (q == std::string::npos) q = v.size();
                fen_at.push_back(std::stoi(v.substr(p, q - p)));
                p = q + 1;
            }
        } else {
            fprintf(stderr, "ref_harness: unknown flag %s\n", s.c_str());
            exit(1);
        }
    }
    if (CAP_FILE.empty() || NET_FILE.empty() || g_out.empty()) {
        fprintf(stderr, "ref_harness: -cap, -net and -out are required\n");
        exit(1);
    }
    if (o.repeat < 1 || (o.repeat > 1 && !o.time_only)) {
        fprintf(stderr, "ref_harness: -repeat needs N >= 1, and -time_only when N > 1\n");
        exit(1);
    }
}

}  // namespace

int main(int argc, char **argv) {
    std::vector<int> fen_at;
    Opts o;
    BIT_PMODEL = true;
    BATCH_PART = true;
    parse(argc, argv, fen_at, o);
    const bool time_only = o.time_only, no_route = o.no_route, plan = !o.time_only || o.dump_plan;
    mkdir(g_out.c_str(), 0755);
    if (OUT_FILE_PATH.empty()) OUT_FILE_PATH = g_out + "/routes.txt";
    // main.cpp:64-67: the route file is written through this logger
    gr_file_logger = spdlog::basic_logger_mt("gr_file_mt_logger", OUT_FILE_PATH, true);
    gr_file_logger->set_pattern("%v");

    auto t0 = std::chrono::steady_clock::now();
    READ_DATA::read_cap_file(CAP_FILE);
    READ_DATA::read_net_file(NET_FILE);
    auto t1 = std::chrono::steady_clock::now();
    const int64_t csize = (int64_t)X * Y * Z;

    if (plan) {
        // the reader's result: capacities as read, nets of two or more pins in
        // order with their pins as left by remove_redundant_pins, one-pin nets
        put("caps.f32", cube_data, csize);
        std::vector<int64_t> ofs(1, 0);
        std::vector<int32_t> pins;
        for (const net_t &n : nets) {
            for (const pin_t &p : n.pins) pins.push_back(UTIL::get_enc<WIRE_ENC>(p.pcd.z, p.pcd.x, p.pcd.y));
            ofs.push_back((int64_t)pins.size());
        }
        put("net_ofs.i64", ofs.data(), ofs.size());
        put("net_pins.i32", pins.data(), pins.size());
    }
    if (!time_only) {
        // names as the route writer prints them (writer_util.hpp:9-12 drops
        // the newlines and spaces the reader keeps around them), one per line
        auto clean = [](std::string s) {
            s.erase(std::remove(s.begin(), s.end(), '\n'), s.end());
            s.erase(std::remove(s.begin(), s.end(), ' '), s.end());
            return s;
        };
        std::string names;
        for (const net_t &n : nets) names += clean(n.net_name) + '\n';
        put("net_names.txt", names.data(), names.size());
        std::string onames;
        for (const net_t &n : one_deg_nets) onames += clean(n.net_name) + '\n';
        put("odeg_names.txt", onames.data(), onames.size());
        // the device cost function at integer capacities
        const int lo = -256, n = 1024 - lo + 1;
        float *d_tab = nullptr;
        check(cudaMalloc(&d_tab, sizeof(float) * n), "cudaMalloc");
        k_ref_cost_table<<<(n + 255) / 256, 256>>>(d_tab, lo, n);
        check(cudaDeviceSynchronize(), "cost table");
        std::vector<float> tab(n);
        check(cudaMemcpy(tab.data(), d_tab, sizeof(float) * n, cudaMemcpyDeviceToHost), "copy");
        cudaFree(d_tab);
        put("cost_table.f32", tab.data(), tab.size());
    }

    // batches (the producer thread of main.cpp:80, run to completion)
    NET_PART::part_nets();
    auto t2 = std::chrono::steady_clock::now();
    if (plan) {
        put("npart_ofst.i32", npart_ofst, PART_ID);
        put("npart_len.i32", npart_len, PART_ID);
        put("npart_ids.i32", npart_ids, (size_t)npart_ofst[PART_ID - 1] + npart_len[PART_ID - 1]);
    }
    if (no_route) {
        FILE *f = fopen((g_out + "/summary.json").c_str(), "w");
        if (f) {
            fprintf(f, "{\"X\": %d, \"Y\": %d, \"Z\": %d, \"nets\": %d, \"one_pin_nets\": %d, \"batches\": %d, "
                       "\"read_s\": %.6f, \"batch_s\": %.6f}\n",
                    (int)X, (int)Y, (int)Z, NUM_NETS, ODEG_NUM_NETS, PART_ID,
                    std::chrono::duration<double>(t1 - t0).count(), std::chrono::duration<double>(t2 - t1).count());
            fclose(f);
        }
        printf("ref_harness: %d nets, %d batches (no route)\n", NUM_NETS, PART_ID);
        return 0;
    }

    // the -bit_pmodel part of test_gpu_lpat's set-up (test_lpat.hpp:237-241)
    BULS::init_bit_data();
    check(cudaDeviceSynchronize(), "init_bit_data");
    auto t3 = std::chrono::steady_clock::now();

    std::vector<float> capr_before, capr_after, fen;
    std::vector<int32_t> marked;
    std::vector<int64_t> marked_ofs(1, 0);
    double route_s = 0.0;
    int64_t total_pairs = 0, total_nets = 0;
    std::vector<double> pass_s;
    for (int pass = 0; pass < o.repeat; pass++) {
        if (pass > 0) {
            // back to the initial cost state: capacities as read, the trees'
            // placement counter at zero (as part_nets leaves it,
            // net_part.hpp:43), the Fenwick cube rebuilt by the reference
            check(cudaMemcpy(d_cube_data_bit, cube_data, sizeof(float) * csize, cudaMemcpyHostToDevice), "capacities");
            MSC::NUM_NODES_OFST = 0;
            BULS::init_bit_data();
            check(cudaDeviceSynchronize(), "init_bit_data");
            route_s = 0.0;
            total_pairs = total_nets = 0;
        }
        for (int batch_id = 0; batch_id < PART_ID; batch_id++) {
            if (!time_only) {
                capr_before.resize(csize);
                check(cudaMemcpy(capr_before.data(), d_cube_data_bit, sizeof(float) * csize, cudaMemcpyDeviceToHost), "capr");
                for (int b : fen_at)
                    if (b == batch_id) {
                        fen.resize(csize);
                        check(cudaMemcpy(fen.data(), d_cost_data_bit, sizeof(float) * csize, cudaMemcpyDeviceToHost), "fen");
                        put("fen_b" + std::to_string(b) + ".f32", fen.data(), fen.size());
                        put("capr_b" + std::to_string(b) + ".f32", capr_before.data(), capr_before.size());
                    }
            }
            auto b0 = std::chrono::steady_clock::now();
            // test_lpat.hpp:288-377 with BIT_PMODEL and RANDOM_GEN == 0
            long num_prs;
            int num_nets = npart_len[batch_id], ofst = npart_ofst[batch_id];
            UTIL::get_num_pts_batch(num_prs, batch_id);
            LPC::hd_ptprs = (genc_dt *)malloc(sizeof(genc_dt) * num_prs * 2);
            rd_enc = (pt_prs *)malloc(sizeof(pt_prs) * num_prs);
            CUDA_MALLOC_1D(LPC::d_ptprs, num_prs * 2, genc_dt);
            CUDA_MALLOC_1D(LPC::d_lpat_res, num_prs, gcb_dt);
            CUDA_MALLOC_1D(LPC::d_lpat_pat, num_prs, lpat_dt);
            int pts_id = 0;
            for (int i = ofst; i < ofst + num_nets; i++) {
                int net_id = npart_ids[i];
                vector<pin_t> pins = nets[net_id].pins;
                for (int j = 0; j < (int)pins.size(); j++) {
                    coord_t ccd = pins[j].pcd;
                    genc_dt enc1 = UTIL::get_enc<CUBE_ENC>(ccd.z, ccd.x, ccd.y);
                    for (int k = 0; k < j; k++) {  // NET_ID_ORDER_REV == 1
                        coord_t ncd = pins[k].pcd;
                        genc_dt enc2 = UTIL::get_enc<CUBE_ENC>(ncd.z, ncd.x, ncd.y);
                        rd_enc[pts_id++] = {enc1 : enc1, enc2 : enc2};
                    }
                }
            }
            for (long i = 0; i < num_prs; i++) {
                LPC::hd_ptprs[2 * i] = rd_enc[i].enc1;
                LPC::hd_ptprs[2 * i + 1] = rd_enc[i].enc2;
            }
            CUDAMEMCPYHD_1D(LPC::d_ptprs, LPC::hd_ptprs, num_prs * 2, genc_dt);
            int num_pts_per_block = NUM_GPU_THREADS / Z1Z2, num_blocks = CEIL_DIV(num_prs, num_pts_per_block);
            if (num_pts_per_block != 5) {
                fprintf(stderr, "ref_harness: the reference's kernel needs 256 / (Z * ceil(Z/2)) == 5 (Z = 9 or 10)\n");
                return 4;
            }
            BULS::get_gpu_lpat_dist<5><<<num_blocks, NUM_GPU_THREADS>>>(LPC::d_lpat_pat, LPC::d_ptprs, LPC::d_lpat_res,
                                                                        num_prs);
            cudaDeviceSynchronize();
            std::vector<float> pc;
            std::vector<int16_t> pp;
            if (!time_only) {
                pc.resize(num_prs);
                pp.resize(num_prs);
                check(cudaMemcpy(pc.data(), LPC::d_lpat_res, sizeof(float) * num_prs, cudaMemcpyDeviceToHost), "costs");
                check(cudaMemcpy(pp.data(), LPC::d_lpat_pat, sizeof(int16_t) * num_prs, cudaMemcpyDeviceToHost), "pats");
            }
            const int slot0 = MSC::NUM_NODES_OFST;
            MSB::get_mst_tree<0>(batch_id, num_prs);
            check(cudaDeviceSynchronize(), "get_mst_tree");
            auto b1 = std::chrono::steady_clock::now();
            route_s += std::chrono::duration<double>(b1 - b0).count();
            total_pairs += num_prs;
            total_nets += num_nets;
            if (!time_only) {
                const bool app = batch_id > 0;
                put("pairs.i32", LPC::hd_ptprs, 2 * (size_t)num_prs, app);
                put("pair_cost.f32", pc.data(), pc.size(), app);
                put("pair_pat.i16", pp.data(), pp.size(), app);
                const int slots = MSC::NUM_NODES_OFST - slot0;
                put("mst.i64", MSC::net_mst_edges.data() + slot0, slots, app);
                put("mst_pat.i32", MSC::mst_lpat_pat.data() + slot0, slots, app);
                capr_after.resize(csize);
                check(cudaMemcpy(capr_after.data(), d_cube_data_bit, sizeof(float) * csize, cudaMemcpyDeviceToHost), "capr");
                for (int64_t e = 0; e < csize; e++)
                    if (capr_after[e] != capr_before[e]) marked.push_back((int32_t)e);
                marked_ofs.push_back((int64_t)marked.size());
            }
            free(rd_enc);
            free(LPC::hd_ptprs);
            cudaFree(LPC::d_ptprs);
            cudaFree(LPC::d_lpat_res);
            cudaFree(LPC::d_lpat_pat);
        }
        pass_s.push_back(route_s);
    }
    write_route_bsem.release();  // test_lpat.hpp:380
    auto t4 = std::chrono::steady_clock::now();

    if (!time_only) {
        put("marked.i32", marked.data(), marked.size());
        put("marked_ofs.i64", marked_ofs.data(), marked_ofs.size());
        capr_after.resize(csize);
        fen.resize(csize);
        check(cudaMemcpy(capr_after.data(), d_cube_data_bit, sizeof(float) * csize, cudaMemcpyDeviceToHost), "capr");
        check(cudaMemcpy(fen.data(), d_cost_data_bit, sizeof(float) * csize, cudaMemcpyDeviceToHost), "fen");
        put("final_capr.f32", capr_after.data(), capr_after.size());
        put("final_fen.f32", fen.data(), fen.size());
        RW::write_route();  // main.cpp:83 (the writer thread)
        gr_file_logger->flush();
    }
    auto t5 = std::chrono::steady_clock::now();
    auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    // the first pass's figures, then every pass's route time
    route_s = pass_s[0];
    std::string passes;
    for (double t : pass_s) passes += (passes.empty() ? "" : ", ") + std::to_string(t);
    FILE *f = fopen((g_out + "/summary.json").c_str(), "w");
    if (f) {
        fprintf(f,
                "{\"X\": %d, \"Y\": %d, \"Z\": %d, \"nets\": %d, \"one_pin_nets\": %d, \"batches\": %d, "
                "\"pairs\": %lld, \"routed_nets\": %lld, \"read_s\": %.6f, \"batch_s\": %.6f, \"fenwick_init_s\": %.6f, "
                "\"route_s\": %.6f, \"write_s\": %.6f, \"route_nets_per_s\": %.3f, \"pass_route_s\": [%s]}\n",
                (int)X, (int)Y, (int)Z, NUM_NETS, ODEG_NUM_NETS, PART_ID, (long long)total_pairs,
                (long long)total_nets, sec(t0, t1), sec(t1, t2), sec(t2, t3), route_s, sec(t4, t5),
                route_s > 0 ? total_nets / route_s : 0.0, passes.c_str());
        fclose(f);
    }
    printf("ref_harness: %d nets, %d batches, %lld pairs, route %.3f s (%.0f nets/s)\n", NUM_NETS, PART_ID,
           (long long)total_pairs, route_s, route_s > 0 ? total_nets / route_s : 0.0);
    return 0;
}
