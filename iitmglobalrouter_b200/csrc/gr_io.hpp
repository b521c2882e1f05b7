// gr_io.hpp -- host-side design handling around the hot path (C++20).
//
//   Design            grid capacities + nets, as the reference's reader leaves
//                     them (read_data.hpp:94-169, 220-300, 366-432, 525-565)
//   read_cap/read_net the reference's .cap / .net text grammar
//   write_cap/net     emits text in exactly that grammar
//   generate          seeded synthetic designs (grid, capacity, pin mix)
//   make_batches      the x-bucket greedy batcher of -batch_part
//                     (part_net/net_part.hpp:167-379)
//   write_routes      route text of the -wrt_mrg -rseg_fmt -oprd_ppatch writer
//                     (writer_files/writer_util.hpp:166-364)
//   evaluate          overflow / wirelength / via statistics
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace grio {

struct Pin {
    int z, x, y;
};

struct Design {
    int X = 0, Y = 0, Z = 0;
    double ulen = 1.0, uvia = 1.0;
    std::vector<double> layer_cost;       // Z per-layer values of the .cap header
    std::vector<long> hlen, vlen;         // X-1, Y-1 GCELL edge lengths
    std::vector<std::string> layer_name;  // Z
    std::vector<int> layer_dir, layer_minlen;
    std::vector<float> cap;  // X*Y*Z capacities, WIRE_ENC order
    // nets with >= 2 distinct pins, in file order (read_data.hpp:366-412)
    std::vector<std::string> names;
    std::vector<int64_t> pin_ofs;  // size n_nets + 1
    std::vector<int32_t> pins;     // WIRE_ENC, ascending within a net
    // one-pin nets (written by the route writer, never routed)
    std::vector<std::string> odeg_names;
    std::vector<Pin> odeg_pins;

    int64_t csize() const { return (int64_t)X * Y * Z; }
    int32_t n_nets() const { return (int32_t)names.size(); }
    int32_t enc(int z, int x, int y) const {
        return (z & 1) ? (int32_t)((int64_t)z * X * Y + (int64_t)x * Y + y)
                       : (int32_t)((int64_t)z * X * Y + (int64_t)y * X + x);
    }
    void dec(int32_t e, int &z, int &x, int &y) const {
        int64_t XY = (int64_t)X * Y;
        z = (int)(e / XY);
        int64_t r = e - z * XY;
        if (z & 1) {
            x = (int)(r / Y);
            y = (int)(r % Y);
        } else {
            y = (int)(r / X);
            x = (int)(r % X);
        }
    }
};

struct Plan {
    std::vector<int64_t> batch_ofs;  // n_batches + 1
    std::vector<int32_t> net_ids;
};

// 0 on success, negative GR_ERR_* on failure; *err gets a message
int read_cap(const std::string &path, bool new_fmt, Design &d, std::string *err);
int read_net(const std::string &path, bool new_fmt, Design &d, std::string *err);
int write_cap(const std::string &path, const Design &d);
int write_net(const std::string &path, const Design &d);

struct GenParams {
    int X, Y, Z;
    int cap_lo, cap_hi;          // capacity uniform in [lo, hi]
    double hot_frac;             // fraction of cells drawn from [hot_lo, hot_hi]
    int hot_lo, hot_hi;
    int64_t n_nets;
    double tail_frac;            // fraction of nets from the geometric tail
    int tail_lo, tail_hi;        // tail = tail_lo + Geometric(tail_p), clipped
    double tail_p;
    double bbox_median, bbox_sigma;  // log-normal bbox sides
    int pin_layers;              // pins on layers [0, pin_layers)
    int num_xdim_parts;
};
// the five standard workloads (1-based config numbers 1..5; 4/5 reuse 2/3)
GenParams standard_params(int config);
void generate(const GenParams &p, uint64_t seed, Design &d);

// integer capacities (GR_ERR_NONINTEGER if any value is fractional)
int integer_caps(const Design &d, std::vector<int32_t> &out);

// -batch_part -num_xdim_parts k
void make_batches(const Design &d, int num_xdim_parts, Plan &plan);

struct EvalStats {
    int64_t overflow_cells = 0;
    double overflow = 0.0;   // sum over z>=1 of max(0, demand - cap)
    int64_t demand = 0;      // total committed GCELL demand
    int64_t wirelength = 0;  // merged wire segment lengths (GCELLs)
    int64_t vias = 0;        // unit layer transitions
};
int write_routes(const std::string &path, const Design &d, const Plan &plan, const int64_t *mst,
                 const int32_t *mst_pat, bool merge, bool rseg_fmt, bool pin_patch, int threads,
                 EvalStats *stats);
void evaluate_demand(const Design &d, const int32_t *demand, EvalStats &st);

}  // namespace grio
