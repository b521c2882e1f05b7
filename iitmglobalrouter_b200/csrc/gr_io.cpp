// gr_io.cpp -- design I/O, synthetic designs, batching and route writing.
// See gr_io.hpp. Reference citations are files of SammithKanur/iitmGlobalRouter.
#include "gr_io.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <thread>

#include "../../include/iitmgr_b200.h"

namespace grio {

// ------------------------------------------------------------------ text scan
namespace {

struct Buf {
    std::vector<char> b;
    size_t n = 0;
    size_t at = 0;
    char c(size_t i) const { return i < n ? b[i] : '\0'; }
};

bool load(const std::string &path, Buf &buf) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.b.assign((size_t)sz + 1, '\0');
    size_t got = sz > 0 ? fread(buf.b.data(), 1, (size_t)sz, f) : 0;
    fclose(f);
    buf.n = got;
    buf.at = 0;
    return true;
}

bool isdig(char ch) { return ch >= '0' && ch <= '9'; }

// read_data.hpp:17-23 get_long: skip non-digits, read digits
bool get_long(Buf &s, long &v) {
    v = 0;
    while (s.at < s.n && !isdig(s.c(s.at))) s.at++;
    if (s.at >= s.n) return false;
    while (isdig(s.c(s.at))) v = v * 10 + (s.c(s.at++) - '0');
    return true;
}

// read_data.hpp:41-67 get_float (FP32 accumulation) and :68-93 get_double
// (same steps; the reference's gcb_dt is float for both)
bool get_real(Buf &s, float &val) {
    val = 0.0f;
    while (s.at < s.n && s.c(s.at) != '-' && !isdig(s.c(s.at))) s.at++;
    if (s.at >= s.n) return false;
    bool neg = false;
    if (s.c(s.at) == '-') {
        neg = true;
        s.at++;
    }
    while (isdig(s.c(s.at))) val = val * 10.0f + (float)(s.c(s.at++) - '0');
    if (s.c(s.at) == '.') {
        float mul = 0.1f;
        s.at++;
        while (isdig(s.c(s.at))) {
            val = val + (float)(s.c(s.at++) - '0') * mul;
            mul *= 0.1f;
        }
    }
    if (s.c(s.at) == 'e') {
        s.at++;
        bool mneg = false;
        int pw = 0;
        if (s.c(s.at) == '-') {
            mneg = true;
            s.at++;
        }
        if (s.c(s.at) == '+') s.at++;
        while (isdig(s.c(s.at))) pw = pw * 10 + (s.c(s.at++) - '0');
        for (int i = 0; i < pw; i++) val = mneg ? (float)(val * (1.0) / (10.0)) : (float)(val * 10.0);
    }
    val = neg ? -val : val;
    return true;
}

// read_data.hpp:31-40 get_string
std::string get_string(Buf &s) {
    while (s.at < s.n && (s.c(s.at) == ' ' || s.c(s.at) == '\n' || s.c(s.at) == ',')) s.at++;
    std::string r;
    while (s.at < s.n && s.c(s.at) != ' ' && s.c(s.at) != '\n' && s.c(s.at) != ',') r += s.c(s.at++);
    return r;
}

std::string strip_name(const std::string &s) {
    std::string r;
    for (char ch : s)
        if (ch != '\n' && ch != ' ' && ch != '\r') r += ch;
    return r;
}

}  // namespace

// read_data.hpp:94-169,184-195: "Z X Y", ULEN, UVIA, Z layer values (+4 more
// with -new_fmt), X-1 and Y-1 edge lengths, then per layer: name, direction,
// min length and Y rows of X capacities (row i holds y = i).
int read_cap(const std::string &path, bool new_fmt, Design &d, std::string *err) {
    Buf s;
    if (!load(path, s)) {
        if (err) *err = "cannot open " + path;
        return GR_ERR_IO;
    }
    long Z, X, Y;
    if (!get_long(s, Z) || !get_long(s, X) || !get_long(s, Y) || Z < 1 || X < 1 || Y < 1) {
        if (err) *err = "bad grid header";
        return GR_ERR_PARSE;
    }
    d.X = (int)X;
    d.Y = (int)Y;
    d.Z = (int)Z;
    float v;
    if (!get_real(s, v)) return GR_ERR_PARSE;
    d.ulen = v;
    if (!get_real(s, v)) return GR_ERR_PARSE;
    d.uvia = v;
    d.layer_cost.assign(Z, 0.0);
    for (long i = 0; i < Z; i++) {
        if (!get_real(s, v)) return GR_ERR_PARSE;
        d.layer_cost[i] = v;
    }
    if (new_fmt)
        for (int i = 0; i < 4; i++)
            if (!get_real(s, v)) return GR_ERR_PARSE;
    d.hlen.assign(X > 1 ? X - 1 : 0, 0);
    d.vlen.assign(Y > 1 ? Y - 1 : 0, 0);
    for (auto &h : d.hlen)
        if (!get_long(s, h)) return GR_ERR_PARSE;
    for (auto &h : d.vlen)
        if (!get_long(s, h)) return GR_ERR_PARSE;
    d.cap.assign((size_t)X * Y * Z, 0.0f);
    d.layer_name.assign(Z, "");
    d.layer_dir.assign(Z, 0);
    d.layer_minlen.assign(Z, 0);
    for (int z = 0; z < Z; z++) {
        d.layer_name[z] = get_string(s);
        long dir, ml;
        if (!get_long(s, dir) || !get_long(s, ml)) {
            if (err) *err = "bad layer header";
            return GR_ERR_PARSE;
        }
        d.layer_dir[z] = (int)dir;
        d.layer_minlen[z] = (int)ml;
        for (int i = 0; i < Y; i++)
            for (int j = 0; j < X; j++) {
                if (!get_real(s, v)) {
                    if (err) *err = "capacity grid truncated";
                    return GR_ERR_PARSE;
                }
                d.cap[d.enc(z, j, i)] = v;
            }
    }
    return GR_OK;
}

namespace {

// read_data.hpp:254-277: digits up to the delimiter, other characters dropped
bool read_cd(const Buf &s, size_t &bid, char delim, int &out) {
    long v = 0;
    bool any = false;
    while (bid < s.n && s.c(bid) != delim) {
        if (isdig(s.c(bid))) {
            v = v * 10 + (s.c(bid) - '0');
            any = true;
        }
        bid++;
    }
    bid++;
    out = (int)v;
    return any;
}

}  // namespace

// read_data.hpp:220-300,413-432,525-565: nets are the depth-0 "( ... )"
// groups; a net's name is the text between the previous group and its "(".
// -new_fmt pins: skip two commas, then z, x (to ',') and y (to ')').
// Otherwise (ISPD24) pins are "(z, x, y)" groups. Pins are deduplicated and
// ordered by cell id; nets left with one pin are set aside.
int read_net(const std::string &path, bool new_fmt, Design &d, std::string *err) {
    if (d.X <= 0) {
        if (err) *err = "read the .cap file first";
        return GR_ERR_STATE;
    }
    Buf s;
    if (!load(path, s)) {
        if (err) *err = "cannot open " + path;
        return GR_ERR_IO;
    }
    std::vector<std::pair<size_t, size_t>> spans;  // '(' and ')' positions
    int depth = 0;
    for (size_t i = 0; i < s.n; i++) {
        char ch = s.b[i];
        if (ch == '(') {
            if (depth == 0) spans.push_back({i, (size_t)-1});
            depth++;
        } else if (ch == ')') {
            depth--;
            if (depth == 0 && !spans.empty()) spans.back().second = i;
        }
    }
    if (!spans.empty() && spans.back().second == (size_t)-1) {
        if (err) *err = "unterminated net";
        return GR_ERR_PARSE;
    }
    const int64_t n_all = (int64_t)spans.size();
    std::vector<std::string> names(n_all);
    std::vector<std::vector<int32_t>> pins(n_all);
    std::vector<Pin> first_pin(n_all);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t i = 0; i < n_all; i++) {
        size_t st = i == 0 ? 0 : spans[i - 1].second + 1;
        size_t op = spans[i].first, ed = spans[i].second;
        names[i] = strip_name(std::string(s.b.data() + st, s.b.data() + op));
        std::map<int32_t, Pin> mp;
        size_t bid = st;
        while (true) {
            Pin p{};
            if (new_fmt) {
                for (int c = 0; c < 2; c++) {  // read_comma twice
                    while (bid < ed && s.b[bid] != ',') bid++;
                    bid++;
                }
                if (bid >= ed) break;
                read_cd(s, bid, ',', p.z);
                read_cd(s, bid, ',', p.x);
                read_cd(s, bid, ')', p.y);
            } else {  // read_ispd24_net_single (read_data.hpp:332-354)
                while (bid < ed && s.b[bid] != '(') bid++;
                bid++;
                if (bid + 5 >= ed) break;
                read_cd(s, bid, ',', p.z);
                read_cd(s, bid, ',', p.x);
                read_cd(s, bid, ')', p.y);
            }
            if (p.z < 0 || p.z >= d.Z || p.x < 0 || p.x >= d.X || p.y < 0 || p.y >= d.Y) {
                bad = 1;
                break;
            }
            int32_t e = d.enc(p.z, p.x, p.y);
            if (!mp.count(e)) mp[e] = p;
        }
        for (auto &kv : mp) pins[i].push_back(kv.first);
        if (!mp.empty()) first_pin[i] = mp.begin()->second;
    }
    if (bad) {
        if (err) *err = "pin outside the grid";
        return GR_ERR_PARSE;
    }
    d.names.clear();
    d.pin_ofs.assign(1, 0);
    d.pins.clear();
    d.odeg_names.clear();
    d.odeg_pins.clear();
    for (int64_t i = 0; i < n_all; i++) {
        if (pins[i].size() == 1) {  // remove_single_deg_nets (read_data.hpp:366-412)
            d.odeg_names.push_back(names[i]);
            d.odeg_pins.push_back(first_pin[i]);
        } else if (pins[i].size() >= 2) {
            d.names.push_back(names[i]);
            d.pins.insert(d.pins.end(), pins[i].begin(), pins[i].end());
            d.pin_ofs.push_back((int64_t)d.pins.size());
        }
    }
    return GR_OK;
}

namespace {

void put_real(std::string &o, double v) {
    char buf[64];
    if (v == std::floor(v) && std::fabs(v) < 1e15) snprintf(buf, sizeof buf, "%.1f", v);
    else snprintf(buf, sizeof buf, "%.9g", v);
    o += buf;
}

}  // namespace

int write_cap(const std::string &path, const Design &d) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return GR_ERR_IO;
    std::string o;
    o += std::to_string(d.Z) + " " + std::to_string(d.X) + " " + std::to_string(d.Y) + "\n";
    put_real(o, d.ulen);
    o += " ";
    put_real(o, d.uvia);
    o += "\n";
    for (int z = 0; z < d.Z; z++) {
        if (z) o += " ";
        put_real(o, z < (int)d.layer_cost.size() ? d.layer_cost[z] : 1.0);
    }
    o += "\n0.0 0.0 0.0 0.0\n";  // the four -new_fmt header values
    for (size_t i = 0; i < d.hlen.size(); i++) o += (i ? " " : "") + std::to_string(d.hlen[i]);
    o += "\n";
    for (size_t i = 0; i < d.vlen.size(); i++) o += (i ? " " : "") + std::to_string(d.vlen[i]);
    o += "\n";
    fwrite(o.data(), 1, o.size(), f);
    for (int z = 0; z < d.Z; z++) {
        o.clear();
        o += (z < (int)d.layer_name.size() && !d.layer_name[z].empty() ? d.layer_name[z]
                                                                          : "metal" + std::to_string(z + 1));
        o += " " + std::to_string(z < (int)d.layer_dir.size() ? d.layer_dir[z] : (z & 1)) + " " +
             std::to_string(z < (int)d.layer_minlen.size() ? d.layer_minlen[z] : 1) + "\n";
        for (int y = 0; y < d.Y; y++) {
            for (int x = 0; x < d.X; x++) {
                if (x) o += " ";
                put_real(o, d.cap[d.enc(z, x, y)]);
            }
            o += "\n";
        }
        fwrite(o.data(), 1, o.size(), f);
    }
    fclose(f);
    return GR_OK;
}

// -new_fmt net text: "name\n(\n[pinK, 0, (z, x, y)]\n...)\n"
int write_net(const std::string &path, const Design &d) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return GR_ERR_IO;
    std::string o;
    auto pin_line = [&](int k, int z, int x, int y) {
        o += "[p" + std::to_string(k) + ", 0, (" + std::to_string(z) + ", " + std::to_string(x) + ", " +
             std::to_string(y) + ")]\n";
    };
    for (int32_t i = 0; i < d.n_nets(); i++) {
        o += d.names[i] + "\n(\n";
        for (int64_t t = d.pin_ofs[i]; t < d.pin_ofs[i + 1]; t++) {
            int z, x, y;
            d.dec(d.pins[t], z, x, y);
            pin_line((int)(t - d.pin_ofs[i]), z, x, y);
        }
        o += ")\n";
        if (o.size() > (1u << 20)) {
            fwrite(o.data(), 1, o.size(), f);
            o.clear();
        }
    }
    for (size_t i = 0; i < d.odeg_names.size(); i++) {
        o += d.odeg_names[i] + "\n(\n";
        pin_line(0, d.odeg_pins[i].z, d.odeg_pins[i].x, d.odeg_pins[i].y);
        o += ")\n";
    }
    fwrite(o.data(), 1, o.size(), f);
    fclose(f);
    return GR_OK;
}

// ------------------------------------------------------------------ synthetic
namespace {

struct Rng {  // xoshiro256** seeded by splitmix64
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto &v : s) {
            x += 0x9e3779b97f4a7c15ull;
            uint64_t z = x;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            v = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double u01() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    int uni(int lo, int hi) { return lo + (int)(next() % (uint64_t)(hi - lo + 1)); }
    double normal() {
        double u1 = u01(), u2 = u01();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

}  // namespace

GenParams standard_params(int config) {
    GenParams p{};
    switch (config) {
        case 1:  // 64x64x5, 2,000 nets
            p = {64, 64, 5, 4, 8, 0.10, 0, 2, 2000, 0.0, 61, 60, 0.03, 6.0, 0.8, 2, 4};
            break;
        case 2:
        case 4:  // 400x400x9, 150,000 nets, 0.5% tail 61..200
            p = {400, 400, 9, 6, 12, 0.15, 0, 3, 150000, 0.005, 61, 200, 0.03, 12.0, 0.8, 2, 4};
            break;
        case 3:
        case 5:  // 1000x1000x10, 1.2M nets, 1% tail up to 400
        default:
            p = {1000, 1000, 10, 8, 16, 0.0, 0, 0, 1200000, 0.01, 61, 400, 0.03, 15.0, 1.0, 2, 4};
            break;
    }
    return p;
}

void generate(const GenParams &p, uint64_t seed, Design &d) {
    d = Design{};
    d.X = p.X;
    d.Y = p.Y;
    d.Z = p.Z;
    d.ulen = 0.5;
    d.uvia = 4.0;
    d.layer_cost.assign(p.Z, 1.0);
    d.hlen.assign(p.X - 1, 4200);
    d.vlen.assign(p.Y - 1, 4200);
    for (int z = 0; z < p.Z; z++) {
        d.layer_name.push_back("metal" + std::to_string(z + 1));
        d.layer_dir.push_back(z & 1);
        d.layer_minlen.push_back(1);
    }
    Rng rc(seed * 2 + 1);
    d.cap.assign((size_t)d.csize(), 0.0f);
    for (int z = 0; z < p.Z; z++)
        for (int y = 0; y < p.Y; y++)
            for (int x = 0; x < p.X; x++) {
                int c = (p.hot_frac > 0 && rc.u01() < p.hot_frac) ? rc.uni(p.hot_lo, p.hot_hi)
                                                                  : rc.uni(p.cap_lo, p.cap_hi);
                d.cap[d.enc(z, x, y)] = (float)c;
            }
    Rng rn(seed * 2 + 2);
    const double mu = std::log(p.bbox_median);
    d.pin_ofs.assign(1, 0);
    std::vector<int32_t> encs;
    for (int64_t i = 0; i < p.n_nets; i++) {
        int n;
        if (p.tail_frac > 0 && rn.u01() < p.tail_frac) {
            double u = rn.u01();
            if (u < 1e-300) u = 1e-300;
            long g = (long)std::floor(std::log(u) / std::log(1.0 - p.tail_p));
            n = (int)std::min<long>(p.tail_lo + g, p.tail_hi);
        } else {
            double r = rn.u01();
            n = r < 0.60 ? 2 : r < 0.85 ? rn.uni(3, 5) : r < 0.98 ? rn.uni(6, 20) : rn.uni(21, 60);
        }
        auto side = [&](int lim) {
            long w = std::lround(std::exp(mu + p.bbox_sigma * rn.normal()));
            return (int)std::max(1L, std::min<long>(w, lim));
        };
        int w = side(p.X), h = side(p.Y);
        int x0 = rn.uni(0, p.X - w), y0 = rn.uni(0, p.Y - h);
        encs.clear();
        Pin first{};
        for (int k = 0; k < n; k++) {
            Pin q{rn.uni(0, p.pin_layers - 1), x0 + rn.uni(0, w - 1), y0 + rn.uni(0, h - 1)};
            if (k == 0) first = q;
            encs.push_back(d.enc(q.z, q.x, q.y));
        }
        std::sort(encs.begin(), encs.end());
        encs.erase(std::unique(encs.begin(), encs.end()), encs.end());
        std::string name = "net" + std::to_string(i);
        if (encs.size() == 1) {
            d.odeg_names.push_back(name);
            d.odeg_pins.push_back(first);
        } else {
            d.names.push_back(name);
            d.pins.insert(d.pins.end(), encs.begin(), encs.end());
            d.pin_ofs.push_back((int64_t)d.pins.size());
        }
    }
}

int integer_caps(const Design &d, std::vector<int32_t> &out) {
    out.resize(d.cap.size());
    for (size_t i = 0; i < d.cap.size(); i++) {
        float v = d.cap[i];
        if (!(v == std::floor(v)) || std::fabs(v) > 1e8f) return GR_ERR_NONINTEGER;
        out[i] = (int32_t)v;
    }
    return GR_OK;
}

// ------------------------------------------------------------------ batching
namespace {

struct Box {
    int minx, maxx, miny, maxy;
};

// closed-box intersection index over one x-bucket (boost::geometry
// intersects on closed boxes: shared edges and corners intersect)
struct BoxIndex {
    static constexpr int kCell = 16;
    int gx = 0, gy = 0;
    std::vector<std::vector<int>> cells;
    std::vector<Box> boxes;
    std::vector<int> touched;
    void init(int X, int Y) {
        gx = (X + kCell - 1) / kCell;
        gy = (Y + kCell - 1) / kCell;
        cells.assign((size_t)gx * gy, {});
        boxes.clear();
        touched.clear();
    }
    void reset() {
        for (int c : touched) cells[c].clear();
        touched.clear();
        boxes.clear();
    }
    bool hits(const Box &b) const {
        for (int cy = b.miny / kCell; cy <= b.maxy / kCell; cy++)
            for (int cx = b.minx / kCell; cx <= b.maxx / kCell; cx++)
                for (int id : cells[(size_t)cy * gx + cx]) {
                    const Box &o = boxes[id];
                    if (b.minx <= o.maxx && o.minx <= b.maxx && b.miny <= o.maxy && o.miny <= b.maxy) return true;
                }
        return false;
    }
    void insert(const Box &b) {
        int id = (int)boxes.size();
        boxes.push_back(b);
        for (int cy = b.miny / kCell; cy <= b.maxy / kCell; cy++)
            for (int cx = b.minx / kCell; cx <= b.maxx / kCell; cx++) {
                auto &v = cells[(size_t)cy * gx + cx];
                if (v.empty()) touched.push_back(cy * gx + cx);
                v.push_back(id);
            }
    }
};

}  // namespace

// NET_PART::part_nets with BATCH_PART (net_part.hpp:236-379) and part_xdim
// (:167-235). The std::sort calls use the reference's comparators on the same
// input sequences (sorting (key, id) records moves them exactly as sorting
// ids through the comparator would), so each batch holds the same nets as the
// reference built with libstdc++. Two deviations: buckets are appended in
// bucket order (the reference's OpenMP critical section interleaves them) and
// the final pin-count sort is stable; routing results do not depend on the
// order of nets inside a batch. Where every remaining net fits into the
// buckets exactly, the reference's bucket assertion (:203) aborts; here the
// extra bucket is simply processed.
void make_batches(const Design &d, int K, Plan &plan) {
    const int32_t N = d.n_nets();
    if (K < 1) K = 1;
    std::vector<Box> bx(N);
    std::vector<int> npins(N);
    for (int32_t i = 0; i < N; i++) {
        Box b{1 << 30, -1, 1 << 30, -1};
        for (int64_t t = d.pin_ofs[i]; t < d.pin_ofs[i + 1]; t++) {
            int z, x, y;
            d.dec(d.pins[t], z, x, y);
            b.minx = std::min(b.minx, x);
            b.maxx = std::max(b.maxx, x);
            b.miny = std::min(b.miny, y);
            b.maxy = std::max(b.maxy, y);
        }
        bx[i] = b;
        npins[i] = (int)(d.pin_ofs[i + 1] - d.pin_ofs[i]);
    }
    std::vector<int> net_ids(N);
    for (int32_t i = 0; i < N; i++) net_ids[i] = i;
    std::vector<char> vis(N, 0);
    // net_part.hpp:244-263: sort by (minx, maxx)
    {
        struct R {
            int64_t key;
            int id;
        };
        std::vector<R> r(N);
        for (int32_t i = 0; i < N; i++) r[i] = {((int64_t)bx[i].minx << 32) | (uint32_t)bx[i].maxx, i};
        std::sort(r.begin(), r.end(), [](const R &a, const R &b) { return a.key < b.key; });
        for (int32_t i = 0; i < N; i++) net_ids[i] = r[i].id;
    }
    plan.batch_ofs.assign(1, 0);
    plan.net_ids.clear();
    plan.net_ids.reserve(N);
    int rem = N;
    // one intersection index per bucket: the buckets' greedy passes are
    // independent and run in parallel (as the reference's OpenMP loop over
    // buckets does); their picks are joined in bucket order
    std::vector<BoxIndex> idxs(K + 1);
    for (auto &ix : idxs) ix.init(d.X, d.Y);
    std::vector<std::vector<int>> picked(K + 1);
    struct RM {
        int key;
        int id;
    };
    std::vector<RM> rm;
    std::vector<int> batch;
    while (rem > 0) {
        // part_xdim: targ_num, sort by maxx (net_part.hpp:168-188)
        const int targ = (rem + K - 1) / K;
        rm.resize(rem);
        for (int i = 0; i < rem; i++) rm[i] = {bx[net_ids[i]].maxx, net_ids[i]};
        std::sort(rm.begin(), rm.end(), [](const RM &a, const RM &b) { return a.key < b.key; });
        for (int i = 0; i < rem; i++) net_ids[i] = rm[i].id;
        // buckets (net_part.hpp:189-202)
        std::vector<int> xid(rem, -1);
        std::vector<int> part_len(K + 1, 0);
        int cmax = -1, cur = 0, num = 0;
        for (int i = 0; i < rem; i++) {
            const Box &b = bx[net_ids[i]];
            if (cur > K) break;
            if (cmax < b.minx) {
                xid[i] = cur;
                num++;
                part_len[cur]++;
            }
            if (num == targ) {
                num = 0;
                cur++;
                cmax = b.maxx;
            }
        }
        const int nparts = std::min(cur, K) + 1;
        std::vector<std::vector<int>> pick(nparts);
        for (int p = 0; p < nparts; p++) pick[p].assign(part_len[p], 0);
        for (int i = 0; i < rem; i++)
            if (xid[i] != -1 && xid[i] < nparts) {
                int p = xid[i], f = part_len[p]--;
                pick[p][f - 1] = net_ids[i];
            }
        // per bucket: sort by half perimeter, greedy non-overlap (:214-234)
        batch.clear();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nparts)
        for (int p = 0; p < nparts; p++) {
            struct RH {
                int key;
                int id;
            };
            std::vector<RH> rh(pick[p].size());
            for (size_t i = 0; i < pick[p].size(); i++) {
                const Box &b = bx[pick[p][i]];
                rh[i] = {(b.maxx - b.minx + 1) + (b.maxy - b.miny + 1), pick[p][i]};
            }
            std::sort(rh.begin(), rh.end(), [](const RH &a, const RH &b) { return a.key < b.key; });
            BoxIndex &idx = idxs[p];
            idx.reset();
            picked[p].clear();
            for (const RH &h : rh) {
                const Box &b = bx[h.id];
                if (!idx.hits(b)) {
                    idx.insert(b);
                    picked[p].push_back(h.id);
                    vis[h.id] = 1;  // each net lies in one bucket: no two threads write one entry
                }
            }
        }
        for (int p = 0; p < nparts; p++) batch.insert(batch.end(), picked[p].begin(), picked[p].end());
        // compaction of the remaining ids (net_part.hpp:326-337)
        int id = 0, fid = 0;
        while (id < rem) {
            if (vis[net_ids[fid]] == 0) fid++;
            if (id > fid && vis[net_ids[id]] == 0) {
                std::swap(net_ids[fid], net_ids[id]);
                fid++;
            }
            id++;
        }
        rem -= (int)batch.size();
        std::stable_sort(batch.begin(), batch.end(), [&](int a, int b) { return npins[a] < npins[b]; });
        plan.net_ids.insert(plan.net_ids.end(), batch.begin(), batch.end());
        plan.batch_ofs.push_back((int64_t)plan.net_ids.size());
        if (batch.empty()) break;  // cannot happen: the first net of a bucket always fits
    }
}

// ------------------------------------------------------------------ routes
namespace {

struct Seg {
    int32_t e1, e2;
};

long gran(long cd) { return 4200L * cd + 2100L; }

// path of one MST edge as segments (writer_util.hpp:300-358): vias as one
// point per unit layer step, wires as (low end, high end) on their track
void edge_segments(const Design &d, int32_t src, int32_t dst, int cpat, std::vector<Seg> &out) {
    const int Z2 = (d.Z + 1) / 2;
    int z1, x1, y1, z2, x2, y2;
    d.dec(src, z1, x1, y1);
    d.dec(dst, z2, x2, y2);
    int via1 = cpat / Z2, via2 = cpat % Z2;
    bool bth = (x1 != x2 && y1 != y2);
    auto vias = [&](int x, int y, int za, int zb) {
        if (za > zb) std::swap(za, zb);
        for (int i = za; i < zb; i++) {
            int32_t e = d.enc(i, x, y);
            out.push_back({e, e});
        }
    };
    auto wire = [&](int z) {
        if (z & 1) {
            int a = std::min(y1, y2), b = std::max(y1, y2);
            if (a != b) out.push_back({d.enc(z, x1, a), d.enc(z, x1, b)});
            y1 = y2;
        } else {
            int a = std::min(x1, x2), b = std::max(x1, x2);
            if (a != b) out.push_back({d.enc(z, a, y1), d.enc(z, b, y1)});
            x1 = x2;
        }
    };
    if (z1 != via1) {
        vias(x1, y1, z1, via1);
        z1 = via1;
    }
    if (z1 > 0) wire(z1);
    via2 = (z1 & 1) ? 2 * via2 : via2 * 2 + 1;
    if (bth && via2 != 0 && z1 != via2) {
        vias(x1, y1, z1, via2);
        z1 = via2;
        wire(z1);
    }
    if (z1 != z2) vias(x1, y1, z1, z2);
}

// merge_st_edges_nnew (writer_util.hpp:166-210)
void merge_segments(std::vector<Seg> &s) {
    std::vector<Seg> w;
    std::set<int32_t> pts;
    for (const Seg &g : s) {
        if (g.e1 == g.e2) pts.insert(g.e1);
        else w.push_back(g);
    }
    if (!w.empty()) {
        std::sort(w.begin(), w.end(), [](const Seg &a, const Seg &b) {
            return a.e1 == b.e1 ? a.e2 < b.e2 : a.e1 < b.e1;
        });
        size_t f = 0;
        Seg cur = w[0];
        for (size_t i = 1; i < w.size(); i++) {
            if (cur.e2 >= w[i].e1) cur.e2 = std::max(cur.e2, w[i].e2);
            else {
                w[f++] = cur;
                cur = w[i];
            }
        }
        w[f++] = cur;
        w.resize(f);
    }
    for (int32_t e : pts) w.push_back({e, e});
    s.swap(w);
}

// oprd_ppatch (writer_util.hpp:239-289): a pin on a layer above 0 that is
// not an end point of any segment splits the wire that passes over it.
bool pin_patch(const Design &d, const int32_t *pins, int n, std::vector<Seg> &s) {
    std::set<int32_t> ends;
    auto cmp = [](const Seg &a, const Seg &b) { return a.e1 == b.e1 ? a.e2 < b.e2 : a.e1 < b.e1; };
    std::set<Seg, decltype(cmp)> wires(cmp);
    for (const Seg &g : s) {
        if (g.e1 == g.e2) {
            int z, x, y;
            d.dec(g.e1, z, x, y);
            ends.insert(d.enc(z, x, y));
            ends.insert(d.enc(z + 1, x, y));
        } else {
            ends.insert(g.e1);
            ends.insert(g.e2);
            wires.insert(g);
        }
    }
    bool ok = true;
    for (int t = 0; t < n; t++) {
        int z, x, y;
        d.dec(pins[t], z, x, y);
        if (z == 0 || ends.count(pins[t])) continue;
        auto it = wires.upper_bound(Seg{pins[t], pins[t]});
        if (it == wires.begin()) {
            ok = false;
            continue;
        }
        --it;
        Seg g = *it;
        if (!(g.e1 < pins[t] && pins[t] < g.e2)) {
            ok = false;
            continue;
        }
        wires.erase(it);
        wires.insert(Seg{g.e1, pins[t]});
        wires.insert(Seg{pins[t], g.e2});
    }
    std::vector<Seg> out;
    for (const Seg &g : s)
        if (g.e1 == g.e2) out.push_back(g);
    for (const Seg &g : wires) out.push_back(g);
    s.swap(out);
    return ok;
}

void put_seg(const Design &d, std::string &o, const Seg &g, bool rseg) {
    int z1, x1, y1, z2, x2, y2;
    d.dec(g.e1, z1, x1, y1);
    d.dec(g.e2, z2, x2, y2);
    char buf[160];
    if (rseg) {  // add_segment (writer_util.hpp:211-223)
        if (g.e1 == g.e2)
            snprintf(buf, sizeof buf, "%ld %ld metal%d %ld %ld metal%d\n", gran(x1), gran(y1), z1 + 1, gran(x2),
                     gran(y2), z1 + 2);
        else
            snprintf(buf, sizeof buf, "%ld %ld metal%d %ld %ld metal%d\n", gran(x1), gran(y1), z1 + 1, gran(x2),
                     gran(y2), z1 + 1);
    } else {
        snprintf(buf, sizeof buf, "%d %d %d %d %d %d\n", z1, x1, y1, z2, x2, y2);
    }
    o += buf;
}

// writer_util.hpp:20-53 (unmerged writer): one line per via step / wire
void put_edge_plain(const Design &d, std::string &o, const std::vector<Seg> &segs, bool rseg) {
    for (const Seg &g : segs) {
        int z1, x1, y1, z2, x2, y2;
        d.dec(g.e1, z1, x1, y1);
        d.dec(g.e2, z2, x2, y2);
        char buf[160];
        if (g.e1 == g.e2) {
            if (rseg)
                snprintf(buf, sizeof buf, "%ld %ld metal%d %ld %ld metal%d\n", gran(x1), gran(y1), z1 + 1,
                         gran(x1), gran(y1), z1 + 2);
            else
                snprintf(buf, sizeof buf, "%d %d %d %d %d %d\n", z1, x1, y1, z1, x1, y1);
        } else if (rseg) {
            snprintf(buf, sizeof buf, "%ld %ld metal%d %ld %ld metal%d\n", gran(x1), gran(y1), z1 + 1, gran(x2),
                     gran(y2), z1 + 2);
        } else {
            snprintf(buf, sizeof buf, "%d %d %d %d %d %d\n", z1, x1, y1, z2, x2, y2);
        }
        o += buf;
    }
}

}  // namespace

int write_routes(const std::string &path, const Design &d, const Plan &plan, const int64_t *mst,
                 const int32_t *mst_pat, bool merge, bool rseg, bool patch, int threads, EvalStats *stats) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return GR_ERR_IO;
    const int64_t nb = (int64_t)plan.batch_ofs.size() - 1;
    const int64_t total = plan.batch_ofs.empty() ? 0 : plan.batch_ofs.back();
    std::vector<int64_t> slot(total + 1, 0);
    for (int64_t i = 0; i < total; i++) {
        int32_t id = plan.net_ids[i];
        slot[i + 1] = slot[i] + (d.pin_ofs[id + 1] - d.pin_ofs[id]);
    }
    std::vector<std::string> text(total);
    std::vector<int64_t> wl(total, 0), nv(total, 0);
    int bad = 0;
    (void)nb;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1) reduction(| : bad)
    for (int64_t i = 0; i < total; i++) {
        const int32_t id = plan.net_ids[i];
        const int64_t o = d.pin_ofs[id];
        const int n = (int)(d.pin_ofs[id + 1] - o);
        std::string &s = text[i];
        s = d.names[id] + "\n(\n";
        std::vector<Seg> segs, one;
        for (int t = 0; t < n; t++) {
            int64_t E = mst[slot[i] + t];
            if (E == -1) continue;
            int n1 = (int)(E & 0x7fff), n2 = (int)((E >> 15) & 0x7fff);
            if (n1 < n2) std::swap(n1, n2);
            if (n1 >= n) {
                bad = 1;
                continue;
            }
            one.clear();
            edge_segments(d, d.pins[o + n1], d.pins[o + n2], mst_pat[slot[i] + t], one);
            if (merge) segs.insert(segs.end(), one.begin(), one.end());
            else put_edge_plain(d, s, one, rseg);
        }
        if (merge) {
            merge_segments(segs);
            if (patch && !pin_patch(d, d.pins.data() + o, n, segs)) bad = 1;
            for (const Seg &g : segs) {
                put_seg(d, s, g, rseg);
                if (g.e1 == g.e2) nv[i]++;
                else wl[i] += g.e2 - g.e1;
            }
        }
        s += ")\n";
    }
    for (int64_t i = 0; i < total; i++) fwrite(text[i].data(), 1, text[i].size(), f);
    // one-pin nets (writer_util.hpp:79-93): a single via step above the pin
    for (size_t i = 0; i < d.odeg_names.size(); i++) {
        const Pin &p = d.odeg_pins[i];
        std::string s = d.odeg_names[i] + "\n(\n";
        char buf[160];
        if (rseg)
            snprintf(buf, sizeof buf, "%ld %ld metal%d %ld %ld metal%d\n", gran(p.x), gran(p.y), p.z + 1, gran(p.x),
                     gran(p.y), p.z + 2);
        else
            snprintf(buf, sizeof buf, "%d %d %d %d %d %d\n", p.z, p.x, p.y, p.z, p.x, p.y);
        s += buf;
        s += ")\n";
        fwrite(s.data(), 1, s.size(), f);
    }
    fclose(f);
    if (stats) {
        stats->wirelength = 0;
        stats->vias = 0;
        for (int64_t i = 0; i < total; i++) {
            stats->wirelength += wl[i];
            stats->vias += nv[i];
        }
    }
    return bad ? GR_ERR_DEVICE : GR_OK;
}

void evaluate_demand(const Design &d, const int32_t *demand, EvalStats &st) {
    st.overflow = 0;
    st.overflow_cells = 0;
    st.demand = 0;
    const int64_t XY = (int64_t)d.X * d.Y;
    for (int64_t e = 0; e < d.csize(); e++) {
        st.demand += demand[e];
        if (e < XY) continue;  // layer 0 carries no wires
        double of = (double)demand[e] - (double)d.cap[e];
        if (of > 0) {
            st.overflow += of;
            st.overflow_cells++;
        }
    }
}

}  // namespace grio
