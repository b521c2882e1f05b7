// Stand-in for the few Boost.Geometry names the reference's batcher uses
// (part_net/net_part.hpp, part_net/part_util.hpp, common.h:155-158), so that
// the reference's own sources compile without Boost for the parity recipe
// in oracle/ref. TEST INFRASTRUCTURE ONLY: nothing in the product uses it.
//
//   point<T, 2, cs::cartesian>   an (x, y) pair with get<0>/get<1>
//   box<P>                       closed rectangle [min_corner, max_corner]
//   index::rtree<box, rstar<N>>  insert, clear, query(intersects(b), out)
//
// The rtree is a grid of buckets: the batcher only asks whether any stored
// box intersects a query box, so the answer (not its order) is what matters.
// intersects() is Boost's closed-box test: boxes that touch intersect.
#pragma once
#include <algorithm>
#include <cstddef>
#include <unordered_map>
#include <vector>

namespace boost {
namespace geometry {
namespace cs {
struct cartesian {};
}  // namespace cs
namespace model {
template <class T, std::size_t D, class CS>
struct point {
    T v[2] = {T(), T()};
    point() = default;
    point(T x, T y) { v[0] = x; v[1] = y; }
    template <std::size_t K>
    T get() const { return v[K]; }
};
template <class P>
struct box {
    P lo, hi;
    box() = default;
    box(const P &a, const P &b) : lo(a), hi(b) {}
    const P &min_corner() const { return lo; }
    const P &max_corner() const { return hi; }
};
}  // namespace model
namespace index {
template <std::size_t N>
struct rstar {};
template <class B>
struct intersects_pred {
    B b;
};
template <class B>
intersects_pred<B> intersects(const B &b) { return intersects_pred<B>{b}; }
template <class B, class Params>
class rtree {
    // boxes bucketed by the 32 x 32 cells of the plane they cover, so that a
    // query tests only the boxes stored in the cells its own box covers
    std::vector<B> items_;
    std::unordered_map<long long, std::vector<std::size_t>> cells_;
    static long long key(long long cx, long long cy) { return (cx << 32) ^ (cy & 0xffffffffLL); }
    template <class F>
    static void cover(const B &b, F f) {
        for (long long cx = (long long)b.lo.v[0] >> 5; cx <= ((long long)b.hi.v[0] >> 5); cx++)
            for (long long cy = (long long)b.lo.v[1] >> 5; cy <= ((long long)b.hi.v[1] >> 5); cy++) f(key(cx, cy));
    }
    static bool meet(const B &a, const B &b) {
        return !(a.hi.v[0] < b.lo.v[0] || b.hi.v[0] < a.lo.v[0] || a.hi.v[1] < b.lo.v[1] || b.hi.v[1] < a.lo.v[1]);
    }
public:
    void insert(const B &b) {
        const std::size_t id = items_.size();
        items_.push_back(b);
        cover(b, [&](long long k) { cells_[k].push_back(id); });
    }
    void clear() {
        items_.clear();
        cells_.clear();
    }
    std::size_t size() const { return items_.size(); }
    template <class Out>
    std::size_t query(const intersects_pred<B> &q, Out out) const {
        std::vector<std::size_t> hit;
        cover(q.b, [&](long long k) {
            auto it = cells_.find(k);
            if (it == cells_.end()) return;
            for (std::size_t id : it->second)
                if (meet(items_[id], q.b)) hit.push_back(id);
        });
        std::sort(hit.begin(), hit.end());
        hit.erase(std::unique(hit.begin(), hit.end()), hit.end());
        for (std::size_t id : hit) *out++ = items_[id];
        return hit.size();
    }
};
}  // namespace index
}  // namespace geometry
}  // namespace boost
