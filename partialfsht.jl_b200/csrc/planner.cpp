// Host planner: boxes, counted costs, partition and leaf choice (src/Box.jl, src/Cost.jl of
// PartialFSHT.jl). The arithmetic follows the reference step by step so that the same points give
// the same boxes, the same splits and the same leaf.
#include "planner.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <mutex>
#include <string>

#include "geometry.hpp"

namespace pf {

namespace {

std::mutex g_cost_mu;
CostConstants g_cost;

const double kTwoPi = 2 * M_PI;
const double kPolarTol = std::sqrt(DBL_EPSILON);  // sqrt(eps(Float64))

// bucket scratch of the maximum-gap scan (src/Box.jl:203-210), sized once per point set
struct GapWs {
    std::vector<double> bmin, bmax;
    std::vector<char> used;
    explicit GapWs(int64_t n) : bmin(std::max<int64_t>(1, n)), bmax(std::max<int64_t>(1, n)),
                                used(std::max<int64_t>(1, n)) {}
};

struct Gap {
    double lo, hi, gap, at;
};

// _max_gap (src/Box.jl:223-258): extremes of v over the indices, the largest gap between
// consecutive values and the value at its upper edge, by n - 1 equal buckets (the largest gap
// is at least a bucket wide, so it never lies inside one)
template <class Idx>
Gap max_gap(const std::vector<double>& v, const Idx& g, int64_t n, GapWs& ws) {
    double lo = v[g(0)], hi = lo;
    for (int64_t i = 1; i < n; ++i) {
        const double x = v[g(i)];
        lo = std::min(lo, x);
        hi = std::max(hi, x);
    }
    if (n < 2 || hi <= lo) return Gap{lo, hi, 0.0, lo};
    const int64_t nb = n - 1;
    const double w = (hi - lo) / (double)nb;
    std::fill(ws.used.begin(), ws.used.begin() + nb, 0);
    for (int64_t i = 0; i < n; ++i) {
        const double x = v[g(i)];
        int64_t k = (int64_t)std::floor((x - lo) / w);
        k = std::min(std::max<int64_t>(k, 0), nb - 1);
        if (ws.used[k]) {
            ws.bmin[k] = std::min(ws.bmin[k], x);
            ws.bmax[k] = std::max(ws.bmax[k], x);
        } else {
            ws.used[k] = 1;
            ws.bmin[k] = x;
            ws.bmax[k] = x;
        }
    }
    double gap = 0.0, at = hi, prev = lo;
    for (int64_t k = 0; k < nb; ++k) {
        if (!ws.used[k]) continue;
        const double d = ws.bmin[k] - prev;
        if (d > gap) {
            gap = d;
            at = ws.bmin[k];
        }
        prev = ws.bmax[k];
    }
    return Gap{lo, hi, gap, at};
}

struct AllIdx {
    int64_t operator()(int64_t i) const { return i; }
};
struct GroupIdx {
    const std::vector<int32_t>* g;
    int64_t operator()(int64_t i) const { return (*g)[i]; }
};

// longitude arc from a maximum-gap scan: the wrap-around gap closes the circle and the larger
// gap is the one left out (src/Box.jl:82-96, 272-286)
void arc(const Gap& q, double* start, double* extent) {
    double gap = q.gap, st = q.at;
    const double wrap = kTwoPi - q.hi + q.lo;
    if (wrap >= gap) {
        gap = wrap;
        st = q.lo;
    }
    const double ext = kTwoPi - gap;
    if (ext <= 0) {
        *start = q.lo;
        *extent = 0.0;
    } else if (ext >= kTwoPi) {
        *start = 0.0;
        *extent = kTwoPi;
    } else {
        *start = st;
        *extent = ext;
    }
}

// _group_box (src/Box.jl:261-287)
SphereBox group_box(const std::vector<double>& tv, const std::vector<double>& pv,
                    const std::vector<int32_t>& g, GapWs& ws) {
    const GroupIdx gi{&g};
    const Gap t = max_gap(tv, gi, (int64_t)g.size(), ws);
    SphereBox b;
    b.lo = t.lo;
    b.hi = t.hi;
    b.touches_north = t.lo <= kPolarTol;
    b.touches_south = t.hi >= M_PI - kPolarTol;
    if (b.touches_north || b.touches_south) {
        b.phistart = 0.0;
        b.phiext = kTwoPi;
        return b;
    }
    const Gap p = max_gap(pv, gi, (int64_t)g.size(), ws);
    arc(p, &b.phistart, &b.phiext);
    return b;
}

// _split_below (src/Box.jl:310-330): false when a side would be empty
bool split_below(const std::vector<double>& v, const std::vector<int32_t>& g, double thresh,
                 std::vector<int32_t>& a, std::vector<int32_t>& b) {
    size_t na = 0;
    for (int32_t i : g) na += v[i] < thresh;
    if (na == 0 || na == g.size()) return false;
    a.clear();
    b.clear();
    a.reserve(na);
    b.reserve(g.size() - na);
    for (int32_t i : g) (v[i] < thresh ? a : b).push_back(i);
    return true;
}

// _best_gap_split (src/Box.jl:289-307): the larger of the colatitude gap and the longitude gap
// weighted by the ring radius
bool best_gap_split(const std::vector<double>& tv, const std::vector<double>& pv,
                    const std::vector<int32_t>& g, GapWs& ws, std::vector<int32_t>& a,
                    std::vector<int32_t>& b) {
    const GroupIdx gi{&g};
    const Gap t = max_gap(tv, gi, (int64_t)g.size(), ws);
    const Gap p = max_gap(pv, gi, (int64_t)g.size(), ws);
    const double mid = (t.lo + t.hi) / 2;
    const double wphi = p.gap * std::sin(std::min(std::max(mid, kPolarTol), M_PI - kPolarTol));
    if (t.gap >= wphi) {
        if (!(t.gap > 0)) return false;
        return split_below(tv, g, t.at, a, b);
    }
    if (!(p.gap > 0)) return false;
    return split_below(pv, g, p.at, a, b);
}

double fft_units(double n) { return n <= 1 ? 0.0 : n * std::log2(n); }

}  // namespace

CostConstants cost_constants() {
    std::lock_guard<std::mutex> lk(g_cost_mu);
    return g_cost;
}

void set_cost_constants(double ring, double fft, double spread, double ft_conn) {
    std::lock_guard<std::mutex> lk(g_cost_mu);
    g_cost.ring = ring;
    g_cost.fft = fft;
    g_cost.spread = spread;
    g_cost.ft_conn = ft_conn;
    g_cost.calibrated = true;
}

SphereBox bounding_box(const double* theta, const double* phi, int64_t n) {
    SphereBox b;
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        lo = std::min(lo, theta[i]);
        hi = std::max(hi, theta[i]);
    }
    b.lo = std::max(lo, 0.0);
    b.hi = std::min(hi, M_PI);
    b.touches_north = b.lo <= kPolarTol;
    b.touches_south = b.hi >= M_PI - kPolarTol;
    if (b.touches_north || b.touches_south) {
        b.phistart = 0.0;
        b.phiext = kTwoPi;
        return b;
    }
    std::vector<double> ps(n);
    for (int64_t i = 0; i < n; ++i) ps[i] = jl_mod(phi[i], kTwoPi);
    if (n == 1) {
        b.phistart = ps[0];
        b.phiext = 0.0;
        return b;
    }
    GapWs ws(n);
    const Gap q = max_gap(ps, AllIdx{}, n, ws);
    arc(q, &b.phistart, &b.phiext);
    return b;
}

double cost_direct(int64_t npts, int lmax, int ntrans) {
    const CostConstants c = cost_constants();
    return c.ring * (double)npts * ((double)lmax + 1) * ((double)lmax + 1) * ntrans / 2;
}

double cost_stretch(const SphereBox& box, int64_t npts, int lmax, int ntrans, double tol) {
    Leaf lf;
    std::string err;
    // the leaf's own sizing at the default apodisation limit and no oversampling
    const int r = build_leaf(box.lo, box.hi, lmax, ntrans, tol, 1.0, 1.0, 1.0, &lf, &err);
    if (r != 0) return INFINITY;
    const CostConstants c = cost_constants();
    const double fft = fft_units((double)lf.nph) * lf.nth_half + fft_units((double)lf.nth * lf.nph);
    const double taps = 2 * std::ceil(std::fabs(std::log10(std::max(tol, 1e-16)))) + 2;
    const double spread = (double)npts * taps * taps;
    return ntrans * (c.ring * (double)lf.ring_work + c.fft * fft + c.spread * spread);
}

void partition_boxes_costed(const double* theta, const double* phi, int64_t n, int lmax,
                            int ntrans, double tol, int maxboxes, Partition& out) {
    out = Partition{};
    std::vector<double> tv(theta, theta + n), pv(n);
    for (int64_t i = 0; i < n; ++i) pv[i] = jl_mod(phi[i], kTwoPi);
    GapWs ws(n);
    auto cost = [&](const SphereBox& b, int64_t np) { return cost_stretch(b, np, lmax, ntrans, tol); };
    std::vector<int32_t> all(n);
    for (int64_t i = 0; i < n; ++i) all[i] = (int32_t)i;
    out.groups.push_back(std::move(all));
    out.boxes.push_back(group_box(tv, pv, out.groups[0], ws));
    out.costs.push_back(cost(out.boxes[0], n));
    std::vector<int32_t> a, b, ba, bb;
    while ((int)out.groups.size() < maxboxes) {
        double best_gain = 0.0;
        size_t best_at = SIZE_MAX;
        std::vector<int32_t> bga, bgb;
        SphereBox bxa, bxb;
        for (size_t gi = 0; gi < out.groups.size(); ++gi) {
            const std::vector<int32_t>& g = out.groups[gi];
            if (g.size() < 2) continue;
            if (!best_gap_split(tv, pv, g, ws, a, b)) continue;
            const SphereBox xa = group_box(tv, pv, a, ws), xb = group_box(tv, pv, b, ws);
            const double gain = out.costs[gi] - (cost(xa, (int64_t)a.size()) + cost(xb, (int64_t)b.size()));
            if (gain > best_gain) {
                best_gain = gain;
                best_at = gi;
                bga.swap(a);
                bgb.swap(b);
                bxa = xa;
                bxb = xb;
            }
        }
        if (best_at == SIZE_MAX) break;
        out.groups.erase(out.groups.begin() + best_at);
        out.boxes.erase(out.boxes.begin() + best_at);
        out.costs.erase(out.costs.begin() + best_at);
        const double ca = cost(bxa, (int64_t)bga.size()), cb = cost(bxb, (int64_t)bgb.size());
        out.groups.push_back(std::move(bga));
        out.boxes.push_back(bxa);
        out.costs.push_back(ca);
        out.groups.push_back(std::move(bgb));
        out.boxes.push_back(bxb);
        out.costs.push_back(cb);
    }
}

int select_method(const double* theta, const double* phi, int64_t n, int lmax, int ntrans,
                  double tol, Partition* part) {
    const SphereBox box = bounding_box(theta, phi, n);
    const double cd = cost_direct(n, lmax, ntrans);
    const double cs = cost_stretch(box, n, lmax, ntrans, tol);
    int best = 2;  // direct
    double bestc = cd;
    if (cs < bestc) {
        best = 1;
        bestc = cs;
    }
    Partition local;
    Partition& p = part ? *part : local;
    partition_boxes_costed(theta, phi, n, lmax, ntrans, tol, 8, p);
    if (p.groups.size() > 1) {
        double cm = 0;
        for (double c : p.costs) cm += c;
        if (cm < bestc) best = 3;
    }
    return best;
}

}  // namespace pf
