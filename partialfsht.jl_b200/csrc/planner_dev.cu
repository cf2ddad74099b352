// The planner's point-set scans on the device: the bucketed maximum gap (src/Box.jl:223-258),
// boxes of point groups (src/Box.jl:261-287) and the splits of the partition search
// (src/Box.jl:156-200, 289-330). The cost model and the search loop stay on the host
// (planner.cpp); only the O(n) passes over the points move here, with the same floating-point
// operations, so that the groups, boxes and costs equal the host planner's.
//
// Maximum gap of v over a group g (n values): min/max by atomics on order-preserving 64-bit
// keys; n - 1 equal buckets, each bucket's min/max by atomics; an inclusive prefix max of the
// bucket maxima gives every bucket's predecessor; the gap before bucket k is its minimum minus
// that predecessor, and the first bucket with the largest gap is an argmax (CUB returns the
// lowest index among equal maxima, as the host scan keeps the first strictly larger gap).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <memory>
#include <vector>

#include "internal.cuh"
#include "planner.hpp"

namespace pf {

namespace {

constexpr unsigned long long kSign = 0x8000000000000000ull;

// order-preserving key of a double: keys compare as unsigned integers as the values compare
__host__ __device__ inline unsigned long long okey_bits(unsigned long long b) {
    return (b & kSign) ? ~b : (b | kSign);
}
__host__ __device__ inline unsigned long long unkey_bits(unsigned long long k) {
    return (k & kSign) ? (k & ~kSign) : ~k;
}
__device__ inline unsigned long long okey(double x) {
    return okey_bits((unsigned long long)__double_as_longlong(x));
}
__device__ inline double unkey(unsigned long long k) {
    return __longlong_as_double((long long)unkey_bits(k));
}
double unkey_host(unsigned long long k) {
    const unsigned long long b = unkey_bits(k);
    double x;
    memcpy(&x, &b, sizeof(x));
    return x;
}

__device__ inline double vat(const double* v, const int* g, int64_t i) { return g ? v[g[i]] : v[i]; }

__device__ inline double jl_mod_dev(double x, double y) {
    const double r = fmod(x, y);
    if (r == 0.0) return copysign(r, y);
    if ((r > 0) != (y > 0)) return r + y;
    return r;
}

__global__ void mod2pi_kernel(const double* __restrict__ phi, int64_t n, double* __restrict__ out) {
    const double two_pi = 2 * M_PI;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = jl_mod_dev(phi[i], two_pi);
}

__global__ void minmax_kernel(const double* __restrict__ v, const int* __restrict__ g, int64_t n,
                              unsigned long long* __restrict__ mm) {
    unsigned long long lo = ~0ull, hi = 0ull;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = okey(vat(v, g, i));
        lo = min(lo, k);
        hi = max(hi, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}

// bucket k = clamp(floor((x - lo) / w), 0, nb - 1), as the host scan
__global__ void bucket_kernel(const double* __restrict__ v, const int* __restrict__ g, int64_t n,
                              double lo, double w, int64_t nb, unsigned long long* __restrict__ bmin,
                              unsigned long long* __restrict__ bmax) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double x = vat(v, g, i);
        int64_t k = (int64_t)floor((x - lo) / w);
        k = min(max(k, (int64_t)0), nb - 1);
        const unsigned long long key = okey(x);
        atomicMin(bmin + k, key);
        atomicMax(bmax + k, key);
    }
}

// gap before each non-empty bucket (bucket 0 holds lo, so every later bucket has a predecessor)
__global__ void gap_kernel(const unsigned long long* __restrict__ bmin,
                           const unsigned long long* __restrict__ pmax, int64_t nb, double lo,
                           double* __restrict__ d) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nb;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (bmin[k] == ~0ull) {
            d[k] = -INFINITY;
        } else {
            const double prev = k == 0 ? lo : unkey(pmax[k - 1]);
            d[k] = unkey(bmin[k]) - prev;
        }
    }
}

__global__ void flags_kernel(const double* __restrict__ v, const int* __restrict__ g, int64_t n,
                             double thresh, char* __restrict__ below, char* __restrict__ above) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const bool b = vat(v, g, i) < thresh;
        below[i] = b;
        above[i] = !b;
    }
}

__global__ void iota_kernel(int* __restrict__ g, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        g[i] = (int)i;
}

unsigned grid_of(int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8));
}

struct Gap {
    double lo, hi, gap, at;
};

// scratch of the scans, sized once for n points
struct Scratch {
    int64_t cap = 0;
    DevBuf mm, bmin, bmax, pmax, d, kv, tmp, fa, fb, cnt;
    size_t tmp_bytes = 0;
    int alloc(int64_t n, cudaStream_t s) {
        cap = std::max<int64_t>(n, 2);
        PF_TRY(mm.alloc(2 * sizeof(unsigned long long)));
        PF_TRY(bmin.alloc(sizeof(unsigned long long) * cap));
        PF_TRY(bmax.alloc(sizeof(unsigned long long) * cap));
        PF_TRY(pmax.alloc(sizeof(unsigned long long) * cap));
        PF_TRY(d.alloc(sizeof(double) * cap));
        PF_TRY(kv.alloc(sizeof(cub::KeyValuePair<int, double>)));
        PF_TRY(fa.alloc(cap));
        PF_TRY(fb.alloc(cap));
        PF_TRY(cnt.alloc(sizeof(int)));
        size_t a = 0, b = 0, c = 0;
        const int ni = (int)cap;
        PF_CUDA(cub::DeviceScan::InclusiveScan(nullptr, a, bmax.as<unsigned long long>(),
                                               pmax.as<unsigned long long>(), cub::Max(), ni, s));
        PF_CUDA(cub::DeviceReduce::ArgMax(nullptr, b, d.as<double>(),
                                          kv.as<cub::KeyValuePair<int, double>>(), ni, s));
        PF_CUDA(cub::DeviceSelect::Flagged(nullptr, c, (const int*)nullptr, fa.as<char>(),
                                           (int*)nullptr, cnt.as<int>(), ni, s));
        tmp_bytes = std::max(a, std::max(b, c));
        PF_TRY(tmp.alloc(tmp_bytes));
        return 0;
    }
};

int max_gap_dev(const double* v, const int* g, int64_t n, Scratch& sc, cudaStream_t s, Gap* out) {
    unsigned long long mm[2] = {~0ull, 0ull};
    PF_CUDA(cudaMemcpyAsync(sc.mm.p, mm, sizeof(mm), cudaMemcpyHostToDevice, s));
    minmax_kernel<<<grid_of(n), 256, 0, s>>>(v, g, n, sc.mm.as<unsigned long long>());
    PF_TRY(check_launch("minmax_kernel"));
    PF_CUDA(cudaMemcpyAsync(mm, sc.mm.p, sizeof(mm), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    const double lo = unkey_host(mm[0]), hi = unkey_host(mm[1]);
    if (n < 2 || hi <= lo) {
        *out = Gap{lo, hi, 0.0, lo};
        return 0;
    }
    const int64_t nb = n - 1;
    const double w = (hi - lo) / (double)nb;
    PF_CUDA(cudaMemsetAsync(sc.bmin.p, 0xff, sizeof(unsigned long long) * nb, s));
    PF_CUDA(cudaMemsetAsync(sc.bmax.p, 0, sizeof(unsigned long long) * nb, s));
    bucket_kernel<<<grid_of(n), 256, 0, s>>>(v, g, n, lo, w, nb, sc.bmin.as<unsigned long long>(),
                                             sc.bmax.as<unsigned long long>());
    PF_TRY(check_launch("bucket_kernel"));
    size_t tb = sc.tmp_bytes;
    PF_CUDA(cub::DeviceScan::InclusiveScan(sc.tmp.p, tb, sc.bmax.as<unsigned long long>(),
                                           sc.pmax.as<unsigned long long>(), cub::Max(), (int)nb, s));
    gap_kernel<<<grid_of(nb), 256, 0, s>>>(sc.bmin.as<unsigned long long>(),
                                           sc.pmax.as<unsigned long long>(), nb, lo, sc.d.as<double>());
    PF_TRY(check_launch("gap_kernel"));
    tb = sc.tmp_bytes;
    PF_CUDA(cub::DeviceReduce::ArgMax(sc.tmp.p, tb, sc.d.as<double>(),
                                      sc.kv.as<cub::KeyValuePair<int, double>>(), (int)nb, s));
    cub::KeyValuePair<int, double> kv;
    PF_CUDA(cudaMemcpyAsync(&kv, sc.kv.p, sizeof(kv), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    Gap r{lo, hi, 0.0, hi};
    if (kv.value > 0) {
        unsigned long long kb = 0;
        PF_CUDA(cudaMemcpyAsync(&kb, sc.bmin.as<unsigned long long>() + kv.key, sizeof(kb),
                                cudaMemcpyDeviceToHost, s));
        PF_CUDA(cudaStreamSynchronize(s));
        r.gap = kv.value;
        r.at = unkey_host(kb);
    }
    *out = r;
    return 0;
}

// a group of points: its indices on the device
struct DevGroup {
    std::shared_ptr<DevBuf> idx;
    int64_t n = 0;
    const int* p() const { return idx->as<int>(); }
};

const double kTwoPi = 2 * M_PI;

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

int group_box_dev(const double* tv, const double* pv, const DevGroup& g, Scratch& sc,
                  cudaStream_t s, SphereBox* out) {
    const double tol = std::sqrt(2.220446049250313e-16);
    Gap t;
    PF_TRY(max_gap_dev(tv, g.p(), g.n, sc, s, &t));
    SphereBox b;
    b.lo = t.lo;
    b.hi = t.hi;
    b.touches_north = t.lo <= tol;
    b.touches_south = t.hi >= M_PI - tol;
    if (b.touches_north || b.touches_south) {
        b.phistart = 0.0;
        b.phiext = kTwoPi;
    } else {
        Gap q;
        PF_TRY(max_gap_dev(pv, g.p(), g.n, sc, s, &q));
        arc(q, &b.phistart, &b.phiext);
    }
    *out = b;
    return 0;
}

// stable split of g by v < thresh; *ok = false when a side would be empty
int split_below_dev(const double* v, const DevGroup& g, double thresh, Scratch& sc, cudaStream_t s,
                    DevGroup& a, DevGroup& b, bool* ok) {
    flags_kernel<<<grid_of(g.n), 256, 0, s>>>(v, g.p(), g.n, thresh, sc.fa.as<char>(), sc.fb.as<char>());
    PF_TRY(check_launch("flags_kernel"));
    a.idx = std::make_shared<DevBuf>();
    b.idx = std::make_shared<DevBuf>();
    PF_TRY(a.idx->alloc(sizeof(int) * g.n));
    PF_TRY(b.idx->alloc(sizeof(int) * g.n));
    size_t tb = sc.tmp_bytes;
    PF_CUDA(cub::DeviceSelect::Flagged(sc.tmp.p, tb, g.p(), sc.fa.as<char>(), a.idx->as<int>(),
                                       sc.cnt.as<int>(), (int)g.n, s));
    int na = 0;
    PF_CUDA(cudaMemcpyAsync(&na, sc.cnt.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    *ok = na > 0 && na < g.n;
    if (!*ok) return 0;
    tb = sc.tmp_bytes;
    PF_CUDA(cub::DeviceSelect::Flagged(sc.tmp.p, tb, g.p(), sc.fb.as<char>(), b.idx->as<int>(),
                                       sc.cnt.as<int>(), (int)g.n, s));
    a.n = na;
    b.n = g.n - na;
    return 0;
}

int best_gap_split_dev(const double* tv, const double* pv, const DevGroup& g, Scratch& sc,
                       cudaStream_t s, DevGroup& a, DevGroup& b, bool* ok) {
    const double tol = std::sqrt(2.220446049250313e-16);
    Gap t, p;
    PF_TRY(max_gap_dev(tv, g.p(), g.n, sc, s, &t));
    PF_TRY(max_gap_dev(pv, g.p(), g.n, sc, s, &p));
    const double mid = (t.lo + t.hi) / 2;
    const double wphi = p.gap * std::sin(std::min(std::max(mid, tol), M_PI - tol));
    *ok = false;
    if (t.gap >= wphi) {
        if (!(t.gap > 0)) return 0;
        return split_below_dev(tv, g, t.at, sc, s, a, b, ok);
    }
    if (!(p.gap > 0)) return 0;
    return split_below_dev(pv, g, p.at, sc, s, a, b, ok);
}

}  // namespace

// Partition search of src/Box.jl:156-200 with the scans on the device. theta and phi are device
// arrays of n points; groups come back as device index lists (ascending).
int partition_boxes_device(const double* theta, const double* phi, int64_t n, int lmax, int ntrans,
                           double tol, int maxboxes, cudaStream_t s, DevPartition& out) {
    out = DevPartition{};
    Scratch sc;
    PF_TRY(sc.alloc(n, s));
    DevBuf pvb;
    PF_TRY(pvb.alloc(sizeof(double) * std::max<int64_t>(n, 1)));
    mod2pi_kernel<<<grid_of(n), 256, 0, s>>>(phi, n, pvb.as<double>());
    PF_TRY(check_launch("mod2pi_kernel"));
    const double* tv = theta;
    const double* pv = pvb.as<double>();
    auto cost = [&](const SphereBox& b, int64_t np) { return cost_stretch(b, np, lmax, ntrans, tol); };
    DevGroup all;
    all.idx = std::make_shared<DevBuf>();
    PF_TRY(all.idx->alloc(sizeof(int) * std::max<int64_t>(n, 1)));
    all.n = n;
    iota_kernel<<<grid_of(n), 256, 0, s>>>(all.idx->as<int>(), n);
    PF_TRY(check_launch("iota_kernel"));
    std::vector<DevGroup> groups{all};
    std::vector<SphereBox> boxes(1);
    PF_TRY(group_box_dev(tv, pv, all, sc, s, &boxes[0]));
    std::vector<double> costs{cost(boxes[0], n)};
    // a group's best split does not change while the group stays: evaluate it once
    struct Cand {
        bool done = false, ok = false;
        DevGroup a, b;
        SphereBox ba, bb;
        double ca = 0, cb = 0;
    };
    std::vector<Cand> cand(1);
    while ((int)groups.size() < maxboxes) {
        double best_gain = 0.0;
        size_t best_at = SIZE_MAX;
        for (size_t gi = 0; gi < groups.size(); ++gi) {
            Cand& c = cand[gi];
            if (!c.done) {
                c.done = true;
                if (groups[gi].n >= 2) {
                    PF_TRY(best_gap_split_dev(tv, pv, groups[gi], sc, s, c.a, c.b, &c.ok));
                    if (c.ok) {
                        PF_TRY(group_box_dev(tv, pv, c.a, sc, s, &c.ba));
                        PF_TRY(group_box_dev(tv, pv, c.b, sc, s, &c.bb));
                        c.ca = cost(c.ba, c.a.n);
                        c.cb = cost(c.bb, c.b.n);
                    }
                }
            }
            if (!c.ok) continue;
            const double gain = costs[gi] - (c.ca + c.cb);
            if (gain > best_gain) {
                best_gain = gain;
                best_at = gi;
            }
        }
        if (best_at == SIZE_MAX) break;
        Cand c = cand[best_at];
        groups.erase(groups.begin() + best_at);
        boxes.erase(boxes.begin() + best_at);
        costs.erase(costs.begin() + best_at);
        cand.erase(cand.begin() + best_at);
        groups.push_back(c.a);
        boxes.push_back(c.ba);
        costs.push_back(c.ca);
        cand.emplace_back();
        groups.push_back(c.b);
        boxes.push_back(c.bb);
        costs.push_back(c.cb);
        cand.emplace_back();
    }
    for (size_t i = 0; i < groups.size(); ++i) {
        out.idx.push_back(groups[i].idx);
        out.n.push_back(groups[i].n);
    }
    out.boxes = boxes;
    out.costs = costs;
    return 0;
}

int bounding_box_device(const double* theta, const double* phi, int64_t n, cudaStream_t s,
                        SphereBox* out) {
    Scratch sc;
    PF_TRY(sc.alloc(n, s));
    Gap t{};
    {
        unsigned long long mm[2] = {~0ull, 0ull};
        PF_CUDA(cudaMemcpyAsync(sc.mm.p, mm, sizeof(mm), cudaMemcpyHostToDevice, s));
        minmax_kernel<<<grid_of(n), 256, 0, s>>>(theta, nullptr, n, sc.mm.as<unsigned long long>());
        PF_TRY(check_launch("minmax_kernel"));
        PF_CUDA(cudaMemcpyAsync(mm, sc.mm.p, sizeof(mm), cudaMemcpyDeviceToHost, s));
        PF_CUDA(cudaStreamSynchronize(s));
        t.lo = unkey_host(mm[0]);
        t.hi = unkey_host(mm[1]);
    }
    const double tol = std::sqrt(2.220446049250313e-16);
    SphereBox b;
    b.lo = std::max(t.lo, 0.0);
    b.hi = std::min(t.hi, M_PI);
    b.touches_north = b.lo <= tol;
    b.touches_south = b.hi >= M_PI - tol;
    if (b.touches_north || b.touches_south) {
        b.phistart = 0.0;
        b.phiext = kTwoPi;
        *out = b;
        return 0;
    }
    DevBuf pvb;
    PF_TRY(pvb.alloc(sizeof(double) * n));
    mod2pi_kernel<<<grid_of(n), 256, 0, s>>>(phi, n, pvb.as<double>());
    PF_TRY(check_launch("mod2pi_kernel"));
    if (n == 1) {
        double p0 = 0;
        PF_CUDA(cudaMemcpyAsync(&p0, pvb.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        PF_CUDA(cudaStreamSynchronize(s));
        b.phistart = p0;
        b.phiext = 0.0;
        *out = b;
        return 0;
    }
    Gap q;
    PF_TRY(max_gap_dev(pvb.as<double>(), nullptr, n, sc, s, &q));
    arc(q, &b.phistart, &b.phiext);
    *out = b;
    return 0;
}

int select_method_device(const double* theta, const double* phi, int64_t n, int lmax, int ntrans,
                         double tol, cudaStream_t s, int* method, DevPartition* part) {
    SphereBox box;
    PF_TRY(bounding_box_device(theta, phi, n, s, &box));
    const double cd = cost_direct(n, lmax, ntrans);
    const double cs = cost_stretch(box, n, lmax, ntrans, tol);
    int best = 2;
    double bestc = cd;
    if (cs < bestc) {
        best = 1;
        bestc = cs;
    }
    DevPartition local;
    DevPartition& p = part ? *part : local;
    PF_TRY(partition_boxes_device(theta, phi, n, lmax, ntrans, tol, 8, s, p));
    if (p.idx.size() > 1) {
        double cm = 0;
        for (double c : p.costs) cm += c;
        if (cm < bestc) best = 3;
    }
    *method = best;
    return 0;
}

}  // namespace pf
