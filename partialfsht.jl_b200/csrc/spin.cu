// Spin-weighted ring pass: G[j, m] = sum_l sa_{lm} N_l d^l_{m,-s}(theta_j) and its exact
// transpose (src/Spin.jl:319-490, SpinRings), for the stretched and Direct leaves of spin s != 0.
//
// A warp takes one order m (m = -lmax..lmax: the Wigner-d of +m and -m differ, so orders are not
// paired as in the scalar pass) and a tile of up to 32 R rings; a lane owns R rings. Each ring is
// seeded at l0 = max(|m|, |s|) from the extremal closed form, sg 2^(lb2 + pc log2 cos(t/2) +
// ps log2 sin(t/2)), with the log-binomial, exponents and sign tabulated per order and the two
// logarithms per ring (src/Spin.jl:190-245), and carries its own power-of-two exponent (the
// reference shares one per ring chunk; power-of-two scalings are exact, so both give the same
// values to rounding). The recurrence d_{l+1} = (a1 cos t - a2) d_l - a0 d_{l-1}
// (src/Spin.jl:6-8) costs three FP64 operations per (ring, degree). Its coefficients for the next
// 32 degrees are computed one degree per lane and staged in shared memory:
//     a1 = (2l-1) l / (sm sn),  a2 = (2l-1) m n / ((l-1) sm sn),  a0 = l sm' sn' / ((l-1) sm sn),
// sm = sqrt(l^2 - m^2), sn = sqrt(l^2 - n^2) and the primed values at l - 1 (the reference's
// expressions with den = (l-1) sm sn divided through), from one reciprocal square root and one
// square root per lane and a per-degree table of 1/sn, sn, 1/l and N_l. Every 32 degrees the
// state is renormalised by a power of two read from its exponent field.
// Forward: each ring accumulates N_l a_{lm} d_l and writes G (windowed, mirrored into the DFS
// rows with sign (-1)^(m+s), zeros for the rings the order does not retain).
// Adjoint: each ring scales its G value by its window and 2^E once per exponent change; per
// degree the lanes' partial sums are transposed through shared memory and reduced one degree per
// lane, then added into the coefficient (orders split over several tiles add atomically).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace pf {

namespace {

constexpr int kSpinWarps = 4;     // forward: warps per block
constexpr int kSpinAdjWarps = 2;  // adjoint: warps per block (18 KB of shared memory each)
constexpr int kSpinFwdUnroll = 4;  // forward degree loop (measured: 0.357 ms vs 0.370 unrolled by 8)

struct SpinCoef {
    double a1, a2, a0, N;
};

__device__ __forceinline__ int spin_renorm_shift(double q1, double q2) {
    const double mx = fmax(fabs(q1), fabs(q2));
    const int e = (__double2hiint(mx) >> 20) & 0x7ff;
    return (e == 0 || e == 0x7ff) ? 0 : e - 1022;
}

// recurrence coefficients taking d_{L1 - 1}, d_{L1 - 2} to d_{L1} (src/Spin.jl:404-416); L1 > l0,
// so L1^2 - m^2 > 0 and L1 - 1 >= 1
__device__ __forceinline__ SpinCoef spin_coef(const double4* __restrict__ lt, int L1, int m, int n) {
    const int Lc = L1 - 1;
    const double4 t1 = lt[L1], t0 = lt[Lc];  // (1/sn, sn, 1/l, N_l)
    const double q = rsqrt((double)L1 * L1 - (double)m * m) * t1.x;  // 1 / (sm1 sn1)
    const double sm0 = sqrt((double)Lc * Lc - (double)m * m);
    const double c = (double)(2 * Lc + 1);
    SpinCoef k;
    k.a1 = c * (double)L1 * q;
    k.a2 = c * ((double)m * (double)n) * t0.z * q;
    k.a0 = (double)L1 * sm0 * t0.y * t0.z * q;
    k.N = t1.w;
    return k;
}

__device__ __forceinline__ size_t sidx(int l, int m, int L) { return (size_t)l + (size_t)(L + 1) * (m + L); }

struct SpinFwdSmem {
    double a1[32], a2[32], a0[32];
    double2 a[32];  // N_l a_{lm}
};

// seed of ring j at l0: d = sg 2^(e - E), E = ceil(e) (0 and d = 0 when e = -inf)
__device__ __forceinline__ void spin_seed(const SpinTables& t, int m, int j, double& d, int& E) {
    const int mi = m + t.lmax;
    double e = t.lb2[mi];
    const int pc = t.pc[mi], ps = t.ps[mi];
    if (pc != 0) e += (double)pc * t.log2cos[j];
    if (ps != 0) e += (double)ps * t.log2sin[j];
    d = 0.0;
    E = 0;
    if (isfinite(e)) {
        const double Es = ceil(e);
        d = t.sg[mi] * exp2(e - Es);
        E = (int)Es;
    }
}

template <int R>
__device__ void spin_fwd_item(const SpinTables& t, const RingOut& o, const RingItem& item,
                              const double2* __restrict__ alm, double2* __restrict__ out, int b,
                              SpinFwdSmem& sm, int lane) {
    const int m = item.m, L = t.lmax, n = -t.spin;
    const int l0 = max(abs(m), abs(n));
    const double2* ab = alm + (size_t)(L + 1) * (2 * L + 1) * b;
    double x[R], d1[R], d0[R];
    double2 acc[R];
    int E[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        x[r] = 0.0;
        d1[r] = d0[r] = 0.0;
        E[r] = 0;
        acc[r] = make_double2(0.0, 0.0);
        if (k < item.n) {
            x[r] = t.cos_t[item.j0 + k];
            spin_seed(t, m, item.j0 + k, d1[r], E[r]);
        }
    }
    {
        const double N0 = t.lt[l0].w;
        const double2 a = ab[sidx(l0, m, L)];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            acc[r].x = a.x * N0 * d1[r];
            acc[r].y = a.y * N0 * d1[r];
        }
    }
    auto step = [&](int i) {
        const double a1 = sm.a1[i], a2 = sm.a2[i], a0 = sm.a0[i];
        const double2 a = sm.a[i];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double dn = fma(fma(a1, x[r], -a2), d1[r], -(a0 * d0[r]));
            d0[r] = d1[r];
            d1[r] = dn;
            acc[r].x = fma(a.x, dn, acc[r].x);
            acc[r].y = fma(a.y, dn, acc[r].y);
        }
    };
    // the coefficients a_{lm} of the next 32 degrees are loaded while this chunk runs
    double2 a_next = make_double2(0.0, 0.0);
    if (l0 + 1 + lane <= L) a_next = ab[sidx(l0 + 1 + lane, m, L)];
    for (int lb = l0 + 1; lb <= L; lb += 32) {
        const int nl = min(32, L - lb + 1);
        __syncwarp();
        if (lane < nl) {
            const SpinCoef c = spin_coef(t.lt, lb + lane, m, n);
            sm.a1[lane] = c.a1;
            sm.a2[lane] = c.a2;
            sm.a0[lane] = c.a0;
            sm.a[lane] = make_double2(a_next.x * c.N, a_next.y * c.N);
        }
        __syncwarp();
        if (lb + 32 + lane <= L) a_next = ab[sidx(lb + 32 + lane, m, L)];
        if (nl == 32) {
#pragma unroll kSpinFwdUnroll
            for (int i = 0; i < 32; ++i) step(i);
        } else {
            for (int i = 0; i < nl; ++i) step(i);
        }
        // renormalise every 32 degrees (exact powers of two)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int sh = spin_renorm_shift(d1[r], d0[r]);
            if (sh != 0) {
                const double f = scalbn(1.0, -sh);
                d1[r] *= f;
                d0[r] *= f;
                acc[r].x *= f;
                acc[r].y *= f;
                E[r] += sh;
            }
        }
    }
    const double smir = o.spin_sgn * ((m & 1) ? -1.0 : 1.0);
    double2* ob = out + o.bstride * b;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        if (k >= item.n) continue;
        const int j = item.j0 + k;
        const double sc = scalbn(t.w ? t.w[j] : 1.0, E[r]);
        const double2 g = make_double2(acc[r].x * sc, acc[r].y * sc);
        ob[j + o.ld * (o.col_off + m)] = g;
        if (o.reflect) ob[(o.nrows - 1 - j) + o.ld * (o.col_off + m)] = make_double2(g.x * smir, g.y * smir);
    }
}

__global__ void __launch_bounds__(kSpinWarps * 32)
spin_fwd_kernel(SpinTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const int* __restrict__ jlo, const int* __restrict__ jhi, const double2* __restrict__ alm,
                void* const* __restrict__ ptrs, int ptr, double2* __restrict__ out, int B) {
    __shared__ SpinFwdSmem sm[kSpinWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kSpinWarps + warp;
    if (it >= nitems) return;
    // in a batch the coefficient array is read from the batch's pointer table
    if (ptrs) alm = static_cast<const double2*>(ptrs[ptr]);
    const RingItem item = items[it];
    const int m = item.m, am = abs(m);
    for (int b = 0; b < B; ++b) {
        // zeros for the rings the order does not retain (first tile of the order)
        if ((item.flags & kItemFirst) && o.zero_rest) {
            double2* ob = out + o.bstride * b;
            const double2 z = make_double2(0.0, 0.0);
            for (int j = lane; j < o.nrings_out; j += 32) {
                if (j >= jlo[am] && j <= jhi[am]) continue;
                ob[j + o.ld * (o.col_off + m)] = z;
                if (o.reflect) ob[(o.nrows - 1 - j) + o.ld * (o.col_off + m)] = z;
            }
        }
        const int reff = (item.n + 31) >> 5;
        if (reff >= 3) spin_fwd_item<4>(t, o, item, alm, out, b, sm[warp], lane);
        else if (reff == 2) spin_fwd_item<2>(t, o, item, alm, out, b, sm[warp], lane);
        else spin_fwd_item<1>(t, o, item, alm, out, b, sm[warp], lane);
    }
}

struct SpinAdjSmem {
    SpinCoef c[32];
    double2 red[32][33];
};

template <int R>
__device__ void spin_adj_item(const SpinTables& t, const RingOut& o, const RingItem& item,
                              const double2* __restrict__ in, double* __restrict__ almd, int b,
                              SpinAdjSmem& sm, int lane) {
    const int m = item.m, L = t.lmax, n = -t.spin;
    const int l0 = max(abs(m), abs(n));
    const double smir = o.spin_sgn * ((m & 1) ? -1.0 : 1.0);
    const double2* ib = in + o.bstride * b;
    double* ad = almd + 2 * (size_t)(L + 1) * (2 * L + 1) * b;
    double x[R], d1[R], d0[R];
    double2 g[R], gs[R];  // folded ring value; scaled by window and 2^E
    int E[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        x[r] = 0.0;
        d1[r] = d0[r] = 0.0;
        E[r] = 0;
        g[r] = gs[r] = make_double2(0.0, 0.0);
        if (k < item.n) {
            const int j = item.j0 + k;
            x[r] = t.cos_t[j];
            spin_seed(t, m, j, d1[r], E[r]);
            double2 v = ib[j + o.ld * (o.col_off + m)];
            if (o.reflect) {
                const double2 u = ib[(o.nrows - 1 - j) + o.ld * (o.col_off + m)];
                v.x += smir * u.x;
                v.y += smir * u.y;
            }
            const double w = t.w ? t.w[j] : 1.0;
            g[r] = make_double2(v.x * w, v.y * w);
            gs[r] = make_double2(scalbn(g[r].x, E[r]), scalbn(g[r].y, E[r]));
        }
    }
    // degree l0: reduce now
    {
        double2 p = make_double2(0.0, 0.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            p.x = fma(d1[r], gs[r].x, p.x);
            p.y = fma(d1[r], gs[r].y, p.y);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            p.x += __shfl_xor_sync(0xffffffffu, p.x, off);
            p.y += __shfl_xor_sync(0xffffffffu, p.y, off);
        }
        if (lane == 0) {
            const double N0 = t.lt[l0].w;
            atomicAdd(ad + 2 * sidx(l0, m, L), p.x * N0);
            atomicAdd(ad + 2 * sidx(l0, m, L) + 1, p.y * N0);
        }
    }
    auto step = [&](int i) {
        const SpinCoef c = sm.c[i];
        double2 p = make_double2(0.0, 0.0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double dn = fma(fma(c.a1, x[r], -c.a2), d1[r], -(c.a0 * d0[r]));
            d0[r] = d1[r];
            d1[r] = dn;
            p.x = fma(dn, gs[r].x, p.x);
            p.y = fma(dn, gs[r].y, p.y);
        }
        sm.red[i][lane] = p;
    };
    for (int lb = l0 + 1; lb <= L; lb += 32) {
        const int nl = min(32, L - lb + 1);
        __syncwarp();
        if (lane < nl) sm.c[lane] = spin_coef(t.lt, lb + lane, m, n);
        __syncwarp();
        if (nl == 32) {
#pragma unroll 8
            for (int i = 0; i < 32; ++i) step(i);
        } else {
            for (int i = 0; i < nl; ++i) step(i);
        }
        __syncwarp();
        if (lane < nl) {
            double sx0 = 0.0, sy0 = 0.0, sx1 = 0.0, sy1 = 0.0;
#pragma unroll 8
            for (int q = 0; q < 32; q += 2) {
                const double2 v0 = sm.red[lane][q], v1 = sm.red[lane][q + 1];
                sx0 += v0.x;
                sy0 += v0.y;
                sx1 += v1.x;
                sy1 += v1.y;
            }
            const double N = sm.c[lane].N;
            const size_t e = 2 * sidx(lb + lane, m, L);
            if (item.flags & kItemSole) {
                ad[e] = (sx0 + sx1) * N;
                ad[e + 1] = (sy0 + sy1) * N;
            } else {
                atomicAdd(ad + e, (sx0 + sx1) * N);
                atomicAdd(ad + e + 1, (sy0 + sy1) * N);
            }
        }
        // renormalise every 32 degrees (exact powers of two); the scaled ring values follow E
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int sh = spin_renorm_shift(d1[r], d0[r]);
            if (sh != 0) {
                const double f = scalbn(1.0, -sh);
                d1[r] *= f;
                d0[r] *= f;
                E[r] += sh;
                gs[r] = make_double2(scalbn(g[r].x, E[r]), scalbn(g[r].y, E[r]));
            }
        }
    }
}

__global__ void __launch_bounds__(kSpinAdjWarps * 32)
spin_adj_kernel(SpinTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const double2* __restrict__ in, double* __restrict__ almd, void* const* __restrict__ ptrs,
                int ptr, int B) {
    __shared__ SpinAdjSmem sm[kSpinAdjWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kSpinAdjWarps + warp;
    if (it >= nitems) return;
    if (ptrs) almd = static_cast<double*>(ptrs[ptr]);
    const RingItem item = items[it];
    for (int b = 0; b < B; ++b) {
        const int reff = (item.n + 31) >> 5;
        if (reff >= 3) spin_adj_item<4>(t, o, item, in, almd, b, sm[warp], lane);
        else if (reff == 2) spin_adj_item<2>(t, o, item, in, almd, b, sm[warp], lane);
        else spin_adj_item<1>(t, o, item, in, almd, b, sm[warp], lane);
    }
}

}  // namespace

int build_spin_items(const std::vector<int>& jlo, const std::vector<int>& jhi, int lmax, int spin,
                     int rings_per_tile, RingItemsOwner& own, cudaStream_t s) {
    std::vector<RingItem> items;
    std::vector<int64_t> cost;
    const int L = lmax;
    for (int m = -L; m <= L; ++m) {
        const int am = std::abs(m);
        const int l0 = std::max(am, std::abs(spin));
        if (l0 > L || jlo[am] > jhi[am]) continue;
        const int lo = jlo[am], hi = jhi[am];
        const int ntile = (hi - lo + rings_per_tile) / rings_per_tile;
        for (int q = 0; q < ntile; ++q) {
            const int j0 = lo + q * rings_per_tile;
            const int nn = std::min(rings_per_tile, hi - j0 + 1);
            int flags = (q == 0 ? kItemFirst : 0) | (ntile == 1 ? kItemSole : 0);
            items.push_back(RingItem{m, j0, nn, flags, l0, L, -1, 0});
            cost.push_back((int64_t)nn * (L - l0 + 1));
        }
    }
    // heaviest first
    std::vector<int> ord(items.size());
    for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int)i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    own.host.resize(items.size());
    for (size_t i = 0; i < ord.size(); ++i) own.host[i] = items[ord[i]];
    PF_TRY(own.items.alloc(sizeof(RingItem) * std::max<size_t>(own.host.size(), 1)));
    if (!own.host.empty())
        PF_CUDA(cudaMemcpyAsync(own.items.p, own.host.data(), sizeof(RingItem) * own.host.size(),
                                cudaMemcpyHostToDevice, s));
    PF_TRY(own.jlo.alloc(sizeof(int) * (L + 1)));
    PF_TRY(own.jhi.alloc(sizeof(int) * (L + 1)));
    PF_CUDA(cudaMemcpyAsync(own.jlo.p, jlo.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(own.jhi.p, jhi.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, s));
    own.view.items = own.items.as<RingItem>();
    own.view.nitems = (int)own.host.size();
    own.view.rmax = std::max(1, rings_per_tile / 32);
    own.view.jlo = own.jlo.as<int>();
    own.view.jhi = own.jhi.as<int>();
    PF_CUDA(cudaStreamSynchronize(s));
    return 0;
}

int spin_ring_forward(const SpinTables& t, const RingOut& o, const RingItems& it, const double2* alm,
                      double2* out, int B, cudaStream_t s) {
    if (it.nitems == 0) return 0;
    spin_fwd_kernel<<<(it.nitems + kSpinWarps - 1) / kSpinWarps, kSpinWarps * 32, 0, s>>>(
        t, o, it.items, it.nitems, it.jlo, it.jhi, alm, nullptr, 0, out, B);
    return check_launch("spin_fwd_kernel");
}

int spin_ring_forward_ptr(const SpinTables& t, const RingOut& o, const RingItems& it,
                          void* const* ptrs, int ptr, double2* out, int B, cudaStream_t s) {
    if (it.nitems == 0) return 0;
    spin_fwd_kernel<<<(it.nitems + kSpinWarps - 1) / kSpinWarps, kSpinWarps * 32, 0, s>>>(
        t, o, it.items, it.nitems, it.jlo, it.jhi, nullptr, ptrs, ptr, out, B);
    return check_launch("spin_fwd_kernel");
}

int spin_ring_adjoint(const SpinTables& t, const RingOut& o, const RingItems& it, const double2* in,
                      double2* alm, int B, cudaStream_t s, bool clear) {
    // the adjoint overwrites alm: clear it, then every (l, m) the walk reaches is added
    if (clear)
        PF_CUDA(cudaMemsetAsync(alm, 0, sizeof(double2) * (size_t)(t.lmax + 1) * (2 * t.lmax + 1) * B, s));
    if (it.nitems == 0) return 0;
    spin_adj_kernel<<<(it.nitems + kSpinAdjWarps - 1) / kSpinAdjWarps, kSpinAdjWarps * 32, 0, s>>>(
        t, o, it.items, it.nitems, in, reinterpret_cast<double*>(alm), nullptr, 0, B);
    return check_launch("spin_adj_kernel");
}

int spin_ring_adjoint_ptr(const SpinTables& t, const RingOut& o, const RingItems& it,
                          const double2* in, void* const* ptrs, int ptr, int B, cudaStream_t s) {
    if (it.nitems == 0) return 0;
    spin_adj_kernel<<<(it.nitems + kSpinAdjWarps - 1) / kSpinAdjWarps, kSpinAdjWarps * 32, 0, s>>>(
        t, o, it.items, it.nitems, in, nullptr, ptrs, ptr, B);
    return check_launch("spin_adj_kernel");
}

// plan-time spin tables (src/Spin.jl:197-245): ring cosines (sign-flipped when reflected), the
// half-angle logarithms (swapped when reflected) and the per-order seed tables
int build_spin_tables(const std::vector<double>& theta_rings, bool reflect, int lmax, int spin,
                      SpinTablesOwner& own, cudaStream_t s) {
    const int n = (int)theta_rings.size(), L = lmax, nm = 2 * lmax + 1;
    std::vector<double> c(n), l2c(n), l2s(n), lb2(nm), sg(nm);
    std::vector<int> pc(nm), ps(nm);
    const double csgn = reflect ? -1.0 : 1.0;
    for (int j = 0; j < n; ++j) {
        const double t = theta_rings[j];
        c[j] = csgn * std::cos(t);
        double ch = std::cos(t / 2), sh = std::fabs(std::sin(t / 2));
        if (reflect) std::swap(ch, sh);
        l2c[j] = ch > 0 ? std::log2(ch) : -INFINITY;
        l2s[j] = sh > 0 ? std::log2(sh) : -INFINITY;
    }
    const int nn = -spin;
    const double inv_ln2 = 1.0 / std::log(2.0);
    for (int m = -L; m <= L; ++m) {
        const int idx = m + L;
        const int l0 = std::max(std::abs(m), std::abs(nn));
        if (l0 > L) {
            lb2[idx] = -INFINITY;
            pc[idx] = ps[idx] = 0;
            sg[idx] = 1.0;
            continue;
        }
        int a, b;
        double extra;
        if (std::abs(nn) == l0) {
            a = m;
            b = nn == l0 ? l0 : -l0;
            extra = 1.0;
        } else {
            a = nn;
            b = m == l0 ? l0 : -l0;
            extra = (((nn - m) % 2 + 2) % 2 == 1) ? -1.0 : 1.0;
        }
        double sgn;
        if (b == l0) {
            pc[idx] = l0 + a;
            ps[idx] = l0 - a;
            sgn = 1.0;
        } else {
            pc[idx] = l0 - a;
            ps[idx] = l0 + a;
            sgn = ((l0 - a) % 2 == 0) ? 1.0 : -1.0;
        }
        lb2[idx] = (std::lgamma(2.0 * l0 + 1) - std::lgamma((double)(l0 - a) + 1) -
                    std::lgamma((double)(l0 + a) + 1)) / 2 * inv_ln2;
        sg[idx] = sgn * extra;
    }
    auto up = [&](DevBuf& d, const void* h, size_t bytes) -> int {
        PF_TRY(d.alloc(std::max<size_t>(bytes, 8)));
        if (bytes) PF_CUDA(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, s));
        return 0;
    };
    PF_TRY(up(own.cos_t, c.data(), sizeof(double) * n));
    PF_TRY(up(own.log2cos, l2c.data(), sizeof(double) * n));
    PF_TRY(up(own.log2sin, l2s.data(), sizeof(double) * n));
    PF_TRY(up(own.lb2, lb2.data(), sizeof(double) * nm));
    PF_TRY(up(own.sg, sg.data(), sizeof(double) * nm));
    PF_TRY(up(own.pc, pc.data(), sizeof(int) * nm));
    PF_TRY(up(own.ps, ps.data(), sizeof(int) * nm));
    // per degree (1/sqrt(l^2 - n^2), sqrt(l^2 - n^2), 1/l, N_l); the first two only for l > |n|
    std::vector<double4> lt(L + 1);
    for (int l = 0; l <= L; ++l) {
        const double q = (double)l * l - (double)nn * nn;
        lt[l] = make_double4(q > 0 ? 1.0 / std::sqrt(q) : 0.0, q > 0 ? std::sqrt(q) : 0.0,
                             l > 0 ? 1.0 / l : 0.0, std::sqrt((2.0 * l + 1) / (4 * M_PI)));
    }
    PF_TRY(up(own.lt, lt.data(), sizeof(double4) * (L + 1)));
    PF_CUDA(cudaStreamSynchronize(s));
    own.t.cos_t = own.cos_t.as<double>();
    own.t.log2cos = own.log2cos.as<double>();
    own.t.log2sin = own.log2sin.as<double>();
    own.t.lb2 = own.lb2.as<double>();
    own.t.sg = own.sg.as<double>();
    own.t.pc = own.pc.as<int>();
    own.t.ps = own.ps.as<int>();
    own.t.lt = own.lt.as<double4>();
    own.t.lmax = L;
    own.t.spin = spin;
    own.t.nrings = n;
    return 0;
}

}  // namespace pf
