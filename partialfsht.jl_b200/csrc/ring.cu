// Ring pass of the stretched leaf on sm_100a: rings_from_alm! and its exact transpose
// alm_from_rings! (PartialFSHT.jl src/Legendre.jl:310-542; device analogue of
// ext/PartialFSHTKernelAbstractionsExt.jl:86-230).
//
// Work decomposition: one warp per item (order m, tile of consecutive retained rings); a
// lane owns R rings (ring j0 + lane + 32 r, R = ceil(tile / 32) chosen per item) and keeps
// their two-term recurrence state and block-scaling exponent in registers. The recurrence
// is the reference's
//     P_m^m = (-1)^m 2^(m log2 sin + log2 c_m),   P_{m+1}^m = sqrt(2m+3) cos P_m^m,
//     P_l^m = a_l^m cos P_{l-1}^m - b_l^m P_{l-2}^m
// renormalised every 64 degrees (src/Legendre.jl:16,455-459). Each ring keeps its own
// exponent (as the KernelAbstractions kernel does), so no chunk headroom rule is needed.
// a_l^m, b_l^m come from a plan-time table built on the device with the reference's exact
// expressions. Per chunk of 32 degrees a warp stages them and the coefficients a_{l,+-m}
// in shared memory; the chunk is walked in fixed, fully unrolled blocks of degrees with no
// branch inside a block, so successive degrees overlap in the pipeline; renormalisation
// falls on block boundaries because 64 is a multiple of the block.
//
// Forward: acc(ring, +-m) += a_{l,+-m} P_l^m, written once per ring, windowed and, for a
// pole/full periodisation, mirrored into the DFS row with sign (-1)^m (src/DFS.jl:26). The
// first tile of each order also writes the zeros of the rings the order does not retain.
// Adjoint: each lane sums P_l^m g_j over its R rings; per block of degrees the lanes' partial
// sums are transposed through shared memory and each lane reduces one (degree, component)
// over the 32 lanes. An order covered by a single tile stores its coefficients; an order
// split over several tiles adds them atomically (into zeros).
#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace pf {

static constexpr int kWarpsPerBlock = 4;
static constexpr int kStride = 64;  // _RESCALE_STRIDE (src/Legendre.jl:16)

// ---------------------------------------------------------------------------------------
// recurrence coefficient table, exact expressions of src/Legendre.jl:406-408
// ---------------------------------------------------------------------------------------
__global__ void ab_table_kernel(int L, int mmax, const int64_t* __restrict__ aboff,
                                double2* __restrict__ ab) {
    const int m = blockIdx.y;
    if (m > mmax) return;
    const int n = L - m - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int l = m + 2 + i;
        const double a = sqrt((double)(2 * l - 1) * (double)(2 * l + 1) /
                              ((double)(l - m) * (double)(l + m)));
        const double b = sqrt((double)(2 * l + 1) / (double)(2 * l - 3) * (double)(l - m - 1) /
                              (double)(l - m) * (double)(l + m - 1) / (double)(l + m));
        ab[aboff[m] + i] = make_double2(a, b);
    }
}

int build_ab_table(int L, int mmax, DevBuf& ab, DevBuf& aboff, cudaStream_t s) {
    std::vector<int64_t> off(L + 1, 0);
    int64_t tot = 0;
    for (int m = 0; m <= L; ++m) {
        off[m] = tot;
        if (m <= mmax) tot += std::max(0, L - m - 1);
    }
    PF_TRY(aboff.alloc(sizeof(int64_t) * (L + 1)));
    PF_TRY(ab.alloc(sizeof(double2) * std::max<int64_t>(tot, 1)));
    PF_CUDA(cudaMemcpyAsync(aboff.p, off.data(), sizeof(int64_t) * (L + 1),
                            cudaMemcpyHostToDevice, s));
    if (tot > 0) {
        dim3 grid((unsigned)std::min(64, (L + 255) / 256 + 1), (unsigned)(mmax + 1));
        ab_table_kernel<<<grid, 256, 0, s>>>(L, mmax, aboff.as<int64_t>(), ab.as<double2>());
        PF_TRY(check_launch("ab_table_kernel"));
    }
    // the host vector must outlive the async copy
    PF_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// the coefficient-table kernel on caller-provided offsets and storage (no allocation)
int launch_ab_table(int L, int mmax, const int64_t* aboff, double2* ab, cudaStream_t s) {
    dim3 grid((unsigned)std::min(64, (L + 255) / 256 + 1), (unsigned)(mmax + 1));
    ab_table_kernel<<<grid, 256, 0, s>>>(L, mmax, aboff, ab);
    return check_launch("ab_table_kernel");
}

std::vector<RingItem> make_ring_items(const std::vector<int>& jlo, const std::vector<int>& jhi,
                                      int L, int mmax, int tile, const RingSegments* seg) {
    std::vector<RingItem> items;
    std::vector<int64_t> cost;
    for (int m = 0; m <= std::min(mmax, L); ++m) {
        int lo = jlo[m], hi = jhi[m];
        if (hi < lo) continue;
        const int ntiles = (hi - lo + tile) / tile;
        const int K = seg && seg->seg_degrees > 0 ? seg->nseg[m] : 1;
        for (int t = 0; t < ntiles; ++t) {
            const int j0 = lo + t * tile;
            const int n = std::min(tile, hi - j0 + 1);
            int flags = 0;
            if (t == 0) flags |= kItemFirst;
            if (ntiles == 1) flags |= kItemSole;
            for (int s = 0; s < K; ++s) {
                RingItem it = whole_item(m, j0, n, s == 0 ? flags : flags & ~kItemFirst, L);
                if (s > 0) {
                    it.lbeg = seg->seg_first(m, s);
                    it.ck = (int)(seg->ckbase[m] + (int64_t)(s - 1) * (hi - lo + 1) + (j0 - lo));
                }
                if (s + 1 < K) it.lend = seg->seg_first(m, s + 1) - 1;
                items.push_back(it);
                cost.push_back((int64_t)((n + 31) / 32) * (it.lend - it.lbeg + 1));
            }
        }
    }
    std::vector<size_t> idx(items.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<RingItem> out(items.size());
    for (size_t i = 0; i < idx.size(); ++i) out[i] = items[idx[i]];
    return out;
}

// ceil(log2(mx)) for finite mx > 0, exact (no transcendental)
__device__ __forceinline__ int ceil_log2(double mx) {
    int e;
    double f = frexp(mx, &e);
    return f == 0.5 ? e - 1 : e;
}

__device__ __forceinline__ double2 cmad(double2 acc, double2 a, double p) {
    acc.x = fma(a.x, p, acc.x);
    acc.y = fma(a.y, p, acc.y);
    return acc;
}

// seed of ring j for order m (src/Legendre.jl:379-382, exponent per ring as in
// ext/PartialFSHTKernelAbstractionsExt.jl:96-99)
__device__ __forceinline__ void ring_seed(const RingTables& t, int m, int j, double sgn,
                                          double& x, double& p2, int& E) {
    x = t.cos_t[j];
    const double e0 = m == 0 ? t.log2c[0] : (double)m * t.log2sin[j] + t.log2c[m];
    p2 = 0.0;
    E = 0;
    if (isfinite(e0)) {
        const double Es = ceil(e0);
        p2 = sgn * exp2(e0 - Es);
        E = (int)Es;
    }
}

__device__ __forceinline__ void ring_renorm(double& p1, double& p2, int& E) {
    const double mx = fmax(fabs(p1), fabs(p2));
    if (mx > 0.0 && isfinite(mx)) {
        const int s = ceil_log2(mx);
        if (s != 0) {
            const double f = scalbn(1.0, -s);
            p1 *= f;
            p2 *= f;
            E += s;
        }
    }
}

// ---------------------------------------------------------------------------------------
// plan-time recurrence checkpoints: one thread per (order, ring) walks the same recurrence
// and renormalisation schedule as the apply kernels and saves (P_{l-1}, P_{l-2}, E) at the
// first degree l of every later segment
// ---------------------------------------------------------------------------------------
struct CkptJob {
    int m, j0, n, nseg, nblk;
    int ck;        // checkpoint index of (segment 1, ring j0)
    int stride;    // between segments: retained rings of the order
    int pad_;
};

__global__ void ring_ckpt_kernel(RingTables t, const CkptJob* __restrict__ jobs,
                                 double2* __restrict__ ckp, int* __restrict__ ckE) {
    const CkptJob jb = jobs[blockIdx.x];
    const int k = threadIdx.x;
    if (k >= jb.n) return;
    const int m = jb.m, L = t.lmax, j = jb.j0 + k;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    double x, p1, p2;
    int E;
    ring_seed(t, m, j, sgn, x, p2, E);
    p1 = sqrt((double)(2 * m + 3)) * x * p2;
    const double2* abm = t.ab + t.aboff[m];
    int s = 1;
    int lnext = m + 2 + 64 * (int)(((int64_t)jb.nblk) / jb.nseg);
    int steps = 0;
    for (int l = m + 2; l <= L; ++l) {
        if (l == lnext) {
            const int64_t idx = jb.ck + (int64_t)(s - 1) * jb.stride + k;
            ckp[idx] = make_double2(p1, p2);
            ckE[idx] = E;
            if (++s == jb.nseg) break;
            lnext = m + 2 + 64 * (int)(((int64_t)s * jb.nblk) / jb.nseg);
        }
        const double2 ab = abm[l - m - 2];
        const double p = fma(ab.x * x, p1, -(ab.y * p2));
        p2 = p1;
        p1 = p;
        if (++steps == kStride) {
            steps = 0;
            if (l < L) ring_renorm(p1, p2, E);
        }
    }
}

int build_ring_segments(const RingTables& t, const std::vector<int>& jlo,
                        const std::vector<int>& jhi, int L, int mmax, int seg_degrees,
                        int64_t max_bytes, RingSegments& seg, cudaStream_t s) {
    seg.nseg.assign(L + 1, 1);
    seg.nblk.assign(L + 1, 0);
    seg.ckbase.assign(L + 1, 0);
    seg.nstates = 0;
    seg.seg_degrees = 0;
    if (seg_degrees <= 0) return 0;
    const int q = std::max(1, (seg_degrees + 32) / 64);
    std::vector<CkptJob> jobs;
    int64_t tot = 0;
    for (int m = 0; m <= std::min(mmax, L); ++m) {
        const int nret = jhi[m] - jlo[m] + 1;
        const int nb = L >= m + 2 ? (L - m - 1 + 63) / 64 : 0;
        seg.nblk[m] = nb;
        const int K = std::max(1, std::min(nb, (nb + q / 2) / q));
        if (nret <= 0 || K <= 1) continue;
        seg.nseg[m] = K;
        seg.ckbase[m] = tot;
        for (int j0 = jlo[m]; j0 <= jhi[m]; j0 += 128)
            jobs.push_back(CkptJob{m, j0, std::min(128, jhi[m] - j0 + 1), K, nb,
                                   (int)(tot + (j0 - jlo[m])), nret, 0});
        tot += (int64_t)(K - 1) * nret;
    }
    if (jobs.empty()) return 0;
    if (tot * (int64_t)(sizeof(double2) + sizeof(int)) > max_bytes || tot > INT32_MAX) {
        seg.nseg.assign(L + 1, 1);
        return 0;
    }
    DevBuf djobs;
    PF_TRY(djobs.alloc(sizeof(CkptJob) * jobs.size()));
    PF_TRY(seg.ck_p.alloc(sizeof(double2) * tot));
    PF_TRY(seg.ck_E.alloc(sizeof(int) * tot));
    PF_CUDA(cudaMemcpyAsync(djobs.p, jobs.data(), sizeof(CkptJob) * jobs.size(),
                            cudaMemcpyHostToDevice, s));
    ring_ckpt_kernel<<<(unsigned)jobs.size(), 128, 0, s>>>(t, djobs.as<CkptJob>(),
                                                           seg.ck_p.as<double2>(),
                                                           seg.ck_E.as<int>());
    PF_TRY(check_launch("ring_ckpt_kernel"));
    PF_CUDA(cudaStreamSynchronize(s));
    seg.nstates = tot;
    seg.seg_degrees = seg_degrees;
    return 0;
}

// ---------------------------------------------------------------------------------------
// forward: alm -> ring columns
// ---------------------------------------------------------------------------------------
template <int NB>
struct FwdSmem {
    double2 ab[kWarpsPerBlock][32];
    double2 ap[kWarpsPerBlock][NB][32];
    double2 am[kWarpsPerBlock][NB][32];
};

template <int R, int NB>
__device__ __forceinline__ void ring_fwd_item(const RingTables& t, const RingOut& o,
                                              const RingItem& item, const double2* __restrict__ alm,
                                              double2* __restrict__ out, int b0, FwdSmem<NB>& sm,
                                              int warp, int lane) {
    const int m = item.m, L = t.lmax;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    const int64_t albs = (int64_t)(L + 1) * (2 * L + 1);
    const double2* colp = alm + albs * b0 + (int64_t)(L + 1) * (2 * m);
    const double2* colm = alm + albs * b0 + (int64_t)(L + 1) * (m > 0 ? 2 * m - 1 : 0);
    const double2* abm = t.ab + t.aboff[m];
    const double2 zero2 = make_double2(0.0, 0.0);

    double x[R], p1[R], p2[R];
    int E[R];
    double2 accp[R][NB], accm[R][NB];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        x[r] = 0.0;
        p1[r] = 0.0;
        p2[r] = 0.0;
        E[r] = 0;
        if (k < item.n) ring_seed(t, m, item.j0 + k, sgn, x[r], p2[r], E[r]);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            accp[r][b] = zero2;
            accm[r][b] = zero2;
        }
    }
    // l = m: P = seed
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const double2 ap = colp[albs * b];
        double2 am = m > 0 ? colm[albs * b] : zero2;
        am.x *= sgn;
        am.y *= sgn;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            accp[r][b] = cmad(accp[r][b], ap, p2[r]);
            accm[r][b] = cmad(accm[r][b], am, p2[r]);
        }
    }
    if (m < L) {
        const double s23 = sqrt((double)(2 * m + 3));
#pragma unroll
        for (int r = 0; r < R; ++r) p1[r] = s23 * x[r] * p2[r];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double2 ap = colp[1 + albs * b];
            double2 am = m > 0 ? colm[1 + albs * b] : zero2;
            am.x *= sgn;
            am.y *= sgn;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                accp[r][b] = cmad(accp[r][b], ap, p1[r]);
                accm[r][b] = cmad(accm[r][b], am, p1[r]);
            }
        }
        auto step = [&](int i) {
            const double2 ab = sm.ab[warp][i];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double p = fma(ab.x * x[r], p1[r], -(ab.y * p2[r]));
                p2[r] = p1[r];
                p1[r] = p;
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const double2 ap = sm.ap[warp][b][i];
                const double2 am = sm.am[warp][b][i];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    accp[r][b] = cmad(accp[r][b], ap, p1[r]);
                    accm[r][b] = cmad(accm[r][b], am, p1[r]);
                }
            }
        };
        int steps = 0;
        // the coefficients of the next 32 degrees are loaded while this chunk runs
        double2 ab_n = zero2, ap_n[NB], am_n[NB];
        auto fetch = [&](int l) {
            if (l <= L) {
                ab_n = abm[l - m - 2];
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    ap_n[b] = colp[(l - m) + albs * b];
                    am_n[b] = m > 0 ? colm[(l - m) + albs * b] : zero2;
                }
            }
        };
#pragma unroll
        for (int b = 0; b < NB; ++b) ap_n[b] = am_n[b] = zero2;
        fetch(m + 2 + lane);
        for (int l0 = m + 2; l0 <= L; l0 += 32) {
            const int nl = min(32, L - l0 + 1);
            __syncwarp();
            if (lane < nl) {
                sm.ab[warp][lane] = ab_n;
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    sm.ap[warp][b][lane] = ap_n[b];
                    sm.am[warp][b][lane] = make_double2(am_n[b].x * sgn, am_n[b].y * sgn);
                }
            }
            __syncwarp();
            fetch(l0 + 32 + lane);
            const int nblk = nl >> 3;
            for (int blk = 0; blk < nblk; ++blk) {
#pragma unroll
                for (int i = 0; i < 8; ++i) step(blk * 8 + i);
                steps += 8;
                if (steps == kStride) {
                    steps = 0;
                    if (l0 + blk * 8 + 7 < L) {
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            const double mx = fmax(fabs(p1[r]), fabs(p2[r]));
                            if (mx > 0.0 && isfinite(mx)) {
                                const int s = ceil_log2(mx);
                                if (s != 0) {
                                    const double f = scalbn(1.0, -s);
                                    p1[r] *= f;
                                    p2[r] *= f;
#pragma unroll
                                    for (int b = 0; b < NB; ++b) {
                                        accp[r][b].x *= f;
                                        accp[r][b].y *= f;
                                        accm[r][b].x *= f;
                                        accm[r][b].y *= f;
                                    }
                                    E[r] += s;
                                }
                            }
                        }
                    }
                }
            }
            for (int i = nblk * 8; i < nl; ++i) step(i);
        }
    }
    // write the ring columns (window and 2^E folded into one exact scale)
    const double smir = o.spin_sgn * sgn;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        if (k >= item.n) continue;
        const int j = item.j0 + k;
        const double sc = scalbn(t.w ? t.w[j] : 1.0, E[r]);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            double2* ob = out + o.bstride * (b0 + b);
            const double2 gp = make_double2(accp[r][b].x * sc, accp[r][b].y * sc);
            const double2 gm = make_double2(accm[r][b].x * sc, accm[r][b].y * sc);
            ob[j + o.ld * (o.col_off + m)] = gp;
            if (m > 0) ob[j + o.ld * (o.col_off - m)] = gm;
            if (o.reflect) {
                const int jj = o.nrows - 1 - j;
                ob[jj + o.ld * (o.col_off + m)] = make_double2(gp.x * smir, gp.y * smir);
                if (m > 0) ob[jj + o.ld * (o.col_off - m)] = make_double2(gm.x * smir, gm.y * smir);
            }
        }
    }
}

// zeros in the order's columns for the rings it does not retain (first tile only)
template <int NB>
__device__ __forceinline__ void ring_fwd_zero_rest(const RingOut& o, const RingItem& item,
                                                   int lo, int hi, double2* __restrict__ out,
                                                   int b0, int lane) {
    const int m = item.m;
    const double2 z = make_double2(0.0, 0.0);
    for (int b = 0; b < NB; ++b) {
        double2* ob = out + o.bstride * (b0 + b);
        for (int j = lane; j < o.nrings_out; j += 32) {
            if (j >= lo && j <= hi) continue;
            ob[j + o.ld * (o.col_off + m)] = z;
            if (m > 0) ob[j + o.ld * (o.col_off - m)] = z;
            if (o.reflect) {
                const int jj = o.nrows - 1 - j;
                ob[jj + o.ld * (o.col_off + m)] = z;
                if (m > 0) ob[jj + o.ld * (o.col_off - m)] = z;
            }
        }
    }
}

template <int RMAX, int NB>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
ring_fwd_kernel(RingTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const int* __restrict__ jlo, const int* __restrict__ jhi,
                const double2* __restrict__ alm, double2* __restrict__ out, int b0) {
    __shared__ FwdSmem<NB> sm;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kWarpsPerBlock + warp;
    if (it >= nitems) return;
    const RingItem item = items[it];
    if ((item.flags & kItemFirst) && o.zero_rest)
        ring_fwd_zero_rest<NB>(o, item, jlo[item.m], jhi[item.m], out, b0, lane);
    for (int base = 0; base < item.n; base += 32 * RMAX) {
        RingItem sub = item;
        sub.j0 = item.j0 + base;
        sub.n = min(32 * RMAX, item.n - base);
        const int reff = (sub.n + 31) >> 5;
        if (RMAX >= 4 && reff >= 3) ring_fwd_item<(RMAX >= 4 ? 4 : 1), NB>(t, o, sub, alm, out, b0, sm, warp, lane);
        else if (RMAX >= 2 && reff == 2) ring_fwd_item<(RMAX >= 2 ? 2 : 1), NB>(t, o, sub, alm, out, b0, sm, warp, lane);
        else ring_fwd_item<1, NB>(t, o, sub, alm, out, b0, sm, warp, lane);
    }
}

// ---------------------------------------------------------------------------------------
// adjoint: ring columns -> alm
// ---------------------------------------------------------------------------------------
// Two warps per block. With kAdjPipelined each warp double-buffers its reduction area, so
// one block's partial sums are reduced while the next block's degrees are computed; without
// it a block is reduced as soon as it is staged (half the shared memory per warp).
static constexpr int kAdjWarps = 2;
static constexpr bool kAdjPipelined = false;
#ifdef PF_ADJ_MIN_BLOCKS
#define PF_ADJ_BOUNDS __launch_bounds__(kAdjWarps * 32, PF_ADJ_MIN_BLOCKS)
#else
#define PF_ADJ_BOUNDS __launch_bounds__(kAdjWarps * 32)
#endif
struct AdjSmem {
    double red[kAdjWarps][kAdjPipelined ? 2 : 1][32][33];
    double2 ab[kAdjWarps][32];
};

template <int R, int NB>
__device__ __forceinline__ void ring_adj_item(const RingTables& t, const RingOut& o,
                                              const RingItem& item, const double2* __restrict__ in,
                                              double* __restrict__ almd, int b0, bool sole,
                                              AdjSmem& sm, int warp, int lane) {
    constexpr int NV = 4 * NB;   // (+m re, +m im, -m re, -m im) per transform
    constexpr int LB = 32 / NV;  // degrees per reduction block
    const int m = item.m, L = t.lmax;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    const double smir = o.spin_sgn * sgn;
    const int64_t albs = (int64_t)(L + 1) * (2 * L + 1);
    const double2* abm = t.ab + t.aboff[m];
    const int64_t cp = (int64_t)(L + 1) * (2 * m);
    const int64_t cm = (int64_t)(L + 1) * (m > 0 ? 2 * m - 1 : 0);

    double x[R], p1[R], p2[R];
    int E[R];
    double2 gp[R][NB], gm[R][NB];
    // ring data for (ring r, transform b): folded, windowed, scaled by 2^E; the -m column
    // carries the (-1)^m of src/Legendre.jl:511
    auto load_g = [&](int r) {
        const int k = lane + 32 * r;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            gp[r][b] = make_double2(0.0, 0.0);
            gm[r][b] = make_double2(0.0, 0.0);
        }
        if (k >= item.n) return;
        const int j = item.j0 + k;
        const double sc = scalbn(t.w ? t.w[j] : 1.0, E[r]);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double2* ib = in + o.bstride * (b0 + b);
            double2 v = ib[j + o.ld * (o.col_off + m)];
            if (o.reflect) {
                const double2 u = ib[(o.nrows - 1 - j) + o.ld * (o.col_off + m)];
                v.x += smir * u.x;
                v.y += smir * u.y;
            }
            gp[r][b] = make_double2(v.x * sc, v.y * sc);
            if (m > 0) {
                double2 u = ib[j + o.ld * (o.col_off - m)];
                if (o.reflect) {
                    const double2 q = ib[(o.nrows - 1 - j) + o.ld * (o.col_off - m)];
                    u.x += smir * q.x;
                    u.y += smir * q.y;
                }
                gm[r][b] = make_double2(u.x * sc * sgn, u.y * sc * sgn);
            }
        }
    };
    const bool seeded = item.ck < 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        x[r] = 0.0;
        p1[r] = 0.0;
        p2[r] = 0.0;
        E[r] = 0;
        if (k < item.n) {
            if (seeded) {
                ring_seed(t, m, item.j0 + k, sgn, x[r], p2[r], E[r]);
            } else {
                x[r] = t.cos_t[item.j0 + k];
                const double2 c = t.ck_p[item.ck + k];
                p1[r] = c.x;
                p2[r] = c.y;
                E[r] = t.ck_E[item.ck + k];
            }
        }
        load_g(r);
    }
    int cur = 0;     // reduction buffer the current block stages into
    int pend = -1;   // first degree of the block waiting in buffer cur ^ 1 (-1: none)
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;  // this lane's sums of the pending block
    // partial sums over this lane's rings for degree slot `slot`
    auto stage = [&](const double (&P)[R], int slot) {
        double part[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) part[v] = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                part[4 * b + 0] = fma(P[r], gp[r][b].x, part[4 * b + 0]);
                part[4 * b + 1] = fma(P[r], gp[r][b].y, part[4 * b + 1]);
                part[4 * b + 2] = fma(P[r], gm[r][b].x, part[4 * b + 2]);
                part[4 * b + 3] = fma(P[r], gm[r][b].y, part[4 * b + 3]);
            }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.red[warp][kAdjPipelined ? cur : 0][slot * NV + v][lane] = part[v];
    };
    // lane's output (degree lfirst + lane / NV, component lane % NV) of a reduced block
    auto write_out = [&](int lfirst, double s) {
        const int li = lane / NV, v = lane % NV;
        const int l = lfirst + li;
        const int b = v >> 2, comp = v & 3;
        if (comp < 2 || m > 0) {
            const int64_t idx = (l - m) + (comp < 2 ? cp : cm) + albs * (b0 + b);
            double* dst = almd + 2 * idx + (comp & 1);
            if (sole) *dst = s;
            else atomicAdd(dst, s);
        }
    };
    // reduce the staged degrees [lfirst, lfirst + cnt) of buffer cur over the lanes at once
    auto flush = [&](int lfirst, int cnt) {
        __syncwarp();
        if (lane < cnt * NV) {
            // four independent partial sums: the chain of dependent adds is 8 long, not 32
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
            for (int q = 0; q < 32; q += 4) {
                s0 += sm.red[warp][kAdjPipelined ? cur : 0][lane][q];
                s1 += sm.red[warp][kAdjPipelined ? cur : 0][lane][q + 1];
                s2 += sm.red[warp][kAdjPipelined ? cur : 0][lane][q + 2];
                s3 += sm.red[warp][kAdjPipelined ? cur : 0][lane][q + 3];
            }
            write_out(lfirst, (s0 + s1) + (s2 + s3));
        }
        __syncwarp();
    };
    // NV of the pending block's 32 values, read while degree slot i of the next block runs
    auto drain = [&](int i) {
#pragma unroll
        for (int k = 0; k < NV; k += 4) {
            const double* rowp = &sm.red[warp][kAdjPipelined ? cur ^ 1 : 0][lane][i * NV + k];
            a0 += rowp[0];
            a1 += rowp[1];
            a2 += rowp[2];
            a3 += rowp[3];
        }
    };
    auto finish = [&]() {
        write_out(pend, (a0 + a1) + (a2 + a3));
        a0 = a1 = a2 = a3 = 0.0;
        pend = -1;
    };
    int lstart = item.lbeg;
    if (seeded) {
        stage(p2, 0);  // l = m
        if (m == L) {
            flush(m, 1);
            return;
        }
        const double s23 = sqrt((double)(2 * m + 3));
#pragma unroll
        for (int r = 0; r < R; ++r) p1[r] = s23 * x[r] * p2[r];
        stage(p1, 1);  // l = m + 1
        flush(m, 2);
        lstart = m + 2;
    }
    {
        auto rec = [&](int i) {
            const double2 ab = sm.ab[warp][i];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double p = fma(ab.x * x[r], p1[r], -(ab.y * p2[r]));
                p2[r] = p1[r];
                p1[r] = p;
            }
        };
        // segments start on the renormalisation schedule, so the count restarts at 0
        int steps = 0;
        // the coefficients of the next 32 degrees are loaded while this chunk runs
        double2 ab_next = make_double2(0.0, 0.0);
        if (lstart <= item.lend && lane <= item.lend - lstart) ab_next = abm[lstart + lane - m - 2];
        for (int l0 = lstart; l0 <= item.lend; l0 += 32) {
            const int nl = min(32, item.lend - l0 + 1);
            __syncwarp();
            if (lane < nl) sm.ab[warp][lane] = ab_next;
            __syncwarp();
            if (l0 + 32 + lane <= item.lend) ab_next = abm[l0 + 32 + lane - m - 2];
            const int nblk = nl / LB;
            for (int blk = 0; blk < nblk; ++blk) {
                if (!kAdjPipelined) {
#pragma unroll
                    for (int i = 0; i < LB; ++i) {
                        rec(blk * LB + i);
                        stage(p1, i);
                    }
                    flush(l0 + blk * LB, LB);
                } else if (pend >= 0) {
#pragma unroll
                    for (int i = 0; i < LB; ++i) {
                        rec(blk * LB + i);
                        stage(p1, i);
                        drain(i);
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < LB; ++i) {
                        rec(blk * LB + i);
                        stage(p1, i);
                    }
                }
                if (kAdjPipelined) {
                    // this block's sums are visible, and every lane is done with the other buffer
                    __syncwarp();
                    if (pend >= 0) finish();
                    pend = l0 + blk * LB;
                    cur ^= 1;
                }
                steps += LB;
                if (steps == kStride) {
                    steps = 0;
                    if (l0 + blk * LB + LB - 1 < L) {
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            const double mx = fmax(fabs(p1[r]), fabs(p2[r]));
                            if (mx > 0.0 && isfinite(mx)) {
                                const int s = ceil_log2(mx);
                                if (s != 0) {
                                    const double f = scalbn(1.0, -s);
                                    p1[r] *= f;
                                    p2[r] *= f;
                                    const int Eold = E[r];
                                    E[r] += s;
                                    if (Eold >= -900) {
                                        // the scaled ring data were normal: 2^s keeps them
                                        // exactly what a reload would give
                                        const double u = scalbn(1.0, s);
#pragma unroll
                                        for (int b = 0; b < NB; ++b) {
                                            gp[r][b].x *= u;
                                            gp[r][b].y *= u;
                                            gm[r][b].x *= u;
                                            gm[r][b].y *= u;
                                        }
                                    } else {
                                        load_g(r);
                                    }
                                }
                            }
                        }
                    }
                }
            }
            const int rem = nl - nblk * LB;
            if (rem > 0) {
                if (pend >= 0) {
#pragma unroll
                    for (int i = 0; i < LB; ++i) drain(i);
                    finish();
                }
                for (int i = 0; i < rem; ++i) {
                    rec(nblk * LB + i);
                    stage(p1, i);
                }
                flush(l0 + nblk * LB, rem);
            }
        }
        if (pend >= 0) {
#pragma unroll
            for (int i = 0; i < LB; ++i) drain(i);
            finish();
        }
    }
}

template <int RMAX, int NB>
__global__ void PF_ADJ_BOUNDS
ring_adj_kernel(RingTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const double2* __restrict__ in, double* __restrict__ almd, int b0, int allow_sole) {
    __shared__ AdjSmem sm;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kAdjWarps + warp;
    if (it >= nitems) return;
    const RingItem item = items[it];
    const bool multi = item.n > 32 * RMAX;
    const bool sole = allow_sole && (item.flags & kItemSole) && !multi;
    for (int base = 0; base < item.n; base += 32 * RMAX) {
        RingItem sub = item;
        sub.j0 = item.j0 + base;
        sub.n = min(32 * RMAX, item.n - base);
        if (sub.ck >= 0) sub.ck += base;
        const int reff = (sub.n + 31) >> 5;
        if (RMAX >= 8 && reff >= 5) ring_adj_item<(RMAX >= 8 ? 8 : 1), NB>(t, o, sub, in, almd, b0, sole, sm, warp, lane);
        else if (RMAX >= 4 && reff >= 3) ring_adj_item<(RMAX >= 4 ? 4 : 1), NB>(t, o, sub, in, almd, b0, sole, sm, warp, lane);
        else if (RMAX >= 2 && reff == 2) ring_adj_item<(RMAX >= 2 ? 2 : 1), NB>(t, o, sub, in, almd, b0, sole, sm, warp, lane);
        else ring_adj_item<1, NB>(t, o, sub, in, almd, b0, sole, sm, warp, lane);
    }
}

// zero what the adjoint does not overwrite: padding rows of every column, the orders the
// ring set does not retain, and the orders whose items add atomically
__global__ void alm_prepare_kernel(double2* __restrict__ alm, int L, int B,
                                   const unsigned char* __restrict__ sole_m, int allow_sole) {
    const int c = blockIdx.x;  // column
    const int b = blockIdx.y;
    const int am = (c + 1) / 2;
    double2* col = alm + (int64_t)(L + 1) * c + (int64_t)(L + 1) * (2 * L + 1) * b;
    const int first = (allow_sole && sole_m[am]) ? L - am + 1 : 0;
    for (int r = first + threadIdx.x; r <= L; r += blockDim.x) col[r] = make_double2(0.0, 0.0);
}

// ---------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------
template <int RMAX, int NB>
static int launch_fwd(const RingTables& t, const RingOut& o, const RingItem* items, int nitems,
                      const int* jlo, const int* jhi, const double2* alm, double2* out, int b0,
                      cudaStream_t s) {
    const int grid = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    ring_fwd_kernel<RMAX, NB><<<grid, kWarpsPerBlock * 32, 0, s>>>(t, o, items, nitems, jlo, jhi,
                                                                  alm, out, b0);
    return check_launch("ring_fwd_kernel");
}

template <int RMAX, int NB>
static int launch_adj(const RingTables& t, const RingOut& o, const RingItem* items, int nitems,
                      const double2* in, double2* alm, int b0, int allow_sole, cudaStream_t s) {
    const int grid = (nitems + kAdjWarps - 1) / kAdjWarps;
    ring_adj_kernel<RMAX, NB><<<grid, kAdjWarps * 32, 0, s>>>(
        t, o, items, nitems, in, reinterpret_cast<double*>(alm), b0, allow_sole);
    return check_launch("ring_adj_kernel");
}

int ring_forward(const RingTables& t, const RingOut& o, const RingItems& it, const double2* alm,
                 double2* out, int B, cudaStream_t s) {
    if (it.nitems <= 0) return 0;
    int b0 = 0;
    while (b0 < B) {
        const int rem = B - b0;
        if (rem >= 4) {
            PF_TRY((launch_fwd<1, 4>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            b0 += 4;
        } else if (rem >= 2) {
            PF_TRY((launch_fwd<2, 2>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            b0 += 2;
        } else {
            if (it.rmax >= 4) PF_TRY((launch_fwd<4, 1>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            else PF_TRY((launch_fwd<2, 1>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            b0 += 1;
        }
    }
    return 0;
}

int alm_prepare(double2* alm, int L, int B, const unsigned char* sole_m, int allow_sole,
                cudaStream_t s) {
    dim3 grid(2 * L + 1, B);
    alm_prepare_kernel<<<grid, 128, 0, s>>>(alm, L, B, sole_m, allow_sole);
    return check_launch("alm_prepare_kernel");
}

int ring_adjoint(const RingTables& t, const RingOut& o, const RingItems& it, const double2* in,
                 double2* alm, int B, cudaStream_t s) {
    // a single transform with the item's own tile shape stores sole orders directly; the
    // multi-transform kernels split items into passes and always add
    const int allow_sole = (B == 1 && it.rmax >= 2) ? 1 : 0;
    PF_TRY(alm_prepare(alm, t.lmax, B, it.sole_m, allow_sole, s));
    if (it.nitems <= 0) return 0;
    int b0 = 0;
    while (b0 < B) {
        const int rem = B - b0;
        if (rem >= 4) {
            PF_TRY((launch_adj<1, 4>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
            b0 += 4;
        } else if (rem >= 2) {
            PF_TRY((launch_adj<2, 2>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
            b0 += 2;
        } else {
            if (it.rmax >= 8) PF_TRY((launch_adj<8, 1>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
            else if (it.rmax >= 4) PF_TRY((launch_adj<4, 1>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
            else PF_TRY((launch_adj<2, 1>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
            b0 += 1;
        }
    }
    return 0;
}

// item lists of one ring set: tiles of 32 * rmax rings, the order flags, the device tables
int build_ring_items(const std::vector<int>& jlo, const std::vector<int>& jhi, int L, int mmax,
                     int rmax, RingItemsOwner& own, cudaStream_t s, const RingSegments* seg) {
    std::vector<RingItem> items = make_ring_items(jlo, jhi, L, mmax, 32 * rmax, seg);
    std::vector<unsigned char> sole(L + 1, 0);
    for (const RingItem& r : items)
        if (r.flags & kItemSole) sole[r.m] = 1;
    PF_TRY(own.items.alloc(sizeof(RingItem) * std::max<size_t>(items.size(), 1)));
    PF_TRY(own.sole.alloc(L + 1));
    PF_TRY(own.jlo.alloc(sizeof(int) * (L + 1)));
    PF_TRY(own.jhi.alloc(sizeof(int) * (L + 1)));
    if (!items.empty())
        PF_CUDA(cudaMemcpyAsync(own.items.p, items.data(), sizeof(RingItem) * items.size(),
                                cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(own.sole.p, sole.data(), L + 1, cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(own.jlo.p, jlo.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(own.jhi.p, jhi.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaStreamSynchronize(s));
    own.view.items = own.items.as<RingItem>();
    own.view.nitems = (int)items.size();
    own.view.rmax = rmax;
    own.view.sole_m = own.sole.as<unsigned char>();
    own.view.jlo = own.jlo.as<int>();
    own.view.jhi = own.jhi.as<int>();
    return 0;
}

}  // namespace pf
