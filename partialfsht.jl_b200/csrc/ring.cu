// Ring pass of the stretched leaf on sm_100a: rings_from_alm! and its exact transpose
// alm_from_rings! (PartialFSHT.jl src/Legendre.jl:310-542; device analogue of
// ext/PartialFSHTKernelAbstractionsExt.jl:86-230).
//
// Work decomposition: one warp per item (order m, tile of consecutive retained rings, range of
// degrees); a lane owns R rings (ring j0 + lane + 32 r) and keeps their two-term recurrence
// state and block-scaling exponent in registers. The recurrence is the reference's
//     P_m^m = (-1)^m 2^(m log2 sin + log2 c_m),   P_{m+1}^m = sqrt(2m+3) cos P_m^m,
//     P_l^m = a_l^m cos P_{l-1}^m - b_l^m P_{l-2}^m,
// run in monic form inside blocks of `stride` degrees from l = m + 2: P_l = g_l q_l with
// g_l = a_lb ... a_l over the block's degrees so far, and
//     q_l = cos q_{l-1} - beta_l q_{l-2},   beta_l = b_l / (a_l a_{l-1})   (a_{m+1} = sqrt(2m+3)),
// two FP64 operations per (ring, degree) instead of three. The per-degree g_l multiplies the
// coefficients (forward) or the reduced sums (adjoint), shared by all rings. A block enters with
// (q_{lb-1}, q_{lb-2}) = (P_{lb-1}, a_{lb-1} P_{lb-2}) and leaves multiplied by g of its last
// degree, at which point the state is renormalised by a power of two (src/Legendre.jl:16,
// 455-459: every 64 degrees in the FP64 form; every 16 in the mixed form, so the values stay
// inside the FP32 range). Each ring keeps its own exponent, as the KernelAbstractions kernel
// does (ext/PartialFSHTKernelAbstractionsExt.jl:96-99).
//
// Forward: acc(ring, +-m) += a_{l,+-m} P_l, written once per ring, windowed and, for a
// pole/full periodisation, mirrored into the DFS row with sign (-1)^m (src/DFS.jl:26). The
// first tile of each order also writes the zeros of the rings the order does not retain.
// Adjoint: each lane sums P_l^m g_j over its R rings; per block of degrees the lanes' partial
// sums are transposed through shared memory and each lane reduces one (degree, component)
// over the 32 lanes. An order covered by a single tile stores its coefficients; an order
// split over several tiles adds them atomically (into zeros).
//
// Mixed form (MIX): the recurrence and exponents stay FP64; the forward accumulates in FP32
// with paired (float2) FMAs over each 32-degree chunk and adds the chunk into a compensated
// (two-sum) FP32 total; the adjoint keeps the ring data in FP32 and reduces in FP32.
#include <algorithm>
#include <cmath>
#include <map>
#include <type_traits>

#include "internal.cuh"

namespace pf {

static constexpr int kWarpsPerBlock = 4;  // forward
static constexpr int kAdjWarps = 1;       // adjoint (one-warp blocks: a finer tail)
static constexpr int kAdjWarpsPersistent = 2;  // the batches' persistent adjoint (measured faster)

// ---------------------------------------------------------------------------------------
// recurrence coefficient table (beta_l, g_l), from the exact expressions of
// src/Legendre.jl:406-408
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double rec_a(int l, int m) {
    if (l == m + 1) return sqrt((double)(2 * m + 3));
    return sqrt((double)(2 * l - 1) * (double)(2 * l + 1) / ((double)(l - m) * (double)(l + m)));
}
__device__ __forceinline__ double rec_b(int l, int m) {
    return sqrt((double)(2 * l + 1) / (double)(2 * l - 3) * (double)(l - m - 1) / (double)(l - m) *
                (double)(l + m - 1) / (double)(l + m));
}

// one thread per (order, block of `stride` degrees)
__global__ void ab_table_kernel(int L, int mmax, int stride, const int64_t* __restrict__ aboff,
                                double2* __restrict__ ab) {
    const int m = blockIdx.y;
    if (m > mmax || L < m + 2) return;
    const int nblk = (L - m - 1 + stride - 1) / stride;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nblk; k += gridDim.x * blockDim.x) {
        const int lb = m + 2 + k * stride;
        const int le = min(L, lb + stride - 1);
        double aprev = rec_a(lb - 1, m);
        double g = 1.0;
        for (int l = lb; l <= le; ++l) {
            const double a = rec_a(l, m), b = rec_b(l, m);
            g *= a;
            ab[aboff[m] + (l - m - 2)] = make_double2(b / (a * aprev), g);
            aprev = a;
        }
    }
}

static void ab_offsets(int L, int mmax, std::vector<int64_t>& off, int64_t& tot) {
    off.assign(L + 1, 0);
    tot = 0;
    for (int m = 0; m <= L; ++m) {
        off[m] = tot;
        if (m <= mmax) tot += std::max(0, L - m - 1);
    }
}

int launch_ab_table(int L, int mmax, int stride, const int64_t* aboff, double2* ab, cudaStream_t s) {
    const int nblk = (L + stride) / stride + 1;
    dim3 grid((unsigned)((nblk + 31) / 32), (unsigned)(mmax + 1));
    ab_table_kernel<<<grid, 32, 0, s>>>(L, mmax, stride, aboff, ab);
    return check_launch("ab_table_kernel");
}

int build_ab_table(int L, int mmax, int stride, DevBuf& ab, DevBuf& aboff, cudaStream_t s) {
    std::vector<int64_t> off;
    int64_t tot;
    ab_offsets(L, mmax, off, tot);
    PF_TRY(aboff.alloc(sizeof(int64_t) * (L + 1)));
    PF_TRY(ab.alloc(sizeof(double2) * std::max<int64_t>(tot, 1)));
    PF_CUDA(cudaMemcpyAsync(aboff.p, off.data(), sizeof(int64_t) * (L + 1),
                            cudaMemcpyHostToDevice, s));
    if (tot > 0) PF_TRY(launch_ab_table(L, mmax, stride, aboff.as<int64_t>(), ab.as<double2>(), s));
    // the host vector must outlive the async copy
    PF_CUDA(cudaStreamSynchronize(s));
    return 0;
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

// power-of-two exponent that brings max(|q1|, |q2|) into [1/2, 1), read from the exponent
// field (any power of two keeps the scaling exact); 0 for zero, subnormal or non-finite
__device__ __forceinline__ int renorm_shift(double q1, double q2) {
    const double mx = fmax(fabs(q1), fabs(q2));
    const int e = (__double2hiint(mx) >> 20) & 0x7ff;
    return (e == 0 || e == 0x7ff) ? 0 : e - 1022;
}

// 2^k for -1022 <= k <= 1023, built from its exponent field
__device__ __forceinline__ double pow2i(int k) { return __hiloint2double((k + 1023) << 20, 0); }

// ---------------------------------------------------------------------------------------
// plan-time recurrence checkpoints: one thread per (order, ring) walks the same monic
// recurrence, block conversions and renormalisations as the apply kernels and saves
// (q_{l-1}, q_{l-2}, E) at the first degree l of every later segment
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
    double x, p2;
    int E;
    ring_seed(t, m, j, sgn, x, p2, E);
    const double s23 = sqrt((double)(2 * m + 3));
    double q1 = s23 * x * p2, q2 = s23 * p2;
    const double2* abm = t.ab + t.aboff[m];
    int s = 1;
    int lnext = m + 2 + 64 * (int)(((int64_t)jb.nblk) / jb.nseg);
    int steps = 0;
    for (int l = m + 2; l <= L; ++l) {
        if (l == lnext) {
            const int64_t idx = jb.ck + (int64_t)(s - 1) * jb.stride + k;
            ckp[idx] = make_double2(q1, q2);
            ckE[idx] = E;
            if (++s == jb.nseg) break;
            lnext = m + 2 + 64 * (int)(((int64_t)s * jb.nblk) / jb.nseg);
        }
        const double2 bg = abm[l - m - 2];
        const double qn = fma(x, q1, -(bg.x * q2));
        q2 = q1;
        q1 = qn;
        if (++steps == t.stride) {
            steps = 0;
            if (l < L) {
                q1 *= bg.y;
                q2 *= bg.y;
                const int sh = renorm_shift(q1, q2);
                if (sh != 0) {
                    const double f = pow2i(-sh);
                    q1 *= f;
                    q2 *= f;
                    E += sh;
                }
            }
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
template <bool MIX> using CoefT = std::conditional_t<MIX, float2, double2>;

// one warp's staging (a block holds one per warp)
template <int NB, bool MIX>
struct FwdSmem {
    double2 bg[32];               // (beta_l, g_l) of the chunk's degrees
    CoefT<MIX> ap[NB][32];        // g_l a_{l,+m}
    CoefT<MIX> am[NB][32];        // g_l (-1)^m a_{l,-m}
};

// accumulator of one (ring, +-m, transform): FP64, or FP32 blocks into a two-sum total
template <bool MIX> struct FwdAcc;
template <> struct FwdAcc<false> {
    double2 a;
    __device__ __forceinline__ void zero() { a = make_double2(0.0, 0.0); }
    __device__ __forceinline__ void add(double2 c, double p) {
        a.x = fma(c.x, p, a.x);
        a.y = fma(c.y, p, a.y);
    }
    __device__ __forceinline__ void fold() {}
    __device__ __forceinline__ void scale(double f) {
        a.x *= f;
        a.y *= f;
    }
    __device__ __forceinline__ double2 total() const { return a; }
};
template <> struct FwdAcc<true> {
    float2 blk, s, c;
    __device__ __forceinline__ void zero() {
        blk = s = c = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void add(float2 cf, float p) {
        blk = __ffma2_rn(cf, make_float2(p, p), blk);
    }
    // s + blk as a two-sum: the rounding error of each block's addition is kept in c
    __device__ __forceinline__ void fold() {
        const float2 t = __fadd2_rn(s, blk);
        const float2 bp = __fadd2_rn(t, make_float2(-s.x, -s.y));
        const float2 sa = __fadd2_rn(t, make_float2(-bp.x, -bp.y));
        const float2 e = __fadd2_rn(__fadd2_rn(s, make_float2(-sa.x, -sa.y)),
                                    __fadd2_rn(blk, make_float2(-bp.x, -bp.y)));
        c = __fadd2_rn(c, e);
        s = t;
        blk = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void scale(double f) {
        const float2 ff = make_float2((float)f, (float)f);
        blk = __fmul2_rn(blk, ff);
        s = __fmul2_rn(s, ff);
        c = __fmul2_rn(c, ff);
    }
    __device__ __forceinline__ double2 total() const {
        return make_double2((double)s.x + ((double)c.x + (double)blk.x),
                            (double)s.y + ((double)c.y + (double)blk.y));
    }
};

template <bool MIX>
__device__ __forceinline__ CoefT<MIX> to_coef(double2 v) {
    if constexpr (MIX) return make_float2((float)v.x, (float)v.y);
    else return v;
}

template <int R, int NB, bool MIX>
__device__ __forceinline__ void ring_fwd_item(const RingTables& t, const RingOut& o,
                                              const RingItem& item, const double2* __restrict__ alm,
                                              double2* __restrict__ out, int b0,
                                              FwdSmem<NB, MIX>& sm, int warp, int lane) {
    constexpr int STRIDE = MIX ? 16 : 64;
    const int m = item.m, L = t.lmax;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    const int64_t albs = (int64_t)(L + 1) * (2 * L + 1);
    const double2* colp = alm + albs * b0 + (int64_t)(L + 1) * (2 * m);
    const double2* colm = alm + albs * b0 + (int64_t)(L + 1) * (m > 0 ? 2 * m - 1 : 0);
    const double2* abm = t.ab + t.aboff[m];
    const double2 zero2 = make_double2(0.0, 0.0);

    double x[R], q1[R], q2[R];
    int E[R];
    FwdAcc<MIX> accp[R][NB], accm[R][NB];
    const bool seeded = item.ck < 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        x[r] = 0.0;
        q1[r] = 0.0;
        q2[r] = 0.0;
        E[r] = 0;
        if (k < item.n) {
            if (seeded) {
                ring_seed(t, m, item.j0 + k, sgn, x[r], q2[r], E[r]);
            } else {
                x[r] = t.cos_t[item.j0 + k];
                const double2 c = t.ck_p[item.ck + k];
                q1[r] = c.x;
                q2[r] = c.y;
                E[r] = t.ck_E[item.ck + k];
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            accp[r][b].zero();
            accm[r][b].zero();
        }
    }
    // add a_{l,+-m} P for degree l (true P values, the first two degrees)
    auto add_true = [&](int l, const double (&P)[R]) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double2 ap = colp[(l - m) + albs * b];
            double2 am = m > 0 ? colm[(l - m) + albs * b] : zero2;
            am.x *= sgn;
            am.y *= sgn;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (MIX) {
                    accp[r][b].add(to_coef<MIX>(ap), (float)P[r]);
                    accm[r][b].add(to_coef<MIX>(am), (float)P[r]);
                } else {
                    accp[r][b].add(ap, P[r]);
                    accm[r][b].add(am, P[r]);
                }
            }
        }
    };
    int lstart = item.lbeg;
    if (seeded) {
        add_true(m, q2);  // l = m
        if (m < L) {
            const double s23 = sqrt((double)(2 * m + 3));
            double p1[R];
#pragma unroll
            for (int r = 0; r < R; ++r) p1[r] = s23 * x[r] * q2[r];
            add_true(m + 1, p1);  // l = m + 1
            // enter the monic form at l = m + 2: (q1, q2) = (P_{m+1}, a_{m+1} P_m)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                q2[r] = s23 * q2[r];
                q1[r] = p1[r];
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                accp[r][b].fold();
                accm[r][b].fold();
            }
        lstart = m + 2;
    }
    auto step = [&](int i) {
        const double beta = sm.bg[i].x;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double qn = fma(x[r], q1[r], -(beta * q2[r]));
            q2[r] = q1[r];
            q1[r] = qn;
        }
        float pf[R];
        if constexpr (MIX) {
#pragma unroll
            for (int r = 0; r < R; ++r) pf[r] = (float)q1[r];
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const CoefT<MIX> ap = sm.ap[b][i];
            const CoefT<MIX> am = sm.am[b][i];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (MIX) {
                    accp[r][b].add(ap, pf[r]);
                    accm[r][b].add(am, pf[r]);
                } else {
                    accp[r][b].add(ap, q1[r]);
                    accm[r][b].add(am, q1[r]);
                }
            }
        }
    };
    auto fold_all = [&]() {
        if constexpr (MIX) {
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    accp[r][b].fold();
                    accm[r][b].fold();
                }
        }
    };
    if (lstart <= item.lend) {
        // the coefficients of the next 32 degrees are loaded while this chunk runs
        double2 bg_n = zero2, ap_n[NB], am_n[NB];
        auto fetch = [&](int l) {
            if (l <= item.lend) {
                bg_n = abm[l - m - 2];
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    ap_n[b] = colp[(l - m) + albs * b];
                    am_n[b] = m > 0 ? colm[(l - m) + albs * b] : zero2;
                }
            }
        };
#pragma unroll
        for (int b = 0; b < NB; ++b) ap_n[b] = am_n[b] = zero2;
        fetch(lstart + lane);
        int steps = 0;
        for (int l0 = lstart; l0 <= item.lend; l0 += 32) {
            const int nl = min(32, item.lend - l0 + 1);
            __syncwarp();
            if (lane < nl) {
                const double g = bg_n.y;
                sm.bg[lane] = bg_n;
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    sm.ap[b][lane] = to_coef<MIX>(make_double2(ap_n[b].x * g, ap_n[b].y * g));
                    const double gs = g * sgn;
                    sm.am[b][lane] = to_coef<MIX>(make_double2(am_n[b].x * gs, am_n[b].y * gs));
                }
            }
            __syncwarp();
            fetch(l0 + 32 + lane);
            const int nblk = nl >> 3;
            for (int blk = 0; blk < nblk; ++blk) {
#pragma unroll
                for (int i = 0; i < 8; ++i) step(blk * 8 + i);
                steps += 8;
                if (steps == STRIDE) {
                    steps = 0;
                    if (l0 + blk * 8 + 7 < L) {
                        // leave the block: scale the state by g of its last degree, renormalise
                        const double G = sm.bg[blk * 8 + 7].y;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            q1[r] *= G;
                            q2[r] *= G;
                            const int sh = renorm_shift(q1[r], q2[r]);
                            if (sh != 0) {
                                const double f = pow2i(-sh);
                                q1[r] *= f;
                                q2[r] *= f;
#pragma unroll
                                for (int b = 0; b < NB; ++b) {
                                    accp[r][b].scale(f);
                                    accm[r][b].scale(f);
                                }
                                E[r] += sh;
                            }
                        }
                    }
                }
            }
            for (int i = nblk * 8; i < nl; ++i) step(i);
            fold_all();
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
            const double2 tp = accp[r][b].total(), tm = accm[r][b].total();
            const double2 gp = make_double2(tp.x * sc, tp.y * sc);
            const double2 gm = make_double2(tm.x * sc, tm.y * sc);
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

template <int RMAX, int NB, bool MIX>
__device__ __forceinline__ void ring_fwd_body(const RingTables& t, const RingOut& o,
                                              const RingItem& item, const int* __restrict__ jlo,
                                              const int* __restrict__ jhi,
                                              const double2* __restrict__ alm,
                                              double2* __restrict__ out, int b0,
                                              FwdSmem<NB, MIX>& sm, int warp, int lane) {
    if ((item.flags & kItemFirst) && o.zero_rest)
        ring_fwd_zero_rest<NB>(o, item, jlo[item.m], jhi[item.m], out, b0, lane);
    for (int base = 0; base < item.n; base += 32 * RMAX) {
        RingItem sub = item;
        sub.j0 = item.j0 + base;
        sub.n = min(32 * RMAX, item.n - base);
        if (sub.ck >= 0) sub.ck += base;
        const int reff = (sub.n + 31) >> 5;
        if (RMAX >= 4 && reff >= 3) ring_fwd_item<(RMAX >= 4 ? 4 : 1), NB, MIX>(t, o, sub, alm, out, b0, sm, warp, lane);
        else if (RMAX >= 2 && reff == 2) ring_fwd_item<(RMAX >= 2 ? 2 : 1), NB, MIX>(t, o, sub, alm, out, b0, sm, warp, lane);
        else ring_fwd_item<1, NB, MIX>(t, o, sub, alm, out, b0, sm, warp, lane);
    }
}

template <int RMAX, int NB, bool MIX>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
ring_fwd_kernel(RingTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const int* __restrict__ jlo, const int* __restrict__ jhi,
                const double2* __restrict__ alm, double2* __restrict__ out, int b0) {
    __shared__ FwdSmem<NB, MIX> sm[kWarpsPerBlock];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kWarpsPerBlock + warp;
    if (it >= nitems) return;
    ring_fwd_body<RMAX, NB, MIX>(t, o, items[it], jlo, jhi, alm, out, b0, sm[warp], warp, lane);
}

// the forward ring passes of many plans: item i belongs to plan items[i].slot
template <int RMAX, int NB, bool MIX>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
ring_fwd_batch_kernel(const RingSlot* __restrict__ slots, const BatchItem* __restrict__ items,
                      int nitems, void* const* __restrict__ ptrs) {
    __shared__ FwdSmem<NB, MIX> sm[kWarpsPerBlock];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kWarpsPerBlock + warp;
    if (it >= nitems) return;
    const BatchItem bi = items[it];
    const RingSlot& sl = slots[bi.slot];
    const RingTables t = sl.tf;
    const RingOut o = sl.o;
    ring_fwd_body<RMAX, NB, MIX>(t, o, bi.it, sl.jlo, sl.jhi,
                                 static_cast<const double2*>(ptrs[sl.ptr]), sl.H, bi.b0, sm[warp],
                                 warp, lane);
}

// ---------------------------------------------------------------------------------------
// adjoint: ring columns -> alm
// ---------------------------------------------------------------------------------------
template <bool MIX> using RedT = std::conditional_t<MIX, float, double>;
template <bool MIX> using RingDataT = std::conditional_t<MIX, float2, double2>;

template <bool MIX>
struct AdjSmem {  // one warp's staging (a block holds one per warp)
    RedT<MIX> red[32][33];
    double2 bg[32];
};

template <int R, int NB, bool MIX>
__device__ __forceinline__ void ring_adj_item(const RingTables& t, const RingOut& o,
                                              const RingItem& item, const double2* __restrict__ in,
                                              double* __restrict__ almd, int b0, int wmode,
                                              AdjSmem<MIX>& sm, int warp, int lane) {
    constexpr int STRIDE = MIX ? 16 : 64;
    constexpr int NV = 4 * NB;   // (+m re, +m im, -m re, -m im) per transform
    constexpr int LB = 32 / NV;  // degrees per reduction block
    // the scaled ring data g w 2^E stay normal (exactly rescalable) above kMinE, and round to
    // zero below kZeroE for any input smaller than 2^9 (mixed) or 2^125 (FP64)
    constexpr int kMinE = MIX ? -100 : -900;
    constexpr int kZeroE = MIX ? -160 : -1200;
    using GD = RingDataT<MIX>;
    using RT = RedT<MIX>;
    const int m = item.m, L = t.lmax;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    const double smir = o.spin_sgn * sgn;
    const int64_t albs = (int64_t)(L + 1) * (2 * L + 1);
    const double2* abm = t.ab + t.aboff[m];
    const int64_t cp = (int64_t)(L + 1) * (2 * m);
    const int64_t cm = (int64_t)(L + 1) * (m > 0 ? 2 * m - 1 : 0);

    double x[R], q1[R], q2[R];
    int E[R];
    GD gp[R][NB], gm[R][NB];
    auto put = [&](double a, double b) -> GD {
        if constexpr (MIX) return make_float2((float)a, (float)b);
        else return make_double2(a, b);
    };
    // ring data for (ring r, transform b): folded, windowed, scaled by 2^E; the -m column
    // carries the (-1)^m of src/Legendre.jl:511
    auto load_g = [&](int r) {
        const int k = lane + 32 * r;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            gp[r][b] = put(0.0, 0.0);
            gm[r][b] = put(0.0, 0.0);
        }
        if (k >= item.n || E[r] < kZeroE) return;
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
            gp[r][b] = put(v.x * sc, v.y * sc);
            if (m > 0) {
                double2 u = ib[j + o.ld * (o.col_off - m)];
                if (o.reflect) {
                    const double2 q = ib[(o.nrows - 1 - j) + o.ld * (o.col_off - m)];
                    u.x += smir * q.x;
                    u.y += smir * q.y;
                }
                gm[r][b] = put(u.x * sc * sgn, u.y * sc * sgn);
            }
        }
    };
    const bool seeded = item.ck < 0;
    // every global load of the item's start is issued before any of them is used: the first
    // chunk's recurrence coefficients, the ring data, then the seeds or checkpoints
    const int lfirst = seeded ? m + 2 : item.lbeg;
    double2 bg_first = make_double2(0.0, 0.0);
    if (lfirst <= item.lend && lane <= item.lend - lfirst) bg_first = abm[lfirst + lane - m - 2];
    double2 rp[R][NB], rm[R][NB];
    double wr[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        wr[r] = 1.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            rp[r][b] = make_double2(0.0, 0.0);
            rm[r][b] = make_double2(0.0, 0.0);
        }
        if (k < item.n) {
            const int j = item.j0 + k;
            if (t.w) wr[r] = t.w[j];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const double2* ib = in + o.bstride * (b0 + b);
                double2 v = ib[j + o.ld * (o.col_off + m)];
                if (o.reflect) {
                    const double2 u = ib[(o.nrows - 1 - j) + o.ld * (o.col_off + m)];
                    v.x += smir * u.x;
                    v.y += smir * u.y;
                }
                rp[r][b] = v;
                if (m > 0) {
                    double2 u = ib[j + o.ld * (o.col_off - m)];
                    if (o.reflect) {
                        const double2 q = ib[(o.nrows - 1 - j) + o.ld * (o.col_off - m)];
                        u.x += smir * q.x;
                        u.y += smir * q.y;
                    }
                    rm[r][b] = u;
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        x[r] = 0.0;
        q1[r] = 0.0;
        q2[r] = 0.0;
        E[r] = 0;
        if (k < item.n) {
            if (seeded) {
                ring_seed(t, m, item.j0 + k, sgn, x[r], q2[r], E[r]);
            } else {
                x[r] = t.cos_t[item.j0 + k];
                const double2 c = t.ck_p[item.ck + k];
                q1[r] = c.x;
                q2[r] = c.y;
                E[r] = t.ck_E[item.ck + k];
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        const bool live = k < item.n && E[r] >= kZeroE;
        const double sc = live ? scalbn(wr[r], E[r]) : 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            gp[r][b] = live ? put(rp[r][b].x * sc, rp[r][b].y * sc) : put(0.0, 0.0);
            gm[r][b] = live ? put(rm[r][b].x * sc * sgn, rm[r][b].y * sc * sgn) : put(0.0, 0.0);
        }
    }
    // partial sums over this lane's rings for degree slot `slot`
    auto stage = [&](const double (&P)[R], int slot) {
        RT part[NV];
        if constexpr (MIX) {
            float2 pp[2 * NB];
#pragma unroll
            for (int v = 0; v < 2 * NB; ++v) pp[v] = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float pf = (float)P[r];
                const float2 p2 = make_float2(pf, pf);
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    pp[2 * b] = __ffma2_rn(p2, gp[r][b], pp[2 * b]);
                    pp[2 * b + 1] = __ffma2_rn(p2, gm[r][b], pp[2 * b + 1]);
                }
            }
#pragma unroll
            for (int v = 0; v < 2 * NB; ++v) {
                part[2 * v] = pp[v].x;
                part[2 * v + 1] = pp[v].y;
            }
        } else {
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
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.red[slot * NV + v][lane] = part[v];
    };
    // reduce the staged degrees [lfirst, lfirst + cnt) over the lanes and write alm; degree
    // lfirst + i carries the factor g of its chunk slot gslot0 + i (1 for the seed degrees)
    auto flush = [&](int lfirst, int cnt, int gslot0) {
        __syncwarp();
        if (lane < cnt * NV) {
            const int li = lane / NV, v = lane % NV;
            // four independent partial sums: the chain of dependent adds is 8 long, not 32
            RT s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
            for (int q = 0; q < 32; q += 4) {
                s0 += sm.red[lane][q];
                s1 += sm.red[lane][q + 1];
                s2 += sm.red[lane][q + 2];
                s3 += sm.red[lane][q + 3];
            }
            double s = (double)((s0 + s1) + (s2 + s3));
            if (gslot0 >= 0) s *= sm.bg[gslot0 + li].y;
            const int l = lfirst + li;
            const int b = v >> 2, comp = v & 3;
            if (comp < 2 || m > 0) {
                const int64_t idx = (l - m) + (comp < 2 ? cp : cm) + albs * (b0 + b);
                double* dst = almd + 2 * idx + (comp & 1);
                // 0: the only writer; 1: this warp wrote the value before (an earlier ring
                // tile of the same item, the same lane): add in order; 2: other warps add too
                if (wmode == 0) *dst = s;
                else if (wmode == 1) *dst += s;
                else atomicAdd(dst, s);
            }
        }
        __syncwarp();
    };
    int lstart = item.lbeg;
    if (seeded) {
        stage(q2, 0);  // l = m
        if (m == L) {
            flush(m, 1, -1);
            return;
        }
        const double s23 = sqrt((double)(2 * m + 3));
        double p1[R];
#pragma unroll
        for (int r = 0; r < R; ++r) p1[r] = s23 * x[r] * q2[r];
        stage(p1, 1);  // l = m + 1
        flush(m, 2, -1);
        // enter the monic form at l = m + 2: (q1, q2) = (P_{m+1}, a_{m+1} P_m)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            q2[r] = s23 * q2[r];
            q1[r] = p1[r];
        }
        lstart = m + 2;
    }
    auto rec = [&](int i) {
        const double beta = sm.bg[i].x;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double qn = fma(x[r], q1[r], -(beta * q2[r]));
            q2[r] = q1[r];
            q1[r] = qn;
        }
    };
    // the coefficients of the next 32 degrees are loaded while this chunk runs
    double2 bg_next = bg_first;  // lstart == lfirst here
    // segments start on the renormalisation schedule, so the count restarts at 0
    int steps = 0;
    for (int l0 = lstart; l0 <= item.lend; l0 += 32) {
        const int nl = min(32, item.lend - l0 + 1);
        __syncwarp();
        if (lane < nl) sm.bg[lane] = bg_next;
        __syncwarp();
        if (l0 + 32 + lane <= item.lend) bg_next = abm[l0 + 32 + lane - m - 2];
        const int nblk = nl / LB;
        for (int blk = 0; blk < nblk; ++blk) {
#pragma unroll
            for (int i = 0; i < LB; ++i) {
                rec(blk * LB + i);
                stage(q1, i);
            }
            flush(l0 + blk * LB, LB, blk * LB);
            steps += LB;
            if (steps == STRIDE) {
                steps = 0;
                if (l0 + blk * LB + LB - 1 < L) {
                    // leave the block: scale the state by g of its last degree, renormalise
                    const double G = sm.bg[blk * LB + LB - 1].y;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        q1[r] *= G;
                        q2[r] *= G;
                        const int sh = renorm_shift(q1[r], q2[r]);
                        if (sh != 0) {
                            const double f = pow2i(-sh);
                            q1[r] *= f;
                            q2[r] *= f;
                            const int Eold = E[r];
                            E[r] += sh;
                            if (Eold >= kMinE) {
                                // the scaled ring data were normal: 2^sh keeps them exactly
                                // what a reload would give
                                const double u = pow2i(sh);
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
        const int rem = nl - nblk * LB;
        if (rem > 0) {
            for (int i = 0; i < rem; ++i) {
                rec(nblk * LB + i);
                stage(q1, i);
            }
            flush(l0 + nblk * LB, rem, nblk * LB);
        }
    }
}

template <int RMAX, int NB, bool MIX>
__device__ __forceinline__ void ring_adj_body(const RingTables& t, const RingOut& o,
                                              const RingItem& item, const double2* __restrict__ in,
                                              double* __restrict__ almd, int b0, int allow_sole,
                                              AdjSmem<MIX>& sm, int warp, int lane) {
    // an item holding all retained rings of its order writes its degrees alone: its first ring
    // tile stores them and the later ones add in order (deterministic); an order split over
    // several items adds atomically into zeros
    const bool whole = allow_sole && (item.flags & kItemSole);
    for (int base = 0; base < item.n; base += 32 * RMAX) {
        const int wmode = whole ? (base == 0 ? 0 : 1) : 2;
        RingItem sub = item;
        sub.j0 = item.j0 + base;
        sub.n = min(32 * RMAX, item.n - base);
        if (sub.ck >= 0) sub.ck += base;
        const int reff = (sub.n + 31) >> 5;
        if (RMAX >= 8 && reff >= 5) ring_adj_item<(RMAX >= 8 ? 8 : 1), NB, MIX>(t, o, sub, in, almd, b0, wmode, sm, warp, lane);
        else if (RMAX >= 4 && reff >= 3) ring_adj_item<(RMAX >= 4 ? 4 : 1), NB, MIX>(t, o, sub, in, almd, b0, wmode, sm, warp, lane);
        else if (RMAX >= 2 && reff == 2) ring_adj_item<(RMAX >= 2 ? 2 : 1), NB, MIX>(t, o, sub, in, almd, b0, wmode, sm, warp, lane);
        else ring_adj_item<1, NB, MIX>(t, o, sub, in, almd, b0, wmode, sm, warp, lane);
    }
}

template <int RMAX, int NB, bool MIX>
__global__ void __launch_bounds__(kAdjWarps * 32)
ring_adj_kernel(RingTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const double2* __restrict__ in, double* __restrict__ almd, int b0, int allow_sole) {
    __shared__ AdjSmem<MIX> sm[kAdjWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kAdjWarps + warp;
    if (it >= nitems) return;
    ring_adj_body<RMAX, NB, MIX>(t, o, items[it], in, almd, b0, allow_sole, sm[warp], warp, lane);
}

// the adjoint ring passes of many plans: item i belongs to plan items[i].slot
template <int RMAX, int NB, bool MIX>
__global__ void __launch_bounds__(kAdjWarps * 32)
ring_adj_batch_kernel(const RingSlot* __restrict__ slots, const BatchItem* __restrict__ items,
                      int nitems, void* const* __restrict__ ptrs) {
    __shared__ AdjSmem<MIX> sm[kAdjWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kAdjWarps + warp;
    if (it >= nitems) return;
    const BatchItem bi = items[it];
    const RingSlot& sl = slots[bi.slot];
    const RingTables t = sl.t;
    const RingOut o = sl.o;
    ring_adj_body<RMAX, NB, MIX>(t, o, bi.it, sl.H, static_cast<double*>(ptrs[sl.ptr]), bi.b0,
                                      sl.allow_sole, sm[warp], warp, lane);
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
template <int RMAX, int NB, bool MIX>
static int launch_fwd(const RingTables& t, const RingOut& o, const RingItem* items, int nitems,
                      const int* jlo, const int* jhi, const double2* alm, double2* out, int b0,
                      cudaStream_t s) {
    const int grid = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    ring_fwd_kernel<RMAX, NB, MIX><<<grid, kWarpsPerBlock * 32, 0, s>>>(t, o, items, nitems, jlo, jhi,
                                                                       alm, out, b0);
    return check_launch("ring_fwd_kernel");
}

template <int RMAX, int NB, bool MIX>
static int launch_adj(const RingTables& t, const RingOut& o, const RingItem* items, int nitems,
                      const double2* in, double2* alm, int b0, int allow_sole, cudaStream_t s) {
    const int grid = (nitems + kAdjWarps - 1) / kAdjWarps;
    ring_adj_kernel<RMAX, NB, MIX><<<grid, kAdjWarps * 32, 0, s>>>(
        t, o, items, nitems, in, reinterpret_cast<double*>(alm), b0, allow_sole);
    return check_launch("ring_adj_kernel");
}

template <bool MIX>
static int ring_forward_t(const RingTables& t, const RingOut& o, const RingItems& it,
                          const double2* alm, double2* out, int B, cudaStream_t s) {
    int b0 = 0;
    while (b0 < B) {
        const int rem = B - b0;
        if (rem >= 4) {
            PF_TRY((launch_fwd<1, 4, MIX>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            b0 += 4;
        } else if (rem >= 2) {
            PF_TRY((launch_fwd<2, 2, MIX>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            b0 += 2;
        } else {
            if (it.rmax >= 4) PF_TRY((launch_fwd<4, 1, MIX>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            else PF_TRY((launch_fwd<2, 1, MIX>(t, o, it.items, it.nitems, it.jlo, it.jhi, alm, out, b0, s)));
            b0 += 1;
        }
    }
    return 0;
}

int ring_forward(const RingTables& t, const RingOut& o, const RingItems& it, const double2* alm,
                 double2* out, int B, cudaStream_t s) {
    if (it.nitems <= 0) return 0;
    return t.mix ? ring_forward_t<true>(t, o, it, alm, out, B, s)
                 : ring_forward_t<false>(t, o, it, alm, out, B, s);
}

int alm_prepare(double2* alm, int L, int B, const unsigned char* sole_m, int allow_sole,
                cudaStream_t s) {
    dim3 grid(2 * L + 1, B);
    alm_prepare_kernel<<<grid, 128, 0, s>>>(alm, L, B, sole_m, allow_sole);
    return check_launch("alm_prepare_kernel");
}

template <bool MIX>
static int ring_adjoint_t(const RingTables& t, const RingOut& o, const RingItems& it,
                          const double2* in, double2* alm, int B, int allow_sole, cudaStream_t s) {
    // one pass per transform: the multi-transform shapes share the recurrence but stage NB times
    // the partial sums per ring through shared memory, the adjoint's co-limit (at lmax 1024,
    // ntrans 4: 0.59 ms with four transforms per pass against 4 x 0.073 ms one by one)
    for (int b0 = 0; b0 < B; ++b0) {
        if (it.rmax >= 8) PF_TRY((launch_adj<8, 1, MIX>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
        else if (it.rmax >= 4) PF_TRY((launch_adj<4, 1, MIX>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
        else PF_TRY((launch_adj<2, 1, MIX>(t, o, it.items, it.nitems, in, alm, b0, allow_sole, s)));
    }
    return 0;
}

// each transform's pass with the items' own tile shape stores the orders covered by a single
// tile directly (the other orders add into zeros)
static int adjoint_allow_sole(const RingItems& it, int B) {
    (void)B;
    return it.rmax >= 2 ? 1 : 0;
}

int ring_adjoint_prepare(const RingTables& t, const RingItems& it, double2* alm, int B, cudaStream_t s) {
    return alm_prepare(alm, t.lmax, B, it.sole_m, adjoint_allow_sole(it, B), s);
}

int ring_adjoint(const RingTables& t, const RingOut& o, const RingItems& it, const double2* in,
                 double2* alm, int B, cudaStream_t s, bool prepare) {
    const int allow_sole = adjoint_allow_sole(it, B);
    if (prepare) PF_TRY(alm_prepare(alm, t.lmax, B, it.sole_m, allow_sole, s));
    if (it.nitems <= 0) return 0;
    return t.mix ? ring_adjoint_t<true>(t, o, it, in, alm, B, allow_sole, s)
                 : ring_adjoint_t<false>(t, o, it, in, alm, B, allow_sole, s);
}

// item lists of one ring set: tiles of 32 * rmax rings, the order flags, the device tables
int build_ring_items(const std::vector<int>& jlo, const std::vector<int>& jhi, int L, int mmax,
                     int rmax, RingItemsOwner& own, cudaStream_t s, const RingSegments* seg,
                     int tile) {
    std::vector<RingItem> items = make_ring_items(jlo, jhi, L, mmax, tile > 0 ? tile : 32 * rmax, seg);
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
    own.host = items;
    own.view.rmax = rmax;
    own.view.sole_m = own.sole.as<unsigned char>();
    own.view.jlo = own.jlo.as<int>();
    own.view.jhi = own.jhi.as<int>();
    return 0;
}

// ---------------------------------------------------------------------------------------
// batched ring passes: the items of many plans, grouped by kernel shape
// ---------------------------------------------------------------------------------------
__global__ void alm_prepare_ptr_kernel(void* const* __restrict__ ptrs, int ptr, int L, int B,
                                       const unsigned char* __restrict__ sole_m, int allow_sole) {
    double2* alm = static_cast<double2*>(ptrs[ptr]);
    const int c = blockIdx.x, b = blockIdx.y;
    const int am = (c + 1) / 2;
    double2* col = alm + (int64_t)(L + 1) * c + (int64_t)(L + 1) * (2 * L + 1) * b;
    const int first = (allow_sole && sole_m[am]) ? L - am + 1 : 0;
    for (int r = first + threadIdx.x; r <= L; r += blockDim.x) col[r] = make_double2(0.0, 0.0);
}

int alm_prepare_ptr(void* const* ptrs, int ptr, int L, int B, const unsigned char* sole_m,
                    int allow_sole, cudaStream_t s) {
    dim3 grid(2 * L + 1, B);
    alm_prepare_ptr_kernel<<<grid, 128, 0, s>>>(ptrs, ptr, L, B, sole_m, allow_sole);
    return check_launch("alm_prepare_ptr_kernel");
}

// the passes a single-plan launch would make over B transforms: (rings per lane, transforms)
static std::vector<std::pair<int, int>> ring_passes(int B, int rmax, bool adjoint, std::vector<int>& b0s) {
    std::vector<std::pair<int, int>> v;
    b0s.clear();
    int b0 = 0;
    while (b0 < B) {
        const int rem = B - b0;
        b0s.push_back(b0);
        if (adjoint) {
            // one pass per transform (ring_adjoint_t)
            v.push_back({rmax >= 8 ? 8 : rmax >= 4 ? 4 : 2, 1});
            b0 += 1;
        } else if (rem >= 4) {
            v.push_back({1, 4});
            b0 += 4;
        } else if (rem >= 2) {
            v.push_back({2, 2});
            b0 += 2;
        } else {
            v.push_back({rmax >= 4 ? 4 : 2, 1});
            b0 += 1;
        }
    }
    return v;
}

int build_ring_batch(const std::vector<RingBatchPlan>& plans, bool adjoint,
                     std::vector<std::unique_ptr<RingBatchGroup>>& groups, cudaStream_t s) {
    groups.clear();
    struct Key {
        int rmax, nb, mix;
        bool operator<(const Key& o) const {
            return rmax != o.rmax ? rmax < o.rmax : nb != o.nb ? nb < o.nb : mix < o.mix;
        }
    };
    std::map<Key, std::vector<std::pair<int64_t, BatchItem>>> by;
    std::vector<int> b0s;
    for (size_t p = 0; p < plans.size(); ++p) {
        const RingBatchPlan& pl = plans[p];
        const auto passes = ring_passes(pl.B, pl.rmax, adjoint, b0s);
        for (size_t k = 0; k < passes.size(); ++k) {
            auto& vec = by[Key{passes[k].first, passes[k].second, pl.mix}];
            for (const RingItem& it : *pl.items) {
                const int64_t cost = (int64_t)((it.n + 31) / 32) * (it.lend - it.lbeg + 1) *
                                     passes[k].second;
                vec.push_back({cost, BatchItem{it, (int)p, b0s[k]}});
            }
        }
    }
    for (auto& kv : by) {
        auto& vec = kv.second;
        if (vec.empty()) continue;  // plans without merged items (spin plans) make no launch
        std::stable_sort(vec.begin(), vec.end(),
                         [](const auto& a, const auto& b) { return a.first > b.first; });
        std::vector<BatchItem> items(vec.size());
        for (size_t i = 0; i < vec.size(); ++i) items[i] = vec[i].second;
        auto g = std::make_unique<RingBatchGroup>();
        g->rmax = kv.first.rmax;
        g->nb = kv.first.nb;
        g->mix = kv.first.mix;
        g->nitems = (int)items.size();
        PF_TRY(g->items.alloc(sizeof(BatchItem) * std::max<size_t>(items.size(), 1)));
        if (!items.empty())
            PF_CUDA(cudaMemcpyAsync(g->items.p, items.data(), sizeof(BatchItem) * items.size(),
                                    cudaMemcpyHostToDevice, s));
        PF_CUDA(cudaStreamSynchronize(s));
        groups.push_back(std::move(g));
    }
    return 0;
}

template <int RMAX, int NB, bool MIX>
static int launch_fwd_batch(const RingSlot* slots, const RingBatchGroup& g, void* const* ptrs,
                            cudaStream_t s) {
    const int grid = (g.nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    ring_fwd_batch_kernel<RMAX, NB, MIX><<<grid, kWarpsPerBlock * 32, 0, s>>>(
        slots, g.items.as<BatchItem>(), g.nitems, ptrs);
    return check_launch("ring_fwd_batch_kernel");
}

template <int RMAX, int NB, bool MIX>
static int launch_adj_batch(const RingSlot* slots, const RingBatchGroup& g, void* const* ptrs,
                            cudaStream_t s) {
    const int grid = (g.nitems + kAdjWarps - 1) / kAdjWarps;
    ring_adj_batch_kernel<RMAX, NB, MIX><<<grid, kAdjWarps * 32, 0, s>>>(
        slots, g.items.as<BatchItem>(), g.nitems, ptrs);
    return check_launch("ring_adj_batch_kernel");
}

template <bool MIX>
static int fwd_batch_shape(const RingSlot* slots, const RingBatchGroup& g, void* const* ptrs,
                           cudaStream_t s) {
    if (g.nb == 4) return launch_fwd_batch<1, 4, MIX>(slots, g, ptrs, s);
    if (g.nb == 2) return launch_fwd_batch<2, 2, MIX>(slots, g, ptrs, s);
    if (g.rmax >= 4) return launch_fwd_batch<4, 1, MIX>(slots, g, ptrs, s);
    return launch_fwd_batch<2, 1, MIX>(slots, g, ptrs, s);
}

template <bool MIX>
static int adj_batch_shape(const RingSlot* slots, const RingBatchGroup& g, void* const* ptrs,
                           cudaStream_t s) {
    if (g.nb == 4) return launch_adj_batch<1, 4, MIX>(slots, g, ptrs, s);
    if (g.nb == 2) return launch_adj_batch<2, 2, MIX>(slots, g, ptrs, s);
    if (g.rmax >= 8) return launch_adj_batch<8, 1, MIX>(slots, g, ptrs, s);
    if (g.rmax >= 4) return launch_adj_batch<4, 1, MIX>(slots, g, ptrs, s);
    return launch_adj_batch<2, 1, MIX>(slots, g, ptrs, s);
}

// ---------------------------------------------------------------------------------------
// one persistent launch per direction for the ring passes of many plans: each warp pulls the next
// item (any plan, any tile shape; all items heaviest first) from a counter in device memory until
// none is left, and the item's shape code (RingItem::pad_) selects the pass it runs. A block
// holds one staging area per warp, sized for the largest shape, so warps of one block may run
// different shapes. No warp waits for another.
// ---------------------------------------------------------------------------------------
// forward shapes: (rings per lane, transforms per pass) = (1, 4), (2, 2), (4, 1), (2, 1); the
// mixed form adds 4
static int fwd_shape(int rmax, int nb, int mix) {
    const int k = nb == 4 ? 0 : nb == 2 ? 1 : rmax >= 4 ? 2 : 3;
    return k + 4 * (mix ? 1 : 0);
}
// adjoint shapes (one transform per pass): rings per lane 4 or 2; the mixed form adds 2
static int adj_shape(int rmax, int mix) { return (rmax >= 4 ? 0 : 1) + 2 * (mix ? 1 : 0); }

union FwdAnySmem {
    FwdSmem<4, false> a;
    FwdSmem<2, false> b;
    FwdSmem<1, false> c;
    FwdSmem<4, true> d;
    FwdSmem<2, true> e;
    FwdSmem<1, true> f;
};
union AdjAnySmem {
    AdjSmem<false> a;
    AdjSmem<true> b;
};

__device__ __forceinline__ int pull_item(int* counter, int lane) {
    int it = 0;
    if (lane == 0) it = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, it, 0);
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32, 3)
ring_fwd_persistent_kernel(const RingSlot* __restrict__ slots, const BatchItem* __restrict__ items,
                           int nitems, void* const* __restrict__ ptrs, int* __restrict__ counter) {
    __shared__ FwdAnySmem sm[kWarpsPerBlock];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int it = pull_item(counter, lane); it < nitems; it = pull_item(counter, lane)) {
        const BatchItem bi = items[it];
        const RingSlot& sl = slots[bi.slot];
        const RingTables t = sl.tf;
        const RingOut o = sl.o;
        const double2* alm = static_cast<const double2*>(ptrs[sl.ptr]);
        FwdAnySmem& w = sm[warp];
        switch (bi.it.pad_) {
            case 0: ring_fwd_body<1, 4, false>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.a, warp, lane); break;
            case 1: ring_fwd_body<2, 2, false>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.b, warp, lane); break;
            case 2: ring_fwd_body<4, 1, false>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.c, warp, lane); break;
            case 3: ring_fwd_body<2, 1, false>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.c, warp, lane); break;
            case 4: ring_fwd_body<1, 4, true>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.d, warp, lane); break;
            case 5: ring_fwd_body<2, 2, true>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.e, warp, lane); break;
            case 6: ring_fwd_body<4, 1, true>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.f, warp, lane); break;
            default: ring_fwd_body<2, 1, true>(t, o, bi.it, sl.jlo, sl.jhi, alm, sl.H, bi.b0, w.f, warp, lane); break;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kAdjWarpsPersistent * 32)
ring_adj_persistent_kernel(const RingSlot* __restrict__ slots, const BatchItem* __restrict__ items,
                           int nitems, void* const* __restrict__ ptrs, int* __restrict__ counter) {
    __shared__ AdjAnySmem sm[kAdjWarpsPersistent];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int it = pull_item(counter, lane); it < nitems; it = pull_item(counter, lane)) {
        const BatchItem bi = items[it];
        const RingSlot& sl = slots[bi.slot];
        const RingTables t = sl.t;
        const RingOut o = sl.o;
        double* almd = static_cast<double*>(ptrs[sl.ptr]);
        AdjAnySmem& w = sm[warp];
        switch (bi.it.pad_) {
            case 0: ring_adj_body<4, 1, false>(t, o, bi.it, sl.H, almd, bi.b0, sl.allow_sole, w.a, warp, lane); break;
            case 1: ring_adj_body<2, 1, false>(t, o, bi.it, sl.H, almd, bi.b0, sl.allow_sole, w.a, warp, lane); break;
            case 2: ring_adj_body<4, 1, true>(t, o, bi.it, sl.H, almd, bi.b0, sl.allow_sole, w.b, warp, lane); break;
            default: ring_adj_body<2, 1, true>(t, o, bi.it, sl.H, almd, bi.b0, sl.allow_sole, w.b, warp, lane); break;
        }
        __syncwarp();
    }
}

int build_ring_merged(const std::vector<RingBatchPlan>& plans, bool adjoint, RingMerged& mg,
                      std::vector<std::unique_ptr<RingBatchGroup>>& rest, cudaStream_t s) {
    std::vector<std::unique_ptr<RingBatchGroup>> groups;
    PF_TRY(build_ring_batch(plans, adjoint, groups, s));
    std::vector<std::pair<int64_t, BatchItem>> all;
    rest.clear();
    for (auto& g : groups) {
        // the eight-rings-per-lane adjoint keeps its own launch (its register count would set
        // every shape's occupancy)
        if (adjoint && g->rmax >= 8) {
            rest.push_back(std::move(g));
            continue;
        }
        std::vector<BatchItem> v(g->nitems);
        if (g->nitems)
            PF_CUDA(cudaMemcpy(v.data(), g->items.p, sizeof(BatchItem) * v.size(), cudaMemcpyDeviceToHost));
        const int code = adjoint ? adj_shape(g->rmax, g->mix) : fwd_shape(g->rmax, g->nb, g->mix);
        for (BatchItem& b : v) {
            b.it.pad_ = code;
            const int64_t cost = (int64_t)((b.it.n + 31) / 32) * (b.it.lend - b.it.lbeg + 1) * g->nb;
            all.push_back({cost, b});
        }
    }
    std::stable_sort(all.begin(), all.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<BatchItem> items(all.size());
    for (size_t i = 0; i < all.size(); ++i) items[i] = all[i].second;
    mg.nitems = (int)items.size();
    PF_TRY(mg.items.alloc(sizeof(BatchItem) * std::max<size_t>(items.size(), 1)));
    PF_TRY(mg.counter.alloc(sizeof(int)));
    if (!items.empty())
        PF_CUDA(cudaMemcpy(mg.items.p, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice));
    // one block per resident slot: the persistent grid
    int dev = 0, sms = 148, per = 1;
    PF_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (adjoint)
        PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, ring_adj_persistent_kernel, kAdjWarpsPersistent * 32, 0));
    else
        PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, ring_fwd_persistent_kernel, kWarpsPerBlock * 32, 0));
    const int wpb = adjoint ? kAdjWarpsPersistent : kWarpsPerBlock;
    mg.grid = std::max(1, std::min(sms * std::max(1, per), (mg.nitems + wpb - 1) / wpb));
    return 0;
}

int ring_merged_launch(const RingSlot* slots, const RingMerged& mg, bool adjoint, void* const* ptrs,
                       cudaStream_t s) {
    if (mg.nitems == 0) return 0;
    PF_CUDA(cudaMemsetAsync(mg.counter.p, 0, sizeof(int), s));
    if (adjoint) {
        ring_adj_persistent_kernel<<<mg.grid, kAdjWarpsPersistent * 32, 0, s>>>(slots, mg.items.as<BatchItem>(),
                                                                      mg.nitems, ptrs, mg.counter.as<int>());
        return check_launch("ring_adj_persistent_kernel");
    }
    ring_fwd_persistent_kernel<<<mg.grid, kWarpsPerBlock * 32, 0, s>>>(slots, mg.items.as<BatchItem>(),
                                                                       mg.nitems, ptrs, mg.counter.as<int>());
    return check_launch("ring_fwd_persistent_kernel");
}

int ring_forward_batch(const RingSlot* slots, const std::vector<std::unique_ptr<RingBatchGroup>>& groups,
                       void* const* ptrs, cudaStream_t s) {
    for (const auto& g : groups) {
        if (g->nitems == 0) continue;
        PF_TRY(g->mix ? fwd_batch_shape<true>(slots, *g, ptrs, s)
                      : fwd_batch_shape<false>(slots, *g, ptrs, s));
    }
    return 0;
}

int ring_adjoint_batch(const RingSlot* slots, const std::vector<std::unique_ptr<RingBatchGroup>>& groups,
                       void* const* ptrs, cudaStream_t s) {
    for (const auto& g : groups) {
        if (g->nitems == 0) continue;
        PF_TRY(g->mix ? adj_batch_shape<true>(slots, *g, ptrs, s)
                      : adj_batch_shape<false>(slots, *g, ptrs, s));
    }
    return 0;
}

}  // namespace pf
