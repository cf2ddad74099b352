// libpfsht_b200: plan construction and the C ABI (include/pfsht_b200.h).
//
// A plan is PartialFSHT.jl's Plan + StretchLeaf (src/Plan.jl:84-116, src/Stretch.jl:129-248)
// on one device: geometry and sizes on the host, the point transform, bin sort and
// recurrence tables on the device, and an apply that runs
//   forward : ring pass -> FFT along Theta -> NUFFT type 2         (src/Stretch.jl:262-277)
//   adjoint : NUFFT type 1 -> inverse FFT along Theta -> ring pass (src/Stretch.jl:279-295)
// The reference's pack / bfft-along-phi / window / DFS / 2-D FFT / phase sequence
// (src/Stretch.jl:269-273) is applied in closed form: the phi shift by pi of the DFS
// reflection is (-1)^m on order columns and fft_phi o bfft_phi = n_phi I on the packed
// orders, so the whole sequence is, per retained order column, the window and the mirrored
// DFS rows (written by the ring pass) followed by one FFT along Theta and the half-cell
// phase / n_theta (folded into the NUFFT's per-mode factor).
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <queue>
#include <string>
#include <vector>

#include "../../include/pfsht_b200.h"
#include "internal.cuh"
#include "plan_internal.hpp"
#include "planner.hpp"

namespace pf {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const std::string& get_error() { return g_err; }

}  // namespace pf

using namespace pf;

struct pfsht_nufft {
    int device = 0;
    int type = 2, iflag = 1, B = 1;
    int n1 = 0, n2 = 0;
    int64_t M = 0;
    NufftGrid g;
    NufftDev d;
};

namespace {

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

template <class T>
int upload(DevBuf& d, const std::vector<T>& h, cudaStream_t s) {
    PF_TRY(d.alloc(sizeof(T) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) PF_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaStreamSynchronize(s));
    return 0;
}

int mode_k(int i, int n) { return i < (n + 1) / 2 ? i : i - n; }

// NUFFT grid and per-mode factors; n1 modes along dim 1, columns -> k2 via colk2
// lengths: 0 = fine-grid FFT lengths picked by timing (fine_fft_length), 1 = the minimum
// 2,3,5-smooth lengths, 2 = nf1 x nf2 as given
int setup_nufft_grid(NufftGrid& g, NufftDev& d, int n1, int nmodes2, const std::vector<int>& colk2,
                     const std::vector<double2>& phase1, double tol, int64_t M, double xmin,
                     double xmax, bool full_rows, int bin_rows, int bin_cols, bool fp32, int lengths,
                     int nf1, int nf2, cudaStream_t s) {
    g.w = es_width(tol);
    g.beta = 2.30 * g.w;
    g.fp32 = fp32 ? 1 : 0;
    g.nf1 = (int)next_smooth(std::max<int64_t>(2 * (int64_t)n1, 2 * g.w));
    g.nf2 = (int)next_smooth(std::max<int64_t>(2 * (int64_t)nmodes2, 2 * g.w));
    g.n1 = n1;
    g.ncols = (int)colk2.size();
    const bool timed = lengths == 0;
    if (lengths == 2) {
        if (nf1 < std::max(2 * n1, 2 * g.w) || nf2 < std::max(2 * nmodes2, 2 * g.w) || nf1 > (1 << 24) ||
            nf2 > (1 << 24))
            return fail(PFSHT_ERR_ARGUMENT, "fine-grid lengths must be at least " +
                                                std::to_string(std::max(2 * n1, 2 * g.w)) + " x " +
                                                std::to_string(std::max(2 * nmodes2, 2 * g.w)));
        g.nf1 = nf1;
        g.nf2 = nf2;
    }
    // timed for one transform, so that plans of one geometry share lengths whatever ntrans
    if (timed) PF_TRY(fine_fft_length(g.nf1, g.ncols, fp32, s, &g.nf1));
    g.M = M;
    // the spreading tile (bin width + w - 1 columns) is half a warp wide for kernels up to
    // 10 cells (two half-warps share its rows by parity), one warp wide beyond
    const bool half = g.w <= 10;
    g.bin_rows = bin_rows > 0 ? bin_rows : (half ? 24 : 12);
    g.bin_cols = (half ? 17 : 33) - g.w;
    if (bin_cols > 0 && bin_cols < g.bin_cols) g.bin_cols = bin_cols;
    // interpolation tiles of up to 32 columns: as many whole bins as fit
    g.igroup = std::max(1, (33 - g.w) / g.bin_cols);
    if (full_rows) {
        g.row0 = 0;
        g.nrows = g.nf1;
        g.row_wrap = 1;
    } else {
        const double s1 = (double)g.nf1 / (2 * M_PI);
        const double g1lo = xmin * s1, g1hi = xmax * s1;
        const int r0 = (int)std::floor(g1lo - 0.5 * g.w) - 2;
        const int r1 = (int)std::ceil(g1hi + 0.5 * g.w) + 2;
        if (r1 - r0 + 1 >= g.nf1) {
            g.row0 = 0;
            g.nrows = g.nf1;
            g.row_wrap = 1;
        } else {
            g.row0 = r0;
            g.nrows = r1 - r0 + 1;
            g.row_wrap = 0;
        }
    }
    if (timed) PF_TRY(fine_fft_length(g.nf2, g.nrows, fp32, s, &g.nf2));
    std::vector<double2> mult1(n1);
    for (int i = 0; i < n1; ++i) {
        const double dec = es_deconv(mode_k(i, n1), g.nf1, g.w, g.beta);
        mult1[i] = make_double2(phase1[i].x * dec, phase1[i].y * dec);
    }
    std::vector<double> dec2(g.ncols);
    std::vector<int> colp2(g.ncols), p2col(g.nf2, -1);
    for (int c = 0; c < g.ncols; ++c) {
        const int k2 = colk2[c];
        dec2[c] = es_deconv(k2, g.nf2, g.w, g.beta);
        int p2 = k2 % g.nf2;
        if (p2 < 0) p2 += g.nf2;
        colp2[c] = p2;
        p2col[p2] = c;
    }
    // the fine columns without a mode column form one run when the mode columns are the two
    // ends of the fine grid (non-negative k2 first, negative k2 last)
    {
        int lo = g.nf2, hi = -1, n = 0;
        for (int q = 0; q < g.nf2; ++q)
            if (p2col[q] < 0) {
                lo = std::min(lo, q);
                hi = std::max(hi, q);
                ++n;
            }
        g.gap_lo = n ? lo : 0;
        g.gap_hi = n ? hi + 1 : 0;
        g.gap_ok = (n == 0 || hi + 1 - lo == n) ? 1 : 0;
    }
    PF_TRY(upload(d.mult1, mult1, s));
    PF_TRY(upload(d.dec2, dec2, s));
    PF_TRY(upload(d.colp2, colp2, s));
    PF_TRY(upload(d.p2col, p2col, s));
    return 0;
}

int validate_common(int64_t npts, int lmax, int ntrans, double tol) {
    if (npts < 1) return fail(PFSHT_ERR_ARGUMENT, "need at least one point");
    if (npts > INT32_MAX) return fail(PFSHT_ERR_ARGUMENT, "at most 2^31 - 1 points per plan");
    if (lmax < 0) return fail(PFSHT_ERR_ARGUMENT, "lmax must be nonnegative");
    if (ntrans < 1) return fail(PFSHT_ERR_ARGUMENT, "ntrans must be >= 1");
    if (!(tol > 0) || !(tol < 1)) return fail(PFSHT_ERR_ARGUMENT, "tol must lie in (0, 1)");
    return 0;
}

void fill_info(pfsht_plan* p) {
    pfsht_plan_info& in = p->info;
    in = pfsht_plan_info{};
    in.kind = p->kind;
    in.flip = p->leaf.flip ? 1 : 0;
    in.lmax = p->L;
    in.ntrans = p->B;
    in.precision = p->precision;
    in.npts = p->M;
    in.tol = p->tol;
    in.spin = p->spin;
    if (p->kind == kMultiBox) {
        for (const auto& c : p->boxes) {
            in.ring_work += c->info.ring_work;
            in.device_bytes += c->info.device_bytes;
        }
        in.device_bytes += (int64_t)(p->gidx.bytes + p->fg.bytes + p->acc.bytes + p->st_alm.bytes +
                                     p->st_f.bytes + p->st_alm2.bytes + p->st_f2.bytes);
        return;
    }
    if (p->kind == kDirect) {
        in.nrings = (int)p->M;
        in.mmax = p->L;
        in.ring_work = 0;
    } else {
        const Leaf& lf = p->leaf;
        in.nth_half = lf.nth_half;
        in.nth = lf.nth;
        in.nph = lf.nph;
        in.mmax = lf.mmax;
        in.nrings = lf.nth_half;
        in.K = lf.g.K;
        in.ring_work = lf.ring_work;
        in.beta = lf.g.beta;
        in.h = lf.g.h;
        in.theta_lo = lf.g.lo;
        in.theta_hi = lf.g.hi;
        in.eps_apo = lf.g.eps_apo;
        in.Theta1 = lf.g.Theta1;
        in.sigma = lf.g.sigma;
        in.ThetaT = lf.g.ThetaT;
        in.nufft_w = p->ng.w;
        in.nufft_beta = p->ng.beta;
        in.nf1 = p->ng.nf1;
        in.nf2 = p->ng.nf2;
        in.row0 = p->ng.row0;
        in.nrows = p->ng.nrows;
        in.ncols = p->ng.ncols;
    }
    int64_t bytes = 0;
    for (const DevBuf* b : {&p->cos_t, &p->log2sin, &p->log2c, &p->w, &p->ab, &p->aboff, &p->fwd_items.items, &p->adj_items.items,
                            &p->adj_seg.ck_p, &p->adj_seg.ck_E,
                            &p->H, &p->phi_pts, &p->nd.pts, &p->nd.perm, &p->nd.binstart,
                            &p->nd.binorder, &p->nd.sorder, &p->nd.bslot, &p->nd.sslot,
                            &p->nd.iorder, &p->nd.ipts, &p->nd.iperm, &p->nd.counter,
                            &p->nd.colp2, &p->nd.p2col, &p->nd.mult1, &p->nd.dec2, &p->nd.pad,
                            &p->nd.U, &p->st_alm, &p->st_f, &p->ab_fwd, &p->st_alm2,
                            &p->st_f2, &p->blk_fwd_items, &p->blk_adj_items})
        bytes += (int64_t)b->bytes;
    in.device_bytes = bytes;
}

// Adjoint items: tiles of 32 * R rings whose sums add atomically when an order spans several;
// with the deterministic option, all retained rings of an order in one item when no order retains
// more than four tiles (the warp walks them tile after tile and adds each tile's sums to the
// previous ones in order: a pass without atomics, measured ~8% slower at lmax 2048); each order split into degree segments of about seg_degrees when the
// unsplit items would give fewer than ~8 warps per resident warp slot (12 per SM at the
// adjoint's register count). The saved recurrence state is bounded by 512 MiB; past that, or
// with seg_degrees < 0, the items stay whole.
// Degree-segment length of the adjoint's items, from a model of the ring pass: an item of d
// degrees whose lanes hold R rings costs d (6 R + 4) (the recurrence and the four sums per ring,
// the transpose-reduce per degree) plus 400 for its start (seed or saved state, ring data, first
// coefficients: about 60 degrees' work); items are dealt heaviest first to the resident warp
// slots, and the segment length of 64 q degrees (q = 2..8) with the shortest schedule wins.
// Measured against fixed lengths at lmax 256 / 1024 / 2048, the adjoint's best lengths were
// 128 / 128 / 448 degrees (0.021 / 0.066 / 0.263 ms against 0.031 / 0.074 / 0.270 ms at 256),
// which the model picks.
static int choose_segment_degrees(const std::vector<int>& jlo, const std::vector<int>& jhi, int L,
                                  int mmax, int tile, int rmax, int slots) {
    std::vector<double> cost;
    double best = 0.0;
    int best_q = 0;
    for (int q = 2; q <= 8; ++q) {
        cost.clear();
        for (int m = 0; m <= std::min(mmax, L); ++m) {
            if (jhi[m] < jlo[m]) continue;
            const int nb = L >= m + 2 ? (L - m - 1 + 63) / 64 : 0;
            const int K = std::max(1, std::min(nb, (nb + q / 2) / q));
            for (int j0 = jlo[m]; j0 <= jhi[m]; j0 += tile) {
                const int n = std::min(tile, jhi[m] - j0 + 1);
                for (int base = 0; base < n; base += 32 * rmax) {
                    const int reff = (std::min(32 * rmax, n - base) + 31) / 32;
                    const int R = reff >= 3 ? 4 : reff;
                    for (int k = 0; k < K; ++k) {
                        const int first = k == 0 ? m : m + 2 + 64 * (int)(((int64_t)k * nb) / K);
                        const int last = k + 1 < K ? m + 1 + 64 * (int)(((int64_t)(k + 1) * nb) / K) : L;
                        cost.push_back((double)(last - first + 1) * (6.0 * R + 4.0) + 400.0);
                    }
                }
            }
        }
        std::sort(cost.begin(), cost.end(), std::greater<double>());
        std::priority_queue<double, std::vector<double>, std::greater<double>> busy;
        for (int w = 0; w < slots; ++w) busy.push(0.0);
        double span = 0.0;
        for (double c : cost) {
            const double t = busy.top() + c;
            busy.pop();
            busy.push(t);
            span = std::max(span, t);
        }
        if (best_q == 0 || span < best) {
            best = span;
            best_q = q;
        }
    }
    return 64 * best_q;
}

int build_adjoint_items(pfsht_plan* p, const std::vector<int>& jlo, const std::vector<int>& jhi,
                        int mmax, cudaStream_t s) {
    const int L = p->L;
    const int rmax = p->R > 0 ? p->R : 4;
    int maxret = 0;
    for (int m = 0; m <= std::min(mmax, L); ++m) maxret = std::max(maxret, jhi[m] - jlo[m] + 1);
    const int tile = p->deterministic && maxret <= 4 * 32 * rmax ? std::max(maxret, 1) : 32 * rmax;
    int seg = p->seg_degrees;
    if (seg == 0) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
        const size_t whole = make_ring_items(jlo, jhi, L, mmax, tile).size();
        seg = whole >= (size_t)sms * 12 * 8 ? -1
                                            : choose_segment_degrees(jlo, jhi, L, mmax, tile, rmax, sms * 11);
    }
    if (seg > 0) {
        PF_TRY(build_ring_segments(p->rt, jlo, jhi, L, mmax, seg, (int64_t)512 << 20, p->adj_seg, s));
        p->rt.ck_p = p->adj_seg.ck_p.as<double2>();
        p->rt.ck_E = p->adj_seg.ck_E.as<int>();
    }
    return build_ring_items(jlo, jhi, L, mmax, rmax, p->adj_items, s,
                            p->adj_seg.seg_degrees > 0 ? &p->adj_seg : nullptr, tile);
}

int build_stretch(pfsht_plan* p, const double* d_theta, const double* d_phi, const pfsht_opts& o,
                  cudaStream_t s) {
    Leaf& lf = p->leaf;
    const int L = p->L, B = p->B;
    p->kind = lf.g.kind;
    p->nrings = lf.nth_half;
    PF_TRY(upload(p->w, lf.w, s));
    if (p->spin != 0) {
        // the Wigner-d ring pass (spin.cu) in FP64 whatever the precision mode; tiles of 128 rings
        PF_TRY(build_spin_tables(lf.theta_rings, lf.flip, L, p->spin, p->spt, s));
        p->spt.t.w = p->w.as<double>();
        PF_TRY(build_spin_items(lf.jlo, lf.jhi, L, p->spin, 128, p->fwd_items, s));
    } else {
        PF_TRY(upload(p->cos_t, lf.cos_t, s));
        PF_TRY(upload(p->log2sin, lf.log2sin, s));
        PF_TRY(upload(p->log2c, lf.log2c, s));
        const bool mix = p->precision == PFSHT_PRECISION_MIXED;
        PF_TRY(build_ab_table(L, lf.mmax, mix ? 16 : 64, p->ab, p->aboff, s));
        p->rt.mix = mix;
        p->rt.stride = mix ? 16 : 64;
        p->rt.cos_t = p->cos_t.as<double>();
        p->rt.log2sin = p->log2sin.as<double>();
        p->rt.log2c = p->log2c.as<double>();
        p->rt.w = p->w.as<double>();
        p->rt.ab = p->ab.as<double2>();
        p->rt.aboff = p->aboff.as<int64_t>();
        p->rt.lmax = L;
        p->rt.nrings = lf.nth_half;
        // forward tiles of 64 rings in the FP64 form (more warps) and of 128 in the mixed form
        // (measured faster), adjoint tiles of 128 (amortises its reduction), split along the
        // degree axis when the tiles alone leave the GPU under-filled
        p->rt_fwd = p->rt;
        if (mix) {
            DevBuf off_unused;  // the offsets equal p->aboff (they depend on lmax and mmax only)
            PF_TRY(build_ab_table(L, lf.mmax, 64, p->ab_fwd, off_unused, s));
            p->rt_fwd.ab = p->ab_fwd.as<double2>();
            p->rt_fwd.mix = 0;
            p->rt_fwd.stride = 64;
        }
        PF_TRY(build_ring_items(lf.jlo, lf.jhi, L, lf.mmax, p->R > 0 ? p->R : 2, p->fwd_items, s));
        PF_TRY(build_adjoint_items(p, lf.jlo, lf.jhi, lf.mmax, s));
    }
    p->ncols = 2 * lf.mmax + 1;
    p->ro_cols.ld = lf.nth;
    p->ro_cols.bstride = (int64_t)lf.nth * p->ncols;
    p->ro_cols.col_off = lf.mmax;
    p->ro_cols.nrows = lf.nth;
    p->ro_cols.reflect = lf.g.kind == kInterior ? 0 : 1;
    // the DFS mirror rows carry (-1)^s (src/DFS.jl:13-33)
    p->ro_cols.spin_sgn = (p->spin & 1) ? -1.0 : 1.0;
    p->ro_cols.nrings_out = lf.nth_half;
    p->ro_cols.zero_rest = 1;
    PF_TRY(p->H.alloc(sizeof(double2) * (size_t)lf.nth * p->ncols * B));
    int n[1] = {lf.nth};
    PF_CUFFT(cufftPlanMany(&p->fth, 1, n, n, 1, lf.nth, n, 1, lf.nth, CUFFT_Z2Z, p->ncols * B));
    p->have_fth = true;

    // points: stretched colatitude and longitude on the device (src/Stretch.jl:202-213)
    DevBuf Th, ph;
    PF_TRY(Th.alloc(sizeof(double) * p->M));
    PF_TRY(ph.alloc(sizeof(double) * p->M));
    PF_TRY(leaf_points(lf.g, lf.flip, d_theta, d_phi, p->M, Th.as<double>(), ph.as<double>(), s));
    double Tmin = 0, Tmax = 0;
    PF_TRY(minmax_device(Th.as<double>(), p->M, &Tmin, &Tmax, s));

    // half-cell phase and 1/n_theta per Theta mode (src/Stretch.jl:229-233 with the n_phi of
    // the phi round trip cancelled)
    const double shift = lf.g.kind == kInterior ? 0.0 : M_PI / lf.nth;
    std::vector<double2> phase(lf.nth);
    for (int i = 0; i < lf.nth; ++i) {
        const double a = -(double)mode_k(i, lf.nth) * shift;
        phase[i] = make_double2(std::cos(a) / lf.nth, std::sin(a) / lf.nth);
    }
    std::vector<int> colk2(p->ncols);
    for (int c = 0; c < p->ncols; ++c) colk2[c] = c - lf.mmax;
    PF_TRY(setup_nufft_grid(p->ng, p->nd, lf.nth, lf.nph, colk2, phase, p->tol, p->M, Tmin, Tmax,
                            false, o.nufft_bin_rows, o.nufft_bin_cols,
                            p->precision == PFSHT_PRECISION_MIXED, o.nufft_fft_lengths, o.nufft_nf1,
                            o.nufft_nf2, s));
    PF_TRY(nufft_setpts(p->ng, p->nd, Th.as<double>(), ph.as<double>(), s));
    p->ng.plain_transpose = o.nufft_transpose == 1 ? 1 : 0;
    p->ng.spread_reg = o.nufft_spread == 1 ? 0 : 1;
    p->ng.deterministic = p->deterministic;
    PF_TRY(nufft_alloc(p->ng, p->nd, B));
    return 0;
}

// the Direct leaf's ring set: every point a ring, every order on every point (eps = 0,
// src/Direct.jl:43-44)
int build_direct_rings(pfsht_plan* p, const double* h_theta, cudaStream_t s) {
    const int L = p->L;
    const int64_t M = p->M;
    std::vector<int> jlo(L + 1, 0), jhi(L + 1, (int)M - 1);
    if (p->spin != 0) {
        // SpinDirectLeaf (src/Spin.jl:557-630); the points keep their order (the walk needs no
        // sorted rings)
        std::vector<double> th(h_theta, h_theta + M);
        PF_TRY(build_spin_tables(th, false, L, p->spin, p->spt, s));
        p->spt.t.w = nullptr;
        return build_spin_items(jlo, jhi, L, p->spin, 128, p->fwd_items, s);
    }
    std::vector<double> cs(M), l2s(M);
    for (int64_t i = 0; i < M; ++i) {
        const double sn = std::sin(h_theta[i]), c = std::cos(h_theta[i]);
        const double as = std::fabs(sn);
        cs[i] = c;
        l2s[i] = as > 0 ? std::log2(as) : -INFINITY;
    }
    std::vector<double> l2c;
    sectorial_log2c(L, l2c);
    PF_TRY(upload(p->cos_t, cs, s));
    PF_TRY(upload(p->log2sin, l2s, s));
    PF_TRY(upload(p->log2c, l2c, s));
    const bool mix = p->precision == PFSHT_PRECISION_MIXED;
    PF_TRY(build_ab_table(L, L, mix ? 16 : 64, p->ab, p->aboff, s));
    p->rt.mix = mix;
    p->rt.stride = mix ? 16 : 64;
    p->rt.cos_t = p->cos_t.as<double>();
    p->rt.log2sin = p->log2sin.as<double>();
    p->rt.log2c = p->log2c.as<double>();
    p->rt.w = nullptr;
    p->rt.ab = p->ab.as<double2>();
    p->rt.aboff = p->aboff.as<int64_t>();
    p->rt.lmax = L;
    p->rt.nrings = (int)M;
    p->rt_fwd = p->rt;
    PF_TRY(build_ring_items(jlo, jhi, L, L, p->R > 0 ? p->R : 2, p->fwd_items, s));
    return build_adjoint_items(p, jlo, jhi, L, s);
}

int build_direct(pfsht_plan* p, const double* h_theta, const double* h_phi, cudaStream_t s) {
    const int L = p->L, B = p->B;
    const int64_t M = p->M;
    if (M > INT32_MAX) return fail(PFSHT_ERR_ARGUMENT, "too many points for the direct method");
    p->kind = kDirect;
    p->nrings = (int)M;
    PF_TRY(build_direct_rings(p, h_theta, s));
    PF_TRY(upload(p->phi_pts, std::vector<double>(h_phi, h_phi + M), s));
    p->ncols = 2 * L + 1;
    p->ro_cols.ld = M;
    p->ro_cols.bstride = M * (2 * L + 1);
    p->ro_cols.col_off = L;
    p->ro_cols.nrows = (int)M;
    p->ro_cols.reflect = 0;
    p->ro_cols.spin_sgn = 1.0;
    p->ro_cols.nrings_out = (int)M;
    p->ro_cols.zero_rest = 0;  // every point keeps every order
    PF_TRY(p->H.alloc(sizeof(double2) * (size_t)M * (2 * L + 1) * B));
    return 0;
}

int plan_create(const double* theta, const double* phi, int64_t npts, int lmax, int ntrans,
                double tol, int precision, const pfsht_opts* opts_in, pfsht_plan** out);

// point sets from this size on are planned by the device scans (planner_dev.cu)
constexpr int64_t kDevicePlannerMin = 1 << 15;

// MultiBoxLeaf (src/MultiBox.jl:32-66): one stretched-leaf plan per group of the partition
int build_multibox(pfsht_plan* p, const Partition& part, const double* th, const double* ph,
                   int precision, const pfsht_opts& o) {
    p->kind = kMultiBox;
    const int nb = (int)part.groups.size();
    if (nb < 1) return fail(PFSHT_ERR_ARGUMENT, "partition produced no boxes");
    p->box_off.assign(nb + 1, 0);
    std::vector<int32_t> idx;
    idx.reserve(p->M);
    for (int i = 0; i < nb; ++i) {
        const std::vector<int32_t>& g = part.groups[i];
        std::vector<double> tg(g.size()), pg(g.size());
        for (size_t k = 0; k < g.size(); ++k) {
            tg[k] = th[g[k]];
            pg[k] = ph[g[k]];
        }
        pfsht_opts oc = o;
        oc.method = PFSHT_METHOD_STRETCH;
        oc.points_on_device = 0;
        oc.device = p->device;
        pfsht_plan* c = nullptr;
        PF_TRY(plan_create(tg.data(), pg.data(), (int64_t)g.size(), p->L, p->B, p->tol, precision,
                           &oc, &c));
        p->boxes.emplace_back(c);
        idx.insert(idx.end(), g.begin(), g.end());
        p->box_off[i + 1] = p->box_off[i] + (int64_t)g.size();
    }
    p->precision = p->boxes[0]->precision;
    PF_TRY(upload(p->gidx, idx, p->st_stream));
    PF_TRY(p->fg.alloc(sizeof(double2) * (size_t)p->M * p->B));
    if (nb > 1) PF_TRY(p->acc.alloc(sizeof(double2) * (size_t)(p->L + 1) * (2 * p->L + 1) * p->B));
    return 0;
}

// the same from a partition computed on the device: each box's points are gathered on the device
// and its plan is built from them there
__global__ void gather_points_by_index(const double* __restrict__ th, const double* __restrict__ ph,
                                       const int* __restrict__ idx, int64_t n, double* __restrict__ tg,
                                       double* __restrict__ pg) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        tg[t] = th[idx[t]];
        pg[t] = ph[idx[t]];
    }
}

int build_multibox_device(pfsht_plan* p, const DevPartition& part, const double* th, const double* ph,
                          int precision, const pfsht_opts& o) {
    p->kind = kMultiBox;
    const int nb = (int)part.idx.size();
    if (nb < 1) return fail(PFSHT_ERR_ARGUMENT, "partition produced no boxes");
    cudaStream_t s = p->st_stream;
    p->box_off.assign(nb + 1, 0);
    for (int i = 0; i < nb; ++i) p->box_off[i + 1] = p->box_off[i] + part.n[i];
    PF_TRY(p->gidx.alloc(sizeof(int32_t) * (size_t)p->M));
    for (int i = 0; i < nb; ++i) {
        const int64_t n = part.n[i];
        PF_CUDA(cudaMemcpyAsync(p->gidx.as<int32_t>() + p->box_off[i], part.idx[i]->p, sizeof(int32_t) * n,
                                cudaMemcpyDeviceToDevice, s));
        DevBuf tg, pg;
        PF_TRY(tg.alloc(sizeof(double) * n));
        PF_TRY(pg.alloc(sizeof(double) * n));
        gather_points_by_index<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(
            th, ph, part.idx[i]->as<int>(), n, tg.as<double>(), pg.as<double>());
        PF_TRY(check_launch("gather_points_by_index"));
        PF_CUDA(cudaStreamSynchronize(s));
        pfsht_opts oc = o;
        oc.method = PFSHT_METHOD_STRETCH;
        oc.points_on_device = 1;
        oc.device = p->device;
        pfsht_plan* c = nullptr;
        PF_TRY(plan_create(tg.as<double>(), pg.as<double>(), n, p->L, p->B, p->tol, precision, &oc, &c));
        p->boxes.emplace_back(c);
    }
    p->precision = p->boxes[0]->precision;
    PF_TRY(p->fg.alloc(sizeof(double2) * (size_t)p->M * p->B));
    if (nb > 1) PF_TRY(p->acc.alloc(sizeof(double2) * (size_t)(p->L + 1) * (2 * p->L + 1) * p->B));
    PF_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// f[idx[j], b] = fg[j, b] (the boxes' fields are a disjoint union, src/MultiBox.jl:83-94)
__global__ void box_scatter_kernel(const double2* __restrict__ fg, const int* __restrict__ idx,
                                   int64_t mb, int64_t M, int B, double2* __restrict__ f) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < mb * B;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / mb, j = t - b * mb;
        f[idx[j] + M * b] = fg[t];
    }
}

// fg[j, b] = f[idx[j], b]
__global__ void box_gather_kernel(const double2* __restrict__ f, const int* __restrict__ idx,
                                  int64_t mb, int64_t M, int B, double2* __restrict__ fg) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < mb * B;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / mb, j = t - b * mb;
        fg[t] = f[idx[j] + M * b];
    }
}

// a += c (the adjoint sums the boxes' coefficient arrays, src/MultiBox.jl:96-110)
__global__ void coeff_add_kernel(double2* __restrict__ a, const double2* __restrict__ c, int64_t n) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const double2 x = a[t], y = c[t];
        a[t] = make_double2(x.x + y.x, x.y + y.y);
    }
}

// blocks of 256 threads for n elements (grid-stride loops beyond 148 x 16 blocks)
unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

int apply_forward(pfsht_plan* p, const double2* alm, double2* f, cudaStream_t s);
int apply_adjoint(pfsht_plan* p, const double2* f, double2* alm, cudaStream_t s);

int multibox_forward(pfsht_plan* p, const double2* alm, double2* f, cudaStream_t s) {
    for (size_t i = 0; i < p->boxes.size(); ++i) {
        const int64_t mb = p->box_off[i + 1] - p->box_off[i];
        double2* fgi = p->fg.as<double2>() + p->B * p->box_off[i];
        PF_TRY(apply_forward(p->boxes[i].get(), alm, fgi, s));
        box_scatter_kernel<<<grid_for(mb * p->B), 256, 0, s>>>(
            fgi, p->gidx.as<int>() + p->box_off[i], mb, p->M, p->B, f);
        PF_TRY(check_launch("box_scatter_kernel"));
    }
    return 0;
}

int multibox_adjoint(pfsht_plan* p, const double2* f, double2* alm, cudaStream_t s) {
    const int64_t nc = (int64_t)(p->L + 1) * (2 * p->L + 1) * p->B;
    for (size_t i = 0; i < p->boxes.size(); ++i) {
        const int64_t mb = p->box_off[i + 1] - p->box_off[i];
        double2* fgi = p->fg.as<double2>() + p->B * p->box_off[i];
        box_gather_kernel<<<grid_for(mb * p->B), 256, 0, s>>>(
            f, p->gidx.as<int>() + p->box_off[i], mb, p->M, p->B, fgi);
        PF_TRY(check_launch("box_gather_kernel"));
        // each box's adjoint overwrites its output: the first writes alm, the others are added
        PF_TRY(apply_adjoint(p->boxes[i].get(), fgi, i == 0 ? alm : p->acc.as<double2>(), s));
        if (i > 0) {
            coeff_add_kernel<<<grid_for(nc), 256, 0, s>>>(alm, p->acc.as<double2>(), nc);
            PF_TRY(check_launch("coeff_add_kernel"));
        }
    }
    return 0;
}

int plan_create(const double* theta, const double* phi, int64_t npts, int lmax, int ntrans,
                double tol, int precision, const pfsht_opts* opts_in, pfsht_plan** out) {
    if (!out) return fail(PFSHT_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!theta || !phi) return fail(PFSHT_ERR_ARGUMENT, "theta and phi must not be NULL");
    PF_TRY(validate_common(npts, lmax, ntrans, tol));
    if (precision != PFSHT_PRECISION_FP64 && precision != PFSHT_PRECISION_MIXED)
        return fail(PFSHT_ERR_ARGUMENT, "unknown precision mode");
    pfsht_opts o;
    pfsht_opts_default(&o);
    if (opts_in) o = *opts_in;
    if (o.method < 0 || o.method > 3) return fail(PFSHT_ERR_ARGUMENT, "unknown method");
    if (!(o.oversample_theta >= 1) || !(o.oversample_phi >= 1))
        return fail(PFSHT_ERR_ARGUMENT, "oversampling factors must be >= 1");
    if (!(o.eps_apo_max > 0)) return fail(PFSHT_ERR_ARGUMENT, "eps_apo_max must be positive");
    if (o.spin != 0 && std::abs(o.spin) > lmax)
        return fail(PFSHT_ERR_ARGUMENT, "(|spin| = " + std::to_string(std::abs(o.spin)) +
                                            ") > lmax = " + std::to_string(lmax));
    if (o.nufft_fft_lengths < 0 || o.nufft_fft_lengths > 2)
        return fail(PFSHT_ERR_ARGUMENT, "nufft_fft_lengths must be 0 (timed), 1 (minimal) or 2 (given)");
    DeviceGuard dg(o.device);
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));

    std::unique_ptr<pfsht_plan> p(new pfsht_plan());
    p->device = dev;
    // the mixed form applies where the tolerance allows FP32 (tol >= 1e-6); below that the
    // plan runs the FP64 form and reports so in its info
    p->precision = (precision == PFSHT_PRECISION_MIXED && tol >= 1e-6) ? PFSHT_PRECISION_MIXED
                                                                        : PFSHT_PRECISION_FP64;
    p->L = lmax;
    p->B = ntrans;
    p->M = npts;
    p->tol = tol;
    p->R = o.ring_rings_per_lane == 2 || o.ring_rings_per_lane == 4 || o.ring_rings_per_lane == 8
               ? o.ring_rings_per_lane : 0;
    p->seg_degrees = o.ring_segment_degrees;
    p->deterministic = o.deterministic ? 1 : 0;
    p->spin = o.spin;
    PF_CUDA(cudaStreamCreateWithFlags(&p->st_stream, cudaStreamNonBlocking));
    PF_CUDA(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
    PF_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
    PF_CUDA(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
    cudaStream_t s = p->st_stream;

    // host and device copies of the points
    std::vector<double> h_theta, h_phi;
    DevBuf d_theta, d_phi;
    const double* dth;
    const double* dph;
    double lo, hi;
    if (o.points_on_device) {
        dth = theta;
        dph = phi;
        PF_TRY(minmax_device(theta, npts, &lo, &hi, s));
    } else {
        PF_TRY(d_theta.alloc(sizeof(double) * npts));
        PF_TRY(d_phi.alloc(sizeof(double) * npts));
        PF_CUDA(cudaMemcpyAsync(d_theta.p, theta, sizeof(double) * npts, cudaMemcpyHostToDevice, s));
        PF_CUDA(cudaMemcpyAsync(d_phi.p, phi, sizeof(double) * npts, cudaMemcpyHostToDevice, s));
        dth = d_theta.as<double>();
        dph = d_phi.as<double>();
        lo = INFINITY;
        hi = -INFINITY;
        for (int64_t i = 0; i < npts; ++i) {
            lo = std::fmin(lo, theta[i]);
            hi = std::fmax(hi, theta[i]);
        }
    }
    if (!(std::isfinite(lo) && std::isfinite(hi)))
        return fail(PFSHT_ERR_ARGUMENT, "colatitudes must be finite");
    // bounding_box colatitude extent (src/Box.jl:51-59)
    lo = std::fmax(lo, 0.0);
    hi = std::fmin(hi, M_PI);

    // the planner reads the points on the host (src/Cost.jl:171-201)
    const double* hth = theta;
    const double* hph = phi;
    auto host_points = [&]() -> int {
        if (!o.points_on_device) return 0;
        if (h_theta.empty()) {
            h_theta.resize(npts);
            h_phi.resize(npts);
            PF_CUDA(cudaMemcpyAsync(h_theta.data(), theta, sizeof(double) * npts, cudaMemcpyDeviceToHost, s));
            PF_CUDA(cudaMemcpyAsync(h_phi.data(), phi, sizeof(double) * npts, cudaMemcpyDeviceToHost, s));
            PF_CUDA(cudaStreamSynchronize(s));
        }
        hth = h_theta.data();
        hph = h_phi.data();
        return 0;
    };
    int method = o.method;
    const int mb = o.maxboxes > 0 ? o.maxboxes : 8;
    if (npts >= kDevicePlannerMin) {
        // large point sets: the planner's scans run on the device copies of the points
        DevPartition dpart;
        bool have_dpart = false;
        if (method == PFSHT_METHOD_AUTO) {
            PF_TRY(select_method_device(dth, dph, npts, lmax, ntrans, tol, s, &method, &dpart));
            have_dpart = true;
        }
        if (method == PFSHT_METHOD_MULTIBOX) {
            if (!have_dpart || mb != 8)
                PF_TRY(partition_boxes_device(dth, dph, npts, lmax, ntrans, tol, mb, s, dpart));
            PF_TRY(build_multibox_device(p.get(), dpart, dth, dph, precision, o));
            PF_CUDA(cudaStreamSynchronize(s));
            fill_info(p.get());
            *out = p.release();
            return 0;
        }
    }
    Partition part;
    bool have_part = false;
    if (method == PFSHT_METHOD_AUTO) {
        PF_TRY(host_points());
        method = select_method(hth, hph, npts, lmax, ntrans, tol, &part);
        have_part = true;
    }
    if (method == PFSHT_METHOD_MULTIBOX) {
        PF_TRY(host_points());
        if (!have_part || mb != 8) partition_boxes_costed(hth, hph, npts, lmax, ntrans, tol, mb, part);
        PF_TRY(build_multibox(p.get(), part, hth, hph, precision, o));
        PF_CUDA(cudaStreamSynchronize(s));
        fill_info(p.get());
        *out = p.release();
        return 0;
    }
    bool direct = method == PFSHT_METHOD_DIRECT;
    if (!direct) {
        std::string err;
        int r = build_leaf(lo, hi, lmax, ntrans, tol, o.eps_apo_max, o.oversample_theta,
                           o.oversample_phi, &p->leaf, &err, o.spin);
        if (r == 2) return fail(PFSHT_ERR_ARGUMENT, err);
        if (r == 1) {
            if (o.method == PFSHT_METHOD_STRETCH) return fail(PFSHT_ERR_REFUSED, err);
            direct = true;  // what the reference's AutoAlgorithm answers (src/Cost.jl:121-122,184-186)
        }
    }
    if (direct) {
        PF_TRY(host_points());
        PF_TRY(build_direct(p.get(), hth, hph, s));
    } else {
        PF_TRY(build_stretch(p.get(), dth, dph, o, s));
    }
    PF_CUDA(cudaStreamSynchronize(s));
    fill_info(p.get());
    *out = p.release();
    return 0;
}

int apply_forward(pfsht_plan* p, const double2* alm, double2* f, cudaStream_t s) {
    if (p->kind == kMultiBox) return multibox_forward(p, alm, f, s);
    clock_begin(&p->clk, s);
    if (p->spin != 0)
        PF_TRY(spin_ring_forward(p->spt.t, p->ro_cols, p->fwd_items.view, alm, p->H.as<double2>(), p->B, s));
    else
        PF_TRY(ring_forward(p->rt_fwd, p->ro_cols, p->fwd_items.view, alm, p->H.as<double2>(), p->B, s));
    if (p->kind != kDirect) clock_mark(&p->clk, kStRingFwd, s);
    return plan_forward_after_ring(p, f, s);
}

int apply_adjoint(pfsht_plan* p, const double2* f, double2* alm, cudaStream_t s) {
    if (p->kind == kMultiBox) return multibox_adjoint(p, f, alm, s);
    // zero what the ring pass will not store on the side stream, overlapped with the NUFFT and
    // Theta-FFT stages (a bandwidth-bound fill beside compute-bound kernels); joined before the pass
    PF_CUDA(cudaEventRecord(p->ev_fork, s));
    PF_CUDA(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    if (p->spin != 0)
        PF_CUDA(cudaMemsetAsync(alm, 0, sizeof(double2) * (size_t)(p->L + 1) * (2 * p->L + 1) * p->B,
                                p->side));
    else
        PF_TRY(ring_adjoint_prepare(p->rt, p->adj_items.view, alm, p->B, p->side));
    PF_CUDA(cudaEventRecord(p->ev_join, p->side));
    clock_begin(&p->clk, s);
    PF_TRY(plan_adjoint_before_ring(p, f, s));
    PF_CUDA(cudaStreamWaitEvent(s, p->ev_join, 0));
    if (p->spin != 0)
        PF_TRY(spin_ring_adjoint(p->spt.t, p->ro_cols, p->fwd_items.view, p->H.as<double2>(), alm, p->B,
                                 s, false));
    else
        PF_TRY(ring_adjoint(p->rt, p->ro_cols, p->adj_items.view, p->H.as<double2>(), alm, p->B, s,
                            false));
    clock_mark(&p->clk, p->kind == kDirect ? kStDirect : kStRingAdj, s);
    return 0;
}

}  // namespace

namespace pf {

int plan_forward_after_ring(pfsht_plan* p, double2* f, cudaStream_t s) {
    StageClock* clk = &p->clk;
    if (p->kind == kDirect) {
        PF_TRY(direct_phase_sum(p->H.as<double2>(), p->phi_pts.as<double>(), p->M, p->L, p->B, f, s));
        clock_mark(clk, kStDirect, s);
        return 0;
    }
    PF_CUFFT(cufftSetStream(p->fth, s));
    PF_CUFFT(cufftExecZ2Z(p->fth, p->H.as<cufftDoubleComplex>(), p->H.as<cufftDoubleComplex>(),
                          CUFFT_FORWARD));
    clock_mark(clk, kStFftThetaFwd, s);
    return nufft_type2(p->ng, p->nd, p->H.as<double2>(), f, p->B, +1, s, clk);
}

int plan_adjoint_before_ring(pfsht_plan* p, const double2* f, cudaStream_t s) {
    StageClock* clk = &p->clk;
    if (p->kind == kDirect)
        return direct_phase_spread(f, p->phi_pts.as<double>(), p->M, p->L, p->B, p->H.as<double2>(), s);
    PF_TRY(nufft_type1(p->ng, p->nd, f, p->H.as<double2>(), p->B, -1, s, clk));
    PF_CUFFT(cufftSetStream(p->fth, s));
    PF_CUFFT(cufftExecZ2Z(p->fth, p->H.as<cufftDoubleComplex>(), p->H.as<cufftDoubleComplex>(),
                          CUFFT_INVERSE));
    clock_mark(clk, kStFftThetaAdj, s);
    return 0;
}

}  // namespace pf

extern "C" {

pfsht_status pfsht_opts_default(pfsht_opts* o) {
    if (!o) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "opts is NULL");
    std::memset(o, 0, sizeof(*o));
    o->method = PFSHT_METHOD_AUTO;
    o->points_on_device = 0;
    o->device = -1;
    o->ring_rings_per_lane = 0;
    o->nufft_bin_rows = 0;
    o->nufft_bin_cols = 0;
    o->oversample_theta = 1.0;
    o->oversample_phi = 1.0;
    o->eps_apo_max = 1.0;
    return PFSHT_OK;
}

pfsht_status pfsht_plan_create(const double* theta, const double* phi, int64_t npts, int32_t lmax,
                               int32_t ntrans, double tol, int32_t precision,
                               const pfsht_opts* opts, pfsht_plan** out) {
    return (pfsht_status)plan_create(theta, phi, npts, lmax, ntrans, tol, precision, opts, out);
}

pfsht_status pfsht_plan_destroy(pfsht_plan* p) {
    if (!p) return PFSHT_OK;
    DeviceGuard dg(p->device);
    delete p;
    return PFSHT_OK;
}

pfsht_status pfsht_forward(pfsht_plan* p, const void* alm, void* f, void* stream) {
    if (!p || !alm || !f) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    DeviceGuard dg(p->device);
    return (pfsht_status)apply_forward(p, (const double2*)alm, (double2*)f, (cudaStream_t)stream);
}

pfsht_status pfsht_adjoint(pfsht_plan* p, const void* f, void* alm, void* stream) {
    if (!p || !alm || !f) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    DeviceGuard dg(p->device);
    return (pfsht_status)apply_adjoint(p, (const double2*)f, (double2*)alm, (cudaStream_t)stream);
}

// The sph_mode coefficient array (src/Layout.jl:13-20) holds order m in the columns 2m - 1 and
// 2m, rows 0 .. lmax - m: a staircase filling half of the (lmax + 1) x (2 lmax + 1) array.
// Host copies move the orders up to the plan's highest retained order (host_mmax) as blocks of
// orders [m0, m1): the contiguous columns
// [max(0, 2 m0 - 1), 2 m1 - 1), rows 0 .. lmax - m0, one 2-D copy each. Blocks of about
// (lmax + 1) / 16 orders keep both the number of copies and the padding they carry small.
struct AlmBlock {
    int c0, c1, rows;
};
// blocks of the orders 0 .. mu
static std::vector<AlmBlock> alm_blocks(int L, int mu) {
    const int G = std::max(32, (L + 1 + 15) / 16);
    std::vector<AlmBlock> v;
    for (int m0 = 0; m0 <= mu; m0 += G) {
        const int m1 = std::min(mu + 1, m0 + G);
        v.push_back(AlmBlock{m0 == 0 ? 0 : 2 * m0 - 1, 2 * m1 - 1, L + 1 - m0});
    }
    return v;
}

// The highest order a plan's applies read or write: the retained orders of the polar truncation
// (src/Legendre.jl:48-57); the forward reads no coefficient of a higher order and the adjoint
// writes zeros there, so host applies move only the orders up to it and zero the rest on the host
static int host_mmax(const pfsht_plan* p) {
    if (p->kind == kMultiBox) {
        int mu = 0;
        for (const auto& c : p->boxes) mu = std::max(mu, host_mmax(c.get()));
        return mu;
    }
    if (p->kind == kDirect) return p->L;
    return std::min(p->L, p->leaf.mmax);
}

// bytes a host apply moves: the coefficient blocks of the orders up to host_mmax (for a spin
// plan, whose (l, m + lmax) layout has no staircase, the columns of those orders) and the field
static void host_bytes(const pfsht_plan* p, int64_t* alm_bytes, int64_t* f_bytes) {
    int64_t a = 0;
    const int mu = host_mmax(p);
    if (p->spin != 0) a = (int64_t)(p->L + 1) * (2 * mu + 1);
    else
        for (const AlmBlock& b : alm_blocks(p->L, mu)) a += (int64_t)b.rows * (b.c1 - b.c0);
    *alm_bytes = a * (int64_t)sizeof(double2) * p->B;
    *f_bytes = (int64_t)sizeof(double2) * p->M * p->B;
}

static int alm_copy(pfsht_plan* p, void* host, double2* dev, bool to_device, cudaStream_t s) {
    const int L = p->L;
    const int mu = host_mmax(p);
    const size_t col = sizeof(double2) * (size_t)(L + 1);
    const size_t tr = col * (2 * L + 1);
    char* h = static_cast<char*>(host);
    char* d = reinterpret_cast<char*>(dev);
    if (p->spin != 0) {
        // columns m + lmax for m = -mu .. mu, contiguous in each transform
        const size_t off = col * (size_t)(L - mu), n = col * (size_t)(2 * mu + 1);
        for (int b = 0; b < p->B; ++b) {
            if (to_device) PF_CUDA(cudaMemcpyAsync(d + tr * b + off, h + tr * b + off, n, cudaMemcpyHostToDevice, s));
            else PF_CUDA(cudaMemcpyAsync(h + tr * b + off, d + tr * b + off, n, cudaMemcpyDeviceToHost, s));
        }
        return 0;
    }
    for (int b = 0; b < p->B; ++b) {
        for (const AlmBlock& k : alm_blocks(L, mu)) {
            const size_t off = tr * b + col * k.c0;
            const size_t width = sizeof(double2) * (size_t)k.rows;
            if (to_device)
                PF_CUDA(cudaMemcpy2DAsync(d + off, col, h + off, col, width, k.c1 - k.c0,
                                          cudaMemcpyHostToDevice, s));
            else
                PF_CUDA(cudaMemcpy2DAsync(h + off, col, d + off, col, width, k.c1 - k.c0,
                                          cudaMemcpyDeviceToHost, s));
        }
    }
    return 0;
}

// zero what the block copies leave out of the host array (rows past each block's height, and the
// columns of orders above host_mmax), on host threads while the copies run
static void alm_zero_host_padding(const pfsht_plan* p, void* host) {
    const int L = p->L;
    const int mu = host_mmax(p);
    std::vector<int> rows(2 * L + 1, 0);
    if (p->spin != 0) {
        for (int c = L - mu; c <= L + mu; ++c) rows[c] = L + 1;  // copied whole
    } else {
        for (const AlmBlock& k : alm_blocks(L, mu))
            for (int c = k.c0; c < k.c1; ++c) rows[c] = k.rows;
    }
    double2* h = static_cast<double2*>(host);
    const int64_t ncol = (int64_t)(2 * L + 1) * p->B;
#pragma omp parallel for schedule(static) num_threads(16) if (ncol > 512)
    for (int64_t q = 0; q < ncol; ++q) {
        const int c = (int)(q % (2 * L + 1));
        if (rows[c] <= L)
            std::memset(h + q * (L + 1) + rows[c], 0, sizeof(double2) * (size_t)(L + 1 - rows[c]));
    }
}

}  // extern "C"

namespace pf {

// copy order block k of the coefficient staircase (all transforms) between host and device
static int alm_copy_block(pfsht_plan* p, const AlmBlock& k, void* host, double2* dev, bool to_device,
                          cudaStream_t s) {
    const int L = p->L;
    const size_t col = sizeof(double2) * (size_t)(L + 1);
    const size_t tr = col * (2 * L + 1);
    char* h = static_cast<char*>(host);
    char* d = reinterpret_cast<char*>(dev);
    for (int b = 0; b < p->B; ++b) {
        const size_t off = tr * b + col * k.c0;
        const size_t width = sizeof(double2) * (size_t)k.rows;
        if (to_device)
            PF_CUDA(cudaMemcpy2DAsync(d + off, col, h + off, col, width, k.c1 - k.c0,
                                      cudaMemcpyHostToDevice, s));
        else
            PF_CUDA(cudaMemcpy2DAsync(h + off, col, d + off, col, width, k.c1 - k.c0,
                                      cudaMemcpyDeviceToHost, s));
    }
    return 0;
}

// ring items grouped by the order blocks of the host copies, each group in its launch order
static int group_items_by_block(pfsht_plan* p, const std::vector<RingItem>& items,
                                const std::vector<AlmBlock>& blocks, DevBuf& out,
                                std::vector<int>& off) {
    std::vector<RingItem> v;
    v.reserve(items.size());
    off.assign(blocks.size() + 1, 0);
    for (size_t k = 0; k < blocks.size(); ++k) {
        const int m0 = (blocks[k].c0 + 1) / 2, m1 = (blocks[k].c1 + 1) / 2;
        for (const RingItem& it : items)
            if (it.m >= m0 && it.m < m1) v.push_back(it);
        off[k + 1] = (int)v.size();
    }
    if (v.size() != items.size()) return fail(PFSHT_ERR_ARGUMENT, "ring items outside the copied orders");
    PF_TRY(out.alloc(sizeof(RingItem) * std::max<size_t>(v.size(), 1)));
    if (!v.empty())
        PF_CUDA(cudaMemcpyAsync(out.p, v.data(), sizeof(RingItem) * v.size(), cudaMemcpyHostToDevice,
                                p->st_stream));
    PF_CUDA(cudaStreamSynchronize(p->st_stream));
    return 0;
}

int plan_host_staging(pfsht_plan* p) {
    const size_t na = sizeof(double2) * (size_t)(p->L + 1) * (2 * p->L + 1) * p->B;
    const size_t nf = sizeof(double2) * (size_t)p->M * p->B;
    if (!p->st_alm.p) PF_TRY(p->st_alm.alloc(na));
    if (!p->st_f.p) PF_TRY(p->st_f.alloc(nf));
    if (!p->st_alm2.p) PF_TRY(p->st_alm2.alloc(na));
    if (!p->st_f2.p) PF_TRY(p->st_f2.alloc(nf));
    if (!p->h2d) {
        PF_CUDA(cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking));
        PF_CUDA(cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&p->ev_alm_in_free, &p->ev_f_out_free, &p->ev_f_in_free,
                               &p->ev_alm_out_free, &p->ev_fwd_done, &p->ev_f_in_ready, &p->ev_copied})
            PF_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    // the blocked ring passes: stretched scalar leaves (spin, Direct and MultiBox plans copy
    // whole and apply on the compute stream)
    const bool blocked = p->kind != kDirect && p->kind != kMultiBox && p->spin == 0;
    if (blocked && !p->host_pipeline) {
        const std::vector<AlmBlock> blocks = alm_blocks(p->L, host_mmax(p));
        PF_TRY(group_items_by_block(p, p->fwd_items.host, blocks, p->blk_fwd_items, p->blk_fwd_off));
        PF_TRY(group_items_by_block(p, p->adj_items.host, blocks, p->blk_adj_items, p->blk_adj_off));
        p->ev_blk.assign(blocks.size(), nullptr);
        for (cudaEvent_t& e : p->ev_blk) PF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        p->host_pipeline = true;
    }
    return 0;
}

// the forward from host coefficients: each order block's copy on h2d, joined by an event before
// the ring items of its orders on s; the field copied back on d2h once the forward ends
static int host_forward_pipelined(pfsht_plan* p, const void* in, void* out, cudaStream_t s) {
    const std::vector<AlmBlock> blocks = alm_blocks(p->L, host_mmax(p));
    const size_t nf = sizeof(double2) * (size_t)p->M * p->B;
    double2* alm = p->st_alm.as<double2>();
    // the previous forward's ring pass has finished reading the staging coefficients
    PF_CUDA(cudaStreamWaitEvent(p->h2d, p->ev_alm_in_free, 0));
    for (size_t k = 0; k < blocks.size(); ++k) {
        PF_TRY(alm_copy_block(p, blocks[k], const_cast<void*>(in), alm, true, p->h2d));
        PF_CUDA(cudaEventRecord(p->ev_blk[k], p->h2d));
    }
    clock_begin(&p->clk, s);
    for (size_t k = 0; k < blocks.size(); ++k) {
        PF_CUDA(cudaStreamWaitEvent(s, p->ev_blk[k], 0));
        RingItems v = p->fwd_items.view;
        v.items = p->blk_fwd_items.as<RingItem>() + p->blk_fwd_off[k];
        v.nitems = p->blk_fwd_off[k + 1] - p->blk_fwd_off[k];
        PF_TRY(ring_forward(p->rt_fwd, p->ro_cols, v, alm, p->H.as<double2>(), p->B, s));
    }
    clock_mark(&p->clk, kStRingFwd, s);
    PF_CUDA(cudaEventRecord(p->ev_alm_in_free, s));
    // the previous forward's field has left the staging buffer
    PF_CUDA(cudaStreamWaitEvent(s, p->ev_f_out_free, 0));
    PF_TRY(plan_forward_after_ring(p, p->st_f.as<double2>(), s));
    PF_CUDA(cudaEventRecord(p->ev_fwd_done, s));
    PF_CUDA(cudaStreamWaitEvent(p->d2h, p->ev_fwd_done, 0));
    PF_CUDA(cudaMemcpyAsync(out, p->st_f.p, nf, cudaMemcpyDeviceToHost, p->d2h));
    PF_CUDA(cudaEventRecord(p->ev_f_out_free, p->d2h));
    return 0;
}

// the adjoint to host coefficients: the field copied in on h2d; each order block's ring items on
// s, then that block's coefficients copied out on d2h while the next block computes
static int host_adjoint_pipelined(pfsht_plan* p, const void* in, void* out, cudaStream_t s) {
    const std::vector<AlmBlock> blocks = alm_blocks(p->L, host_mmax(p));
    const size_t nf = sizeof(double2) * (size_t)p->M * p->B;
    double2* alm = p->st_alm2.as<double2>();
    PF_CUDA(cudaStreamWaitEvent(p->h2d, p->ev_f_in_free, 0));
    PF_CUDA(cudaMemcpyAsync(p->st_f2.p, in, nf, cudaMemcpyHostToDevice, p->h2d));
    PF_CUDA(cudaEventRecord(p->ev_f_in_ready, p->h2d));
    // the output zero fill on the side stream, once the previous adjoint's copies have left
    PF_CUDA(cudaEventRecord(p->ev_fork, s));
    PF_CUDA(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    PF_CUDA(cudaStreamWaitEvent(p->side, p->ev_alm_out_free, 0));
    PF_TRY(ring_adjoint_prepare(p->rt, p->adj_items.view, alm, p->B, p->side));
    PF_CUDA(cudaEventRecord(p->ev_join, p->side));
    clock_begin(&p->clk, s);
    PF_CUDA(cudaStreamWaitEvent(s, p->ev_f_in_ready, 0));
    PF_TRY(plan_adjoint_before_ring(p, p->st_f2.as<double2>(), s));
    PF_CUDA(cudaEventRecord(p->ev_f_in_free, s));
    PF_CUDA(cudaStreamWaitEvent(s, p->ev_join, 0));
    for (size_t k = 0; k < blocks.size(); ++k) {
        RingItems v = p->adj_items.view;
        v.items = p->blk_adj_items.as<RingItem>() + p->blk_adj_off[k];
        v.nitems = p->blk_adj_off[k + 1] - p->blk_adj_off[k];
        PF_TRY(ring_adjoint(p->rt, p->ro_cols, v, p->H.as<double2>(), alm, p->B, s, false));
        PF_CUDA(cudaEventRecord(p->ev_blk[k], s));
        PF_CUDA(cudaStreamWaitEvent(p->d2h, p->ev_blk[k], 0));
        PF_TRY(alm_copy_block(p, blocks[k], out, alm, false, p->d2h));
    }
    clock_mark(&p->clk, kStRingAdj, s);
    PF_CUDA(cudaEventRecord(p->ev_alm_out_free, p->d2h));
    return 0;
}

void plan_host_wait(pfsht_plan* p) {
    if (p->host_zero.valid()) p->host_zero.get();
}

int plan_host_enqueue(pfsht_plan* p, const void* in, void* out, bool fwd, cudaStream_t s,
                      bool order_on_s, bool zero_async) {
    PF_TRY(plan_host_staging(p));
    const size_t nf = sizeof(double2) * (size_t)p->M * p->B;
    if (p->host_pipeline) {
        if (fwd) {
            PF_TRY(host_forward_pipelined(p, in, out, s));
        } else {
            PF_TRY(host_adjoint_pipelined(p, in, out, s));
            // the padding rows (tens of MB at large lmax) are zeroed while the device works,
            // so the caller can issue its next apply at once
            plan_host_wait(p);
            if (zero_async)
                p->host_zero = std::async(std::launch::async, [p, out] { alm_zero_host_padding(p, out); });
            else
                alm_zero_host_padding(p, out);
        }
    } else {
        // whole copies around the apply on the compute stream
        PF_CUDA(cudaStreamWaitEvent(s, p->ev_copied, 0));
        if (fwd) {
            PF_TRY(alm_copy(p, const_cast<void*>(in), p->st_alm.as<double2>(), true, s));
            PF_TRY(apply_forward(p, p->st_alm.as<double2>(), p->st_f.as<double2>(), s));
            PF_CUDA(cudaMemcpyAsync(out, p->st_f.p, nf, cudaMemcpyDeviceToHost, s));
        } else {
            PF_CUDA(cudaMemcpyAsync(p->st_f2.p, in, nf, cudaMemcpyHostToDevice, s));
            PF_TRY(apply_adjoint(p, p->st_f2.as<double2>(), p->st_alm2.as<double2>(), s));
            PF_TRY(alm_copy(p, out, p->st_alm2.as<double2>(), false, s));
            alm_zero_host_padding(p, out);
        }
        // the plan's d2h stream marks the end of every host apply
        PF_CUDA(cudaEventRecord(p->ev_copied, s));
        PF_CUDA(cudaStreamWaitEvent(p->d2h, p->ev_copied, 0));
    }
    if (order_on_s) {
        PF_CUDA(cudaEventRecord(p->ev_copied, p->d2h));
        PF_CUDA(cudaStreamWaitEvent(s, p->ev_copied, 0));
    }
    return 0;
}

}  // namespace pf

extern "C" {

static int host_apply(pfsht_plan* p, const void* in, void* out, bool fwd) {
    DeviceGuard dg(p->device);
    cudaStream_t s = p->st_stream;
    PF_TRY(plan_host_enqueue(p, in, out, fwd, s, true, true));
    PF_CUDA(cudaStreamSynchronize(s));
    plan_host_wait(p);
    return 0;
}

pfsht_status pfsht_host_bytes(const pfsht_plan* p, int64_t* h2d_forward, int64_t* d2h_forward,
                              int64_t* h2d_adjoint, int64_t* d2h_adjoint) {
    if (!p) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL plan");
    int64_t a = 0, f = 0;
    host_bytes(p, &a, &f);
    if (h2d_forward) *h2d_forward = a;
    if (d2h_forward) *d2h_forward = f;
    if (h2d_adjoint) *h2d_adjoint = f;
    if (d2h_adjoint) *d2h_adjoint = a;
    return PFSHT_OK;
}

pfsht_status pfsht_forward_host(pfsht_plan* p, const void* alm, void* f) {
    if (!p || !alm || !f) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    return (pfsht_status)host_apply(p, alm, f, true);
}

pfsht_status pfsht_adjoint_host(pfsht_plan* p, const void* f, void* alm) {
    if (!p || !alm || !f) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    return (pfsht_status)host_apply(p, f, alm, false);
}

static int host_apply_async(pfsht_plan* p, const void* in, void* out, bool fwd, void* stream) {
    DeviceGuard dg(p->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : p->st_stream;
    return plan_host_enqueue(p, in, out, fwd, s, false, true);
}

pfsht_status pfsht_forward_host_async(pfsht_plan* p, const void* alm, void* f, void* stream) {
    if (!p || !alm || !f) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    return (pfsht_status)host_apply_async(p, alm, f, true, stream);
}

pfsht_status pfsht_adjoint_host_async(pfsht_plan* p, const void* f, void* alm, void* stream) {
    if (!p || !alm || !f) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    return (pfsht_status)host_apply_async(p, f, alm, false, stream);
}

static int host_sync(pfsht_plan* p) {
    if (!p->d2h) return 0;  // no host apply was issued
    DeviceGuard dg(p->device);
    PF_CUDA(cudaStreamSynchronize(p->d2h));
    plan_host_wait(p);
    return 0;
}

pfsht_status pfsht_host_sync(pfsht_plan* p) {
    if (!p) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL plan");
    return (pfsht_status)host_sync(p);
}

pfsht_status pfsht_wait_timeouts(int32_t* count) {
    if (!count) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    int n = 0;
    const int r = tma_timeouts(&n);
    *count = n;
    return (pfsht_status)r;
}

pfsht_status pfsht_ring_forward(pfsht_plan* p, const void* alm, void* G, void* stream) {
    if (!p || !alm || !G) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (p->kind == kDirect) return (pfsht_status)fail(PFSHT_ERR_UNSUPPORTED, "direct plan has no ring set");
    if (p->kind == kMultiBox)
        return (pfsht_status)fail(PFSHT_ERR_UNSUPPORTED, "a multi-box plan has one ring set per box");
    DeviceGuard dg(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    RingTables t = p->rt_fwd;
    t.w = nullptr;
    RingOut o;
    o.ld = p->nrings;
    o.bstride = (int64_t)p->nrings * (2 * p->L + 1);
    o.col_off = p->L;
    o.nrows = p->nrings;
    o.reflect = 0;
    o.nrings_out = p->nrings;
    o.zero_rest = 0;  // the whole G is cleared first: orders above mmax have no item
    const size_t bytes = sizeof(double2) * (size_t)o.bstride * p->B;
    cudaError_t e = cudaMemsetAsync(G, 0, bytes, s);
    if (e != cudaSuccess) return (pfsht_status)fail(PFSHT_ERR_CUDA, cudaGetErrorString(e));
    if (p->spin != 0) {
        SpinTables st = p->spt.t;
        st.w = nullptr;
        return (pfsht_status)spin_ring_forward(st, o, p->fwd_items.view, (const double2*)alm,
                                               (double2*)G, p->B, s);
    }
    return (pfsht_status)ring_forward(t, o, p->fwd_items.view,
                                      (const double2*)alm, (double2*)G, p->B, s);
}

pfsht_status pfsht_ring_adjoint(pfsht_plan* p, const void* G, void* alm, void* stream) {
    if (!p || !alm || !G) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (p->kind == kDirect) return (pfsht_status)fail(PFSHT_ERR_UNSUPPORTED, "direct plan has no ring set");
    if (p->kind == kMultiBox)
        return (pfsht_status)fail(PFSHT_ERR_UNSUPPORTED, "a multi-box plan has one ring set per box");
    DeviceGuard dg(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    RingTables t = p->rt;
    t.w = nullptr;
    RingOut o;
    o.ld = p->nrings;
    o.bstride = (int64_t)p->nrings * (2 * p->L + 1);
    o.col_off = p->L;
    o.nrows = p->nrings;
    o.reflect = 0;
    o.nrings_out = p->nrings;
    if (p->spin != 0) {
        SpinTables st = p->spt.t;
        st.w = nullptr;
        return (pfsht_status)spin_ring_adjoint(st, o, p->fwd_items.view, (const double2*)G,
                                               (double2*)alm, p->B, s);
    }
    return (pfsht_status)ring_adjoint(t, o, p->adj_items.view,
                                      (const double2*)G, (double2*)alm, p->B, s);
}

int64_t pfsht_ring_work(const pfsht_plan* p) { return p ? p->info.ring_work : -1; }

pfsht_status pfsht_plan_get_info(const pfsht_plan* p, pfsht_plan_info* info) {
    if (!p || !info) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    *info = p->info;
    return PFSHT_OK;
}

int64_t pfsht_workspace_bytes(const pfsht_plan* p) { return p ? p->info.device_bytes : -1; }

int32_t pfsht_plan_num_boxes(const pfsht_plan* p) {
    if (!p) return -1;
    return p->kind == kMultiBox ? (int32_t)p->boxes.size() : 1;
}

pfsht_status pfsht_plan_box(const pfsht_plan* p, int32_t box, pfsht_plan_info* info, int64_t* indices) {
    if (!p) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL plan");
    const int32_t nb = pfsht_plan_num_boxes(p);
    if (box < 0 || box >= nb) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "box index out of range");
    if (p->kind != kMultiBox) {
        if (info) *info = p->info;
        if (indices)
            for (int64_t i = 0; i < p->M; ++i) indices[i] = i;
        return PFSHT_OK;
    }
    const pfsht_plan* c = p->boxes[box].get();
    if (info) *info = c->info;
    if (indices) {
        const int64_t mb = p->box_off[box + 1] - p->box_off[box];
        std::vector<int32_t> h(mb);
        DeviceGuard dg(p->device);
        if (mb > 0 && cudaMemcpy(h.data(), p->gidx.as<int32_t>() + p->box_off[box], sizeof(int32_t) * mb,
                                 cudaMemcpyDeviceToHost) != cudaSuccess)
            return (pfsht_status)fail(PFSHT_ERR_CUDA, "copying box indices");
        for (int64_t i = 0; i < mb; ++i) indices[i] = h[i];
    }
    return PFSHT_OK;
}

static pfsht_box to_abi(const SphereBox& b) {
    pfsht_box o;
    o.theta_lo = b.lo;
    o.theta_hi = b.hi;
    o.phi_start = b.phistart;
    o.phi_extent = b.phiext;
    o.touches_north = b.touches_north ? 1 : 0;
    o.touches_south = b.touches_south ? 1 : 0;
    return o;
}

static SphereBox from_abi(const pfsht_box& o) {
    SphereBox b;
    b.lo = o.theta_lo;
    b.hi = o.theta_hi;
    b.phistart = o.phi_start;
    b.phiext = o.phi_extent;
    b.touches_north = o.touches_north != 0;
    b.touches_south = o.touches_south != 0;
    return b;
}

pfsht_status pfsht_bounding_box(const double* theta, const double* phi, int64_t npts, pfsht_box* box) {
    if (!theta || !phi || !box) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (npts < 1) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "need at least one point");
    *box = to_abi(bounding_box(theta, phi, npts));
    return PFSHT_OK;
}

double pfsht_cost_direct(int64_t npts, int32_t lmax, int32_t ntrans) {
    return cost_direct(npts, lmax, ntrans);
}

double pfsht_cost_stretch(const pfsht_box* box, int64_t npts, int32_t lmax, int32_t ntrans, double tol) {
    if (!box) return NAN;
    return cost_stretch(from_abi(*box), npts, lmax, ntrans, tol);
}

pfsht_status pfsht_partition_boxes(const double* theta, const double* phi, int64_t npts,
                                   int32_t lmax, int32_t ntrans, double tol, int32_t maxboxes,
                                   int32_t* group_of_point, int32_t* nboxes, pfsht_box* boxes,
                                   double* costs) {
    if (!theta || !phi || !nboxes) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    const int v = validate_common(npts, lmax, ntrans, tol);
    if (v) return (pfsht_status)v;
    if (maxboxes < 1) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "maxboxes must be >= 1");
    Partition part;
    partition_boxes_costed(theta, phi, npts, lmax, ntrans, tol, maxboxes, part);
    *nboxes = (int32_t)part.groups.size();
    for (size_t i = 0; i < part.groups.size(); ++i) {
        if (group_of_point)
            for (int32_t k : part.groups[i]) group_of_point[k] = (int32_t)i;
        if (boxes) boxes[i] = to_abi(part.boxes[i]);
        if (costs) costs[i] = part.costs[i];
    }
    return PFSHT_OK;
}

pfsht_status pfsht_select_method(const double* theta, const double* phi, int64_t npts, int32_t lmax,
                                 int32_t ntrans, double tol, int32_t* method) {
    if (!theta || !phi || !method) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    const int v = validate_common(npts, lmax, ntrans, tol);
    if (v) return (pfsht_status)v;
    *method = select_method(theta, phi, npts, lmax, ntrans, tol, nullptr);
    return PFSHT_OK;
}

pfsht_status pfsht_partition_boxes_device(const double* theta, const double* phi, int64_t npts,
                                          int32_t lmax, int32_t ntrans, double tol, int32_t maxboxes,
                                          int32_t* group_of_point, int32_t* nboxes, pfsht_box* boxes,
                                          double* costs, void* stream) {
    if (!theta || !phi || !nboxes) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    const int v = validate_common(npts, lmax, ntrans, tol);
    if (v) return (pfsht_status)v;
    if (maxboxes < 1) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "maxboxes must be >= 1");
    cudaStream_t s = (cudaStream_t)stream;
    DevPartition part;
    int r = partition_boxes_device(theta, phi, npts, lmax, ntrans, tol, maxboxes, s, part);
    if (r) return (pfsht_status)r;
    *nboxes = (int32_t)part.idx.size();
    for (size_t i = 0; i < part.idx.size(); ++i) {
        if (group_of_point) {
            std::vector<int32_t> h(part.n[i]);
            if (part.n[i] > 0 && cudaMemcpy(h.data(), part.idx[i]->p, sizeof(int32_t) * part.n[i],
                                            cudaMemcpyDeviceToHost) != cudaSuccess)
                return (pfsht_status)fail(PFSHT_ERR_CUDA, "copying box indices");
            for (int32_t k : h) group_of_point[k] = (int32_t)i;
        }
        if (boxes) boxes[i] = to_abi(part.boxes[i]);
        if (costs) costs[i] = part.costs[i];
    }
    return PFSHT_OK;
}

pfsht_status pfsht_select_method_device(const double* theta, const double* phi, int64_t npts,
                                        int32_t lmax, int32_t ntrans, double tol, int32_t* method,
                                        void* stream) {
    if (!theta || !phi || !method) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    const int v = validate_common(npts, lmax, ntrans, tol);
    if (v) return (pfsht_status)v;
    int m = 0;
    const int r = select_method_device(theta, phi, npts, lmax, ntrans, tol, (cudaStream_t)stream, &m, nullptr);
    if (r) return (pfsht_status)r;
    *method = m;
    return PFSHT_OK;
}

pfsht_status pfsht_bounding_box_device(const double* theta, const double* phi, int64_t npts,
                                       pfsht_box* box, void* stream) {
    if (!theta || !phi || !box) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (npts < 1) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "need at least one point");
    SphereBox b;
    const int r = bounding_box_device(theta, phi, npts, (cudaStream_t)stream, &b);
    if (r) return (pfsht_status)r;
    *box = to_abi(b);
    return PFSHT_OK;
}

pfsht_status pfsht_set_cost_constants(double ring, double fft, double spread, double ft_conn) {
    if (!(ring > 0) || !(fft > 0) || !(spread > 0) || !(ft_conn > 0))
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "cost constants must be positive");
    set_cost_constants(ring, fft, spread, ft_conn);
    return PFSHT_OK;
}

pfsht_status pfsht_get_cost_constants(double* ring, double* fft, double* spread, double* ft_conn,
                                      int32_t* calibrated) {
    const CostConstants c = cost_constants();
    if (ring) *ring = c.ring;
    if (fft) *fft = c.fft;
    if (spread) *spread = c.spread;
    if (ft_conn) *ft_conn = c.ft_conn;
    if (calibrated) *calibrated = c.calibrated ? 1 : 0;
    return PFSHT_OK;
}

pfsht_status pfsht_plan_geometry(const double* theta, const double* phi, int64_t npts, int32_t lmax,
                                 int32_t ntrans, double tol, const pfsht_opts* opts_in,
                                 pfsht_plan_info* info) {
    if (!theta || !phi || !info) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    int v = validate_common(npts, lmax, ntrans, tol);
    if (v) return (pfsht_status)v;
    pfsht_opts o;
    pfsht_opts_default(&o);
    if (opts_in) o = *opts_in;
    if (o.spin != 0 && std::abs(o.spin) > lmax)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "|spin| > lmax");
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t i = 0; i < npts; ++i) {
        lo = std::fmin(lo, theta[i]);
        hi = std::fmax(hi, theta[i]);
    }
    lo = std::fmax(lo, 0.0);
    hi = std::fmin(hi, M_PI);
    *info = pfsht_plan_info{};
    info->lmax = lmax;
    info->ntrans = ntrans;
    info->npts = npts;
    info->tol = tol;
    info->spin = o.spin;
    int method = o.method;
    Partition part;
    bool have_part = false;
    if (method == PFSHT_METHOD_AUTO) {
        method = select_method(theta, phi, npts, lmax, ntrans, tol, &part);
        have_part = true;
    }
    if (method == PFSHT_METHOD_MULTIBOX) {
        const int mb = o.maxboxes > 0 ? o.maxboxes : 8;
        if (!have_part || mb != 8) partition_boxes_costed(theta, phi, npts, lmax, ntrans, tol, mb, part);
        info->kind = kMultiBox;
        for (const SphereBox& b : part.boxes) {
            Leaf lb;
            std::string eb;
            const int rb = build_leaf(b.lo, b.hi, lmax, ntrans, tol, o.eps_apo_max, o.oversample_theta,
                                      o.oversample_phi, &lb, &eb, o.spin);
            if (rb == 2) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, eb);
            if (rb == 1) return (pfsht_status)fail(PFSHT_ERR_REFUSED, eb);
            info->ring_work += lb.ring_work;
        }
        return PFSHT_OK;
    }
    if (method == PFSHT_METHOD_DIRECT) {
        info->kind = kDirect;
        info->mmax = lmax;
        info->nrings = (int)npts;
        return PFSHT_OK;
    }
    Leaf lf;
    std::string err;
    int r = build_leaf(lo, hi, lmax, ntrans, tol, o.eps_apo_max, o.oversample_theta,
                       o.oversample_phi, &lf, &err, o.spin);
    if (r == 2) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, err);
    if (r == 1) {
        if (o.method == PFSHT_METHOD_STRETCH) return (pfsht_status)fail(PFSHT_ERR_REFUSED, err);
        info->kind = kDirect;
        info->mmax = lmax;
        info->nrings = (int)npts;
        return PFSHT_OK;
    }
    info->kind = lf.g.kind;
    info->flip = lf.flip;
    info->nth_half = lf.nth_half;
    info->nth = lf.nth;
    info->nph = lf.nph;
    info->mmax = lf.mmax;
    info->nrings = lf.nth_half;
    info->K = lf.g.K;
    info->ring_work = lf.ring_work;
    info->beta = lf.g.beta;
    info->h = lf.g.h;
    info->theta_lo = lf.g.lo;
    info->theta_hi = lf.g.hi;
    info->eps_apo = lf.g.eps_apo;
    info->Theta1 = lf.g.Theta1;
    info->sigma = lf.g.sigma;
    info->ThetaT = lf.g.ThetaT;
    info->nufft_w = es_width(tol);
    info->nufft_beta = 2.30 * info->nufft_w;
    info->nf1 = (int)next_smooth(std::max<int64_t>(2 * (int64_t)lf.nth, 2 * info->nufft_w));
    info->nf2 = (int)next_smooth(std::max<int64_t>(2 * (int64_t)lf.nph, 2 * info->nufft_w));
    info->ncols = 2 * lf.mmax + 1;
    return PFSHT_OK;
}

pfsht_status pfsht_dfs_double(const void* F, void* Ft, int32_t Nth, int32_t Nph, int32_t B,
                              int32_t spin, void* stream) {
    if (!F || !Ft || Nth < 1 || Nph < 1 || B < 1)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "bad DFS arguments");
    return (pfsht_status)dfs_double((const double2*)F, (double2*)Ft, Nth, Nph, B, spin, (cudaStream_t)stream);
}

pfsht_status pfsht_dfs_fold(void* F, const void* Ft, int32_t Nth, int32_t Nph, int32_t B,
                            int32_t spin, void* stream) {
    if (!F || !Ft || Nth < 1 || Nph < 1 || B < 1)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "bad DFS arguments");
    return (pfsht_status)dfs_fold((double2*)F, (const double2*)Ft, Nth, Nph, B, spin, (cudaStream_t)stream);
}

pfsht_status pfsht_nufft_create(int32_t type, int32_t n1, int32_t n2, int32_t iflag, int32_t ntrans,
                                double tol, const double* x, const double* y, int64_t M,
                                pfsht_nufft** out) {
    if (!out) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (type != 1 && type != 2)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NUFFT type must be 1 or 2");
    if (n1 < 1 || n2 < 1 || ntrans < 1 || M < 1 || !x || !y)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "bad NUFFT arguments");
    if (!(tol > 0) || !(tol < 1)) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "tol must lie in (0, 1)");
    std::unique_ptr<pfsht_nufft> p(new pfsht_nufft());
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (pfsht_status)fail(PFSHT_ERR_CUDA, cudaGetErrorString(e));
    p->device = dev;
    p->type = type;
    p->iflag = iflag >= 0 ? 1 : -1;
    p->B = ntrans;
    p->n1 = n1;
    p->n2 = n2;
    p->M = M;
    DevBuf dx, dy;
    int r = dx.alloc(sizeof(double) * M);
    if (!r) r = dy.alloc(sizeof(double) * M);
    if (r) return (pfsht_status)r;
    if (cudaMemcpy(dx.p, x, sizeof(double) * M, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dy.p, y, sizeof(double) * M, cudaMemcpyHostToDevice) != cudaSuccess)
        return (pfsht_status)fail(PFSHT_ERR_CUDA, "copying NUFFT points");
    std::vector<int> colk2(n2);
    for (int c = 0; c < n2; ++c) colk2[c] = mode_k(c, n2);
    std::vector<double2> ones(n1, make_double2(1.0, 0.0));
    r = setup_nufft_grid(p->g, p->d, n1, n2, colk2, ones, tol, M, 0.0, 0.0, true, 0, 0, false, 0,
                         0, 0, nullptr);
    if (!r) r = nufft_setpts(p->g, p->d, dx.as<double>(), dy.as<double>(), nullptr);
    if (!r) r = nufft_alloc(p->g, p->d, ntrans);
    if (r) return (pfsht_status)r;
    *out = p.release();
    return PFSHT_OK;
}

pfsht_status pfsht_nufft_exec(pfsht_nufft* p, const void* in, void* out, void* stream) {
    if (!p || !in || !out) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    DeviceGuard dg(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (p->type == 2)
        return (pfsht_status)nufft_type2(p->g, p->d, (const double2*)in, (double2*)out, p->B, p->iflag, s);
    return (pfsht_status)nufft_type1(p->g, p->d, (const double2*)in, (double2*)out, p->B, p->iflag, s);
}

pfsht_status pfsht_nufft_destroy(pfsht_nufft* p) {
    if (!p) return PFSHT_OK;
    DeviceGuard dg(p->device);
    delete p;
    return PFSHT_OK;
}

size_t pfsht_last_error(char* buf, size_t len) {
    const std::string& e = get_error();
    if (buf && len > 0) {
        size_t n = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), n);
        buf[n] = 0;
    }
    return e.size();
}

const char* pfsht_version(void) { return "pfsht_b200 0.1.0 (sm_100a)"; }

int64_t pfsht_launch_count(void) { return (int64_t)launch_count(); }

static const char* kStageNames[kNumStages] = {
    "ring_fwd", "fft_theta_fwd", "nufft_pad", "fft_fine1_fwd", "rows_fwd", "fft_fine2_fwd",
    "interp", "spread", "fft_fine2_adj", "rows_adj", "fft_fine1_adj", "nufft_unpad",
    "fft_theta_adj", "ring_adj", "direct"};

int32_t pfsht_num_stages(void) { return kNumStages; }

const char* pfsht_stage_name(int32_t stage) {
    return stage >= 0 && stage < kNumStages ? kStageNames[stage] : "";
}

pfsht_status pfsht_profile_start(pfsht_plan* p, int32_t max_marks) {
    if (!p || max_marks < 2) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "bad profile arguments");
    for (auto& c : p->boxes) {
        const pfsht_status r = pfsht_profile_start(c.get(), max_marks);
        if (r) return r;
    }
    DeviceGuard dg(p->device);
    StageClock& c = p->clk;
    while ((int)c.ev.size() < max_marks) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return (pfsht_status)fail(PFSHT_ERR_CUDA, "cudaEventCreate");
        c.ev.push_back(e);
    }
    c.stage.assign(c.ev.size(), -1);
    c.cap = (int)c.ev.size();
    c.used = 0;
    c.prev = nullptr;
    c.on = true;
    return PFSHT_OK;
}

pfsht_status pfsht_profile_stop(pfsht_plan* p, double* stage_ms, int32_t* stage_count) {
    if (!p || !stage_ms || !stage_count) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (p->kind == kMultiBox) {
        // the boxes' stages, summed
        std::vector<double> ms(kNumStages);
        std::vector<int32_t> cnt(kNumStages);
        for (int i = 0; i < kNumStages; ++i) {
            stage_ms[i] = 0.0;
            stage_count[i] = 0;
        }
        for (auto& c : p->boxes) {
            const pfsht_status r = pfsht_profile_stop(c.get(), ms.data(), cnt.data());
            if (r) return r;
            for (int i = 0; i < kNumStages; ++i) {
                stage_ms[i] += ms[i];
                stage_count[i] += cnt[i];
            }
        }
        return PFSHT_OK;
    }
    DeviceGuard dg(p->device);
    StageClock& c = p->clk;
    for (int i = 0; i < kNumStages; ++i) {
        stage_ms[i] = 0.0;
        stage_count[i] = 0;
    }
    if (c.used > 0 && cudaEventSynchronize(c.ev[c.used - 1]) != cudaSuccess)
        return (pfsht_status)fail(PFSHT_ERR_CUDA, "cudaEventSynchronize");
    for (int i = 1; i < c.used; ++i) {
        const int st = c.stage[i];
        if (st < 0) continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c.ev[i - 1], c.ev[i]) != cudaSuccess)
            return (pfsht_status)fail(PFSHT_ERR_CUDA, "cudaEventElapsedTime");
        stage_ms[st] += ms;
        stage_count[st] += 1;
    }
    const int overflow = c.used >= c.cap;
    c.on = false;
    c.used = 0;
    c.prev = nullptr;
    if (overflow) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "profile buffer filled; raise max_marks");
    return PFSHT_OK;
}

}  // extern "C"
