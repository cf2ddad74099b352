// Ring pass of the stretched leaf on sm_100a: rings_from_alm! and its exact transpose
// alm_from_rings! (PartialFSHT.jl src/Legendre.jl:310-542; device analogue of
// ext/PartialFSHTKernelAbstractionsExt.jl:86-230).
//
// Work decomposition: one warp per item (order m, tile of up to 128 consecutive retained
// rings); a lane owns R rings (ring j0 + lane + 32 r) and carries their two-term recurrence
// state and block-scaling exponent in registers. The recurrence is the reference's
//     P_m^m = (-1)^m 2^(m log2 sin + log2 c_m),   P_{m+1}^m = sqrt(2m+3) cos P_m^m,
//     P_l^m = a_l^m cos P_{l-1}^m - b_l^m P_{l-2}^m
// renormalised every 64 degrees (src/Legendre.jl:16,455-459). Each ring keeps its own
// exponent (as the KernelAbstractions kernel does), so no chunk headroom rule is needed.
// a_l^m, b_l^m come from a plan-time table built on the device with the reference's exact
// expressions; per block of 32 degrees a warp stages them and the coefficients a_{l,+-m}
// in shared memory, so the inner loop reads them as broadcasts.
//
// Forward: acc(ring, +-m) += a_{l,+-m} P_l^m, written once per ring, windowed and, for a
// pole/full periodisation, mirrored into the DFS row with sign (-1)^m (src/DFS.jl:26).
// Adjoint: each lane sums P_l^m g_j over its R rings; per block of degrees the lanes'
// partial sums are transposed through shared memory and each lane reduces one
// (degree, component) over the 32 lanes, then adds it to alm once per item.
#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace pf {

static constexpr int kWarpsPerBlock = 4;
static constexpr int kTileRings = 128;  // rings per work item
static constexpr int kStride = 64;      // _RESCALE_STRIDE (src/Legendre.jl:16)

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

std::vector<RingItem> make_ring_items(const std::vector<int>& jlo, const std::vector<int>& jhi,
                                      int L, int mmax, int /*R*/) {
    std::vector<RingItem> items;
    std::vector<int64_t> cost;
    for (int m = 0; m <= std::min(mmax, L); ++m) {
        int lo = jlo[m], hi = jhi[m];
        for (int j0 = lo; j0 <= hi; j0 += kTileRings) {
            int n = std::min(kTileRings, hi - j0 + 1);
            items.push_back(RingItem{m, j0, n, 0});
            cost.push_back((int64_t)((n + 31) / 32) * (L - m + 1));
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

// ---------------------------------------------------------------------------------------
// forward: alm -> ring columns
// ---------------------------------------------------------------------------------------
template <int R, int NB>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
ring_fwd_kernel(RingTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const double2* __restrict__ alm, double2* __restrict__ out, int b0) {
    __shared__ double2 s_ab[kWarpsPerBlock][32];
    __shared__ double2 s_ap[kWarpsPerBlock][NB][32];
    __shared__ double2 s_am[kWarpsPerBlock][NB][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kWarpsPerBlock + warp;
    if (it >= nitems) return;
    const RingItem item = items[it];
    const int m = item.m, L = t.lmax;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    const int64_t albs = (int64_t)(L + 1) * (2 * L + 1);
    const double2* colp = alm + albs * b0 + (int64_t)(L + 1) * (2 * m);
    const double2* colm = alm + albs * b0 + (int64_t)(L + 1) * (m > 0 ? 2 * m - 1 : 0);
    const double2* abm = t.ab + t.aboff[m];
    const double s23 = sqrt((double)(2 * m + 3));
    const double2 zero2 = make_double2(0.0, 0.0);

    for (int pass = 0; pass * 32 * R < item.n; ++pass) {
        const int kbase = pass * 32 * R;
        double x[R], p1[R], p2[R];
        int E[R];
        double2 accp[R][NB], accm[R][NB];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = kbase + lane + 32 * r;
            x[r] = 0.0;
            p1[r] = 0.0;
            p2[r] = 0.0;
            E[r] = 0;
            if (k < item.n) {
                const int j = item.j0 + k;
                x[r] = t.cos_t[j];
                const double e0 = m == 0 ? t.log2c[0] : (double)m * t.log2sin[j] + t.log2c[m];
                if (isfinite(e0)) {
                    const double Es = ceil(e0);
                    p2[r] = sgn * exp2(e0 - Es);
                    E[r] = (int)Es;
                }
            }
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
            // l = m + 1
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
            int steps = 0;
            for (int l0 = m + 2; l0 <= L; l0 += 32) {
                const int nl = min(32, L - l0 + 1);
                __syncwarp();
                if (lane < nl) {
                    const int l = l0 + lane;
                    s_ab[warp][lane] = abm[l - m - 2];
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        s_ap[warp][b][lane] = colp[(l - m) + albs * b];
                        double2 am = m > 0 ? colm[(l - m) + albs * b] : zero2;
                        am.x *= sgn;
                        am.y *= sgn;
                        s_am[warp][b][lane] = am;
                    }
                }
                __syncwarp();
                for (int i = 0; i < nl; ++i) {
                    const double2 ab = s_ab[warp][i];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const double p = fma(ab.x * x[r], p1[r], -(ab.y * p2[r]));
                        p2[r] = p1[r];
                        p1[r] = p;
                    }
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        const double2 ap = s_ap[warp][b][i];
                        const double2 am = s_am[warp][b][i];
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            accp[r][b] = cmad(accp[r][b], ap, p1[r]);
                            accm[r][b] = cmad(accm[r][b], am, p1[r]);
                        }
                    }
                    if (++steps == kStride && l0 + i < L) {
                        steps = 0;
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
        }
        // write the ring columns (window and 2^E folded into one exact scale)
        const double smir = o.spin_sgn * sgn;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = kbase + lane + 32 * r;
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
}

// ---------------------------------------------------------------------------------------
// adjoint: ring columns -> alm (alm must be zeroed; one atomic add per item and output)
// ---------------------------------------------------------------------------------------
template <int R, int NB>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
ring_adj_kernel(RingTables t, RingOut o, const RingItem* __restrict__ items, int nitems,
                const double2* __restrict__ in, double* __restrict__ almd, int b0) {
    constexpr int NV = 4 * NB;   // (+m re, +m im, -m re, -m im) per transform
    constexpr int LB = 32 / NV;  // degrees per reduction block
    __shared__ double s_red[kWarpsPerBlock][32][33];
    __shared__ double2 s_ab[kWarpsPerBlock][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kWarpsPerBlock + warp;
    if (it >= nitems) return;
    const RingItem item = items[it];
    const int m = item.m, L = t.lmax;
    const double sgn = (m & 1) ? -1.0 : 1.0;
    const double smir = o.spin_sgn * sgn;
    const int64_t albs = (int64_t)(L + 1) * (2 * L + 1);
    const double2* abm = t.ab + t.aboff[m];
    const double s23 = sqrt((double)(2 * m + 3));
    const int64_t cp = (int64_t)(L + 1) * (2 * m);
    const int64_t cm = (int64_t)(L + 1) * (m > 0 ? 2 * m - 1 : 0);

    for (int pass = 0; pass * 32 * R < item.n; ++pass) {
        const int kbase = pass * 32 * R;
        double x[R], p1[R], p2[R];
        int E[R];
        double2 gp[R][NB], gm[R][NB];
        // ring data for (ring r, transform b): folded, windowed, scaled by 2^E; the -m
        // column carries the (-1)^m of src/Legendre.jl:511
        auto load_g = [&](int r) {
            const int k = kbase + lane + 32 * r;
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
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = kbase + lane + 32 * r;
            x[r] = 0.0;
            p1[r] = 0.0;
            p2[r] = 0.0;
            E[r] = 0;
            if (k < item.n) {
                const int j = item.j0 + k;
                x[r] = t.cos_t[j];
                const double e0 = m == 0 ? t.log2c[0] : (double)m * t.log2sin[j] + t.log2c[m];
                if (isfinite(e0)) {
                    const double Es = ceil(e0);
                    p2[r] = sgn * exp2(e0 - Es);
                    E[r] = (int)Es;
                }
            }
            load_g(r);
        }
        int lb = 0, lfirst = m;
        // reduce the staged degrees [lfirst, lfirst + cnt) over the lanes and add to alm
        auto flush = [&](int cnt) {
            __syncwarp();
            if (lane < cnt * NV) {
                const int li = lane / NV, v = lane % NV;
                double s = 0.0;
#pragma unroll 8
                for (int q = 0; q < 32; ++q) s += s_red[warp][lane][q];
                const int l = lfirst + li;
                const int b = v >> 2, comp = v & 3;
                if (comp < 2 || m > 0) {
                    const int64_t idx = (l - m) + (comp < 2 ? cp : cm) + albs * (b0 + b);
                    atomicAdd(almd + 2 * idx + (comp & 1), s);
                }
            }
            __syncwarp();
        };
        auto stage = [&](const double (&P)[R]) {
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
            for (int v = 0; v < NV; ++v) s_red[warp][lb * NV + v][lane] = part[v];
            if (++lb == LB) {
                flush(LB);
                lfirst += LB;
                lb = 0;
            }
        };
        stage(p2);  // l = m
        if (m < L) {
#pragma unroll
            for (int r = 0; r < R; ++r) p1[r] = s23 * x[r] * p2[r];
            stage(p1);  // l = m + 1
            int steps = 0;
            for (int l0 = m + 2; l0 <= L; l0 += 32) {
                const int nl = min(32, L - l0 + 1);
                __syncwarp();
                if (lane < nl) s_ab[warp][lane] = abm[l0 + lane - m - 2];
                __syncwarp();
                for (int i = 0; i < nl; ++i) {
                    const double2 ab = s_ab[warp][i];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const double p = fma(ab.x * x[r], p1[r], -(ab.y * p2[r]));
                        p2[r] = p1[r];
                        p1[r] = p;
                    }
                    stage(p1);
                    if (++steps == kStride && l0 + i < L) {
                        steps = 0;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            const double mx = fmax(fabs(p1[r]), fabs(p2[r]));
                            if (mx > 0.0 && isfinite(mx)) {
                                const int s = ceil_log2(mx);
                                if (s != 0) {
                                    const double f = scalbn(1.0, -s);
                                    p1[r] *= f;
                                    p2[r] *= f;
                                    E[r] += s;
                                    load_g(r);
                                }
                            }
                        }
                    }
                }
            }
        }
        if (lb > 0) flush(lb);
    }
}

template <int R, int NB>
static int launch_fwd(const RingTables& t, const RingOut& o, const RingItem* items, int nitems,
                      const double2* alm, double2* out, int b0, cudaStream_t s) {
    const int grid = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    ring_fwd_kernel<R, NB><<<grid, kWarpsPerBlock * 32, 0, s>>>(t, o, items, nitems, alm, out, b0);
    return check_launch("ring_fwd_kernel");
}

template <int R, int NB>
static int launch_adj(const RingTables& t, const RingOut& o, const RingItem* items, int nitems,
                      const double2* in, double2* alm, int b0, cudaStream_t s) {
    const int grid = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    ring_adj_kernel<R, NB><<<grid, kWarpsPerBlock * 32, 0, s>>>(t, o, items, nitems, in,
                                                                 reinterpret_cast<double*>(alm), b0);
    return check_launch("ring_adj_kernel");
}

int ring_forward(const RingTables& t, const RingOut& o, const RingItem* items, int nitems, int R,
                 const double2* alm, double2* out, int B, cudaStream_t s) {
    if (nitems <= 0) return 0;
    int b0 = 0;
    while (b0 < B) {
        int rem = B - b0;
        if (rem >= 4) {
            PF_TRY((launch_fwd<1, 4>(t, o, items, nitems, alm, out, b0, s)));
            b0 += 4;
        } else if (rem >= 2) {
            PF_TRY((launch_fwd<2, 2>(t, o, items, nitems, alm, out, b0, s)));
            b0 += 2;
        } else {
            if (R >= 4) PF_TRY((launch_fwd<4, 1>(t, o, items, nitems, alm, out, b0, s)));
            else if (R >= 2) PF_TRY((launch_fwd<2, 1>(t, o, items, nitems, alm, out, b0, s)));
            else PF_TRY((launch_fwd<1, 1>(t, o, items, nitems, alm, out, b0, s)));
            b0 += 1;
        }
    }
    return 0;
}

int ring_adjoint(const RingTables& t, const RingOut& o, const RingItem* items, int nitems, int R,
                 const double2* in, double2* alm, int B, cudaStream_t s) {
    if (nitems <= 0) return 0;
    int b0 = 0;
    while (b0 < B) {
        int rem = B - b0;
        if (rem >= 4) {
            PF_TRY((launch_adj<1, 4>(t, o, items, nitems, in, alm, b0, s)));
            b0 += 4;
        } else if (rem >= 2) {
            PF_TRY((launch_adj<2, 2>(t, o, items, nitems, in, alm, b0, s)));
            b0 += 2;
        } else {
            if (R >= 4) PF_TRY((launch_adj<4, 1>(t, o, items, nitems, in, alm, b0, s)));
            else if (R >= 2) PF_TRY((launch_adj<2, 1>(t, o, items, nitems, in, alm, b0, s)));
            else PF_TRY((launch_adj<1, 1>(t, o, items, nitems, in, alm, b0, s)));
            b0 += 1;
        }
    }
    return 0;
}

}  // namespace pf
