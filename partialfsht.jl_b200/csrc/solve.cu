// solve!(alm, plan, f; mode, rtol, maxiter, prior, w) (src/Analysis.jl:375-436) on the device:
// conjugate gradients on the normal equations (A^H W A + C^-1) alm = A^H W f.
//
// The loop stays on the device. One iteration -- forward apply, point weights, adjoint apply,
// prior, the two dot products and the three vector updates -- is captured once as a CUDA graph;
// every scalar (alpha, beta, the residual norms, the iteration count) lives in device memory and
// is computed by the kernels, so a launch needs nothing from the host. Once the relative residual
// reaches the tolerance a device flag freezes the updates, exactly where the reference's loop
// breaks. The host keeps one iteration in flight: it launches iteration i, then waits for the
// state copied out after iteration i - 1, and stops when that says done (the iteration in flight
// is then a frozen no-op). Dot products reduce in a fixed order (per-block partials, then one
// block); the adjoint apply inside an iteration adds floating-point atomically (ring tiles of one
// order, spread rows shared by neighbouring bins), so two solves agree to round-off, not bit for
// bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "plan_internal.hpp"

namespace {

using namespace pf;

struct SolveState {
    double2 rsold, rsnew, pAp, alpha, beta;
    double rhsn, rel, tol;
    int iters, done;
};

struct HostState {
    double rel;
    int iters, done;
};

constexpr int kDotBlocks = 592;  // 4 x 148 SMs
constexpr int kThreads = 256;

int fail(int code, const char* msg) {
    set_error(msg);
    return code;
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    // a / b for complex numbers (b != 0); Smith's scaling keeps intermediates in range
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const double r = b.x / b.y, d = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

// per-block partial sums of conj(x) y
__global__ void __launch_bounds__(kThreads) dot_partial_kernel(const double2* __restrict__ x,
                                                               const double2* __restrict__ y,
                                                               int64_t n, double2* __restrict__ part) {
    __shared__ double2 sh[kThreads];
    double sr = 0.0, si = 0.0, tr = 0.0, ti = 0.0;
    const int64_t step = (int64_t)gridDim.x * kThreads;
    int64_t t = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    for (; t + step < n; t += 2 * step) {  // two loads of each array in flight
        const double2 a = x[t], b = y[t], c = x[t + step], e = y[t + step];
        sr += a.x * b.x + a.y * b.y;
        si += a.x * b.y - a.y * b.x;
        tr += c.x * e.x + c.y * e.y;
        ti += c.x * e.y - c.y * e.x;
    }
    if (t < n) {
        const double2 a = x[t], b = y[t];
        sr += a.x * b.x + a.y * b.y;
        si += a.x * b.y - a.y * b.x;
    }
    sh[threadIdx.x] = make_double2(sr + tr, si + ti);
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[threadIdx.x].x += sh[threadIdx.x + o].x;
            sh[threadIdx.x].y += sh[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__device__ double2 reduce_parts(const double2* __restrict__ part) {
    __shared__ double2 sh[kThreads];
    double sr = 0.0, si = 0.0;
    for (int k = threadIdx.x; k < kDotBlocks; k += kThreads) {
        sr += part[k].x;
        si += part[k].y;
    }
    sh[threadIdx.x] = make_double2(sr, si);
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sh[threadIdx.x].x += sh[threadIdx.x + o].x;
            sh[threadIdx.x].y += sh[threadIdx.x + o].y;
        }
        __syncthreads();
    }
    return sh[0];
}

// initial state: rsold = dot(r, r), rhsn = sqrt|dot(rhs, rhs)| (r = rhs)
__global__ void __launch_bounds__(kThreads) init_state_kernel(const double2* __restrict__ part,
                                                              SolveState* st, double tol) {
    const double2 d = reduce_parts(part);
    if (threadIdx.x == 0) {
        st->rsold = d;
        st->rhsn = sqrt(hypot(d.x, d.y));
        st->rel = 1.0;
        st->tol = tol;
        st->iters = 0;
        st->done = 0;
        st->alpha = st->beta = st->rsnew = st->pAp = make_double2(0.0, 0.0);
    }
}

// alpha = rsold / dot(p, Ap) (0 when the denominator is 0)
__global__ void __launch_bounds__(kThreads) alpha_kernel(const double2* __restrict__ part, SolveState* st) {
    const double2 d = reduce_parts(part);
    if (threadIdx.x == 0 && !st->done) {
        st->pAp = d;
        st->alpha = (d.x == 0.0 && d.y == 0.0) ? make_double2(0.0, 0.0) : cdiv(st->rsold, d);
    }
}

// alm += alpha p; r -= alpha Ap; and the per-block partial sums of |r|^2 of the new residual
// (for dot(r, r)) in the same pass. Frozen: r is unchanged and the partials are its norm.
__global__ void __launch_bounds__(kThreads) update_xr_kernel(double2* __restrict__ alm,
                                                             double2* __restrict__ r,
                                                             const double2* __restrict__ p,
                                                             const double2* __restrict__ Ap, int64_t n,
                                                             const SolveState* __restrict__ st,
                                                             double2* __restrict__ part) {
    __shared__ double2 sh[kThreads];
    const bool frozen = st->done != 0;
    const double2 a = st->alpha;
    double sr = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)kThreads + threadIdx.x; t < n; t += (int64_t)gridDim.x * kThreads) {
        double2 y = r[t];
        if (!frozen) {
            const double2 pv = p[t], qv = Ap[t];
            double2 x = alm[t];
            x.x += a.x * pv.x - a.y * pv.y;
            x.y += a.x * pv.y + a.y * pv.x;
            y.x -= a.x * qv.x - a.y * qv.y;
            y.y -= a.x * qv.y + a.y * qv.x;
            alm[t] = x;
            r[t] = y;
        }
        sr += y.x * y.x + y.y * y.y;
    }
    sh[threadIdx.x] = make_double2(sr, 0.0);
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x].x += sh[threadIdx.x + o].x;
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// rsnew = dot(r, r); count the iteration; stop at rel <= tol, else beta = rsnew / rsold
__global__ void __launch_bounds__(kThreads) rsnew_kernel(const double2* __restrict__ part, SolveState* st) {
    const double2 d = reduce_parts(part);
    if (threadIdx.x == 0 && !st->done) {
        st->iters += 1;
        st->rsnew = d;
        st->rel = sqrt(hypot(d.x, d.y)) / st->rhsn;
        if (st->rel <= st->tol) {
            st->done = 1;
        } else {
            st->beta = cdiv(d, st->rsold);
            st->rsold = d;
        }
    }
}

// p = r + beta p
__global__ void update_p_kernel(double2* __restrict__ p, const double2* __restrict__ r, int64_t n,
                                const SolveState* __restrict__ st) {
    if (st->done) return;
    const double2 b = st->beta;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const double2 pv = p[t], rv = r[t];
        p[t] = make_double2(rv.x + b.x * pv.x - b.y * pv.y, rv.y + b.x * pv.y + b.y * pv.x);
    }
}

// f[i, b] *= w[i] (src/Analysis.jl:106-117)
__global__ void weight_kernel(double2* __restrict__ f, const double* __restrict__ w, int64_t M, int B) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M * B; t += (int64_t)gridDim.x * blockDim.x) {
        const double s = w[t % M];
        f[t].x *= s;
        f[t].y *= s;
    }
}

// Ap[l, m] += reg[l] p[l, m] over the sph_mode slots (src/Analysis.jl:449-458)
__global__ void prior_kernel(double2* __restrict__ Ap, const double2* __restrict__ p,
                             const double* __restrict__ reg, int L, int B) {
    const int64_t nr = L + 1, nc = 2 * L + 1, n = nr * nc * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(t % nr);
        const int col = (int)((t / nr) % nc);
        const int l = row + (col + 1) / 2;
        if (l > L) continue;
        const double s = reg[l];
        if (s == 0.0) continue;
        const double2 pv = p[t];
        Ap[t].x += s * pv.x;
        Ap[t].y += s * pv.y;
    }
}

unsigned grid_n(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 148 * 16)); }

struct SolveBufs {
    DevBuf rhs, r, p, Ap, fbuf, fw, part, state, reg;
};

int run_solve(pfsht_plan* pl, const double2* f, double2* alm, int mode, double rtol, int maxiter,
              const double* prior, const double* w, cudaStream_t s, int* iters_out, double* rel_out) {
    const int L = pl->L, B = pl->B;
    const int64_t nc = (int64_t)(L + 1) * (2 * L + 1) * B;
    const int64_t nf = pl->M * B;
    const size_t ca = sizeof(double2) * nc, cf = sizeof(double2) * nf;
    SolveBufs b;
    PF_TRY(b.rhs.alloc(ca));
    PF_TRY(b.r.alloc(ca));
    PF_TRY(b.p.alloc(ca));
    PF_TRY(b.Ap.alloc(ca));
    PF_TRY(b.fbuf.alloc(cf));
    PF_TRY(b.fw.alloc(cf));
    PF_TRY(b.part.alloc(sizeof(double2) * kDotBlocks));
    PF_TRY(b.state.alloc(sizeof(SolveState)));
    const double2* d_rhs = b.rhs.as<double2>();
    double2* d_r = b.r.as<double2>();
    double2* d_p = b.p.as<double2>();
    double2* d_Ap = b.Ap.as<double2>();
    double2* d_f = b.fbuf.as<double2>();
    double2* d_part = b.part.as<double2>();
    SolveState* st = b.state.as<SolveState>();
    const double* d_reg = nullptr;
    if (mode == PFSHT_SOLVE_WIENER) {
        // _prior_inverse! (src/Analysis.jl:437-447): 1 / C_l where C_l > 0, else 0
        std::vector<double> reg(L + 1);
        for (int l = 0; l <= L; ++l) reg[l] = prior[l] > 0 ? 1.0 / prior[l] : 0.0;
        PF_TRY(b.reg.alloc(sizeof(double) * (L + 1)));
        PF_CUDA(cudaMemcpyAsync(b.reg.p, reg.data(), sizeof(double) * (L + 1), cudaMemcpyHostToDevice, s));
        d_reg = b.reg.as<double>();
    }
    const double tol = mode == PFSHT_SOLVE_MINNORM ? std::min(rtol, 1e-12) : rtol;
    // the solve's applies are not stage-timed
    const bool clk_on = pl->clk.on;
    pl->clk.on = false;
    struct Restore {
        pfsht_plan* p;
        bool on;
        ~Restore() { p->clk.on = on; }
    } restore{pl, clk_on};

    // rhs = A^H (w f); alm = 0; r = p = rhs
    PF_CUDA(cudaMemcpyAsync(b.fw.p, f, cf, cudaMemcpyDeviceToDevice, s));
    if (w) {
        weight_kernel<<<grid_n(nf), kThreads, 0, s>>>(b.fw.as<double2>(), w, pl->M, B);
        PF_TRY(check_launch("weight_kernel"));
    }
    PF_TRY(pfsht_adjoint(pl, b.fw.p, b.rhs.p, s) == PFSHT_OK ? 0 : PFSHT_ERR_CUDA);
    PF_CUDA(cudaMemsetAsync(alm, 0, ca, s));
    PF_CUDA(cudaMemcpyAsync(d_r, d_rhs, ca, cudaMemcpyDeviceToDevice, s));
    PF_CUDA(cudaMemcpyAsync(d_p, d_rhs, ca, cudaMemcpyDeviceToDevice, s));
    dot_partial_kernel<<<kDotBlocks, kThreads, 0, s>>>(d_r, d_r, nc, d_part);
    PF_TRY(check_launch("dot_partial_kernel"));
    init_state_kernel<<<1, kThreads, 0, s>>>(d_part, st, tol);
    PF_TRY(check_launch("init_state_kernel"));
    SolveState h0;
    PF_CUDA(cudaMemcpyAsync(&h0, st, sizeof(h0), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    if (h0.rhsn == 0.0 || maxiter <= 0) {
        *iters_out = 0;
        *rel_out = h0.rhsn == 0.0 ? 0.0 : 1.0;
        return 0;
    }

    // one iteration, captured
    cudaStream_t cs;
    PF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Cleanup {
        cudaStream_t s;
        cudaGraph_t* g;
        cudaGraphExec_t* e;
        ~Cleanup() {
            if (*e) cudaGraphExecDestroy(*e);
            if (*g) cudaGraphDestroy(*g);
            cudaStreamDestroy(s);
        }
    } cleanup{cs, &graph, &exec};
    PF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int rc = pfsht_forward(pl, d_p, d_f, cs) == PFSHT_OK ? 0 : PFSHT_ERR_CUDA;
    if (!rc && w) {
        weight_kernel<<<grid_n(nf), kThreads, 0, cs>>>(d_f, w, pl->M, B);
        rc = check_launch("weight_kernel");
    }
    if (!rc) rc = pfsht_adjoint(pl, d_f, d_Ap, cs) == PFSHT_OK ? 0 : PFSHT_ERR_CUDA;
    if (!rc && d_reg) {
        prior_kernel<<<grid_n(nc), kThreads, 0, cs>>>(d_Ap, d_p, d_reg, L, B);
        rc = check_launch("prior_kernel");
    }
    if (!rc) {
        dot_partial_kernel<<<kDotBlocks, kThreads, 0, cs>>>(d_p, d_Ap, nc, d_part);
        alpha_kernel<<<1, kThreads, 0, cs>>>(d_part, st);
        update_xr_kernel<<<kDotBlocks, kThreads, 0, cs>>>(alm, d_r, d_p, d_Ap, nc, st, d_part);
        rsnew_kernel<<<1, kThreads, 0, cs>>>(d_part, st);
        update_p_kernel<<<grid_n(nc), kThreads, 0, cs>>>(d_p, d_r, nc, st);
        rc = check_launch("solve iteration kernels");
    }
    const cudaError_t ec = cudaStreamEndCapture(cs, &graph);
    if (rc) return rc;
    if (ec != cudaSuccess) return fail(PFSHT_ERR_CUDA, cudaGetErrorString(ec));
    PF_CUDA(cudaGraphInstantiate(&exec, graph, 0));

    // one iteration in flight: launch i, then read the state copied out after i - 1
    HostState* hs = nullptr;
    PF_CUDA(cudaHostAlloc(&hs, 2 * sizeof(HostState), cudaHostAllocDefault));
    struct FreeHost {
        HostState* h;
        ~FreeHost() { cudaFreeHost(h); }
    } free_host{hs};
    cudaEvent_t ev[2];
    PF_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    PF_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    struct FreeEv {
        cudaEvent_t* e;
        ~FreeEv() {
            cudaEventDestroy(e[0]);
            cudaEventDestroy(e[1]);
        }
    } free_ev{ev};
    for (int i = 0; i < maxiter; ++i) {
        PF_CUDA(cudaGraphLaunch(exec, s));
        PF_CUDA(cudaMemcpyAsync(&hs[i & 1].rel, &st->rel, sizeof(double), cudaMemcpyDeviceToHost, s));
        PF_CUDA(cudaMemcpyAsync(&hs[i & 1].iters, &st->iters, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        PF_CUDA(cudaEventRecord(ev[i & 1], s));
        if (i >= 1) {
            PF_CUDA(cudaEventSynchronize(ev[(i - 1) & 1]));
            if (hs[(i - 1) & 1].done) break;
        }
    }
    PF_CUDA(cudaStreamSynchronize(s));
    SolveState fin;
    PF_CUDA(cudaMemcpy(&fin, st, sizeof(fin), cudaMemcpyDeviceToHost));
    *iters_out = fin.iters;
    *rel_out = fin.rel;
    return 0;
}

}  // namespace

extern "C" {

pfsht_status pfsht_solve(pfsht_plan* plan, const void* f, void* alm, int32_t mode, double rtol,
                         int32_t maxiter, const double* prior, const double* w, void* stream,
                         int32_t* iters, double* relres) {
    if (!plan || !f || !alm || !iters || !relres) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (mode < PFSHT_SOLVE_CG || mode > PFSHT_SOLVE_MINNORM)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "mode must be CG, WIENER or MINNORM");
    if (mode == PFSHT_SOLVE_WIENER && !prior)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "WIENER needs a prior C_l: that prior is what makes "
                                                      "the problem well posed");
    if (!(rtol > 0)) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "rtol must be positive");
    if (maxiter < 0) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "maxiter must be >= 0");
    DeviceGuard dg(plan->device);
    int it = 0;
    double rel = 0;
    const int r = run_solve(plan, (const double2*)f, (double2*)alm, mode, rtol, maxiter, prior, w,
                            (cudaStream_t)stream, &it, &rel);
    if (r) return (pfsht_status)r;
    *iters = it;
    *relres = rel;
    return PFSHT_OK;
}

}  // extern "C"
