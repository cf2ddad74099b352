// 2-D NUFFT of the stretched leaf and the NUFFT seam, on sm_100a: an exponential-of-
// semicircle (ES) kernel NUFFT with upsampling 2 (the published FINUFFT algorithm that the
// reference calls through ext/PartialFSHTFINUFFTExt.jl and ext/PartialFSHTcuFINUFFTExt.jl;
// its exact semantics are DirectSum's, src/NUFFT.jl:85-129).
//
// Type 2 (modes -> values), per transform:
//   pad   : mode columns (n1 x ncols, FFT order along dim 1) times the per-mode factors
//           (deconvolution, and for the leaf the half-cell phase and 1/n_theta) into the
//           zero-padded fine columns (nf1 x ncols)
//   FFT   : along dim 1 (length nf1) on the ncols non-zero columns only
//   rows  : the fine-grid rows that points can reach, [row0, row0 + nrows), transposed to
//           row-major U (nrows x nf2) with the unused fine columns zero
//   FFT   : along dim 2 (length nf2) on those rows only
//   interp: w x w taps per point, points in bin order
// Type 1 is the exact transpose (spread -> FFT -> rows^T -> FFT -> unpad).
//
// Points are transformed and bin-sorted on the device at plan time (radix sort on bin key).
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>

#include <map>
#include <mutex>
#include <tuple>

#include "es_horner_table.h"
#include "internal.cuh"
#include "tma.cuh"

namespace pf {

DevBuf::~DevBuf() {
    if (p) cudaFree(p);
}

int DevBuf::alloc(size_t n) {
    if (p) {
        cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        set_error(std::string("cudaMalloc of ") + std::to_string(n) + " bytes: " +
                  cudaGetErrorString(e));
        return 5;
    }
    bytes = n;
    return 0;
}

void StageClock::begin(cudaStream_t s) {
    if (used >= cap) return;
    cudaEventRecord(ev[used], s);
    stage[used] = -1;
    prev = ev[used];
    ++used;
}

void StageClock::mark(int st, cudaStream_t s) {
    if (used >= cap || !prev) return;
    cudaEventRecord(ev[used], s);
    stage[used] = st;
    prev = ev[used];
    ++used;
}

NufftDev::~NufftDev() {
    if (have_f1) cufftDestroy(f1);
    if (have_f2) cufftDestroy(f2);
}

static std::atomic<long long> g_launches{0};
long long launch_count() { return g_launches.load(); }

// every launch of this library's kernels is followed by this check, which also counts it
int check_launch(const char* what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string(what) + ": " + cudaGetErrorString(e));
        return 4;
    }
    return 0;
}

static inline unsigned nblk(int64_t n, int bs) {
    int64_t b = (n + bs - 1) / bs;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 1 << 20));
}

// ---------------------------------------------------------------------------------------
// leaf point transform (src/Stretch.jl:202-213, src/Windows.jl:289-298)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double dev_jl_mod(double x, double y) {
    double r = fmod(x, y);
    if (r == 0.0) return copysign(r, y);
    if ((r > 0) != (y > 0)) return r + y;
    return r;
}

__global__ void leaf_points_kernel(int kind, int north, double thmax, double lo_ext,
                                   double period, int flip, const double* __restrict__ theta,
                                   const double* __restrict__ phi, int64_t M,
                                   double* __restrict__ Th, double* __restrict__ ph) {
    const double pi = 3.141592653589793;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        double t = theta[i];
        if (flip) t = pi - t;
        double T;
        if (kind == kFull) {
            T = t;
        } else if (kind == kPole) {
            const double d = north ? t : pi - t;
            T = pi * d / thmax;
        } else {
            T = 2 * pi * (t - lo_ext) / period;
        }
        Th[i] = T;
        ph[i] = dev_jl_mod(phi[i], 2 * pi);
    }
}

int leaf_points(const Geom& g, bool flip, const double* theta, const double* phi, int64_t M,
                double* Th, double* ph, cudaStream_t s) {
    const double thmax = g.h * (1 + g.eps_apo);
    const int north = g.lo <= std::sqrt(2.220446049250313e-16) ? 1 : 0;
    const double lo_ext = g.lo - g.h * g.eps_apo;
    leaf_points_kernel<<<nblk(M, 256), 256, 0, s>>>(g.kind, north, thmax, lo_ext, g.period,
                                                    flip ? 1 : 0, theta, phi, M, Th, ph);
    return check_launch("leaf_points_kernel");
}

int minmax_device(const double* x, int64_t M, double* mn, double* mx, cudaStream_t s) {
    DevBuf out, tmp;
    PF_TRY(out.alloc(2 * sizeof(double)));
    size_t tb = 0, tb2 = 0;
    PF_CUDA(cub::DeviceReduce::Min(nullptr, tb, x, out.as<double>(), (int)M, s));
    PF_CUDA(cub::DeviceReduce::Max(nullptr, tb2, x, out.as<double>() + 1, (int)M, s));
    PF_TRY(tmp.alloc(std::max(tb, tb2)));
    PF_CUDA(cub::DeviceReduce::Min(tmp.p, tb, x, out.as<double>(), (int)M, s));
    PF_CUDA(cub::DeviceReduce::Max(tmp.p, tb2, x, out.as<double>() + 1, (int)M, s));
    double h[2];
    PF_CUDA(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    *mn = h[0];
    *mx = h[1];
    return 0;
}

// ---------------------------------------------------------------------------------------
// plan-time: grid coordinates, bin keys, sort
// ---------------------------------------------------------------------------------------
// Bins are aligned to the kernel's first cell (origin) i0 = ceil(g - w/2) of each point:
// bin (br, bc) holds the points with origin row in [br BR, br BR + BR) and origin column in
// [bc BC, bc BC + BC) (columns, and rows when every row is kept, taken modulo the grid).
// Within a bin the points are sorted by origin row, then origin column.
__global__ void bin_keys_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                int64_t M, double s1, double s2, int row0, int row_wrap,
                                int nf1, int nf2, int nrows, int w, int bin_rows, int bin_cols,
                                int nbr, int nbc, double2* __restrict__ g, int* __restrict__ key,
                                int* __restrict__ idx, int* __restrict__ counts) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        double g1 = x[i] * s1;
        double g2 = y[i] * s2;
        if (row_wrap) {
            g1 = dev_jl_mod(g1, (double)nf1);
            if (g1 >= nf1) g1 -= nf1;
        } else {
            g1 = g1 - (double)row0;
        }
        g2 = dev_jl_mod(g2, (double)nf2);
        if (g2 >= nf2) g2 -= nf2;
        int r = (int)ceil(g1 - 0.5 * w);
        int c = (int)ceil(g2 - 0.5 * w);
        if (row_wrap) r = ((r % nrows) + nrows) % nrows;
        r = min(max(r, 0), nrows - 1);
        c = ((c % nf2) + nf2) % nf2;
        const int br = min(r / bin_rows, nbr - 1);
        const int bc = min(c / bin_cols, nbc - 1);
        const int k = br * nbc + bc;
        g[i] = make_double2(g1, g2);
        key[i] = (k * bin_rows + (r - br * bin_rows)) * bin_cols + (c - bc * bin_cols);
        idx[i] = (int)i;
        atomicAdd(counts + k, 1);
    }
}

__global__ void gather_points_kernel(const double2* __restrict__ g, const int* __restrict__ sidx,
                                     int64_t M, double2* __restrict__ pts, int* __restrict__ perm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int j = sidx[i];
        pts[i] = g[j];
        perm[i] = j;
    }
}

// bin offsets on the host (nbins + 1)
static std::vector<int> binstart_host(const NufftGrid& g, const NufftDev& d, cudaStream_t s) {
    std::vector<int> bs((size_t)g.nbr * g.nbc + 1, 0);
    if (cudaMemcpyAsync(bs.data(), d.binstart.p, sizeof(int) * bs.size(), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        bs.clear();
    return bs;
}

// The interpolation's order of the points (ipts / iperm): within each interpolation group, the
// points dealt round-robin over the shared-memory bank class of their tile origin (element
// offset (r0 TC + c0) mod KM, KM elements per 128 bytes), so that the KM lanes that read the
// tile together in one shared-memory phase start at different banks and each tap's loads need
// no replay. The group's point range is unchanged.
int interp_point_order(const NufftGrid& g, NufftDev& d, const std::vector<int>& bs, cudaStream_t s) {
    const int64_t M = g.M;
    if (bs.empty()) {
        set_error("copying the NUFFT bin offsets failed");
        return 4;
    }
    std::vector<double2> pts(M);
    std::vector<int> perm(M);
    PF_CUDA(cudaMemcpyAsync(pts.data(), d.pts.p, sizeof(double2) * M, cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaMemcpyAsync(perm.data(), d.perm.p, sizeof(int) * M, cudaMemcpyDeviceToHost, s));
    PF_CUDA(cudaStreamSynchronize(s));
    const int W = g.w, KM = g.fp32 ? 16 : 8;
    const int G = g.igroup, TS = (G * g.bin_cols + W - 1) | 1;  // the kernel's tile row stride
    std::vector<double2> opts(M);
    std::vector<int> operm(M);
    std::vector<std::vector<int>> bucket(KM);
#pragma omp parallel for schedule(dynamic, 16) num_threads(16) firstprivate(bucket) if (M > 100000)
    for (int q = 0; q < g.nbr * g.nsbc; ++q) {
        const int br = q / g.nsbc, sg = q % g.nsbc;
        const int a = bs[br * g.nbc + sg * G], e = bs[br * g.nbc + std::min(g.nbc, sg * G + G)];
        const int tr0 = br * g.bin_rows, tc0 = sg * G * g.bin_cols;
        for (auto& v : bucket) v.clear();
        for (int i = a; i < e; ++i) {
            int r = (int)std::ceil(pts[i].x - 0.5 * W);
            if (g.row_wrap) r = ((r % g.nrows) + g.nrows) % g.nrows;
            int c = (int)std::ceil(pts[i].y - 0.5 * W);
            c = ((c % g.nf2) + g.nf2) % g.nf2;
            const int64_t off = (int64_t)(r - tr0) * TS + (c - tc0);
            bucket[(int)(((off % KM) + KM) % KM)].push_back(i);
        }
        int o = a;
        for (size_t j = 0; o < e; ++j)
            for (int k = 0; k < KM; ++k)
                if (j < bucket[k].size()) {
                    opts[o] = pts[bucket[k][j]];
                    operm[o] = perm[bucket[k][j]];
                    ++o;
                }
    }
    PF_TRY(d.ipts.alloc(sizeof(double2) * std::max<int64_t>(M, 1)));
    PF_TRY(d.iperm.alloc(sizeof(int) * std::max<int64_t>(M, 1)));
    PF_CUDA(cudaMemcpyAsync(d.ipts.p, opts.data(), sizeof(double2) * M, cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaMemcpyAsync(d.iperm.p, operm.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaStreamSynchronize(s));
    return 0;
}

int nufft_setpts(NufftGrid& g, NufftDev& d, const double* x, const double* y, cudaStream_t s) {
    const int64_t M = g.M;
    if (M > INT32_MAX) {
        set_error("more than 2^31-1 points in one plan");
        return 1;
    }
    g.nbr = std::max(1, (g.nrows + g.bin_rows - 1) / g.bin_rows);
    g.nbc = std::max(1, (g.nf2 + g.bin_cols - 1) / g.bin_cols);
    const int nbins = g.nbr * g.nbc;
    DevBuf gg, key, key2, idx, idx2, counts, tmp;
    PF_TRY(gg.alloc(sizeof(double2) * M));
    PF_TRY(key.alloc(sizeof(int) * M));
    PF_TRY(key2.alloc(sizeof(int) * M));
    PF_TRY(idx.alloc(sizeof(int) * M));
    PF_TRY(idx2.alloc(sizeof(int) * M));
    PF_TRY(counts.alloc(sizeof(int) * (nbins + 1)));
    PF_TRY(d.binstart.alloc(sizeof(int) * (nbins + 1)));
    PF_TRY(d.pts.alloc(sizeof(double2) * M));
    PF_TRY(d.perm.alloc(sizeof(int) * M));
    PF_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * (nbins + 1), s));
    const double s1 = (double)g.nf1 / (2 * M_PI), s2 = (double)g.nf2 / (2 * M_PI);
    bin_keys_kernel<<<nblk(M, 256), 256, 0, s>>>(x, y, M, s1, s2, g.row0, g.row_wrap, g.nf1,
                                                 g.nf2, g.nrows, g.w, g.bin_rows, g.bin_cols,
                                                 g.nbr, g.nbc,
                                                 gg.as<double2>(), key.as<int>(), idx.as<int>(),
                                                 counts.as<int>());
    PF_TRY(check_launch("bin_keys_kernel"));
    const int64_t nkeys = (int64_t)nbins * g.bin_rows * g.bin_cols;
    if (nkeys > INT32_MAX) {
        set_error("NUFFT fine grid too large for 32-bit bin keys");
        return 1;
    }
    int end_bit = 1;
    while ((1ll << end_bit) < nkeys && end_bit < 31) ++end_bit;
    size_t tb = 0, tb2 = 0;
    PF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<int>(), key2.as<int>(),
                                            idx.as<int>(), idx2.as<int>(), (int)M, 0, end_bit, s));
    PF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, counts.as<int>(), d.binstart.as<int>(),
                                          nbins + 1, s));
    PF_TRY(tmp.alloc(std::max(tb, tb2)));
    PF_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.as<int>(), key2.as<int>(),
                                            idx.as<int>(), idx2.as<int>(), (int)M, 0, end_bit, s));
    PF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, counts.as<int>(), d.binstart.as<int>(),
                                          nbins + 1, s));
    gather_points_kernel<<<nblk(M, 256), 256, 0, s>>>(gg.as<double2>(), idx2.as<int>(), M,
                                                      d.pts.as<double2>(), d.perm.as<int>());
    PF_TRY(check_launch("gather_points_kernel"));
    // launch order of the bins: non-empty bins, most points first, so the heavy bins start
    // in the first wave and the tail of the grid is the light ones
    std::vector<int> cnt(nbins);
    PF_CUDA(cudaMemcpyAsync(cnt.data(), counts.p, sizeof(int) * nbins, cudaMemcpyDeviceToHost, s));
    // temporaries are freed when this returns, so finish using them first
    PF_CUDA(cudaStreamSynchronize(s));
    std::vector<int> order;
    order.reserve(nbins);
    for (int b = 0; b < nbins; ++b)
        if (cnt[b] > 0) order.push_back(b);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cnt[a] > cnt[b]; });
    g.nbusy = (int)order.size();
    PF_TRY(d.binorder.alloc(sizeof(int) * std::max<size_t>(order.size(), 1)));
    if (!order.empty())
        PF_CUDA(cudaMemcpyAsync(d.binorder.p, order.data(), sizeof(int) * order.size(),
                                cudaMemcpyHostToDevice, s));
    // spreading colours: tiles of bins rcol rows or ccol columns of bins apart are disjoint when
    // the kernel's reach w - 1 fits in (rcol - 1) bins. Tiles that run past the grid's last column
    // (or, when rows wrap, its last row) wrap onto its first ones, so those bins get colour
    // classes of their own, one set for column wrap, one for row wrap and one for both; within
    // such a set no two bins of one class both wrap, so their tiles stay disjoint as well.
    {
        const int rcol = 1 + (g.w - 1 + g.bin_rows - 1) / g.bin_rows;
        const int ccol = 1 + (g.w - 1 + g.bin_cols - 1) / g.bin_cols;
        const int K = rcol * ccol;
        g.ncolors = 4 * K;
        std::vector<int> sord;
        g.color_off.assign(1, 0);
        auto colour = [&](int b) {
            const int br = b / g.nbc, bc = b % g.nbc;
            const int cw = bc * g.bin_cols + g.bin_cols + g.w - 1 > g.nf2 ? 1 : 0;
            const int rw = g.row_wrap && br * g.bin_rows + g.bin_rows + g.w - 1 > g.nrows ? 1 : 0;
            return (br % rcol) * ccol + bc % ccol + K * (cw + 2 * rw);
        };
        for (int k = 0; k < g.ncolors; ++k) {
            for (int b : order)
                if (colour(b) == k) sord.push_back(b);
            g.color_off.push_back((int)sord.size());
        }
        PF_TRY(d.sorder.alloc(sizeof(int) * std::max<size_t>(sord.size(), 1)));
        if (!sord.empty())
            PF_CUDA(cudaMemcpyAsync(d.sorder.p, sord.data(), sizeof(int) * sord.size(),
                                    cudaMemcpyHostToDevice, s));
        // the register-tile spreading reads a bin's number and point range in one load
        std::vector<int> first(nbins + 1, 0);
        for (int b = 0; b < nbins; ++b) first[b + 1] = first[b] + cnt[b];
        auto slots = [&](const std::vector<int>& ord, DevBuf& out) -> int {
            std::vector<int4> v(std::max<size_t>(ord.size(), 1), make_int4(0, 0, 0, 0));
            for (size_t i = 0; i < ord.size(); ++i)
                v[i] = make_int4(ord[i], first[ord[i]], first[ord[i] + 1], 0);
            PF_TRY(out.alloc(sizeof(int4) * v.size()));
            PF_CUDA(cudaMemcpyAsync(out.p, v.data(), sizeof(int4) * v.size(), cudaMemcpyHostToDevice, s));
            PF_CUDA(cudaStreamSynchronize(s));
            return 0;
        };
        PF_TRY(slots(order, d.bslot));
        PF_TRY(slots(sord, d.sslot));
    }
    // interpolation groups igroup consecutive bins of a bin row; non-empty groups, most
    // points first
    g.igroup = std::max(1, g.igroup);
    g.nsbc = (g.nbc + g.igroup - 1) / g.igroup;
    std::vector<int> gcnt((size_t)g.nbr * g.nsbc, 0);
    for (int b = 0; b < nbins; ++b) gcnt[(size_t)(b / g.nbc) * g.nsbc + (b % g.nbc) / g.igroup] += cnt[b];
    std::vector<int> gorder;
    for (int q = 0; q < (int)gcnt.size(); ++q)
        if (gcnt[q] > 0) gorder.push_back(q);
    std::stable_sort(gorder.begin(), gorder.end(), [&](int a, int b) { return gcnt[a] > gcnt[b]; });
    g.nisb = (int)gorder.size();
    PF_TRY(d.iorder.alloc(sizeof(int) * std::max<size_t>(gorder.size(), 1)));
    if (!gorder.empty())
        PF_CUDA(cudaMemcpyAsync(d.iorder.p, gorder.data(), sizeof(int) * gorder.size(),
                                cudaMemcpyHostToDevice, s));
    PF_CUDA(cudaStreamSynchronize(s));
    return interp_point_order(g, d, binstart_host(g, d, s), s);
}

// ---------------------------------------------------------------------------------------
// fine-grid FFT lengths: any length >= the minimum serves the NUFFT (the deconvolution uses the
// actual length), and the library FFT's speed varies by a factor ~3 between neighbouring smooth
// lengths, so the lengths are picked by timing.
// ---------------------------------------------------------------------------------------
namespace {

bool smooth7(int64_t n) {
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

struct LenKey {
    int nmin;
    int64_t batch;
    int fp32;
    bool operator<(const LenKey& o) const {
        return std::tie(nmin, batch, fp32) < std::tie(o.nmin, o.batch, o.fp32);
    }
};
std::mutex g_len_mu;
std::map<LenKey, int> g_len_cache;

// device time of one batched in-place FFT of length n (ms), or a large value when the library
// cannot plan it
double time_fft(int n, int64_t batch, bool fp32, void* buf, cudaStream_t s) {
    cufftHandle h;
    int nn[1] = {n};
    if (cufftPlanMany(&h, 1, nn, nn, 1, n, nn, 1, n, fp32 ? CUFFT_C2C : CUFFT_Z2Z, (int)batch) !=
        CUFFT_SUCCESS)
        return 1e30;
    cufftSetStream(h, s);
    auto run = [&] {
        if (fp32) cufftExecC2C(h, (cufftComplex*)buf, (cufftComplex*)buf, CUFFT_FORWARD);
        else cufftExecZ2Z(h, (cufftDoubleComplex*)buf, (cufftDoubleComplex*)buf, CUFFT_FORWARD);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    run();
    run();
    cudaEventRecord(e0, s);
    for (int k = 0; k < 3; ++k) run();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cufftDestroy(h);
    return ms / 3;
}

}  // namespace

int fine_fft_length(int nmin, int64_t batch, bool fp32, cudaStream_t s, int* out) {
    *out = nmin;
    std::vector<int> cand;
    for (int64_t n = nmin; n <= nmin + nmin / 10 && cand.size() < 12; ++n)
        if (smooth7(n)) cand.push_back((int)n);
    if (cand.size() < 2 || batch < 1) return 0;
    const LenKey key{nmin, batch, fp32 ? 1 : 0};
    std::lock_guard<std::mutex> lk(g_len_mu);
    auto it = g_len_cache.find(key);
    if (it != g_len_cache.end()) {
        *out = it->second;
        return 0;
    }
    // time on at most 256 MB of scratch (a smaller batch ranks the lengths alike)
    const size_t el = fp32 ? sizeof(float2) : sizeof(double2);
    const int64_t bm = std::max<int64_t>(1, std::min<int64_t>(batch, ((int64_t)256 << 20) / ((int64_t)cand.back() * el)));
    DevBuf scratch;
    PF_TRY(scratch.alloc(el * (size_t)bm * cand.back()));
    PF_CUDA(cudaMemsetAsync(scratch.p, 0, el * (size_t)bm * cand.back(), s));
    std::vector<double> t(cand.size());
    for (size_t i = 0; i < cand.size(); ++i) t[i] = time_fft(cand[i], bm, fp32, scratch.p, s);
    PF_CUDA(cudaStreamSynchronize(s));
    PF_CUDA(cudaGetLastError());
    // the shortest length within 5% of the fastest (a longer grid costs the other stages more)
    const double best = *std::min_element(t.begin(), t.end());
    for (size_t i = 0; i < cand.size(); ++i)
        if (t[i] <= 1.05 * best) {
            *out = cand[i];
            break;
        }
    g_len_cache[key] = *out;
    return 0;
}

int nufft_alloc(NufftGrid& g, NufftDev& d, int B) {
    const size_t el = g.fp32 ? sizeof(float2) : sizeof(double2);
    const cufftType ty = g.fp32 ? CUFFT_C2C : CUFFT_Z2Z;
    PF_TRY(d.pad.alloc(el * (size_t)g.nf1 * g.ncols * B));
    PF_TRY(d.U.alloc(el * (size_t)g.nrows * g.nf2 * B));
    PF_TRY(d.counter.alloc(sizeof(int)));
    int n1[1] = {g.nf1};
    PF_CUFFT(cufftPlanMany(&d.f1, 1, n1, n1, 1, g.nf1, n1, 1, g.nf1, ty, g.ncols * B));
    d.have_f1 = true;
    int n2[1] = {g.nf2};
    PF_CUFFT(cufftPlanMany(&d.f2, 1, n2, n2, 1, g.nf2, n2, 1, g.nf2, ty, g.nrows * B));
    d.have_f2 = true;
    // tensor maps for the TMA row transposes (the plain kernels serve when the driver has no
    // encoder or the layout does not fit one)
    d.have_maps = g.gap_ok && !g.plain_transpose &&
                  make_tile_map(&d.pad_map, d.pad.p, (int)el, g.nf1, (int64_t)g.ncols * B, 128 / (int)el, 32) == 0 &&
                  make_tile_map(&d.U_map, d.U.p, (int)el, g.nf2, (int64_t)g.nrows * B, 128 / (int)el, 32) == 0;
    return 0;
}

// in-place fine-grid FFT of either element type
static int fine_fft(cufftHandle h, void* data, bool fp32, int dir) {
    if (fp32)
        PF_CUFFT(cufftExecC2C(h, static_cast<cufftComplex*>(data), static_cast<cufftComplex*>(data), dir));
    else
        PF_CUFFT(cufftExecZ2Z(h, static_cast<cufftDoubleComplex*>(data),
                              static_cast<cufftDoubleComplex*>(data), dir));
    return 0;
}

// ---------------------------------------------------------------------------------------
// complex element of the fine grids: double2 in the FP64 form, float2 in the mixed form (whose
// mode columns, points and per-mode factors stay FP64)
// ---------------------------------------------------------------------------------------
template <class T> struct Cx;
template <> struct Cx<double> {
    using t = double2;
    __device__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <> struct Cx<float> {
    using t = float2;
    __device__ static float2 make(float x, float y) { return make_float2(x, y); }
};
template <class T> using cx = typename Cx<T>::t;

// ---------------------------------------------------------------------------------------
// pad / unpad along dim 1
// ---------------------------------------------------------------------------------------
template <class T>
__global__ void pad_kernel(const double2* __restrict__ in, int n1, int ncols, int nf1,
                           const double2* __restrict__ mult1, const double* __restrict__ dec2,
                           cx<T>* __restrict__ pad) {
    const int c = blockIdx.y, b = blockIdx.z;
    const int pos = (n1 + 1) / 2, neg = n1 / 2;
    const double2* ic = in + (int64_t)n1 * c + (int64_t)n1 * ncols * b;
    cx<T>* oc = pad + (int64_t)nf1 * c + (int64_t)nf1 * ncols * b;
    const double d2 = dec2[c];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nf1; p += gridDim.x * blockDim.x) {
        int i1 = -1;
        if (p < pos) i1 = p;
        else if (p >= nf1 - neg) i1 = n1 + (p - nf1);
        double2 v = make_double2(0.0, 0.0);
        if (i1 >= 0) {
            const double2 a = ic[i1];
            const double2 f = mult1[i1];
            v.x = (a.x * f.x - a.y * f.y) * d2;
            v.y = (a.x * f.y + a.y * f.x) * d2;
        }
        oc[p] = Cx<T>::make((T)v.x, (T)v.y);
    }
}

template <class T>
__global__ void unpad_kernel(const cx<T>* __restrict__ pad, int n1, int ncols, int nf1,
                             const double2* __restrict__ mult1, const double* __restrict__ dec2,
                             double2* __restrict__ out) {
    const int c = blockIdx.y, b = blockIdx.z;
    const cx<T>* ic = pad + (int64_t)nf1 * c + (int64_t)nf1 * ncols * b;
    double2* oc = out + (int64_t)n1 * c + (int64_t)n1 * ncols * b;
    const double d2 = dec2[c];
    for (int i1 = blockIdx.x * blockDim.x + threadIdx.x; i1 < n1; i1 += gridDim.x * blockDim.x) {
        const int k1 = i1 < (n1 + 1) / 2 ? i1 : i1 - n1;
        const int p = k1 >= 0 ? k1 : nf1 + k1;
        const cx<T> a0 = ic[p];
        const double2 a = make_double2((double)a0.x, (double)a0.y);
        const double2 f = mult1[i1];  // conj(f)
        double2 v;
        v.x = (a.x * f.x + a.y * f.y) * d2;
        v.y = (a.y * f.x - a.x * f.y) * d2;
        oc[i1] = v;
    }
}

// ---------------------------------------------------------------------------------------
// fine rows <-> fine columns (tile transpose through shared memory)
// ---------------------------------------------------------------------------------------
// U[r, p2] = pad[(row0 + r) mod nf1, p2col[p2]] (or 0)
template <class T>
__global__ void rows_fwd_kernel(const cx<T>* __restrict__ pad, int nf1, int ncols, int row0,
                                int nrows, int nf2, const int* __restrict__ p2col,
                                cx<T>* __restrict__ U) {
    __shared__ cx<T> tile[32][33];
    const int b = blockIdx.z;
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;  // c0 indexes p2
    const cx<T>* pb = pad + (int64_t)nf1 * ncols * b;
    cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int p2 = c0 + k;
        const int r = r0 + threadIdx.x;
        cx<T> v = Cx<T>::make(0, 0);
        if (p2 < nf2 && r < nrows) {
            const int c = p2col[p2];
            if (c >= 0) {
                int p1 = row0 + r;
                p1 %= nf1;
                if (p1 < 0) p1 += nf1;
                v = pb[p1 + (int64_t)nf1 * c];
            }
        }
        tile[k][threadIdx.x] = v;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k;
        const int p2 = c0 + threadIdx.x;
        if (r < nrows && p2 < nf2) ub[(int64_t)r * nf2 + p2] = tile[threadIdx.x][k];
    }
}

// pad[p1, c] = U[(p1 - row0) mod nf1, colp2[c]] when that row is kept, else 0
template <class T>
__global__ void rows_adj_kernel(const cx<T>* __restrict__ U, int nf1, int ncols, int row0,
                                int nrows, int nf2, const int* __restrict__ colp2,
                                cx<T>* __restrict__ pad) {
    __shared__ cx<T> tile[32][33];
    const int b = blockIdx.z;
    const int p0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    cx<T>* pb = pad + (int64_t)nf1 * ncols * b;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int p1 = p0 + k;
        const int c = c0 + threadIdx.x;
        cx<T> v = Cx<T>::make(0, 0);
        if (p1 < nf1 && c < ncols) {
            int r = (p1 - row0) % nf1;
            if (r < 0) r += nf1;
            if (r < nrows) v = ub[(int64_t)r * nf2 + colp2[c]];
        }
        tile[k][threadIdx.x] = v;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k;
        const int p1 = p0 + threadIdx.x;
        if (c < ncols && p1 < nf1) pb[p1 + (int64_t)nf1 * c] = tile[threadIdx.x][k];
    }
}

// ---------------------------------------------------------------------------------------
// the same transposes with TMA-staged tiles: a block per 32 x 32 tile loads it into shared
// memory with 2-D tensor copies (128-byte lines, 128-byte swizzle so that the transposed reads
// fill each bank once), waits on an mbarrier (bounded) and writes the transposed tile with
// coalesced stores. Tiles whose rows wrap around the fine grid, or whose columns are not one
// contiguous run (or, for 8-byte elements, start on an odd element), are read with plain loads.
// ---------------------------------------------------------------------------------------
constexpr int kTmaWaitLimit = 1 << 20;

// U[r, p2] = pad[(row0 + r) mod nf1, p2col[p2]]; blocks past the tiles zero the fine columns
// [gap_lo, gap_hi) that hold no mode column (the only such columns), 32 rows x 256 columns each
template <class T>
__global__ void __launch_bounds__(256)
rows_fwd_tma_kernel(const __grid_constant__ CUtensorMap pmap, const cx<T>* __restrict__ pad,
                    int nf1, int ncols, int row0, int nrows, int nf2,
                    const int* __restrict__ colp2, int gap_lo, int gap_hi, int ntc, int ntr,
                    int nzc, cx<T>* __restrict__ U) {
    constexpr int E = sizeof(cx<T>);  // 16 (FP64) or 8 (FP32) bytes
    constexpr int SUB = 128 / E;       // fine rows per 128-byte line
    constexpr int NSUB = 32 / SUB;     // line blocks per 32-row tile
    __shared__ __align__(1024) unsigned char tile[NSUB][32 * 128];
    __shared__ __align__(8) uint64_t bar;
    const int b = blockIdx.z, tx = threadIdx.x, ty = threadIdx.y;
    cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    const int ntiles = ntc * ntr;
    if ((int)blockIdx.x >= ntiles) {
        const int zb = (int)blockIdx.x - ntiles;
        const int zr = (zb / nzc) * 32, z0 = gap_lo + (zb % nzc) * 256;
        const int z1 = min(z0 + 256, gap_hi);
        const cx<T> z = Cx<T>::make(0, 0);
        for (int r = zr + ty; r < min(zr + 32, nrows); r += 8)
            for (int p2 = z0 + tx; p2 < z1; p2 += 32) ub[(int64_t)r * nf2 + p2] = z;
        return;
    }
    const int c0 = ((int)blockIdx.x % ntc) * 32, r0 = ((int)blockIdx.x / ntc) * 32;
    const int p0 = row0 + r0;
    const bool tma = p0 >= 0 && p0 + 32 <= nf1 && (E == 16 || (p0 & 1) == 0);
    if (tma) {
        if (tx == 0 && ty == 0) {
            mbar_init(&bar, 1);
            mbar_expect_tx(&bar, NSUB * 32 * 128);
#pragma unroll
            for (int j = 0; j < NSUB; ++j)
                tma_load_2d(tile[j], &pmap, &bar, (p0 + j * SUB) * (E / 8), c0 + ncols * b);
        }
        __syncthreads();
        if (!mbar_wait_bounded(&bar, 0, kTmaWaitLimit)) return;
    }
    const int c = c0 + tx;
    if (c >= ncols) return;
    const int p2 = colp2[c];
    for (int rr = ty; rr < 32; rr += 8) {
        const int r = r0 + rr;
        if (r >= nrows) break;
        cx<T> v;
        if (tma) {
            v = *reinterpret_cast<const cx<T>*>(tile[rr / SUB] + swz128(tx, (rr % SUB) * E));
        } else {
            int p1 = (row0 + r) % nf1;
            if (p1 < 0) p1 += nf1;
            v = pad[p1 + (int64_t)nf1 * (c + (int64_t)ncols * b)];
        }
        ub[(int64_t)r * nf2 + p2] = v;
    }
}

// pad[p1, c] = U[(p1 - row0) mod nf1, colp2[c]] when that row is kept, else 0
template <class T>
__global__ void __launch_bounds__(256)
rows_adj_tma_kernel(const __grid_constant__ CUtensorMap umap, const cx<T>* __restrict__ U,
                    int nf1, int ncols, int row0, int nrows, int nf2,
                    const int* __restrict__ colp2, int ntc, cx<T>* __restrict__ pad) {
    constexpr int E = sizeof(cx<T>);
    constexpr int SUB = 128 / E;  // fine columns per 128-byte line
    constexpr int NSUB = 32 / SUB;
    __shared__ __align__(1024) unsigned char tile[NSUB][32 * 128];
    __shared__ __align__(8) uint64_t bar;
    const int b = blockIdx.z, tx = threadIdx.x, ty = threadIdx.y;
    const int c0 = ((int)blockIdx.x % ntc) * 32, p0 = ((int)blockIdx.x / ntc) * 32;
    // kept rows of the tile: r = (p1 - row0) mod nf1, one run when it does not wrap
    int rf = (p0 - row0) % nf1;
    if (rf < 0) rf += nf1;
    const int ncv = min(32, ncols - c0);
    const int q0 = colp2[c0];
    // the tile's columns are one run of fine columns
    const bool run = __syncthreads_and(tx >= ncv || colp2[c0 + tx] == q0 + tx) != 0;
    const bool tma = run && rf + 32 <= nf1 && rf < nrows && (E == 16 || (q0 & 1) == 0);
    if (tma) {
        if (tx == 0 && ty == 0) {
            mbar_init(&bar, 1);
            mbar_expect_tx(&bar, NSUB * 32 * 128);
#pragma unroll
            for (int j = 0; j < NSUB; ++j)
                tma_load_2d(tile[j], &umap, &bar, (q0 + j * SUB) * (E / 8), rf + nrows * b);
        }
        __syncthreads();
        if (!mbar_wait_bounded(&bar, 0, kTmaWaitLimit)) return;
    }
    const int p1 = p0 + tx;
    if (p1 >= nf1) return;
    const int r = tma ? rf + tx : ((p1 - row0) % nf1 + nf1) % nf1;
    const cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    for (int k = ty; k < ncv; k += 8) {
        const int c = c0 + k;
        cx<T> v = Cx<T>::make(0, 0);
        if (r < nrows) {
            if (tma) v = *reinterpret_cast<const cx<T>*>(tile[k / SUB] + swz128(tx, (k % SUB) * E));
            else v = ub[(int64_t)r * nf2 + colp2[c]];
        }
        pad[p1 + (int64_t)nf1 * (c + (int64_t)ncols * b)] = v;
    }
}

int tma_timeouts(int* out) {
    PF_CUDA(cudaMemcpyFromSymbol(out, g_tma_timeouts, sizeof(int)));
    return 0;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_tile_map(CUtensorMap* map, void* base, int esize, int64_t inner, int64_t outer,
                  int box_inner, int box_outer) {
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    if (!fn || esize % 8 != 0 || ((uintptr_t)base & 15) != 0) return 1;
    // 8-byte units: the complex values move as (re, im) pairs of 8-byte words
    const int u = esize / 8;
    const cuuint64_t dims[2] = {(cuuint64_t)(inner * u), (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)(inner * esize)};
    const cuuint32_t box[2] = {(cuuint32_t)(box_inner * u), (cuuint32_t)box_outer};
    const cuuint32_t estr[2] = {1, 1};
    if (strides[0] % 16 != 0 || box[0] * 8 != 128) return 1;
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
               ? 0 : 1;
}

// ---------------------------------------------------------------------------------------
// interpolation and spreading
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ int wrap(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

// tile of a bin: the rows and columns its points' kernels reach,
// rows [br BR, br BR + BR + W - 1) x columns [bc BC, bc BC + BC + W - 1)
struct TileGeom {
    int tr0, tc0, TR, TC;
};
template <int W>
__device__ __forceinline__ TileGeom tile_geom(int bin, int nbc, int BR, int BC) {
    const int br = bin / nbc, bc = bin % nbc;
    return TileGeom{br * BR, bc * BC, BR + W - 1, BC + W - 1};
}

// origin cell of a point inside its bin's tile (the binning of bin_keys_kernel)
template <int W>
__device__ __forceinline__ void local_origin(double2 g, const TileGeom& tg, int nrows, int nf2,
                                             int row_wrap, int& r0, int& c0, double& v1,
                                             double& v2) {
    const int i10 = (int)ceil(g.x - 0.5 * W);
    const int i20 = (int)ceil(g.y - 0.5 * W);
    v1 = ((double)i10 - g.x) + (0.5 * W - 0.5);
    v2 = ((double)i20 - g.y) + (0.5 * W - 0.5);
    int r = i10, c = i20;
    if (row_wrap) r = wrap(r, nrows);
    c = wrap(c, nf2);
    r0 = r - tg.tr0;
    c0 = c - tg.tc0;
}

template <int W, class T> struct EsCoef;
template <int W> struct EsCoef<W, double> {
    __device__ static const double* get() { return EsHorner<W>::coef(); }
};
template <int W> struct EsCoef<W, float> {
    __device__ static const float* get() { return EsHorner<W>::coef_f(); }
};

// Weights of the mirrored taps a and W - 1 - a (a < W / 2) at offset v, u = v^2, in the grid's
// precision. Tap W - 1 - a is tap a reflected (v -> -v; the table holds the same coefficients
// with the odd powers negated), so with p_a(v) = E(v^2) + v O(v^2) the pair costs one even and
// one odd Horner chain in u: NC multiply-adds for two taps instead of 2 (NC - 1).
template <int W, class T>
__device__ __forceinline__ void es_pair(int a, T v, T u, T& ka, T& kb) {
    constexpr int NC = EsHorner<W>::NC;
    constexpr int NE = (NC + 1) / 2, NO = NC / 2;
    const T* cf = EsCoef<W, T>::get() + a * NC;
    T e = cf[2 * (NE - 1)];
#pragma unroll
    for (int i = NE - 2; i >= 0; --i) e = fma(e, u, cf[2 * i]);
    T o = cf[2 * (NO - 1) + 1];
#pragma unroll
    for (int i = NO - 2; i >= 0; --i) o = fma(o, u, cf[2 * i + 1]);
    ka = fma(v, o, e);
    kb = fma(-v, o, e);
}

// weight of the middle tap of an odd width (an even polynomial: its odd coefficients are 0)
template <int W, class T>
__device__ __forceinline__ T es_mid(T u) {
    constexpr int NC = EsHorner<W>::NC;
    constexpr int NE = (NC + 1) / 2;
    const T* cf = EsCoef<W, T>::get() + (W / 2) * NC;
    T e = cf[2 * (NE - 1)];
#pragma unroll
    for (int i = NE - 2; i >= 0; --i) e = fma(e, u, cf[2 * i]);
    return e;
}

// all W tap weights at offset v: mirrored pairs in FP64; one Horner chain per tap in FP32, where
// the spreading kernel measured faster that way (0.133 vs 0.142 ms at lmax 2048)
template <int W, class T>
__device__ __forceinline__ void es_weights(T v, T (&k)[W]) {
    if constexpr (sizeof(T) == 8) {
        const T u = v * v;
#pragma unroll
        for (int a = 0; a < W / 2; ++a) es_pair<W, T>(a, v, u, k[a], k[W - 1 - a]);
        if constexpr (W & 1) k[W / 2] = es_mid<W, T>(u);
    } else {
        constexpr int NC = EsHorner<W>::NC;
        const T* cf = EsCoef<W, T>::get();
#pragma unroll
        for (int a = 0; a < W; ++a) {
            T p = cf[a * NC + NC - 1];
#pragma unroll
            for (int q = NC - 2; q >= 0; --q) p = fma(p, v, cf[a * NC + q]);
            k[a] = p;
        }
    }
}

// one point's interpolation from its group's tile (rows TS elements apart): the w x w taps,
// rows in mirrored pairs with the column weights held in registers; 0 for a point outside the
// tile (which binning excludes)
template <int W, class T>
__device__ __forceinline__ cx<T> interp_point(double2 g, const TileGeom& tg, int TS,
                                              const cx<T>* tile, int nrows, int nf2, int row_wrap) {
    int r0, c0;
    double v1, v2;
    local_origin<W>(g, tg, nrows, nf2, row_wrap, r0, c0, v1, v2);
    T k2[W];
    es_weights<W, T>((T)v2, k2);
    cx<T> acc = Cx<T>::make(0, 0);
    if (r0 >= 0 && r0 + W <= tg.TR && c0 >= 0 && c0 + W <= tg.TC) {
        const T w1 = (T)v1, u1 = w1 * w1;
        auto row_sum = [&](int a) {
            const cx<T>* row = tile + (r0 + a) * TS + c0;
            cx<T> sr = Cx<T>::make(0, 0);
#pragma unroll
            for (int c = 0; c < W; ++c) {
                const cx<T> u = row[c];
                sr.x = fma(u.x, k2[c], sr.x);
                sr.y = fma(u.y, k2[c], sr.y);
            }
            return sr;
        };
        // rows in mirrored pairs (a, W - 1 - a): one pair of row weights at a time
#pragma unroll
        for (int a = 0; a < W / 2; ++a) {
            T ka, kb;
            es_pair<W, T>(a, w1, u1, ka, kb);
            const cx<T> sa = row_sum(a), sb = row_sum(W - 1 - a);
            acc.x = fma(sa.x, ka, acc.x);
            acc.y = fma(sa.y, ka, acc.y);
            acc.x = fma(sb.x, kb, acc.x);
            acc.y = fma(sb.y, kb, acc.y);
        }
        if constexpr (W & 1) {
            const T km = es_mid<W, T>(u1);
            const cx<T> sm = row_sum(W / 2);
            acc.x = fma(sm.x, km, acc.x);
            acc.y = fma(sm.y, km, acc.y);
        }
    }
    return acc;
}

// Type-2 interpolation: one CTA per group of consecutive bins of a bin row copies the group's
// tile of U (at most 32 columns) into shared memory, then each thread interpolates points of
// the group from it. The row weights are evaluated row by
// row inside the tap loop so only the column weights are held in registers.
template <int W, class T>
__global__ void __launch_bounds__(128, sizeof(T) == 8 ? 5 : 4)
interp_kernel(const double2* __restrict__ pts, const int* __restrict__ perm,
              const int* __restrict__ binstart, const int* __restrict__ iorder, int nbc, int G,
              int nsbc, int BR, int BC, int64_t M, const cx<T>* __restrict__ U, int nrows,
              int nf2, int row_wrap, int B, double2* __restrict__ f) {
    extern __shared__ __align__(16) unsigned char interp_smem[];
    cx<T>* tile = reinterpret_cast<cx<T>*>(interp_smem);
    // a group of G consecutive bins of one bin row: their points are contiguous in bin order
    const int sb = iorder[blockIdx.x];
    const int br = sb / nsbc, sg = sb % nsbc;
    const int s = binstart[br * nbc + sg * G];
    const int e = binstart[br * nbc + min(nbc, sg * G + G)];
    const TileGeom tg{br * BR, sg * G * BC, BR + W - 1, G * BC + W - 1};
    // the tile is at most 32 columns wide (G BC <= 33 - W): lane = column, warps stride the rows
    const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int gcol = wrap(tg.tc0 + ln, nf2);
    // tile rows an odd number of elements apart: a tap's bank class then depends on its row as
    // well as its column, which evens out the classes the points are dealt over
    const int TS = tg.TC | 1;
    for (int b = 0; b < B; ++b) {
        const cx<T>* ub = U + (int64_t)nrows * nf2 * b;
        if (tg.TC <= 32) {
            if (ln < tg.TC) {
                for (int rr = wid; rr < tg.TR; rr += nw) {
                    int r = tg.tr0 + rr;
                    if (row_wrap) r = wrap(r, nrows);
                    cx<T> v = Cx<T>::make(0, 0);
                    if (r >= 0 && r < nrows) v = ub[(int64_t)r * nf2 + gcol];
                    tile[rr * TS + ln] = v;
                }
            }
        } else {
            for (int t = threadIdx.x; t < tg.TR * tg.TC; t += blockDim.x) {
                int r = tg.tr0 + t / tg.TC;
                if (row_wrap) r = wrap(r, nrows);
                cx<T> v = Cx<T>::make(0, 0);
                if (r >= 0 && r < nrows) v = ub[(int64_t)r * nf2 + wrap(tg.tc0 + t % tg.TC, nf2)];
                tile[(t / tg.TC) * TS + t % tg.TC] = v;
            }
        }
        // each thread's first point loads while the tile copy completes; FP32 grids also issue
        // each later point's load one iteration ahead (in FP64 the extra registers would cost
        // more occupancy than the hidden latency gains)
        constexpr bool kAhead = sizeof(T) == 4;
        int p = s + threadIdx.x;
        double2 gn = make_double2(0.0, 0.0);
        int jn = 0;
        if (p < e) {
            gn = pts[p];
            jn = perm[p];
        }
        __syncthreads();
        for (bool first = true; p < e; p += blockDim.x, first = false) {
            double2 g;
            int j;
            if constexpr (kAhead) {
                g = gn;
                j = jn;
                if (p + (int)blockDim.x < e) {
                    gn = pts[p + blockDim.x];
                    jn = perm[p + blockDim.x];
                }
            } else {
                // FP64: only each thread's first point is loaded under the tile copy
                if (first) {
                    g = gn;
                    j = jn;
                } else {
                    g = pts[p];
                    j = perm[p];
                }
            }
            const cx<T> acc = interp_point<W, T>(g, tg, TS, tile, nrows, nf2, row_wrap);
            f[j + M * b] = make_double2((double)acc.x, (double)acc.y);
        }
        __syncthreads();
    }
}

// asynchronous global -> shared copy of one grid value, or zeros (src_bytes = 0); each thread
// later waits for its own copies
template <class T>
__device__ __forceinline__ void cp_async_value(cx<T>* dst, const cx<T>* src, bool valid) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const int n = valid ? (int)sizeof(cx<T>) : 0;
    if constexpr (sizeof(cx<T>) == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n)
                     : "memory");
}

// Type-2 interpolation, pipelined (one transform): a resident grid of blocks pulls groups of
// bins from a counter, heaviest first; while a block interpolates the points of one group from
// its tile, the next group's tile is copied into the other half of its shared memory with
// cp.async, so the copy's latency is not exposed between groups. Points and results as in
// interp_kernel.
template <int W, class T>
__global__ void __launch_bounds__(128, sizeof(T) == 8 ? 5 : 4)
interp_pipe_kernel(const double2* __restrict__ pts, const int* __restrict__ perm,
                   const int* __restrict__ binstart, const int* __restrict__ iorder, int ngroups,
                   int nbc, int G, int nsbc, int BR, int BC, const cx<T>* __restrict__ U, int nrows,
                   int nf2, int row_wrap, int tile_elems, double2* __restrict__ f,
                   int* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char interp_smem[];
    cx<T>* tiles = reinterpret_cast<cx<T>*>(interp_smem);  // two tiles of tile_elems values
    __shared__ int s_next;
    const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31, nw = blockDim.x >> 5;
    auto geom = [&](int q) {
        const int sb = iorder[q];
        const int br = sb / nsbc, sg = sb % nsbc;
        return TileGeom{br * BR, sg * G * BC, BR + W - 1, G * BC + W - 1};
    };
    // the tile is at most 32 columns wide (G BC <= 33 - W): lane = column, warps stride the rows
    auto copy_tile = [&](int q, cx<T>* tile) {
        const TileGeom tg = geom(q);
        const int TS = tg.TC | 1;
        if (ln < tg.TC) {
            const int gcol = wrap(tg.tc0 + ln, nf2);
            for (int rr = wid; rr < tg.TR; rr += nw) {
                int r = tg.tr0 + rr;
                if (row_wrap) r = wrap(r, nrows);
                const bool ok = r >= 0 && r < nrows;
                cp_async_value<T>(tile + rr * TS + ln, U + (ok ? (int64_t)r * nf2 + gcol : 0), ok);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    if (threadIdx.x == 0) s_next = atomicAdd(counter, 1);
    __syncthreads();
    int cur = s_next;
    if (cur >= ngroups) return;
    copy_tile(cur, tiles);
    for (int buf = 0;; buf ^= 1) {
        __syncthreads();  // every thread has read s_next
        if (threadIdx.x == 0) s_next = atomicAdd(counter, 1);
        __syncthreads();
        const int nxt = s_next;
        if (nxt < ngroups) copy_tile(nxt, tiles + (buf ^ 1) * tile_elems);
        else asm volatile("cp.async.commit_group;\n" ::: "memory");
        // this thread's copies of the current tile are done; the barrier makes everyone's visible
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        const TileGeom tg = geom(cur);
        const int sb = iorder[cur];
        const int br = sb / nsbc, sg = sb % nsbc;
        const int s = binstart[br * nbc + sg * G];
        const int e = binstart[br * nbc + min(nbc, sg * G + G)];
        const cx<T>* tile = tiles + buf * tile_elems;
        for (int p = s + threadIdx.x; p < e; p += blockDim.x) {
            const double2 g = pts[p];
            const int j = perm[p];
            const cx<T> acc = interp_point<W, T>(g, tg, tg.TC | 1, tile, nrows, nf2, row_wrap);
            f[j] = make_double2((double)acc.x, (double)acc.y);
        }
        __syncthreads();  // the tile is read before it is refilled
        if (nxt >= ngroups) break;
        cur = nxt;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Type-1 spreading, output stationary: one warp per bin, lane l owns tile column l (the
// tile is BC + W - 1 = 32 columns wide) and keeps in registers the W rows a point's kernel
// can reach. The bin's points arrive sorted by origin row, so when the origin row advances
// the rows left behind are complete: each is added to U exactly once (atomically, since
// neighbouring bins' tiles overlap it). Per batch of 32 points each lane evaluates one
// point's row weights and its value times the column weights into a per-warp staging area;
// the points are then applied one by one from it, the next point's operands loaded while the
// current one's W complex FMA pairs run, with no shared-memory read-modify-write.
template <int W, class T>
struct SpreadStage {
    static constexpr int KP = (W + 1) / 2;  // row weights as pairs
    cx<T> k1[32][KP];          // row weights (pairs; the odd tail padded with 0)
    cx<T> vk[32][W + 1];       // value x column weight; slot W is 0 for lanes off the point
    int2 org[32];              // origin row (or -1: skip) and column inside the tile
};

// warps (bins) per block: the staging area of the wide kernels needs more shared memory
template <int W> struct SpreadWarps { static constexpr int N = W > 12 ? 2 : 4; };

template <int W, class T>
__global__ void __launch_bounds__(SpreadWarps<W>::N * 32)
spread_kernel(const double2* __restrict__ pts, const int* __restrict__ perm,
              const int* __restrict__ binstart, const int* __restrict__ binorder, int nbusy,
              int nbc, int BR, int BC, int64_t M, const double2* __restrict__ fin, int b,
              int nrows, int nf2, int row_wrap, int plain, cx<T>* __restrict__ U) {
    constexpr int KP = SpreadStage<W, T>::KP;
    constexpr int NW = SpreadWarps<W>::N;
    __shared__ SpreadStage<W, T> stg[NW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = blockIdx.x * NW + warp;
    if (slot >= nbusy) return;
    const int bin = binorder[slot];
    const int s = binstart[bin], e = binstart[bin + 1];
    const TileGeom tg = tile_geom<W>(bin, nbc, BR, BC);
    SpreadStage<W, T>& st = stg[warp];
    cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    const bool col_ok = lane < tg.TC;
    const int gcol = wrap(tg.tc0 + lane, nf2);
    cx<T> acc[W];
#pragma unroll
    for (int a = 0; a < W; ++a) acc[a] = Cx<T>::make(0, 0);
    int rbase = -1;
    // add tile row r (a local row) held in acc[a] to U
    auto flush = [&](int r, const cx<T>& v) {
        int gr = tg.tr0 + r;
        if (row_wrap) gr = wrap(gr, nrows);
        if (col_ok && gr >= 0 && gr < nrows && (v.x != 0.0 || v.y != 0.0)) {
            cx<T>* qd = ub + (int64_t)gr * nf2 + gcol;
            if (plain) {
                // no other tile of this launch reaches the cell (bins launched by colour)
                cx<T> u = *qd;
                u.x += v.x;
                u.y += v.y;
                *qd = u;
            } else {
                atomicAdd(reinterpret_cast<T*>(qd), v.x);
                atomicAdd(reinterpret_cast<T*>(qd) + 1, v.y);
            }
        }
    };
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 32; ++q) st.vk[q][W] = Cx<T>::make(0, 0);
    }
    for (int base = s; base < e; base += 32) {
        const int nb = min(32, e - base);
        __syncwarp();
        if (lane < nb) {
            const double2 g = pts[base + lane];
            const double2 v = fin[perm[base + lane] + M * b];
            int r0, c0;
            double v1, v2;
            local_origin<W>(g, tg, nrows, nf2, row_wrap, r0, c0, v1, v2);
            {
                T k1[W];
                es_weights<W, T>((T)v1, k1);
#pragma unroll
                for (int q = 0; q < KP; ++q)
                    st.k1[lane][q] = Cx<T>::make(k1[2 * q], 2 * q + 1 < W ? k1[2 * q + 1] : (T)0);
            }
            {
                T k2[W];
                es_weights<W, T>((T)v2, k2);
#pragma unroll
                for (int q = 0; q < W; ++q)
                    st.vk[lane][q] = Cx<T>::make((T)v.x * k2[q], (T)v.y * k2[q]);
            }
            const bool inside = r0 >= 0 && r0 + W <= tg.TR && c0 >= 0 && c0 + W <= tg.TC;
            st.org[lane] = make_int2(inside ? r0 : -1, c0);
        }
        __syncwarp();
        // operands of point q for this lane
        auto fetch = [&](int q, int2& o, cx<T>& vk, cx<T> (&k1)[KP]) {
            o = st.org[q];
            const unsigned dc = (unsigned)(lane - o.y);
            vk = st.vk[q][dc < (unsigned)W ? dc : W];
#pragma unroll
            for (int a2 = 0; a2 < KP; ++a2) k1[a2] = st.k1[q][a2];
        };
        int2 o_n;
        cx<T> vk_n, k1_n[KP];
        fetch(0, o_n, vk_n, k1_n);
        for (int q = 0; q < nb; ++q) {
            const int2 o = o_n;
            const cx<T> vk = vk_n;
            cx<T> k1[KP];
#pragma unroll
            for (int a2 = 0; a2 < KP; ++a2) k1[a2] = k1_n[a2];
            if (q + 1 < nb) fetch(q + 1, o_n, vk_n, k1_n);
            const int r0 = o.x;
            if (r0 < 0) continue;  // outside its bin's tile: cannot happen for binned points
            if (r0 != rbase) {
                if (rbase < 0) rbase = r0;
                int d = r0 - rbase;
                if (d >= W) {
#pragma unroll
                    for (int a = 0; a < W; ++a) {
                        flush(rbase + a, acc[a]);
                        acc[a] = Cx<T>::make(0, 0);
                    }
                    rbase = r0;
                    d = 0;
                }
                for (; d > 0; --d) {
                    flush(rbase, acc[0]);
#pragma unroll
                    for (int a = 0; a < W - 1; ++a) acc[a] = acc[a + 1];
                    acc[W - 1] = Cx<T>::make(0, 0);
                    ++rbase;
                }
            }
#pragma unroll
            for (int a2 = 0; a2 < KP; ++a2) {
                acc[2 * a2].x = fma(vk.x, k1[a2].x, acc[2 * a2].x);
                acc[2 * a2].y = fma(vk.y, k1[a2].x, acc[2 * a2].y);
                if (2 * a2 + 1 < W) {
                    acc[2 * a2 + 1].x = fma(vk.x, k1[a2].y, acc[2 * a2 + 1].x);
                    acc[2 * a2 + 1].y = fma(vk.y, k1[a2].y, acc[2 * a2 + 1].y);
                }
            }
        }
    }
    if (rbase >= 0) {
#pragma unroll
        for (int a = 0; a < W; ++a) flush(rbase + a, acc[a]);
    }
}

// Type-1 spreading for tiles at most 16 columns wide (bins of BC <= 17 - W columns): one warp
// per bin, lane (h, c) = (lane / 16, lane % 16) owns tile column c and, of the W rows a point's
// kernel reaches, those of parity h, RH = ceil(W / 2) of them in registers (row base_h + 2 i,
// base_h the first row of parity h at or after the current origin row). A point of origin row
// r0 gives lanes of parity r0 & 1 its even-offset row weights and the other half its odd ones,
// so each lane does RH complex FMA pairs per point where the 32-column layout does W. When the
// origin row advances past a row, the half holding it adds it to U and slides its window by
// one register; the other half is untouched.
template <int W, class T>
struct Spread16Stage {
    static constexpr int RH = (W + 1) / 2;
    static constexpr int RP = (RH + 1) / 2;  // row weights of one parity, as pairs
    cx<T> k1[32][2][RP];       // [point][parity][pair]: even / odd offset row weights, 0-padded
    cx<T> vk[32][W + 1];       // value x column weight; slot W is 0 for lanes off the point
    int2 org[32];              // origin row (or -1: skip) and column inside the tile
};

template <int W, class T>
__global__ void __launch_bounds__(128)
spread16_kernel(const double2* __restrict__ pts, const int* __restrict__ perm,
                const int* __restrict__ binstart, const int* __restrict__ binorder, int nbusy,
                int nbc, int BR, int BC, int64_t M, const double2* __restrict__ fin, int b,
                int nrows, int nf2, int row_wrap, int plain, cx<T>* __restrict__ U) {
    constexpr int RH = Spread16Stage<W, T>::RH;
    constexpr int RP = Spread16Stage<W, T>::RP;
    __shared__ Spread16Stage<W, T> stg[4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h = lane >> 4, c = lane & 15;
    const int slot = blockIdx.x * 4 + warp;
    if (slot >= nbusy) return;
    const int bin = binorder[slot];
    const int s = binstart[bin], e = binstart[bin + 1];
    const TileGeom tg = tile_geom<W>(bin, nbc, BR, BC);
    Spread16Stage<W, T>& st = stg[warp];
    cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    const bool col_ok = c < tg.TC;
    const int gcol = wrap(tg.tc0 + c, nf2);
    cx<T> acc[RH];
#pragma unroll
    for (int i = 0; i < RH; ++i) acc[i] = Cx<T>::make(0, 0);
    int rbase = -1;  // current origin row (local); this half holds rows base_h + 2 i
    auto flush = [&](int r, const cx<T>& v) {
        int gr = tg.tr0 + r;
        if (row_wrap) gr = wrap(gr, nrows);
        if (col_ok && gr >= 0 && gr < nrows && (v.x != 0.0 || v.y != 0.0)) {
            cx<T>* qd = ub + (int64_t)gr * nf2 + gcol;
            if (plain) {
                // no other tile of this launch reaches the cell (bins launched by colour)
                cx<T> u = *qd;
                u.x += v.x;
                u.y += v.y;
                *qd = u;
            } else {
                atomicAdd(reinterpret_cast<T*>(qd), v.x);
                atomicAdd(reinterpret_cast<T*>(qd) + 1, v.y);
            }
        }
    };
    // add every row this half holds and clear the window
    auto flush_all = [&]() {
        const int base_h = rbase + ((h - rbase) & 1);
#pragma unroll
        for (int i = 0; i < RH; ++i) {
            flush(base_h + 2 * i, acc[i]);
            acc[i] = Cx<T>::make(0, 0);
        }
    };
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 32; ++q) st.vk[q][W] = Cx<T>::make(0, 0);
    }
    for (int base = s; base < e; base += 32) {
        const int nb = min(32, e - base);
        __syncwarp();
        if (lane < nb) {
            const double2 g = pts[base + lane];
            const double2 v = fin[perm[base + lane] + M * b];
            int r0, c0;
            double v1, v2;
            local_origin<W>(g, tg, nrows, nf2, row_wrap, r0, c0, v1, v2);
            {
                T k1[W];
                es_weights<W, T>((T)v1, k1);
#pragma unroll
                for (int par = 0; par < 2; ++par) {
#pragma unroll
                    for (int p = 0; p < RP; ++p) {
                        const int a0 = par + 4 * p, a1 = par + 4 * p + 2;
                        st.k1[lane][par][p] = Cx<T>::make(a0 < W ? k1[a0 < W ? a0 : 0] : (T)0,
                                                          a1 < W ? k1[a1 < W ? a1 : 0] : (T)0);
                    }
                }
            }
            {
                T k2[W];
                es_weights<W, T>((T)v2, k2);
#pragma unroll
                for (int q = 0; q < W; ++q)
                    st.vk[lane][q] = Cx<T>::make((T)v.x * k2[q], (T)v.y * k2[q]);
            }
            const bool inside = r0 >= 0 && r0 + W <= tg.TR && c0 >= 0 && c0 + W <= tg.TC;
            st.org[lane] = make_int2(inside ? r0 : -1, c0);
        }
        __syncwarp();
        for (int q = 0; q < nb; ++q) {
            const int2 o = st.org[q];
            const int r0 = o.x;
            if (r0 < 0) continue;  // outside its bin's tile: cannot happen for binned points
            if (r0 != rbase) {
                if (rbase >= 0 && r0 - rbase >= W) flush_all();
                if (rbase < 0 || r0 - rbase >= W) {
                    rbase = r0;
                } else {
                    // rows rbase .. r0 - 1 are complete: the half of each row's parity adds it
                    // and slides its window
                    for (; rbase < r0; ++rbase) {
                        if ((rbase & 1) == h) {
                            flush(rbase, acc[0]);
#pragma unroll
                            for (int i = 0; i < RH - 1; ++i) acc[i] = acc[i + 1];
                            acc[RH - 1] = Cx<T>::make(0, 0);
                        }
                    }
                }
            }
            const unsigned dc = (unsigned)(c - o.y);
            const cx<T> vk = st.vk[q][dc < (unsigned)W ? dc : W];
            const int par = (h ^ r0) & 1;  // 0: this half holds the even-offset rows
#pragma unroll
            for (int p = 0; p < RP; ++p) {
                const cx<T> kk = st.k1[q][par][p];
                acc[2 * p].x = fma(vk.x, kk.x, acc[2 * p].x);
                acc[2 * p].y = fma(vk.y, kk.x, acc[2 * p].y);
                if (2 * p + 1 < RH) {
                    acc[2 * p + 1].x = fma(vk.x, kk.y, acc[2 * p + 1].x);
                    acc[2 * p + 1].y = fma(vk.y, kk.y, acc[2 * p + 1].y);
                }
            }
        }
    }
    if (rbase >= 0) flush_all();
}

// Type-1 spreading with the bin's whole tile in registers: one warp per bin, lane (h, c) owns
// tile column c (the tile is at most 16 columns wide) and every row of parity h, 2 NRH rows
// at most (row 2 k + h in acc[k]). A point of origin row r0 = 2 j + p reaches, in each half,
// registers j .. j + RW - 1 (RW = W / 2 + 1): register j + i of half h holds row offset
// 2 i + h - p. Per batch of 32 points each lane stages one point's row weights and its value
// times its column weights; the bin's points are sorted by origin row, so the batch splits
// into runs of one row pair j, and each run is added by a warp-uniform switch on j that names
// the registers statically: per point and lane, RW row weights, one column value and 2 RW
// FMAs. Nothing is added to U until the bin ends, when each lane adds its rows once: no window
// slides, no row is flushed twice, and a cell's sum runs over the bin's points in the same
// order as in spread16_kernel, so the two give the same values.
//
// Two staging layouts, each the faster one measured for its precision:
// - FP64 (SpreadPickStage): the row weights zero-padded, [0, 0, k_0 .. k_{W-1}, 0 ..], which a
//   lane reads at stride 2 from 2 + h - p; the W column values and a 0, of which a lane picks
//   its own by its offset from the point's first column; runs found point by point.
// - FP32 (SpreadRowStage): each half's RW row weights in 16-byte vectors, and the value at
//   every tile column (0 off the point), one load per lane; runs found by a ballot.
template <int W, class T>
struct SpreadPickStage {
    static constexpr int RW = W / 2 + 1;       // registers a point reaches in one half
    // [0, 0, k_0 .. k_{W-1}, 0 ..]; both rows an odd number of elements long, so that the lanes'
    // stores of their points' rows fall in distinct banks
    static constexpr int NK = 2 * RW + 3;
    static constexpr int NV = (W + 1) % 2 ? W + 1 : W + 2;
    T k1[32][NK];              // row weights, zero-padded
    cx<T> vk[32][NV];          // value x column weight; slot W is 0 for lanes off the point
    int2 org[32];              // origin row (or -1: skip) and column inside the tile
    long long roff[32];        // element offset of local row r in U (or -1: outside the grid)
};

template <int W, class T>
struct SpreadRowStage {  // T = float (the FP64 grids use SpreadPickStage)
    static constexpr int RW = W / 2 + 1;
    static constexpr int VPL = 16 / (int)sizeof(T);        // T per 16-byte load
    static constexpr int KP = (RW + VPL - 1) / VPL * VPL;  // row weights per half
    // rows padded to odd multiples of 16 bytes: the lanes' 16-byte stores of their points'
    // rows fall in distinct banks
    static constexpr int KS = 2 * KP + VPL;
    static constexpr int NV = 17;  // an odd number of values, for the same reason
    alignas(16) T kw[32][KS];  // [point][half KP + i]: weight of register j + i (0-padded)
    cx<T> vc[32][NV];          // [point][column]: value x column weight (0 off the point)
    long long roff[32];
};

template <int W, class T> struct SpreadRegLayout {
    using type = std::conditional_t<sizeof(T) == 8, SpreadPickStage<W, T>, SpreadRowStage<W, T>>;
};

// FP64: the points q, q + 1, .. < nb of origin row pair J; each point's operands are read
// before its run test, so the test does not hold up the loads. Returns the first point after
// the run.
template <int J, int W, int NRH, class T>
__device__ __forceinline__ int add_run(const SpreadPickStage<W, T>& st, int q, int nb, int h,
                                       int c, cx<T> (&acc)[NRH]) {
    constexpr int RW = SpreadPickStage<W, T>::RW;
    if constexpr (J + RW <= NRH) {
        do {
            const int2 o = st.org[q];
            const T* kr = st.k1[q] + 2 + h - (o.x & 1);
            T kw[RW];
#pragma unroll
            for (int i = 0; i < RW; ++i) kw[i] = kr[2 * i];
            const unsigned dc = (unsigned)(c - o.y);
            const cx<T> vk = st.vk[q][dc < (unsigned)W ? dc : W];
            if ((o.x >> 1) != J) break;  // the next pair (or a point outside the tile: -1)
#pragma unroll
            for (int i = 0; i < RW; ++i) {
                acc[J + i].x = fma(vk.x, kw[i], acc[J + i].x);
                acc[J + i].y = fma(vk.y, kw[i], acc[J + i].y);
            }
        } while (++q < nb);
        return q;
    } else {
        return q + 1;  // no point of a fitting grid reaches this pair
    }
}

// FP32: the points q0 .. q1 - 1, all of origin row pair J (row weights read as float4)
template <int J, int W, int NRH, class T>
__device__ __forceinline__ void add_run(const SpreadRowStage<W, T>& st, int q0, int q1, int h,
                                        int c, cx<T> (&acc)[NRH]) {
    using S = SpreadRowStage<W, T>;
    constexpr int RW = S::RW, KP = S::KP, KS = S::KS, NV = S::NV;
    if constexpr (J + RW <= NRH) {
        const T* kp = st.kw[q0] + h * KP;
        const cx<T>* vp = &st.vc[q0][c];
        for (int q = q0; q < q1; ++q, kp += KS, vp += NV) {
            T kw[KP];
#pragma unroll
            for (int u = 0; u < KP / 4; ++u) {
                const float4 t4 = reinterpret_cast<const float4*>(kp)[u];
                kw[4 * u] = t4.x;
                kw[4 * u + 1] = t4.y;
                kw[4 * u + 2] = t4.z;
                kw[4 * u + 3] = t4.w;
            }
            const cx<T> vk = *vp;
#pragma unroll
            for (int i = 0; i < RW; ++i) {
                acc[J + i].x = fma(vk.x, kw[i], acc[J + i].x);
                acc[J + i].y = fma(vk.y, kw[i], acc[J + i].y);
            }
        }
    }
}

// register pairs of rows each lane holds: the tile may be 2 NRH rows high
constexpr int kSpreadRegRows = 16;

// whether spread_reg_kernel covers a grid's bins: tiles at most 16 columns wide and origin
// rows r0 <= bin_rows - 1 whose window ends inside the held rows
__host__ __device__ constexpr bool spread_reg_fits(int w, int bin_rows, int bin_cols) {
    return w <= 10 && bin_cols + w - 1 <= 16 && bin_rows >= 1 &&
           (bin_rows - 1) / 2 <= kSpreadRegRows - (w / 2 + 1);
}

#define PF_ROW_PAIR_CASES(CASE)                                                               \
    CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) \
    CASE(11) CASE(12) CASE(13) CASE(14) CASE(15)

template <int W, class T>
__global__ void __launch_bounds__(128, 4)
spread_reg_kernel(const double2* __restrict__ pts, const int* __restrict__ perm,
                  const int4* __restrict__ slots, int nbusy, int nbc, int BR, int BC, int64_t M,
                  const double2* __restrict__ fin, int b, int nrows, int nf2, int row_wrap,
                  int plain, cx<T>* __restrict__ U) {
    using S = typename SpreadRegLayout<W, T>::type;
    constexpr bool kPick = std::is_same_v<S, SpreadPickStage<W, T>>;
    constexpr int RW = S::RW;
    constexpr int NRH = kSpreadRegRows;
    static_assert(NRH <= 16, "the row switch names 16 cases");
    static_assert(W <= 16, "a point's columns fit the 16-column tile");
    extern __shared__ __align__(16) unsigned char spread_reg_smem[];  // 4 stages
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h = lane >> 4, c = lane & 15;
    const int slot = blockIdx.x * 4 + warp;
    if (slot >= nbusy) return;
    const int4 sl = slots[slot];  // bin, first point, end
    const int bin = sl.x, s = sl.y, e = sl.z;
    const TileGeom tg = tile_geom<W>(bin, nbc, BR, BC);
    S& st = reinterpret_cast<S*>(spread_reg_smem)[warp];
    cx<T>* ub = U + (int64_t)nrows * nf2 * b;
    {
        // lane r: where local row r lands in U
        int gr = tg.tr0 + lane;
        if (row_wrap) gr = wrap(gr, nrows);
        st.roff[lane] = (lane < tg.TR && gr >= 0 && gr < nrows) ? (long long)gr * nf2 : -1;
        if constexpr (kPick) st.vk[lane][W] = Cx<T>::make(0, 0);
    }
    cx<T> acc[NRH];
#pragma unroll
    for (int i = 0; i < NRH; ++i) acc[i] = Cx<T>::make(0, 0);
    for (int base = s; base < e; base += 32) {
        const int nb = min(32, e - base);
        __syncwarp();
        int jl = -1;  // this lane's point's origin row pair (-1: none, or outside the tile)
        if (lane < nb) {
            const double2 g = pts[base + lane];
            const double2 v = fin[perm[base + lane] + M * b];
            int r0, c0;
            double v1, v2;
            local_origin<W>(g, tg, nrows, nf2, row_wrap, r0, c0, v1, v2);
            const bool inside = r0 >= 0 && r0 + W <= tg.TR && c0 >= 0 && c0 + W <= tg.TC;
            {
                T k1[W];
                es_weights<W, T>((T)v1, k1);
                auto at = [&](int a) -> T { return (a >= 0 && a < W) ? k1[(a >= 0 && a < W) ? a : 0] : (T)0; };
                if constexpr (kPick) {
#pragma unroll
                    for (int n = 0; n < S::NK; ++n) st.k1[lane][n] = at(n - 2);
                } else {
                    // even offsets for the half of parity p, odd ones for the other, stored
                    // as 16-byte vectors
                    constexpr int KP = S::KP;
                    T w[2 * KP];
                    if (r0 & 1) {
#pragma unroll
                        for (int i = 0; i < KP; ++i) {
                            w[i] = i < RW ? at(2 * i - 1) : (T)0;
                            w[KP + i] = i < RW ? at(2 * i) : (T)0;
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < KP; ++i) {
                            w[i] = i < RW ? at(2 * i) : (T)0;
                            w[KP + i] = i < RW ? at(2 * i + 1) : (T)0;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < KP / 2; ++u)
                        reinterpret_cast<float4*>(st.kw[lane])[u] =
                            make_float4(w[4 * u], w[4 * u + 1], w[4 * u + 2], w[4 * u + 3]);
                }
            }
            {
                T k2[W];
                es_weights<W, T>((T)v2, k2);
                if constexpr (kPick) {
#pragma unroll
                    for (int d = 0; d < W; ++d)
                        st.vk[lane][d] = Cx<T>::make((T)v.x * k2[d], (T)v.y * k2[d]);
                    st.org[lane] = make_int2(inside ? r0 : -1, c0);
                } else {
                    cx<T>* vr = st.vc[lane];
#pragma unroll
                    for (int cc = 0; cc < 16; ++cc) vr[cc] = Cx<T>::make(0, 0);
                    // (a point outside the tile writes somewhere in its row and is skipped)
                    vr += min(max(c0, 0), 16 - W);
#pragma unroll
                    for (int d = 0; d < W; ++d) vr[d] = Cx<T>::make((T)v.x * k2[d], (T)v.y * k2[d]);
                }
            }
            // a point outside its bin's tile (cannot happen for binned points) is skipped
            jl = inside ? (r0 >> 1) : -1;
        }
        __syncwarp();
        if constexpr (kPick) {
            // one switch per run of points of one origin row pair
            for (int q = 0; q < nb;) {
                const int r0 = st.org[q].x;
                if (r0 < 0) {
                    ++q;
                    continue;
                }
                switch (r0 >> 1) {
#define PF_RUN_CASE(J) case J: q = add_run<J, W, NRH, T>(st, q, nb, h, c, acc); break;
                    PF_ROW_PAIR_CASES(PF_RUN_CASE)
#undef PF_RUN_CASE
                    default: ++q; break;
                }
            }
        } else {
            // runs found by a ballot, one switch per run
            const int jprev = __shfl_up_sync(0xffffffffu, jl, 1);
            unsigned starts = __ballot_sync(0xffffffffu, lane < nb && (lane == 0 || jl != jprev));
            while (starts) {
                const int q0 = __ffs(starts) - 1;
                starts &= starts - 1;
                const int q1 = starts ? __ffs(starts) - 1 : nb;
                switch (__shfl_sync(0xffffffffu, jl, q0)) {
#define PF_RUN_CASE(J) case J: add_run<J, W, NRH, T>(st, q0, q1, h, c, acc); break;
                    PF_ROW_PAIR_CASES(PF_RUN_CASE)
#undef PF_RUN_CASE
                    default: break;
                }
            }
        }
    }
    __syncwarp();
    if (c < tg.TC) {
        const int gcol = wrap(tg.tc0 + c, nf2);
#pragma unroll
        for (int k = 0; k < NRH; ++k) {
            const cx<T> v = acc[k];
            const long long off = st.roff[2 * k + h];
            if (off >= 0 && (v.x != 0.0 || v.y != 0.0)) {
                cx<T>* qd = ub + off + gcol;
                if (plain) {
                    // no other tile of this launch reaches the cell (bins launched by colour)
                    cx<T> u = *qd;
                    u.x += v.x;
                    u.y += v.y;
                    *qd = u;
                } else {
                    atomicAdd(reinterpret_cast<T*>(qd), v.x);
                    atomicAdd(reinterpret_cast<T*>(qd) + 1, v.y);
                }
            }
        }
    }
}
#undef PF_ROW_PAIR_CASES

// groups per resident block from which the one-transform interpolation is pipelined
constexpr int kInterpPipeGroups = 4;

template <int W, class T>
static int launch_interp(const NufftGrid& g, NufftDev& d, double2* f, int B, cudaStream_t s) {
    const int tile_elems = (g.bin_rows + W - 1) * ((g.igroup * g.bin_cols + W - 1) | 1);
    if (B == 1 && g.interp_pipe && g.igroup * g.bin_cols + W - 1 <= 32 && g.nisb > 0) {
        const size_t smem2 = 2 * sizeof(cx<T>) * (size_t)tile_elems;
        if (smem2 > 48 * 1024)
            PF_CUDA(cudaFuncSetAttribute(interp_pipe_kernel<W, T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
        int per = 0, dev = 0, nsm = 0;
        PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, interp_pipe_kernel<W, T>, 128, smem2));
        PF_CUDA(cudaGetDevice(&dev));
        PF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const int grid = std::max(1, std::min(g.nisb, std::max(1, per) * nsm));
        // the copy ahead pays once each resident block takes several groups (measured: 3-4%
        // faster at lmax 2048, 4 to 8 groups per block; 32% slower at lmax 1024, under 2)
        if (g.nisb >= kInterpPipeGroups * grid) {
            PF_CUDA(cudaMemsetAsync(d.counter.p, 0, sizeof(int), s));
            interp_pipe_kernel<W, T><<<grid, 128, smem2, s>>>(
                d.ipts.as<double2>(), d.iperm.as<int>(), d.binstart.as<int>(), d.iorder.as<int>(),
                g.nisb, g.nbc, g.igroup, g.nsbc, g.bin_rows, g.bin_cols, d.U.as<cx<T>>(), g.nrows,
                g.nf2, g.row_wrap, tile_elems, f, d.counter.as<int>());
            return check_launch("interp_pipe_kernel");
        }
    }
    const size_t smem = sizeof(cx<T>) * (size_t)tile_elems;
    if (smem > 48 * 1024)
        PF_CUDA(cudaFuncSetAttribute(interp_kernel<W, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    interp_kernel<W, T><<<g.nisb, 128, smem, s>>>(
        d.ipts.as<double2>(), d.iperm.as<int>(), d.binstart.as<int>(), d.iorder.as<int>(), g.nbc,
        g.igroup, g.nsbc, g.bin_rows, g.bin_cols, g.M, d.U.as<cx<T>>(), g.nrows, g.nf2,
        g.row_wrap, B, f);
    return check_launch("interp_kernel");
}

template <int W, class T>
static int launch_spread(const NufftGrid& g, NufftDev& d, const double2* f, int B, cudaStream_t s) {
    // with the deterministic option, one launch per bin colour in a fixed order and plain adds
    const bool col = g.deterministic && g.ncolors > 0;
    const int nl = col ? g.ncolors : 1;
    for (int b = 0; b < B; ++b) {
        for (int k = 0; k < nl; ++k) {
            const int n = col ? g.color_off[k + 1] - g.color_off[k] : g.nbusy;
            const int* order = col ? d.sorder.as<int>() + g.color_off[k] : d.binorder.as<int>();
            if (n == 0) continue;
            if (g.spread_reg && spread_reg_fits(W, g.bin_rows, g.bin_cols)) {
                constexpr int WR = W <= 10 ? W : 2;
                const size_t smem = 4 * sizeof(typename SpreadRegLayout<WR, T>::type);
                if (smem > 48 * 1024)
                    PF_CUDA(cudaFuncSetAttribute(spread_reg_kernel<WR, T>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                const int4* sl = col ? d.sslot.as<int4>() + g.color_off[k] : d.bslot.as<int4>();
                spread_reg_kernel<WR, T><<<(n + 3) / 4, 128, smem, s>>>(
                    d.pts.as<double2>(), d.perm.as<int>(), sl, n, g.nbc, g.bin_rows, g.bin_cols,
                    g.M, f, b, g.nrows, g.nf2, g.row_wrap, col ? 1 : 0, d.U.as<cx<T>>());
                PF_TRY(check_launch("spread_reg_kernel"));
            } else if (W <= 10 && g.bin_cols + W - 1 <= 16) {
                spread16_kernel<(W <= 10 ? W : 2), T><<<(n + 3) / 4, 128, 0, s>>>(
                    d.pts.as<double2>(), d.perm.as<int>(), d.binstart.as<int>(), order, n, g.nbc,
                    g.bin_rows, g.bin_cols, g.M, f, b, g.nrows, g.nf2, g.row_wrap, col ? 1 : 0,
                    d.U.as<cx<T>>());
                PF_TRY(check_launch("spread16_kernel"));
            } else {
                constexpr int NW = SpreadWarps<W>::N;
                spread_kernel<W, T><<<(n + NW - 1) / NW, NW * 32, 0, s>>>(
                    d.pts.as<double2>(), d.perm.as<int>(), d.binstart.as<int>(), order, n, g.nbc,
                    g.bin_rows, g.bin_cols, g.M, f, b, g.nrows, g.nf2, g.row_wrap, col ? 1 : 0,
                    d.U.as<cx<T>>());
                PF_TRY(check_launch("spread_kernel"));
            }
        }
    }
    return 0;
}

// kernel widths: 2..16 in FP64; the mixed form runs at tol >= 1e-6, so w <= 8 there
#define PF_WIDTH_SWITCH(CALL)                                                               \
    switch (g.w) {                                                                          \
        case 2: return CALL(2); case 3: return CALL(3); case 4: return CALL(4);             \
        case 5: return CALL(5); case 6: return CALL(6); case 7: return CALL(7);             \
        case 8: return CALL(8);                                                             \
        default: break;                                                                     \
    }                                                                                       \
    if constexpr (sizeof(T) == sizeof(double)) {                                            \
        switch (g.w) {                                                                      \
            case 9: return CALL(9); case 10: return CALL(10); case 11: return CALL(11);     \
            case 12: return CALL(12); case 13: return CALL(13); case 14: return CALL(14);   \
            case 15: return CALL(15); case 16: return CALL(16);                             \
            default: break;                                                                 \
        }                                                                                   \
    }                                                                                       \
    set_error("unsupported NUFFT kernel width");                                            \
    return 7;

template <class T>
static int interp_any(const NufftGrid& g, NufftDev& d, double2* f, int B, cudaStream_t s) {
#define PF_CALL(WW) launch_interp<WW, T>(g, d, f, B, s)
    PF_WIDTH_SWITCH(PF_CALL)
#undef PF_CALL
}

template <class T>
static int spread_any(const NufftGrid& g, NufftDev& d, const double2* f, int B, cudaStream_t s) {
#define PF_CALL(WW) launch_spread<WW, T>(g, d, f, B, s)
    PF_WIDTH_SWITCH(PF_CALL)
#undef PF_CALL
}
#undef PF_WIDTH_SWITCH

template <class T>
static int type2_impl(const NufftGrid& g, NufftDev& d, const double2* modes, double2* f, int B,
                      int dir, cudaStream_t s, StageClock* clk) {
    {
        dim3 grid(nblk(g.nf1, 256), g.ncols, B);
        pad_kernel<T><<<grid, 256, 0, s>>>(modes, g.n1, g.ncols, g.nf1, d.mult1.as<double2>(),
                                           d.dec2.as<double>(), d.pad.as<cx<T>>());
        PF_TRY(check_launch("pad_kernel"));
    }
    clock_mark(clk, kStPad, s);
    PF_CUFFT(cufftSetStream(d.f1, s));
    PF_TRY(fine_fft(d.f1, d.pad.p, g.fp32, dir));
    clock_mark(clk, kStFft1Fwd, s);
    if (d.have_maps) {
        const int ntc = (g.ncols + 31) / 32, ntr = (g.nrows + 31) / 32;
        const int nzc = (g.gap_hi - g.gap_lo + 255) / 256;
        dim3 grid(ntc * ntr + ntr * nzc, 1, B);
        rows_fwd_tma_kernel<T><<<grid, dim3(32, 8), 0, s>>>(
            d.pad_map, d.pad.as<cx<T>>(), g.nf1, g.ncols, g.row0, g.nrows, g.nf2,
            d.colp2.as<int>(), g.gap_lo, g.gap_hi, ntc, ntr, nzc, d.U.as<cx<T>>());
        PF_TRY(check_launch("rows_fwd_tma_kernel"));
    } else {
        dim3 grid((g.nf2 + 31) / 32, (g.nrows + 31) / 32, B);
        rows_fwd_kernel<T><<<grid, dim3(32, 8), 0, s>>>(d.pad.as<cx<T>>(), g.nf1, g.ncols, g.row0,
                                                        g.nrows, g.nf2, d.p2col.as<int>(),
                                                        d.U.as<cx<T>>());
        PF_TRY(check_launch("rows_fwd_kernel"));
    }
    clock_mark(clk, kStRowsFwd, s);
    PF_CUFFT(cufftSetStream(d.f2, s));
    PF_TRY(fine_fft(d.f2, d.U.p, g.fp32, dir));
    clock_mark(clk, kStFft2Fwd, s);
    PF_TRY(interp_any<T>(g, d, f, B, s));
    clock_mark(clk, kStInterp, s);
    return 0;
}

template <class T>
static int type1_impl(const NufftGrid& g, NufftDev& d, const double2* f, double2* modes, int B,
                      int dir, cudaStream_t s, StageClock* clk) {
    PF_CUDA(cudaMemsetAsync(d.U.p, 0, sizeof(cx<T>) * (size_t)g.nrows * g.nf2 * B, s));
    PF_TRY(spread_any<T>(g, d, f, B, s));
    clock_mark(clk, kStSpread, s);
    PF_CUFFT(cufftSetStream(d.f2, s));
    PF_TRY(fine_fft(d.f2, d.U.p, g.fp32, dir));
    clock_mark(clk, kStFft2Adj, s);
    if (d.have_maps) {
        const int ntc = (g.ncols + 31) / 32, ntp = (g.nf1 + 31) / 32;
        dim3 grid(ntc * ntp, 1, B);
        rows_adj_tma_kernel<T><<<grid, dim3(32, 8), 0, s>>>(
            d.U_map, d.U.as<cx<T>>(), g.nf1, g.ncols, g.row0, g.nrows, g.nf2, d.colp2.as<int>(),
            ntc, d.pad.as<cx<T>>());
        PF_TRY(check_launch("rows_adj_tma_kernel"));
    } else {
        dim3 grid((g.ncols + 31) / 32, (g.nf1 + 31) / 32, B);
        rows_adj_kernel<T><<<grid, dim3(32, 8), 0, s>>>(d.U.as<cx<T>>(), g.nf1, g.ncols, g.row0,
                                                        g.nrows, g.nf2, d.colp2.as<int>(),
                                                        d.pad.as<cx<T>>());
        PF_TRY(check_launch("rows_adj_kernel"));
    }
    clock_mark(clk, kStRowsAdj, s);
    PF_CUFFT(cufftSetStream(d.f1, s));
    PF_TRY(fine_fft(d.f1, d.pad.p, g.fp32, dir));
    clock_mark(clk, kStFft1Adj, s);
    {
        dim3 grid(nblk(g.n1, 256), g.ncols, B);
        unpad_kernel<T><<<grid, 256, 0, s>>>(d.pad.as<cx<T>>(), g.n1, g.ncols, g.nf1,
                                             d.mult1.as<double2>(), d.dec2.as<double>(), modes);
        PF_TRY(check_launch("unpad_kernel"));
    }
    clock_mark(clk, kStUnpad, s);
    return 0;
}

int nufft_type2(const NufftGrid& g, NufftDev& d, const double2* modes, double2* f, int B,
                int iflag, cudaStream_t s, StageClock* clk) {
    const int dir = iflag > 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
    return g.fp32 ? type2_impl<float>(g, d, modes, f, B, dir, s, clk)
                  : type2_impl<double>(g, d, modes, f, B, dir, s, clk);
}

int nufft_type1(const NufftGrid& g, NufftDev& d, const double2* f, double2* modes, int B,
                int iflag, cudaStream_t s, StageClock* clk) {
    const int dir = iflag > 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
    return g.fp32 ? type1_impl<float>(g, d, f, modes, B, dir, s, clk)
                  : type1_impl<double>(g, d, f, modes, B, dir, s, clk);
}

// ---------------------------------------------------------------------------------------
// Direct leaf phases (src/Direct.jl:74-84,102-114): exact cis(m phi) per (point, order)
// ---------------------------------------------------------------------------------------
__global__ void direct_sum_kernel(const double2* __restrict__ G, const double* __restrict__ phi,
                                  int64_t M, int L, int B, double2* __restrict__ f) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ph = phi[i];
        for (int b = 0; b < B; ++b) {
            const double2* Gb = G + (int64_t)M * (2 * L + 1) * b;
            double2 acc = Gb[i + M * (int64_t)L];
            for (int m = 1; m <= L; ++m) {
                double sn, cs;
                sincos((double)m * ph, &sn, &cs);
                const double2 gp = Gb[i + M * (int64_t)(L + m)];
                const double2 gm = Gb[i + M * (int64_t)(L - m)];
                acc.x += (gp.x * cs - gp.y * sn) + (gm.x * cs + gm.y * sn);
                acc.y += (gp.x * sn + gp.y * cs) + (gm.y * cs - gm.x * sn);
            }
            f[i + M * b] = acc;
        }
    }
}

__global__ void direct_spread_kernel(const double2* __restrict__ f, const double* __restrict__ phi,
                                     int64_t M, int L, int B, double2* __restrict__ G) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double ph = phi[i];
        for (int b = 0; b < B; ++b) {
            double2* Gb = G + (int64_t)M * (2 * L + 1) * b;
            const double2 v = f[i + M * b];
            Gb[i + M * (int64_t)L] = v;
            for (int m = 1; m <= L; ++m) {
                double sn, cs;
                sincos((double)m * ph, &sn, &cs);
                Gb[i + M * (int64_t)(L + m)] = make_double2(v.x * cs + v.y * sn, v.y * cs - v.x * sn);
                Gb[i + M * (int64_t)(L - m)] = make_double2(v.x * cs - v.y * sn, v.y * cs + v.x * sn);
            }
        }
    }
}

int direct_phase_sum(const double2* G, const double* phi, int64_t M, int L, int B, double2* f,
                     cudaStream_t s) {
    direct_sum_kernel<<<nblk(M, 128), 128, 0, s>>>(G, phi, M, L, B, f);
    return check_launch("direct_sum_kernel");
}

int direct_phase_spread(const double2* f, const double* phi, int64_t M, int L, int B, double2* G,
                        cudaStream_t s) {
    direct_spread_kernel<<<nblk(M, 128), 128, 0, s>>>(f, phi, M, L, B, G);
    return check_launch("direct_spread_kernel");
}

// ---------------------------------------------------------------------------------------
// DFS periodisation (src/DFS.jl:13-56)
// ---------------------------------------------------------------------------------------
__global__ void dfs_double_kernel(const double2* __restrict__ F, double2* __restrict__ Ft, int Nth,
                                  int Nph, int B, double sgn) {
    const int64_t n = (int64_t)2 * Nth * Nph * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % (2 * Nth));
        const int64_t rest = t / (2 * Nth);
        const int j = (int)(rest % Nph);
        const int b = (int)(rest / Nph);
        double2 v;
        if (i < Nth) {
            v = F[i + (int64_t)Nth * j + (int64_t)Nth * Nph * b];
        } else {
            const int ii = i - Nth;
            const int js = (j + Nph / 2) % Nph;
            const double2 u = F[(Nth - 1 - ii) + (int64_t)Nth * js + (int64_t)Nth * Nph * b];
            v = make_double2(sgn * u.x, sgn * u.y);
        }
        Ft[t] = v;
    }
}

__global__ void dfs_fold_kernel(double2* __restrict__ F, const double2* __restrict__ Ft, int Nth,
                                int Nph, int B, double sgn) {
    const int64_t n = (int64_t)Nth * Nph * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % Nth);
        const int64_t rest = t / Nth;
        const int j = (int)(rest % Nph);
        const int b = (int)(rest / Nph);
        const int js = ((j - Nph / 2) % Nph + Nph) % Nph;
        const double2 a = Ft[i + (int64_t)2 * Nth * j + (int64_t)2 * Nth * Nph * b];
        const double2 u = Ft[(2 * Nth - 1 - i) + (int64_t)2 * Nth * js + (int64_t)2 * Nth * Nph * b];
        F[t] = make_double2(a.x + sgn * u.x, a.y + sgn * u.y);
    }
}

int dfs_double(const double2* F, double2* Ft, int Nth, int Nph, int B, int spin, cudaStream_t s) {
    const double sgn = (spin % 2 == 0) ? 1.0 : -1.0;
    dfs_double_kernel<<<nblk((int64_t)2 * Nth * Nph * B, 256), 256, 0, s>>>(F, Ft, Nth, Nph, B, sgn);
    return check_launch("dfs_double_kernel");
}

int dfs_fold(double2* F, const double2* Ft, int Nth, int Nph, int B, int spin, cudaStream_t s) {
    const double sgn = (spin % 2 == 0) ? 1.0 : -1.0;
    dfs_fold_kernel<<<nblk((int64_t)Nth * Nph * B, 256), 256, 0, s>>>(F, Ft, Nth, Nph, B, sgn);
    return check_launch("dfs_fold_kernel");
}

}  // namespace pf
