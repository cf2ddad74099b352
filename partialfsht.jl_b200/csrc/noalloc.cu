// Direct synthesis that allocates nothing: pfsht_direct_forward_noalloc.
//
// Some callers cannot allocate device memory when they need a transform: code running
// inside a framework that owns all of the device's memory through its own pool (so a
// cudaMalloc of the library would fail or fragment it), code on a device whose memory a
// graph or another process has reserved in advance, or small utility calls for which a
// plan's allocations and their cudaMalloc/cudaFree synchronisation cost more than the work.
// This entry point evaluates f_i = sum_lm a_lm Y_lm(theta_i, phi_i) for a small point set
// (the Direct leaf's synthesis, src/Direct.jl:60-86) with every intermediate held in one
// fixed array of device memory that the library declares at file scope, so it makes no
// cudaMalloc, cudaFree or other allocating call at all. The caller still passes the points,
// the coefficients and the output buffer, all on the device.
//
// Limits and behaviour:
//   - the scratch array is kNoAllocScratchBytes (32 MiB); it holds the per-point tables,
//     the recurrence coefficients for lmax and the npts x (2 lmax + 1) ring columns, and a
//     call whose sizes need more is rejected with PFSHT_ERR_ARGUMENT before any launch;
//   - every device that loads the library holds this array until the process exits;
//   - the first call on a device looks up the array's device address (cudaGetSymbolAddress)
//     with that device current; make that first call before any stream capture. The address
//     is kept per device ordinal, which assumes the device's primary context (the one the CUDA
//     runtime uses); after cudaDeviceReset, or from another driver-API context on the same
//     device, the kept address is stale and the entry point must not be called;
//   - lmax is at most kNoAllocMaxLmax (the recurrence table alone would not fit above it);
//   - all calls share the one array and the array keeps the last call's contents, so calls
//     that overlap on the GPU (different streams, or different host threads on one device)
//     race and must be serialised by the caller. Every region a call reads is written by the
//     same call first, so no clearing between calls is needed.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <string>

#include "../../include/pfsht_b200.h"
#include "internal.cuh"

namespace pf {

static constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
static constexpr int kNoAllocTile = 64;                    // rings (points) per work item
static constexpr int kNoAllocMaxLmax = 2048;               // its (beta, g) table alone nearly fills the array

// the scratch array: host code must not take its address directly (see below)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// device address of g_noalloc_scratch per device ordinal, looked up once per device
static constexpr int kMaxDevices = 64;
static std::atomic<void*> g_noalloc_ptr[kMaxDevices];

static int noalloc_scratch(void** out) {
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal out of range for the no-allocation path");
        return 1;
    }
    void* p = g_noalloc_ptr[dev].load();
    if (!p) {
        // in host code the array's name is only a host-side stand-in; the device address
        // comes from the runtime, with this device current
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error(std::string("cudaGetSymbolAddress of the no-allocation scratch: ") +
                      cudaGetErrorString(e));
            return 4;
        }
        g_noalloc_ptr[dev].store(p);
    }
    *out = p;
    return 0;
}

// scratch layout (byte offsets, 256-aligned sections)
struct NoAllocLayout {
    size_t cos_t, log2sin, log2c, aboff, ab, items, G, total;
    int nitems;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// all sizes in 64-bit arithmetic: callers bound lmax <= kNoAllocMaxLmax and npts < 2^31, so
// no product below can overflow, and the total decides whether the call fits
static NoAllocLayout noalloc_layout(int64_t M, int64_t L) {
    NoAllocLayout y;
    const int64_t nab = L >= 1 ? L * (L - 1) / 2 + 1 : 1;  // sum over m of max(0, L-m-1)
    const int64_t ntile = (M + kNoAllocTile - 1) / kNoAllocTile;
    const int64_t nitems = (L + 1) * ntile;
    y.nitems = nitems > INT32_MAX ? -1 : (int)nitems;
    size_t o = 0;
    y.cos_t = o; o = align256(o + sizeof(double) * (size_t)M);
    y.log2sin = o; o = align256(o + sizeof(double) * (size_t)M);
    y.log2c = o; o = align256(o + sizeof(double) * (size_t)(L + 1));
    y.aboff = o; o = align256(o + sizeof(int64_t) * (size_t)(L + 1));
    y.ab = o; o = align256(o + sizeof(double2) * (size_t)nab);
    y.items = o; o = align256(o + sizeof(RingItem) * (size_t)nitems);
    y.G = o; o = align256(o + sizeof(double2) * (size_t)M * (size_t)(2 * L + 1));
    y.total = o;
    return y;
}

// point tables, the sectorial log-prefactor (src/Legendre.jl:65-75), the coefficient-table
// offsets and the work items (order m, tile of points), all written into the scratch
__global__ void noalloc_prep_kernel(const double* __restrict__ theta, int64_t M, int L,
                                    double* __restrict__ cos_t, double* __restrict__ log2sin,
                                    double* __restrict__ log2c, int64_t* __restrict__ aboff,
                                    RingItem* __restrict__ items, int64_t ntile) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = tid; i < M; i += nthr) {
        double s, c;
        sincos(theta[i], &s, &c);
        const double as = fabs(s);
        cos_t[i] = c;
        log2sin[i] = as > 0 ? log2(as) : -INFINITY;
    }
    for (int64_t k = tid; k < (int64_t)(L + 1) * ntile; k += nthr) {
        const int m = (int)(k / ntile), t = (int)(k % ntile);
        const int j0 = t * kNoAllocTile;
        const int n = (int)min((int64_t)kNoAllocTile, M - j0);
        items[k] = whole_item(m, j0, n, (t == 0 ? kItemFirst : 0) | (ntile == 1 ? kItemSole : 0), L);
    }
    for (int m = (int)tid; m <= L; m += (int)nthr) {
        int64_t off = 0;
        // offsets of the per-order coefficient runs: sum over m' < m of max(0, L - m' - 1)
        const int64_t full = min(m, max(L - 1, 0));
        off = full * (L - 1) - full * (full - 1) / 2;
        aboff[m] = off;
    }
    if (tid == 0) {
        double acc = -log2(sqrt(4.0 * 3.141592653589793));
        log2c[0] = acc;
        for (int m = 1; m <= L; ++m) {
            acc += log2(sqrt((double)(2 * m + 1) / (double)(2 * m)));
            log2c[m] = acc;
        }
    }
}

static int direct_forward_noalloc(const double* theta, const double* phi, int64_t M, int L,
                                  const double2* alm, double2* f, cudaStream_t s) {
    const NoAllocLayout y = noalloc_layout(M, L);
    if (y.total > kNoAllocScratchBytes || y.nitems < 0) {
        set_error("pfsht_direct_forward_noalloc: npts = " + std::to_string(M) + " at lmax = " +
                  std::to_string(L) + " needs " + std::to_string(y.total) +
                  " bytes of scratch, above the fixed " + std::to_string(kNoAllocScratchBytes) +
                  " (about npts * (2 lmax + 1) * 16 bytes must fit); use a plan instead");
        return 1;
    }
    void* base = nullptr;
    PF_TRY(noalloc_scratch(&base));
    unsigned char* b = static_cast<unsigned char*>(base);
    double* cos_t = reinterpret_cast<double*>(b + y.cos_t);
    double* log2sin = reinterpret_cast<double*>(b + y.log2sin);
    double* log2c = reinterpret_cast<double*>(b + y.log2c);
    int64_t* aboff = reinterpret_cast<int64_t*>(b + y.aboff);
    double2* ab = reinterpret_cast<double2*>(b + y.ab);
    RingItem* items = reinterpret_cast<RingItem*>(b + y.items);
    double2* G = reinterpret_cast<double2*>(b + y.G);
    const int64_t ntile = (M + kNoAllocTile - 1) / kNoAllocTile;
    const int64_t work = std::max<int64_t>(M, (int64_t)(L + 1) * ntile);
    const unsigned grid = (unsigned)std::min<int64_t>((work + 255) / 256, 4096);
    noalloc_prep_kernel<<<grid, 256, 0, s>>>(theta, M, L, cos_t, log2sin, log2c, aboff, items, ntile);
    PF_TRY(check_launch("noalloc_prep_kernel"));
    if (L >= 2) PF_TRY(launch_ab_table(L, L, 64, aboff, ab, s));
    RingTables t;
    t.cos_t = cos_t;
    t.log2sin = log2sin;
    t.log2c = log2c;
    t.w = nullptr;
    t.ab = ab;
    t.aboff = aboff;
    t.lmax = L;
    t.nrings = (int)M;
    RingOut o;
    o.ld = M;
    o.bstride = M * (2 * L + 1);
    o.col_off = L;
    o.nrows = (int)M;
    o.reflect = 0;
    o.nrings_out = (int)M;
    o.zero_rest = 0;  // every point keeps every order: all of G is written
    RingItems it;
    it.items = items;
    it.nitems = y.nitems;
    it.rmax = 2;
    PF_TRY(ring_forward(t, o, it, alm, G, 1, s));
    return direct_phase_sum(G, phi, M, L, 1, f, s);
}

}  // namespace pf

extern "C" pfsht_status pfsht_direct_forward_noalloc(const double* theta, const double* phi,
                                                     int64_t npts, int32_t lmax, const void* alm,
                                                     void* f, void* stream) {
    if (!theta || !phi || !alm || !f) {
        pf::set_error("pfsht_direct_forward_noalloc: NULL argument");
        return PFSHT_ERR_ARGUMENT;
    }
    if (npts < 1 || lmax < 0 || npts > INT32_MAX) {
        pf::set_error("pfsht_direct_forward_noalloc: need npts >= 1 and lmax >= 0");
        return PFSHT_ERR_ARGUMENT;
    }
    if (lmax > pf::kNoAllocMaxLmax) {
        pf::set_error("pfsht_direct_forward_noalloc: lmax = " + std::to_string(lmax) +
                      " is above the fixed scratch's limit of " +
                      std::to_string(pf::kNoAllocMaxLmax) + "; use a plan instead");
        return PFSHT_ERR_ARGUMENT;
    }
    return (pfsht_status)pf::direct_forward_noalloc(theta, phi, npts, lmax, (const double2*)alm,
                                                    (double2*)f, (cudaStream_t)stream);
}
