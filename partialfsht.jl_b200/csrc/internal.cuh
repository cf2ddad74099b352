// Internal declarations shared by the CUDA sources of libpfsht_b200.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "geometry.hpp"
#include "planner.hpp"

namespace pf {

// ---------------------------------------------------------------------------------------
// error plumbing (thread-local last error; C ABI returns codes)
// ---------------------------------------------------------------------------------------
void set_error(const std::string& msg);
const std::string& get_error();

struct Status {
    int code = 0;
    static Status ok() { return Status{}; }
};

#define PF_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            ::pf::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));       \
            return _e == cudaErrorMemoryAllocation ? 5 : 4;                             \
        }                                                                               \
    } while (0)

#define PF_CUFFT(call)                                                                  \
    do {                                                                                \
        cufftResult _r = (call);                                                        \
        if (_r != CUFFT_SUCCESS) {                                                      \
            ::pf::set_error(std::string(#call) + ": cuFFT error " + std::to_string((int)_r)); \
            return _r == CUFFT_ALLOC_FAILED ? 5 : 4;                                    \
        }                                                                               \
    } while (0)

#define PF_TRY(call)                                                                    \
    do {                                                                                \
        int _s = (call);                                                                \
        if (_s != 0) return _s;                                                         \
    } while (0)

// device allocation owned by a plan; freed in the destructor
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf();
    int alloc(size_t n);
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// ---------------------------------------------------------------------------------------
// ring pass (ring.cu)
// ---------------------------------------------------------------------------------------
// One work item: order m, rings [j0, j0 + n), degrees [lbeg, lend]. An item that starts at
// lbeg = m seeds its recurrence from the sectorial value; a later degree segment (lbeg > m)
// starts from the recurrence state saved at plan time, ck_p/ck_E[ck + k] for ring j0 + k.
enum { kItemFirst = 1, kItemSole = 2 };  // first tile of its order / only tile of its order
struct RingItem {
    int m, j0, n, flags;
    int lbeg, lend;
    int ck;   // checkpoint index of ring j0 (-1: seed at l = m)
    int pad_;
};
__host__ __device__ inline RingItem whole_item(int m, int j0, int n, int flags, int lmax) {
    return RingItem{m, j0, n, flags, m, lmax, -1, 0};
}

struct RingTables {
    const double* cos_t = nullptr;    // nrings, reflection sign folded in
    const double* log2sin = nullptr;  // nrings
    const double* log2c = nullptr;    // lmax + 1
    const double* w = nullptr;        // nrings window, or null for 1
    const double2* ab = nullptr;      // (beta_l, g_l) of the monic recurrence, per m from l = m + 2
    const int64_t* aboff = nullptr;   // lmax + 1 offsets into ab
    const double2* ck_p = nullptr;    // saved monic state (q_{l-1}, q_{l-2}) at segment starts
    const int* ck_E = nullptr;        // and its block exponent
    int lmax = 0;
    int nrings = 0;
    int mix = 0;       // FP32 accumulation (mixed form)
    int stride = 64;   // renormalisation block in degrees: 64 (FP64), 16 (mixed)
};

// Degree segments of the ring pass: order m is walked as nseg[m] pieces that start on the
// renormalisation schedule (l = m + 2 + 64 q), so each piece can run as its own item from
// a recurrence state saved once at plan time. Checkpoint of segment s >= 1, ring j:
// ckbase[m] + (s - 1) * (jhi[m] - jlo[m] + 1) + (j - jlo[m]).
struct RingSegments {
    int seg_degrees = 0;               // target segment length (multiple of 64); 0 = none
    std::vector<int> nseg;             // lmax + 1
    std::vector<int> nblk;             // lmax + 1: 64-degree blocks from l = m + 2
    std::vector<int64_t> ckbase;       // lmax + 1
    int64_t nstates = 0;
    DevBuf ck_p, ck_E;
    // first degree of segment s of order m (s >= 1)
    int seg_first(int m, int s) const {
        return m + 2 + 64 * (int)(((int64_t)s * nblk[m]) / nseg[m]);
    }
};

// Layout of the ring-side array: column-major (ld x ncols x B), column of order m at
// col_off + m; reflect writes/reads the mirrored row nrows - 1 - j too (DFS rows).
struct RingOut {
    int64_t ld = 0;       // leading dimension (rows)
    int64_t bstride = 0;  // elements between transforms
    int col_off = 0;
    int nrows = 0;
    int reflect = 0;
    double spin_sgn = 1.0;
    int nrings_out = 0;   // rings of the ring set (rows 0..nrings_out-1 belong to rings)
    int zero_rest = 0;    // forward writes zeros for the rings an order does not retain
};

// device view of one item list
struct RingItems {
    const RingItem* items = nullptr;
    int nitems = 0;
    int rmax = 4;                          // tile = 32 * rmax rings
    const unsigned char* sole_m = nullptr; // lmax + 1: order covered by a single tile
    const int* jlo = nullptr;              // lmax + 1 retained ring range
    const int* jhi = nullptr;
};

struct RingItemsOwner {
    DevBuf items, sole, jlo, jhi;
    RingItems view;
    std::vector<RingItem> host;  // the items, in launch order
};

// one plan of a batched ring pass, as the batched kernels read it from device memory
struct RingSlot {
    RingTables t;   // the adjoint's tables
    RingTables tf;  // the forward's (the mixed form's forward runs in FP64 on its own table)
    RingOut o;
    const int* jlo = nullptr;
    const int* jhi = nullptr;
    double2* H = nullptr;     // the plan's column array
    int allow_sole = 0;       // adjoint: orders covered by one tile store instead of adding
    int ptr = 0;              // index of the plan's coefficient array in the pointer table
};
struct BatchItem {
    RingItem it;
    int slot;   // plan
    int b0;     // first transform of the pass
};
// the items of one kernel shape: rings per lane (rmax), transforms per pass (nb), mixed
struct RingBatchGroup {
    int rmax = 1, nb = 1, mix = 0;
    DevBuf items;
    int nitems = 0;
};
// what the grouping needs of one plan
struct RingBatchPlan {
    const std::vector<RingItem>* items;
    int B, rmax, mix;
};
// all plans' items of one direction in one persistent launch (every tile shape, heaviest first)
struct RingMerged {
    DevBuf items;    // BatchItem[nitems], it.pad_ = shape code
    DevBuf counter;  // next item to pull
    int nitems = 0;
    int grid = 1;    // resident blocks
};
// one group per kernel shape, items of all plans heaviest first
int build_ring_batch(const std::vector<RingBatchPlan>& plans, bool adjoint,
                     std::vector<std::unique_ptr<RingBatchGroup>>& groups, cudaStream_t s);
// the ring passes of all plans: one launch per group; coefficient arrays through ptrs
int ring_forward_batch(const RingSlot* slots, const std::vector<std::unique_ptr<RingBatchGroup>>& groups,
                       void* const* ptrs, cudaStream_t s);
int ring_adjoint_batch(const RingSlot* slots, const std::vector<std::unique_ptr<RingBatchGroup>>& groups,
                       void* const* ptrs, cudaStream_t s);
// the merged list of one direction; shapes the persistent kernel does not take stay in `rest`
// (launched per shape as above)
int build_ring_merged(const std::vector<RingBatchPlan>& plans, bool adjoint, RingMerged& mg,
                      std::vector<std::unique_ptr<RingBatchGroup>>& rest, cudaStream_t s);
// zero the counter and launch the persistent pass (inside a capture: a memset node and a kernel)
int ring_merged_launch(const RingSlot* slots, const RingMerged& mg, bool adjoint, void* const* ptrs,
                       cudaStream_t s);
// alm_prepare of one plan whose coefficient array is ptrs[ptr]
int alm_prepare_ptr(void* const* ptrs, int ptr, int L, int B, const unsigned char* sole_m,
                    int allow_sole, cudaStream_t s);

int build_ab_table(int lmax, int mmax, int stride, DevBuf& ab, DevBuf& aboff, cudaStream_t s);
int launch_ab_table(int lmax, int mmax, int stride, const int64_t* aboff, double2* ab, cudaStream_t s);
// items over the retained (m, ring) set, tiles of `tile` rings, split into the degree
// segments of `seg` when given, heaviest first
std::vector<RingItem> make_ring_items(const std::vector<int>& jlo, const std::vector<int>& jhi,
                                      int lmax, int mmax, int tile,
                                      const RingSegments* seg = nullptr);
int build_ring_items(const std::vector<int>& jlo, const std::vector<int>& jhi, int lmax, int mmax,
                     int rmax, RingItemsOwner& own, cudaStream_t s,
                     const RingSegments* seg = nullptr, int tile = 0);
// choose the degree segments for a ring set (seg_degrees > 0: target length; 0: none) and
// save the recurrence state at every segment start; t.ab/aboff must be built. Returns the
// segments unused (nseg all 1) when the state would exceed max_bytes.
int build_ring_segments(const RingTables& t, const std::vector<int>& jlo,
                        const std::vector<int>& jhi, int lmax, int mmax, int seg_degrees,
                        int64_t max_bytes, RingSegments& seg, cudaStream_t s);
// launchers: B transforms, alm complex (lmax+1, 2lmax+1, B); the adjoint writes all of alm
int ring_forward(const RingTables& t, const RingOut& o, const RingItems& it, const double2* alm,
                 double2* out, int B, cudaStream_t s);
// prepare = false: the caller has run ring_adjoint_prepare on alm (zeroing what the pass does
// not store), e.g. on another stream ahead of the pass
int ring_adjoint(const RingTables& t, const RingOut& o, const RingItems& it, const double2* in,
                 double2* alm, int B, cudaStream_t s, bool prepare = true);
int ring_adjoint_prepare(const RingTables& t, const RingItems& it, double2* alm, int B, cudaStream_t s);

// ---------------------------------------------------------------------------------------
// spin-weighted ring pass (spin.cu): G[j, m] = sum_l sa_{lm} N_l d^l_{m,-s}(theta_j) for
// m = -lmax..lmax and its transpose (src/Spin.jl:319-490); coefficients (l, m) at
// l + (lmax + 1)(m + lmax) (src/Layout.jl:28-29)
// ---------------------------------------------------------------------------------------
struct SpinTables {
    const double* cos_t = nullptr;    // nrings, reflection sign folded in
    const double* log2cos = nullptr;  // nrings: log2 cos(t/2) (log2 sin(t/2) when reflected)
    const double* log2sin = nullptr;  // nrings: log2 |sin(t/2)| (log2 cos(t/2) when reflected)
    const double* lb2 = nullptr;      // 2 lmax + 1: seed log2 binomial per order (-inf: none)
    const double* sg = nullptr;       // 2 lmax + 1: seed sign
    const int* pc = nullptr;          // 2 lmax + 1: seed power of cos(t/2)
    const int* ps = nullptr;          // 2 lmax + 1: seed power of sin(t/2)
    const double* w = nullptr;        // nrings window, or null for 1
    const double4* lt = nullptr;      // lmax + 1: (1/sqrt(l^2 - s^2), sqrt(l^2 - s^2), 1/l, N_l)
    int lmax = 0, spin = 0, nrings = 0;
};
struct SpinTablesOwner {
    DevBuf cos_t, log2cos, log2sin, lb2, sg, pc, ps, lt;
    SpinTables t;
};
// tables of a ring set (ring colatitudes theta_rings; reflect: the rings stand for pi - theta)
int build_spin_tables(const std::vector<double>& theta_rings, bool reflect, int lmax, int spin,
                      SpinTablesOwner& own, cudaStream_t s);
// items over (m = -lmax..lmax, tiles of rings_per_tile retained rings), heaviest first; jlo/jhi
// indexed by |m| (uploaded into own.jlo / own.jhi)
int build_spin_items(const std::vector<int>& jlo, const std::vector<int>& jhi, int lmax, int spin,
                     int rings_per_tile, RingItemsOwner& own, cudaStream_t s);
int spin_ring_forward(const SpinTables& t, const RingOut& o, const RingItems& it,
                      const double2* alm, double2* out, int B, cudaStream_t s);
// overwrites alm (entries below l = max(|m|, |s|) zero); clear = false: the caller has zeroed it
int spin_ring_adjoint(const SpinTables& t, const RingOut& o, const RingItems& it,
                      const double2* in, double2* alm, int B, cudaStream_t s, bool clear = true);
// the same with the coefficient array at ptrs[ptr] (a batch's device pointer table); the adjoint
// adds into that array, which the caller zeroes first
int spin_ring_forward_ptr(const SpinTables& t, const RingOut& o, const RingItems& it,
                          void* const* ptrs, int ptr, double2* out, int B, cudaStream_t s);
int spin_ring_adjoint_ptr(const SpinTables& t, const RingOut& o, const RingItems& it,
                          const double2* in, void* const* ptrs, int ptr, int B, cudaStream_t s);

// ---------------------------------------------------------------------------------------
// per-stage CUDA-event timing of applies (diagnostics; off unless a profile is active)
// ---------------------------------------------------------------------------------------
enum Stage {
    kStRingFwd, kStFftThetaFwd, kStPad, kStFft1Fwd, kStRowsFwd, kStFft2Fwd, kStInterp,
    kStSpread, kStFft2Adj, kStRowsAdj, kStFft1Adj, kStUnpad, kStFftThetaAdj, kStRingAdj,
    kStDirect, kNumStages
};
struct StageClock {
    bool on = false;
    int cap = 0, used = 0;
    cudaEvent_t prev = nullptr;
    std::vector<cudaEvent_t> ev;       // cap events, reused
    std::vector<int> stage;            // stage ending at ev[i] (-1: a start mark)
    void begin(cudaStream_t s);
    void mark(int st, cudaStream_t s);
};
inline void clock_begin(StageClock* c, cudaStream_t s) { if (c && c->on) c->begin(s); }
inline void clock_mark(StageClock* c, int st, cudaStream_t s) { if (c && c->on) c->mark(st, s); }

// ---------------------------------------------------------------------------------------
// NUFFT stages (nufft.cu)
// ---------------------------------------------------------------------------------------
struct NufftGrid {
    int w = 9;
    double beta = 0;
    int nf1 = 0, nf2 = 0;
    int row0 = 0, nrows = 0;   // fine-grid rows [row0, row0 + nrows) (mod nf1) are kept
    int row_wrap = 0;          // 1 when all nf1 rows are kept and taps wrap
    int n1 = 0;                // modes along dim 1 (FFT order)
    int ncols = 0;             // mode columns
    int bin_rows = 16, bin_cols = 16, nbr = 0, nbc = 0;
    int nbusy = 0;             // bins holding at least one point
    int igroup = 1;            // interpolation: consecutive bins of a bin row per block
    int nsbc = 0, nisb = 0;    // groups per bin row; non-empty groups
    int fp32 = 0;              // fine grids, FFTs, spreading and interpolation in FP32
    int64_t M = 0;
    // spreading in bin colours: bins (br, bc) of one colour (br mod rcol, bc mod ccol) have
    // disjoint tiles, so launching the colours one after the other (deterministic != 0) lets
    // every tile add its rows with plain loads and stores, in a fixed order (a deterministic
    // type-1 NUFFT); bins whose tiles wrap around the grid have colour classes of their own
    int deterministic = 0;
    int ncolors = 0;
    std::vector<int> color_off;  // ncolors + 1 offsets into NufftDev::sorder
    // the fine columns that hold no mode column: one run [gap_lo, gap_hi) (gap_ok), which the
    // TMA row transposes zero directly
    int gap_lo = 0, gap_hi = 0, gap_ok = 0;
    int plain_transpose = 0;   // 1: the plain-load transposes only
    int spread_reg = 1;        // spreading holds each bin's tile in registers where it fits
    int interp_pipe = 1;       // one-transform interpolation copies the next group's tile ahead
};

struct NufftDev {
    DevBuf pts;       // double2 (g1 - row0, g2) in bin order
    DevBuf perm;      // int32 original index, bin order
    DevBuf binstart;  // int32 nbins + 1
    DevBuf binorder;  // int32 nbusy: non-empty bins, most points first
    DevBuf iorder;    // int32 nisb: non-empty interpolation groups, most points first
    DevBuf sorder;    // int32 nbusy: non-empty bins by spreading colour, most points first in each
    DevBuf bslot;     // int4 nbusy: (bin, first point, end, 0) in binorder's order
    DevBuf sslot;     // int4 nbusy: the same in sorder's order
    DevBuf ipts;      // double2: pts in the interpolation's order (each group's points dealt over
    DevBuf iperm;     // int32    their shared-memory bank class), and their original indices
    DevBuf colp2;     // int32 ncols: fine column of each mode column
    DevBuf p2col;     // int32 nf2: mode column of each fine column or -1
    DevBuf mult1;     // double2 n1: per-mode complex factor along dim 1 (deconv incl.)
    DevBuf dec2;      // double ncols: deconvolution along dim 2
    DevBuf pad;       // double2 nf1 x ncols x B
    DevBuf U;         // double2 nrows x nf2 x B
    DevBuf counter;   // int: the next interpolation group to pull
    cufftHandle f1 = 0, f2 = 0;
    bool have_f1 = false, have_f2 = false;
    // 2-D tensor maps of pad (nf1 x ncols B) and U (nf2 x nrows B) for the TMA row transposes
    alignas(64) CUtensorMap pad_map;
    alignas(64) CUtensorMap U_map;
    bool have_maps = false;
    ~NufftDev();
};

// bounded device-side waits that gave up (the TMA row transposes), on the current device
int tma_timeouts(int* out);

// transform points (x = stretched colatitude, y = longitude; both radians) into grid
// coordinates, sort them into bins, fill pts/perm/binstart. x,y are device arrays.
int nufft_setpts(NufftGrid& g, NufftDev& d, const double* x, const double* y, cudaStream_t s);
// fine-grid FFT length for a dimension of minimum length nmin: the fastest batched library FFT
// (batch sequences, FP32 or FP64) among the 7-smooth lengths in [nmin, 1.1 nmin], timed on the
// device once per process for each (nmin, batch, type)
int fine_fft_length(int nmin, int64_t batch, bool fp32, cudaStream_t s, int* out);
// allocate pad/U and plan the fine-grid FFTs for B transforms
int nufft_alloc(NufftGrid& g, NufftDev& d, int B);
// type 2 from mode columns (n1 x ncols x B, FFT order along dim 1) to values f (M x B)
int nufft_type2(const NufftGrid& g, NufftDev& d, const double2* modes, double2* f, int B,
                int iflag, cudaStream_t s, StageClock* clk = nullptr);
// type 1 from values to mode columns
int nufft_type1(const NufftGrid& g, NufftDev& d, const double2* f, double2* modes, int B,
                int iflag, cudaStream_t s, StageClock* clk = nullptr);

// point transform of the leaf (src/Stretch.jl:202-213) on the device
int leaf_points(const Geom& g, bool flip, const double* theta, const double* phi, int64_t M,
                double* Theta, double* phi_out, cudaStream_t s);
int minmax_device(const double* x, int64_t M, double* mn, double* mx, cudaStream_t s);

// Direct leaf helpers (src/Direct.jl:60-117) on the device
int direct_phase_sum(const double2* G, const double* phi, int64_t M, int lmax, int B,
                     double2* f, cudaStream_t s);
int direct_phase_spread(const double2* f, const double* phi, int64_t M, int lmax, int B,
                        double2* G, cudaStream_t s);

// DFS (src/DFS.jl:13-56)
int dfs_double(const double2* F, double2* Ft, int Nth, int Nph, int B, int spin, cudaStream_t s);
int dfs_fold(double2* F, const double2* Ft, int Nth, int Nph, int B, int spin, cudaStream_t s);

// the planner's point scans on the device (planner_dev.cu); theta / phi are device arrays and
// the groups come back as device index lists, equal to the host planner's
struct DevPartition {
    std::vector<std::shared_ptr<DevBuf>> idx;
    std::vector<int64_t> n;
    std::vector<SphereBox> boxes;
    std::vector<double> costs;
};
int bounding_box_device(const double* theta, const double* phi, int64_t n, cudaStream_t s,
                        SphereBox* out);
int partition_boxes_device(const double* theta, const double* phi, int64_t n, int lmax, int ntrans,
                           double tol, int maxboxes, cudaStream_t s, DevPartition& out);
// *method: 1 stretch, 2 direct, 3 multi-box (select_method of src/Cost.jl:171-201)
int select_method_device(const double* theta, const double* phi, int64_t n, int lmax, int ntrans,
                         double tol, cudaStream_t s, int* method, DevPartition* part);

// launch-error check after a kernel (also counts the launch)
int check_launch(const char* what);
long long launch_count();

}  // namespace pf
