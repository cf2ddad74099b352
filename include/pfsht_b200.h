/*
 * pfsht_b200.h -- C ABI of libpfsht_b200, a B200 (sm_100a) backend for PartialFSHT.jl's
 * partial-sky spherical harmonic synthesis and its exact adjoint.
 *
 * The entry points are what a PartialFSHT.jl device extension would ccall in place of the
 * reference's Julia leaf. Plain pointers and sizes only.
 *
 * Layouts are the reference's, column-major:
 *   alm : (lmax+1) x (2lmax+1) x ntrans complex double, FastSphericalHarmonics sph_mode
 *         packing (src/Layout.jl:13-20): 0-based column 2m for m >= 0, 2|m|-1 for m < 0,
 *         row l-|m|. Padding slots are ignored on input and written as zero by the adjoint.
 *   f   : npts x ntrans complex double, points in the caller's order.
 *   G   : nrings x (2lmax+1) x ntrans complex double, column m+lmax (src/Legendre.jl:306).
 * Complex numbers are interleaved (re, im) pairs of doubles.
 *
 * Every function returns a pfsht_status; a non-zero status leaves a message readable with
 * pfsht_last_error (thread-local). Validation happens before any launch.
 */
#ifndef PFSHT_B200_H
#define PFSHT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PFSHT_OK = 0,
    PFSHT_ERR_ARGUMENT = 1,       /* Julia ArgumentError (src/Plan.jl:98-102) */
    PFSHT_ERR_DIMENSION = 2,      /* Julia DimensionMismatch (src/Layout.jl:35-56) */
    PFSHT_ERR_REFUSED = 3,        /* degenerate stretch geometry (src/Windows.jl:66-75) */
    PFSHT_ERR_CUDA = 4,           /* a CUDA or cuFFT call failed */
    PFSHT_ERR_OUT_OF_MEMORY = 5,  /* device allocation failed, or a budget was exceeded */
    PFSHT_ERR_TIMEOUT = 6,        /* a bounded device-side wait gave up */
    PFSHT_ERR_UNSUPPORTED = 7     /* option not built into this library */
} pfsht_status;

/* AbstractAlgorithm (src/Cost.jl:15-30): AUTO is the cost model's choice (select_method,
 * src/Cost.jl:171-201) among the stretched leaf, Direct and MultiBox. */
typedef enum {
    PFSHT_METHOD_AUTO = 0,
    PFSHT_METHOD_STRETCH = 1,
    PFSHT_METHOD_DIRECT = 2,
    PFSHT_METHOD_MULTIBOX = 3   /* one stretched leaf per box of a partition (src/MultiBox.jl) */
} pfsht_method;

typedef enum {
    PFSHT_PRECISION_FP64 = 0,   /* plain form: FP64 everywhere */
    PFSHT_PRECISION_MIXED = 1   /* FP64 recurrence + exponents; FP32 compensated ring sums and FP32 NUFFT.
                                   Applies when tol >= 1e-6; a plan asked for it at a smaller tol runs
                                   the FP64 form (pfsht_plan_info.precision says which). */
} pfsht_precision;

typedef enum {
    PFSHT_KIND_POLE = 0, PFSHT_KIND_INTERIOR = 1, PFSHT_KIND_FULL = 2, PFSHT_KIND_DIRECT = 3,
    PFSHT_KIND_MULTIBOX = 4
} pfsht_kind;

/* Plan options: the keyword arguments of Plan(...) (src/Plan.jl:84-97) that change the
 * apply, plus the device knobs. Fill with pfsht_opts_default first. */
typedef struct pfsht_opts {
    int32_t method;             /* pfsht_method */
    int32_t points_on_device;   /* theta/phi are device pointers */
    int32_t device;             /* CUDA device ordinal; -1 = current */
    int32_t ring_rings_per_lane;/* ring-pass tile shape: rings per lane (1, 2 or 4; 0 = auto) */
    int32_t nufft_bin_rows;     /* NUFFT spreading bin height in fine cells (0 = auto) */
    int32_t nufft_bin_cols;     /* NUFFT spreading bin width in fine cells (0 = auto) */
    double oversample_theta;    /* src/Plan.jl:95 */
    double oversample_phi;      /* src/Plan.jl:96 */
    double eps_apo_max;         /* src/Plan.jl:97 */
    int32_t ring_segment_degrees; /* adjoint ring pass: split each order into degree segments of
                                     about this length, started from recurrence states saved at
                                     plan time (0 = auto, < 0 = never split) */
    int32_t nufft_fft_lengths;  /* NUFFT fine-grid FFT lengths: 0 = the fastest library FFT among
                                   the 7-smooth lengths within 10% above the minimum (timed at
                                   plan time, once per process and shape); 1 = the minimum
                                   2,3,5-smooth lengths >= 2n (deterministic, as FINUFFT);
                                   2 = nufft_nf1 x nufft_nf2 as given (each >= its minimum) */
    int32_t nufft_nf1, nufft_nf2;
    int32_t maxboxes;           /* MultiBox: at most this many boxes (src/Plan.jl:93; 0 = 8) */
    int32_t spin;               /* spin weight s, |s| <= lmax (src/Plan.jl:87,101-102): s != 0
                                   transforms spin-s fields with coefficients sa_lm at
                                   l + (lmax+1)(m+lmax) (src/Layout.jl:28-29), the ring pass in
                                   FP64 whatever the precision mode */
    int32_t nufft_transpose;    /* NUFFT fine-row transposes: 0 = TMA-staged tiles where the grid
                                   layout allows (plain loads for the rest), 1 = plain loads only */
    int32_t deterministic;      /* 1: adjoints that are bitwise reproducible run to run (each order's
                                   ring sums added in a fixed order by one warp, spreading bins
                                   launched in colours whose tiles are disjoint); 0 (default): the
                                   faster adjoint, whose atomic additions vary at round-off */
    int32_t nufft_spread;       /* NUFFT spreading: 0 = each bin's whole tile held in registers
                                   where the tile fits (16 columns, 32 rows), 1 = a sliding window
                                   of the kernel's rows (same values, in the same order) */
} pfsht_opts;

typedef struct pfsht_plan pfsht_plan;

/* Geometry and sizes of a plan (the fields of StretchLeaf, src/Stretch.jl:94-127). */
typedef struct pfsht_plan_info {
    int32_t kind;        /* pfsht_kind */
    int32_t flip;        /* south periodisation reflected to the north */
    int32_t lmax, ntrans, precision;
    int32_t nth_half, nth, nph, mmax, nrings;
    int64_t npts, K, ring_work;
    double tol, beta, h, theta_lo, theta_hi, eps_apo, Theta1, sigma, ThetaT;
    /* NUFFT */
    int32_t nufft_w, nf1, nf2, row0, nrows, ncols;
    double nufft_beta;
    int64_t device_bytes; /* device memory the plan holds */
    int32_t spin;         /* spin weight */
    int32_t pad_;
} pfsht_plan_info;

/* Fill defaults (method AUTO, host points, current device, oversampling 1, eps_apo_max 1). */
pfsht_status pfsht_opts_default(pfsht_opts* opts);

/* Plan(theta, phi; lmax, tol, ntrans) (src/Plan.jl:84-116). Geometry on the host; the
 * point transform, the NUFFT bin sort and the recurrence tables on the device. */
pfsht_status pfsht_plan_create(const double* theta, const double* phi, int64_t npts,
                               int32_t lmax, int32_t ntrans, double tol, int32_t precision,
                               const pfsht_opts* opts, pfsht_plan** out);
pfsht_status pfsht_plan_destroy(pfsht_plan* plan);

/* mul!(f, plan, alm) (src/Plan.jl:137-141): device pointers, enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream). */
pfsht_status pfsht_forward(pfsht_plan* plan, const void* alm, void* f, void* stream);
/* mul!(alm, plan', f) (src/Plan.jl:143-148): overwrites alm, padding zeroed. */
pfsht_status pfsht_adjoint(pfsht_plan* plan, const void* f, void* alm, void* stream);

/* The same two applies on host buffers: copies in, apply, copies out, synchronous.
 * The plan keeps staging buffers for this (src/Stretch.jl:393-410 role), one set per direction.
 * The coefficients cross in blocks of orders, and the ring pass of a block runs while the next
 * block is copied (in for the forward, out for the adjoint). */
pfsht_status pfsht_forward_host(pfsht_plan* plan, const void* alm, void* f);
pfsht_status pfsht_adjoint_host(pfsht_plan* plan, const void* f, void* alm);

/* The host-buffer applies without waiting for them (no reference counterpart; mul! on host
 * arrays returns with the result, these let a caller with independent inputs keep the link busy):
 * the compute is enqueued on `stream` (NULL = the plan's own stream) and the copies on the plan's
 * two copy streams, one per direction, so a forward's field copy out can run beside an adjoint's
 * field copy in and compute. The outputs are complete, and the inputs free for reuse, once
 * pfsht_host_sync returns. Host buffers must be page-locked (cudaHostAlloc / cudaHostRegister) for
 * the copies to overlap. One plan's host applies run in the order issued. */
pfsht_status pfsht_forward_host_async(pfsht_plan* plan, const void* alm, void* f, void* stream);
pfsht_status pfsht_adjoint_host_async(pfsht_plan* plan, const void* f, void* alm, void* stream);
/* Waits for every host-buffer apply of the plan issued so far, including an asynchronous
 * adjoint's zeroing of the padding and unretained orders of its host output, which runs on a
 * host thread of its own. */
pfsht_status pfsht_host_sync(pfsht_plan* plan);

/* Bytes the two host-buffer applies move across PCIe per call (no reference counterpart):
 * the coefficient array travels as the sph_mode staircase of the orders the plan retains
 * (rows 0..lmax-m of each order m <= mmax, in blocks of orders; for a spin plan the columns of
 * those orders), since the forward reads no other coefficient and the adjoint's others are zero,
 * which the library writes into the host array itself; the field travels whole. */
pfsht_status pfsht_host_bytes(const pfsht_plan* plan, int64_t* h2d_forward, int64_t* d2h_forward,
                              int64_t* h2d_adjoint, int64_t* d2h_adjoint);

/* rings_from_alm! / alm_from_rings! (src/Legendre.jl:310-341) on the plan's ring set:
 * G is nrings x (2lmax+1) x ntrans on the device. For parity tests of the ring pass. */
pfsht_status pfsht_ring_forward(pfsht_plan* plan, const void* alm, void* G, void* stream);
pfsht_status pfsht_ring_adjoint(pfsht_plan* plan, const void* G, void* alm, void* stream);

/* Queries: ring_work (src/Plan.jl:44), sizes (src/Stretch.jl:94-127). */
int64_t pfsht_ring_work(const pfsht_plan* plan);
pfsht_status pfsht_plan_get_info(const pfsht_plan* plan, pfsht_plan_info* info);
int64_t pfsht_workspace_bytes(const pfsht_plan* plan);

/* ---- planner (src/Box.jl, src/Cost.jl), host only ---------------------------------------- */

/* SphereBox (src/Box.jl:23-30): colatitude extent and the longitude arc from phi_start. */
typedef struct pfsht_box {
    double theta_lo, theta_hi, phi_start, phi_extent;
    int32_t touches_north, touches_south;
} pfsht_box;

/* bounding_box (src/Box.jl:42-73): exact colatitude extent, longitude arc = complement of the
 * largest circular gap (O(n), no sort). */
pfsht_status pfsht_bounding_box(const double* theta, const double* phi, int64_t npts, pfsht_box* box);
/* cost_direct / cost_stretch (src/Cost.jl:107-142) in the cost constants' units; cost_stretch is
 * +inf where the stretched construction refuses the geometry. */
double pfsht_cost_direct(int64_t npts, int32_t lmax, int32_t ntrans);
double pfsht_cost_stretch(const pfsht_box* box, int64_t npts, int32_t lmax, int32_t ntrans, double tol);
/* partition_boxes_costed (src/Box.jl:156-200) with cost_stretch: group_of_point[i] = box of point
 * i (0-based, in the order boxes are reported); boxes / costs hold maxboxes entries. */
pfsht_status pfsht_partition_boxes(const double* theta, const double* phi, int64_t npts,
                                   int32_t lmax, int32_t ntrans, double tol, int32_t maxboxes,
                                   int32_t* group_of_point, int32_t* nboxes, pfsht_box* boxes,
                                   double* costs);
/* select_method (src/Cost.jl:171-201) for AUTO: *method = STRETCH, DIRECT or MULTIBOX. */
pfsht_status pfsht_select_method(const double* theta, const double* phi, int64_t npts,
                                 int32_t lmax, int32_t ntrans, double tol, int32_t* method);
/* The same three on device arrays of points (the O(n) scans run on the device, the cost model and
 * the search loop on the host; results equal the host versions'). Plans of 2^15 points or more
 * are planned this way. */
pfsht_status pfsht_bounding_box_device(const double* theta, const double* phi, int64_t npts,
                                       pfsht_box* box, void* stream);
pfsht_status pfsht_partition_boxes_device(const double* theta, const double* phi, int64_t npts,
                                          int32_t lmax, int32_t ntrans, double tol, int32_t maxboxes,
                                          int32_t* group_of_point, int32_t* nboxes, pfsht_box* boxes,
                                          double* costs, void* stream);
pfsht_status pfsht_select_method_device(const double* theta, const double* phi, int64_t npts,
                                        int32_t lmax, int32_t ntrans, double tol, int32_t* method,
                                        void* stream);
/* set_cost_constants! / cost_calibrated (src/Cost.jl:60-74): process-wide per-unit costs. */
pfsht_status pfsht_set_cost_constants(double ring, double fft, double spread, double ft_conn);
pfsht_status pfsht_get_cost_constants(double* ring, double* fft, double* spread, double* ft_conn,
                                      int32_t* calibrated);

/* Boxes of a MultiBox plan (1 for a single-leaf plan, whose box is the plan itself): the box's
 * stretched leaf geometry and, if indices is not NULL, its points (ascending 0-based indices
 * into the plan's point set; info.npts of them). */
int32_t pfsht_plan_num_boxes(const pfsht_plan* plan);
pfsht_status pfsht_plan_box(const pfsht_plan* plan, int32_t box, pfsht_plan_info* info,
                            int64_t* indices);

/* ---- analysis: solve! (src/Analysis.jl:375-436) -------------------------------------------- */

typedef enum {
    PFSHT_SOLVE_CG = 0,      /* :cg -- stopped at rtol (the stopping rule is the regularisation) */
    PFSHT_SOLVE_WIENER = 1,  /* :wiener -- Tikhonov with the prior C_l (required) */
    PFSHT_SOLVE_MINNORM = 2  /* :minnorm -- rtol tightened to min(rtol, 1e-12) */
} pfsht_solve_mode;

/* Conjugate gradients on (A^H W A + C^-1) alm = A^H W f on the device: f and alm are device
 * arrays in the plan's layouts (alm is overwritten with the solution); prior is a host array of
 * lmax + 1 values C_l (WIENER only, NULL otherwise); w is a device array of npts point weights or
 * NULL. Each iteration is one CUDA graph with device-side scalars; the updates freeze where the
 * reference's loop breaks. *iters and *relres are the reference's info.iters and info.relres. */
pfsht_status pfsht_solve(pfsht_plan* plan, const void* f, void* alm, int32_t mode, double rtol,
                         int32_t maxiter, const double* prior, const double* w, void* stream,
                         int32_t* iters, double* relres);

/* Host-only plan geometry, no device touched: what pfsht_plan_create would choose for
 * these points (kind, sizes, ring_work). Points are host pointers. nf1/nf2 are the minimum
 * fine-grid lengths; a plan built with timed lengths may use longer ones (pfsht_plan_get_info). */
pfsht_status pfsht_plan_geometry(const double* theta, const double* phi, int64_t npts,
                                 int32_t lmax, int32_t ntrans, double tol,
                                 const pfsht_opts* opts, pfsht_plan_info* info);

/* dfs_double! / dfs_fold! (src/DFS.jl:13-56) on device arrays, column-major
 * F: Nth x Nph x B, Ft: 2Nth x Nph x B. */
pfsht_status pfsht_dfs_double(const void* F, void* Ft, int32_t Nth, int32_t Nph, int32_t B,
                              int32_t spin, void* stream);
pfsht_status pfsht_dfs_fold(void* F, const void* Ft, int32_t Nth, int32_t Nph, int32_t B,
                            int32_t spin, void* stream);

/* The NUFFT seam (src/NUFFT.jl:17-25, _nufft_makeplan/_nufft_exec!): a 2-D type-1/type-2
 * NUFFT with modes n1 x n2 in FFT order (modeord = 1), points x, y (host pointers, any
 * real values; taken modulo 2 pi). type 2: modes -> M values; type 1: M values -> modes. */
typedef struct pfsht_nufft pfsht_nufft;
pfsht_status pfsht_nufft_create(int32_t type, int32_t n1, int32_t n2, int32_t iflag,
                                int32_t ntrans, double tol, const double* x, const double* y,
                                int64_t M, pfsht_nufft** out);
pfsht_status pfsht_nufft_exec(pfsht_nufft* p, const void* in, void* out, void* stream);
pfsht_status pfsht_nufft_destroy(pfsht_nufft* p);

/* Many plans applied together (the farmed mul! over independent plans,
 * ext/PartialFSHTOhMyThreadsExt.jl:151-159, on one GPU). A batch holds borrowed plans of one
 * device, which must outlive it and must not be applied elsewhere while a batch apply runs.
 * Each direction is one CUDA graph, captured at its first call and replayed by one
 * cudaGraphLaunch: the ring passes of all plans run as one launch per kernel shape (at most a
 * few), the remaining stages of the plans concurrently on nstreams internal streams (0 = 8).
 * alms[i] and fs[i] are plan i's device arrays, in the layouts of pfsht_forward / pfsht_adjoint;
 * they may change from call to call. A call returns once the graph is enqueued on `stream`;
 * it first waits for the batch's previous call to finish on the device. */
typedef struct pfsht_batch pfsht_batch;
pfsht_status pfsht_batch_create(pfsht_plan* const* plans, int32_t nplans, int32_t nstreams,
                                pfsht_batch** out);
pfsht_status pfsht_batch_forward(pfsht_batch* batch, const void* const* alms, void* const* fs,
                                 void* stream);
pfsht_status pfsht_batch_adjoint(pfsht_batch* batch, const void* const* fs, void* const* alms,
                                 void* stream);
/* ring-pass launches per direction and nodes of the captured graphs (0 before the first call) */
pfsht_status pfsht_batch_info(const pfsht_batch* batch, int32_t* ring_launches_fwd,
                              int32_t* ring_launches_adj, int64_t* graph_nodes_fwd,
                              int64_t* graph_nodes_adj);
pfsht_status pfsht_batch_destroy(pfsht_batch* batch);

/* Serving loop (no reference counterpart): plans resident on one device and a worker thread
 * that runs synthesis (forward = 1) and adjoint requests on HOST arrays as they arrive. Plans are
 * registered against hbm_budget_bytes (each counts its device memory plus its staging buffers;
 * a registration past the budget returns PFSHT_ERR_OUT_OF_MEMORY). A request starts as soon as
 * one of nslots streams is free and its plan is idle: requests for different plans overlap on
 * the device, requests for one plan run in arrival order. submit returns at once with an id;
 * wait blocks until that request is done (timeout_s < 0: no limit; PFSHT_ERR_TIMEOUT when it
 * runs out) and gives its latency from submission. Host arrays must stay valid until their
 * request is done; pinned arrays let copies of one request overlap another's kernels.
 * Registered plans must outlive the server and must not be applied elsewhere meanwhile.
 * Times are seconds since the server was created; release forgets a finished request. */
typedef struct pfsht_server pfsht_server;
pfsht_status pfsht_server_create(int32_t device, int64_t hbm_budget_bytes, int32_t nslots,
                                 pfsht_server** out);
pfsht_status pfsht_server_add_plan(pfsht_server* server, pfsht_plan* plan, int32_t* plan_id);
pfsht_status pfsht_server_submit(pfsht_server* server, int32_t plan_id, int32_t forward,
                                 const void* in, void* out, int64_t* request_id);
pfsht_status pfsht_server_wait(pfsht_server* server, int64_t request_id, double timeout_s,
                               double* latency_s);
pfsht_status pfsht_server_request_times(pfsht_server* server, int64_t request_id,
                                        double* t_submit, double* t_start, double* t_done);
pfsht_status pfsht_server_release(pfsht_server* server, int64_t request_id);
pfsht_status pfsht_server_stats(pfsht_server* server, int64_t* completed, int64_t* queued,
                                int64_t* running, int64_t* bytes_resident);
pfsht_status pfsht_server_destroy(pfsht_server* server);

/* FMA-throughput microbenchmark on the current device (no reference counterpart): runs a
 * grid of independent FP64 (fp64 = 1) or FP32 FMA chains and reports FLOP/s (2 per FMA).
 * These are the denominators of the ring-pass and NUFFT FLOP rooflines. */
pfsht_status pfsht_fma_peak(int32_t fp64, int32_t iters, double* flops_per_s, double* ms);

/* Number of this library's own kernel launches since load (diagnostics; cuFFT and CUB
 * kernels are not counted). */
int64_t pfsht_launch_count(void);

/* Per-stage CUDA-event timing of a plan's applies (no reference counterpart; the reference's
 * benchmark/calibrate.jl:68-79 times stages on the host). Between start and stop every apply
 * records an event at each stage boundary on its stream; stop sums the durations per stage
 * (stage_ms and stage_count sized pfsht_num_stages()). max_marks bounds the events kept. */
pfsht_status pfsht_profile_start(pfsht_plan* plan, int32_t max_marks);
pfsht_status pfsht_profile_stop(pfsht_plan* plan, double* stage_ms, int32_t* stage_count);
int32_t pfsht_num_stages(void);
const char* pfsht_stage_name(int32_t stage);

/* Direct synthesis without any allocation (no counterpart in the reference): for callers
 * that cannot allocate device memory at the call (a framework owning the device's memory
 * through its own pool, memory reserved in advance, or calls too small to pay for a plan).
 * Computes f_i = sum_lm a_lm Y_lm(theta_i, phi_i) exactly, as a Direct plan's synthesis does,
 * for device arrays theta, phi (npts), alm ((lmax+1) x (2lmax+1)) and f (npts), with all
 * intermediates in one fixed 32 MiB array the library declares in device memory; it makes no
 * cudaMalloc, cudaFree or other allocating call. Sizes needing more (about
 * npts (2 lmax + 1) 16 bytes), and lmax above 2048, are rejected with PFSHT_ERR_ARGUMENT.
 * The first call on a device looks up the array's address and should come before any stream
 * capture; the address is kept per device for the device's primary context (the CUDA
 * runtime's), so the call is not for other driver-API contexts or after cudaDeviceReset.
 * Calls share the array: calls that overlap on the GPU race and must be serialised by the
 * caller. */
pfsht_status pfsht_direct_forward_noalloc(const double* theta, const double* phi, int64_t npts,
                                          int32_t lmax, const void* alm, void* f, void* stream);

/* Number of bounded device-side waits (the TMA tile loads of the NUFFT row transposes) that gave
 * up on the current device since the library was loaded (no reference counterpart). A kernel
 * whose wait runs out records it here, skips that tile and returns; 0 means every wait ended. */
pfsht_status pfsht_wait_timeouts(int32_t* count);

/* Thread-local message of the last failing call; returns its length. */
size_t pfsht_last_error(char* buf, size_t len);
/* Library version string. */
const char* pfsht_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PFSHT_B200_H */
