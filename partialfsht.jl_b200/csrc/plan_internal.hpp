// The plan object behind the C ABI's opaque pfsht_plan, shared by plan.cu (construction and
// single-plan applies) and batch.cu (many plans in one captured graph).
#pragma once
#include <cufft.h>

#include <future>
#include <memory>
#include <vector>

#include "../../include/pfsht_b200.h"
#include "internal.cuh"

using namespace pf;

struct pfsht_plan {
    int device = 0;
    int precision = 0;
    int kind = kPole;
    int L = 0, B = 1;
    int64_t M = 0;
    double tol = 0;
    int R = 0;  // ring tile rings-per-lane override (0 = defaults)
    int deterministic = 0;  // fixed-order adjoint sums (pfsht_opts.deterministic)
    pf::Leaf leaf;
    int ncols = 0;
    int nrings = 0;
    // ring pass
    DevBuf cos_t, log2sin, log2c, w, ab, aboff;
    RingItemsOwner fwd_items, adj_items;
    RingSegments adj_seg;  // degree segments of the adjoint items
    int seg_degrees = 0;   // requested segment length (0 = auto, < 0 = none)
    RingTables rt;
    // the forward ring pass's tables: rt itself, except in the mixed form, whose forward runs the
    // FP64 pass (FP32 accumulation saves nothing there: each ring value's conversion costs as
    // much as the FP64 multiply-adds) on its own (beta, g) table of 64-degree blocks
    RingTables rt_fwd;
    DevBuf ab_fwd;
    // spin weight s (src/Spin.jl): s != 0 runs the Wigner-d ring pass on spt with the items in
    // fwd_items for both directions; coefficients in the (l, m + lmax) layout
    int spin = 0;
    SpinTablesOwner spt;
    RingOut ro_cols;  // the apply's column array H (or G for the direct leaf)
    // column array: nth x ncols x B (stretch) or M x (2L+1) x B (direct)
    DevBuf H;
    cufftHandle fth = 0;
    bool have_fth = false;
    // NUFFT
    NufftGrid ng;
    NufftDev nd;
    // direct leaf
    DevBuf phi_pts;
    // host-buffer staging: st_alm / st_f serve the forward (coefficients in, field out),
    // st_alm2 / st_f2 the adjoint (field in, coefficients out), so that a forward's output copy
    // and an adjoint's input copy (or the next call's) can be in flight while the other computes
    DevBuf st_alm, st_f, st_alm2, st_f2;
    cudaStream_t st_stream = nullptr;
    // host copies run on their own streams, one per direction of the link, ordered against the
    // compute stream by events; blk_* hold the ring items grouped by the order blocks in which
    // the coefficients cross (items of block k at [off[k], off[k + 1]), heaviest first in each),
    // so the ring pass of one block runs while the next block is copied
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_alm_in_free = nullptr, ev_f_out_free = nullptr, ev_f_in_free = nullptr,
                ev_alm_out_free = nullptr, ev_fwd_done = nullptr, ev_f_in_ready = nullptr,
                ev_copied = nullptr;
    std::vector<cudaEvent_t> ev_blk;
    DevBuf blk_fwd_items, blk_adj_items;
    std::vector<int> blk_fwd_off, blk_adj_off;
    bool host_pipeline = false;  // the blocked host path is set up
    // the adjoint zeroes its output on `side` while the NUFFT and Theta-FFT stages run
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // MultiBox (src/MultiBox.jl): one stretched-leaf plan per box; gidx holds the boxes' point
    // indices one box after the other (box i at [box_off[i], box_off[i + 1])), fg the boxes'
    // fields in the same order (box i at B box_off[i]), acc one coefficient array for the sum
    std::vector<std::unique_ptr<pfsht_plan>> boxes;
    std::vector<int64_t> box_off;
    DevBuf gidx, fg, acc;
    pfsht_plan_info info{};
    StageClock clk;
    // an asynchronous host adjoint's zeroing of its output's padding rows, on a host thread
    std::future<void> host_zero;
    ~pfsht_plan() {
        if (host_zero.valid()) host_zero.wait();
        if (have_fth) cufftDestroy(fth);
        if (st_stream) cudaStreamDestroy(st_stream);
        if (side) cudaStreamDestroy(side);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
        for (cudaEvent_t e : {ev_alm_in_free, ev_f_out_free, ev_f_in_free, ev_alm_out_free,
                              ev_fwd_done, ev_f_in_ready, ev_copied})
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ev_blk) cudaEventDestroy(e);
        for (cudaEvent_t e : clk.ev) cudaEventDestroy(e);
    }
};

namespace pf {

// selects a device for the lifetime of a call and restores the caller's
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (dev >= 0 && dev != prev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// The pieces of one apply around its ring pass: the forward after the ring pass (FFT along
// Theta and NUFFT type 2, or the Direct leaf's phase sum) and the adjoint before it.
int plan_forward_after_ring(pfsht_plan* p, double2* f, cudaStream_t s);
int plan_adjoint_before_ring(pfsht_plan* p, const double2* f, cudaStream_t s);

// The host-buffer apply without its final synchronisation: copies in (the coefficient
// staircase or the field), applies on the plan's staging buffers and copies out. The compute
// runs on `s`, the copies on the plan's h2d / d2h streams; with order_on_s the end of the output
// copy is ordered before whatever is enqueued on `s` afterwards, otherwise only the plan's d2h
// stream (pfsht_host_sync) marks it. For the adjoint it also zeroes the host array's padding rows
// on host threads: before it returns, or with zero_async on a host thread of its own that
// plan_host_wait joins. The host arrays must stay valid until the copies end.
int plan_host_enqueue(pfsht_plan* p, const void* in, void* out, bool fwd, cudaStream_t s,
                      bool order_on_s = true, bool zero_async = false);
// wait for the plan's asynchronous padding zeroing, if one is running
void plan_host_wait(pfsht_plan* p);
// allocate the plan's staging buffers for host-buffer applies
int plan_host_staging(pfsht_plan* p);

}  // namespace pf
