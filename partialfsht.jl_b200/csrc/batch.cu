// Many plans applied together (pfsht_batch_*): the role of the reference's farmed mul! over
// independent plans (ext/PartialFSHTOhMyThreadsExt.jl:151-159), done on one GPU.
//
// One direction of a batch is one CUDA graph, captured on first use and replayed with a single
// cudaGraphLaunch:
//   forward : pointer table -> ring passes of all scalar plans (one persistent launch: warps
//             pull the items of every plan and tile shape, heaviest first, from a counter) ->
//             per plan, on one of several streams: the
//             spin ring pass of a spin plan, FFT along Theta and NUFFT type 2 into the plan's
//             own field buffer -> one copy kernel into the callers' fields
//   adjoint : pointer table -> one copy kernel from the callers' fields -> per plan on the
//             streams: NUFFT type 1, inverse FFT along Theta, zeroing of the caller's
//             coefficient array (and a spin plan's own ring pass) -> ring passes of all scalar
//             plans (one persistent launch; tiles of eight rings per lane, if a plan asks for
//             them, run in launches of their own after it)
// Callers' arrays are reached through a device pointer table that the graph's first node
// copies from pinned host memory, so new arrays on each call need no new capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "plan_internal.hpp"

namespace pf {

// a contiguous piece of one plan's field (M x B values) for the copy kernel
struct FChunk {
    int plan;
    int64_t off, n;
};
static constexpr int64_t kFChunk = 1 << 16;

// to_user: plans' buffers -> callers' fields (ptrs[nplans + p]); else the reverse
__global__ void field_copy_kernel(const FChunk* __restrict__ chunks, double2* const* __restrict__ stf,
                                  void* const* __restrict__ ptrs, int nplans, int to_user) {
    const FChunk c = chunks[blockIdx.x];
    double2* own = stf[c.plan] + c.off;
    double2* user = static_cast<double2*>(ptrs[nplans + c.plan]) + c.off;
    for (int64_t i = threadIdx.x; i < c.n; i += blockDim.x) {
        if (to_user) user[i] = own[i];
        else own[i] = user[i];
    }
}

}  // namespace pf

struct pfsht_batch {
    int device = 0;
    int n = 0;
    std::vector<pfsht_plan*> plans;
    pf::RingMerged mf, ma;                                    // all ring items per direction
    std::vector<std::unique_ptr<pf::RingBatchGroup>> gf, ga;  // shapes outside the merged launch
    pf::DevBuf slots;    // RingSlot[n]
    pf::DevBuf ptrs;     // void*[2n]: coefficient arrays, then fields
    void** ptrs_host = nullptr;  // pinned source of the table
    pf::DevBuf stf;      // double2*[n]: each plan's field buffer
    pf::DevBuf chunks;   // FChunk[nchunks]
    int nchunks = 0;
    cudaStream_t main = nullptr;
    std::vector<cudaStream_t> side;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // [0] adjoint, [1] forward
    int64_t nodes[2] = {0, 0};
    bool launched = false;
    ~pfsht_batch() {
        for (cudaGraphExec_t e : exec)
            if (e) cudaGraphExecDestroy(e);
        for (cudaStream_t s : side) cudaStreamDestroy(s);
        for (cudaEvent_t e : join) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (done) cudaEventDestroy(done);
        if (main) cudaStreamDestroy(main);
        if (ptrs_host) cudaFreeHost(ptrs_host);
    }
};

namespace {

using namespace pf;

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

// everything of one direction, recorded on b->main (inside a capture)
int record(pfsht_batch* b, bool fwd) {
    cudaStream_t m = b->main;
    const int n = b->n;
    void* const* ptrs = b->ptrs.as<void*>();
    const RingSlot* slots = b->slots.as<RingSlot>();
    double2* const* stf = b->stf.as<double2*>();
    PF_CUDA(cudaMemcpyAsync(b->ptrs.p, b->ptrs_host, sizeof(void*) * 2 * n,
                            cudaMemcpyHostToDevice, m));
    if (fwd) {
        PF_TRY(ring_merged_launch(slots, b->mf, false, ptrs, m));
        PF_TRY(ring_forward_batch(slots, b->gf, ptrs, m));
    }
    else {
        field_copy_kernel<<<b->nchunks, 256, 0, m>>>(b->chunks.as<FChunk>(), stf, ptrs, n, 0);
        PF_TRY(check_launch("field_copy_kernel"));
    }
    PF_CUDA(cudaEventRecord(b->fork, m));
    for (size_t k = 0; k < b->side.size(); ++k) PF_CUDA(cudaStreamWaitEvent(b->side[k], b->fork, 0));
    for (int i = 0; i < n; ++i) {
        pfsht_plan* p = b->plans[i];
        cudaStream_t s = b->side[i % b->side.size()];
        if (fwd) {
            if (p->spin)
                PF_TRY(spin_ring_forward_ptr(p->spt.t, p->ro_cols, p->fwd_items.view, ptrs, i,
                                             p->H.as<double2>(), p->B, s));
            PF_TRY(plan_forward_after_ring(p, p->st_f.as<double2>(), s));
        } else if (p->spin) {
            PF_TRY(plan_adjoint_before_ring(p, p->st_f.as<double2>(), s));
            PF_TRY(alm_prepare_ptr(ptrs, i, p->L, p->B, nullptr, 0, s));
            PF_TRY(spin_ring_adjoint_ptr(p->spt.t, p->ro_cols, p->fwd_items.view, p->H.as<double2>(),
                                         ptrs, i, p->B, s));
        } else {
            PF_TRY(plan_adjoint_before_ring(p, p->st_f.as<double2>(), s));
            const int allow_sole = p->adj_items.view.rmax >= 2 ? 1 : 0;
            PF_TRY(alm_prepare_ptr(ptrs, i, p->L, p->B, p->adj_items.view.sole_m, allow_sole, s));
        }
    }
    for (size_t k = 0; k < b->side.size(); ++k) {
        PF_CUDA(cudaEventRecord(b->join[k], b->side[k]));
        PF_CUDA(cudaStreamWaitEvent(m, b->join[k], 0));
    }
    if (fwd) {
        field_copy_kernel<<<b->nchunks, 256, 0, m>>>(b->chunks.as<FChunk>(), stf, ptrs, n, 1);
        PF_TRY(check_launch("field_copy_kernel"));
    } else {
        PF_TRY(ring_merged_launch(slots, b->ma, true, ptrs, m));
        PF_TRY(ring_adjoint_batch(slots, b->ga, ptrs, m));
    }
    return 0;
}

int capture(pfsht_batch* b, bool fwd) {
    PF_CUDA(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    const int rc = record(b, fwd);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->main, &graph);
    if (rc) {
        if (e == cudaSuccess && graph) cudaGraphDestroy(graph);
        return rc;
    }
    PF_CUDA(e);
    size_t nn = 0;
    cudaGraphGetNodes(graph, nullptr, &nn);
    b->nodes[fwd] = (int64_t)nn;
    const cudaError_t ei = cudaGraphInstantiate(&b->exec[fwd], graph, 0);
    cudaGraphDestroy(graph);
    PF_CUDA(ei);
    return 0;
}

int batch_apply(pfsht_batch* b, bool fwd, const void* const* in, void* const* out,
                cudaStream_t stream) {
    DeviceGuard dg(b->device);
    if (!b->exec[fwd]) PF_TRY(capture(b, fwd));
    // the previous replay has copied the table once it is done
    if (b->launched) PF_CUDA(cudaEventSynchronize(b->done));
    for (int i = 0; i < b->n; ++i) {
        b->ptrs_host[i] = const_cast<void*>(fwd ? in[i] : static_cast<const void*>(out[i]));
        b->ptrs_host[b->n + i] = const_cast<void*>(fwd ? static_cast<const void*>(out[i]) : in[i]);
    }
    PF_CUDA(cudaGraphLaunch(b->exec[fwd], stream));
    PF_CUDA(cudaEventRecord(b->done, stream));
    b->launched = true;
    return 0;
}

int batch_create(pfsht_plan* const* plans, int n, int nstreams, pfsht_batch** out) {
    if (!plans || !out || n < 1) return fail(PFSHT_ERR_ARGUMENT, "need at least one plan");
    if (nstreams < 0 || nstreams > 32) return fail(PFSHT_ERR_ARGUMENT, "nstreams must lie in 0..32");
    for (int i = 0; i < n; ++i) {
        if (!plans[i]) return fail(PFSHT_ERR_ARGUMENT, "NULL plan in the batch");
        if (plans[i]->kind == kMultiBox)
            return fail(PFSHT_ERR_UNSUPPORTED, "a multi-box plan cannot join a batch; batch its boxes' "
                                               "geometries as plans of their own");
    }
    const int dev = plans[0]->device;
    for (int i = 0; i < n; ++i) {
        if (plans[i]->device != dev) return fail(PFSHT_ERR_ARGUMENT, "all plans of a batch must share a device");
        for (int j = 0; j < i; ++j)
            if (plans[j] == plans[i]) return fail(PFSHT_ERR_ARGUMENT, "a plan appears twice in the batch");
    }
    DeviceGuard dg(dev);
    std::unique_ptr<pfsht_batch> b(new pfsht_batch());
    b->device = dev;
    b->n = n;
    b->plans.assign(plans, plans + n);
    PF_CUDA(cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking));
    const int ns = std::max(1, std::min(nstreams > 0 ? nstreams : 8, n));
    b->side.resize(ns);
    b->join.resize(ns);
    for (int k = 0; k < ns; ++k) {
        PF_CUDA(cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking));
        PF_CUDA(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
    }
    PF_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    PF_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    PF_CUDA(cudaHostAlloc(&b->ptrs_host, sizeof(void*) * 2 * n, cudaHostAllocDefault));
    PF_TRY(b->ptrs.alloc(sizeof(void*) * 2 * n));
    std::vector<RingSlot> slots(n);
    std::vector<double2*> stf(n);
    std::vector<FChunk> chunks;
    std::vector<RingBatchPlan> fw(n), ad(n);
    for (int i = 0; i < n; ++i) {
        pfsht_plan* p = plans[i];
        const size_t nf = sizeof(double2) * (size_t)p->M * p->B;
        if (!p->st_f.p) PF_TRY(p->st_f.alloc(nf));
        stf[i] = p->st_f.as<double2>();
        RingSlot& s = slots[i];
        s.t = p->rt;
        s.tf = p->rt_fwd;
        s.o = p->ro_cols;
        s.jlo = p->adj_items.view.jlo;
        s.jhi = p->adj_items.view.jhi;
        s.H = p->H.as<double2>();
        s.allow_sole = p->adj_items.view.rmax >= 2 ? 1 : 0;
        s.ptr = i;
        // spin plans run their own ring passes on the side streams (the merged launches are the
        // scalar recurrence)
        static const std::vector<RingItem> kNone;
        fw[i] = RingBatchPlan{p->spin ? &kNone : &p->fwd_items.host, p->B, p->fwd_items.view.rmax, p->rt_fwd.mix};
        ad[i] = RingBatchPlan{p->spin ? &kNone : &p->adj_items.host, p->B, p->adj_items.view.rmax, p->rt.mix};
        const int64_t tot = p->M * p->B;
        for (int64_t o = 0; o < tot; o += kFChunk) chunks.push_back(FChunk{i, o, std::min(kFChunk, tot - o)});
    }
    PF_TRY(b->slots.alloc(sizeof(RingSlot) * n));
    PF_TRY(b->stf.alloc(sizeof(double2*) * n));
    PF_TRY(b->chunks.alloc(sizeof(FChunk) * chunks.size()));
    b->nchunks = (int)chunks.size();
    PF_CUDA(cudaMemcpy(b->slots.p, slots.data(), sizeof(RingSlot) * n, cudaMemcpyHostToDevice));
    PF_CUDA(cudaMemcpy(b->stf.p, stf.data(), sizeof(double2*) * n, cudaMemcpyHostToDevice));
    PF_CUDA(cudaMemcpy(b->chunks.p, chunks.data(), sizeof(FChunk) * chunks.size(),
                       cudaMemcpyHostToDevice));
    PF_TRY(build_ring_merged(fw, false, b->mf, b->gf, b->main));
    PF_TRY(build_ring_merged(ad, true, b->ma, b->ga, b->main));
    *out = b.release();
    return 0;
}

}  // namespace

extern "C" {

pfsht_status pfsht_batch_create(pfsht_plan* const* plans, int32_t nplans, int32_t nstreams,
                                pfsht_batch** out) {
    if (out) *out = nullptr;
    return (pfsht_status)batch_create(plans, nplans, nstreams, out);
}

pfsht_status pfsht_batch_forward(pfsht_batch* b, const void* const* alms, void* const* fs,
                                 void* stream) {
    if (!b || !alms || !fs) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    for (int i = 0; i < b->n; ++i)
        if (!alms[i] || !fs[i]) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL array in the batch");
    return (pfsht_status)batch_apply(b, true, alms, fs, (cudaStream_t)stream);
}

pfsht_status pfsht_batch_adjoint(pfsht_batch* b, const void* const* fs, void* const* alms,
                                 void* stream) {
    if (!b || !alms || !fs) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    for (int i = 0; i < b->n; ++i)
        if (!alms[i] || !fs[i]) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL array in the batch");
    return (pfsht_status)batch_apply(b, false, fs, alms, (cudaStream_t)stream);
}

pfsht_status pfsht_batch_info(const pfsht_batch* b, int32_t* ring_launches_fwd,
                              int32_t* ring_launches_adj, int64_t* graph_nodes_fwd,
                              int64_t* graph_nodes_adj) {
    if (!b) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL batch");
    if (ring_launches_fwd) *ring_launches_fwd = (int32_t)b->gf.size() + (b->mf.nitems > 0 ? 1 : 0);
    if (ring_launches_adj) *ring_launches_adj = (int32_t)b->ga.size() + (b->ma.nitems > 0 ? 1 : 0);
    if (graph_nodes_fwd) *graph_nodes_fwd = b->nodes[1];
    if (graph_nodes_adj) *graph_nodes_adj = b->nodes[0];
    return PFSHT_OK;
}

pfsht_status pfsht_batch_destroy(pfsht_batch* b) {
    if (!b) return PFSHT_OK;
    DeviceGuard dg(b->device);
    if (b->launched) cudaEventSynchronize(b->done);
    delete b;
    return PFSHT_OK;
}

}  // extern "C"
