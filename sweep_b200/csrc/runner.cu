// runner.cu -- stepped runners: a forward or backward pass advanced segment
// by segment over the time axis, as the reference's persistent runner API
// (reference src/sweep/csrc/core/capi.h:236-243, driven by
// src/sweep/csrc/cuda/common/eq_driver.cuh:199-453 and 715-925).
//
// A runner is created once over a problem and its caller-owned buffers
// (descriptor, record / gradients, tape, workspace: all kept valid until
// destroy), then run() advances it: a forward runner over [it_begin, it_end),
// segments in order from 0 to nt; a backward runner over the reverse segment
// [bw_it_end, bw_it_begin), segments in order from nt down to 0.  After a
// forward segment the record holds every step run so far, and the tape is
// complete after the segment that ends at nt; after a backward segment the
// gradients (and illuminations) hold the contribution of every step reversed
// so far.  The segments compute exactly what one call computes: the same
// kernels in the same order on the same state.  Boundary saving only (every
// strip format, device or host tape), as the reference's runners; step_phase
// must be 0 (its 1 / 2, the split of a step around a domain-decomposition
// halo exchange, have no counterpart here).
#include "acoustic2d.cuh"
#include "elastic2d.cuh"

namespace sweep {
namespace a3d {
void forward_segment(const sweep_acoustic_desc*, int, float*, void*, void*, int64_t, cudaStream_t, StepState&, int,
                     int);
void backward_segment(const sweep_acoustic_desc*, int, const float*, const void*, float*, float*, float*, float*,
                      void*, int64_t, cudaStream_t, StepState&, int, int);
void sizes(const sweep_acoustic_desc*, int, int, int64_t*, int64_t*);
}  // namespace a3d

namespace {

struct Runner {
    bool elastic = false, backward = false;
    int device = 0;
    sweep_acoustic_desc ad{};
    sweep_elastic_desc ed{};
    int mem_mode = 0;
    float* record = nullptr;
    const float* adj = nullptr;
    void* tape = nullptr;
    void* ws = nullptr;
    int64_t ws_bytes = 0;
    float *g0 = nullptr, *g1 = nullptr, *g2 = nullptr, *is = nullptr, *ir = nullptr;
    StepState seg;
    int nt() const { return elastic ? ed.nt : ad.nt; }
};

void check_mode(int mem_mode)
{
    const int base = mem_mode & ~SWEEP_MEM_HOST_TAPE;
    SWEEP_REQUIRE(base == SWEEP_MEM_BOUNDARY || base == SWEEP_MEM_BOUNDARY_FP16 || base == SWEEP_MEM_BOUNDARY_BF16 ||
                      base == SWEEP_MEM_BOUNDARY_INT8,
                  "runner: stepped runners take boundary saving only (memory mode %d)", mem_mode);
}

void check_sizes(const Runner& r)
{
    int64_t ws = 0, tape = 0;
    if (r.elastic) el2d::sizes(&r.ed, r.mem_mode, 0, &ws, &tape);
    else if (r.ad.ndim == 2) a2d::sizes(&r.ad, r.mem_mode, 0, &ws, &tape);
    else a3d::sizes(&r.ad, r.mem_mode, 0, &ws, &tape);
    SWEEP_REQUIRE(r.ws != nullptr && r.ws_bytes >= ws, "runner: workspace too small (%lld < %lld)",
                  (long long)r.ws_bytes, (long long)ws);
    SWEEP_REQUIRE(r.tape != nullptr, "runner: null tape");
}

Runner* make(bool elastic, bool backward, int mem_mode)
{
    check_mode(mem_mode);
    Runner* r = new Runner();
    r->elastic = elastic;
    r->backward = backward;
    r->mem_mode = mem_mode;
    SWEEP_CUDA(cudaGetDevice(&r->device));
    return r;
}

// Runs `fn` with the runner's device current, restoring the caller's.
template <class F>
void on_device(const Runner& r, F&& fn)
{
    int prev = 0;
    SWEEP_CUDA(cudaGetDevice(&prev));
    if (prev != r.device) SWEEP_CUDA(cudaSetDevice(r.device));
    try {
        fn();
    } catch (...) {
        if (prev != r.device) cudaSetDevice(prev);
        throw;
    }
    if (prev != r.device) SWEEP_CUDA(cudaSetDevice(prev));
}

Runner* live(void* h, bool backward)
{
    SWEEP_REQUIRE(h != nullptr, "runner: null handle");
    Runner* r = static_cast<Runner*>(h);
    SWEEP_REQUIRE(r->backward == backward, "runner: a %s runner handed to the %s entry",
                  r->backward ? "backward" : "forward", backward ? "backward" : "forward");
    return r;
}

}  // namespace
}  // namespace sweep

using namespace sweep;

extern "C" int sweep_b200_acoustic_forward_runner_create(const sweep_acoustic_desc* d, int32_t mem_mode,
                                                         float* record, void* tape, void* workspace,
                                                         int64_t workspace_bytes, void** handle, char* err,
                                                         int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr && handle != nullptr, "null argument");
        SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
        SWEEP_REQUIRE(record != nullptr || d->nrec == 0, "acoustic forward runner: null record");
        Runner* r = make(false, false, mem_mode);
        r->ad = *d; r->record = record; r->tape = tape; r->ws = workspace; r->ws_bytes = workspace_bytes;
        try {
            check_sizes(*r);
        } catch (...) {
            delete r;
            throw;
        }
        *handle = r;
    });
}

extern "C" int sweep_b200_acoustic_backward_runner_create(const sweep_acoustic_desc* d, int32_t mem_mode,
                                                          const float* adj, const void* tape, float* grad_vp,
                                                          float* grad_wavelet, float* illum_src, float* illum_rec,
                                                          void* workspace, int64_t workspace_bytes, void** handle,
                                                          char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr && handle != nullptr && grad_vp != nullptr, "null argument");
        SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
        SWEEP_REQUIRE(adj != nullptr || d->nrec == 0, "acoustic backward runner: null record cotangent");
        SWEEP_REQUIRE((illum_src == nullptr) == (illum_rec == nullptr),
                      "acoustic backward runner: pass both illuminations or neither");
        Runner* r = make(false, true, mem_mode);
        r->ad = *d; r->adj = adj; r->tape = const_cast<void*>(tape); r->ws = workspace; r->ws_bytes = workspace_bytes;
        r->g0 = grad_vp; r->g1 = grad_wavelet; r->is = illum_src; r->ir = illum_rec;
        r->seg.next = d->nt;
        try {
            check_sizes(*r);
        } catch (...) {
            delete r;
            throw;
        }
        *handle = r;
    });
}

extern "C" int sweep_b200_elastic_forward_runner_create(const sweep_elastic_desc* d, int32_t mem_mode, float* record,
                                                        void* tape, void* workspace, int64_t workspace_bytes,
                                                        void** handle, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr && handle != nullptr, "null argument");
        SWEEP_REQUIRE(record != nullptr || d->nrec == 0, "elastic forward runner: null record");
        Runner* r = make(true, false, mem_mode);
        r->ed = *d; r->record = record; r->tape = tape; r->ws = workspace; r->ws_bytes = workspace_bytes;
        try {
            check_sizes(*r);
        } catch (...) {
            delete r;
            throw;
        }
        *handle = r;
    });
}

extern "C" int sweep_b200_elastic_backward_runner_create(const sweep_elastic_desc* d, int32_t mem_mode,
                                                         const float* adj, const void* tape, float* grad_vp,
                                                         float* grad_vs, float* grad_rho, void* workspace,
                                                         int64_t workspace_bytes, void** handle, char* err,
                                                         int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr && handle != nullptr && grad_vp && grad_vs && grad_rho, "null argument");
        SWEEP_REQUIRE(adj != nullptr || d->nrec == 0, "elastic backward runner: null record cotangent");
        Runner* r = make(true, true, mem_mode);
        r->ed = *d; r->adj = adj; r->tape = const_cast<void*>(tape); r->ws = workspace; r->ws_bytes = workspace_bytes;
        r->g0 = grad_vp; r->g1 = grad_vs; r->g2 = grad_rho;
        r->seg.next = d->nt;
        try {
            check_sizes(*r);
        } catch (...) {
            delete r;
            throw;
        }
        *handle = r;
    });
}

extern "C" int sweep_b200_forward_runner_run(void* handle, int32_t it_begin, int32_t it_end, int32_t step_phase,
                                             void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        Runner* r = live(handle, false);
        SWEEP_REQUIRE(step_phase == 0,
                      "forward runner: step_phase %d -- only 0 (whole steps) is built; the domain-decomposition "
                      "split of a step (1 boundary strips, 2 interior) has no counterpart here", step_phase);
        SWEEP_REQUIRE(0 <= it_begin && it_begin <= it_end && it_end <= r->nt(),
                      "forward runner: require 0 <= it_begin <= it_end <= nt, got [%d, %d) with nt = %d", it_begin,
                      it_end, r->nt());
        SWEEP_REQUIRE(it_begin == r->seg.next,
                      "forward runner: segments run in order; the next one starts at step %d (got %d)", r->seg.next,
                      it_begin);
        if (it_begin == it_end) return;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        on_device(*r, [&] {
            if (r->elastic)
                el2d::forward_segment(&r->ed, r->mem_mode, r->record, r->tape, r->ws, r->ws_bytes, st, r->seg,
                                      it_begin, it_end);
            else if (r->ad.ndim == 2)
                a2d::forward_segment(&r->ad, r->mem_mode, r->record, r->tape, r->ws, r->ws_bytes, st, r->seg,
                                     it_begin, it_end);
            else
                a3d::forward_segment(&r->ad, r->mem_mode, r->record, r->tape, r->ws, r->ws_bytes, st, r->seg,
                                     it_begin, it_end);
        });
        r->seg.next = it_end;
    });
}

extern "C" int sweep_b200_backward_runner_run(void* handle, int32_t bw_it_begin, int32_t bw_it_end,
                                              int32_t step_phase, void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        Runner* r = live(handle, true);
        SWEEP_REQUIRE(step_phase == 0, "backward runner: step_phase %d -- only 0 (whole steps) is built",
                      step_phase);
        SWEEP_REQUIRE(0 <= bw_it_end && bw_it_end <= bw_it_begin && bw_it_begin <= r->nt(),
                      "backward runner: require 0 <= bw_it_end <= bw_it_begin <= nt, got [%d, %d) with nt = %d",
                      bw_it_end, bw_it_begin, r->nt());
        SWEEP_REQUIRE(bw_it_begin == r->seg.next,
                      "backward runner: segments run in order from nt down; the next one begins at step %d (got %d)",
                      r->seg.next, bw_it_begin);
        if (bw_it_begin == bw_it_end) return;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        on_device(*r, [&] {
            if (r->elastic)
                el2d::backward_segment(&r->ed, r->mem_mode, r->adj, r->tape, r->g0, r->g1, r->g2, r->ws,
                                       r->ws_bytes, st, r->seg, bw_it_begin, bw_it_end);
            else if (r->ad.ndim == 2)
                a2d::backward_segment(&r->ad, r->mem_mode, r->adj, r->tape, r->g0, r->g1, r->is, r->ir, r->ws,
                                      r->ws_bytes, st, r->seg, bw_it_begin, bw_it_end);
            else
                a3d::backward_segment(&r->ad, r->mem_mode, r->adj, r->tape, r->g0, r->g1, r->is, r->ir, r->ws,
                                      r->ws_bytes, st, r->seg, bw_it_begin, bw_it_end);
        });
        r->seg.next = bw_it_end;
    });
}

extern "C" int sweep_b200_runner_device_index(void* handle)
{
    return handle ? static_cast<Runner*>(handle)->device : -1;
}

extern "C" void sweep_b200_runner_destroy(void* handle)
{
    delete static_cast<Runner*>(handle);
}
