// common.cuh -- shared host/device helpers of libsweep_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sweep_b200.h"

namespace sweep {

// Host-side error: thrown inside the library, caught at the C boundary and
// turned into (non-zero return, message), as the reference's guarded()
// (reference src/sweep/csrc/cuda/common/capi.cu:578-580).
struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define SWEEP_REQUIRE(cond, ...)                                                  \
    do {                                                                          \
        if (!(cond)) {                                                            \
            char _buf[512];                                                       \
            snprintf(_buf, sizeof(_buf), __VA_ARGS__);                            \
            throw ::sweep::Error(_buf);                                           \
        }                                                                         \
    } while (0)

#define SWEEP_CUDA(call)                                                          \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess)                                                    \
            throw ::sweep::Error(std::string(#call " failed: ") + cudaGetErrorString(_e)); \
    } while (0)

#define SWEEP_LAUNCH_CHECK()                                                      \
    do {                                                                          \
        cudaError_t _e = cudaGetLastError();                                      \
        if (_e != cudaSuccess)                                                    \
            throw ::sweep::Error(std::string("kernel launch failed: ") + cudaGetErrorString(_e)); \
    } while (0)

// Run `fn` and convert any exception into the C ABI's (rc, message) pair.
template <class F>
int guarded(char* err, int32_t cap, F&& fn)
{
    try {
        fn();
        if (err && cap > 0) err[0] = '\0';
        return 0;
    } catch (const std::exception& e) {
        if (err && cap > 0) {
            strncpy(err, e.what(), (size_t)cap - 1);
            err[cap - 1] = '\0';
        }
        return 1;
    } catch (...) {
        if (err && cap > 0) {
            strncpy(err, "unknown error", (size_t)cap - 1);
            err[cap - 1] = '\0';
        }
        return 2;
    }
}

// Bump allocator over a caller-owned byte range: every sub-buffer 256-byte
// aligned.  With base == nullptr it only measures (the sizes query and the
// carve then agree by construction).
struct Carve {
    char* base;
    int64_t off = 0;
    explicit Carve(void* b) : base(static_cast<char*>(b)) {}
    template <class T>
    T* take(int64_t count)
    {
        off = (off + 255) & ~int64_t(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * (int64_t)sizeof(T);
        return p;
    }
};

// Boundary-saving tape in pinned host memory (reference
// BoundarySaving(storage='cpu'), boundary/runtime.cuh:91-620): the step
// kernels write a ring of R device slots; a copy stream moves forward slot it
// to host slot it and, in the reverse, brings host slots back into the ring
// ahead of their use.  Events order every reuse of a ring slot; close() makes
// the caller's stream wait for every copy.
struct HostRing {
    static constexpr int R = 4;
    char* ring = nullptr;            // R device slots of `step` bytes
    char* host = nullptr;            // the host tape (pinned)
    long long step = 0;
    cudaStream_t main = nullptr, copy = nullptr;
    cudaEvent_t ready[R], freed[R];

    void open(void* ring_, void* host_, long long step_, cudaStream_t st)
    {
        ring = static_cast<char*>(ring_);
        host = static_cast<char*>(host_);
        step = step_;
        main = st;
        SWEEP_CUDA(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
        for (int i = 0; i < R; ++i) {
            SWEEP_CUDA(cudaEventCreateWithFlags(&ready[i], cudaEventDisableTiming));
            SWEEP_CUDA(cudaEventCreateWithFlags(&freed[i], cudaEventDisableTiming));
        }
        after(main, copy);           // the copies start after the work queued so far
    }
    void* slot(int t) const { return ring + (long long)(t % R) * step; }
    // forward: the copy that last emptied slot(t) must be done before step t writes it
    void before_write(int t)
    {
        if (t >= R) SWEEP_CUDA(cudaStreamWaitEvent(main, freed[t % R], 0));
    }
    // forward: once step t's kernels are done, move slot(t) to host slot t
    void after_write(int t)
    {
        SWEEP_CUDA(cudaEventRecord(ready[t % R], main));
        SWEEP_CUDA(cudaStreamWaitEvent(copy, ready[t % R], 0));
        SWEEP_CUDA(cudaMemcpyAsync(host + (long long)t * step, slot(t), step, cudaMemcpyDeviceToHost, copy));
        SWEEP_CUDA(cudaEventRecord(freed[t % R], copy));
    }
    // reverse: host slot t into the ring, after the slot's last reader when `reused`
    void fetch(int t, bool reused)
    {
        if (reused) SWEEP_CUDA(cudaStreamWaitEvent(copy, freed[t % R], 0));
        SWEEP_CUDA(cudaMemcpyAsync(slot(t), host + (long long)t * step, step, cudaMemcpyHostToDevice, copy));
        SWEEP_CUDA(cudaEventRecord(ready[t % R], copy));
    }
    void before_read(int t) { SWEEP_CUDA(cudaStreamWaitEvent(main, ready[t % R], 0)); }
    void after_read(int t) { SWEEP_CUDA(cudaEventRecord(freed[t % R], main)); }
    void close()
    {
        if (!copy) return;
        after(copy, main);
        for (int i = 0; i < R; ++i) {
            cudaEventDestroy(ready[i]);
            cudaEventDestroy(freed[i]);
        }
        cudaStreamDestroy(copy);     // released once its queued work is done
        copy = nullptr;
    }
    // `later` waits for the work queued on `earlier` so far
    static void after(cudaStream_t earlier, cudaStream_t later)
    {
        cudaEvent_t e;
        SWEEP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        SWEEP_CUDA(cudaEventRecord(e, earlier));
        SWEEP_CUDA(cudaStreamWaitEvent(later, e, 0));
        SWEEP_CUDA(cudaEventDestroy(e));
    }
};

// Per-shape launch schedule (sweep_b200_schedule): the recorded one, or all
// built-in (zeros, graph_steps -1).  Thread-safe; defined in schedule.cu.
sweep_b200_schedule recorded_schedule(const sweep_acoustic_desc* d);
sweep_b200_schedule recorded_schedule(const sweep_elastic_desc* d);

// Time steps per captured graph when neither the schedule nor the
// environment (SWEEP_B200_GRAPH_STEPS) sets it.
constexpr int kGraphStepsDefault = 64;
int resolve_graph_steps(int recorded);

// A run of time steps issued as CUDA graphs of up to `steps` steps each.  The
// launches of a chunk are captured on a private non-blocking stream (capture
// runs nothing), the graph is instantiated and launched on the caller's
// stream, and the next chunk is captured while the previous one runs on the
// GPU.  The captured launches are the stream path's launches in the same
// order, so results are identical.  steps <= 0: every launch goes straight to
// the caller's stream.  Use: take stream() for each step's launches, call
// step_done() after them, and flush() once after the loop, before anything
// else is queued on the caller's stream.
class StepGraphs {
public:
    StepGraphs(cudaStream_t st, int steps) : st_(st), steps_(steps)
    {
        if (steps_ > 0) SWEEP_CUDA(cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking));
    }
    StepGraphs(const StepGraphs&) = delete;
    StepGraphs& operator=(const StepGraphs&) = delete;
    ~StepGraphs()
    {
        abort_capture();
        if (cs_) cudaStreamDestroy(cs_);
    }
    cudaStream_t stream()
    {
        if (steps_ <= 0) return st_;
        if (!capturing_) {
            SWEEP_CUDA(cudaStreamBeginCapture(cs_, cudaStreamCaptureModeThreadLocal));
            capturing_ = true;
        }
        return cs_;
    }
    void step_done()
    {
        if (capturing_ && ++n_ >= steps_) flush();
    }
    void flush()
    {
        if (!capturing_) return;
        capturing_ = false;
        n_ = 0;
        cudaGraph_t g = nullptr;
        SWEEP_CUDA(cudaStreamEndCapture(cs_, &g));
        cudaGraphExec_t ge = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        SWEEP_CUDA(ei);
        const cudaError_t el = cudaGraphLaunch(ge, st_);
        cudaGraphExecDestroy(ge);    // an executable graph in flight is freed when it completes
        SWEEP_CUDA(el);
        ++launched_;
    }
    int graphs_launched() const { return launched_; }

private:
    void abort_capture()
    {
        if (!capturing_) return;
        capturing_ = false;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs_, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
    }
    cudaStream_t st_, cs_ = nullptr;
    int steps_, n_ = 0, launched_ = 0;
    bool capturing_ = false;
};

// Between the segments of a stepped run (the sweep_b200_*_runner entries):
// where the next segment starts and the rotating buffer state of the pass --
// wavefield buffer indices, swapped CPML pointers -- which an equation saves
// after a segment and restores before the next.  Segments run in order: a
// forward [it_begin, it_end) starts where the last one ended, a backward
// reverses [bw_end, bw_begin) starting where the last one stopped.
struct StepState {
    int next = 0;            // forward: next step; backward: the step above the next segment
    bool begun = false;      // the first segment has run (fields set up)
    int idx[8] = {};
    void* ptr[8] = {};
};

// Source / receiver events grouped by (shot, tile): a CSR table so that the
// CTA owning a tile finds its point sources and receivers without scanning the
// whole list.  `cell` is the tile-local linear cell index, `id` the global
// event index (b * n + s).
struct EventTable {
    const int32_t* off = nullptr;   // (B * ntiles + 1)
    const int2* ev = nullptr;       // (count)
};


}  // namespace sweep
