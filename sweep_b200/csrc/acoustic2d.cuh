// acoustic2d.cuh -- host-side interface of acoustic2d.cu shared with the C ABI files.
#pragma once

#include "common.cuh"

namespace sweep {
namespace a2d {

// Host staging of the source / receiver event tables.  The regular entry
// points size it with std::vector; the allocation-free entry point hands
// fixed static storage.
struct HostStage {
    int32_t *loc_src, *loc_rec;      // (B, nsrc, 2), (B, nrec, 2)
    int32_t *off_src, *off_rec;      // (B * ntiles + 1)
    int2 *ev_src, *ev_rec;           // (B * nsrc), (B * nrec)
    int32_t* fill;                   // (B * ntiles)
    int32_t* order;                  // (ntiles)
};

void sizes(const sweep_acoustic_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_acoustic_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_acoustic_desc*, int, int, const float*, const void*, float*, float*,
              float*, float*, void*, int64_t, cudaStream_t);
// Workspace bytes of a forward without a tape (no backward to follow).
int64_t forward_only_bytes(const sweep_acoustic_desc* d);
// Event-table staging sizes: shot-tile keys (+1) and events of each kind.
void stage_sizes(const sweep_acoustic_desc* d, int64_t* nkey, int64_t* nev_src, int64_t* nev_rec);
// Forward with an explicit workspace and host staging (stage == nullptr: growable);
// `mem_mode` as in the C ABI; ckpt_every > 0 writes the checkpoint-mode tape.
// seg != nullptr: a stepped run of [seg0, seg1) (boundary saving only).
void forward_with(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape, void* ws,
                  int64_t ws_bytes, cudaStream_t st, const HostStage* stage, StepState* seg, int seg0, int seg1);
// Stepped runs (boundary saving): forward steps [it0, it1) after the
// segments before; backward reverse steps [bw1, bw0) after the segments above
// (grad_vp / illum overwritten with the gradient of every step reversed so far).
void forward_segment(const sweep_acoustic_desc* d, int mem_mode, float* record, void* tape, void* ws,
                     int64_t ws_bytes, cudaStream_t st, StepState& seg, int it0, int it1);
void backward_segment(const sweep_acoustic_desc* d, int mem_mode, const float* adj, const void* tape,
                      float* grad_vp, float* grad_w, float* illum_s, float* illum_r, void* ws, int64_t ws_bytes,
                      cudaStream_t st, StepState& seg, int bw0, int bw1);

}  // namespace a2d
}  // namespace sweep
