// elastic2d.cuh -- host-side interface of elastic2d.cu shared with the C ABI file.
#pragma once

#include "common.cuh"

namespace sweep {
namespace el2d {

void sizes(const sweep_elastic_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_elastic_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_elastic_desc*, int, int, const float*, const void*, float*, float*, float*,
              void*, int64_t, cudaStream_t);
// Stepped runs (boundary saving): forward steps [it0, it1) after the
// segments before; backward reverse steps [bw1, bw0) after the segments above
// (the gradients overwritten with those of every step reversed so far).
void forward_segment(const sweep_elastic_desc* d, int mem_mode, float* record, void* tape, void* ws,
                     int64_t ws_bytes, cudaStream_t st, StepState& seg, int it0, int it1);
void backward_segment(const sweep_elastic_desc* d, int mem_mode, const float* adj, const void* tape,
                      float* grad_vp, float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st,
                      StepState& seg, int bw0, int bw1);

}  // namespace el2d
}  // namespace sweep
