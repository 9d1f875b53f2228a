// acoustic_orders.cuh -- host-side interface of acoustic_orders.cu (the
// acoustic path at spatial orders other than 8) shared with the C ABI file.
#pragma once

#include "common.cuh"

namespace sweep {
namespace aord {

void sizes(const sweep_acoustic_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_acoustic_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_acoustic_desc*, int, int, const float*, const void*, float*, float*, float*, float*, void*,
              int64_t, cudaStream_t);

}  // namespace aord
}  // namespace sweep
