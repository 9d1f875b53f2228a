// elastic_orders.cuh -- host-side interface of elastic_orders.cu (the 2-D
// elastic path at spatial orders other than 8) shared with the C ABI file.
#pragma once

#include "common.cuh"

namespace sweep {
namespace eord {

void sizes(const sweep_elastic_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_elastic_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_elastic_desc*, int, int, const float*, const void*, float*, float*, float*, void*, int64_t,
              cudaStream_t);

}  // namespace eord
}  // namespace sweep
