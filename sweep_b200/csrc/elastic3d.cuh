// elastic3d.cuh -- host-side interface of elastic3d.cu shared with the C ABI file.
#pragma once

#include "common.cuh"

namespace sweep {
namespace el3d {

void sizes(const sweep_elastic3d_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_elastic3d_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_elastic3d_desc*, int, int, const float*, const void*, float*, float*, float*,
              void*, int64_t, cudaStream_t);

}  // namespace el3d
}  // namespace sweep
