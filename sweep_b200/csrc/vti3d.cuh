// vti3d.cuh -- host-side interface of vti3d.cu (3-D first-order acoustic VTI)
// shared with the C ABI file.
#pragma once

#include "common.cuh"

namespace sweep {
namespace vti3 {

void sizes(const sweep_vti3d_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_vti3d_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_vti3d_desc*, int, int, const float*, const void*, float*, float*, float*, float*, void*,
              int64_t, cudaStream_t);

}  // namespace vti3
}  // namespace sweep
