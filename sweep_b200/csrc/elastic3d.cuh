// elastic3d.cuh -- host-side interface of elastic3d.cu shared with the C ABI file.
#pragma once

#include "common.cuh"

namespace sweep {

// the entry points of one spatial order (elastic3d_impl.cuh, built once per
// order: el3d_m4 in elastic3d.cu, el3d_m1..el3d_m3 in elastic3d_orders.cu)
#define SWEEP_EL3D_DECLARE(NS)                                                                              \
    namespace NS {                                                                                          \
    void sizes(const sweep_elastic3d_desc*, int, int, int64_t*, int64_t*);                                  \
    void forward(const sweep_elastic3d_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);       \
    void backward(const sweep_elastic3d_desc*, int, int, const float*, const void*, float*, float*, float*, \
                  void*, int64_t, cudaStream_t);                                                            \
    }
SWEEP_EL3D_DECLARE(el3d_m1)
SWEEP_EL3D_DECLARE(el3d_m2)
SWEEP_EL3D_DECLARE(el3d_m3)
SWEEP_EL3D_DECLARE(el3d_m4)
#undef SWEEP_EL3D_DECLARE

// the entry points the C ABI calls: dispatch on the descriptor's order
namespace el3d {

void sizes(const sweep_elastic3d_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_elastic3d_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_elastic3d_desc*, int, int, const float*, const void*, float*, float*, float*,
              void*, int64_t, cudaStream_t);

}  // namespace el3d
}  // namespace sweep
