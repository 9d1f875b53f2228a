// elastic3d_orders.cu -- the 3-D isotropic elastic path at spatial orders 2,
// 4 and 6 (stencil half-widths 1, 2, 3): the body of elastic3d_impl.cuh built
// once per order, each in its own namespace; elastic3d.cu holds order 8 and
// the dispatch.  The reference's Elastic3D defaults to order 4.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <vector>

#include "common.cuh"
#include "elastic3d.cuh"

#define EL3D_M 1
#define EL3D_NS el3d_m1
#include "elastic3d_impl.cuh"
#undef EL3D_NS
#undef EL3D_M

#define EL3D_M 2
#define EL3D_NS el3d_m2
#include "elastic3d_impl.cuh"
#undef EL3D_NS
#undef EL3D_M

#define EL3D_M 3
#define EL3D_NS el3d_m3
#include "elastic3d_impl.cuh"
#undef EL3D_NS
#undef EL3D_M
