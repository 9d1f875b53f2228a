// elastic3d.cu -- 3-D isotropic elastic (velocity-stress, staggered grid)
// forward and boundary-saving adjoint for sm_100a, at spatial orders 2, 4, 6
// and 8 (this file: order 8 and the dispatch by order; elastic3d_orders.cu:
// orders 2, 4, 6; the body of every order is elastic3d_impl.cuh).
//
// Restates the reference's elastic3d path (src/sweep/csrc/cuda/equations/
// elastic3d/kernels.cuh, driver_traits.cuh; common/sg_driver.cuh):
//
//   forward, per step:
//     vel3      velocity update; the nine stress-derivative CPML memories
//               outside the physical box shrunk by one cell  kernels.cuh:104-248
//     str3      stress update with the nine velocity-derivative memories
//                                                             kernels.cuh:290-483
//     src3 / strips3 / rec3   source injection per source field, the nine
//               fields' boundary strips, the receiver gather  driver_traits.cuh:265-300
//   reverse, per step (driver_traits.cuh:680-905):
//     vsrc3     body-force rho correction (before the residuals)
//     res3      signed residual injection (stress -1, velocity +1); src3 with
//               -w takes the forward source back out
//     srev3     stress reconstruction on the box minus one cell   kernels.cuh:653-768
//     strips3   stress strips of step it - 1 restored
//     sprep3    stress-adjoint prepare (q and the adjoint memories of the
//               velocity derivatives) with the fused vp / vs / rho imaging
//                                                             kernels.cuh:1367-1615
//     rrho3     receiver rho correction                       common/common.cu:77-116
//     sapp3     stress-adjoint apply (adjoint velocities)     kernels.cuh:1683-1780
//     vprep3 / vapp3   velocity-adjoint prepare / apply       kernels.cuh:959-1236
//     cap3, vrev3, strips3   v(it) carriers, velocity reconstruction,
//               velocity strips of step it - 1                kernels.cuh:536-652
//
// One thread per cell on 32 x 4 x 2 (x, y, z) blocks, two z planes of a shot
// per grid row (against 32 x 8 tiles of one plane: 4.47 against 4.2 Gcell/s);
// the stencils read global memory through the read-only path.  (A z-marching
// variant with shared-memory planes and register z-queues, run at two CTAs
// per SM without a load pipeline, measured 2.8x slower in the forward; four
// cells of a column per thread with the z taps in a register window, at
// three CTAs per SM, 1.23x slower; the kernels that beat this layout need the
// 3-D acoustic kernels' TMA plane rings.)
// Layout: fields (B, nz, ny, nx), x fastest; CPML memories in per-axis slabs
// covering the cells outside the box shrunk by one cell along their axis
// (x: (B, nz, ny, WX), y: (B, nz, WY, nx), z: (B, WZ, ny, nx)).  Cells in the
// CPML branch because of another axis have zero coefficients on this one and
// keep no memory (as the reference's stored() gating).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <vector>

#include "common.cuh"
#include "elastic3d.cuh"

#define EL3D_M 4
#define EL3D_NS el3d_m4
#include "elastic3d_impl.cuh"
#undef EL3D_NS
#undef EL3D_M

namespace sweep {
namespace el3d {

// the entry points of the order the descriptor asks for
#define SWEEP_EL3D_BY_ORDER(CALL)                                                                          \
    switch (d->M) {                                                                                          \
    case 1: el3d_m1::CALL; break;                                                                            \
    case 2: el3d_m2::CALL; break;                                                                            \
    case 3: el3d_m3::CALL; break;                                                                            \
    case 4: el3d_m4::CALL; break;                                                                            \
    default: SWEEP_REQUIRE(false, "elastic3d: spatial orders 2, 4, 6 and 8 are built (got order %d)", 2 * d->M); \
    }

void sizes(const sweep_elastic3d_desc* d, int mem_mode, int ckpt_every, int64_t* ws_bytes, int64_t* tape_bytes)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_EL3D_BY_ORDER(sizes(d, mem_mode, ckpt_every, ws_bytes, tape_bytes))
}

void forward(const sweep_elastic3d_desc* d, int mem_mode, int ckpt_every, float* record, void* tape, void* ws,
             int64_t ws_bytes, cudaStream_t st)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_EL3D_BY_ORDER(forward(d, mem_mode, ckpt_every, record, tape, ws, ws_bytes, st))
}

void backward(const sweep_elastic3d_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
              float* grad_vp, float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_EL3D_BY_ORDER(backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_vs, grad_rho, ws, ws_bytes, st))
}

#undef SWEEP_EL3D_BY_ORDER

}  // namespace el3d
}  // namespace sweep
