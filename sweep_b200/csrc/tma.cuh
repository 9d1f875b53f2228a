// tma.cuh -- Tensor Memory Accelerator tile loads and mbarrier pipelines for
// sm_100a, written directly in PTX.  Loads only, never multicast: every tensor
// map covers memory of the GPU the kernel runs on.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace sweep {
namespace tma {

// Upper bound of one mbarrier wait, in SM clock cycles (~2 s at 1.9 GHz).
// Every wait in this library gives up after it, raises the call's error flag
// and returns: the host reports the failure instead of the GPU hanging.
constexpr long long kWaitCycles = 4000000000LL;

// ----------------------------------------------------------------- host side
// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        SWEEP_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        SWEEP_REQUIRE(q == cudaDriverEntryPointSuccess && p != nullptr,
                      "cuTensorMapEncodeTiled is not available from the driver");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// A rank-`rank` float32 tensor map: dims[0] fastest, strides in ELEMENTS for
// dims 1.. (each a multiple of 4 floats), box[] the tile loaded per copy.
// Out-of-range elements of a tile read as zero.
inline CUtensorMap make_map(const float* base, int rank, const uint64_t* dims, const uint64_t* strides_el,
                            const uint32_t* box)
{
    CUtensorMap m;
    cuuint64_t gd[5], gs[4];
    cuuint32_t bd[5], es[5];
    for (int i = 0; i < rank; ++i) {
        gd[i] = dims[i];
        bd[i] = box[i];
        es[i] = 1;
    }
    for (int i = 0; i + 1 < rank; ++i) {
        SWEEP_REQUIRE((strides_el[i] * 4) % 16 == 0, "TMA stride must be a multiple of 16 bytes");
        gs[i] = strides_el[i] * 4;
    }
    SWEEP_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0, "TMA base must be 16-byte aligned");
    SWEEP_REQUIRE((box[0] * 4) % 16 == 0, "TMA box row must be a multiple of 16 bytes");
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<float*>(base), gd, gs, bd, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    SWEEP_REQUIRE(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return m;
}

// --------------------------------------------------------------- device side
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`; false (and *err = code) after `budget`
// SM clock cycles.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, int* err, int code, long long budget)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > budget) {
            atomicExch(err, code);
            return false;
        }
    }
    return true;
}

// The library's wait: gives up after kWaitCycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code)
{
    return mbar_wait_for(bar, parity, err, code, kWaitCycles);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 3-D tiled load of the box at (x, y, z) of `map` into shared memory `dst`;
// completion is counted on `bar` in bytes.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Prefetch the box at (x, y, z) of `map` into L2 (no shared memory, no
// completion to wait for).
__device__ __forceinline__ void prefetch_3d(const CUtensorMap* map, int x, int y, int z)
{
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z)
                 : "memory");
}

__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z, int w)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace tma
}  // namespace sweep
