// conv_bf16.cu -- BF16 3x3 convolutions (stride 1, zero padding 1) as
// implicit GEMMs on the tensor cores with FP32 accumulation, for the U-Net
// preconditioner of the FWI update.  No counterpart in the reference (it has
// no learned preconditioner); checked against PyTorch's float64 conv2d.
//
// Layout: activations NHWC bf16 with C a multiple of 8 (16-byte channel
// groups); weights (Co, 3, 3, C) bf16.  Tap t = (dy + 1) * 3 + (dx + 1).
//
//   forward  y[p, co]  = sum_{t, c} x[p + off(t), c] w[co, t, c]          (M = pixels, N = Co, K = 9 C)
//   data     dx[p, c]  = sum_{t, co} dy[p - off(t), co] w[co, t, c]       (M = pixels, N = C,  K = 9 Co)
//   weight   dw[co, t, c] = sum_p dy[p, co] x[p + off(t), c]              (M = Co, N = 9 C, K = pixels)
//
// The forward and data passes share one kernel on the 5th-generation tensor
// cores: the CTA gathers a 128-pixel x 64-K tile of A (8-channel groups of an
// NHWC tensor at the tap-shifted pixel: sign +1 forward, -1 data) and a 64 x 64
// tile of B (the weights, or their per-tap transpose for the data pass) into
// shared memory in the UMMA K-major no-swizzle layout, and one thread issues
// tcgen05.mma (M 128, N 64, K 16) into an FP32 accumulator in tensor memory;
// tcgen05.commit on a per-stage mbarrier releases each of the two shared-memory
// stages, so the gather of one K tile overlaps the MMAs of the previous one.
// The epilogue reads the accumulator with tcgen05.ld.  The weight gradient
// (K = pixels) runs on the same tensor-core path, transposed (wgrad_umma).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "tma.cuh"

namespace sweep {
namespace conv {

constexpr int BM = 128, BN = 64, NT = 256;

// ------------------------------------------------------------ tcgen05 path
namespace umma {

constexpr int TK = 64;                       // K per shared-memory stage (4 MMAs of K 16)
constexpr int A_BYTES = BM * TK * 2;         // 16 KB
constexpr int B_BYTES = BN * TK * 2;         // 8 KB
constexpr int TMEM_COLS = 64;                // FP32 accumulator: 128 lanes x 64 columns

enum ErrCode { ERR_MMA_WAIT = 11 };

struct Smem {
    alignas(128) unsigned char a[2][A_BYTES];
    alignas(128) unsigned char b[2][B_BYTES];
    uint64_t done[2];                        // MMAs of a stage finished (tcgen05.commit)
    uint32_t tmem;                           // accumulator base address from tcgen05.alloc
};

// Byte offset of the 16-byte chunk (row r, K chunk kc) in the K-major
// no-swizzle layout: 8 x 16-byte core matrices, the 8 K chunks of a row group
// adjacent (leading byte offset 128), row groups 1024 bytes apart (stride
// byte offset), rows 16 bytes apart inside a core matrix.
__device__ __forceinline__ uint32_t chunk_off(int r, int kc) { return ((r >> 3) * 8 + kc) * 128 + (r & 7) * 16; }

// Shared-memory matrix descriptor: start address, leading / stride byte
// offsets (16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    constexpr uint64_t lbo = 128 >> 4, sbo = 1024 >> 4;
    return (uint64_t)((addr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: D F32, A and B BF16, both K-major, N 64, M 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tma::smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void ld8(uint32_t taddr, float (&v)[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace umma

struct Shape {
    int N, H, W;        // images, height, width
    int C;              // channels of the gathered tensor (multiple of 8)
    int Nout;           // output channels
    int sign;           // +1 forward (p + off), -1 data gradient (p - off)
};

// out[p, n] = sum_k A[p, k] B[n, k] (+ bias[n]);  A gathered from act.
// One CTA = 128 pixels x 64 outputs; thread 0 issues the MMAs, all threads
// gather and run the epilogue (warp w reads TMEM lanes 32 (w % 4) .. + 31,
// columns 32 (w / 4) .. + 31).
__global__ void __launch_bounds__(NT) gather_gemm(const __nv_bfloat16* __restrict__ act,
                                                  const __nv_bfloat16* __restrict__ Bt,
                                                  const float* __restrict__ bias, float* __restrict__ out, Shape S,
                                                  int* err)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    umma::Smem& sm = *reinterpret_cast<umma::Smem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long P = (long long)S.N * S.H * S.W;
    const long long HW = (long long)S.H * S.W;
    const long long p0 = (long long)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int K = 9 * S.C;
    const int nk = (K + umma::TK - 1) / umma::TK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tma::smem_u32(&sm.tmem)),
                     "r"(umma::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        tma::mbar_init(&sm.done[0], 1);
        tma::mbar_init(&sm.done[1], 1);
        tma::fence_barrier_init();
    }
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tmem = sm.tmem;

    // this thread's gather rows: A chunks id = tid + 256 u (row id % 128, K chunk id / 128),
    // B chunks likewise over 64 rows; the pixel decomposition is fixed per row
    const int ar = tid & (BM - 1);
    const long long pa = p0 + ar;
    const bool arow = pa < P;
    const int aimg = arow ? (int)(pa / HW) : 0;
    const int arem = arow ? (int)(pa - (long long)aimg * HW) : 0;
    const int ah = arem / S.W, aw = arem - (arem / S.W) * S.W;
    bool ok = true;

    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt & 1;
        if (kt >= 2) {
            // the MMAs that read this stage two tiles ago are done
            ok = ok && tma::mbar_wait(&sm.done[st], ((kt >> 1) - 1) & 1, err, umma::ERR_MMA_WAIT);
        }
        const int kbase = kt * umma::TK;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int kc = (tid >> 7) + 2 * u;           // 0..7
            const int k = kbase + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (arow && k < K) {
                const int t = k / S.C, c = k - t * S.C;
                const int h = ah + S.sign * (t / 3 - 1), w = aw + S.sign * (t % 3 - 1);
                if (h >= 0 && h < S.H && w >= 0 && w < S.W)
                    v = *reinterpret_cast<const uint4*>(act + (((long long)aimg * S.H + h) * S.W + w) * S.C + c);
            }
            *reinterpret_cast<uint4*>(sm.a[st] + umma::chunk_off(ar, kc)) = v;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int id = tid + NT * u;
            const int r = id & (BN - 1), kc = id >> 6;   // 64 rows x 8 chunks
            const int n = n0 + r, k = kbase + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (n < S.Nout && k < K) v = *reinterpret_cast<const uint4*>(Bt + (long long)n * K + k);
            *reinterpret_cast<uint4*>(sm.b[st] + umma::chunk_off(r, kc)) = v;
        }
        umma::fence_async_smem();                        // generic writes -> tensor-core reads
        __syncthreads();
        if (tid == 0) {
            umma::fence_after();
            const uint32_t a0 = tma::smem_u32(sm.a[st]), b0 = tma::smem_u32(sm.b[st]);
#pragma unroll
            for (int kk = 0; kk < umma::TK / 16; ++kk)
                umma::mma(tmem, umma::smem_desc(a0 + kk * 256), umma::smem_desc(b0 + kk * 256),
                          (kt > 0 || kk > 0) ? 1u : 0u);
            umma::commit(&sm.done[st]);
        }
    }
    // the last commit covers every MMA issued before it
    const int last = nk - 1;
    ok = ok && tma::mbar_wait(&sm.done[last & 1], (last >> 1) & 1, err, umma::ERR_MMA_WAIT);
    umma::fence_after();

    const int q = warp & 3, half = warp >> 2;
    const long long p = p0 + 32 * q + lane;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float v[8];
        umma::ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * half + 8 * j), v);
        umma::wait_ld();
        const int n = n0 + 32 * half + 8 * j;
        if (ok && p < P && n < S.Nout) {
            float* o = out + p * S.Nout + n;
#pragma unroll
            for (int e = 0; e < 8; ++e) v[e] += bias ? bias[n + e] : 0.f;
            *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
            *reinterpret_cast<float4*>(o + 4) = make_float4(v[4], v[5], v[6], v[7]);
        }
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(umma::TMEM_COLS));
}

// Weight gradient on the 5th-generation tensor cores, transposed:
//   dw[co, k] = sum_p X[p, k] dy[p, co],  X[p, k = t C + c] = x[p + off(t), c],
// as D[k, co] = A[k, p] B[co, p] with M = 9 C (128 per CTA), N = Co (64 per
// CTA) and K = pixels (64 per shared-memory stage; the pixel range split
// over blockIdx.z, partial sums added atomically).  Both operands are
// gathered K-major (pixels contiguous): a 16-byte load of x (8 channels of one
// tap-shifted pixel) or of dy (8 output channels of one pixel) fills one
// K column of 8 rows.  Same shared-memory layout, descriptors and MMA shape
// (M 128, N 64, K 16) as gather_gemm; the epilogue reads the accumulator with
// tcgen05.ld and adds it into dw.
__global__ void __launch_bounds__(NT) wgrad_umma(const __nv_bfloat16* __restrict__ x,
                                                 const __nv_bfloat16* __restrict__ dy, float* __restrict__ dw,
                                                 int Nimg, int H, int W, int C, int Co, int pix_per_split, int* err)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    umma::Smem& sm = *reinterpret_cast<umma::Smem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long P = (long long)Nimg * H * W, HW = (long long)H * W;
    const int K = 9 * C;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const long long pbeg = (long long)blockIdx.z * pix_per_split;
    const long long pend = min(P, pbeg + pix_per_split);
    const int nk = (int)((pend - pbeg + umma::TK - 1) / umma::TK);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tma::smem_u32(&sm.tmem)),
                     "r"(umma::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        tma::mbar_init(&sm.done[0], 1);
        tma::mbar_init(&sm.done[1], 1);
        tma::fence_barrier_init();
    }
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tmem = sm.tmem;
    // this thread's pixel column of the stage: the same for every unit it gathers
    const int pc = tid & (umma::TK - 1);
    bool ok = true;
    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt & 1;
        if (kt >= 2) ok = ok && tma::mbar_wait(&sm.done[st], ((kt >> 1) - 1) & 1, err, umma::ERR_MMA_WAIT);
        const long long p = pbeg + (long long)kt * umma::TK + pc;
        const bool pin = p < pend;
        const int img = pin ? (int)(p / HW) : 0;
        const int rem = pin ? (int)(p - (long long)img * HW) : 0;
        const int ph = rem / W, pw = rem - (rem / W) * W;
        const uint32_t col = (uint32_t)(pc & 7) * 2;
        // A: 16 row groups of 8 (k = m0 + 8 g .. + 7, one tap, 8 channels) x 64 pixels
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int g = (tid >> 6) + 4 * u;             // 0..15
            const int k = m0 + 8 * g;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (pin && k < K) {
                const int t = k / C, c = k - t * C;
                const int h = ph + (t / 3 - 1), w = pw + (t % 3 - 1);
                if (h >= 0 && h < H && w >= 0 && w < W)
                    v = *reinterpret_cast<const uint4*>(x + (((long long)img * H + h) * W + w) * C + c);
            }
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
            for (int r = 0; r < 8; ++r)
                *reinterpret_cast<__nv_bfloat16*>(sm.a[st] + umma::chunk_off(8 * g + r, pc >> 3) + col) = e[r];
        }
        // B: 8 row groups of 8 output channels x 64 pixels
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int g = (tid >> 6) + 4 * u;             // 0..7
            const int co = n0 + 8 * g;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (pin && co < Co) v = *reinterpret_cast<const uint4*>(dy + p * Co + co);
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
            for (int r = 0; r < 8; ++r)
                *reinterpret_cast<__nv_bfloat16*>(sm.b[st] + umma::chunk_off(8 * g + r, pc >> 3) + col) = e[r];
        }
        umma::fence_async_smem();                        // generic writes -> tensor-core reads
        __syncthreads();
        if (tid == 0) {
            umma::fence_after();
            const uint32_t a0 = tma::smem_u32(sm.a[st]), b0 = tma::smem_u32(sm.b[st]);
#pragma unroll
            for (int kk = 0; kk < umma::TK / 16; ++kk)
                umma::mma(tmem, umma::smem_desc(a0 + kk * 256), umma::smem_desc(b0 + kk * 256),
                          (kt > 0 || kk > 0) ? 1u : 0u);
            umma::commit(&sm.done[st]);
        }
    }
    if (nk > 0) {
        const int last = nk - 1;
        ok = ok && tma::mbar_wait(&sm.done[last & 1], (last >> 1) & 1, err, umma::ERR_MMA_WAIT);
    }
    umma::fence_after();
    const int q = warp & 3, half = warp >> 2;
    const int k = m0 + 32 * q + lane;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float v[8];
        umma::ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * half + 8 * j), v);
        umma::wait_ld();
        const int co = n0 + 32 * half + 8 * j;
        if (ok && nk > 0 && k < K) {
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (co + e < Co) atomicAdd(dw + (long long)(co + e) * K + k, v[e]);
        }
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(umma::TMEM_COLS));
}

// Device error flag of the convolution kernels (one per process; zeroed
// when made and by every status call).
int* error_flag()
{
    static int* flag = nullptr;
    if (!flag) {
        SWEEP_CUDA(cudaMalloc(&flag, sizeof(int)));
        SWEEP_CUDA(cudaMemset(flag, 0, sizeof(int)));
    }
    return flag;
}

}  // namespace conv
}  // namespace sweep

using namespace sweep;

extern "C" int sweep_b200_conv3x3_gemm(const void* act, const void* bt, const float* bias, float* out,
                                                      int32_t n, int32_t h, int32_t w, int32_t c, int32_t nout,
                                                      int32_t sign, void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(act && bt && out, "conv3x3: null pointer");
        SWEEP_REQUIRE(n >= 1 && h >= 1 && w >= 1 && nout >= 1, "conv3x3: empty shape");
        SWEEP_REQUIRE(c >= 8 && c % 8 == 0, "conv3x3: channels must be a positive multiple of 8 (got %d)", c);
        SWEEP_REQUIRE(sign == 1 || sign == -1, "conv3x3: sign must be +1 or -1");
        SWEEP_REQUIRE(((uintptr_t)act & 15) == 0 && ((uintptr_t)bt & 15) == 0, "conv3x3: operands must be 16-byte aligned");
        SWEEP_REQUIRE(nout % 8 == 0, "conv3x3: output channels must be a multiple of 8 (got %d)", nout);
        SWEEP_REQUIRE(((uintptr_t)out & 15) == 0, "conv3x3: output must be 16-byte aligned");
        conv::Shape S{n, h, w, c, nout, sign};
        const long long P = (long long)n * h * w;
        const dim3 grid((unsigned)((P + conv::BM - 1) / conv::BM), (unsigned)((nout + conv::BN - 1) / conv::BN));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        static bool attr = false;
        if (!attr) {
            SWEEP_CUDA(cudaFuncSetAttribute(conv::gather_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)sizeof(conv::umma::Smem)));
            attr = true;
        }
        conv::gather_gemm<<<grid, conv::NT, sizeof(conv::umma::Smem), st>>>(
            static_cast<const __nv_bfloat16*>(act), static_cast<const __nv_bfloat16*>(bt), bias, out, S,
            conv::error_flag());
        SWEEP_LAUNCH_CHECK();
    });
}

extern "C" int sweep_b200_conv3x3_wgrad(const void* x, const void* dy, float* dw, int32_t n, int32_t h,
                                                       int32_t w, int32_t c, int32_t co, void* stream, char* err,
                                                       int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(x && dy && dw, "conv3x3 wgrad: null pointer");
        SWEEP_REQUIRE(c >= 8 && c % 8 == 0 && co >= 8 && co % 8 == 0,
                      "conv3x3 wgrad: channel counts must be positive multiples of 8 (got %d, %d)", c, co);
        SWEEP_REQUIRE(((uintptr_t)x & 15) == 0 && ((uintptr_t)dy & 15) == 0, "conv3x3 wgrad: operands must be 16-byte aligned");
        const long long P = (long long)n * h * w;
        const int K = 9 * c;
        // tensor cores: M = 9 c (128 per CTA), N = co (64 per CTA), K = pixels
        const unsigned gx = (unsigned)((K + conv::BM - 1) / conv::BM), gy = (unsigned)((co + conv::BN - 1) / conv::BN);
        // pixel splits: about four CTAs per SM in all, each split a multiple of 64 pixels
        long long splits = std::max(1LL, (4LL * 148) / ((long long)gx * gy));
        long long per = (P + splits - 1) / splits;
        per = (per + 63) / 64 * 64;
        splits = (P + per - 1) / per;
        const dim3 grid(gx, gy, (unsigned)splits);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        static bool attr = false;
        if (!attr) {
            SWEEP_CUDA(cudaFuncSetAttribute(conv::wgrad_umma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)sizeof(conv::umma::Smem)));
            attr = true;
        }
        SWEEP_CUDA(cudaMemsetAsync(dw, 0, sizeof(float) * (size_t)co * K, st));
        conv::wgrad_umma<<<grid, conv::NT, sizeof(conv::umma::Smem), st>>>(
            static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), dw, n, h, w, c, co,
            (int)per, conv::error_flag());
        SWEEP_LAUNCH_CHECK();
    });
}

extern "C" int sweep_b200_conv3x3_status(void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        int* flag = conv::error_flag();
        int h_flag = 0;
        SWEEP_CUDA(cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        SWEEP_CUDA(cudaStreamSynchronize(st));
        if (h_flag) SWEEP_CUDA(cudaMemset(flag, 0, sizeof(int)));
        SWEEP_REQUIRE(h_flag == 0, "conv3x3: a tensor-core wait did not complete in time (code %d); "
                                   "outputs since the last status call are invalid", h_flag);
    });
}
