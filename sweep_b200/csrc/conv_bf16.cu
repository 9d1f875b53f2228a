// conv_bf16.cu -- BF16 3x3 convolutions (stride 1, zero padding 1) as
// implicit GEMMs on the tensor cores (mma.sync m16n8k16, FP32 accumulation),
// for the U-Net preconditioner of the FWI update.  No counterpart in the
// reference (it has no learned preconditioner); checked against PyTorch's
// float32 conv2d.
//
// Layout: activations NHWC bf16 with C a multiple of 8 (16-byte channel
// groups); weights (Co, 3, 3, C) bf16.  Tap t = (dy + 1) * 3 + (dx + 1).
//
//   forward  y[p, co]  = sum_{t, c} x[p + off(t), c] w[co, t, c]          (M = pixels, N = Co, K = 9 C)
//   data     dx[p, c]  = sum_{t, co} dy[p - off(t), co] w[co, t, c]       (M = pixels, N = C,  K = 9 Co)
//   weight   dw[co, t, c] = sum_p dy[p, co] x[p + off(t), c]              (M = Co, N = 9 C, K = pixels)
//
// The forward and data passes share one kernel: A gathers 8-channel groups of
// an NHWC tensor at the tap-shifted pixel (sign +1 forward, -1 data), B is a
// K-contiguous (N, K) matrix (the weights, or their per-tap transpose for the
// data pass).  Tiles: 128 pixels x 64 outputs x 32 K, 8 warps of 32 x 32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace sweep {
namespace conv {

constexpr int BM = 128, BN = 64, BK = 32, PADK = 8, NT = 256;

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

struct Shape {
    int N, H, W;        // images, height, width
    int C;              // channels of the gathered tensor (multiple of 8)
    int Nout;           // output channels
    int sign;           // +1 forward (p + off), -1 data gradient (p - off)
};

// out[p, n] = sum_k A[p, k] B[n, k] (+ bias[n]);  A gathered from act.
__global__ void __launch_bounds__(NT) gather_gemm(const __nv_bfloat16* __restrict__ act,
                                                  const __nv_bfloat16* __restrict__ Bt,
                                                  const float* __restrict__ bias, float* __restrict__ out, Shape S)
{
    __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PADK];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PADK];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
    const long long P = (long long)S.N * S.H * S.W;
    const long long p0 = (long long)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int K = 9 * S.C;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    for (int k0 = 0; k0 < K; k0 += BK) {
        // A: 128 rows x 4 groups of 8 channels, two groups per thread
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int id = tid + u * NT;
            const int r = id >> 2, gk = (id & 3) * 8;
            const long long p = p0 + r;
            const int k = k0 + gk;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < P && k < K) {
                const int t = k / S.C, c = k - t * S.C;
                const int dy = t / 3 - 1, dx = t % 3 - 1;
                const int img = (int)(p / ((long long)S.H * S.W));
                const int rem = (int)(p - (long long)img * S.H * S.W);
                const int h = rem / S.W + S.sign * dy, w = rem % S.W + S.sign * dx;
                if (h >= 0 && h < S.H && w >= 0 && w < S.W)
                    v = *reinterpret_cast<const uint4*>(act + (((long long)img * S.H + h) * S.W + w) * S.C + c);
            }
            *reinterpret_cast<uint4*>(&As[r][gk]) = v;
        }
        // B: 64 rows x 4 groups
        {
            const int r = tid >> 2, gk = (tid & 3) * 8;
            const int n = n0 + r, k = k0 + gk;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (n < S.Nout && k < K) v = *reinterpret_cast<const uint4*>(Bt + (long long)n * K + k);
            *reinterpret_cast<uint4*>(&Bs[r][gk]) = v;
        }
        __syncthreads();
        const int g = lane >> 2, q = lane & 3;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + g;
                a[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * q]);
                a[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * q]);
                a[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * q + 8]);
                a[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * q + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn + j * 8 + g;
                b[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * q]);
                b[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * q + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long long p = p0 + wm + i * 16 + g + 8 * h;
                const int n = n0 + wn + j * 8 + 2 * q;
                if (p >= P) continue;
                float* o = out + p * S.Nout + n;
                if (n < S.Nout) o[0] = acc[i][j][2 * h] + (bias ? bias[n] : 0.f);
                if (n + 1 < S.Nout) o[1] = acc[i][j][2 * h + 1] + (bias ? bias[n + 1] : 0.f);
            }
}

// dw[co, k] += sum over this CTA's pixel range of dy[p, co] * X[p, k], where
// X[p, k = t C + c] = x[p + off(t), c].  M = Co (64 per CTA), N = 9 C (64 per
// CTA), K = pixels (split over blockIdx.z, partial sums added atomically).
__global__ void __launch_bounds__(NT) weight_grad(const __nv_bfloat16* __restrict__ x,
                                                  const __nv_bfloat16* __restrict__ dy, float* __restrict__ dw,
                                                  int Nimg, int H, int W, int C, int Co, int pix_per_split)
{
    constexpr int WM = 64;
    __shared__ __align__(16) __nv_bfloat16 As[WM][BK + PADK];   // [co][pixel]
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PADK];   // [k][pixel]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;       // 8 warps: 2 (M) x 4 (N) of 32 x 16
    const long long P = (long long)Nimg * H * W;
    const int co0 = blockIdx.x * WM, kb0 = blockIdx.y * BN;
    const int K = 9 * C;
    const long long pbeg = (long long)blockIdx.z * pix_per_split;
    const long long pend = min(P, pbeg + pix_per_split);
    float acc[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
    for (long long pp = pbeg; pp < pend; pp += BK) {
        // A^T: dy[pp + r, co0 .. co0+63] -> As[co][r]; 32 pixels x 8 groups = 256 units
        {
            const int r = tid >> 3, gc = (tid & 7) * 8;
            const long long p = pp + r;
            const int co = co0 + gc;
            __nv_bfloat16 v[8];
            if (p < pend && co < Co) {
                const uint4 u = *reinterpret_cast<const uint4*>(dy + p * Co + co);
                memcpy(v, &u, 16);
            } else {
#pragma unroll
                for (int e = 0; e < 8; ++e) v[e] = __float2bfloat16(0.f);
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) As[gc + e][r] = v[e];
        }
        // B^T: X[pp + r, kb0 .. kb0+63] -> Bs[k][r]
        {
            const int r = tid >> 3, gk = (tid & 7) * 8;
            const long long p = pp + r;
            const int k = kb0 + gk;
            __nv_bfloat16 v[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) v[e] = __float2bfloat16(0.f);
            if (p < pend && k < K) {
                const int t = k / C, c = k - t * C;
                const int ddy = t / 3 - 1, ddx = t % 3 - 1;
                const int img = (int)(p / ((long long)H * W));
                const int rem = (int)(p - (long long)img * H * W);
                const int h = rem / W + ddy, w = rem % W + ddx;
                if (h >= 0 && h < H && w >= 0 && w < W) {
                    const uint4 u = *reinterpret_cast<const uint4*>(x + (((long long)img * H + h) * W + w) * C + c);
                    memcpy(v, &u, 16);
                }
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) Bs[gk + e][r] = v[e];
        }
        __syncthreads();
        const int g = lane >> 2, q = lane & 3;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t a[2][4], b[2][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + g;
                a[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * q]);
                a[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * q]);
                a[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * q + 8]);
                a[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * q + 8]);
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int c = wn + j * 8 + g;
                b[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * q]);
                b[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * q + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) mma_bf16(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int co = co0 + wm + i * 16 + g + 8 * h;
                const int k = kb0 + wn + j * 8 + 2 * q;
                if (co >= Co) continue;
                if (k < K) atomicAdd(dw + (long long)co * K + k, acc[i][j][2 * h]);
                if (k + 1 < K) atomicAdd(dw + (long long)co * K + k + 1, acc[i][j][2 * h + 1]);
            }
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
        conv::Shape S{n, h, w, c, nout, sign};
        const long long P = (long long)n * h * w;
        const dim3 grid((unsigned)((P + conv::BM - 1) / conv::BM), (unsigned)((nout + conv::BN - 1) / conv::BN));
        conv::gather_gemm<<<grid, conv::NT, 0, static_cast<cudaStream_t>(stream)>>>(
            static_cast<const __nv_bfloat16*>(act), static_cast<const __nv_bfloat16*>(bt), bias, out, S);
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
        const unsigned gx = (unsigned)((co + 63) / 64), gy = (unsigned)((K + conv::BN - 1) / conv::BN);
        // pixel splits: about four CTAs per SM in all, each split a multiple of 32 pixels
        long long splits = std::max(1LL, (4LL * 148) / ((long long)gx * gy));
        long long per = (P + splits - 1) / splits;
        per = (per + 31) / 32 * 32;
        splits = (P + per - 1) / per;
        const dim3 grid(gx, gy, (unsigned)splits);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        SWEEP_CUDA(cudaMemsetAsync(dw, 0, sizeof(float) * (size_t)co * K, st));
        conv::weight_grad<<<grid, conv::NT, 0, st>>>(static_cast<const __nv_bfloat16*>(x),
                                                     static_cast<const __nv_bfloat16*>(dy), dw, n, h, w, c, co, (int)per);
        SWEEP_LAUNCH_CHECK();
    });
}
