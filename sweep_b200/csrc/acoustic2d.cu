// acoustic2d.cu -- 2-D constant-density acoustic propagation on B200 (sm_100a):
// 8th-order-in-space / 2nd-order-in-time leapfrog with CPML, a fused forward
// step and a fused reverse step (exact adjoint + boundary-saving
// reconstruction + vp imaging), both tiled over shared memory and batched over
// shots.
//
// Numerics follow the reference's compiled path (impl='c'):
//   forward step       reference src/sweep/csrc/cuda/equations/acoustic2d/forward_split.cu:40-168
//   adjoint step       reference .../acoustic2d/adjoint_split.cu:27-196
//   reconstruction     reference .../acoustic2d/kernels.cuh:474-528
//   strip imaging      reference .../acoustic2d/kernels.cu:83-131
//   step order         reference src/sweep/csrc/cuda/common/eq_driver.cuh:377-434, 814-880,
//                      .../acoustic2d/driver_traits.cuh:529-635
// with the same expression trees (difference-form Laplacian with __fsub_rn
// taps, fused d(a psi) tap form, the adjoint's transposed CPML terms).
//
// Layout and schedule (the B200 part):
//   * one CTA = one 64x32 (x, z) tile for a group of G shots; the tile of the
//     stencil input plus its 4-cell halo is staged once per shot in shared
//     memory and every tap is read from there;
//   * with a shared model the velocity tile is staged once per CTA for all G
//     shots, and the gradient of the G shots is summed in registers and
//     flushed once per step into a Kahan-compensated per-group accumulator;
//   * point sources, receivers and boundary strips are handled by the CTA
//     that owns the cell, in the same launch as the stencil (no separate
//     injection / gather / strip kernels);
//   * one launch per forward step and one per reverse step.
#include "common.cuh"

namespace sweep {
namespace a2d {

constexpr int M = 4;                 // stencil half-width (order 8)
constexpr int TX = 64, TZ = 32;      // tile
constexpr int NTH = 256;             // threads per CTA (8 warps)
constexpr int SW = TX + 2 * M;       // staged tile width (with halo)
constexpr int SH = TZ + 2 * M;       // staged tile height
constexpr int SN = SW * SH;
constexpr int RPW = TZ / 8;          // rows per warp
constexpr int CPT = 2 * RPW;         // cells per thread

struct Params {
    int B, nz, nx, nt, nsrc, nrec;
    int ntx, ntz, G, per_shot;
    float dt, dz, dx;
    float lc[M + 1], gc[M + 1];
    int z0, z1, x0, x1;              // physical box (runtime grid)
    int bz_lo, bz_hi, bx_lo, bx_hi;  // forward CPML compute band: iz < bz_lo || iz >= bz_hi
    int pz0, pz1, px0, px1;          // adjoint pure interior box
    int rz0, rz1, rx0, rx1;          // reconstruction box (= physical box minus strips)
    int wzl, wzh, wxl, wxh;          // strip widths
    int n_top, n_bot, n_left, nstrip;
    const float *az, *bz, *dbz, *ax, *bx, *dbx;
    const float* vp;
    long long vp_stride;
    const float* wavelet;
    EventTable src, rec;
};

struct FwdPtrs {
    const float* u_prev; const float* u_now; float* u_next;
    const float* psix; const float* psiz; float* psixn; float* psizn;
    float* zetax; float* zetaz;
    float* record;                   // (B, nt, nrec)
    float* strips;                   // this step's strip slot (B, nstrip) or null
};

struct RevPtrs {
    const float* l_prev; const float* l_now; float* l_next;
    const float *apx, *apz, *azx, *azz;   // adjoint CPML memories (read)
    float *apx_o, *apz_o, *azx_o, *azz_o; // adjoint CPML memories (written)
    const float* r_prev; const float* r_now; float* r_next;
    const float* strips;             // saved U[it-1] strips (B, nstrip) or null
    const float* adj;                // (B, nt, nrec)
    float* grad_w;                   // (B, nsrc, nt) or null
    float* gacc; float* gcomp;       // Kahan accumulator slots (nslot, cells)
    float* illum_s; float* illum_r;  // (nslot, cells) or null
};

// ------------------------------------------------------------------ device
__device__ __forceinline__ float tap(float uk, float u0) { return __fsub_rn(uk, u0); }

// Stage a (SH x SW) window of field g (one shot, nz x nx) whose (0,0) is the
// runtime cell (tz0 - M, tx0 - M); cells off the grid read 0.
__device__ __forceinline__ void stage(float* s, const float* __restrict__ g, int nz, int nx,
                                      int tz0, int tx0)
{
    for (int i = threadIdx.x; i < SN; i += NTH) {
        const int r = i / SW, c = i - r * SW;
        const int iz = tz0 - M + r, ix = tx0 - M + c;
        s[i] = (iz >= 0 && iz < nz && ix >= 0 && ix < nx) ? __ldg(g + (long long)iz * nx + ix) : 0.f;
    }
}

// Difference-form Laplacian along the axis of stride `st` (1: x, SW: z) at the
// staged centre p (reference operators/laplace.cuh:327-380; minus tap first).
__device__ __forceinline__ float lap_s(const float* p, int st, const Params& P, float h)
{
    const float u0 = p[0];
    float acc = P.lc[1] * (tap(p[-st], u0) + tap(p[st], u0));
    acc = acc + P.lc[2] * (tap(p[-2 * st], u0) + tap(p[2 * st], u0));
    acc = acc + P.lc[3] * (tap(p[-3 * st], u0) + tap(p[3 * st], u0));
    acc = acc + P.lc[4] * (tap(p[-4 * st], u0) + tap(p[4 * st], u0));
    return acc / (h * h);
}

// Centred first derivative at the staged centre (reference operators/gradient.cuh:49-88).
__device__ __forceinline__ float grad_s(const float* p, int st, const Params& P, float h)
{
    float acc = P.gc[1] * (p[st] - p[-st]);
    acc = acc + P.gc[2] * (p[2 * st] - p[-2 * st]);
    acc = acc + P.gc[3] * (p[3 * st] - p[-3 * st]);
    acc = acc + P.gc[4] * (p[4 * st] - p[-4 * st]);
    return acc / h;
}

// Fused d(a psi)/d axis in tap form (reference acoustic2d/kernels.cuh:30-77):
// profile a at axis index ia, psi read from global memory at linear index i.
__device__ __forceinline__ float grad_apsi(const float* __restrict__ a, int ia,
                                           const float* __restrict__ psi, long long i, long long st,
                                           const Params& P, float h)
{
    float acc = P.gc[1] * (__ldg(a + ia + 1) * __ldg(psi + i + st) - __ldg(a + ia - 1) * __ldg(psi + i - st));
    acc = acc + P.gc[2] * (__ldg(a + ia + 2) * __ldg(psi + i + 2 * st) - __ldg(a + ia - 2) * __ldg(psi + i - 2 * st));
    acc = acc + P.gc[3] * (__ldg(a + ia + 3) * __ldg(psi + i + 3 * st) - __ldg(a + ia - 3) * __ldg(psi + i - 3 * st));
    acc = acc + P.gc[4] * (__ldg(a + ia + 4) * __ldg(psi + i + 4 * st) - __ldg(a + ia - 4) * __ldg(psi + i - 4 * st));
    return acc / h;
}

// Index of (iz, ix) in the boundary-saving strip set (top rows, bottom rows,
// left columns, right columns: reference acoustic2d/kernels.cu:95-107), or -1.
__device__ __forceinline__ int strip_index(const Params& P, int iz, int ix)
{
    if (iz < P.z0 || iz >= P.z1 || ix < P.x0 || ix >= P.x1) return -1;
    const int bw = P.x1 - P.x0, zi0 = P.z0 + P.wzl, zi1 = P.z1 - P.wzh;
    if (iz < zi0) return (iz - P.z0) * bw + (ix - P.x0);
    if (iz >= zi1) return P.n_top + (iz - zi1) * bw + (ix - P.x0);
    if (ix < P.x0 + P.wxl) return P.n_top + P.n_bot + (iz - zi0) * P.wxl + (ix - P.x0);
    if (ix >= P.x1 - P.wxh)
        return P.n_top + P.n_bot + P.n_left + (iz - zi0) * P.wxh + (ix - (P.x1 - P.wxh));
    return -1;
}

__device__ __forceinline__ bool computed(const Params& P, int iz, int ix)
{
    return iz >= M && iz < P.nz - M && ix >= M && ix < P.nx - M;
}

// ----------------------------------------------------------- forward step
// u_next = 2 u - u_prev + vp^2 dt^2 (Lap u + CPML terms) on [M, n-M)^2, then
// (same launch) strip save of u_now, source injection into u_next and receiver
// gather from u_next -- the per-step order of the reference's forward loop.
__global__ void __launch_bounds__(NTH) fwd_kernel(const Params P, const FwdPtrs F, const int it)
{
    extern __shared__ float smem[];
    float* s_u = smem;               // SN
    float* s_o = smem + SN;          // TZ * TX staging of u_next (event tiles)
    const int tx0 = blockIdx.x * TX, tz0 = blockIdx.y * TZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long N = (long long)P.nz * P.nx;
    const int tile = blockIdx.y * P.ntx + blockIdx.x;
    const int ntiles = P.ntx * P.ntz;
    const bool band = tx0 < P.bx_lo || tx0 + TX > P.bx_hi || tz0 < P.bz_lo || tz0 + TZ > P.bz_hi;
    const bool strip_tile = F.strips != nullptr &&
        tx0 < P.x1 && tx0 + TX > P.x0 && tz0 < P.z1 && tz0 + TZ > P.z0 &&
        !(tx0 >= P.x0 + P.wxl && tx0 + TX <= P.x1 - P.wxh &&
          tz0 >= P.z0 + P.wzl && tz0 + TZ <= P.z1 - P.wzh);

    for (int g = 0; g < P.G; ++g) {
        const int b = blockIdx.z * P.G + g;
        if (b >= P.B) break;
        const float* un = F.u_now + b * N;
        const float* vp = P.vp + b * P.vp_stride;
        __syncthreads();
        stage(s_u, un, P.nz, P.nx, tz0, tx0);
        __syncthreads();

        float out[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
            const int iz = tz0 + r, ix = tx0 + c;
            out[k] = 0.f;
            if (!computed(P, iz, ix)) continue;
            const long long i = (long long)iz * P.nx + ix;
            const float* p = s_u + (r + M) * SW + (c + M);
            const float lx = lap_s(p, 1, P, P.dx);
            const float lz = lap_s(p, SW, P, P.dz);
            const float v = __ldg(vp + i);
            const float v2dt2 = ((v * v) * P.dt) * P.dt;
            float w;
            const bool cx = ix < P.bx_lo || ix >= P.bx_hi;
            const bool cz = iz < P.bz_lo || iz >= P.bz_hi;
            if (!band || (!cx && !cz)) {
                w = lx + lz;
            } else {
                w = 0.f;
                if (cx) {
                    const float a = __ldg(P.ax + ix), bb = __ldg(P.bx + ix), db = __ldg(P.dbx + ix);
                    const float du = grad_s(p, 1, P, P.dx);
                    const float* psx = F.psix + b * N;
                    const float dap = grad_apsi(P.ax, ix, psx, i, 1, P, P.dx);
                    const float tmp = ((1.0f + bb) * lx + db * du) + dap;
                    float* zx = F.zetax + b * N;
                    const float z = zx[i];
                    w += (1.0f + bb) * tmp + a * z;
                    F.psixn[b * N + i] = bb * du + a * __ldg(psx + i);
                    zx[i] = bb * tmp + a * z;
                } else {
                    w += lx;
                }
                if (cz) {
                    const float a = __ldg(P.az + iz), bb = __ldg(P.bz + iz), db = __ldg(P.dbz + iz);
                    const float du = grad_s(p, SW, P, P.dz);
                    const float* psz = F.psiz + b * N;
                    const float dap = grad_apsi(P.az, iz, psz, i, P.nx, P, P.dz);
                    const float tmp = ((1.0f + bb) * lz + db * du) + dap;
                    float* zz = F.zetaz + b * N;
                    const float z = zz[i];
                    w += (1.0f + bb) * tmp + a * z;
                    F.psizn[b * N + i] = bb * du + a * __ldg(psz + i);
                    zz[i] = bb * tmp + a * z;
                } else {
                    w += lz;
                }
            }
            out[k] = 2.0f * p[0] - __ldg(F.u_prev + b * N + i) + v2dt2 * w;
            if (strip_tile) {
                const int si = strip_index(P, iz, ix);
                if (si >= 0) F.strips[(long long)b * P.nstrip + si] = p[0];
            }
        }

        // point sources and receivers of this (shot, tile)
        const int key = b * ntiles + tile;
        const int s_beg = P.src.off[key], s_end = P.src.off[key + 1];
        const int r_beg = P.rec.off[key], r_end = P.rec.off[key + 1];
        if (s_beg != s_end || r_beg != r_end) {
#pragma unroll
            for (int k = 0; k < CPT; ++k)
                s_o[(warp + 8 * (k >> 1)) * TX + lane + 32 * (k & 1)] = out[k];
            __syncthreads();
            for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                const int2 ev = P.src.ev[e];
                atomicAdd(s_o + ev.x, __ldg(P.wavelet + (long long)ev.y * P.nt + it));
            }
            __syncthreads();
            for (int e = r_beg + threadIdx.x; e < r_end; e += NTH) {
                const int2 ev = P.rec.ev[e];
                const int rb = ev.y / P.nrec, rr = ev.y - rb * P.nrec;
                F.record[((long long)rb * P.nt + it) * P.nrec + rr] = s_o[ev.x];
            }
#pragma unroll
            for (int k = 0; k < CPT; ++k)
                out[k] = s_o[(warp + 8 * (k >> 1)) * TX + lane + 32 * (k & 1)];
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
            const int iz = tz0 + r, ix = tx0 + c;
            if (computed(P, iz, ix)) F.u_next[b * N + (long long)iz * P.nx + ix] = out[k];
        }
    }
}

// ------------------------------------------------------------ reverse step
// One launch per reverse step `it` of the boundary-saving backward:
//   lambda_next = exact adjoint step of lambda (CPML transposed in the ring),
//   + record cotangent at the receivers               (-> lambda(it))
//   wavelet gradient  g_w[b, s, it] = lambda(it) at the sources
//   when it > 0: u(it-1) rebuilt in the reconstruction box, restored from the
//   saved strips elsewhere in the physical box, and the vp image
//   2 dt^2 u_tt lambda(it) / vp accumulated, u_tt = (u(it-1) - s(it) - 2 u(it) + u(it+1)) / dt^2;
//   then the source added back.
__global__ void __launch_bounds__(NTH) rev_kernel(const Params P, const RevPtrs R, const int it,
                                                   const int do_recon)
{
    extern __shared__ float smem[];
    float* s_l = smem;               // lambda(it+1) tile + halo
    float* s_c = smem + SN;          // vp^2 dt^2 tile + halo
    float* s_r = smem + 2 * SN;      // u(it) tile + halo (reconstruction)
    float* s_lo = smem + 3 * SN;     // staging (event tiles)
    float* s_ro = s_lo + TZ * TX;
    const int tx0 = blockIdx.x * TX, tz0 = blockIdx.y * TZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long N = (long long)P.nz * P.nx;
    const int tile = blockIdx.y * P.ntx + blockIdx.x;
    const int ntiles = P.ntx * P.ntz;
    const float dt2 = P.dt * P.dt;
    const float invdx2 = 1.0f / (P.dx * P.dx), invdz2 = 1.0f / (P.dz * P.dz);
    const float invdx = 1.0f / P.dx, invdz = 1.0f / P.dz;
    const bool ring = tx0 < P.px0 || tx0 + TX > P.px1 || tz0 < P.pz0 || tz0 + TZ > P.pz1;
    const bool phys_any = tx0 < P.x1 && tx0 + TX > P.x0 && tz0 < P.z1 && tz0 + TZ > P.z0;
    const bool phys_tile = do_recon && phys_any;
    const bool recon_tile = phys_tile && tx0 < P.rx1 && tx0 + TX > P.rx0 && tz0 < P.rz1 && tz0 + TZ > P.rz0;

    float gsum[CPT], isum_s[CPT], isum_r[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) { gsum[k] = 0.f; isum_s[k] = 0.f; isum_r[k] = 0.f; }
    bool staged_c = false;

    for (int g = 0; g < P.G; ++g) {
        const int b = blockIdx.z * P.G + g;
        if (b >= P.B) break;
        const long long bo = b * N;
        const float* vp = P.vp + b * P.vp_stride;
        __syncthreads();
        if (!staged_c) {
            // vp^2 dt^2 with halo (GW_AT of reference acoustic2d/kernels.cuh:370)
            for (int i = threadIdx.x; i < SN; i += NTH) {
                const int r = i / SW, c = i - r * SW;
                const int iz = tz0 - M + r, ix = tx0 - M + c;
                float v = 0.f;
                if (iz >= 0 && iz < P.nz && ix >= 0 && ix < P.nx) v = __ldg(vp + (long long)iz * P.nx + ix);
                s_c[i] = (v * v) * dt2;
            }
            staged_c = !P.per_shot;
        }
        stage(s_l, R.l_now + bo, P.nz, P.nx, tz0, tx0);
        if (recon_tile) stage(s_r, R.r_now + bo, P.nz, P.nx, tz0, tx0);
        __syncthreads();

        float lo[CPT], ro[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
            const int iz = tz0 + r, ix = tx0 + c;
            lo[k] = 0.f; ro[k] = 0.f;
            if (!computed(P, iz, ix)) continue;
            const long long i = (long long)iz * P.nx + ix;
            const int sc = (r + M) * SW + (c + M);
            const float* pl = s_l + sc;
            const float* pc = s_c + sc;
            const float gun = pl[0];
            const float gw = pc[0] * gun;
            const bool pure = !ring || (ix >= P.px0 && ix < P.px1 && iz >= P.pz0 && iz < P.pz1);
            if (pure) {
                float lapx = 0.0f, lapz = 0.0f;
#pragma unroll
                for (int kk = 1; kk <= M; ++kk) {
                    lapx += P.lc[kk] * (tap(pc[kk] * pl[kk], gw) + tap(pc[-kk] * pl[-kk], gw));
                    lapz += P.lc[kk] * (tap(pc[kk * SW] * pl[kk * SW], gw) + tap(pc[-kk * SW] * pl[-kk * SW], gw));
                }
                lo[k] = 2.0f * gun - __ldg(R.l_prev + bo + i) + lapx * invdx2 + lapz * invdz2;
            } else {
                const float ax_ = __ldg(P.ax + ix), az_ = __ldg(P.az + iz);
                const float bx_ = __ldg(P.bx + ix), bz_ = __ldg(P.bz + iz);
                const float* zx = R.azx + bo;
                const float* zz = R.azz + bo;
                const float* px = R.apx + bo;
                const float* pz = R.apz + bo;
                const float zx0 = __ldg(zx + i), zz0 = __ldg(zz + i);
                const float gtx0 = bx_ * zx0 + (1.0f + bx_) * gw;
                const float gtz0 = bz_ * zz0 + (1.0f + bz_) * gw;
                const float lx0 = (1.0f + bx_) * gtx0;
                float Lx = 0.0f, Dgx = 0.0f, Dqx = 0.0f;
#pragma unroll
                for (int kk = 1; kk <= M; ++kk) {
                    const int cp = ix + kk, cm = ix - kk;
                    const float bp = __ldg(P.bx + cp), bm = __ldg(P.bx + cm);
                    const float tp = bp * __ldg(zx + i + kk) + ((1.0f + bp) * pc[kk]) * pl[kk];
                    const float tm = bm * __ldg(zx + i - kk) + ((1.0f + bm) * pc[-kk]) * pl[-kk];
                    Lx += P.lc[kk] * (tap((1.0f + bp) * tp, lx0) + tap((1.0f + bm) * tm, lx0));
                    Dgx += P.gc[kk] * ((bp * __ldg(px + i + kk) + __ldg(P.dbx + cp) * tp)
                                     - (bm * __ldg(px + i - kk) + __ldg(P.dbx + cm) * tm));
                    Dqx += P.gc[kk] * (tp - tm);
                }
                Lx *= invdx2; Dgx *= invdx; Dqx *= invdx;
                const float lz0 = (1.0f + bz_) * gtz0;
                float Lz = 0.0f, Dgz = 0.0f, Dqz = 0.0f;
#pragma unroll
                for (int kk = 1; kk <= M; ++kk) {
                    const int cp = iz + kk, cm = iz - kk;
                    const long long o = (long long)kk * P.nx;
                    const float bp = __ldg(P.bz + cp), bm = __ldg(P.bz + cm);
                    const float tp = bp * __ldg(zz + i + o) + ((1.0f + bp) * pc[kk * SW]) * pl[kk * SW];
                    const float tm = bm * __ldg(zz + i - o) + ((1.0f + bm) * pc[-kk * SW]) * pl[-kk * SW];
                    Lz += P.lc[kk] * (tap((1.0f + bp) * tp, lz0) + tap((1.0f + bm) * tm, lz0));
                    Dgz += P.gc[kk] * ((bp * __ldg(pz + i + o) + __ldg(P.dbz + cp) * tp)
                                     - (bm * __ldg(pz + i - o) + __ldg(P.dbz + cm) * tm));
                    Dqz += P.gc[kk] * (tp - tm);
                }
                Lz *= invdz2; Dgz *= invdz; Dqz *= invdz;
                lo[k] = 2.0f * gun - __ldg(R.l_prev + bo + i) + (Lx + Lz - Dgx - Dgz);
                R.apx_o[bo + i] = ax_ * (__ldg(px + i) - Dqx);
                R.apz_o[bo + i] = az_ * (__ldg(pz + i) - Dqz);
                R.azx_o[bo + i] = ax_ * (zx0 + gw);
                R.azz_o[bo + i] = az_ * (zz0 + gw);
            }
            if (phys_tile && iz >= P.z0 && iz < P.z1 && ix >= P.x0 && ix < P.x1) {
                if (iz >= P.rz0 && iz < P.rz1 && ix >= P.rx0 && ix < P.rx1) {
                    const float* pr = s_r + sc;
                    const float v = __ldg(vp + i);
                    const float wsum = lap_s(pr, 1, P, P.dx) + lap_s(pr, SW, P, P.dz);
                    ro[k] = 2.0f * pr[0] - __ldg(R.r_prev + bo + i) + (v * v) * P.dt * P.dt * wsum;
                } else {
                    ro[k] = __ldg(R.strips + (long long)b * P.nstrip + strip_index(P, iz, ix));
                }
            }
        }

        const int key = b * ntiles + tile;
        const int s_beg = P.src.off[key], s_end = P.src.off[key + 1];
        const int r_beg = P.rec.off[key], r_end = P.rec.off[key + 1];
        const bool events = s_beg != s_end || r_beg != r_end;
        if (events) {
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int o = (warp + 8 * (k >> 1)) * TX + lane + 32 * (k & 1);
                s_lo[o] = lo[k]; s_ro[o] = ro[k];
            }
            __syncthreads();
            for (int e = r_beg + threadIdx.x; e < r_end; e += NTH) {
                const int2 ev = P.rec.ev[e];
                const int rb = ev.y / P.nrec, rr = ev.y - rb * P.nrec;
                atomicAdd(s_lo + ev.x, __ldg(R.adj + ((long long)rb * P.nt + it) * P.nrec + rr));
            }
            if (do_recon) {
                for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                    const int2 ev = P.src.ev[e];
                    const int iz = tz0 + ev.x / TX, ix = tx0 + ev.x % TX;
                    if (strip_index(P, iz, ix) >= 0)
                        atomicAdd(s_ro + ev.x, -__ldg(P.wavelet + (long long)ev.y * P.nt + it));
                }
            }
            __syncthreads();
            if (R.grad_w) {
                for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                    const int2 ev = P.src.ev[e];
                    R.grad_w[(long long)ev.y * P.nt + it] = s_lo[ev.x];
                }
            }
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int o = (warp + 8 * (k >> 1)) * TX + lane + 32 * (k & 1);
                lo[k] = s_lo[o]; ro[k] = s_ro[o];
            }
        }

        // imaging (physical box), illumination, stores
        float gl[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
            const int iz = tz0 + r, ix = tx0 + c;
            gl[k] = 0.f;
            if (!computed(P, iz, ix)) continue;
            const long long i = (long long)iz * P.nx + ix;
            R.l_next[bo + i] = lo[k];
            if (!(phys_any && iz >= P.z0 && iz < P.z1 && ix >= P.x0 && ix < P.x1)) continue;
            if (do_recon) {
                const float u0 = recon_tile ? s_r[(r + M) * SW + (c + M)] : __ldg(R.r_now + bo + i);
                const float up = __ldg(R.r_prev + bo + i);
                const float v = __ldg(vp + i);
                const float utt = (ro[k] - 2 * u0 + up) / dt2;
                gl[k] = 2.f * P.dt * P.dt * utt * lo[k] / v;
                if (R.illum_s) isum_s[k] += utt * utt;
            }
            if (R.illum_s) isum_r[k] += lo[k] * lo[k];
        }
        if (events && do_recon) {
            __syncthreads();
            for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                const int2 ev = P.src.ev[e];
                atomicAdd(s_ro + ev.x, __ldg(P.wavelet + (long long)ev.y * P.nt + it));
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < CPT; ++k)
                ro[k] = s_ro[(warp + 8 * (k >> 1)) * TX + lane + 32 * (k & 1)];
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
            const int iz = tz0 + r, ix = tx0 + c;
            if (phys_tile && iz >= P.z0 && iz < P.z1 && ix >= P.x0 && ix < P.x1)
                R.r_next[bo + (long long)iz * P.nx + ix] = ro[k];
            gsum[k] += gl[k];
        }
        if (P.per_shot && (do_recon || R.illum_s)) {
            // flush this shot into its own slot
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
                const int iz = tz0 + r, ix = tx0 + c;
                if (!(phys_any && iz >= P.z0 && iz < P.z1 && ix >= P.x0 && ix < P.x1)) continue;
                const long long o = bo + (long long)iz * P.nx + ix;
                const float y = gsum[k] - R.gcomp[o];
                const float t = R.gacc[o] + y;
                R.gcomp[o] = (t - R.gacc[o]) - y;
                R.gacc[o] = t;
                gsum[k] = 0.f;
                if (R.illum_s) {
                    R.illum_s[o] += isum_s[k]; R.illum_r[o] += isum_r[k];
                    isum_s[k] = 0.f; isum_r[k] = 0.f;
                }
            }
        }
    }
    if (!P.per_shot && phys_any && (do_recon || R.illum_s)) {
        const long long so = (long long)blockIdx.z * N;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = warp + 8 * (k >> 1), c = lane + 32 * (k & 1);
            const int iz = tz0 + r, ix = tx0 + c;
            if (!(iz >= P.z0 && iz < P.z1 && ix >= P.x0 && ix < P.x1)) continue;
            const long long o = so + (long long)iz * P.nx + ix;
            const float y = gsum[k] - R.gcomp[o];
            const float t = R.gacc[o] + y;
            R.gcomp[o] = (t - R.gacc[o]) - y;
            R.gacc[o] = t;
            if (R.illum_s) { R.illum_s[o] += isum_s[k]; R.illum_r[o] += isum_r[k]; }
        }
    }
}

// Sum the Kahan slots (value minus compensation) into the output gradient.
__global__ void finalize_kernel(const float* __restrict__ acc, const float* __restrict__ comp,
                                const float* __restrict__ is, const float* __restrict__ ir,
                                int nslot_in, int nout, long long N,
                                float* __restrict__ grad, float* __restrict__ ois, float* __restrict__ oir)
{
    const long long n = (long long)nout * N;
    const int per = nslot_in / nout;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = i / N, c = i - o * N;
        float s = 0.f, a = 0.f, bsum = 0.f;
        for (int k = 0; k < per; ++k) {
            const long long j = (o * per + k) * N + c;
            s += acc[j] - comp[j];
            if (is) { a += is[j]; bsum += ir[j]; }
        }
        grad[i] = s;
        if (ois) { ois[i] = a; oir[i] = bsum; }
    }
}

// ------------------------------------------------------------------- host
struct Plan {
    Params P;
    int nslot;            // gradient accumulator slots
    long long N;
    dim3 grid;
};

static void build_events(const Plan& pl, const std::vector<int32_t>& loc, int n, HostEvents& out)
{
    const Params& P = pl.P;
    const int ntiles = P.ntx * P.ntz;
    std::vector<int32_t> cnt((size_t)P.B * ntiles + 1, 0);
    std::vector<int> key(loc.size() / 2, -1);
    for (int b = 0; b < P.B; ++b)
        for (int s = 0; s < n; ++s) {
            const int e = b * n + s;
            const int ix = loc[2 * e], iz = loc[2 * e + 1];
            // cells of the outer stencil halo are never updated: treated as off-grid
            if (ix < M || ix >= P.nx - M || iz < M || iz >= P.nz - M) continue;
            key[e] = b * ntiles + (iz / TZ) * P.ntx + ix / TX;
            cnt[key[e] + 1]++;
        }
    for (size_t i = 1; i < cnt.size(); ++i) cnt[i] += cnt[i - 1];
    out.off = cnt;
    out.ev.assign(cnt.back(), make_int2(0, 0));
    std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
    for (int e = 0; e < (int)key.size(); ++e) {
        if (key[e] < 0) continue;
        const int ix = loc[2 * e], iz = loc[2 * e + 1];
        out.ev[fill[key[e]]++] = make_int2((iz % TZ) * TX + ix % TX, e);
    }
}

static Plan make_plan(const sweep_acoustic_desc* d)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->ndim == 2, "acoustic2d: ndim must be 2 (got %d)", d->ndim);
    SWEEP_REQUIRE(d->M == M, "acoustic2d: only spatial order 8 (M = 4) is built (got M = %d)", d->M);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1, "acoustic2d: B and nt must be >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "acoustic2d: negative source/receiver count");
    for (int f = 0; f < 4; ++f) {
        const int p = d->pad[f < 2 ? f : f + 2];
        SWEEP_REQUIRE(p >= 1, "acoustic2d: every face needs a PML pad >= 1 (face %d has %d)", f, p);
    }
    Plan pl{};
    Params& P = pl.P;
    P.B = d->B; P.nz = d->nz; P.nx = d->nx; P.nt = d->nt;
    P.nsrc = d->nsrc; P.nrec = d->nrec;
    const int pzl = d->pad[0], pzh = d->pad[1], pxl = d->pad[4], pxh = d->pad[5];
    P.z0 = pzl + M; P.z1 = d->nz - pzh - M;
    P.x0 = pxl + M; P.x1 = d->nx - pxh - M;
    SWEEP_REQUIRE(P.z1 - P.z0 >= 1 && P.x1 - P.x0 >= 1, "acoustic2d: empty physical box");
    P.dt = d->dt; P.dz = d->dz; P.dx = d->dx;
    for (int k = 0; k <= M; ++k) { P.lc[k] = d->lap[k]; P.gc[k] = d->grad[k]; }
    P.bz_lo = pzl + 2 * M; P.bz_hi = d->nz - pzh - 2 * M;
    P.bx_lo = pxl + 2 * M; P.bx_hi = d->nx - pxh - 2 * M;
    P.pz0 = pzl + 2 * M + 1; P.pz1 = d->nz - (pzh + 2 * M + 1);
    P.px0 = pxl + 2 * M + 1; P.px1 = d->nx - (pxh + 2 * M + 1);
    auto widths = [](int extent, int w, int& lo, int& hi) {
        lo = std::min(w, std::max(extent, 0));
        hi = std::min(w, std::max(extent - lo, 0));
    };
    const int w = M + 1;
    widths(P.z1 - P.z0, w, P.wzl, P.wzh);
    widths(P.x1 - P.x0, w, P.wxl, P.wxh);
    const int bw = P.x1 - P.x0, bh = std::max(0, (P.z1 - P.wzh) - (P.z0 + P.wzl));
    P.n_top = P.wzl * bw; P.n_bot = P.wzh * bw; P.n_left = P.wxl * bh;
    P.nstrip = P.n_top + P.n_bot + P.n_left + P.wxh * bh;
    P.rz0 = P.z0 + P.wzl; P.rz1 = P.z1 - P.wzh;
    P.rx0 = P.x0 + P.wxl; P.rx1 = P.x1 - P.wxh;
    P.az = d->az; P.bz = d->bz; P.dbz = d->dbz; P.ax = d->ax; P.bx = d->bx; P.dbx = d->dbx;
    P.vp = d->vp; P.vp_stride = d->vp_stride;
    P.per_shot = d->vp_stride != 0;
    P.wavelet = d->wavelet;
    P.ntx = (d->nx + TX - 1) / TX;
    P.ntz = (d->nz + TZ - 1) / TZ;
    const int ntiles = P.ntx * P.ntz;
    // shots per CTA: enough CTAs for ~4 waves over 148 SMs
    int G = (int)((long long)ntiles * P.B / (148LL * 4));
    G = std::max(1, std::min(G, 8));
    G = std::min(G, P.B);
    P.G = G;
    pl.N = (long long)d->nz * d->nx;
    const int ngroups = (P.B + G - 1) / G;
    pl.nslot = P.per_shot ? P.B : ngroups;
    pl.grid = dim3(P.ntx, P.ntz, ngroups);
    return pl;
}

struct FwdWork {
    float* u[3];
    float *psix, *psiz, *psixn, *psizn, *zetax, *zetaz;
    int32_t *src_off, *rec_off;
    int2 *src_ev, *rec_ev;
};

struct RevWork {
    float* l[3];
    float* aux[8];
    float* r[3];
    float *gacc, *gcomp, *is, *ir;
    int32_t *src_off, *rec_off;
    int2 *src_ev, *rec_ev;
};

static void carve_events(Carve& c, const Plan& pl, int32_t*& so, int32_t*& ro, int2*& se, int2*& re)
{
    const long long nkey = (long long)pl.P.B * pl.P.ntx * pl.P.ntz + 1;
    so = c.take<int32_t>(nkey);
    ro = c.take<int32_t>(nkey);
    se = c.take<int2>((long long)pl.P.B * std::max(pl.P.nsrc, 1));
    re = c.take<int2>((long long)pl.P.B * std::max(pl.P.nrec, 1));
}

static FwdWork carve_fwd(Carve& c, const Plan& pl)
{
    FwdWork w{};
    const long long n = (long long)pl.P.B * pl.N;
    for (auto& p : w.u) p = c.take<float>(n);
    w.psix = c.take<float>(n); w.psiz = c.take<float>(n);
    w.psixn = c.take<float>(n); w.psizn = c.take<float>(n);
    w.zetax = c.take<float>(n); w.zetaz = c.take<float>(n);
    carve_events(c, pl, w.src_off, w.rec_off, w.src_ev, w.rec_ev);
    return w;
}

static RevWork carve_rev(Carve& c, const Plan& pl, bool illum)
{
    RevWork w{};
    const long long n = (long long)pl.P.B * pl.N;
    for (auto& p : w.l) p = c.take<float>(n);
    for (auto& p : w.aux) p = c.take<float>(n);
    for (auto& p : w.r) p = c.take<float>(n);
    w.gacc = c.take<float>((long long)pl.nslot * pl.N);
    w.gcomp = c.take<float>((long long)pl.nslot * pl.N);
    if (illum) {
        w.is = c.take<float>((long long)pl.nslot * pl.N);
        w.ir = c.take<float>((long long)pl.nslot * pl.N);
    }
    carve_events(c, pl, w.src_off, w.rec_off, w.src_ev, w.rec_ev);
    return w;
}

static int64_t tape_bytes(const Plan& pl)
{
    Carve c(nullptr);
    c.take<float>((long long)pl.P.nt * pl.P.B * pl.P.nstrip);
    c.take<float>(2LL * pl.P.B * pl.N);
    return c.off;
}

static void upload_events(const sweep_acoustic_desc* d, Plan& pl, cudaStream_t st,
                          int32_t* so, int32_t* ro, int2* se, int2* re, HostEvents& hs, HostEvents& hr)
{
    const int B = d->B;
    std::vector<int32_t> sl((size_t)B * d->nsrc * 2), rl((size_t)B * d->nrec * 2);
    if (!sl.empty()) SWEEP_CUDA(cudaMemcpyAsync(sl.data(), d->src_loc, sl.size() * 4, cudaMemcpyDeviceToHost, st));
    if (!rl.empty()) SWEEP_CUDA(cudaMemcpyAsync(rl.data(), d->rec_loc, rl.size() * 4, cudaMemcpyDeviceToHost, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    build_events(pl, sl, d->nsrc, hs);
    build_events(pl, rl, d->nrec, hr);
    SWEEP_CUDA(cudaMemcpyAsync(so, hs.off.data(), hs.off.size() * 4, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemcpyAsync(ro, hr.off.data(), hr.off.size() * 4, cudaMemcpyHostToDevice, st));
    if (!hs.ev.empty()) SWEEP_CUDA(cudaMemcpyAsync(se, hs.ev.data(), hs.ev.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    if (!hr.ev.empty()) SWEEP_CUDA(cudaMemcpyAsync(re, hr.ev.data(), hr.ev.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    pl.P.src.off = so; pl.P.src.ev = se;
    pl.P.rec.off = ro; pl.P.rec.ev = re;
}

static size_t fwd_smem() { return (SN + TZ * TX) * sizeof(float); }
static size_t rev_smem() { return (3 * SN + 2 * TZ * TX) * sizeof(float); }

static void set_attrs()
{
    static bool done = false;
    if (done) return;
    SWEEP_CUDA(cudaFuncSetAttribute(fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem()));
    SWEEP_CUDA(cudaFuncSetAttribute(rev_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rev_smem()));
    done = true;
}

void sizes(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, int64_t* ws, int64_t* tape)
{
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY, "acoustic2d: only boundary saving is built for 2-D");
    (void)ckpt_every;
    Plan pl = make_plan(d);
    Carve cf(nullptr);
    carve_fwd(cf, pl);
    Carve cr(nullptr);
    carve_rev(cr, pl, true);
    *ws = std::max(cf.off, cr.off);
    *tape = tape_bytes(pl);
}

void forward(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape,
             void* ws, int64_t ws_bytes, cudaStream_t st)
{
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, ckpt_every, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic2d forward: workspace too small (%lld < %lld)",
                  (long long)ws_bytes, (long long)need_ws);
    SWEEP_REQUIRE(record != nullptr || d->nrec == 0, "acoustic2d forward: null record");
    set_attrs();
    Plan pl = make_plan(d);
    Carve c(ws);
    FwdWork w = carve_fwd(c, pl);
    HostEvents hs, hr;
    upload_events(d, pl, st, w.src_off, w.rec_off, w.src_ev, w.rec_ev, hs, hr);
    const long long n = (long long)pl.P.B * pl.N;
    for (auto* p : w.u) SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
    for (auto* p : {w.psix, w.psiz, w.psixn, w.psizn, w.zetax, w.zetaz})
        SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
    if (d->nrec > 0)
        SWEEP_CUDA(cudaMemsetAsync(record, 0, (size_t)d->B * d->nt * d->nrec * 4, st));
    float* strips = static_cast<float*>(tape);
    FwdPtrs F{};
    F.record = record;
    float *up = w.u[0], *un = w.u[1], *ux = w.u[2];
    float *px = w.psix, *pz = w.psiz, *pxn = w.psixn, *pzn = w.psizn;
    for (int it = 0; it < d->nt; ++it) {
        F.u_prev = up; F.u_now = un; F.u_next = ux;
        F.psix = px; F.psiz = pz; F.psixn = pxn; F.psizn = pzn;
        F.zetax = w.zetax; F.zetaz = w.zetaz;
        F.strips = strips ? strips + (long long)it * pl.P.B * pl.P.nstrip : nullptr;
        fwd_kernel<<<pl.grid, NTH, fwd_smem(), st>>>(pl.P, F, it);
        SWEEP_LAUNCH_CHECK();
        float* t = up; up = un; un = ux; ux = t;
        std::swap(px, pxn); std::swap(pz, pzn);
    }
    if (strips) {
        float* last = strips + (long long)d->nt * pl.P.B * pl.P.nstrip;
        // (U[nt-1], U[nt]) per shot
        SWEEP_CUDA(cudaMemcpyAsync(last, up, n * 4, cudaMemcpyDeviceToDevice, st));
        SWEEP_CUDA(cudaMemcpyAsync(last + n, un, n * 4, cudaMemcpyDeviceToDevice, st));
    }
}

void backward(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
              float* grad_vp, float* grad_w, float* illum_s, float* illum_r,
              void* ws, int64_t ws_bytes, cudaStream_t st)
{
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, ckpt_every, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic2d backward: workspace too small");
    SWEEP_REQUIRE(tape != nullptr, "acoustic2d backward: null tape");
    SWEEP_REQUIRE(grad_vp != nullptr, "acoustic2d backward: null grad_vp");
    SWEEP_REQUIRE((illum_s == nullptr) == (illum_r == nullptr), "acoustic2d backward: pass both illuminations or neither");
    set_attrs();
    Plan pl = make_plan(d);
    Carve c(ws);
    const bool illum = illum_s != nullptr;
    RevWork w = carve_rev(c, pl, illum);
    HostEvents hs, hr;
    upload_events(d, pl, st, w.src_off, w.rec_off, w.src_ev, w.rec_ev, hs, hr);
    const long long n = (long long)pl.P.B * pl.N;
    for (auto* p : w.l) SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
    for (auto* p : w.aux) SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
    SWEEP_CUDA(cudaMemsetAsync(w.r[2], 0, n * 4, st));
    SWEEP_CUDA(cudaMemsetAsync(w.gacc, 0, (size_t)pl.nslot * pl.N * 4, st));
    SWEEP_CUDA(cudaMemsetAsync(w.gcomp, 0, (size_t)pl.nslot * pl.N * 4, st));
    if (illum) {
        SWEEP_CUDA(cudaMemsetAsync(w.is, 0, (size_t)pl.nslot * pl.N * 4, st));
        SWEEP_CUDA(cudaMemsetAsync(w.ir, 0, (size_t)pl.nslot * pl.N * 4, st));
    }
    if (grad_w && d->nsrc > 0)
        SWEEP_CUDA(cudaMemsetAsync(grad_w, 0, (size_t)d->B * d->nsrc * d->nt * 4, st));
    const float* strips = static_cast<const float*>(tape);
    const float* last = strips + (long long)d->nt * pl.P.B * pl.P.nstrip;
    // seed: prev = U[nt], now = U[nt-1]  (reference driver_traits.cuh:493-505; the
    // rim outside the physical box is never read by the reconstruction)
    SWEEP_CUDA(cudaMemcpyAsync(w.r[0], last + n, n * 4, cudaMemcpyDeviceToDevice, st));
    SWEEP_CUDA(cudaMemcpyAsync(w.r[1], last, n * 4, cudaMemcpyDeviceToDevice, st));
    RevPtrs R{};
    R.adj = adj; R.grad_w = grad_w;
    R.gacc = w.gacc; R.gcomp = w.gcomp;
    R.illum_s = w.is; R.illum_r = w.ir;
    float *lp = w.l[0], *ln = w.l[1], *lx = w.l[2];
    float *rp = w.r[0], *rn = w.r[1], *rx = w.r[2];
    int cur = 0;
    for (int it = d->nt - 1; it >= 0; --it) {
        const int do_recon = it > 0 ? 1 : 0;
        R.l_prev = lp; R.l_now = ln; R.l_next = lx;
        R.apx = w.aux[0 + cur]; R.apz = w.aux[2 + cur]; R.azx = w.aux[4 + cur]; R.azz = w.aux[6 + cur];
        R.apx_o = w.aux[1 - cur]; R.apz_o = w.aux[3 - cur]; R.azx_o = w.aux[5 - cur]; R.azz_o = w.aux[7 - cur];
        R.r_prev = rp; R.r_now = rn; R.r_next = rx;
        R.strips = do_recon ? strips + (long long)(it - 1) * pl.P.B * pl.P.nstrip : nullptr;
        rev_kernel<<<pl.grid, NTH, rev_smem(), st>>>(pl.P, R, it, do_recon);
        SWEEP_LAUNCH_CHECK();
        float* t = lp; lp = ln; ln = lx; lx = t;
        cur = 1 - cur;
        if (do_recon) { t = rp; rp = rn; rn = rx; rx = t; }
    }
    const int nout = pl.P.per_shot ? d->B : 1;
    finalize_kernel<<<1184, 256, 0, st>>>(w.gacc, w.gcomp, w.is, w.ir, pl.nslot, nout, pl.N,
                                          grad_vp, illum_s, illum_r);
    SWEEP_LAUNCH_CHECK();
}

}  // namespace a2d
}  // namespace sweep
