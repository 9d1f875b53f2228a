// acoustic2d.cu -- 2-D constant-density acoustic propagation on B200 (sm_100a):
// 8th-order-in-space / 2nd-order-in-time leapfrog with CPML, a fused forward
// step and a fused reverse step (exact adjoint + boundary-saving
// reconstruction + vp imaging), both tiled over shared memory, fed by TMA and
// batched over shots.
//
// Numerics follow the reference's compiled path (impl='c'):
//   forward step       reference src/sweep/csrc/cuda/equations/acoustic2d/forward_split.cu:40-168
//   adjoint step       reference .../acoustic2d/adjoint_split.cu:27-196
//   reconstruction     reference .../acoustic2d/kernels.cuh:474-528
//   strip imaging      reference .../acoustic2d/kernels.cu:83-131
//   step order         reference src/sweep/csrc/cuda/common/eq_driver.cuh:377-434, 814-880,
//                      .../acoustic2d/driver_traits.cuh:529-635
// with the same expression trees (difference-form Laplacian with __fsub_rn
// taps, fused d(a psi) tap form, the adjoint's transposed CPML terms) in the
// reference CUDA core's arithmetic mode (flush-to-zero, fast division).
//
// Layout and schedule (the B200 part):
//   * every internal field is pitched: rows of P floats (P = nx rounded up to
//     32), so each row starts on a 128-byte line and TMA can address it;
//   * one CTA = one 64 x 32 (x, z) tile for a group of G shots; per shot, one
//     thread issues TMA tile loads (the stencil input with its 4-cell halo,
//     and the centre tiles) into shared memory, double-buffered across the
//     shot loop so the next shot's tiles are in flight while this one computes;
//   * the model enters as precomputed coefficient fields (vp^2 dt^2 in the two
//     roundings the reference uses, and vp itself), read once per CTA for a
//     shared model;
//   * the gradient of the G shots is summed in registers and flushed once per
//     step into a Kahan-compensated per-group accumulator;
//   * point sources, receivers and boundary strips are handled by the CTA that
//     owns the cell, in the same launch as the stencil;
//   * one launch per forward step and one per reverse step.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <functional>

#include "acoustic2d.cuh"
#include "tma.cuh"

namespace sweep {
namespace a2d {

constexpr int M = 4;                 // stencil half-width (order 8)
constexpr int TX = 64, TZ = 32;      // tile
constexpr int NTH = 256;             // threads per CTA (8 warps)
constexpr int SW = TX + 2 * M;       // staged tile width (with halo)
constexpr int SH = TZ + 2 * M;       // staged tile height
constexpr int SN = SW * SH;          // staged halo tile, floats
constexpr int TN = TX * TZ;          // centre tile, floats
constexpr int CPT = TN / NTH;        // cells per thread (8)
constexpr int kMaxG = 16;            // shots per CTA, at most

enum ErrCode { ERR_TMA_WAIT_FWD = 1, ERR_TMA_WAIT_REV = 2 };

// Boundary-strip storage of the boundary-saving tape.  fp32 and bf16 keep the
// strip set (each cell once, strip_index order); fp16 and int8 keep the
// reference's four faces (top and bottom rows across the box, left and right
// columns down the whole box, corners in two faces), each quantised per shot
// in blocks of kQB cells against the block's max |value|
// (reference boundarysaver.cu:906-1100).
enum StripFmt { SF_F32 = 0, SF_F16 = 1, SF_BF16 = 2, SF_I8 = 3 };
constexpr int kQB = 256;

struct StripStore {
    int fmt;                         // StripFmt
    int w;                           // face band width (M + 1)
    int cells[4], blocks[4];         // per shot and face (top, bottom, left, right): scaled formats
    long long pay[4], scl[4];        // byte offsets of each face's codes and scales in a step slot
    long long step;                  // bytes of one step slot
};

struct Params {
    int B, nz, nx, nt, nsrc, nrec;
    int P;                           // row pitch (floats)
    int ntx, ntz, G, per_shot;
    long long S;                     // shot stride (nz * P)
    long long ms;                    // model stride: 0 (shared) or S
    float dt, dz, dx;
    float lc[M + 1], gc[M + 1];
    int z0, z1, x0, x1;              // physical box (runtime grid)
    int bz_lo, bz_hi, bx_lo, bx_hi;  // forward CPML compute band: iz < bz_lo || iz >= bz_hi
    int pz0, pz1, px0, px1;          // adjoint pure interior box
    int rz0, rz1, rx0, rx1;          // reconstruction box (= physical box minus strips)
    int wzl, wzh, wxl, wxh;          // strip widths
    int n_top, n_bot, n_left, nstrip;
    const float *az, *bz, *dbz, *ax, *bx, *dbx;
    const float* cf;                 // ((v*v)*dt)*dt, pitched (forward / reconstruction)
    const float* vv;                 // v, pitched (imaging)
    const float* wavelet;
    EventTable src, rec;
    const int* order;                // tile slots, heaviest (CPML ring) tiles first
    int* err;
    StripStore st;
};

struct FwdMaps {
    CUtensorMap halo[3];             // the three wavefield buffers, (SW x SH) boxes
    CUtensorMap tile[3];             // the same buffers, (TX x TZ) boxes
};

struct RevMaps {
    CUtensorMap lh[3], lt[3];        // adjoint field buffers: halo / centre boxes
    CUtensorMap rh[3], rt[3];        // reconstruction buffers: halo / centre boxes
    CUtensorMap ch;                  // (v*v)*(dt*dt), halo box
    CUtensorMap am[8];               // adjoint CPML memories: x ones with an x halo, z ones with a z halo
};

struct FwdPtrs {
    float* u_next;
    const float* psix; const float* psiz; float* psixn; float* psizn;
    float* zetax; float* zetaz;
    float* record;                   // (B, nt, nrec)
    void* strips;                    // this step's strips (B, nstrip): float, or bf16 when sbf16; or null
    int sbf16;
    int now, prev;                   // buffer indices of u_now / u_prev
};

struct RevPtrs {
    float* l_next;
    const float *apx, *apz, *azx, *azz;   // adjoint CPML memories (read)
    float *apx_o, *apz_o, *azx_o, *azz_o; // adjoint CPML memories (written)
    float* r_next;
    const void* strips;              // step slot holding the strips of U[it-1] (format P.st), or null
    const float* adj;                // (B, nt, nrec)
    float* grad_w;                   // (B, nsrc, nt) or null
    float* gacc; float* gcomp;       // Kahan accumulator slots (nslot, S)
    float* illum_s; float* illum_r;  // (nslot, S) or null
    int lnow, lprev, rnow, rprev;    // buffer indices
    int cur;                         // CPML memories read this step: am[0 + cur], am[2 + cur], am[4 + cur], am[6 + cur]
};

// ------------------------------------------------------------------ device
__device__ __forceinline__ float tap(float uk, float u0) { return __fsub_rn(uk, u0); }

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
// profile a at axis index ia, psi read from global memory at offset i.
__device__ __forceinline__ float grad_apsi(const float* __restrict__ a, int ia,
                                           const float* __restrict__ psi, int i, int st,
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

// Face f (0 top, 1 bottom, 2 left, 3 right) cell `idx` of the scaled
// formats -> grid cell (reference boundarysaver.cu:72-112 face indexing:
// top / bottom (width, box width), left / right (box height, width)).
__device__ __forceinline__ void face_cell(const Params& P, int f, int idx, int& iz, int& ix)
{
    const int w = P.st.w, bw = P.x1 - P.x0;
    if (f < 2) {
        const int r = idx / bw;
        iz = (f == 0 ? P.z0 : P.z1 - w) + r;
        ix = P.x0 + (idx - r * bw);
    } else {
        const int r = idx / w;
        iz = P.z0 + r;
        ix = (f == 2 ? P.x0 : P.x1 - w) + (idx - r * w);
    }
}

// The face a scaled-format restore reads strip cell (iz, ix) from: the last of
// the faces holding it in the reference's restore order top, bottom, left,
// right (a corner cell takes its left or right face's value).
__device__ __forceinline__ int face_index(const Params& P, int iz, int ix, int& f)
{
    const int w = P.st.w, bw = P.x1 - P.x0;
    if (ix >= P.x1 - w) { f = 3; return (iz - P.z0) * w + (ix - (P.x1 - w)); }
    if (ix < P.x0 + w) { f = 2; return (iz - P.z0) * w + (ix - P.x0); }
    if (iz >= P.z1 - w) { f = 1; return (iz - (P.z1 - w)) * bw + (ix - P.x0); }
    f = 0;
    return (iz - P.z0) * bw + (ix - P.x0);
}

// Saved value of strip cell (iz, ix) of shot b from a step slot (dequantised
// as the reference does: fp16 code x scale; int8 (code - 128) x scale / 127).
__device__ __forceinline__ float strip_value(const Params& P, const void* slot, int b, int iz, int ix)
{
    const StripStore& S = P.st;
    if (S.fmt == SF_F32) return __ldg(static_cast<const float*>(slot) + (long long)b * P.nstrip + strip_index(P, iz, ix));
    if (S.fmt == SF_BF16)
        return __bfloat162float(static_cast<const __nv_bfloat16*>(slot)[(long long)b * P.nstrip + strip_index(P, iz, ix)]);
    int f;
    const int i = face_index(P, iz, ix, f);
    const char* base = static_cast<const char*>(slot);
    const float scale = reinterpret_cast<const float*>(base + S.scl[f])[(long long)b * S.blocks[f] + i / kQB];
    const long long e = (long long)b * S.cells[f] + i;
    if (S.fmt == SF_F16) return __half2float(reinterpret_cast<const __half*>(base + S.pay[f])[e]) * scale;
    const float s = scale * (1.0f / 127.0f);
    return ((float)reinterpret_cast<const uint8_t*>(base + S.pay[f])[e] - 128.0f) * s;
}

__device__ __forceinline__ bool computed(const Params& P, int iz, int ix)
{
    return iz >= M && iz < P.nz - M && ix >= M && ix < P.nx - M;
}


__device__ __forceinline__ int cell_r(int k) { return (threadIdx.x >> 5) + 8 * (k >> 1); }
__device__ __forceinline__ int cell_c(int k) { return (threadIdx.x & 31) + 32 * (k & 1); }

// Reverse-step cell ownership: thread t holds rows 4 (t / 32) .. + 3 and
// columns 2 (t % 32), + 1 of the tile -- cell k = 2 j + i is (row j, column i)
// of that block -- so the x and z stencil windows of its 8 cells are read
// once as float2 rows and shared between them.
__device__ __forceinline__ int rcell_r(int k) { return 4 * (threadIdx.x >> 5) + (k >> 1); }
__device__ __forceinline__ int rcell_c(int k) { return 2 * (threadIdx.x & 31) + (k & 1); }

__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ float2 ldg2(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ float comp(const float2 v, int e) { return e ? v.y : v.x; }

// Save u_now of this tile's boundary strips from its staged copy `now`
// (rows of SW floats, origin at (tz0 - M, tx0 - M)) into the strip set of one
// shot, `dst`: the four strip rectangles of strip_index, cut to the tile and
// walked by the whole CTA (rows of 8 or 64 slots, one cell per thread).
template <class T>
__device__ __forceinline__ void save_strips(const Params& P, const float* now, T* __restrict__ dst,
                                            int tx0, int tz0)
{
    const int bw = P.x1 - P.x0, zi0 = P.z0 + P.wzl, zi1 = P.z1 - P.wzh;
    auto rect = [&](int za, int zb, int xa, int xb, int base, int rw, int rz, int rx) {
        za = max(za, tz0); zb = min(zb, tz0 + TZ);
        xa = max(xa, tx0); xb = min(xb, tx0 + TX);
        if (za >= zb || xa >= xb) return;
        const int w = xb - xa;
        const int sh = w <= 8 ? 3 : 6;
        const int n = (zb - za) << sh;
        for (int e = threadIdx.x; e < n; e += NTH) {
            const int c = e & ((1 << sh) - 1);
            if (c >= w) continue;
            const int iz = za + (e >> sh), ix = xa + c;
            dst[base + (iz - rz) * rw + (ix - rx)] = static_cast<T>(now[(iz - tz0 + M) * SW + (ix - tx0 + M)]);
        }
    };
    rect(P.z0, zi0, P.x0, P.x1, 0, bw, P.z0, P.x0);
    rect(zi1, P.z1, P.x0, P.x1, P.n_top, bw, zi1, P.x0);
    rect(zi0, zi1, P.x0, P.x0 + P.wxl, P.n_top + P.n_bot, P.wxl, zi0, P.x0);
    rect(zi0, zi1, P.x1 - P.wxh, P.x1, P.n_top + P.n_bot + P.n_left, P.wxh, zi0, P.x1 - P.wxh);
}

// ----------------------------------------------------------- forward step
struct FwdSmem {
    float now[2][SN];
    float prev[2][TN];
    float out[TN];
    int4 evr[kMaxG];                 // per shot of the CTA: source and receiver event ranges
    uint64_t bar[2];
};

// u_next = 2 u - u_prev + vp^2 dt^2 (Lap u + CPML terms) on [M, n-M)^2, then
// (same launch) strip save of u_now, source injection into u_next and receiver
// gather from u_next -- the per-step order of the reference's forward loop.
__global__ void __launch_bounds__(NTH) fwd_kernel(const __grid_constant__ FwdMaps MP, const Params P,
                                                  const FwdPtrs F, const int it)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    FwdSmem& sm = *reinterpret_cast<FwdSmem*>(smem_raw);
    const int tile = P.order[blockIdx.y];
    const int tx0 = (tile % P.ntx) * TX, tz0 = (tile / P.ntx) * TZ;
    const int b0 = blockIdx.x * P.G;
    const int nloc = min(P.G, P.B - b0);
    const int ntiles = P.ntx * P.ntz;
    const bool band = tx0 < P.bx_lo || tx0 + TX > P.bx_hi || tz0 < P.bz_lo || tz0 + TZ > P.bz_hi;
    const bool full = tx0 >= M && tx0 + TX <= P.nx - M && tz0 >= M && tz0 + TZ <= P.nz - M;
    const bool strip_tile = F.strips != nullptr &&
        tx0 < P.x1 && tx0 + TX > P.x0 && tz0 < P.z1 && tz0 + TZ > P.z0 &&
        !(tx0 >= P.x0 + P.wxl && tx0 + TX <= P.x1 - P.wxh &&
          tz0 >= P.z0 + P.wzl && tz0 + TZ <= P.z1 - P.wzh);
    constexpr uint32_t kBytes = (SN + TN) * 4;

    if (threadIdx.x == 0) {
        tma::mbar_init(&sm.bar[0], 1);
        tma::mbar_init(&sm.bar[1], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    auto issue = [&](int s, int b) {
        tma::mbar_expect_tx(&sm.bar[s], kBytes);
        tma::load_3d(sm.now[s], &MP.halo[F.now], &sm.bar[s], tx0 - M, tz0 - M, b);
        tma::load_3d(sm.prev[s], &MP.tile[F.prev], &sm.bar[s], tx0, tz0, b);
    };
    if (threadIdx.x == 0) {
        issue(0, b0);
        if (nloc > 1) issue(1, b0 + 1);
    }
    if (threadIdx.x < nloc) {
        const int key = (b0 + threadIdx.x) * ntiles + tile;
        sm.evr[threadIdx.x] = make_int4(P.src.off[key], P.src.off[key + 1], P.rec.off[key], P.rec.off[key + 1]);
    }

    // model coefficients of this thread's cells (shared model: once per CTA)
    float cf[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int iz = tz0 + cell_r(k), ix = tx0 + cell_c(k);
        cf[k] = computed(P, iz, ix) ? __ldg(P.cf + b0 * P.ms + iz * P.P + ix) : 0.f;
    }

    __syncthreads();                     // the event ranges (sm.evr) are written
    // Each thread waits for shot g's tiles itself; a failed wait is noted and
    // the CTA leaves together at the barrier that ends the shot, after
    // thread 0 has waited (bounded) for the loads still in flight.
    bool bad = false;
    auto leave = [&](int g) {
        if (threadIdx.x == 0)
            for (int h = g; h < min(g + 2, nloc); ++h)
                tma::mbar_wait(&sm.bar[h & 1], (h >> 1) & 1, P.err, ERR_TMA_WAIT_FWD);
    };
    for (int g = 0; g < nloc; ++g) {
        const int b = b0 + g;
        const int s = g & 1;
        if (!tma::mbar_wait(&sm.bar[s], (g >> 1) & 1, P.err, ERR_TMA_WAIT_FWD)) bad = true;
        const float* now = sm.now[s];
        const float* prev = sm.prev[s];
        const long long bo = (long long)b * P.S;

        float out[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int r = cell_r(k), c = cell_c(k);
            const int iz = tz0 + r, ix = tx0 + c;
            out[k] = 0.f;
            if (!full && !computed(P, iz, ix)) continue;
            const float* p = now + (r + M) * SW + (c + M);
            const float lx = lap_s(p, 1, P, P.dx);
            const float lz = lap_s(p, SW, P, P.dz);
            float w;
            const bool cx = ix < P.bx_lo || ix >= P.bx_hi;
            const bool cz = iz < P.bz_lo || iz >= P.bz_hi;
            if (!band || (!cx && !cz)) {
                w = lx + lz;
            } else {
                const int i = iz * P.P + ix;
                w = 0.f;
                if (cx) {
                    const float a = __ldg(P.ax + ix), bb = __ldg(P.bx + ix), db = __ldg(P.dbx + ix);
                    const float du = grad_s(p, 1, P, P.dx);
                    const float* __restrict__ psx = F.psix + bo;
                    const float dap = grad_apsi(P.ax, ix, psx, i, 1, P, P.dx);
                    const float tmp = ((1.0f + bb) * lx + db * du) + dap;
                    float* __restrict__ zx = F.zetax + bo;
                    float* __restrict__ pxn = F.psixn + bo;
                    const float z = zx[i];
                    w += (1.0f + bb) * tmp + a * z;
                    pxn[i] = bb * du + a * __ldg(psx + i);
                    zx[i] = bb * tmp + a * z;
                } else {
                    w += lx;
                }
                if (cz) {
                    const float a = __ldg(P.az + iz), bb = __ldg(P.bz + iz), db = __ldg(P.dbz + iz);
                    const float du = grad_s(p, SW, P, P.dz);
                    const float* __restrict__ psz = F.psiz + bo;
                    const float dap = grad_apsi(P.az, iz, psz, i, P.P, P, P.dz);
                    const float tmp = ((1.0f + bb) * lz + db * du) + dap;
                    float* __restrict__ zz = F.zetaz + bo;
                    float* __restrict__ pzn = F.psizn + bo;
                    const float z = zz[i];
                    w += (1.0f + bb) * tmp + a * z;
                    pzn[i] = bb * du + a * __ldg(psz + i);
                    zz[i] = bb * tmp + a * z;
                } else {
                    w += lz;
                }
            }
            out[k] = 2.0f * p[0] - prev[r * TX + c] + cf[k] * w;
        }
        if (strip_tile) {
            if (F.sbf16)
                save_strips(P, now, static_cast<__nv_bfloat16*>(F.strips) + (long long)b * P.nstrip, tx0, tz0);
            else
                save_strips(P, now, static_cast<float*>(F.strips) + (long long)b * P.nstrip, tx0, tz0);
        }

        // point sources and receivers of this (shot, tile)
        const int4 er = sm.evr[g];
        const int s_beg = er.x, s_end = er.y, r_beg = er.z, r_end = er.w;
        if (s_beg != s_end || r_beg != r_end) {
#pragma unroll
            for (int k = 0; k < CPT; ++k) sm.out[cell_r(k) * TX + cell_c(k)] = out[k];
            __syncthreads();
            for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                const int2 ev = P.src.ev[e];
                atomicAdd(sm.out + ev.x, __ldg(P.wavelet + (long long)ev.y * P.nt + it));
            }
            __syncthreads();
            for (int e = r_beg + threadIdx.x; F.record && e < r_end; e += NTH) {
                const int2 ev = P.rec.ev[e];
                const int rb = ev.y / P.nrec, rr = ev.y - rb * P.nrec;
                F.record[((long long)rb * P.nt + it) * P.nrec + rr] = sm.out[ev.x];
            }
#pragma unroll
            for (int k = 0; k < CPT; ++k) out[k] = sm.out[cell_r(k) * TX + cell_c(k)];
        }
        float* un = F.u_next + bo;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int iz = tz0 + cell_r(k), ix = tx0 + cell_c(k);
            if (full || computed(P, iz, ix)) un[iz * P.P + ix] = out[k];
        }
        // every thread is done with stage s (and has waited for it)
        if (__syncthreads_or(bad)) { leave(g); return; }
        if (threadIdx.x == 0 && g + 2 < nloc) issue(s, b + 2);
    }
}

// ------------------------------------------------------------ reverse step
struct RevSmem {
    float l[2][SN];                  // lambda(it+1) tile + halo
    float lp[2][TN];                 // lambda(it+2) centre
    float r[2][SN];                  // u(it) tile + halo
    float rp[2][TN];                 // u(it+1) centre
    float c[SN];                     // (v*v)*(dt*dt) tile + halo
    float lo[TN];                    // staging (event tiles)
    float ro[TN];
    float bx[SW], dbx[SW];           // CPML b and db/dx at the staged columns (0 off the grid)
    float bz[SH], dbz[SH];           // the same at the staged rows
    int4 evr[kMaxG];                 // per shot of the CTA: source and receiver event ranges
    uint64_t bar[3];
    int bad[2];                      // a thread's wait for shot g failed: bad[g & 1] (read after the
                                     // shot's barrier; by parity, so shot g + 1's write cannot meet
                                     // a slower thread's read for shot g)
};

// One launch per reverse step `it` of the boundary-saving backward:
//   lambda_next = exact adjoint step of lambda (CPML transposed in the ring),
//   + record cotangent at the receivers               (-> lambda(it))
//   wavelet gradient  g_w[b, s, it] = lambda(it) at the sources
//   when it > 0: u(it-1) rebuilt in the reconstruction box, restored from the
//   saved strips elsewhere in the physical box, and the vp image
//   2 dt^2 u_tt lambda(it) / vp accumulated, u_tt = (u(it-1) - s(it) - 2 u(it) + u(it+1)) / dt^2;
//   then the source added back.
// The CPML form of the adjoint is applied per axis: a cell whose x (z)
// neighbourhood has b = db = 0 takes the plain x (z) Laplacian, which is what
// the CPML form reduces to there, and leaves that axis's memories untouched
// (they enter every update multiplied by b of their own cell).
__global__ void __launch_bounds__(NTH, 2) rev_kernel(const __grid_constant__ RevMaps MP, const Params P,
                                                     const RevPtrs R, const int it, const int do_recon)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    RevSmem& sm = *reinterpret_cast<RevSmem*>(smem_raw);
    const int tile = P.order[blockIdx.y];
    const int tx0 = (tile % P.ntx) * TX, tz0 = (tile / P.ntx) * TZ;
    const int b0 = blockIdx.x * P.G;
    const int nloc = min(P.G, P.B - b0);
    const int ntiles = P.ntx * P.ntz;
    const float dt2 = P.dt * P.dt;
    const float invdx2 = 1.0f / (P.dx * P.dx), invdz2 = 1.0f / (P.dz * P.dz);
    const float invdx = 1.0f / P.dx, invdz = 1.0f / P.dz;
    const bool ring = tx0 < P.px0 || tx0 + TX > P.px1 || tz0 < P.pz0 || tz0 + TZ > P.pz1;
    const bool phys_any = tx0 < P.x1 && tx0 + TX > P.x0 && tz0 < P.z1 && tz0 + TZ > P.z0;
    const bool phys_tile = do_recon && phys_any;
    const uint32_t kBytes = (SN + TN + (phys_tile ? SN + TN : 0)) * 4;

    // this thread's block: rows r0 .. r0+3, columns c0, c0+1 (global gz0.., gx0..)
    const int r0 = 4 * (threadIdx.x >> 5), c0 = 2 * (threadIdx.x & 31);
    const int gz0 = tz0 + r0, gx0 = tx0 + c0;
    unsigned cm = 0, pm = 0, rm = 0;  // bit k: computed / physical box / reconstruction box
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int iz = gz0 + (k >> 1), ix = gx0 + (k & 1);
        if (computed(P, iz, ix)) cm |= 1u << k;
        if (iz >= P.z0 && iz < P.z1 && ix >= P.x0 && ix < P.x1) pm |= 1u << k;
        if (iz >= P.rz0 && iz < P.rz1 && ix >= P.rx0 && ix < P.rx1) rm |= 1u << k;
    }
    auto xband = [&](int ix) { return ix < P.px0 || ix >= P.px1; };
    auto zband = [&](int iz) { return iz < P.pz0 || iz >= P.pz1; };
    const bool xc = ring && cm && (xband(gx0) || xband(gx0 + 1));
    const bool zc = ring && cm && (zband(gz0) || zband(gz0 + 1) || zband(gz0 + 2) || zband(gz0 + 3));

    if (threadIdx.x == 0) {
        for (int i = 0; i < 3; ++i) tma::mbar_init(&sm.bar[i], 1);
        tma::fence_barrier_init();
        sm.bad[0] = sm.bad[1] = 0;
    }
    __syncthreads();
    auto issue = [&](int s, int b) {
        tma::mbar_expect_tx(&sm.bar[s], kBytes);
        tma::load_3d(sm.l[s], &MP.lh[R.lnow], &sm.bar[s], tx0 - M, tz0 - M, b);
        tma::load_3d(sm.lp[s], &MP.lt[R.lprev], &sm.bar[s], tx0, tz0, b);
        if (phys_tile) {
            tma::load_3d(sm.r[s], &MP.rh[R.rnow], &sm.bar[s], tx0 - M, tz0 - M, b);
            tma::load_3d(sm.rp[s], &MP.rt[R.rprev], &sm.bar[s], tx0, tz0, b);
        }
        if (ring) {
            // the CPML memories this shot's ring cells read, into L2 ahead of use
            tma::prefetch_3d(&MP.am[0 + R.cur], tx0 - M, tz0, b);
            tma::prefetch_3d(&MP.am[4 + R.cur], tx0 - M, tz0, b);
            tma::prefetch_3d(&MP.am[2 + R.cur], tx0, tz0 - M, b);
            tma::prefetch_3d(&MP.am[6 + R.cur], tx0, tz0 - M, b);
        }
    };
    if (threadIdx.x == 0) {
        tma::mbar_expect_tx(&sm.bar[2], SN * 4);
        tma::load_3d(sm.c, &MP.ch, &sm.bar[2], tx0 - M, tz0 - M, P.ms ? b0 : 0);
        issue(0, b0);
        if (nloc > 1) issue(1, b0 + 1);
    }
    if (threadIdx.x < nloc) {
        const int key = (b0 + threadIdx.x) * ntiles + tile;
        sm.evr[threadIdx.x] = make_int4(P.src.off[key], P.src.off[key + 1], P.rec.off[key], P.rec.off[key + 1]);
    }
    if (ring) {
        for (int t = threadIdx.x; t < SW + SH; t += NTH) {
            if (t < SW) {
                const int ix = tx0 - M + t;
                const bool in = ix >= 0 && ix < P.nx;
                sm.bx[t] = in ? __ldg(P.bx + ix) : 0.f;
                sm.dbx[t] = in ? __ldg(P.dbx + ix) : 0.f;
            } else {
                const int q = t - SW, iz = tz0 - M + q;
                const bool in = iz >= 0 && iz < P.nz;
                sm.bz[q] = in ? __ldg(P.bz + iz) : 0.f;
                sm.dbz[q] = in ? __ldg(P.dbz + iz) : 0.f;
            }
        }
    }
    // per-cell vp (shared model or one shot per CTA: loaded once; the
    // reconstruction coefficient ((v*v)*dt)*dt is formed from it as the
    // forward's is); a column pair is computed together or its second cell is not
    float vr[CPT];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float2 v2 = make_float2(1.f, 1.f);
        if (cm >> (2 * j) & 1) v2 = ldg2(P.vv + b0 * P.ms + (long long)(gz0 + j) * P.P + gx0);
        vr[2 * j] = v2.x; vr[2 * j + 1] = (cm >> (2 * j + 1) & 1) ? v2.y : 1.f;
    }
    {
        const bool ok = tma::mbar_wait(&sm.bar[2], 0, P.err, ERR_TMA_WAIT_REV);
        if (__syncthreads_or(!ok)) return;
    }

    // illumination (when asked for) goes straight to this CTA's slot, shot by shot
    const long long slot = (long long)(P.per_shot ? b0 : blockIdx.x) * P.S;
    float gsum[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) gsum[k] = 0.f;

    // one block barrier per shot, as in fwd_kernel (the failure flag in
    // shared memory: a register kept across the shot loop would spill)
    auto leave = [&](int g) {
        if (threadIdx.x == 0)
            for (int h = g; h < min(g + 2, nloc); ++h)
                tma::mbar_wait(&sm.bar[h & 1], (h >> 1) & 1, P.err, ERR_TMA_WAIT_REV);
    };
    for (int g = 0; g < nloc; ++g) {
        const int b = b0 + g;
        const int s = g & 1;
        if (!tma::mbar_wait(&sm.bar[s], (g >> 1) & 1, P.err, ERR_TMA_WAIT_REV)) sm.bad[s] = 1;
        const long long bo = (long long)b * P.S;
        const float* sl = sm.l[s];
        const float* slp = sm.lp[s];
        const float* sr = sm.r[s];
        const float* srp = sm.rp[s];
        const float* sc = sm.c;

        float lo[CPT], ro[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) { lo[k] = 0.f; ro[k] = 0.f; }
        if (cm) {
            // c * lambda down the block's two columns, staged rows r0 .. r0+11
            float2 G[12];
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                const int o = (r0 + q) * SW + c0 + M;
                const float2 l2 = ld2(sl + o), c2 = ld2(sc + o);
                G[q] = make_float2(c2.x * l2.x, c2.y * l2.y);
            }
            float ux[CPT];               // x part of the adjoint update
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int so = (r0 + M + j) * SW + c0;      // window start (staged column c0)
                if (!xc) {
                    float gw[10];
#pragma unroll
                    for (int p = 0; p < 5; ++p) {
                        if (p == 2) continue;
                        const float2 l2 = ld2(sl + so + 2 * p), c2 = ld2(sc + so + 2 * p);
                        gw[2 * p] = c2.x * l2.x; gw[2 * p + 1] = c2.y * l2.y;
                    }
                    gw[4] = G[4 + j].x; gw[5] = G[4 + j].y;
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const float g0 = gw[4 + i];
                        float a = 0.0f;
#pragma unroll
                        for (int kk = 1; kk <= M; ++kk)
                            a += P.lc[kk] * (tap(gw[4 + i + kk], g0) + tap(gw[4 + i - kk], g0));
                        ux[2 * j + i] = a * invdx2;
                    }
                } else {
                    const int iz = gz0 + j;
                    const bool rowin = iz < P.nz;
                    const long long ro_ = bo + (long long)iz * P.P;
                    float tq[10], sq[10], hq[10], zc0[2], pc0[2];
#pragma unroll
                    for (int p = 0; p < 5; ++p) {
                        const float2 l2 = ld2(sl + so + 2 * p), c2 = ld2(sc + so + 2 * p);
                        const int ix = gx0 - M + 2 * p;
                        float2 z2 = make_float2(0.f, 0.f), p2 = make_float2(0.f, 0.f);
                        if (rowin && ix >= 0 && ix < P.nx) {
                            z2 = ldg2(R.azx + ro_ + ix);
                            p2 = ldg2(R.apx + ro_ + ix);
                        }
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int q = 2 * p + e;
                            const float bq = sm.bx[c0 + q], dbq = sm.dbx[c0 + q];
                            const float zq = comp(z2, e), pq = comp(p2, e);
                            tq[q] = bq * zq + ((1.0f + bq) * comp(c2, e)) * comp(l2, e);
                            sq[q] = (1.0f + bq) * tq[q];
                            hq[q] = bq * pq + dbq * tq[q];
                            if (q == 4 || q == 5) { zc0[q - 4] = zq; pc0[q - 4] = pq; }
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const float b_ = sm.bx[c0 + M + i];
                        const float gwc = comp(G[4 + j], i);
                        const float l0 = (1.0f + b_) * (b_ * zc0[i] + (1.0f + b_) * gwc);
                        float L = 0.0f, Dg = 0.0f, Dq = 0.0f;
#pragma unroll
                        for (int kk = 1; kk <= M; ++kk) {
                            L += P.lc[kk] * (tap(sq[4 + i + kk], l0) + tap(sq[4 + i - kk], l0));
                            Dg += P.gc[kk] * (hq[4 + i + kk] - hq[4 + i - kk]);
                            Dq += P.gc[kk] * (tq[4 + i + kk] - tq[4 + i - kk]);
                        }
                        ux[2 * j + i] = L * invdx2 - Dg * invdx;
                        if (cm >> (2 * j + i) & 1) {
                            const float a = __ldg(P.ax + gx0 + i);
                            R.apx_o[ro_ + gx0 + i] = a * (pc0[i] - Dq * invdx);
                            R.azx_o[ro_ + gx0 + i] = a * (zc0[i] + gwc);
                        }
                    }
                }
            }
            // z part, then lambda_next = 2 lambda - lambda_prev + x part + z part
            if (!zc) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const float g0 = comp(G[4 + j], i);
                        float a = 0.0f;
#pragma unroll
                        for (int kk = 1; kk <= M; ++kk)
                            a += P.lc[kk] * (tap(comp(G[4 + j + kk], i), g0) + tap(comp(G[4 + j - kk], i), g0));
                        ux[2 * j + i] += a * invdz2;
                    }
            } else {
                // centre terms (and the zeta update, which needs nothing else)
                float l0[CPT];
                const bool colin = gx0 < P.nx;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int iz = gz0 + j;
                    const float b_ = sm.bz[r0 + M + j];
                    float2 z2 = make_float2(0.f, 0.f);
                    const long long o = bo + (long long)iz * P.P + gx0;
                    if (colin && iz < P.nz) z2 = ldg2(R.azz + o);
                    const float a = (cm >> (2 * j) & 1) ? __ldg(P.az + iz) : 0.f;
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const float gwc = comp(G[4 + j], i);
                        l0[2 * j + i] = (1.0f + b_) * (b_ * comp(z2, i) + (1.0f + b_) * gwc);
                        if (cm >> (2 * j + i) & 1) R.azz_o[o + i] = a * (comp(z2, i) + gwc);
                    }
                }
                // one column at a time (keeps the accumulators of 4 cells live)
#pragma unroll 1
                for (int i = 0; i < 2; ++i) {
                    float L[4], Dg[4], Dq[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) { L[j] = 0.f; Dg[j] = 0.f; Dq[j] = 0.f; }
                    const bool cin = colin && (i == 0 || gx0 + 1 < P.nx);
#pragma unroll
                    for (int q = 0; q < 12; ++q) {
                        const int iz = gz0 - M + q;
                        const int o = (r0 + q) * SW + c0 + M + i;
                        float zq = 0.f, pq = 0.f;
                        if (cin && iz >= 0 && iz < P.nz) {
                            const long long go = bo + (long long)iz * P.P + gx0 + i;
                            zq = __ldg(R.azz + go); pq = __ldg(R.apz + go);
                        }
                        const float bq = sm.bz[r0 + q], dbq = sm.dbz[r0 + q];
                        const float t = bq * zq + ((1.0f + bq) * sc[o]) * sl[o];
                        const float sv = (1.0f + bq) * t;
                        const float h = bq * pq + dbq * t;
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int kk = q - M - j;
                            if (kk == 0 || kk < -M || kk > M) continue;
                            const int ka = kk < 0 ? -kk : kk;
                            L[j] += P.lc[ka] * tap(sv, i ? l0[2 * j + 1] : l0[2 * j]);
                            Dg[j] += kk > 0 ? P.gc[ka] * h : -(P.gc[ka] * h);
                            Dq[j] += kk > 0 ? P.gc[ka] * t : -(P.gc[ka] * t);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int k = 2 * j + i;
                        const float d = L[j] * invdz2 - Dg[j] * invdz;
                        if (i) ux[2 * j + 1] += d; else ux[2 * j] += d;
                        if (cm >> k & 1) {
                            const long long o = bo + (long long)(gz0 + j) * P.P + gx0 + i;
                            R.apz_o[o] = __ldg(P.az + gz0 + j) * (__ldg(R.apz + o) - Dq[j] * invdz);
                        }
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 lp2 = ld2(slp + (r0 + j) * TX + c0);
                const float2 l2 = ld2(sl + (r0 + M + j) * SW + c0 + M);
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int k = 2 * j + i;
                    if (cm >> k & 1) lo[k] = 2.0f * comp(l2, i) - comp(lp2, i) + ux[k];
                }
            }

            // reconstruction of u(it-1): stencil in the reconstruction box,
            // saved strips in the rest of the physical box
            if (phys_tile && pm) {
                float2 U[12];
#pragma unroll
                for (int q = 0; q < 12; ++q) U[q] = ld2(sr + (r0 + q) * SW + c0 + M);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int so = (r0 + M + j) * SW + c0;
                    float u[10];
#pragma unroll
                    for (int p = 0; p < 5; ++p) {
                        if (p == 2) continue;
                        const float2 v = ld2(sr + so + 2 * p);
                        u[2 * p] = v.x; u[2 * p + 1] = v.y;
                    }
                    u[4] = U[4 + j].x; u[5] = U[4 + j].y;
                    const float2 up2 = ld2(srp + (r0 + j) * TX + c0);
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const int k = 2 * j + i;
                        if (rm >> k & 1) {
                            const float u0 = u[4 + i];
                            float ax = 0.0f, az = 0.0f;
#pragma unroll
                            for (int kk = 1; kk <= M; ++kk) {
                                ax += P.lc[kk] * (tap(u[4 + i + kk], u0) + tap(u[4 + i - kk], u0));
                                az += P.lc[kk] * (tap(comp(U[4 + j + kk], i), u0) + tap(comp(U[4 + j - kk], i), u0));
                            }
                            const float wsum = ax / (P.dx * P.dx) + az / (P.dz * P.dz);
                            const float cf = ((vr[k] * vr[k]) * P.dt) * P.dt;
                            ro[k] = 2.0f * u0 - comp(up2, i) + cf * wsum;
                        } else if (pm >> k & 1) {
                            ro[k] = strip_value(P, R.strips, b, gz0 + j, gx0 + i);
                        }
                    }
                }
            }
        }

        const int4 er = sm.evr[g];
        const int s_beg = er.x, s_end = er.y, r_beg = er.z, r_end = er.w;
        const bool events = s_beg != s_end || r_beg != r_end;
        if (events) {
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int o = rcell_r(k) * TX + rcell_c(k);
                sm.lo[o] = lo[k]; sm.ro[o] = ro[k];
            }
            __syncthreads();
            for (int e = r_beg + threadIdx.x; e < r_end; e += NTH) {
                const int2 ev = P.rec.ev[e];
                const int rb = ev.y / P.nrec, rr = ev.y - rb * P.nrec;
                atomicAdd(sm.lo + ev.x, __ldg(R.adj + ((long long)rb * P.nt + it) * P.nrec + rr));
            }
            if (do_recon) {
                for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                    const int2 ev = P.src.ev[e];
                    const int iz = tz0 + ev.x / TX, ix = tx0 + ev.x % TX;
                    if (strip_index(P, iz, ix) >= 0)
                        atomicAdd(sm.ro + ev.x, -__ldg(P.wavelet + (long long)ev.y * P.nt + it));
                }
            }
            __syncthreads();
            if (R.grad_w) {
                for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                    const int2 ev = P.src.ev[e];
                    R.grad_w[(long long)ev.y * P.nt + it] = sm.lo[ev.x];
                }
            }
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int o = rcell_r(k) * TX + rcell_c(k);
                lo[k] = sm.lo[o]; ro[k] = sm.ro[o];
            }
        }

        // imaging (physical box), illumination, stores
        float* ln = R.l_next + bo;
        float gl[CPT];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const long long o = (long long)(gz0 + j) * P.P + gx0;
            const int k0 = 2 * j;
            if ((cm >> k0 & 3) == 3) {
                *reinterpret_cast<float2*>(ln + o) = make_float2(lo[k0], lo[k0 + 1]);
            } else if (cm >> k0 & 1) {
                ln[o] = lo[k0];
            }
            const float2 u02 = ld2(sr + (r0 + M + j) * SW + c0 + M);
            const float2 up2 = ld2(srp + (r0 + j) * TX + c0);
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int k = k0 + i;
                gl[k] = 0.f;
                if (!(pm >> k & 1)) continue;
                float utt = 0.f;
                if (do_recon) {
                    utt = (ro[k] - 2 * comp(u02, i) + comp(up2, i)) / dt2;
                    gl[k] = 2.f * P.dt * P.dt * utt * lo[k] / vr[k];
                }
                if (R.illum_s) {
                    R.illum_s[slot + o + i] += utt * utt;
                    R.illum_r[slot + o + i] += lo[k] * lo[k];
                }
            }
        }
        if (events && do_recon) {
            __syncthreads();
            for (int e = s_beg + threadIdx.x; e < s_end; e += NTH) {
                const int2 ev = P.src.ev[e];
                atomicAdd(sm.ro + ev.x, __ldg(P.wavelet + (long long)ev.y * P.nt + it));
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < CPT; ++k) ro[k] = sm.ro[rcell_r(k) * TX + rcell_c(k)];
        }
        if (phys_tile) {
            float* rn = R.r_next + bo;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const long long o = (long long)(gz0 + j) * P.P + gx0;
                const int k0 = 2 * j;
                if ((pm >> k0 & 3) == 3) {
                    *reinterpret_cast<float2*>(rn + o) = make_float2(ro[k0], ro[k0 + 1]);
                } else {
                    if (pm >> k0 & 1) rn[o] = ro[k0];
                    if (pm >> (k0 + 1) & 1) rn[o + 1] = ro[k0 + 1];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) gsum[k] += gl[k];
        // every thread is done with stage s (and has waited for it)
        __syncthreads();
        if (sm.bad[s]) { leave(g); return; }
        if (threadIdx.x == 0 && g + 2 < nloc) issue(s, b + 2);
    }

    // Kahan-compensated flush into this CTA's accumulator slot (per shot for
    // per-shot models, which run one shot per CTA; per shot group otherwise)
    if (pm && do_recon) {
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!(pm >> k & 1)) continue;
            const long long o = slot + (long long)(gz0 + (k >> 1)) * P.P + gx0 + (k & 1);
            const float y = gsum[k] - R.gcomp[o];
            const float t = R.gacc[o] + y;
            R.gcomp[o] = (t - R.gacc[o]) - y;
            R.gacc[o] = t;
        }
    }
}

// One step's strips (fp32 strip set, `strips`) into the scaled faces of a step
// slot: one CTA per (shot, face, block of kQB cells) -- max |value| of the
// block, its scale, the codes (reference boundarysaver.cu:957-990, 1050-1080:
// int8 round(v 127 / max) + 128 clamped to [0, 255]; fp16 v / max rounded).
__global__ void __launch_bounds__(kQB) quantize_strips(const Params P, const float* __restrict__ strips, void* slot)
{
    const StripStore& S = P.st;
    const int per = S.blocks[0] + S.blocks[1] + S.blocks[2] + S.blocks[3];
    const int b = blockIdx.x / per;
    int j = blockIdx.x - b * per, f = 0;
    while (f < 3 && j >= S.blocks[f]) { j -= S.blocks[f]; ++f; }
    const int idx = j * kQB + threadIdx.x;
    const bool in = idx < S.cells[f];
    float v = 0.f;
    if (in) {
        int iz, ix;
        face_cell(P, f, idx, iz, ix);
        v = strips[(long long)b * P.nstrip + strip_index(P, iz, ix)];
    }
    float m = fabsf(v);
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wmax[kQB / 32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    m = wmax[0];
#pragma unroll
    for (int i = 1; i < kQB / 32; ++i) m = fmaxf(m, wmax[i]);
    char* base = static_cast<char*>(slot);
    if (threadIdx.x == 0) reinterpret_cast<float*>(base + S.scl[f])[(long long)b * S.blocks[f] + j] = m;
    if (!in) return;
    const long long e = (long long)b * S.cells[f] + idx;
    if (S.fmt == SF_F16) {
        const float inv = m > 0.0f ? 1.0f / m : 0.0f;
        reinterpret_cast<__half*>(base + S.pay[f])[e] = __float2half(v * inv);
    } else {
        const float qs = m > 0.0f ? 127.0f / m : 0.0f;
        int q = __float2int_rn(v * qs) + 128;
        q = q < 0 ? 0 : (q > 255 ? 255 : q);
        reinterpret_cast<uint8_t*>(base + S.pay[f])[e] = (uint8_t)q;
    }
}

// Model-derived fields, pitched: cf = ((v*v)*dt)*dt (forward, reconstruction),
// ca = (v*v)*(dt*dt) (adjoint taps), vv = v (imaging); 0 (vv: 1) in the pitch pad.
__global__ void prep_kernel(const float* __restrict__ vp, int nm, int nz, int nx, int P, float dt,
                            float* __restrict__ cf, float* __restrict__ ca, float* __restrict__ vv)
{
    const long long n = (long long)nm * nz * P;
    const float dt2 = dt * dt;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / P;
        const int ix = (int)(i - row * P);
        if (ix < nx) {
            const float v = vp[row * nx + ix];
            cf[i] = ((v * v) * dt) * dt;
            ca[i] = (v * v) * dt2;
            vv[i] = v;
        } else {
            cf[i] = 0.f; ca[i] = 0.f; vv[i] = 1.f;
        }
    }
}

// Sum the Kahan slots (value minus compensation) into the caller's unpitched
// gradient (and illuminations).
__global__ void finalize_kernel(const float* __restrict__ acc, const float* __restrict__ comp,
                                const float* __restrict__ is, const float* __restrict__ ir,
                                int nslot_in, int nout, int nz, int nx, int P,
                                float* __restrict__ grad, float* __restrict__ ois, float* __restrict__ oir)
{
    const long long N = (long long)nz * nx, S = (long long)nz * P;
    const long long n = (long long)nout * N;
    const int per = nslot_in / nout;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = i / N, c = i - o * N;
        const long long iz = c / nx, ix = c - iz * nx;
        float s = 0.f, a = 0.f, bsum = 0.f;
        for (int k = 0; k < per; ++k) {
            const long long j = (o * per + k) * S + iz * P + ix;
            s += acc[j] - comp[j];
            if (is) { a += is[j]; bsum += ir[j]; }
        }
        grad[i] = s;
        if (ois) { ois[i] = a; oir[i] = bsum; }
    }
}

// Unpitched (B, nz, nx) <-> pitched (B, nz, P) copies of whole wavefields.
__global__ void pitch_copy_kernel(const float* __restrict__ src, float* __restrict__ dst, int B, int nz, int nx,
                                  int P, int to_pitched)
{
    const long long n = (long long)B * nz * nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / nx, ix = i - row * nx;
        if (to_pitched) dst[row * P + ix] = src[i];
        else dst[i] = src[row * P + ix];
    }
}

// ------------------------------------------------------------------- host
struct Plan {
    Params P;
    bool host_tape = false;          // boundary-saving tape in pinned host memory (SWEEP_MEM_HOST_TAPE)
    int nslot;                       // gradient accumulator slots (backward)
    int nm;                          // model copies (1 shared, B per-shot)
    int Gf, Gr;                      // shots per CTA: forward, backward
    dim3 gridf, gridr;
    int graph_steps;                 // time steps per captured CUDA graph (0: stream launches)
};

// CSR of the events of (shot, tile): off[key .. key+1) indexes ev, each
// (tile-local cell, global event id), in event order.  `loc` is the host copy
// of the (B, n, 2) coordinates; `fill` is (B * ntiles) scratch.
static int build_events(const Params& P, const int32_t* loc, int n, int32_t* off, int2* ev, int32_t* fill)
{
    const int ntiles = P.ntx * P.ntz;
    const int nkey = P.B * ntiles;
    for (int i = 0; i <= nkey; ++i) off[i] = 0;
    auto key_of = [&](int e) -> int {
        const int ix = loc[2 * e], iz = loc[2 * e + 1];
        // cells of the outer stencil halo are never updated: treated as off-grid
        if (ix < M || ix >= P.nx - M || iz < M || iz >= P.nz - M) return -1;
        return (e / n) * ntiles + (iz / TZ) * P.ntx + ix / TX;
    };
    for (int e = 0; e < P.B * n; ++e) {
        const int k = key_of(e);
        if (k >= 0) off[k + 1]++;
    }
    for (int i = 1; i <= nkey; ++i) off[i] += off[i - 1];
    for (int i = 0; i < nkey; ++i) fill[i] = off[i];
    for (int e = 0; e < P.B * n; ++e) {
        const int k = key_of(e);
        if (k < 0) continue;
        const int ix = loc[2 * e], iz = loc[2 * e + 1];
        ev[fill[k]++] = make_int2((iz % TZ) * TX + ix % TX, e);
    }
    return off[nkey];
}

// Shots per CTA: the shape's recorded schedule value if any, else the
// environment variable `env`, else `preferred` (measured best on B200 for this
// kernel) capped so the grid still fills the GPU.
static int choose_group(int ntiles, int B, const char* env, int preferred, int recorded)
{
    if (recorded >= 1) return std::min({recorded, B, kMaxG});
    if (const char* e = getenv(env)) {
        const int g = atoi(e);
        if (g >= 1) return std::min({g, B, kMaxG});
    }
    int G = std::min({preferred, B, kMaxG});
    while (G > 1 && (long long)ntiles * ((B + G - 1) / G) < 2LL * 148) --G;
    return std::max(G, 1);
}

static Plan make_plan(const sweep_acoustic_desc* d)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->ndim == 2, "acoustic2d: ndim must be 2 (got %d)", d->ndim);
    SWEEP_REQUIRE(d->M == M, "acoustic2d: only spatial order 8 (M = 4) is built (got M = %d)", d->M);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1, "acoustic2d: B and nt must be >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "acoustic2d: negative source/receiver count");
    SWEEP_REQUIRE(d->nz >= 2 * M + 1 && d->nx >= 2 * M + 1, "acoustic2d: grid too small");
    // a free surface is a face without PML cells (pad 0): the M halo cells
    // beyond it are never updated and stay zero
    for (int f = 0; f < 4; ++f) {
        const int p = d->pad[f < 2 ? f : f + 2];
        SWEEP_REQUIRE(p >= 0, "acoustic2d: negative PML pad on face %d (%d)", f, p);
    }
    Plan pl{};
    Params& P = pl.P;
    P.B = d->B; P.nz = d->nz; P.nx = d->nx; P.nt = d->nt;
    P.nsrc = d->nsrc; P.nrec = d->nrec;
    P.P = (d->nx + 31) / 32 * 32;
    P.S = (long long)d->nz * P.P;
    SWEEP_REQUIRE(P.S < (1LL << 31), "acoustic2d: one shot's grid must hold < 2^31 cells");
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
    P.per_shot = d->vp_stride != 0;
    P.ms = P.per_shot ? P.S : 0;
    pl.nm = P.per_shot ? d->B : 1;
    P.wavelet = d->wavelet;
    P.ntx = (d->nx + TX - 1) / TX;
    P.ntz = (d->nz + TZ - 1) / TZ;
    const int ntiles = P.ntx * P.ntz;
    const sweep_b200_schedule sc = recorded_schedule(d);
    pl.Gf = P.per_shot ? 1 : choose_group(ntiles, P.B, "SWEEP_B200_SHOTS_PER_CTA_FWD", 2, sc.shots_fwd);
    pl.Gr = P.per_shot ? 1 : choose_group(ntiles, P.B, "SWEEP_B200_SHOTS_PER_CTA_REV", 8, sc.shots_rev);
    pl.graph_steps = resolve_graph_steps(sc.graph_steps);
    // blockIdx.x = shot group (fastest), blockIdx.y = tile slot
    pl.gridf = dim3((P.B + pl.Gf - 1) / pl.Gf, ntiles);
    pl.gridr = dim3((P.B + pl.Gr - 1) / pl.Gr, ntiles);
    pl.nslot = P.per_shot ? P.B : (int)pl.gridr.x;
    P.G = pl.Gr;
    return pl;
}

struct Common {
    float *cf, *ca, *vv;
    int32_t *src_off, *rec_off;
    int2 *src_ev, *rec_ev;
    int* order;
    int* err;
};

struct FwdWork {
    Common c;
    float* u[3];
    float *psix, *psiz, *psixn, *psizn, *zetax, *zetaz;
    float* scratch;                  // one step's fp32 strips ahead of their quantisation (scaled formats)
    char* ring;                      // host tape: HostRing::R device strip slots
};

struct RevWork {
    Common c;
    float* l[3];
    float* aux[8];
    float* r[3];
    float *gacc, *gcomp, *is, *ir;
    char* ring;                      // host tape: HostRing::R device strip slots
};

static Common carve_common(Carve& c, const Plan& pl)
{
    Common w{};
    const long long nmS = (long long)pl.nm * pl.P.S;
    w.cf = c.take<float>(nmS);
    w.ca = c.take<float>(nmS);
    w.vv = c.take<float>(nmS);
    const long long nkey = (long long)pl.P.B * pl.P.ntx * pl.P.ntz + 1;
    w.src_off = c.take<int32_t>(nkey);
    w.rec_off = c.take<int32_t>(nkey);
    w.src_ev = c.take<int2>((long long)pl.P.B * std::max(pl.P.nsrc, 1));
    w.rec_ev = c.take<int2>((long long)pl.P.B * std::max(pl.P.nrec, 1));
    w.order = c.take<int>((long long)pl.P.ntx * pl.P.ntz);
    w.err = c.take<int>(1);
    return w;
}

static FwdWork carve_fwd(Carve& c, const Plan& pl)
{
    FwdWork w{};
    w.c = carve_common(c, pl);
    const long long n = (long long)pl.P.B * pl.P.S;
    for (auto& p : w.u) p = c.take<float>(n);
    w.psix = c.take<float>(n); w.psiz = c.take<float>(n);
    w.psixn = c.take<float>(n); w.psizn = c.take<float>(n);
    w.zetax = c.take<float>(n); w.zetaz = c.take<float>(n);
    if (pl.P.st.fmt == SF_F16 || pl.P.st.fmt == SF_I8) w.scratch = c.take<float>((long long)pl.P.B * pl.P.nstrip);
    if (pl.host_tape) w.ring = c.take<char>((long long)HostRing::R * pl.P.st.step);
    return w;
}

static RevWork carve_rev(Carve& c, const Plan& pl, bool illum)
{
    RevWork w{};
    w.c = carve_common(c, pl);
    const long long n = (long long)pl.P.B * pl.P.S;
    for (auto& p : w.l) p = c.take<float>(n);
    for (auto& p : w.aux) p = c.take<float>(n);
    for (auto& p : w.r) p = c.take<float>(n);
    w.gacc = c.take<float>((long long)pl.nslot * pl.P.S);
    w.gcomp = c.take<float>((long long)pl.nslot * pl.P.S);
    if (illum) {
        w.is = c.take<float>((long long)pl.nslot * pl.P.S);
        w.ir = c.take<float>((long long)pl.nslot * pl.P.S);
    }
    if (pl.host_tape) w.ring = c.take<char>((long long)HostRing::R * pl.P.st.step);
    return w;
}

// Strip storage of a memory mode: the step-slot layout of the boundary-saving
// tape (the checkpoint mode keeps its chunk strips as fp32).
static void set_store(Plan& pl, int mem_mode)
{
    pl.host_tape = (mem_mode & SWEEP_MEM_HOST_TAPE) != 0;
    mem_mode &= ~SWEEP_MEM_HOST_TAPE;
    Params& P = pl.P;
    StripStore& S = P.st;
    S = StripStore{};
    S.w = M + 1;
    S.fmt = mem_mode == SWEEP_MEM_BOUNDARY_FP16 ? SF_F16
          : mem_mode == SWEEP_MEM_BOUNDARY_BF16 ? SF_BF16
          : mem_mode == SWEEP_MEM_BOUNDARY_INT8 ? SF_I8 : SF_F32;
    auto up = [](long long v, long long a) { return (v + a - 1) / a * a; };
    if (S.fmt == SF_F32 || S.fmt == SF_BF16) {
        S.step = up((long long)P.B * P.nstrip * (S.fmt == SF_F32 ? 4 : 2), 256);
        return;
    }
    const int bw = P.x1 - P.x0, bh = P.z1 - P.z0;
    SWEEP_REQUIRE(bw >= 2 * S.w && bh >= 2 * S.w,
                  "acoustic2d: fp16 / int8 strip storage needs a physical box of at least %d cells per axis "
                  "(got %d x %d)", 2 * S.w, bh, bw);
    const int cells[4] = {S.w * bw, S.w * bw, bh * S.w, bh * S.w};
    const int esz = S.fmt == SF_F16 ? 2 : 1;
    long long off = 0;
    for (int f = 0; f < 4; ++f) {
        S.cells[f] = cells[f];
        S.blocks[f] = (cells[f] + kQB - 1) / kQB;
        S.pay[f] = off;
        off = up(off + (long long)P.B * cells[f] * esz, 16);
    }
    for (int f = 0; f < 4; ++f) {
        S.scl[f] = off;
        off = up(off + (long long)P.B * S.blocks[f] * 4, 16);
    }
    S.step = up(off, 256);
}

// tape: one strip slot per step (P.st.step bytes), then (U[nt-1], U[nt]) pitched
static int64_t tape_bytes(const Plan& pl)
{
    return (int64_t)pl.P.nt * pl.P.st.step + 2LL * pl.P.B * pl.P.S * 4;
}

static void* tape_slot(const void* tape, const Plan& pl, int it)
{
    return const_cast<char*>(static_cast<const char*>(tape)) + (long long)it * pl.P.st.step;
}

static float* tape_last(void* tape, const Plan& pl)
{
    return static_cast<float*>(tape_slot(tape, pl, pl.P.nt));
}

// Checkpointed boundary saving (SWEEP_MEM_CHECKPOINT, chunk length k): for
// every chunk c >= 1 the tape holds the forward state before step c k -- the
// wavefield pair (U[ck-1], U[ck]), the CPML psi (x, z) and zeta (x, z) -- and
// the strips of U[ck-1].  The backward replays each chunk from its checkpoint,
// keeping that chunk's strips only, and runs the boundary-saving reverse step
// over it (the reference re-runs each chunk from a checkpoint as well,
// checkpoint_runtime.cuh:15-362, eq_driver.cuh:928-1135).
constexpr int kStateFields = 6;

static int nchunks(const Plan& pl, int k)
{
    SWEEP_REQUIRE(k >= 1, "acoustic2d: checkpoint interval must be >= 1 (got %d)", k);
    return (pl.P.nt + k - 1) / k;
}

static long long ckpt_stride(const Plan& pl)
{
    Carve c(nullptr);
    c.take<float>(kStateFields * (long long)pl.P.B * pl.P.S);
    c.take<float>((long long)pl.P.B * pl.P.nstrip);
    return (c.off + 255) & ~255LL;
}

static int64_t tape_bytes_ckpt(const Plan& pl, int k)
{
    return (int64_t)std::max(nchunks(pl, k) - 1, 1) * ckpt_stride(pl);
}

// state field f of checkpoint c (c >= 1), then its strips
static float* ckpt_field(void* tape, const Plan& pl, int c, int f)
{
    char* base = static_cast<char*>(tape) + (long long)(c - 1) * ckpt_stride(pl);
    return reinterpret_cast<float*>(base) + (long long)f * pl.P.B * pl.P.S;
}

static float* ckpt_strips(void* tape, const Plan& pl, int c)
{
    return ckpt_field(tape, pl, c, kStateFields);
}

struct VecStage {
    std::vector<int32_t> ls, lr, os, orr, fill, ord;
    std::vector<int2> es, er;
    HostStage h{};
    VecStage(const Params& P)
        : ls((size_t)P.B * P.nsrc * 2 + 1), lr((size_t)P.B * P.nrec * 2 + 1),
          os((size_t)P.B * P.ntx * P.ntz + 1), orr((size_t)P.B * P.ntx * P.ntz + 1),
          fill((size_t)P.B * P.ntx * P.ntz + 1), ord((size_t)P.ntx * P.ntz),
          es((size_t)P.B * P.nsrc + 1), er((size_t)P.B * P.nrec + 1)
    {
        h = HostStage{ls.data(), lr.data(), os.data(), orr.data(), es.data(), er.data(), fill.data(), ord.data()};
    }
};

// Tile slots, heaviest first (the block scheduler hands out blocks in order):
// tiles crossing both CPML rings, then one, then the interior.  No allocation.
static void tile_order(const Params& P, int32_t* order)
{
    const int ntiles = P.ntx * P.ntz;
    int n = 0;
    for (int want = 2; want >= 0; --want)
        for (int t = 0; t < ntiles; ++t) {
            const int tx0 = (t % P.ntx) * TX, tz0 = (t / P.ntx) * TZ;
            const bool rx = tx0 < P.px0 || tx0 + TX > P.px1, rz = tz0 < P.pz0 || tz0 + TZ > P.pz1;
            if ((rx ? 1 : 0) + (rz ? 1 : 0) == want) order[n++] = t;
        }
}

// Per-call set-up shared by both passes: model fields, event tables, error flag.
static void setup_common(const sweep_acoustic_desc* d, Plan& pl, const Common& w, cudaStream_t st,
                         const HostStage& h)
{
    Params& P = pl.P;
    prep_kernel<<<592, 256, 0, st>>>(d->vp, pl.nm, d->nz, d->nx, P.P, d->dt, w.cf, w.ca, w.vv);
    SWEEP_LAUNCH_CHECK();
    P.cf = w.cf; P.vv = w.vv;
    const size_t ns = (size_t)d->B * d->nsrc * 2, nr = (size_t)d->B * d->nrec * 2;
    if (ns) SWEEP_CUDA(cudaMemcpyAsync(h.loc_src, d->src_loc, ns * 4, cudaMemcpyDeviceToHost, st));
    if (nr) SWEEP_CUDA(cudaMemcpyAsync(h.loc_rec, d->rec_loc, nr * 4, cudaMemcpyDeviceToHost, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    const int nsev = build_events(P, h.loc_src, d->nsrc, h.off_src, h.ev_src, h.fill);
    const int nrev = build_events(P, h.loc_rec, d->nrec, h.off_rec, h.ev_rec, h.fill);
    const size_t nkey = (size_t)P.B * P.ntx * P.ntz + 1;
    SWEEP_CUDA(cudaMemcpyAsync(w.src_off, h.off_src, nkey * 4, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemcpyAsync(w.rec_off, h.off_rec, nkey * 4, cudaMemcpyHostToDevice, st));
    if (nsev) SWEEP_CUDA(cudaMemcpyAsync(w.src_ev, h.ev_src, nsev * sizeof(int2), cudaMemcpyHostToDevice, st));
    if (nrev) SWEEP_CUDA(cudaMemcpyAsync(w.rec_ev, h.ev_rec, nrev * sizeof(int2), cudaMemcpyHostToDevice, st));
    // the host staging may be reused or released once the copies have read it
    SWEEP_CUDA(cudaStreamSynchronize(st));
    P.src.off = w.src_off; P.src.ev = w.src_ev;
    P.rec.off = w.rec_off; P.rec.ev = w.rec_ev;
    tile_order(P, h.order);
    SWEEP_CUDA(cudaMemcpyAsync(w.order, h.order, (size_t)P.ntx * P.ntz * sizeof(int), cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    P.order = w.order;
    SWEEP_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    P.err = w.err;
}

static void check_err(const Common& w, cudaStream_t st, const char* what)
{
    int h = 0;
    SWEEP_CUDA(cudaMemcpyAsync(&h, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    SWEEP_REQUIRE(h == 0, "acoustic2d %s: a tile load did not complete in time (code %d); results are invalid", what, h);
}

static CUtensorMap field_map(const float* base, const Params& P, int nb, bool halo)
{
    const uint64_t dims[3] = {(uint64_t)P.nx, (uint64_t)P.nz, (uint64_t)nb};
    const uint64_t strides[2] = {(uint64_t)P.P, (uint64_t)P.S};
    const uint32_t box[3] = {(uint32_t)(halo ? SW : TX), (uint32_t)(halo ? SH : TZ), 1u};
    return tma::make_map(base, 3, dims, strides, box);
}

// A CPML memory (full grid, pitched) with the box its ring cells read: x
// memories (TX + 2M) x TZ, z memories TX x (TZ + 2M).
static CUtensorMap mem_map(const float* base, const Params& P, bool xmem)
{
    const uint64_t dims[3] = {(uint64_t)P.nx, (uint64_t)P.nz, (uint64_t)P.B};
    const uint64_t strides[2] = {(uint64_t)P.P, (uint64_t)P.S};
    const uint32_t box[3] = {(uint32_t)(xmem ? SW : TX), (uint32_t)(xmem ? TZ : SH), 1u};
    return tma::make_map(base, 3, dims, strides, box);
}

static size_t fwd_smem() { return sizeof(FwdSmem); }
static size_t rev_smem() { return sizeof(RevSmem); }

static void set_attrs()
{
    static bool done = false;
    if (done) return;
    SWEEP_CUDA(cudaFuncSetAttribute(fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem()));
    SWEEP_CUDA(cudaFuncSetAttribute(rev_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rev_smem()));
    done = true;
}

// Backward workspace of the checkpoint mode: the reverse set, the forward set
// the replay runs in, and the strips of one chunk (k + 1 steps).
static void carve_rev_ckpt(Carve& c, const Plan& pl, bool illum, int k, RevWork& rw, FwdWork& fw, float*& chunk)
{
    rw = carve_rev(c, pl, illum);
    const long long n = (long long)pl.P.B * pl.P.S;
    for (auto& p : fw.u) p = c.take<float>(n);
    fw.psix = c.take<float>(n); fw.psiz = c.take<float>(n);
    fw.psixn = c.take<float>(n); fw.psizn = c.take<float>(n);
    fw.zetax = c.take<float>(n); fw.zetaz = c.take<float>(n);
    fw.c = rw.c;
    chunk = c.take<float>((long long)(k + 1) * pl.P.B * pl.P.nstrip);
}

static void check_mode(int mem_mode, int ckpt_every)
{
    if (mem_mode & SWEEP_MEM_HOST_TAPE) {
        mem_mode &= ~SWEEP_MEM_HOST_TAPE;
        SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT && mem_mode != SWEEP_MEM_RECURSIVE,
                      "acoustic2d: a host tape goes with boundary saving only");
    }
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY || mem_mode == SWEEP_MEM_CHECKPOINT ||
                      mem_mode == SWEEP_MEM_BOUNDARY_FP16 || mem_mode == SWEEP_MEM_BOUNDARY_BF16 ||
                      mem_mode == SWEEP_MEM_BOUNDARY_INT8 || mem_mode == SWEEP_MEM_RECURSIVE,
                  "acoustic2d: unknown memory mode %d", mem_mode);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT || ckpt_every >= 1,
                  "acoustic2d: checkpoint interval must be >= 1 (got %d)", ckpt_every);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_RECURSIVE || ckpt_every >= 1,
                  "acoustic2d: the recursive checkpoint budget must be >= 1 (got %d)", ckpt_every);
}

static void copy_any(void* dst, const void* src, long long bytes, cudaStream_t st)
{
    SWEEP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st));
}

void sizes(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, int64_t* ws, int64_t* tape)
{
    check_mode(mem_mode, ckpt_every);
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    Carve cf(nullptr);
    carve_fwd(cf, pl);
    Carve cr(nullptr);
    if (mem_mode == SWEEP_MEM_CHECKPOINT) {
        RevWork rw; FwdWork fw; float* chunk;
        carve_rev_ckpt(cr, pl, true, ckpt_every, rw, fw, chunk);
        *tape = tape_bytes_ckpt(pl, ckpt_every);
    } else if (mem_mode == SWEEP_MEM_RECURSIVE) {
        RevWork rw; FwdWork fw; float* chunk;
        carve_rev_ckpt(cr, pl, true, SWEEP_RECURSIVE_LEAF, rw, fw, chunk);
        cr.take<char>((long long)ckpt_every * ckpt_stride(pl));      // the snapshot slots
        *tape = 256;                                                   // nothing is kept
    } else {
        carve_rev(cr, pl, true);
        *tape = tape_bytes(pl);
    }
    *ws = std::max(cf.off, cr.off);
}

void schedule_of(const sweep_acoustic_desc* d, sweep_b200_schedule* out)
{
    const Plan pl = make_plan(d);
    out->shots_fwd = pl.Gf;
    out->shots_rev = pl.Gr;
    out->z_chunks = 0;
    out->graph_steps = pl.graph_steps;
    out->tile_y = 0;
}

int64_t forward_only_bytes(const sweep_acoustic_desc* d)
{
    Plan pl = make_plan(d);
    Carve c(nullptr);
    carve_fwd(c, pl);
    return c.off;
}

void stage_sizes(const sweep_acoustic_desc* d, int64_t* nkey, int64_t* nev_src, int64_t* nev_rec)
{
    Plan pl = make_plan(d);
    *nkey = (int64_t)pl.P.B * pl.P.ntx * pl.P.ntz + 1;
    *nev_src = (int64_t)d->B * d->nsrc;
    *nev_rec = (int64_t)d->B * d->nrec;
}

// Rotating forward state: wavefield buffer indices and the CPML psi pair.
struct FwdState {
    int ip = 0, in = 1, ix = 2;
    float *px, *pz, *pxn, *pzn;
};

static FwdMaps fwd_maps(const FwdWork& w, const Params& P)
{
    FwdMaps maps;
    for (int i = 0; i < 3; ++i) {
        maps.halo[i] = field_map(w.u[i], P, P.B, true);
        maps.tile[i] = field_map(w.u[i], P, P.B, false);
    }
    return maps;
}

// Forward steps [it0, it1): one fwd_kernel launch per step; `strips_of(it)`
// is the strip slot step `it` writes (null: none), `record` may be null.
template <class StripsOf>
static void forward_steps(const Plan& pl, const FwdMaps& maps, const FwdWork& w, float* record, FwdState& S,
                          int it0, int it1, StripsOf strips_of, cudaStream_t st, HostRing* hr = nullptr,
                          bool graphs = true)
{
    StepGraphs gs(st, (hr || !graphs) ? 0 : pl.graph_steps);
    Params PF = pl.P;
    PF.G = pl.Gf;
    FwdPtrs F{};
    F.record = record;
    F.zetax = w.zetax; F.zetaz = w.zetaz;
    const bool scaled = PF.st.fmt == SF_F16 || PF.st.fmt == SF_I8;
    const int qblocks = PF.B * (PF.st.blocks[0] + PF.st.blocks[1] + PF.st.blocks[2] + PF.st.blocks[3]);
    for (int it = it0; it < it1; ++it) {
        F.now = S.in; F.prev = S.ip; F.u_next = w.u[S.ix];
        F.psix = S.px; F.psiz = S.pz; F.psixn = S.pxn; F.psizn = S.pzn;
        void* slot = strips_of(it);
        if (slot && hr) hr->before_write(it);
        F.strips = (slot && scaled) ? static_cast<void*>(w.scratch) : slot;
        F.sbf16 = PF.st.fmt == SF_BF16;
        const cudaStream_t ls = gs.stream();
        fwd_kernel<<<pl.gridf, NTH, fwd_smem(), ls>>>(maps, PF, F, it);
        SWEEP_LAUNCH_CHECK();
        if (slot && scaled) {
            quantize_strips<<<qblocks, kQB, 0, ls>>>(PF, w.scratch, slot);
            SWEEP_LAUNCH_CHECK();
        }
        if (slot && hr) hr->after_write(it);
        gs.step_done();
        const int t = S.ip; S.ip = S.in; S.in = S.ix; S.ix = t;
        std::swap(S.px, S.pxn); std::swap(S.pz, S.pzn);
    }
    gs.flush();
}

static void copy_dd(float* dst, const float* src, long long n, cudaStream_t st)
{
    SWEEP_CUDA(cudaMemcpyAsync(dst, src, n * 4, cudaMemcpyDeviceToDevice, st));
}

void forward_with(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape, void* ws,
                  int64_t ws_bytes, cudaStream_t st, const HostStage* stage, StepState* seg, int seg0, int seg1)
{
    // a stepped run covers [seg0, seg1) of the time axis, continuing seg's state
    const bool stepped = seg != nullptr;
    const int a = stepped ? seg0 : 0, b = stepped ? seg1 : d->nt;
    SWEEP_REQUIRE(!stepped || ckpt_every <= 0, "acoustic2d stepped forward: boundary saving only");
    SWEEP_REQUIRE(record != nullptr || d->nrec == 0, "acoustic2d forward: null record");
    SWEEP_REQUIRE(d->vp != nullptr, "acoustic2d forward: null vp");
    set_attrs();
    Plan pl = make_plan(d);
    set_store(pl, ckpt_every > 0 ? SWEEP_MEM_CHECKPOINT : mem_mode);
    Carve c(ws);
    FwdWork w = carve_fwd(c, pl);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= c.off, "acoustic2d forward: workspace too small (%lld < %lld)",
                  (long long)ws_bytes, (long long)c.off);
    if (stage) {
        setup_common(d, pl, w.c, st, *stage);
    } else {
        VecStage vs(pl.P);
        setup_common(d, pl, w.c, st, vs.h);
    }
    const Params& P = pl.P;
    const long long n = (long long)P.B * P.S;
    if (a == 0) {
        for (auto* p : w.u) SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
        for (auto* p : {w.psix, w.psiz, w.psixn, w.psizn, w.zetax, w.zetaz})
            SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
        if (d->nrec > 0)
            SWEEP_CUDA(cudaMemsetAsync(record, 0, (size_t)d->B * d->nt * d->nrec * 4, st));
    }
    const FwdMaps maps = fwd_maps(w, P);
    FwdState S;
    S.px = w.psix; S.pz = w.psiz; S.pxn = w.psixn; S.pzn = w.psizn;
    if (stepped && a > 0) {
        S.ip = seg->idx[0]; S.in = seg->idx[1]; S.ix = seg->idx[2];
        S.px = static_cast<float*>(seg->ptr[0]); S.pz = static_cast<float*>(seg->ptr[1]);
        S.pxn = static_cast<float*>(seg->ptr[2]); S.pzn = static_cast<float*>(seg->ptr[3]);
    }
    // a caller-staged call (the allocation-free entry) issues plain launches:
    // instantiating a graph allocates
    const bool graphs = stage == nullptr;
    if (ckpt_every <= 0 && tape && pl.host_tape) {
        HostRing hr;
        hr.open(w.ring, tape, P.st.step, st);
        forward_steps(pl, maps, w, record, S, a, b, [&](int it) { return hr.slot(it); }, st, &hr);
        hr.close();
        if (b == d->nt) {
            float* last = tape_last(tape, pl);
            copy_any(last, w.u[S.ip], n * 4, st);
            copy_any(last + n, w.u[S.in], n * 4, st);
        }
    } else if (ckpt_every <= 0) {
        forward_steps(pl, maps, w, record, S, a, b,
                      [&](int it) { return tape ? tape_slot(tape, pl, it) : nullptr; }, st, nullptr, graphs);
        if (tape && b == d->nt) {
            float* last = tape_last(tape, pl);
            // (U[nt-1], U[nt]) per shot, pitched
            copy_dd(last, w.u[S.ip], n, st);
            copy_dd(last + n, w.u[S.in], n, st);
        }
    } else {
        const int k = ckpt_every, C = nchunks(pl, k);
        for (int ch = 0; ch < C; ++ch) {
            const int it0 = ch * k, it1 = std::min(d->nt, it0 + k);
            if (tape && ch >= 1) {
                const float* state[kStateFields] = {w.u[S.ip], w.u[S.in], S.px, S.pz, w.zetax, w.zetaz};
                for (int f = 0; f < kStateFields; ++f) copy_dd(ckpt_field(tape, pl, ch, f), state[f], n, st);
            }
            // the last step of a chunk keeps its strips with the next checkpoint
            forward_steps(pl, maps, w, record, S, it0, it1,
                          [&](int it) {
                              return (tape && it == it1 - 1 && ch + 1 < C) ? ckpt_strips(tape, pl, ch + 1) : nullptr;
                          },
                          st, nullptr, graphs);
        }
    }
    if (stepped) {
        seg->idx[0] = S.ip; seg->idx[1] = S.in; seg->idx[2] = S.ix;
        seg->ptr[0] = S.px; seg->ptr[1] = S.pz; seg->ptr[2] = S.pxn; seg->ptr[3] = S.pzn;
    }
    check_err(w.c, st, "forward");
}

void forward(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape,
             void* ws, int64_t ws_bytes, cudaStream_t st)
{
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, ckpt_every, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic2d forward: workspace too small (%lld < %lld)",
                  (long long)ws_bytes, (long long)need_ws);
    // recursive checkpointing keeps nothing from the forward: the backward
    // replays from the initial state
    forward_with(d, mem_mode == SWEEP_MEM_RECURSIVE ? SWEEP_MEM_BOUNDARY : mem_mode,
                 mem_mode == SWEEP_MEM_CHECKPOINT ? ckpt_every : 0, record,
                 mem_mode == SWEEP_MEM_RECURSIVE ? nullptr : tape, ws, ws_bytes, st, nullptr, nullptr, 0, 0);
}

void forward_segment(const sweep_acoustic_desc* d, int mem_mode, float* record, void* tape, void* ws,
                     int64_t ws_bytes, cudaStream_t st, StepState& seg, int it0, int it1)
{
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, 0, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic2d forward runner: workspace too small (%lld < %lld)",
                  (long long)ws_bytes, (long long)need_ws);
    forward_with(d, mem_mode, 0, record, tape, ws, ws_bytes, st, nullptr, &seg, it0, it1);
}

// Recursive checkpointing (SWEEP_MEM_RECURSIVE; reference
// Ckpt(mode='recursive', count), sg_driver.cuh / eq_driver.cuh recursive
// runners): reverse [0, nt) leaf by leaf, last leaf first.  An interval
// [a, b) longer than one leaf is bisected at a leaf boundary m: the forward is
// replayed from the state at a to m, the state at m (and the strips of
// U[m - 1]) goes into the next free snapshot slot, [m, b) is processed, the
// slot is freed and [a, m) follows.  With no slot left, each leaf of [a, b)
// replays from the state at a.  A leaf [a, e) is replayed from the state at a
// into its strips and reversed by the boundary-saving step, exactly as a
// checkpoint chunk; the leaves are the chunks of SWEEP_MEM_CHECKPOINT with
// interval SWEEP_RECURSIVE_LEAF, so the gradient is that mode's.
template <class Reverse>
static void backward_recursive(const Plan& pl, FwdWork& fw, RevWork& w, float* chunk, char* snaps, int count,
                               cudaStream_t st, Reverse& reverse)
{
    const Params& P = pl.P;
    const int L = SWEEP_RECURSIVE_LEAF;
    const long long n = (long long)P.B * P.S, cs = (long long)P.B * P.nstrip;
    const FwdMaps fmaps = fwd_maps(fw, P);
    float* state[kStateFields] = {fw.u[0], fw.u[1], fw.psix, fw.psiz, fw.zetax, fw.zetaz};
    // the replay set starts clear (see the checkpoint mode)
    for (auto* p : {fw.u[0], fw.u[1], fw.u[2], fw.psix, fw.psiz, fw.psixn, fw.psizn, fw.zetax, fw.zetaz})
        SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
    FwdState S;
    // the state before step a: snapshot slot k, or the initial (zero) state for k < 0
    auto restore = [&](int k) {
        S = FwdState{};
        S.px = fw.psix; S.pz = fw.psiz; S.pxn = fw.psixn; S.pzn = fw.psizn;
        for (int f = 0; f < kStateFields; ++f) {
            if (k < 0) SWEEP_CUDA(cudaMemsetAsync(state[f], 0, n * 4, st));
            else copy_dd(state[f], ckpt_field(snaps, pl, k + 1, f), n, st);
        }
    };
    auto save = [&](int k) {
        const float* cur[kStateFields] = {fw.u[S.ip], fw.u[S.in], S.px, S.pz, fw.zetax, fw.zetaz};
        for (int f = 0; f < kStateFields; ++f) copy_dd(ckpt_field(snaps, pl, k + 1, f), cur[f], n, st);
    };
    // replay [a, e) from the current state into the chunk's strips, then reverse it
    auto leaf = [&](int a, int e) {
        forward_steps(pl, fmaps, fw, nullptr, S, a, e, [&](int it) { return chunk + (long long)(it - a + 1) * cs; },
                      st);
        copy_dd(w.r[0], fw.u[S.in], n, st);       // U[e]
        copy_dd(w.r[1], fw.u[S.ip], n, st);       // U[e - 1]
        reverse(a, e, [&](int t) { return chunk + (long long)(t - (a - 1)) * cs; });
    };
    std::function<void(int, int, int, int)> process = [&](int a, int b, int ka, int free) {
        const int nleaf = (b - a + L - 1) / L;
        if (nleaf <= 1) {
            restore(ka);
            if (a > 0) copy_dd(chunk, ckpt_strips(snaps, pl, ka + 1), cs, st);   // strips of U[a - 1]
            leaf(a, b);
            return;
        }
        if (free > 0) {
            const int k = count - free, m = a + L * ((nleaf + 1) / 2);
            restore(ka);
            forward_steps(pl, fmaps, fw, nullptr, S, a, m,
                          [&](int it) { return it == m - 1 ? ckpt_strips(snaps, pl, k + 1) : nullptr; }, st);
            save(k);
            process(m, b, k, free - 1);
            process(a, m, ka, free);
            return;
        }
        for (int c0 = a + (nleaf - 1) * L; c0 >= a; c0 -= L) {
            restore(ka);
            if (c0 > a)
                forward_steps(pl, fmaps, fw, nullptr, S, a, c0, [&](int it) { return it == c0 - 1 ? chunk : nullptr; },
                              st);
            else if (a > 0)
                copy_dd(chunk, ckpt_strips(snaps, pl, ka + 1), cs, st);
            leaf(c0, std::min(b, c0 + L));
        }
    };
    // a snapshot slot k holds the state before its step and the strips of the step before
    SWEEP_REQUIRE(count >= 1, "acoustic2d: the recursive checkpoint budget must be >= 1");
    process(0, P.nt, -1, count);
}

void backward_with(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
                   float* grad_vp, float* grad_w, float* illum_s, float* illum_r,
                   void* ws, int64_t ws_bytes, cudaStream_t st, StepState* seg, int bw0, int bw1)
{
    // a stepped run reverses [bw1, bw0) top down, continuing seg's state
    const bool stepped = seg != nullptr;
    const int top = stepped ? bw0 : d->nt, bottom = stepped ? bw1 : 0;
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, ckpt_every, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic2d backward: workspace too small");
    SWEEP_REQUIRE(tape != nullptr, "acoustic2d backward: null tape");
    SWEEP_REQUIRE(grad_vp != nullptr, "acoustic2d backward: null grad_vp");
    SWEEP_REQUIRE(adj != nullptr || d->nrec == 0, "acoustic2d backward: null record cotangent");
    SWEEP_REQUIRE((illum_s == nullptr) == (illum_r == nullptr), "acoustic2d backward: pass both illuminations or neither");
    set_attrs();
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    Carve c(ws);
    const bool illum = illum_s != nullptr;
    const bool ckpt = mem_mode == SWEEP_MEM_CHECKPOINT;
    const bool recursive = mem_mode == SWEEP_MEM_RECURSIVE;
    SWEEP_REQUIRE(!stepped || (!ckpt && !recursive), "acoustic2d stepped backward: boundary saving only");
    const bool first = top == d->nt;
    RevWork w;
    FwdWork fw{};
    float* chunk = nullptr;
    char* snaps = nullptr;
    if (ckpt) carve_rev_ckpt(c, pl, illum, ckpt_every, w, fw, chunk);
    else if (recursive) {
        carve_rev_ckpt(c, pl, illum, SWEEP_RECURSIVE_LEAF, w, fw, chunk);
        snaps = c.take<char>((long long)ckpt_every * ckpt_stride(pl));
    } else w = carve_rev(c, pl, illum);
    {
        VecStage vs(pl.P);
        setup_common(d, pl, w.c, st, vs.h);
    }
    const Params& P = pl.P;
    const long long n = (long long)P.B * P.S;
    if (first) {
        for (auto* p : w.l) SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
        for (auto* p : w.aux) SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
        SWEEP_CUDA(cudaMemsetAsync(w.r[2], 0, n * 4, st));
        SWEEP_CUDA(cudaMemsetAsync(w.gacc, 0, (size_t)pl.nslot * P.S * 4, st));
        SWEEP_CUDA(cudaMemsetAsync(w.gcomp, 0, (size_t)pl.nslot * P.S * 4, st));
        if (illum) {
            SWEEP_CUDA(cudaMemsetAsync(w.is, 0, (size_t)pl.nslot * P.S * 4, st));
            SWEEP_CUDA(cudaMemsetAsync(w.ir, 0, (size_t)pl.nslot * P.S * 4, st));
        }
        if (grad_w && d->nsrc > 0)
            SWEEP_CUDA(cudaMemsetAsync(grad_w, 0, (size_t)d->B * d->nsrc * d->nt * 4, st));
    }
    RevMaps maps;
    for (int i = 0; i < 3; ++i) {
        maps.lh[i] = field_map(w.l[i], P, P.B, true);
        maps.lt[i] = field_map(w.l[i], P, P.B, false);
        maps.rh[i] = field_map(w.r[i], P, P.B, true);
        maps.rt[i] = field_map(w.r[i], P, P.B, false);
    }
    maps.ch = field_map(w.c.ca, P, pl.nm, true);
    for (int i = 0; i < 8; ++i) maps.am[i] = mem_map(w.aux[i], P, (i >> 1) == 0 || (i >> 1) == 2);
    RevPtrs R{};
    R.adj = adj; R.grad_w = grad_w;
    R.gacc = w.gacc; R.gcomp = w.gcomp;
    R.illum_s = w.is; R.illum_r = w.ir;
    int lp = 0, ln = 1, lx = 2;
    int cur = 0;
    int rp = 0, rn = 1, rx = 2;
    if (stepped && !first) {
        lp = seg->idx[0]; ln = seg->idx[1]; lx = seg->idx[2]; cur = seg->idx[3];
        rp = seg->idx[4]; rn = seg->idx[5]; rx = seg->idx[6];
    }
    // Reverse steps [it0, it1) top down; a fresh run starts the reconstruction
    // from r[0] = U[it1], r[1] = U[it1 - 1], a continued one where the last
    // stopped; strips_of(it) holds the strips of U[it].
    HostRing hr;
    const bool host = pl.host_tape && !ckpt && !recursive;
    auto reverse = [&](int it0, int it1, auto strips_of, bool fresh) {
        StepGraphs gs(st, host ? 0 : pl.graph_steps);
        if (fresh) { rp = 0; rn = 1; rx = 2; }
        for (int it = it1 - 1; it >= it0; --it) {
            const int do_recon = it > 0 ? 1 : 0;
            R.lprev = lp; R.lnow = ln; R.l_next = w.l[lx];
            R.apx = w.aux[0 + cur]; R.apz = w.aux[2 + cur]; R.azx = w.aux[4 + cur]; R.azz = w.aux[6 + cur];
            R.apx_o = w.aux[1 - cur]; R.apz_o = w.aux[3 - cur]; R.azx_o = w.aux[5 - cur]; R.azz_o = w.aux[7 - cur];
            R.cur = cur;
            R.rprev = rp; R.rnow = rn; R.r_next = w.r[rx];
            R.strips = do_recon ? strips_of(it - 1) : nullptr;
            if (host && do_recon) hr.before_read(it - 1);
            rev_kernel<<<pl.gridr, NTH, rev_smem(), gs.stream()>>>(maps, P, R, it, do_recon);
            SWEEP_LAUNCH_CHECK();
            if (host && do_recon) {
                hr.after_read(it - 1);
                if (it - 1 - HostRing::R >= std::max(it0 - 1, 0)) hr.fetch(it - 1 - HostRing::R, true);
            }
            gs.step_done();
            int t = lp; lp = ln; ln = lx; lx = t;
            cur = 1 - cur;
            if (do_recon) { t = rp; rp = rn; rn = rx; rx = t; }
        }
        gs.flush();
    };
    if (recursive) {
        auto rev = [&](int it0, int it1, auto strips_of) { reverse(it0, it1, strips_of, true); };
        backward_recursive(pl, fw, w, chunk, snaps, ckpt_every, st, rev);
    } else if (!ckpt) {
        if (first) {
            const float* last = tape_last(const_cast<void*>(tape), pl);
            // seed: prev = U[nt], now = U[nt-1]  (reference driver_traits.cuh:493-505; the
            // rim outside the physical box is never read by the reconstruction)
            copy_any(w.r[0], last + n, n * 4, st);
            copy_any(w.r[1], last, n * 4, st);
        }
        if (host) {
            hr.open(w.ring, const_cast<void*>(tape), P.st.step, st);
            for (int t = top - 2; t >= std::max(bottom - 1, 0) && t > top - 2 - HostRing::R; --t) hr.fetch(t, false);
            reverse(bottom, top, [&](int t) { return hr.slot(t); }, first);
            hr.close();
        } else {
            reverse(bottom, top, [&](int t) { return tape_slot(tape, pl, t); }, first);
        }
    } else {
        const int k = ckpt_every, C = nchunks(pl, k);
        const FwdMaps fmaps = fwd_maps(fw, P);
        void* tp = const_cast<void*>(tape);
        const long long cs = (long long)P.B * P.nstrip;
        // the replay set starts clear: the fields a checkpoint does not hold
        // (the third wavefield buffer, the next psi pair) are read in their
        // stencil halo and outside the CPML band, which no step writes
        for (auto* p : {fw.u[0], fw.u[1], fw.u[2], fw.psix, fw.psiz, fw.psixn, fw.psizn, fw.zetax, fw.zetaz})
            SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
        for (int ch = C - 1; ch >= 0; --ch) {
            const int it0 = ch * k, it1 = std::min(d->nt, it0 + k);
            FwdState S;
            S.px = fw.psix; S.pz = fw.psiz; S.pxn = fw.psixn; S.pzn = fw.psizn;
            if (ch == 0) {
                for (auto* p : {fw.u[0], fw.u[1], fw.psix, fw.psiz, fw.zetax, fw.zetaz})
                    SWEEP_CUDA(cudaMemsetAsync(p, 0, n * 4, st));
            } else {
                float* state[kStateFields] = {fw.u[0], fw.u[1], fw.psix, fw.psiz, fw.zetax, fw.zetaz};
                for (int f = 0; f < kStateFields; ++f) copy_dd(state[f], ckpt_field(tp, pl, ch, f), n, st);
                copy_dd(chunk, ckpt_strips(tp, pl, ch), cs, st);          // strips of U[it0 - 1]
            }
            // replay: chunk slot j holds the strips of U[it0 - 1 + j]
            forward_steps(pl, fmaps, fw, nullptr, S, it0, it1,
                          [&](int it) { return chunk + (long long)(it - it0 + 1) * cs; }, st);
            copy_dd(w.r[0], fw.u[S.in], n, st);       // U[it1]
            copy_dd(w.r[1], fw.u[S.ip], n, st);       // U[it1 - 1]
            reverse(it0, it1, [&](int t) { return chunk + (long long)(t - (it0 - 1)) * cs; }, true);
        }
    }
    if (stepped) {
        const int keep[7] = {lp, ln, lx, cur, rp, rn, rx};
        for (int k = 0; k < 7; ++k) seg->idx[k] = keep[k];
    }
    const int nout = P.per_shot ? d->B : 1;
    finalize_kernel<<<1184, 256, 0, st>>>(w.gacc, w.gcomp, w.is, w.ir, pl.nslot, nout, d->nz, d->nx, P.P,
                                          grad_vp, illum_s, illum_r);
    SWEEP_LAUNCH_CHECK();
    check_err(w.c, st, "backward");
}

void backward(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
              float* grad_vp, float* grad_w, float* illum_s, float* illum_r,
              void* ws, int64_t ws_bytes, cudaStream_t st)
{
    backward_with(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_w, illum_s, illum_r, ws, ws_bytes, st, nullptr,
                  0, 0);
}

void backward_segment(const sweep_acoustic_desc* d, int mem_mode, const float* adj, const void* tape,
                      float* grad_vp, float* grad_w, float* illum_s, float* illum_r, void* ws, int64_t ws_bytes,
                      cudaStream_t st, StepState& seg, int bw0, int bw1)
{
    backward_with(d, mem_mode, 0, adj, tape, grad_vp, grad_w, illum_s, illum_r, ws, ws_bytes, st, &seg, bw0, bw1);
}

}  // namespace a2d
}  // namespace sweep
