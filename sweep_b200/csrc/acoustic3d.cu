// acoustic3d.cu -- 3-D constant-density acoustic propagation on B200 (sm_100a):
// 8th-order-in-space / 2nd-order-in-time leapfrog with CPML, exact adjoint,
// boundary-saving reconstruction and vp imaging.
//
// Numerics follow the reference's compiled path (impl='c'):
//   forward step       reference src/sweep/csrc/cuda/equations/acoustic3d/forward_split.cu:79-290
//                      (interior; CPML shell with the product-rule split
//                      a * d(psi) + d(a) * psi on the band plus one cell)
//   adjoint step       reference .../acoustic3d/adjoint_split.cu:14-320
//   reconstruction     reference .../acoustic3d/forward_split.cu:292-372
//   reverse step order reference .../acoustic3d/driver_traits.cuh:481-590
//
// Schedule (the B200 part): the stencil kernels stream along z.  A CTA owns a
// 32 x 8 block of (x, y) columns for one shot; each thread keeps the nine
// z-taps of its column in a register queue and reads the x / y taps from a
// shared-memory plane (with its 4-cell halo) that is loaded one plane ahead
// while the current plane computes.  Every field is pitched (x rows of
// P = round_up(nx, 32) floats).  Point sources, receivers and boundary strips
// are small gather / scatter kernels between the stencil launches.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <functional>

#include "common.cuh"
#include "tma.cuh"

namespace sweep {
namespace a3d {

constexpr int M = 4;
// Ring depths and CTAs per SM of the three stencil kernels: build-time knobs
// (the shared-memory ring and the L1 share the same on-chip memory).
#ifndef SWEEP_A3D_FWD_STAGES
#define SWEEP_A3D_FWD_STAGES 11
#endif
#ifndef SWEEP_A3D_ADJ_STAGES
#define SWEEP_A3D_ADJ_STAGES 8
#endif
#ifndef SWEEP_A3D_REC_STAGES
#define SWEEP_A3D_REC_STAGES 9
#endif
#ifndef SWEEP_A3D_CTAS
#define SWEEP_A3D_CTAS 4
#endif
constexpr int BXC = 32;                        // columns per CTA along x
constexpr int PW = BXC + 2 * M;                // staged plane width, floats
// A CTA covers BXC x BY columns; BY (8 or 16) is the schedule's tile height.
template <int BY>
struct TileY {
    static constexpr int PH = BY + 2 * M;      // staged plane height
    static constexpr int PN = PW * PH;         // staged plane, floats
    static constexpr int NT = BXC * BY;        // threads per CTA
    static constexpr int CN = BXC * BY;        // centre tile, floats
    static constexpr int CTAS = SWEEP_A3D_CTAS * 8 / BY;   // CTAs per SM
};

// Boundary-strip storage of the boundary-saving tape.  fp32 and bf16 keep the
// strip set (each cell once, strip_coord order); fp16 and int8 keep the
// reference's six faces (z faces across the box, y faces down the whole box,
// x faces through it; edges in two or three faces), each quantised per shot
// in blocks of kQB cells against the block's max |value| (reference
// boundarysaver.cu:207-330 face layout, 906-1100 quantisation).
enum StripFmt { SF_F32 = 0, SF_F16 = 1, SF_BF16 = 2, SF_I8 = 3 };
constexpr int kQB = 256;

struct StripStore {
    int fmt;                         // StripFmt
    int w;                           // face band width (M + 1)
    int cells[6], blocks[6];         // per shot and face (top, bottom, front, back, left, right)
    long long pay[6], scl[6];        // byte offsets of each face's codes and scales in a step slot
    long long step;                  // bytes of one step slot
    int host;                        // the tape is pinned host memory (SWEEP_MEM_HOST_TAPE)
};

constexpr int kMaxXBlocks = 48;
constexpr int kMaxYBlocks = 160;

struct Params {
    int B, nz, ny, nx, nt, nsrc, nrec;
    int P;                                     // x pitch (floats)
    long long SP, S;                           // plane stride, shot stride
    int zc, nzc;                               // z chunk length, chunks
    int rows;                                  // rows of a stencil CTA (tile height: 8 or 16)
    int graph_steps;                           // host only: time steps per captured CUDA graph
    float dt, dz, dy, dx;
    float ih2z, ih2y, ih2x;                    // 1 / h^2 per axis
    float ihz, ihy, ihx;                       // 1 / h per axis
    float lc[M + 1], gc[M + 1];
    int z0, z1, y0, y1, x0, x1;                // physical box
    int ex0, ex1, ey0, ey1, ez0, ez1;          // forward CPML branch: ix < ex0 || ix >= ex1 ...
    int qx0, qx1, qy0, qy1, qz0, qz1;          // adjoint clear box / reconstruction box
    int wzl, wzh, wyl, wyh, wxl, wxh;          // strip widths
    long long n_top, n_bot, nring, nstrip;
    const float *az, *bz, *dbz, *ay, *by, *dby, *ax, *bx, *dbx;
    // the same profiles packed per index as {a, b, d b / d axis, d a / d axis}
    // (one 16-byte load per neighbour in the CPML terms); d a / d axis is the
    // centred derivative grad_p(a + i) on [M, n - M), 0 outside
    const float4 *pz, *py, *px;
    const float *cf, *ca, *vv;                 // model fields, pitched (one copy: shared model)
    const int* soff;                           // strip cell -> its offset in a shot's field (strip_coord, tabled)
    StripStore st;
    // x tiling of the forward (0) and adjoint (1) stencil grids: column block
    // b starts at x = xo[k][b] (a multiple of 4, for the TMA row origin) and
    // updates only the columns it owns, [xl[k][b], xh[k][b]); the blocks own
    // [M, nx - M) exactly once, each lies wholly in the CPML x band or wholly
    // clear of it, so no warp of a clear block takes the band path
    int nbx[2];
    short xo[2][kMaxXBlocks], xl[2][kMaxXBlocks], xh[2][kMaxXBlocks];
    // the same along y with 8-row blocks (a row origin needs no alignment)
    int nby[2];
    short yo[2][kMaxYBlocks], yl[2][kMaxYBlocks], yh[2][kMaxYBlocks];
};

// ------------------------------------------------------------------ device
__device__ __forceinline__ float tap(float uk, float u0) { return __fsub_rn(uk, u0); }

// difference-form Laplacian at p along stride st (reference laplace.cuh:327-380),
// scaled by ih2 = 1 / h^2
__device__ __forceinline__ float lap_p(const float* p, long long st, const Params& P, float ih2)
{
    const float u0 = p[0];
    float acc = P.lc[1] * (tap(p[-st], u0) + tap(p[st], u0));
    acc = acc + P.lc[2] * (tap(p[-2 * st], u0) + tap(p[2 * st], u0));
    acc = acc + P.lc[3] * (tap(p[-3 * st], u0) + tap(p[3 * st], u0));
    acc = acc + P.lc[4] * (tap(p[-4 * st], u0) + tap(p[4 * st], u0));
    return acc * ih2;
}

// the same on a register queue q[0..8] (q[4] the centre)
__device__ __forceinline__ float lap_q(const float* q, const Params& P, float ih2)
{
    const float u0 = q[M];
    float acc = P.lc[1] * (tap(q[M - 1], u0) + tap(q[M + 1], u0));
    acc = acc + P.lc[2] * (tap(q[M - 2], u0) + tap(q[M + 2], u0));
    acc = acc + P.lc[3] * (tap(q[M - 3], u0) + tap(q[M + 3], u0));
    acc = acc + P.lc[4] * (tap(q[M - 4], u0) + tap(q[M + 4], u0));
    return acc * ih2;
}

// centred first derivative at p along stride st (reference gradient.cuh:49-88),
// scaled by ih = 1 / h
__device__ __forceinline__ float grad_p(const float* p, long long st, const Params& P, float ih)
{
    float acc = P.gc[1] * (p[st] - p[-st]);
    acc = acc + P.gc[2] * (p[2 * st] - p[-2 * st]);
    acc = acc + P.gc[3] * (p[3 * st] - p[-3 * st]);
    acc = acc + P.gc[4] * (p[4 * st] - p[-4 * st]);
    return acc * ih;
}

// the same on a read-only global field (non-coherent cache path)
__device__ __forceinline__ float grad_g(const float* __restrict__ p, long long st, const Params& P, float ih)
{
    float acc = P.gc[1] * (__ldg(p + st) - __ldg(p - st));
    acc = acc + P.gc[2] * (__ldg(p + 2 * st) - __ldg(p - 2 * st));
    acc = acc + P.gc[3] * (__ldg(p + 3 * st) - __ldg(p - 3 * st));
    acc = acc + P.gc[4] * (__ldg(p + 4 * st) - __ldg(p - 4 * st));
    return acc * ih;
}

__device__ __forceinline__ float grad_q(const float* q, const Params& P, float ih)
{
    float acc = P.gc[1] * (q[M + 1] - q[M - 1]);
    acc = acc + P.gc[2] * (q[M + 2] - q[M - 2]);
    acc = acc + P.gc[3] * (q[M + 3] - q[M - 3]);
    acc = acc + P.gc[4] * (q[M + 4] - q[M - 4]);
    return acc * ih;
}

// strip cell s -> (iz, iy, ix): z faces (full x-y), y faces over the inner z
// planes, x faces over the inner z planes and inner y rows
__device__ __forceinline__ void strip_coord(const Params& P, long long s, int& iz, int& iy, int& ix)
{
    const int bx = P.x1 - P.x0, by = P.y1 - P.y0;
    const long long pl = (long long)bx * by;
    if (s < P.n_top) {
        iz = P.z0 + (int)(s / pl); const long long r = s % pl; iy = P.y0 + (int)(r / bx); ix = P.x0 + (int)(r % bx);
        return;
    }
    s -= P.n_top;
    if (s < P.n_bot) {
        iz = P.z1 - P.wzh + (int)(s / pl); const long long r = s % pl; iy = P.y0 + (int)(r / bx); ix = P.x0 + (int)(r % bx);
        return;
    }
    s -= P.n_bot;
    iz = P.z0 + P.wzl + (int)(s / P.nring);
    long long r = s % P.nring;
    if (r < (long long)P.wyl * bx) { iy = P.y0 + (int)(r / bx); ix = P.x0 + (int)(r % bx); return; }
    r -= (long long)P.wyl * bx;
    if (r < (long long)P.wyh * bx) { iy = P.y1 - P.wyh + (int)(r / bx); ix = P.x0 + (int)(r % bx); return; }
    r -= (long long)P.wyh * bx;
    const int ww = P.wxl + P.wxh;
    iy = P.y0 + P.wyl + (int)(r / ww);
    const int c = (int)(r % ww);
    ix = c < P.wxl ? P.x0 + c : P.x1 - P.wxh + (c - P.wxl);
}

// Inverse of strip_coord: the strip-set index of a strip cell.
__device__ __forceinline__ long long strip_index3(const Params& P, int iz, int iy, int ix)
{
    const long long bx = P.x1 - P.x0, by = P.y1 - P.y0;
    if (iz < P.z0 + P.wzl) return ((long long)(iz - P.z0) * by + (iy - P.y0)) * bx + (ix - P.x0);
    if (iz >= P.z1 - P.wzh) return P.n_top + ((long long)(iz - (P.z1 - P.wzh)) * by + (iy - P.y0)) * bx + (ix - P.x0);
    long long s = P.n_top + P.n_bot + (long long)(iz - (P.z0 + P.wzl)) * P.nring;
    if (iy < P.y0 + P.wyl) return s + (long long)(iy - P.y0) * bx + (ix - P.x0);
    s += (long long)P.wyl * bx;
    if (iy >= P.y1 - P.wyh) return s + (long long)(iy - (P.y1 - P.wyh)) * bx + (ix - P.x0);
    s += (long long)P.wyh * bx;
    const int ww = P.wxl + P.wxh;
    return s + (long long)(iy - (P.y0 + P.wyl)) * ww + (ix < P.x0 + P.wxl ? ix - P.x0 : P.wxl + ix - (P.x1 - P.wxh));
}

// Face f (0 top, 1 bottom, 2 front, 3 back, 4 left, 5 right) cell `idx` of
// the scaled formats -> grid cell (z faces (width, box y, box x); y faces
// (box z, width, box x); x faces (box z, box y, width)).
__device__ __forceinline__ void face_cell3(const Params& P, int f, long long idx, int& iz, int& iy, int& ix)
{
    const int w = P.st.w, bx = P.x1 - P.x0, by = P.y1 - P.y0;
    if (f < 2) {
        ix = P.x0 + (int)(idx % bx); idx /= bx;
        iy = P.y0 + (int)(idx % by);
        iz = (f == 0 ? P.z0 : P.z1 - w) + (int)(idx / by);
    } else if (f < 4) {
        ix = P.x0 + (int)(idx % bx); idx /= bx;
        iy = (f == 2 ? P.y0 : P.y1 - w) + (int)(idx % w);
        iz = P.z0 + (int)(idx / w);
    } else {
        ix = (f == 4 ? P.x0 : P.x1 - w) + (int)(idx % w); idx /= w;
        iy = P.y0 + (int)(idx % by);
        iz = P.z0 + (int)(idx / by);
    }
}

// The face a scaled-format restore reads strip cell (iz, iy, ix) from: the
// last of the faces holding it in the reference's restore order (top, bottom,
// front, back, left, right).
__device__ __forceinline__ long long face_index3(const Params& P, int iz, int iy, int ix, int& f)
{
    const int w = P.st.w, bx = P.x1 - P.x0, by = P.y1 - P.y0;
    if (ix >= P.x1 - w) { f = 5; return ((long long)(iz - P.z0) * by + (iy - P.y0)) * w + (ix - (P.x1 - w)); }
    if (ix < P.x0 + w) { f = 4; return ((long long)(iz - P.z0) * by + (iy - P.y0)) * w + (ix - P.x0); }
    if (iy >= P.y1 - w) { f = 3; return ((long long)(iz - P.z0) * w + (iy - (P.y1 - w))) * bx + (ix - P.x0); }
    if (iy < P.y0 + w) { f = 2; return ((long long)(iz - P.z0) * w + (iy - P.y0)) * bx + (ix - P.x0); }
    if (iz >= P.z1 - w) { f = 1; return ((long long)(iz - (P.z1 - w)) * by + (iy - P.y0)) * bx + (ix - P.x0); }
    f = 0;
    return ((long long)(iz - P.z0) * by + (iy - P.y0)) * bx + (ix - P.x0);
}

__device__ __forceinline__ bool in_phys(const Params& P, int iz, int iy, int ix)
{
    return iz >= P.z0 && iz < P.z1 && iy >= P.y0 && iy < P.y1 && ix >= P.x0 && ix < P.x1;
}

__device__ __forceinline__ bool in_recon(const Params& P, int iz, int iy, int ix)
{
    return iz >= P.qz0 && iz < P.qz1 && iy >= P.qy0 && iy < P.qy1 && ix >= P.qx0 && ix < P.qx1;
}

// ----------------------------------------------------------- forward step
struct F3 {
    const float* u_now; const float* u_prev; float* u_next;
    const float *psx, *psy, *psz;              // CPML psi (read)
    float *psxn, *psyn, *pszn;                 // CPML psi (written)
    float *zx, *zy, *zz;                       // CPML zeta (in place)
};

// Forward plane ring: stage q holds the wavefield plane u(q) with its x / y
// halo, and the centre tiles of u_prev(q - M) and of the model for plane
// q - M.  Each thread keeps the nine z-taps of its column in a register
// queue: plane z reads its x / y taps from stage z and pushes the centre of
// stage z + M into the queue, so stages z .. z + M must have landed; with NF3
// stages the loads run NF3 - M - 1 planes ahead of the compute, TMA-issued by
// one thread on one mbarrier per stage.
constexpr int NF3 = SWEEP_A3D_FWD_STAGES;
static_assert(NF3 >= 2 * M + 1, "the forward ring must hold the first plane's z-taps and one more stage");
template <int BY>
struct F3Smem {
    float u[NF3][TileY<BY>::PN];
    float up[NF3][TileY<BY>::CN];
    float cf[NF3][TileY<BY>::CN];
    uint64_t bar[NF3];
};

struct F3Maps {
    CUtensorMap uh[3];              // the three wavefield buffers, (PW x PH) boxes
    CUtensorMap uc[3];              // the same buffers, (BXC x BYC) boxes
    CUtensorMap cf;                 // ((v*v)*dt)*dt, (BXC x BYC) boxes
};

enum { ERR_WAIT_F3 = 1 };

// u_next = 2 u - u_prev + vp^2 dt^2 (Lap u + CPML terms) on [M, n-M)^3.
// The CPML branch of an axis runs on its band plus one cell (reference
// forward_split.cu:150-156) and uses the product-rule split
// tmp = (((1 + b) Lap + db du) + a dpsi) + da psi (forward_split.cu:171-172).
template <int BY>
__global__ void __launch_bounds__(TileY<BY>::NT, TileY<BY>::CTAS)
    f3_step(const __grid_constant__ F3Maps MP, const Params P, const F3 F, const int uin, const int uprev, int* err)
{
    constexpr int PN = TileY<BY>::PN, CN3 = TileY<BY>::CN;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    F3Smem<BY>& sm = *reinterpret_cast<F3Smem<BY>*>(smem_raw);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BXC + tx;
    const int xb = P.xo[0][blockIdx.x], yb = P.yo[0][blockIdx.y];
    const int gx0 = xb - M, gy0 = yb - M;
    const int ix = xb + tx, iy = yb + ty;
    const int b = blockIdx.z / P.nzc, zci = blockIdx.z - b * P.nzc;
    const int zb = max(M, zci * P.zc), ze = min(P.nz - M, (zci + 1) * P.zc);
    if (zb >= ze) return;
    const bool col = ix >= P.xl[0][blockIdx.x] && ix < P.xh[0][blockIdx.x] && iy >= P.yl[0][blockIdx.y] &&
                     iy < P.yh[0][blockIdx.y];
    const long long bo = (long long)b * P.S;
    const long long colo = (long long)iy * P.P + ix;
    const int q0 = zb - M, q1 = ze + M;                // stages [q0, q1)
    auto slot = [&](int q) { return (q - q0) % NF3; };
    auto parity = [&](int q) { return (uint32_t)(((q - q0) / NF3) & 1); };
    auto issue = [&](int q) {
        const int sl = slot(q);
        const bool cen = q - M >= zb && q - M < ze;     // u_prev / model of plane q - M
        tma::mbar_expect_tx(&sm.bar[sl], (uint32_t)(PN + (cen ? 2 * CN3 : 0)) * 4u);
        tma::load_4d(sm.u[sl], &MP.uh[uin], &sm.bar[sl], gx0, gy0, q, b);
        if (cen) {
            tma::load_4d(sm.up[sl], &MP.uc[uprev], &sm.bar[sl], gx0 + M, gy0 + M, q - M, b);
            tma::load_3d(sm.cf[sl], &MP.cf, &sm.bar[sl], gx0 + M, gy0 + M, q - M);
        }
    };
    if (tid == 0) {
        for (int i = 0; i < NF3; ++i) tma::mbar_init(&sm.bar[i], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    int next = q0;                                     // first stage not yet issued (thread 0)
    if (tid == 0)
        for (; next < min(q1, q0 + NF3); ++next) issue(next);
    // a failed wait: drain (bounded) every stage still in flight, then exit
    auto fail = [&](int q) {
        if (tid == 0)
            for (int r = q; r < next; ++r) tma::mbar_wait(&sm.bar[slot(r)], parity(r), err, ERR_WAIT_F3);
    };
    // Each thread waits for the stages it reads itself; a failed wait is
    // noted and the whole CTA leaves at the end of that plane, at the one
    // block barrier a plane has (results are then invalid and the host
    // reports the error).  Leaving, thread 0 waits (bounded) for every stage
    // still in flight: from q0 at the first plane (no slot reused yet), else
    // from z + M (every earlier stage was waited for at an earlier plane).
    bool bad = false;
    auto await = [&](int q) {
        if (!tma::mbar_wait(&sm.bar[slot(q)], parity(q), err, ERR_WAIT_F3)) bad = true;
    };
    const int cidx = (ty + M) * PW + (tx + M), cc = ty * BXC + tx;
    // the z-queue: u of planes z - M .. z + M at this column (q[M] the centre)
    float q[2 * M + 1];
#pragma unroll
    for (int k = 0; k < 2 * M; ++k) {
        await(q0 + k);
        q[k] = sm.u[slot(q0 + k)][cidx];
    }
    // rolling slots of stages z and z + M and the phase of z + M
    int sz = M % NF3, sq = (2 * M) % NF3;
    uint32_t ph = (uint32_t)(((2 * M) / NF3) & 1);
    const bool inx = ix < P.ex0 || ix >= P.ex1;
    const bool iny = iy < P.ey0 || iy >= P.ey1;
    long long i = bo + (long long)zb * P.SP + colo;
    for (int z = zb; z < ze; ++z, i += P.SP) {
        if (!tma::mbar_wait(&sm.bar[sq], ph, err, ERR_WAIT_F3)) bad = true;
        q[2 * M] = sm.u[sq][cidx];
        if (col) {
            const float* p = sm.u[sz] + cidx;
            const float lx = lap_p(p, 1, P, P.ih2x);
            const float ly = lap_p(p, PW, P, P.ih2y);
            const float lz = lap_q(q, P, P.ih2z);
            const bool inz = z < P.ez0 || z >= P.ez1;
            float w;
            if (!inx && !iny && !inz) {
                w = (lx + ly) + lz;
            } else {
                w = 0.f;
                if (inx) {
                    const float du = grad_p(p, 1, P, P.ihx);
                    const float dps = grad_g(F.psx + i, 1, P, P.ihx);
                    const float4 pr = __ldg(P.px + ix);
                    const float a = pr.x, bb = pr.y, db = pr.z, da = pr.w;
                    const float ps = __ldg(F.psx + i), zt = F.zx[i];
                    const float tmp = (((1.f + bb) * lx + db * du) + a * dps) + da * ps;
                    w += (1.f + bb) * tmp + a * zt;
                    F.psxn[i] = bb * du + a * ps;
                    F.zx[i] = bb * tmp + a * zt;
                } else {
                    w += lx;
                }
                if (iny) {
                    const float du = grad_p(p, PW, P, P.ihy);
                    const float dps = grad_g(F.psy + i, P.P, P, P.ihy);
                    const float4 pr = __ldg(P.py + iy);
                    const float a = pr.x, bb = pr.y, db = pr.z, da = pr.w;
                    const float ps = __ldg(F.psy + i), zt = F.zy[i];
                    const float tmp = (((1.f + bb) * ly + db * du) + a * dps) + da * ps;
                    w += (1.f + bb) * tmp + a * zt;
                    F.psyn[i] = bb * du + a * ps;
                    F.zy[i] = bb * tmp + a * zt;
                } else {
                    w += ly;
                }
                if (inz) {
                    const float du = grad_q(q, P, P.ihz);
                    const float dps = grad_g(F.psz + i, P.SP, P, P.ihz);
                    const float4 pr = __ldg(P.pz + z);
                    const float a = pr.x, bb = pr.y, db = pr.z, da = pr.w;
                    const float ps = __ldg(F.psz + i), zt = F.zz[i];
                    const float tmp = (((1.f + bb) * lz + db * du) + a * dps) + da * ps;
                    w += (1.f + bb) * tmp + a * zt;
                    F.pszn[i] = bb * du + a * ps;
                    F.zz[i] = bb * tmp + a * zt;
                } else {
                    w += lz;
                }
            }
            F.u_next[i] = 2.f * q[M] - sm.up[sq][cc] + sm.cf[sq][cc] * w;
        }
#pragma unroll
        for (int k = 0; k < 2 * M; ++k) q[k] = q[k + 1];
        sz = sz + 1 == NF3 ? 0 : sz + 1;
        if (++sq == NF3) { sq = 0; ph ^= 1u; }
        // every thread is done with stage z and has waited for z + M
        if (__syncthreads_or(bad)) { fail(z == zb ? q0 : z + M); return; }
        if (tid == 0)
            for (; next < q1 && next <= z + NF3; ++next) issue(next);     // slots of stages <= z are free
    }
}

// ------------------------------------------------- point events and strips
// A coordinate in the outer stencil halo (never updated) counts as off the grid.
__device__ __forceinline__ bool event_cell(const Params& P, const int* loc, long long e, long long& off)
{
    const int x = loc[3 * e], y = loc[3 * e + 1], z = loc[3 * e + 2];
    if (x < M || x >= P.nx - M || y < M || y >= P.ny - M || z < M || z >= P.nz - M) return false;
    off = (long long)z * P.SP + (long long)y * P.P + x;
    return true;
}

// u[b, cell] += sign * amplitude of event (b, s) at step it.  rec_layout: the
// amplitudes are a record cotangent (B, nt, n); else a wavelet (B, n, nt).
// strip_only: only events whose cell lies in the restored boundary strips.
__global__ void inject3(const Params P, float* __restrict__ u, const float* __restrict__ amp,
                        const int* __restrict__ loc, int n, int it, int rec_layout, float sign, int strip_only)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)P.B * n) return;
    const int b = (int)(e / n), s = (int)(e - (long long)b * n);
    long long off;
    if (!event_cell(P, loc, e, off)) return;
    if (strip_only) {
        const int x = loc[3 * e], y = loc[3 * e + 1], z = loc[3 * e + 2];
        if (!in_phys(P, z, y, x) || in_recon(P, z, y, x)) return;
    }
    const float a = rec_layout ? amp[((long long)b * P.nt + it) * n + s] : amp[((long long)b * n + s) * P.nt + it];
    atomicAdd(u + (long long)b * P.S + off, sign * a);
}

// out[b, it, r] = u[b, cell]  (record layout)  or  out[b, s, it] = u[b, cell]
// (wavelet-gradient layout)
__global__ void gather3(const Params P, const float* __restrict__ u, float* __restrict__ out,
                        const int* __restrict__ loc, int n, int it, int rec_layout)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)P.B * n) return;
    const int b = (int)(e / n), s = (int)(e - (long long)b * n);
    long long off;
    if (!event_cell(P, loc, e, off)) return;
    const float v = u[(long long)b * P.S + off];
    if (rec_layout) out[((long long)b * P.nt + it) * n + s] = v;
    else out[((long long)b * n + s) * P.nt + it] = v;
}

// boundary strips: save (slot <- u; the scaled formats into `scratch`, for
// quantise_strips3) or restore (u <- slot, dequantised as the reference does:
// fp16 code x scale; int8 (code - 128) x scale / 127), every shot
__global__ void strips3(const Params P, float* __restrict__ u, void* slot, float* __restrict__ scratch, int restore)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)P.B * P.nstrip) return;
    const int b = (int)(e / P.nstrip);
    const long long sidx = e - (long long)b * P.nstrip;
    float* c = u + (long long)b * P.S + __ldg(P.soff + sidx);
    const StripStore& S = P.st;
    if (!restore) {
        if (S.fmt == SF_F32) static_cast<float*>(slot)[e] = *c;
        else if (S.fmt == SF_BF16) static_cast<__nv_bfloat16*>(slot)[e] = __float2bfloat16(*c);
        else scratch[e] = *c;
        return;
    }
    if (S.fmt == SF_F32) { *c = static_cast<const float*>(slot)[e]; return; }
    if (S.fmt == SF_BF16) { *c = __bfloat162float(static_cast<const __nv_bfloat16*>(slot)[e]); return; }
    int iz, iy, ix, f;
    strip_coord(P, sidx, iz, iy, ix);
    const long long i = face_index3(P, iz, iy, ix, f);
    const char* base = static_cast<const char*>(slot);
    const float scale = reinterpret_cast<const float*>(base + S.scl[f])[(long long)b * S.blocks[f] + i / kQB];
    const long long q = (long long)b * S.cells[f] + i;
    if (S.fmt == SF_F16) {
        *c = __half2float(reinterpret_cast<const __half*>(base + S.pay[f])[q]) * scale;
    } else {
        const float sc = scale * (1.0f / 127.0f);
        *c = ((float)reinterpret_cast<const uint8_t*>(base + S.pay[f])[q] - 128.0f) * sc;
    }
}

// One step's strips (fp32 strip set in `scratch`) into the scaled faces of a
// step slot: one CTA per (shot, face, block of kQB cells) -- max |value| of
// the block, its scale, the codes (reference boundarysaver.cu:957-990,
// 1050-1080: int8 round(v 127 / max) + 128 clamped to [0, 255]; fp16 v / max).
__global__ void __launch_bounds__(kQB) quantize_strips3(const Params P, const float* __restrict__ scratch, void* slot)
{
    const StripStore& S = P.st;
    int per = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) per += S.blocks[f];
    const int b = blockIdx.x / per;
    int j = blockIdx.x - b * per, f = 0;
    while (f < 5 && j >= S.blocks[f]) { j -= S.blocks[f]; ++f; }
    const long long idx = (long long)j * kQB + threadIdx.x;
    const bool in = idx < S.cells[f];
    float v = 0.f;
    if (in) {
        int iz, iy, ix;
        face_cell3(P, f, idx, iz, iy, ix);
        v = scratch[(long long)b * P.nstrip + strip_index3(P, iz, iy, ix)];
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
    const long long q = (long long)b * S.cells[f] + idx;
    if (S.fmt == SF_F16) {
        const float inv = m > 0.0f ? 1.0f / m : 0.0f;
        reinterpret_cast<__half*>(base + S.pay[f])[q] = __float2half(v * inv);
    } else {
        const float qs = m > 0.0f ? 127.0f / m : 0.0f;
        int c = __float2int_rn(v * qs) + 128;
        c = c < 0 ? 0 : (c > 255 ? 255 : c);
        reinterpret_cast<uint8_t*>(base + S.pay[f])[q] = (uint8_t)c;
    }
}

__device__ __forceinline__ void kahan_add(float* acc, float* comp, long long o, float g)
{
    const float y = g - comp[o];
    const float t = acc[o] + y;
    comp[o] = (t - acc[o]) - y;
    acc[o] = t;
}

struct Img {
    const float *r_prev, *r_now, *r_next, *lam;   // u(it+1), u(it), u(it-1) - s(it), lambda(it)
    float *gacc, *gcomp, *is, *ir;              // per-shot slots (B, S)
};

// vp imaging of the strip cells (reference acoustic2d/kernels.cu:83-131; the
// 3-D twin acoustic3d/kernels.cu), after the restore and the strip-source removal
__global__ void strip_image3(const Params P, const Img I)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)P.B * P.nstrip) return;
    const int b = (int)(e / P.nstrip);
    const long long c = __ldg(P.soff + (e - (long long)b * P.nstrip));
    const long long o = (long long)b * P.S + c;
    const float dt2 = P.dt * P.dt;
    const float utt = (I.r_next[o] - 2 * I.r_now[o] + I.r_prev[o]) / dt2;
    const float lam = I.lam[o];
    kahan_add(I.gacc, I.gcomp, o, 2.f * P.dt * P.dt * utt * lam / __ldg(P.vv + c));
    if (I.is) { I.is[o] += utt * utt; I.ir[o] += lam * lam; }
}

// ------------------------------------------------------------ adjoint step
// gw = ((v*v)*dt^2) * lambda is the tap value of the adjoint Laplacian
// (reference adjoint_split.cu GW_AT).

struct A3 {
    const float* l_now; const float* l_prev; float* l_next;
    const float *px, *py, *pz, *zx, *zy, *zz;          // adjoint CPML memories (read)
    float *pxo, *pyo, *pzo, *zxo, *zyo, *zzo;          // (written)
};

// The transposed CPML terms of one axis at linear offset i, stride st,
// packed profiles pr = {a, b, db, da} at axis index c (reference
// adjoint_split.cu:205-255).  g: gw = ((v*v)*dt^2) * lambda at the 2M+1
// cells along the axis around i (g[M] at i, from shared memory or the
// z-queue).
__device__ __forceinline__ void adj_axis(const Params& P, const float4* __restrict__ pr,
                                         const float (&g)[2 * M + 1], const float* __restrict__ psi,
                                         const float* __restrict__ zeta, long long i, long long st, int c,
                                         float ih2, float ih, float& L, float& Dg, float* pso, float* zto)
{
    const float gw = g[M];
    const float4 p0 = __ldg(pr + c);
    const float a_ = p0.x, b_ = p0.y, da = p0.w;
    const float* zp = zeta + i;
    const float* pp_ = psi + i;
    const float z0 = __ldg(zp);
    const float gt0 = b_ * z0 + (1.0f + b_) * gw;
    const float l0 = (1.0f + b_) * gt0;
    float Lq = 0.0f, Dgg = 0.0f, Dq = 0.0f;
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        const float4 pp = __ldg(pr + c + k), pm = __ldg(pr + c - k);
        const float bp = pp.y, bm = pm.y;
        const float tp = bp * __ldg(zp + k * st) + (1.0f + bp) * g[M + k];
        const float tm = bm * __ldg(zp - k * st) + (1.0f + bm) * g[M - k];
        Lq += P.lc[k] * (tap((1.0f + bp) * tp, l0) + tap((1.0f + bm) * tm, l0));
        Dgg += P.gc[k] * ((bp * __ldg(pp_ + k * st) + pp.z * tp) - (bm * __ldg(pp_ - k * st) + pm.z * tm));
        Dq += P.gc[k] * (pp.x * tp - pm.x * tm);
    }
    L = Lq * ih2;
    Dg = Dgg * ih;
    Dq = Dq * ih;
    pso[i] = (a_ * __ldg(pp_) + da * gt0) - Dq;
    zto[i] = a_ * (z0 + gw);
}

// Adjoint plane ring: stage q holds lambda(q) and (v*v)*dt^2 of plane q with
// their x / y halo, and lambda(it+1) of plane q - M.  Each thread keeps
// gw = ((v*v)*dt^2) * lambda of the nine z-taps of its column in a register
// queue (plane z pushes the centre of stage z + M), and the CTA forms the gw
// plane of the next plane's x / y taps once, in a double buffer, at the end
// of each plane.  Stages z .. z + M must have landed at plane z; with NA3
// stages the loads run NA3 - M - 1 planes ahead.
constexpr int NA3 = SWEEP_A3D_ADJ_STAGES;
static_assert(NA3 >= 2 * M, "the adjoint ring must hold the 2M stages of the first plane's z-queue");

template <int BY>
struct A3Smem {
    float l[NA3][TileY<BY>::PN];
    float c[NA3][TileY<BY>::PN];
    float lp[NA3][TileY<BY>::CN];
    float gw[2][TileY<BY>::PN];
    uint64_t bar[NA3];
};

struct A3Maps {
    CUtensorMap lh[3];              // lambda buffers, (PW x PH) boxes
    CUtensorMap lc[3];              // the same, centre boxes
    CUtensorMap ch;                 // (v*v)*(dt*dt), (PW x PH) boxes
};

// lambda_next = exact transpose of the forward step (reference adjoint_split.cu:14-320):
// pure interior  2 l - l_prev + Lap(gw) (difference form around gw);
// shell          per axis outside the clear box the transposed CPML terms,
//                inside it the bare Laplacian of gw.
template <int BY>
__global__ void __launch_bounds__(TileY<BY>::NT, TileY<BY>::CTAS)
    a3_step(const __grid_constant__ A3Maps MP, const Params P, const A3 A, const int lnow, const int lprev, int* err)
{
    constexpr int PN = TileY<BY>::PN, CN3 = TileY<BY>::CN, NTH = TileY<BY>::NT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    A3Smem<BY>& sm = *reinterpret_cast<A3Smem<BY>*>(smem_raw);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BXC + tx;
    const int xb = P.xo[1][blockIdx.x], yb = P.yo[1][blockIdx.y];
    const int gx0 = xb - M, gy0 = yb - M;
    const int ix = xb + tx, iy = yb + ty;
    const int b = blockIdx.z / P.nzc, zci = blockIdx.z - b * P.nzc;
    const int zb = max(M, zci * P.zc), ze = min(P.nz - M, (zci + 1) * P.zc);
    if (zb >= ze) return;
    const bool col = ix >= P.xl[1][blockIdx.x] && ix < P.xh[1][blockIdx.x] && iy >= P.yl[1][blockIdx.y] &&
                     iy < P.yh[1][blockIdx.y];
    const long long bo = (long long)b * P.S;
    const long long colo = (long long)iy * P.P + ix;
    const bool inx = ix < P.qx0 || ix >= P.qx1;
    const bool iny = iy < P.qy0 || iy >= P.qy1;
    const int q0 = zb - M, q1 = ze + M;
    auto slot = [&](int q) { return (q - q0) % NA3; };
    auto parity = [&](int q) { return (uint32_t)(((q - q0) / NA3) & 1); };
    auto issue = [&](int q) {
        const int sl = slot(q), z = q - M;
        const bool cen = z >= zb && z < ze;
        tma::mbar_expect_tx(&sm.bar[sl], (uint32_t)(2 * PN + (cen ? CN3 : 0)) * 4u);
        tma::load_4d(sm.l[sl], &MP.lh[lnow], &sm.bar[sl], gx0, gy0, q, b);
        tma::load_3d(sm.c[sl], &MP.ch, &sm.bar[sl], gx0, gy0, q);
        if (cen) tma::load_4d(sm.lp[sl], &MP.lc[lprev], &sm.bar[sl], gx0 + M, gy0 + M, z, b);
    };
    if (tid == 0) {
        for (int i = 0; i < NA3; ++i) tma::mbar_init(&sm.bar[i], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    int next = q0;
    if (tid == 0)
        for (; next < min(q1, q0 + NA3); ++next) issue(next);
    auto fail = [&](int q) {
        if (tid == 0)
            for (int r = q; r < next; ++r) tma::mbar_wait(&sm.bar[slot(r)], parity(r), err, ERR_WAIT_F3);
    };
    // Each thread waits for the stages it reads itself; a failed wait is
    // noted and the CTA leaves together at the next block barrier, thread 0
    // draining the loads in flight (from q0 before the first plane's barrier,
    // else from z + M).
    bool bad = false;
    auto await = [&](int q) {
        if (!tma::mbar_wait(&sm.bar[slot(q)], parity(q), err, ERR_WAIT_F3)) bad = true;
    };
    // the gw plane of plane q into gw buffer q & 1 (stage q has landed)
    auto convert = [&](int q) {
        float* g = sm.gw[q & 1];
        const float* c = sm.c[slot(q)];
        const float* l = sm.l[slot(q)];
        for (int e = tid; e < PN; e += NTH) g[e] = c[e] * l[e];
    };
    const int cidx = (ty + M) * PW + (tx + M), cc = ty * BXC + tx;
    float qg[2 * M + 1];                                // gw of planes z - M .. z + M at this column
#pragma unroll
    for (int k = 0; k < 2 * M; ++k) {
        await(q0 + k);
        qg[k] = sm.c[slot(q0 + k)][cidx] * sm.l[slot(q0 + k)][cidx];
    }
    convert(zb);
    if (__syncthreads_or(bad)) { fail(q0); return; }
    // the stages before zb fed only the queue: their slots are free now, and
    // refilling them brings stage zb + M (NA3 < 2M + 1 holds it back so far)
    if (tid == 0)
        for (; next < q1 && next < zb + NA3; ++next) issue(next);
    // rolling slots of stages z and z + M and the phase of z + M
    int sz = M % NA3, sq = (2 * M) % NA3;
    uint32_t ph = (uint32_t)(((2 * M) / NA3) & 1);
    long long ic = (long long)zb * P.SP + colo;
    for (int z = zb; z < ze; ++z, ic += P.SP) {
        if (!tma::mbar_wait(&sm.bar[sq], ph, err, ERR_WAIT_F3)) bad = true;
        qg[2 * M] = sm.c[sq][cidx] * sm.l[sq][cidx];
        if (col) {
            const float* g = sm.gw[z & 1] + cidx;
            const long long i = bo + ic;
            const float gun = sm.l[sz][cidx];
            const float gw = qg[M];
            const bool inz = z < P.qz0 || z >= P.qz1;
            const float lprevv = sm.lp[sq][cc];
            if (!inx && !iny && !inz) {
                float lapx = 0.0f, lapy = 0.0f, lapz = 0.0f;
#pragma unroll
                for (int k = 1; k <= M; ++k) {
                    lapx += P.lc[k] * (tap(g[k], gw) + tap(g[-k], gw));
                    lapy += P.lc[k] * (tap(g[k * PW], gw) + tap(g[-k * PW], gw));
                    lapz += P.lc[k] * (tap(qg[M + k], gw) + tap(qg[M - k], gw));
                }
                A.l_next[i] = 2.0f * gun - lprevv + lapx * P.ih2x + lapy * P.ih2y + lapz * P.ih2z;
            } else {
                float Lx, Ly, Lz, Dgx = 0.f, Dgy = 0.f, Dgz = 0.f;
                float ga[2 * M + 1];
                if (inx) {
#pragma unroll
                    for (int k = -M; k <= M; ++k) ga[M + k] = g[k];
                    adj_axis(P, P.px, ga, A.px + bo, A.zx + bo, ic, 1, ix, P.ih2x, P.ihx, Lx, Dgx, A.pxo + bo,
                             A.zxo + bo);
                } else {
                    Lx = 0.0f;
#pragma unroll
                    for (int k = 1; k <= M; ++k) Lx += P.lc[k] * (tap(g[k], gw) + tap(g[-k], gw));
                    Lx *= P.ih2x;
                }
                if (iny) {
#pragma unroll
                    for (int k = -M; k <= M; ++k) ga[M + k] = g[k * PW];
                    adj_axis(P, P.py, ga, A.py + bo, A.zy + bo, ic, P.P, iy, P.ih2y, P.ihy, Ly, Dgy, A.pyo + bo,
                             A.zyo + bo);
                } else {
                    Ly = 0.0f;
#pragma unroll
                    for (int k = 1; k <= M; ++k) Ly += P.lc[k] * (tap(g[k * PW], gw) + tap(g[-k * PW], gw));
                    Ly *= P.ih2y;
                }
                if (inz) {
                    adj_axis(P, P.pz, qg, A.pz + bo, A.zz + bo, ic, P.SP, z, P.ih2z, P.ihz, Lz, Dgz, A.pzo + bo,
                             A.zzo + bo);
                } else {
                    Lz = 0.0f;
#pragma unroll
                    for (int k = 1; k <= M; ++k) Lz += P.lc[k] * (tap(qg[M + k], gw) + tap(qg[M - k], gw));
                    Lz *= P.ih2z;
                }
                A.l_next[i] = 2.0f * gun - lprevv + (Lx + Ly + Lz - Dgx - Dgy - Dgz);
            }
        }
#pragma unroll
        for (int k = 0; k < 2 * M; ++k) qg[k] = qg[k + 1];
        sz = sz + 1 == NA3 ? 0 : sz + 1;
        // the next plane's gw (stage z + 1, now in slot sz, has landed:
        // z + 1 <= z + M); the buffer it overwrites was last read in plane z - 1
        if (z + 1 < ze) {
            float* gb = sm.gw[(z + 1) & 1];
            const float* c = sm.c[sz];
            const float* l = sm.l[sz];
            for (int e = tid; e < PN; e += NTH) gb[e] = c[e] * l[e];
        }
        if (++sq == NA3) { sq = 0; ph ^= 1u; }
        if (__syncthreads_or(bad)) { fail(z + M); return; }
        if (tid == 0)
            for (; next < q1 && next <= z + NA3; ++next) issue(next);    // slots of stages <= z are free
    }
}

// ---------------------------------------------- reconstruction and imaging
struct R3 {
    const float* r_now; const float* r_prev; float* r_next;  // u(it), u(it+1), u(it-1) - s(it)
    const float* lam;                                       // lambda(it)
    float *gacc, *gcomp, *is, *ir;                          // per-shot slots (B, S)
};

// Reconstruction plane ring: stage q holds the halo plane u(it)(q); the
// per-plane centre tiles of plane q - M -- u(it+1), lambda(it), the two model
// fields and the two Kahan slots -- sit in a ring of NRC3 stages indexed by
// plane, filled with stage q and counted on its barrier.  Each thread keeps
// the nine z-taps of its column in a register queue (plane z pushes the
// centre of stage z + M), so stages z .. z + M must have landed at plane z:
// the halo loads run NR3 - M - 1 planes ahead, the centre tiles NRC3 - 1.
constexpr int NR3 = SWEEP_A3D_REC_STAGES;
static_assert(NR3 >= 2 * M + 1, "the reconstruction ring must hold the first plane's z-taps and one more stage");
constexpr int NRC3 = NR3 - M;
template <int BY>
struct R3Smem {
    float u[NR3][TileY<BY>::PN];
    float c[NRC3][6][TileY<BY>::CN];
    uint64_t bar[NR3];
};

struct R3Maps {
    CUtensorMap uh[3];              // reconstruction buffers, (PW x PH) boxes
    CUtensorMap uc[3];              // the same, centre boxes
    CUtensorMap lc[3];              // lambda buffers, centre boxes
    CUtensorMap cf, vv;             // model fields, centre boxes
    CUtensorMap ga, gc;             // Kahan accumulator and compensation slots, centre boxes
};

// u(it-1) = 2 u(it) - u(it+1) + vp^2 dt^2 Lap u(it) on the reconstruction box
// (the physical box minus the restored strips) with the fused vp image
// 2 dt^2 u_tt lambda(it) / vp (reference forward_split.cu:292-372).
template <int BY>
__global__ void __launch_bounds__(TileY<BY>::NT, TileY<BY>::CTAS)
    r3_recon(const __grid_constant__ R3Maps MP, const Params P, const R3 R, const int rnow, const int rprev,
             const int lnow, int* err)
{
    constexpr int PN = TileY<BY>::PN, CN3 = TileY<BY>::CN;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R3Smem<BY>& sm = *reinterpret_cast<R3Smem<BY>*>(smem_raw);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BXC + tx;
    const int gx0 = blockIdx.x * BXC - M, gy0 = blockIdx.y * BY - M;
    const int ix = blockIdx.x * BXC + tx, iy = blockIdx.y * BY + ty;
    const int b = blockIdx.z / P.nzc, zci = blockIdx.z - b * P.nzc;
    const int zb = max(P.qz0, zci * P.zc), ze = min(P.qz1, (zci + 1) * P.zc);
    if (zb >= ze) return;
    const bool col = ix >= P.qx0 && ix < P.qx1 && iy >= P.qy0 && iy < P.qy1;
    const long long bo = (long long)b * P.S;
    const long long colo = (long long)iy * P.P + ix;
    const float dt2 = P.dt * P.dt;
    const int q0 = zb - M, q1 = ze + M;
    auto slot = [&](int q) { return (q - q0) % NR3; };
    auto cslot = [&](int z) { return (z - zb) % NRC3; };
    auto parity = [&](int q) { return (uint32_t)(((q - q0) / NR3) & 1); };
    auto issue = [&](int q) {
        const int sl = slot(q), z = q - M;
        const bool cen = z >= zb && z < ze;
        tma::mbar_expect_tx(&sm.bar[sl], (uint32_t)(PN + (cen ? 6 * CN3 : 0)) * 4u);
        tma::load_4d(sm.u[sl], &MP.uh[rnow], &sm.bar[sl], gx0, gy0, q, b);
        if (cen) {
            float(*c)[CN3] = sm.c[cslot(z)];
            const int x = gx0 + M, y = gy0 + M;
            tma::load_4d(c[0], &MP.uc[rprev], &sm.bar[sl], x, y, z, b);
            tma::load_4d(c[1], &MP.lc[lnow], &sm.bar[sl], x, y, z, b);
            tma::load_3d(c[2], &MP.cf, &sm.bar[sl], x, y, z);
            tma::load_3d(c[3], &MP.vv, &sm.bar[sl], x, y, z);
            tma::load_4d(c[4], &MP.ga, &sm.bar[sl], x, y, z, b);
            tma::load_4d(c[5], &MP.gc, &sm.bar[sl], x, y, z, b);
        }
    };
    if (tid == 0) {
        for (int i = 0; i < NR3; ++i) tma::mbar_init(&sm.bar[i], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    // The first issue fills the halo ring; a centre slot is refilled with a
    // halo stage, so the halo stages issued up front are capped at M + NRC3
    // (their centre tiles cover planes zb .. zb + NRC3 - 1).
    int next = q0;
    if (tid == 0)
        for (; next < min(q1, q0 + M + NRC3); ++next) issue(next);
    auto fail = [&](int q) {
        if (tid == 0)
            for (int r = q; r < next; ++r) tma::mbar_wait(&sm.bar[slot(r)], parity(r), err, ERR_WAIT_F3);
    };
    // one block barrier per plane; a failed wait leaves at it (as f3_step)
    bool bad = false;
    auto await = [&](int q) {
        if (!tma::mbar_wait(&sm.bar[slot(q)], parity(q), err, ERR_WAIT_F3)) bad = true;
    };
    const int cidx = (ty + M) * PW + (tx + M), cc = ty * BXC + tx;
    float q[2 * M + 1];
#pragma unroll
    for (int k = 0; k < 2 * M; ++k) {
        await(q0 + k);
        q[k] = sm.u[slot(q0 + k)][cidx];
    }
    // rolling slots: halo stages z and z + M, the phase of z + M, centre plane z
    int sz = M % NR3, sq = (2 * M) % NR3, sc = 0;
    uint32_t ph = (uint32_t)(((2 * M) / NR3) & 1);
    long long i = bo + (long long)zb * P.SP + colo;
    for (int z = zb; z < ze; ++z, i += P.SP) {
        if (!tma::mbar_wait(&sm.bar[sq], ph, err, ERR_WAIT_F3)) bad = true;
        q[2 * M] = sm.u[sq][cidx];
        if (col) {
            const float* p = sm.u[sz] + cidx;
            const float w = (lap_p(p, 1, P, P.ih2x) + lap_p(p, PW, P, P.ih2y)) + lap_q(q, P, P.ih2z);
            const float(*c)[CN3] = sm.c[sc];
            const float u0 = q[M], up = c[0][cc];
            const float un = 2.0f * u0 - up + c[2][cc] * w;
            R.r_next[i] = un;
            const float utt = (un - 2 * u0 + up) / dt2;
            const float lam = c[1][cc];
            const float g = 2.f * P.dt * P.dt * utt * lam / c[3][cc];
            const float y = g - c[5][cc];
            const float t = c[4][cc] + y;
            R.gcomp[i] = (t - c[4][cc]) - y;
            R.gacc[i] = t;
            if (R.is) { R.is[i] += utt * utt; R.ir[i] += lam * lam; }
        }
#pragma unroll
        for (int k = 0; k < 2 * M; ++k) q[k] = q[k + 1];
        sz = sz + 1 == NR3 ? 0 : sz + 1;
        sc = sc + 1 == NRC3 ? 0 : sc + 1;
        if (++sq == NR3) { sq = 0; ph ^= 1u; }
        if (__syncthreads_or(bad)) { fail(z == zb ? q0 : z + M); return; }
        // after plane z the halo slots of stages <= z and the centre slot of
        // plane z are free: stage s refills centre slot s - M, so s <= z + NRC3
        if (tid == 0)
            for (; next < q1 && next <= min(z + NR3, z + M + NRC3); ++next) issue(next);
    }
}

// receiver illumination of the last adjoint step (it == 0), physical box
__global__ void illum_tail3(const Params P, const float* __restrict__ lam, float* __restrict__ ir)
{
    const long long bx = P.x1 - P.x0, by = P.y1 - P.y0, bz = P.z1 - P.z0;
    const long long n = (long long)P.B * bz * by * bx;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        long long r = e;
        const int ix = P.x0 + (int)(r % bx); r /= bx;
        const int iy = P.y0 + (int)(r % by); r /= by;
        const int iz = P.z0 + (int)(r % bz); const int b = (int)(r / bz);
        const long long o = (long long)b * P.S + (long long)iz * P.SP + (long long)iy * P.P + ix;
        ir[o] += lam[o] * lam[o];
    }
}

// strip cell s -> offset of (iz, iy, ix) in a shot's pitched field, once per
// call: the strip kernels of every step read it instead of decoding strip_coord
__global__ void strip_table3(const Params P, int* __restrict__ soff)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < P.nstrip;
         s += (long long)gridDim.x * blockDim.x) {
        int iz, iy, ix;
        strip_coord(P, s, iz, iy, ix);
        soff[s] = (int)((long long)iz * P.SP + (long long)iy * P.P + ix);
    }
}

// model fields, pitched: cf = ((v*v)*dt)*dt, ca = (v*v)*(dt*dt), vv = v
// {a, b, d b, d a} per index of one axis (d a: grad_p of the a profile on
// [M, n - M), as the stencil kernels computed it in place before).
__global__ void pack_prof3(const float* __restrict__ a, const float* __restrict__ b, const float* __restrict__ db,
                           int n, float h, const Params P, float4* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float da = (i >= M && i < n - M) ? grad_p(a + i, 1, P, 1.0f / h) : 0.f;
        out[i] = make_float4(a[i], b[i], db[i], da);
    }
}

__global__ void prep3(const float* __restrict__ vp, int rows, int nx, int P, float dt,
                      float* __restrict__ cf, float* __restrict__ ca, float* __restrict__ vv)
{
    const long long n = (long long)rows * P;
    const float dt2 = dt * dt;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / P;
        const int ix = (int)(i - row * P);
        if (ix < nx) {
            const float v = vp[row * nx + ix];
            cf[i] = ((v * v) * dt) * dt; ca[i] = (v * v) * dt2; vv[i] = v;
        } else {
            cf[i] = 0.f; ca[i] = 0.f; vv[i] = 1.f;
        }
    }
}

// sum of the per-shot Kahan slots into the caller's unpitched (1, nz, ny, nx) gradient
__global__ void finalize3(const float* __restrict__ acc, const float* __restrict__ comp,
                          const float* __restrict__ is, const float* __restrict__ ir, int B, int rows, int nx,
                          int P, long long S, float* __restrict__ g, float* __restrict__ ois, float* __restrict__ oir)
{
    const long long n = (long long)rows * nx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / nx, ix = i - row * nx;
        const long long c = row * P + ix;
        float s = 0.f, a = 0.f, r = 0.f;
        for (int b = 0; b < B; ++b) {
            s += acc[b * S + c] - comp[b * S + c];
            if (is) { a += is[b * S + c]; r += ir[b * S + c]; }
        }
        g[i] = s;
        if (ois) { ois[i] = a; oir[i] = r; }
    }
}

// ------------------------------------------------------------------- host
static Params make_params(const sweep_acoustic_desc* d)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->ndim == 3, "acoustic3d: ndim must be 3 (got %d)", d->ndim);
    SWEEP_REQUIRE(d->M == M, "acoustic3d: only spatial order 8 (M = 4) is built (got M = %d)", d->M);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1, "acoustic3d: B and nt must be >= 1");
    SWEEP_REQUIRE(d->vp_stride == 0, "acoustic3d takes one model shared by every shot");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "acoustic3d: negative source/receiver count");
    // a free surface is the top face without PML cells (pad 0): its M halo
    // planes above the surface are never updated and stay zero
    for (int f = 0; f < 6; ++f)
        SWEEP_REQUIRE(d->pad[f] >= (f == 0 ? 0 : 1),
                      "acoustic3d: every face but the top (free surface) needs a PML pad >= 1 (face %d has %d)", f,
                      d->pad[f]);
    Params P{};
    P.B = d->B; P.nz = d->nz; P.ny = d->ny; P.nx = d->nx; P.nt = d->nt;
    P.nsrc = d->nsrc; P.nrec = d->nrec;
    P.P = (d->nx + 31) / 32 * 32;
    P.SP = (long long)d->ny * P.P;
    P.S = (long long)d->nz * P.SP;
    SWEEP_REQUIRE(P.S < (1LL << 31), "acoustic3d: a shot's field of %lld cells exceeds the 2^31 offsets of the strip "
                  "table", P.S);
    P.dt = d->dt; P.dz = d->dz; P.dy = d->dy; P.dx = d->dx;
    P.ih2z = 1.0f / (d->dz * d->dz); P.ih2y = 1.0f / (d->dy * d->dy); P.ih2x = 1.0f / (d->dx * d->dx);
    P.ihz = 1.0f / d->dz; P.ihy = 1.0f / d->dy; P.ihx = 1.0f / d->dx;
    for (int k = 0; k <= M; ++k) { P.lc[k] = d->lap[k]; P.gc[k] = d->grad[k]; }
    P.z0 = d->pad[0] + M; P.z1 = d->nz - d->pad[1] - M;
    P.y0 = d->pad[2] + M; P.y1 = d->ny - d->pad[3] - M;
    P.x0 = d->pad[4] + M; P.x1 = d->nx - d->pad[5] - M;
    SWEEP_REQUIRE(P.z1 > P.z0 && P.y1 > P.y0 && P.x1 > P.x0, "acoustic3d: empty physical box");
    P.ex0 = P.x0 + 1; P.ex1 = P.x1 - 1; P.ey0 = P.y0 + 1; P.ey1 = P.y1 - 1; P.ez0 = P.z0 + 1; P.ez1 = P.z1 - 1;
    P.qz0 = d->pad[0] + 2 * M + 1; P.qz1 = d->nz - (d->pad[1] + 2 * M + 1);
    P.qy0 = d->pad[2] + 2 * M + 1; P.qy1 = d->ny - (d->pad[3] + 2 * M + 1);
    P.qx0 = d->pad[4] + 2 * M + 1; P.qx1 = d->nx - (d->pad[5] + 2 * M + 1);
    auto widths = [](int extent, int w, int& lo, int& hi) {
        lo = std::min(w, std::max(extent, 0));
        hi = std::min(w, std::max(extent - lo, 0));
    };
    const int w = M + 1;
    widths(P.z1 - P.z0, w, P.wzl, P.wzh);
    widths(P.y1 - P.y0, w, P.wyl, P.wyh);
    widths(P.x1 - P.x0, w, P.wxl, P.wxh);
    const long long bx = P.x1 - P.x0, by = P.y1 - P.y0;
    const long long bzi = std::max(0, (P.z1 - P.wzh) - (P.z0 + P.wzl));
    const long long byi = std::max(0LL, by - P.wyl - P.wyh);
    P.n_top = P.wzl * bx * by; P.n_bot = P.wzh * bx * by;
    P.nring = (P.wyl + P.wyh) * bx + byi * (P.wxl + P.wxh);
    P.nstrip = P.n_top + P.n_bot + bzi * P.nring;
    P.az = d->az; P.bz = d->bz; P.dbz = d->dbz; P.ay = d->ay; P.by = d->by; P.dby = d->dby;
    P.ax = d->ax; P.bx = d->bx; P.dbx = d->dbx;
    // z chunks: enough CTAs for eight waves at 4 CTAs per SM (the stencil
    // kernels are capped at 64 registers for that occupancy; CTAs in the CPML
    // shell take ~3x an interior CTA's time, and many short CTAs balance them
    // across the SMs: measured on the 256^3 survey, 4-shot calls, 1 / 2 / 4
    // chunks per column took 96.7 / 86.7 / 83.2 ms for 16 steps), chunks of
    // at least 16 planes -- or the shape's recorded schedule value
    const sweep_b200_schedule sc = recorded_schedule(d);
    P.rows = sc.tile_y == 16 ? 16 : 8;
    const long long cols = (long long)((d->nx + BXC - 1) / BXC) * ((d->ny + P.rows - 1) / P.rows) * d->B;
    int nzc = sc.z_chunks >= 1 ? sc.z_chunks : (int)std::max(1LL, (8LL * 4 * 148 + cols - 1) / cols);
    nzc = std::max(1, std::min(nzc, d->nz / 16));
    P.graph_steps = resolve_graph_steps(sc.graph_steps);
    P.zc = (d->nz + nzc - 1) / nzc;
    P.nzc = (d->nz + P.zc - 1) / P.zc;
    // x / y tiling: [M, n - M) cut at the CPML band edges (forward: the
    // product-rule band ex / ey; adjoint: the clear box q), each piece tiled
    // by blocks of `w` from an origin rounded down to `align`
    auto tile = [&](int n_axis, int b0, int b1, int w, int align, int cap, int& nb, short* o_, short* l_, short* h_) {
        const int lo = M, hi = n_axis - M;
        b0 = std::min(std::max(b0, lo), hi);
        b1 = std::min(std::max(b1, b0), hi);
        const int cut[4] = {lo, b0, b1, hi};
        int n = 0;
        for (int sgm = 0; sgm < 3; ++sgm) {
            const int a = cut[sgm], e = cut[sgm + 1];
            for (int o = a / align * align; o < e; o += w) {
                SWEEP_REQUIRE(n < cap, "acoustic3d: an axis of %d cells needs more than %d blocks", n_axis, cap);
                o_[n] = (short)o;
                l_[n] = (short)std::max(o, a);
                h_[n] = (short)std::min(o + w, e);
                ++n;
            }
        }
        nb = n;
    };
    tile(d->nx, P.ex0, P.ex1, BXC, 4, kMaxXBlocks, P.nbx[0], P.xo[0], P.xl[0], P.xh[0]);
    tile(d->nx, P.qx0, P.qx1, BXC, 4, kMaxXBlocks, P.nbx[1], P.xo[1], P.xl[1], P.xh[1]);
    tile(d->ny, P.ey0, P.ey1, P.rows, 1, kMaxYBlocks, P.nby[0], P.yo[0], P.yl[0], P.yh[0]);
    tile(d->ny, P.qy0, P.qy1, P.rows, 1, kMaxYBlocks, P.nby[1], P.yo[1], P.yl[1], P.yh[1]);
    return P;
}

// kind: 0 the forward step, 1 the adjoint step (their band-aligned x
// tilings), 2 the reconstruction (plain 32-column blocks)
static dim3 stencil_grid(const Params& P, int kind = 2)
{
    if (kind < 2) return dim3((unsigned)P.nbx[kind], (unsigned)P.nby[kind], P.B * P.nzc);
    return dim3((P.nx + BXC - 1) / BXC, (P.ny + P.rows - 1) / P.rows, P.B * P.nzc);
}

struct Work {
    float *cf, *ca, *vv;
    float* f[34];                    // forward: u x3, psi x6, zeta x3; reverse: see backward()
    int* err;                        // bounded-wait failure flag
    float* scratch;                  // one step's fp32 strips ahead of their quantisation (scaled formats)
    char* ring;                      // host tape: HostRing::R device strip slots
    float4 *pz, *py, *px;            // packed CPML profiles per axis
    int* soff;                       // strip cell offsets (strip_table3)
};

static Work carve(Carve& c, const Params& P, int nfields)
{
    Work w{};
    w.cf = c.take<float>(P.S); w.ca = c.take<float>(P.S); w.vv = c.take<float>(P.S);
    w.pz = c.take<float4>(P.nz); w.py = c.take<float4>(P.ny); w.px = c.take<float4>(P.nx);
    for (int i = 0; i < nfields; ++i) w.f[i] = c.take<float>((long long)P.B * P.S);
    w.err = c.take<int>(1);
    w.soff = c.take<int>(std::max(P.nstrip, 1LL));
    if (P.st.fmt == SF_F16 || P.st.fmt == SF_I8) w.scratch = c.take<float>((long long)P.B * P.nstrip);
    if (P.st.host) w.ring = c.take<char>((long long)HostRing::R * P.st.step);
    return w;
}

// Model fields and packed profiles of a call (shared by both passes).
static void prep_call(const sweep_acoustic_desc* d, Params& P, const Work& w, cudaStream_t st)
{
    const long long rows = (long long)d->nz * d->ny;
    prep3<<<592, 256, 0, st>>>(d->vp, (int)rows, d->nx, P.P, d->dt, w.cf, w.ca, w.vv);
    SWEEP_LAUNCH_CHECK();
    P.cf = w.cf; P.ca = w.ca; P.vv = w.vv;
    pack_prof3<<<1, 256, 0, st>>>(d->az, d->bz, d->dbz, d->nz, d->dz, P, w.pz);
    pack_prof3<<<1, 256, 0, st>>>(d->ay, d->by, d->dby, d->ny, d->dy, P, w.py);
    pack_prof3<<<1, 256, 0, st>>>(d->ax, d->bx, d->dbx, d->nx, d->dx, P, w.px);
    SWEEP_LAUNCH_CHECK();
    P.pz = w.pz; P.py = w.py; P.px = w.px;
    if (P.nstrip > 0) {
        strip_table3<<<592, 256, 0, st>>>(P, w.soff);
        SWEEP_LAUNCH_CHECK();
    }
    P.soff = w.soff;
}

static void check_err(const Work& w, cudaStream_t st, const char* what)
{
    int h = 0;
    SWEEP_CUDA(cudaMemcpyAsync(&h, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    SWEEP_REQUIRE(h == 0, "acoustic3d %s: a plane load did not complete in time (code %d); results are invalid", what, h);
}

// 4-D (x, y, z, shot) map of a wavefield buffer, or 3-D (x, y, z) of the model.
static CUtensorMap plane_map(const float* base, const Params& P, int nb, bool halo)
{
    const uint32_t bx = halo ? PW : BXC, by = halo ? P.rows + 2 * M : P.rows;
    if (nb == 0) {
        const uint64_t dims[3] = {(uint64_t)P.nx, (uint64_t)P.ny, (uint64_t)P.nz};
        const uint64_t strides[2] = {(uint64_t)P.P, (uint64_t)P.SP};
        const uint32_t box[3] = {bx, by, 1u};
        return tma::make_map(base, 3, dims, strides, box);
    }
    const uint64_t dims[4] = {(uint64_t)P.nx, (uint64_t)P.ny, (uint64_t)P.nz, (uint64_t)nb};
    const uint64_t strides[3] = {(uint64_t)P.P, (uint64_t)P.SP, (uint64_t)P.S};
    const uint32_t box[4] = {bx, by, 1u, 1u};
    return tma::make_map(base, 4, dims, strides, box);
}

// Strip storage of a memory mode: the step-slot layout of the boundary-saving
// tape (the checkpoint mode keeps its chunk strips as fp32).
static void set_store(Params& P, int mem_mode)
{
    StripStore& S = P.st;
    S = StripStore{};
    S.host = (mem_mode & SWEEP_MEM_HOST_TAPE) != 0;
    mem_mode &= ~SWEEP_MEM_HOST_TAPE;
    S.w = M + 1;
    S.fmt = mem_mode == SWEEP_MEM_BOUNDARY_FP16 ? SF_F16
          : mem_mode == SWEEP_MEM_BOUNDARY_BF16 ? SF_BF16
          : mem_mode == SWEEP_MEM_BOUNDARY_INT8 ? SF_I8 : SF_F32;
    auto up = [](long long v, long long a) { return (v + a - 1) / a * a; };
    if (S.fmt == SF_F32 || S.fmt == SF_BF16) {
        S.step = up((long long)P.B * P.nstrip * (S.fmt == SF_F32 ? 4 : 2), 256);
        return;
    }
    const long long bx = P.x1 - P.x0, by = P.y1 - P.y0, bz = P.z1 - P.z0;
    SWEEP_REQUIRE(bx >= 2 * S.w && by >= 2 * S.w && bz >= 2 * S.w,
                  "acoustic3d: fp16 / int8 strip storage needs a physical box of at least %d cells per axis", 2 * S.w);
    const long long cells[6] = {S.w * by * bx, S.w * by * bx, bz * S.w * bx, bz * S.w * bx, bz * by * S.w, bz * by * S.w};
    const int esz = S.fmt == SF_F16 ? 2 : 1;
    long long off = 0;
    for (int f = 0; f < 6; ++f) {
        SWEEP_REQUIRE(cells[f] < (1LL << 31), "acoustic3d: a strip face holds too many cells");
        S.cells[f] = (int)cells[f];
        S.blocks[f] = (int)((cells[f] + kQB - 1) / kQB);
        S.pay[f] = off;
        off = up(off + (long long)P.B * cells[f] * esz, 16);
    }
    for (int f = 0; f < 6; ++f) {
        S.scl[f] = off;
        off = up(off + (long long)P.B * S.blocks[f] * 4, 16);
    }
    S.step = up(off, 256);
}

// tape: one strip slot per step (P.st.step bytes), then (U[nt-1], U[nt]) pitched
static int64_t tape_bytes(const Params& P)
{
    return (int64_t)P.nt * P.st.step + 2LL * P.B * P.S * 4;
}

static void* tape_slot(const void* tape, const Params& P, int it)
{
    return const_cast<char*>(static_cast<const char*>(tape)) + (long long)it * P.st.step;
}

static float* tape_last(void* tape, const Params& P)
{
    return static_cast<float*>(tape_slot(tape, P, P.nt));
}

static constexpr int kFwdFields = 12, kRevFields = 22;

// Checkpointed boundary saving (SWEEP_MEM_CHECKPOINT, chunk length k): for
// every chunk c >= 1 the tape holds the forward state before step c k -- the
// wavefield pair (U[ck-1], U[ck]), CPML psi (x, y, z) and zeta (x, y, z) --
// and the strips of U[ck-1]; the backward replays each chunk from its
// checkpoint into the strips of that chunk and runs the boundary-saving
// reverse steps over it (reference checkpoint_runtime.cuh:15-362,
// eq_driver.cuh:928-1135: chunked replay).
static constexpr int kStateFields = 8;

static int nchunks(const Params& P, int k)
{
    SWEEP_REQUIRE(k >= 1, "acoustic3d: checkpoint interval must be >= 1 (got %d)", k);
    return (P.nt + k - 1) / k;
}

static long long ckpt_stride(const Params& P)
{
    Carve c(nullptr);
    c.take<float>(kStateFields * (long long)P.B * P.S);
    c.take<float>((long long)P.B * std::max(P.nstrip, 1LL));
    return (c.off + 255) & ~255LL;
}

static float* ckpt_field(void* tape, const Params& P, int c, int f)
{
    char* base = static_cast<char*>(tape) + (long long)(c - 1) * ckpt_stride(P);
    return reinterpret_cast<float*>(base) + (long long)f * P.B * P.S;
}

static float* ckpt_strips(void* tape, const Params& P, int c) { return ckpt_field(tape, P, c, kStateFields); }

void schedule_of(const sweep_acoustic_desc* d, sweep_b200_schedule* out)
{
    const Params P = make_params(d);
    out->shots_fwd = 0;
    out->shots_rev = 0;
    out->z_chunks = P.nzc;
    out->graph_steps = P.graph_steps;
    out->tile_y = P.rows;
}

void sizes(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, int64_t* ws, int64_t* tape)
{
    const int base_mode = mem_mode & ~SWEEP_MEM_HOST_TAPE;
    SWEEP_REQUIRE(base_mode == SWEEP_MEM_BOUNDARY || base_mode == SWEEP_MEM_CHECKPOINT ||
                      base_mode == SWEEP_MEM_BOUNDARY_FP16 || base_mode == SWEEP_MEM_BOUNDARY_BF16 ||
                      base_mode == SWEEP_MEM_BOUNDARY_INT8 || base_mode == SWEEP_MEM_RECURSIVE,
                  "acoustic3d: unknown memory mode %d", mem_mode);
    SWEEP_REQUIRE(!(mem_mode & SWEEP_MEM_HOST_TAPE) ||
                      (base_mode != SWEEP_MEM_CHECKPOINT && base_mode != SWEEP_MEM_RECURSIVE),
                  "acoustic3d: a host tape goes with boundary saving only");
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT || ckpt_every >= 1,
                  "acoustic3d: checkpoint interval must be >= 1 (got %d)", ckpt_every);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_RECURSIVE || ckpt_every >= 1,
                  "acoustic3d: the recursive checkpoint budget must be >= 1 (got %d)", ckpt_every);
    Params P = make_params(d);
    set_store(P, mem_mode);
    Carve c(nullptr);
    if (mem_mode == SWEEP_MEM_CHECKPOINT) {
        carve(c, P, kRevFields + kFwdFields);
        c.take<float>((long long)(ckpt_every + 1) * P.B * P.nstrip);
        *tape = (int64_t)std::max(nchunks(P, ckpt_every) - 1, 1) * ckpt_stride(P);
    } else if (mem_mode == SWEEP_MEM_RECURSIVE) {
        carve(c, P, kRevFields + kFwdFields);
        c.take<float>((long long)(SWEEP_RECURSIVE_LEAF + 1) * P.B * P.nstrip);
        c.take<char>((long long)ckpt_every * ckpt_stride(P));           // the snapshot slots
        *tape = 256;                                                     // nothing is kept
    } else {
        carve(c, P, std::max(kFwdFields, kRevFields));
        *tape = tape_bytes(P);
    }
    *ws = c.off;
}

static inline unsigned blocks_for(long long n, int threads) { return (unsigned)std::max(1LL, (n + threads - 1) / threads); }

static void copy_dd(float* dst, const float* src, long long n, cudaStream_t st)
{
    SWEEP_CUDA(cudaMemcpyAsync(dst, src, n * 4, cudaMemcpyDeviceToDevice, st));
}

// Rotating forward state over the 12 forward fields f[0..11] of a set:
// wavefield buffer indices and the current / next CPML psi triples.
struct FwdState {
    float* const* f;
    int ip = 0, in = 1, ix = 2;
    float* ps[3];
    float* psn[3];
    explicit FwdState(float* const* fields) : f(fields)
    {
        for (int a = 0; a < 3; ++a) { ps[a] = f[3 + a]; psn[a] = f[6 + a]; }
    }
    float* zeta(int a) const { return f[9 + a]; }
};

// The three stencil kernels at the plan's tile height, their shared memory
// opted in once per instantiation.
template <int BY>
static void set_stencil_attrs()
{
    static bool done = false;
    if (done) return;
    SWEEP_CUDA(cudaFuncSetAttribute(f3_step<BY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(F3Smem<BY>)));
    SWEEP_CUDA(cudaFuncSetAttribute(a3_step<BY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(A3Smem<BY>)));
    SWEEP_CUDA(cudaFuncSetAttribute(r3_recon<BY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(R3Smem<BY>)));
    done = true;
}

static void launch_f3(const Params& P, const F3Maps& maps, const F3& F, int uin, int uprev, int* err, cudaStream_t st)
{
    const dim3 grid = stencil_grid(P, 0), block(BXC, P.rows);
    if (P.rows == 16) {
        set_stencil_attrs<16>();
        f3_step<16><<<grid, block, sizeof(F3Smem<16>), st>>>(maps, P, F, uin, uprev, err);
    } else {
        set_stencil_attrs<8>();
        f3_step<8><<<grid, block, sizeof(F3Smem<8>), st>>>(maps, P, F, uin, uprev, err);
    }
}

static void launch_a3(const Params& P, const A3Maps& maps, const A3& A, int lnow, int lprev, int* err,
                      cudaStream_t st)
{
    const dim3 grid = stencil_grid(P, 1), block(BXC, P.rows);
    if (P.rows == 16) {
        set_stencil_attrs<16>();
        a3_step<16><<<grid, block, sizeof(A3Smem<16>), st>>>(maps, P, A, lnow, lprev, err);
    } else {
        set_stencil_attrs<8>();
        a3_step<8><<<grid, block, sizeof(A3Smem<8>), st>>>(maps, P, A, lnow, lprev, err);
    }
}

static void launch_r3(const Params& P, const R3Maps& maps, const R3& R, int rnow, int rprev, int lnow, int* err,
                      cudaStream_t st)
{
    const dim3 grid = stencil_grid(P, 2), block(BXC, P.rows);
    if (P.rows == 16) {
        set_stencil_attrs<16>();
        r3_recon<16><<<grid, block, sizeof(R3Smem<16>), st>>>(maps, P, R, rnow, rprev, lnow, err);
    } else {
        set_stencil_attrs<8>();
        r3_recon<8><<<grid, block, sizeof(R3Smem<8>), st>>>(maps, P, R, rnow, rprev, lnow, err);
    }
}

// Forward steps [it0, it1): stencil, strips of U[it] (strips_of(it), null:
// none), source injection, receiver gather (record may be null).
template <class StripsOf>
static void forward_steps(const sweep_acoustic_desc* d, const Params& P, FwdState& S, float* record, int it0,
                          int it1, StripsOf strips_of, int* err, float* scratch, cudaStream_t st,
                          HostRing* hr = nullptr)
{
    const bool scaled = P.st.fmt == SF_F16 || P.st.fmt == SF_I8;
    int qper = 0;
    for (int f = 0; f < 6; ++f) qper += P.st.blocks[f];
    const unsigned gs = blocks_for((long long)P.B * P.nsrc, 128), gr = blocks_for((long long)P.B * P.nrec, 128);
    const unsigned gst = blocks_for((long long)P.B * P.nstrip, 256);
    F3Maps maps;
    for (int k = 0; k < 3; ++k) {
        maps.uh[k] = plane_map(S.f[k], P, P.B, true);
        maps.uc[k] = plane_map(S.f[k], P, P.B, false);
    }
    maps.cf = plane_map(P.cf, P, 0, false);
    StepGraphs sg(st, hr ? 0 : P.graph_steps);
    for (int it = it0; it < it1; ++it) {
        F3 F{S.f[S.in], S.f[S.ip], S.f[S.ix], S.ps[0], S.ps[1], S.ps[2], S.psn[0], S.psn[1], S.psn[2],
             S.zeta(0), S.zeta(1), S.zeta(2)};
        const cudaStream_t ls = sg.stream();
        launch_f3(P, maps, F, S.in, S.ip, err, ls);
        SWEEP_LAUNCH_CHECK();
        void* slot = strips_of(it);
        if (slot && P.nstrip > 0) {
            if (hr) hr->before_write(it);
            strips3<<<gst, 256, 0, ls>>>(P, S.f[S.in], slot, scratch, 0);
            if (scaled) quantize_strips3<<<(unsigned)(P.B * qper), kQB, 0, ls>>>(P, scratch, slot);
            if (hr) hr->after_write(it);
        }
        if (d->nsrc > 0)
            inject3<<<gs, 128, 0, ls>>>(P, S.f[S.ix], d->wavelet, d->src_loc, d->nsrc, it, 0, 1.f, 0);
        if (d->nrec > 0 && record)
            gather3<<<gr, 128, 0, ls>>>(P, S.f[S.ix], record, d->rec_loc, d->nrec, it, 1);
        SWEEP_LAUNCH_CHECK();
        sg.step_done();
        const int t = S.ip; S.ip = S.in; S.in = S.ix; S.ix = t;
        for (int a = 0; a < 3; ++a) std::swap(S.ps[a], S.psn[a]);
    }
    sg.flush();
}

static void state_fields(const FwdState& S, float* out[kStateFields])
{
    out[0] = S.f[S.ip]; out[1] = S.f[S.in];
    for (int a = 0; a < 3; ++a) { out[2 + a] = S.ps[a]; out[5 + a] = S.zeta(a); }
}

static void forward_with(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape,
                         void* ws, int64_t ws_bytes, cudaStream_t st, StepState* seg, int seg0, int seg1)
{
    // a stepped run covers [seg0, seg1) of the time axis, continuing seg's state
    const bool stepped = seg != nullptr;
    const int a = stepped ? seg0 : 0, b = stepped ? seg1 : d->nt;
    SWEEP_REQUIRE(!stepped || (mem_mode != SWEEP_MEM_CHECKPOINT && mem_mode != SWEEP_MEM_RECURSIVE),
                  "acoustic3d stepped forward: boundary saving only");
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, ckpt_every, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic3d forward: workspace too small (%lld < %lld)",
                  (long long)ws_bytes, (long long)need_ws);
    SWEEP_REQUIRE(record != nullptr || d->nrec == 0, "acoustic3d forward: null record");
    Params P = make_params(d);
    set_store(P, mem_mode);
    Carve c(ws);
    Work w = carve(c, P, kFwdFields);
    prep_call(d, P, w, st);
    const long long n = (long long)P.B * P.S;
    if (a == 0) {
        for (int i = 0; i < kFwdFields; ++i) SWEEP_CUDA(cudaMemsetAsync(w.f[i], 0, n * 4, st));
        if (d->nrec > 0) SWEEP_CUDA(cudaMemsetAsync(record, 0, (size_t)d->B * d->nt * d->nrec * 4, st));
    }
    SWEEP_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    FwdState S(w.f);
    if (stepped && a > 0) {
        S.ip = seg->idx[0]; S.in = seg->idx[1]; S.ix = seg->idx[2];
        for (int k = 0; k < 3; ++k) {
            S.ps[k] = static_cast<float*>(seg->ptr[k]);
            S.psn[k] = static_cast<float*>(seg->ptr[3 + k]);
        }
    }
    auto keep = [&] {
        if (!stepped) return;
        seg->idx[0] = S.ip; seg->idx[1] = S.in; seg->idx[2] = S.ix;
        for (int k = 0; k < 3; ++k) { seg->ptr[k] = S.ps[k]; seg->ptr[3 + k] = S.psn[k]; }
    };
    if (mem_mode == SWEEP_MEM_RECURSIVE) {
        // recursive checkpointing keeps nothing: the backward replays from the initial state
        forward_steps(d, P, S, record, 0, d->nt, [&](int) { return (void*)nullptr; }, w.err, w.scratch, st);
        check_err(w, st, "forward");
        return;
    }
    if (mem_mode != SWEEP_MEM_CHECKPOINT && tape && P.st.host) {
        HostRing hr;
        hr.open(w.ring, tape, P.st.step, st);
        forward_steps(d, P, S, record, a, b, [&](int it) { return hr.slot(it); }, w.err, w.scratch, st, &hr);
        hr.close();
        if (b == d->nt) {
            float* last = tape_last(tape, P);
            SWEEP_CUDA(cudaMemcpyAsync(last, S.f[S.ip], n * 4, cudaMemcpyDefault, st));       // U[nt-1]
            SWEEP_CUDA(cudaMemcpyAsync(last + n, S.f[S.in], n * 4, cudaMemcpyDefault, st));   // U[nt]
        }
        keep();
        check_err(w, st, "forward");
        return;
    } else if (mem_mode != SWEEP_MEM_CHECKPOINT) {
        forward_steps(d, P, S, record, a, b, [&](int it) { return tape ? tape_slot(tape, P, it) : nullptr; },
                      w.err, w.scratch, st);
        if (tape && b == d->nt) {
            float* last = tape_last(tape, P);
            copy_dd(last, S.f[S.ip], n, st);        // U[nt-1]
            copy_dd(last + n, S.f[S.in], n, st);    // U[nt]
        }
        keep();
        check_err(w, st, "forward");
        return;
    }
    const int k = ckpt_every, C = nchunks(P, k);
    for (int ch = 0; ch < C; ++ch) {
        const int it0 = ch * k, it1 = std::min(d->nt, it0 + k);
        if (tape && ch >= 1) {
            float* state[kStateFields];
            state_fields(S, state);
            for (int f = 0; f < kStateFields; ++f) copy_dd(ckpt_field(tape, P, ch, f), state[f], n, st);
        }
        // the last step of a chunk keeps its strips with the next checkpoint
        forward_steps(d, P, S, record, it0, it1,
                      [&](int it) { return (tape && it == it1 - 1 && ch + 1 < C) ? ckpt_strips(tape, P, ch + 1) : nullptr; },
                      w.err, w.scratch, st);
    }
    check_err(w, st, "forward");
}

// Recursive checkpointing (SWEEP_MEM_RECURSIVE): the 2-D driver's bisection
// (acoustic2d.cu backward_recursive) over the 3-D replay set w.f[kRevFields..]:
// at most `count` snapshot slots, each the checkpoint layout (state fields,
// then the strips of the step before); leaves of SWEEP_RECURSIVE_LEAF steps,
// the chunks of SWEEP_MEM_CHECKPOINT with that interval.
template <class Reverse>
static void backward_recursive(const sweep_acoustic_desc* d, const Params& P, Work& w, float* chunk, char* snaps,
                               int count, cudaStream_t st, Reverse& reverse)
{
    const int L = SWEEP_RECURSIVE_LEAF;
    const long long n = (long long)P.B * P.S, cs = (long long)P.B * P.nstrip;
    float* const* fw = w.f + kRevFields;
    // the replay set starts clear (see the checkpoint mode)
    for (int i = 0; i < kFwdFields; ++i) SWEEP_CUDA(cudaMemsetAsync(fw[i], 0, n * 4, st));
    FwdState S(fw);
    auto restore = [&](int k) {
        S = FwdState(fw);
        float* state[kStateFields];
        state_fields(S, state);
        for (int f = 0; f < kStateFields; ++f) {
            if (k < 0) SWEEP_CUDA(cudaMemsetAsync(state[f], 0, n * 4, st));
            else copy_dd(state[f], ckpt_field(snaps, P, k + 1, f), n, st);
        }
    };
    auto save = [&](int k) {
        float* state[kStateFields];
        state_fields(S, state);
        for (int f = 0; f < kStateFields; ++f) copy_dd(ckpt_field(snaps, P, k + 1, f), state[f], n, st);
    };
    auto replay = [&](int a, int e, auto strips_of) {
        forward_steps(d, P, S, nullptr, a, e, strips_of, w.err, w.scratch, st);
    };
    auto leaf = [&](int a, int e) {
        replay(a, e, [&](int it) { return (void*)(chunk + (long long)(it - a + 1) * cs); });
        copy_dd(w.f[15], S.f[S.in], n, st);      // U[e]
        copy_dd(w.f[16], S.f[S.ip], n, st);      // U[e - 1]
        reverse(a, e, [&](int t) { return chunk + (long long)(t - (a - 1)) * cs; });
    };
    std::function<void(int, int, int, int)> process = [&](int a, int b, int ka, int free) {
        const int nleaf = (b - a + L - 1) / L;
        if (nleaf <= 1) {
            restore(ka);
            if (a > 0) copy_dd(chunk, ckpt_strips(snaps, P, ka + 1), cs, st);   // strips of U[a - 1]
            leaf(a, b);
            return;
        }
        if (free > 0) {
            const int k = count - free, m = a + L * ((nleaf + 1) / 2);
            restore(ka);
            replay(a, m, [&](int it) { return (void*)(it == m - 1 ? ckpt_strips(snaps, P, k + 1) : nullptr); });
            save(k);
            process(m, b, k, free - 1);
            process(a, m, ka, free);
            return;
        }
        for (int c0 = a + (nleaf - 1) * L; c0 >= a; c0 -= L) {
            restore(ka);
            if (c0 > a)
                replay(a, c0, [&](int it) { return (void*)(it == c0 - 1 ? chunk : nullptr); });
            else if (a > 0)
                copy_dd(chunk, ckpt_strips(snaps, P, ka + 1), cs, st);
            leaf(c0, std::min(b, c0 + L));
        }
    };
    SWEEP_REQUIRE(count >= 1, "acoustic3d: the recursive checkpoint budget must be >= 1");
    process(0, P.nt, -1, count);
}

static void backward_with(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, const float* adj,
                          const void* tape, float* grad_vp, float* grad_w, float* illum_s, float* illum_r,
                          void* ws, int64_t ws_bytes, cudaStream_t st, StepState* seg, int bw0, int bw1)
{
    // a stepped run reverses [bw1, bw0) top down, continuing seg's state
    const bool stepped = seg != nullptr;
    const int top = stepped ? bw0 : d->nt, bottom = stepped ? bw1 : 0;
    const bool first = top == d->nt;
    int64_t need_ws, need_tape;
    sizes(d, mem_mode, ckpt_every, &need_ws, &need_tape);
    SWEEP_REQUIRE(ws != nullptr && ws_bytes >= need_ws, "acoustic3d backward: workspace too small");
    SWEEP_REQUIRE(tape != nullptr && grad_vp != nullptr, "acoustic3d backward: null tape or gradient");
    SWEEP_REQUIRE(adj != nullptr || d->nrec == 0, "acoustic3d backward: null record cotangent");
    SWEEP_REQUIRE((illum_s == nullptr) == (illum_r == nullptr), "acoustic3d backward: pass both illuminations or neither");
    const bool ckpt = mem_mode == SWEEP_MEM_CHECKPOINT;
    const bool recursive = mem_mode == SWEEP_MEM_RECURSIVE;
    SWEEP_REQUIRE(!stepped || (!ckpt && !recursive), "acoustic3d stepped backward: boundary saving only");
    Params P = make_params(d);
    set_store(P, mem_mode);
    Carve c(ws);
    // fields: 0-2 lambda, 3-14 adjoint CPML (psi x,y,z and zeta x,y,z, two
    // buffers each), 15-17 reconstruction, 18-19 Kahan slots, 20-21
    // illumination; checkpoint mode: 22-33 the forward set of the replay,
    // then the strips of one chunk
    Work w = carve(c, P, (ckpt || recursive) ? kRevFields + kFwdFields : kRevFields);
    float* chunk = ckpt ? c.take<float>((long long)(ckpt_every + 1) * P.B * P.nstrip)
                 : recursive ? c.take<float>((long long)(SWEEP_RECURSIVE_LEAF + 1) * P.B * P.nstrip) : nullptr;
    char* snaps = recursive ? c.take<char>((long long)ckpt_every * ckpt_stride(P)) : nullptr;
    const long long rows = (long long)d->nz * d->ny;
    prep_call(d, P, w, st);
    const long long n = (long long)P.B * P.S;
    const bool illum = illum_s != nullptr;
    if (first) {
        for (int i = 0; i < kRevFields; ++i) SWEEP_CUDA(cudaMemsetAsync(w.f[i], 0, n * 4, st));
        if (grad_w && d->nsrc > 0) SWEEP_CUDA(cudaMemsetAsync(grad_w, 0, (size_t)d->B * d->nsrc * d->nt * 4, st));
    }
    SWEEP_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    const unsigned gs = blocks_for((long long)P.B * P.nsrc, 128), gr = blocks_for((long long)P.B * P.nrec, 128);
    const unsigned gst = blocks_for((long long)P.B * P.nstrip, 256);
    int lp = 0, ln = 1, lx = 2, cur = 0;
    int rp = 15, rn = 16, rx = 17;
    if (stepped && !first) {
        lp = seg->idx[0]; ln = seg->idx[1]; lx = seg->idx[2]; cur = seg->idx[3];
        rp = seg->idx[4]; rn = seg->idx[5]; rx = seg->idx[6];
    }
    float* gacc = w.f[18];
    float* gcomp = w.f[19];
    float* is = illum ? w.f[20] : nullptr;
    float* ir = illum ? w.f[21] : nullptr;
    A3Maps amaps;
    for (int k = 0; k < 3; ++k) {
        amaps.lh[k] = plane_map(w.f[k], P, P.B, true);
        amaps.lc[k] = plane_map(w.f[k], P, P.B, false);
    }
    amaps.ch = plane_map(P.ca, P, 0, true);
    R3Maps rmaps;
    for (int k = 0; k < 3; ++k) {
        rmaps.uh[k] = plane_map(w.f[15 + k], P, P.B, true);
        rmaps.uc[k] = plane_map(w.f[15 + k], P, P.B, false);
        rmaps.lc[k] = plane_map(w.f[k], P, P.B, false);
    }
    rmaps.cf = plane_map(P.cf, P, 0, false);
    rmaps.vv = plane_map(P.vv, P, 0, false);
    rmaps.ga = plane_map(gacc, P, P.B, false);
    rmaps.gc = plane_map(gcomp, P, P.B, false);
    // Reverse steps [it0, it1) top down from prev = U[it1] (f[15]), now =
    // U[it1 - 1] (f[16]); strips_of(t) holds the strips of U[t].
    HostRing hr;
    const bool host = P.st.host && !ckpt && !recursive;
    auto reverse = [&](int it0, int it1, auto strips_of, bool fresh) {
        StepGraphs sg(st, host ? 0 : P.graph_steps);
        if (fresh) { rp = 15; rn = 16; rx = 17; }
        for (int it = it1 - 1; it >= it0; --it) {
            const cudaStream_t ls = sg.stream();
            float* a_in[6];
            float* a_out[6];
            for (int k = 0; k < 6; ++k) { a_in[k] = w.f[3 + 2 * k + cur]; a_out[k] = w.f[3 + 2 * k + 1 - cur]; }
            A3 A{w.f[ln], w.f[lp], w.f[lx], a_in[0], a_in[1], a_in[2], a_in[3], a_in[4], a_in[5],
                 a_out[0], a_out[1], a_out[2], a_out[3], a_out[4], a_out[5]};
            launch_a3(P, amaps, A, ln, lp, w.err, ls);
            SWEEP_LAUNCH_CHECK();
            if (d->nrec > 0)
                inject3<<<gr, 128, 0, ls>>>(P, w.f[lx], adj, d->rec_loc, d->nrec, it, 1, 1.f, 0);
            int t = lp; lp = ln; ln = lx; lx = t;
            cur = 1 - cur;
            if (grad_w && d->nsrc > 0)
                gather3<<<gs, 128, 0, ls>>>(P, w.f[ln], grad_w, d->src_loc, d->nsrc, it, 0);
            if (it > 0) {
                R3 R{w.f[rn], w.f[rp], w.f[rx], w.f[ln], gacc, gcomp, is, ir};
                launch_r3(P, rmaps, R, rn - 15, rp - 15, ln, w.err, ls);
                if (P.nstrip > 0) {
                    if (host) hr.before_read(it - 1);
                    strips3<<<gst, 256, 0, ls>>>(P, w.f[rx], strips_of(it - 1), nullptr, 1);
                    if (host) {
                        hr.after_read(it - 1);
                        if (it - 1 - HostRing::R >= std::max(it0 - 1, 0)) hr.fetch(it - 1 - HostRing::R, true);
                    }
                    if (d->nsrc > 0)
                        inject3<<<gs, 128, 0, ls>>>(P, w.f[rx], d->wavelet, d->src_loc, d->nsrc, it, 0, -1.f, 1);
                    Img I{w.f[rp], w.f[rn], w.f[rx], w.f[ln], gacc, gcomp, is, ir};
                    strip_image3<<<gst, 256, 0, ls>>>(P, I);
                }
                if (d->nsrc > 0)
                    inject3<<<gs, 128, 0, ls>>>(P, w.f[rx], d->wavelet, d->src_loc, d->nsrc, it, 0, 1.f, 0);
                SWEEP_LAUNCH_CHECK();
                t = rp; rp = rn; rn = rx; rx = t;
            } else if (illum) {
                illum_tail3<<<592, 256, 0, ls>>>(P, w.f[ln], ir);
                SWEEP_LAUNCH_CHECK();
            }
            sg.step_done();
        }
        sg.flush();
    };
    if (recursive) {
        auto rev = [&](int it0, int it1, auto strips_of) { reverse(it0, it1, strips_of, true); };
        backward_recursive(d, P, w, chunk, snaps, ckpt_every, st, rev);
    } else if (!ckpt) {
        if (first) {
            const float* last = tape_last(const_cast<void*>(tape), P);
            SWEEP_CUDA(cudaMemcpyAsync(w.f[15], last + n, n * 4, cudaMemcpyDefault, st));   // prev = U[nt]
            SWEEP_CUDA(cudaMemcpyAsync(w.f[16], last, n * 4, cudaMemcpyDefault, st));       // now  = U[nt-1]
        }
        if (host && P.nstrip > 0) {
            hr.open(w.ring, const_cast<void*>(tape), P.st.step, st);
            for (int t = top - 2; t >= std::max(bottom - 1, 0) && t > top - 2 - HostRing::R; --t) hr.fetch(t, false);
            reverse(bottom, top, [&](int t) { return hr.slot(t); }, first);
            hr.close();
        } else {
            reverse(bottom, top, [&](int t) { return tape_slot(tape, P, t); }, first);
        }
    } else {
        const int k = ckpt_every, C = nchunks(P, k);
        void* tp = const_cast<void*>(tape);
        const long long cs = (long long)P.B * P.nstrip;
        float* const* fw = w.f + kRevFields;
        // the replay set starts clear: the fields a checkpoint does not hold
        // (the third wavefield buffer, the next-psi triple) are read in their
        // stencil halo and outside the CPML band, which no step writes
        for (int i = 0; i < kFwdFields; ++i) SWEEP_CUDA(cudaMemsetAsync(fw[i], 0, n * 4, st));
        for (int ch = C - 1; ch >= 0; --ch) {
            const int it0 = ch * k, it1 = std::min(d->nt, it0 + k);
            FwdState S(fw);
            float* state[kStateFields];
            state_fields(S, state);
            if (ch == 0) {
                for (int f = 0; f < kStateFields; ++f) SWEEP_CUDA(cudaMemsetAsync(state[f], 0, n * 4, st));
            } else {
                for (int f = 0; f < kStateFields; ++f) copy_dd(state[f], ckpt_field(tp, P, ch, f), n, st);
                copy_dd(chunk, ckpt_strips(tp, P, ch), cs, st);       // strips of U[it0 - 1]
            }
            // replay: chunk slot j holds the strips of U[it0 - 1 + j]
            forward_steps(d, P, S, nullptr, it0, it1, [&](int it) { return chunk + (long long)(it - it0 + 1) * cs; },
                          w.err, w.scratch, st);
            copy_dd(w.f[15], S.f[S.in], n, st);      // U[it1]
            copy_dd(w.f[16], S.f[S.ip], n, st);      // U[it1 - 1]
            reverse(it0, it1, [&](int t) { return chunk + (long long)(t - (it0 - 1)) * cs; }, true);
        }
    }
    if (stepped) {
        const int keep[7] = {lp, ln, lx, cur, rp, rn, rx};
        for (int k = 0; k < 7; ++k) seg->idx[k] = keep[k];
    }
    finalize3<<<592, 256, 0, st>>>(gacc, gcomp, is, ir, P.B, (int)rows, d->nx, P.P, P.S, grad_vp, illum_s, illum_r);
    SWEEP_LAUNCH_CHECK();
    check_err(w, st, "backward");
}

void forward(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape,
             void* ws, int64_t ws_bytes, cudaStream_t st)
{
    forward_with(d, mem_mode, ckpt_every, record, tape, ws, ws_bytes, st, nullptr, 0, 0);
}

void backward(const sweep_acoustic_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
              float* grad_vp, float* grad_w, float* illum_s, float* illum_r,
              void* ws, int64_t ws_bytes, cudaStream_t st)
{
    backward_with(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_w, illum_s, illum_r, ws, ws_bytes, st, nullptr,
                  0, 0);
}

void forward_segment(const sweep_acoustic_desc* d, int mem_mode, float* record, void* tape, void* ws,
                     int64_t ws_bytes, cudaStream_t st, StepState& seg, int it0, int it1)
{
    forward_with(d, mem_mode, 0, record, tape, ws, ws_bytes, st, &seg, it0, it1);
}

void backward_segment(const sweep_acoustic_desc* d, int mem_mode, const float* adj, const void* tape,
                      float* grad_vp, float* grad_w, float* illum_s, float* illum_r, void* ws, int64_t ws_bytes,
                      cudaStream_t st, StepState& seg, int bw0, int bw1)
{
    backward_with(d, mem_mode, 0, adj, tape, grad_vp, grad_w, illum_s, illum_r, ws, ws_bytes, st, &seg, bw0, bw1);
}

}  // namespace a3d
}  // namespace sweep
