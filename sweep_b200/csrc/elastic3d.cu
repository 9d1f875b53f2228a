// elastic3d.cu -- 3-D isotropic elastic (velocity-stress, staggered grid)
// forward and boundary-saving adjoint for sm_100a.
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
// One thread per cell on (32 x 8) tiles of x / y, one z plane and shot per
// grid row; the stencils read global memory through the read-only path.  (A
// z-marching variant with shared-memory planes and register z-queues, run at
// two CTAs per SM without a load pipeline, measured 2.8x slower in the
// forward; the kernels that beat this layout need the 3-D acoustic kernels'
// TMA plane rings.)
// Layout: fields (B, nz, ny, nx), x fastest; CPML memories in per-axis slabs
// covering the cells outside the box shrunk by one cell along their axis
// (x: (B, nz, ny, WX), y: (B, nz, WY, nx), z: (B, WZ, ny, nx)).  Cells in the
// CPML branch because of another axis have zero coefficients on this one and
// keep no memory (as the reference's stored() gating).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "elastic3d.cuh"

namespace sweep {
namespace el3d {

constexpr int M = 4;
constexpr int NTHX = 32, NTHY = 8;

// Staggered first-derivative weights of order 8 (reference
// operators/staggered.cuh:351-354).
#define W1 (1225.f / 1024.f)
#define W2 (-245.f / 3072.f)
#define W3 (49.f / 5120.f)
#define W4 (-5.f / 7168.f)

enum { VX, VY, VZ, SXX, SYY, SZZ, SXY, SXZ, SYZ, NFLD };
// memories per axis: x {vx, vy, vz, sxx, sxy, sxz}, y {vx, vy, vz, sxy, syy, syz},
// z {vx, vy, vz, sxz, syz, szz} -- the field differenced, the axis of the slab
enum { MX_VX, MX_VY, MX_VZ, MX_SXX, MX_SXY, MX_SXZ };
enum { MY_VX, MY_VY, MY_VZ, MY_SXY, MY_SYY, MY_SYZ };
enum { MZ_VX, MZ_VY, MZ_VZ, MZ_SXZ, MZ_SYZ, MZ_SZZ };

struct Slabs {
    float *x[6], *y[6], *z[6];
};

// the nine field pointers, passed by value to the point kernels
struct Fields {
    float* f[9];
};

struct Geo {
    int B, nz, ny, nx, nt;
    long long S;                    // cells per shot
    int z0, z1, y0, y1, x0, x1;     // physical box
    int SXL, SXH, SYL, SYH, SZL, SZH;   // slab sides (box edge + one cell)
    int WX, WY, WZ;
    float dt, idx, idy, idz;
    const float *az, *bz, *azh, *bzh, *ay, *by, *ayh, *byh, *ax, *bx, *axh, *bxh;
    int nsrc, nrec, nsf, nrf;
    int sf[9], rf[9];
    const int* src_loc;             // (B, nsrc, 3) runtime (x, y, z)
    const int* rec_loc;             // (B, nrec, 3)
    const float* wavelet;           // (B, nsrc, nt)
    long long ms;                   // model stride between shots (0 or S)
    const int* cells;               // strip cell offsets in a shot grid
    int ns;                         // strip cells
    int fst;                        // traction-free top face: the surface is row z0 (no pad above)
};

struct Models {
    const float *lam, *mu, *kv;     // kv = dt * (1 / rho)
    const float *vp, *vs, *rho;     // the caller's models (imaging)
};

__device__ __forceinline__ float dp(const float* __restrict__ u, long long i, long long s, float inv)
{
    return (W1 * (__ldg(u + i + s) - __ldg(u + i)) + W2 * (__ldg(u + i + 2 * s) - __ldg(u + i - s)) +
            W3 * (__ldg(u + i + 3 * s) - __ldg(u + i - 2 * s)) + W4 * (__ldg(u + i + 4 * s) - __ldg(u + i - 3 * s))) *
           inv;
}
__device__ __forceinline__ float dm(const float* __restrict__ u, long long i, long long s, float inv)
{
    return (W1 * (__ldg(u + i) - __ldg(u + i - s)) + W2 * (__ldg(u + i + s) - __ldg(u + i - 2 * s)) +
            W3 * (__ldg(u + i + 2 * s) - __ldg(u + i - 3 * s)) + W4 * (__ldg(u + i + 3 * s) - __ldg(u + i - 4 * s))) *
           inv;
}

// ------------------------------------------------ traction-free top face
// The reference's 3-D image method (common/elastic_free_surface.cuh:723-952,
// elastic3d/kernels.cuh:360-372, 1421-1499): the rows above the surface row z0
// are air, read by a z-derivative as the image of the row mirrored about the
// surface (about z0 for integer fields, z0 - 1/2 for fields half a cell
// below it, negated for odd fields); the full stencil runs over the images.
// Only the M rows from the surface down reach the air; the adjoint is the
// exact transpose, so it differs from the plain one on the M + 1 rows from
// the surface down.  The surface row's sxx and syy take the Robertsson
// correction and its szz is zeroed.
template <bool FS, bool FWD>
__device__ __forceinline__ float dz_fs(const Geo& G, const float* __restrict__ u, long long i, int iz, bool odd,
                                       bool half)
{
    const long long sz = (long long)G.nx * G.ny;
    if (!FS || iz >= G.z0 + M) return FWD ? dp(u, i, sz, G.idz) : dm(u, i, sz, G.idz);
    auto at = [&](int k) {
        if (k >= G.z0) return __ldg(u + i + (long long)(k - iz) * sz);
        const int m = half ? 2 * G.z0 - 1 - k : 2 * G.z0 - k;
        const float v = __ldg(u + i + (long long)(m - iz) * sz);
        return odd ? -v : v;
    };
    const float w[M] = {W1, W2, W3, W4};
    float g = 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m)
        g += w[m] * (FWD ? at(iz + m + 1) - at(iz - m) : at(iz + m) - at(iz - m - 1));
    return g * G.idz;
}
// negated transpose of dz_fs (the plain one: D- for a D+ forward)
template <bool FS, bool FWD>
__device__ __forceinline__ float adz_fs(const Geo& G, const float* __restrict__ q, long long i, int iz, bool odd,
                                        bool half)
{
    const long long sz = (long long)G.nx * G.ny;
    if (!FS || iz > G.z0 + M) return FWD ? dm(q, i, sz, G.idz) : dp(q, i, sz, G.idz);
    const int top = G.z0, lo = half ? top - 1 : top;
    const float par = odd ? -1.f : 1.f;
    auto at = [&](int k) { return __ldg(q + i + (long long)(k - iz) * sz); };
    const float w[M] = {W1, W2, W3, W4};
    float g = 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int jp = FWD ? iz + m : iz + m + 1;
        const int jm = FWD ? iz - m - 1 : iz - m;
        const int jg = FWD ? (half ? 2 * top - 1 + m - iz : 2 * top + m - iz)
                           : (half ? 2 * top + m - iz : 2 * top + m + 1 - iz);
        if (jp >= top) g += w[m] * at(jp);
        if (jm >= top) g -= w[m] * at(jm);
        if (iz > lo && jg >= top) g += w[m] * par * at(jg);
    }
    return g * G.idz;
}

__device__ __forceinline__ bool interior(const Geo& G, int ix, int iy, int iz)
{
    return ix >= G.x0 + 1 && ix < G.x1 - 1 && iy >= G.y0 + 1 && iy < G.y1 - 1 && iz >= G.z0 + 1 && iz < G.z1 - 1;
}
__device__ __forceinline__ bool in_core(const Geo& G, int ix, int iy, int iz)
{
    return ix >= M && ix < G.nx - M && iy >= M && iy < G.ny - M && iz >= M && iz < G.nz - M;
}
__device__ __forceinline__ bool in_box(const Geo& G, int ix, int iy, int iz)
{
    return ix >= G.x0 && ix < G.x1 && iy >= G.y0 && iy < G.y1 && iz >= G.z0 && iz < G.z1;
}
// slab offsets of a cell (-1: no memory along that axis)
__device__ __forceinline__ long long xsl(const Geo& G, int b, int iz, int iy, int ix)
{
    const int s = ix < G.SXL ? ix : (ix >= G.nx - G.SXH ? G.SXL + ix - (G.nx - G.SXH) : -1);
    return s < 0 ? -1 : (((long long)b * G.nz + iz) * G.ny + iy) * G.WX + s;
}
__device__ __forceinline__ long long ysl(const Geo& G, int b, int iz, int iy, int ix)
{
    const int s = iy < G.SYL ? iy : (iy >= G.ny - G.SYH ? G.SYL + iy - (G.ny - G.SYH) : -1);
    return s < 0 ? -1 : (((long long)b * G.nz + iz) * G.WY + s) * G.nx + ix;
}
__device__ __forceinline__ long long zsl(const Geo& G, int b, int iz, int iy, int ix)
{
    const int s = iz < G.SZL ? iz : (iz >= G.nz - G.SZH ? G.SZL + iz - (G.nz - G.SZH) : -1);
    return s < 0 ? -1 : (((long long)b * G.WZ + s) * G.ny + iy) * G.nx + ix;
}

// thread -> (b, iz, iy, ix); false past the grid
__device__ __forceinline__ bool cell_of(const Geo& G, int& b, int& iz, int& iy, int& ix)
{
    ix = blockIdx.x * NTHX + threadIdx.x;
    iy = blockIdx.y * NTHY + threadIdx.y;
    b = blockIdx.z / G.nz;
    iz = blockIdx.z - b * G.nz;
    return ix < G.nx && iy < G.ny;
}

// forward CPML memory update of derivative d along an axis: m = a m + b d,
// d += m (at == -1: no memory, the coefficients are zero there)
__device__ __forceinline__ void mem(float* __restrict__ m, long long at, float a, float b, float& d)
{
    if (at < 0) return;
    const float v = a * m[at] + b * d;
    m[at] = v;
    d += v;
}

// ------------------------------------------------------------------ forward
struct Fwd {
    Geo G;
    Models m;
    float* f[NFLD];
    Slabs mem;
};

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) vel3(Fwd A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !in_core(G, ix, iy, iz)) return;
    const long long sy = G.nx;
    const long long c = (iz * (long long)G.ny + iy) * G.nx + ix, i = b * G.S + c;
    float* const* f = A.f;
    float dsxx_dx = dp(f[SXX], i, 1, G.idx);
    float dsxy_dy = dm(f[SXY], i, sy, G.idy);
    float dsxz_dz = dz_fs<FS, false>(G, f[SXZ], i, iz, true, true);
    float dsxy_dx = dm(f[SXY], i, 1, G.idx);
    float dsyy_dy = dp(f[SYY], i, sy, G.idy);
    float dsyz_dz = dz_fs<FS, false>(G, f[SYZ], i, iz, true, true);
    float dsxz_dx = dm(f[SXZ], i, 1, G.idx);
    float dsyz_dy = dm(f[SYZ], i, sy, G.idy);
    float dszz_dz = dz_fs<FS, true>(G, f[SZZ], i, iz, true, false);
    if (!interior(G, ix, iy, iz)) {
        const long long xo = xsl(G, b, iz, iy, ix), yo = ysl(G, b, iz, iy, ix), zo = zsl(G, b, iz, iy, ix);
        mem(A.mem.z[MZ_SZZ], zo, G.azh[iz], G.bzh[iz], dszz_dz);
        mem(A.mem.x[MX_SXZ], xo, G.ax[ix], G.bx[ix], dsxz_dx);
        mem(A.mem.z[MZ_SXZ], zo, G.az[iz], G.bz[iz], dsxz_dz);
        mem(A.mem.x[MX_SXX], xo, G.axh[ix], G.bxh[ix], dsxx_dx);
        mem(A.mem.y[MY_SXY], yo, G.ay[iy], G.by[iy], dsxy_dy);
        mem(A.mem.x[MX_SXY], xo, G.ax[ix], G.bx[ix], dsxy_dx);
        mem(A.mem.y[MY_SYY], yo, G.ayh[iy], G.byh[iy], dsyy_dy);
        mem(A.mem.z[MZ_SYZ], zo, G.az[iz], G.bz[iz], dsyz_dz);
        mem(A.mem.y[MY_SYZ], yo, G.ay[iy], G.by[iy], dsyz_dy);
    }
    const float k = A.m.kv[b * G.ms + c];
    f[VX][i] += k * (dsxx_dx + dsxy_dy + dsxz_dz);
    f[VY][i] += k * (dsxy_dx + dsyy_dy + dsyz_dz);
    f[VZ][i] += k * (dsxz_dx + dsyz_dy + dszz_dz);
}

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) str3(Fwd A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !in_core(G, ix, iy, iz)) return;
    const long long sy = G.nx;
    const long long c = (iz * (long long)G.ny + iy) * G.nx + ix, i = b * G.S + c;
    float* const* f = A.f;
    float dvx_dx = dm(f[VX], i, 1, G.idx);
    float dvx_dy = dp(f[VX], i, sy, G.idy);
    float dvx_dz = dz_fs<FS, true>(G, f[VX], i, iz, false, false);
    float dvy_dx = dp(f[VY], i, 1, G.idx);
    float dvy_dy = dm(f[VY], i, sy, G.idy);
    float dvy_dz = dz_fs<FS, true>(G, f[VY], i, iz, false, false);
    float dvz_dx = dp(f[VZ], i, 1, G.idx);
    float dvz_dy = dp(f[VZ], i, sy, G.idy);
    float dvz_dz = dz_fs<FS, false>(G, f[VZ], i, iz, true, true);
    if (!interior(G, ix, iy, iz)) {
        const long long xo = xsl(G, b, iz, iy, ix), yo = ysl(G, b, iz, iy, ix), zo = zsl(G, b, iz, iy, ix);
        mem(A.mem.z[MZ_VZ], zo, G.az[iz], G.bz[iz], dvz_dz);
        mem(A.mem.y[MY_VY], yo, G.ay[iy], G.by[iy], dvy_dy);
        mem(A.mem.x[MX_VX], xo, G.ax[ix], G.bx[ix], dvx_dx);
        mem(A.mem.z[MZ_VX], zo, G.azh[iz], G.bzh[iz], dvx_dz);
        mem(A.mem.x[MX_VZ], xo, G.axh[ix], G.bxh[ix], dvz_dx);
        mem(A.mem.y[MY_VX], yo, G.ayh[iy], G.byh[iy], dvx_dy);
        mem(A.mem.x[MX_VY], xo, G.axh[ix], G.bxh[ix], dvy_dx);
        mem(A.mem.z[MZ_VY], zo, G.azh[iz], G.bzh[iz], dvy_dz);
        mem(A.mem.y[MY_VZ], yo, G.ayh[iy], G.byh[iy], dvz_dy);
    }
    const long long mi = b * G.ms + c;
    const float lam = A.m.lam[mi], mu = A.m.mu[mi];
    const float div = dvx_dx + dvy_dy + dvz_dz;
    f[SXX][i] += G.dt * (lam * div + 2.f * mu * dvx_dx);
    f[SYY][i] += G.dt * (lam * div + 2.f * mu * dvy_dy);
    f[SZZ][i] += G.dt * (lam * div + 2.f * mu * dvz_dz);
    f[SXY][i] += G.dt * mu * (dvx_dy + dvy_dx);
    f[SXZ][i] += G.dt * mu * (dvx_dz + dvz_dx);
    f[SYZ][i] += G.dt * mu * (dvy_dz + dvz_dy);
    if (FS && iz == G.z0) {   // surface row: Robertsson sxx / syy, then szz = 0
        const float rob = -G.dt * lam * (lam / (lam + 2.f * mu) * (dvx_dx + dvy_dy) + dvz_dz);
        f[SXX][i] += rob;
        f[SYY][i] += rob;
        f[SZZ][i] = 0.f;
    }
}

// Source injection of step it with sign (+1 forward, -1 taking the forward
// source back out in the reverse) into every source field; one block per shot.
__global__ void src3(const Geo G, const Fields F, int it, float sign)
{
    float* const* f = F.f;
    const int b = blockIdx.x;
    for (int s = threadIdx.x; s < G.nsrc; s += blockDim.x) {
        const int* l = G.src_loc + ((long long)b * G.nsrc + s) * 3;
        if (l[0] < 0 || l[0] >= G.nx || l[1] < 0 || l[1] >= G.ny || l[2] < 0 || l[2] >= G.nz) continue;
        const long long i = b * G.S + ((long long)l[2] * G.ny + l[1]) * G.nx + l[0];
        const float w = sign * G.wavelet[((long long)b * G.nsrc + s) * G.nt + it];
        for (int k = 0; k < G.nsf; ++k) atomicAdd(f[G.sf[k]] + i, w);
    }
}

// receivers: one thread per (shot, receiver), grid (receiver blocks, shots)
__global__ void rec3(const Geo G, const Fields F, float* record, int it)
{
    float* const* f = F.f;
    const int b = blockIdx.y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < G.nrec; r += gridDim.x * blockDim.x) {
        const int* l = G.rec_loc + ((long long)b * G.nrec + r) * 3;
        if (l[0] < 0 || l[0] >= G.nx || l[1] < 0 || l[1] >= G.ny || l[2] < 0 || l[2] >= G.nz) continue;
        const long long i = b * G.S + ((long long)l[2] * G.ny + l[1]) * G.nx + l[0];
        float* out = record + (((long long)b * G.nt + it) * G.nrec + r) * G.nrf;
        for (int k = 0; k < G.nrf; ++k) out[k] = f[G.rf[k]][i];
    }
}

// Strip save (restore = 0) of fields [f0, f1) into / restore out of one step
// slot (B, 9, ns) of the tape.
__global__ void strips3(const Geo G, const Fields F, float* slot, int f0, int f1, int restore)
{
    float* const* f = F.f;
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e / G.ns), k = (int)(e - (long long)b * G.ns);
        const long long i = b * G.S + G.cells[k];
        for (int fl = f0; fl < f1; ++fl) {
            float* t = slot + ((long long)b * NFLD + fl) * G.ns + k;
            if (restore) f[fl][i] = *t;
            else *t = f[fl][i];
        }
    }
}

// ------------------------------------------------------------------ reverse
struct Rev {
    Geo G;
    Models m;
    float* f[NFLD];      // reconstructed forward fields
    float* a[NFLD];      // adjoint fields
    float* cv[3];        // v(it + 1) carriers on the box
    float* q[9];         // prepare -> apply scratch (q, then p)
    Slabs am;            // adjoint memories
    float *gvp, *gvs, *grho;   // per-shot gradient slots (B, S)
    const float* adj;    // (B, nt, nrec, nrf)
    int it;
};

__global__ void vsrc3(Rev A)
{
    const Geo& G = A.G;
    const int b = blockIdx.x;
    for (int s = threadIdx.x; s < G.nsrc; s += blockDim.x) {
        const int* l = G.src_loc + ((long long)b * G.nsrc + s) * 3;
        if (l[0] < 0 || l[0] >= G.nx || l[1] < 0 || l[1] >= G.ny || l[2] < 0 || l[2] >= G.nz) continue;
        const long long c = ((long long)l[2] * G.ny + l[1]) * G.nx + l[0];
        const float w = G.wavelet[((long long)b * G.nsrc + s) * G.nt + A.it];
        for (int k = 0; k < G.nsf; ++k) {
            const int fl = G.sf[k];
            if (fl > VZ) continue;
            atomicAdd(A.grho + b * G.S + c, (A.a[fl][b * G.S + c] * w) / A.m.rho[b * G.ms + c]);
        }
    }
}

__global__ void res3(Rev A)
{
    const Geo& G = A.G;
    const int b = blockIdx.y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < G.nrec; r += gridDim.x * blockDim.x) {
        const int* l = G.rec_loc + ((long long)b * G.nrec + r) * 3;
        if (l[0] < 0 || l[0] >= G.nx || l[1] < 0 || l[1] >= G.ny || l[2] < 0 || l[2] >= G.nz) continue;
        const long long i = b * G.S + ((long long)l[2] * G.ny + l[1]) * G.nx + l[0];
        const float* res = A.adj + (((long long)b * G.nt + A.it) * G.nrec + r) * G.nrf;
        for (int k = 0; k < G.nrf; ++k) {
            const int fl = G.rf[k];
            atomicAdd(A.a[fl] + i, fl >= SXX ? -res[k] : res[k]);
        }
    }
}

// Receiver rho correction after the image (velocity receivers in the core).
__global__ void rrho3(Rev A)
{
    const Geo& G = A.G;
    const int b = blockIdx.y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < G.nrec; r += gridDim.x * blockDim.x) {
        const int* l = G.rec_loc + ((long long)b * G.nrec + r) * 3;
        if (!in_core(G, l[0], l[1], l[2])) continue;
        const long long c = ((long long)l[2] * G.ny + l[1]) * G.nx + l[0];
        const float* res = A.adj + (((long long)b * G.nt + A.it) * G.nrec + r) * G.nrf;
        for (int k = 0; k < G.nrf; ++k) {
            const int fl = G.rf[k];
            if (fl > VZ) continue;
            const float now = A.f[fl][b * G.S + c], nxt = A.cv[fl][b * G.S + c];
            atomicAdd(A.grho + b * G.S + c, -res[k] * (now - nxt) / A.m.rho[b * G.ms + c]);
        }
    }
}

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) srev3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !interior(G, ix, iy, iz)) return;
    const long long sy = G.nx;
    const long long c = (iz * (long long)G.ny + iy) * G.nx + ix, i = b * G.S + c;
    float* const* f = A.f;
    const float dvx_dx = dm(f[VX], i, 1, G.idx), dvx_dy = dp(f[VX], i, sy, G.idy);
    const float dvx_dz = dz_fs<FS, true>(G, f[VX], i, iz, false, false);
    const float dvy_dx = dp(f[VY], i, 1, G.idx), dvy_dy = dm(f[VY], i, sy, G.idy);
    const float dvy_dz = dz_fs<FS, true>(G, f[VY], i, iz, false, false);
    const float dvz_dx = dp(f[VZ], i, 1, G.idx), dvz_dy = dp(f[VZ], i, sy, G.idy);
    const float dvz_dz = dz_fs<FS, false>(G, f[VZ], i, iz, true, true);
    const long long mi = b * G.ms + c;
    const float lam = A.m.lam[mi], mu = A.m.mu[mi];
    const float div = dvx_dx + dvy_dy + dvz_dz;
    f[SXX][i] -= G.dt * (lam * div + 2.f * mu * dvx_dx);
    f[SYY][i] -= G.dt * (lam * div + 2.f * mu * dvy_dy);
    f[SZZ][i] -= G.dt * (lam * div + 2.f * mu * dvz_dz);
    f[SXY][i] -= G.dt * mu * (dvx_dy + dvy_dx);
    f[SXZ][i] -= G.dt * mu * (dvx_dz + dvz_dx);
    f[SYZ][i] -= G.dt * mu * (dvy_dz + dvz_dy);
}

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) vrev3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !interior(G, ix, iy, iz)) return;
    const long long sy = G.nx;
    const long long c = (iz * (long long)G.ny + iy) * G.nx + ix, i = b * G.S + c;
    float* const* f = A.f;
    const float dsxx_dx = dp(f[SXX], i, 1, G.idx), dsxy_dy = dm(f[SXY], i, sy, G.idy);
    const float dsxz_dz = dz_fs<FS, false>(G, f[SXZ], i, iz, true, true), dsxy_dx = dm(f[SXY], i, 1, G.idx);
    const float dsyy_dy = dp(f[SYY], i, sy, G.idy), dsyz_dz = dz_fs<FS, false>(G, f[SYZ], i, iz, true, true);
    const float dsxz_dx = dm(f[SXZ], i, 1, G.idx), dsyz_dy = dm(f[SYZ], i, sy, G.idy);
    const float dszz_dz = dz_fs<FS, true>(G, f[SZZ], i, iz, true, false);
    const float k = A.m.kv[b * G.ms + c];
    f[VX][i] -= k * (dsxx_dx + dsxy_dy + dsxz_dz);
    f[VY][i] -= k * (dsxy_dx + dsyy_dy + dsyz_dz);
    f[VZ][i] -= k * (dsxz_dx + dsyz_dy + dszz_dz);
}

// adjoint CPML memory of one q / p entry: t = m + bar; q = bar + b t; m' = a t
__device__ __forceinline__ float amem(float* __restrict__ m, long long at, float a, float b, float bar)
{
    if (at < 0) return bar;
    const float t = m[at] + bar;
    m[at] = a * t;
    return bar + b * t;
}

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) sprep3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix)) return;
    const long long sy = G.nx;
    const long long c = (iz * (long long)G.ny + iy) * G.nx + ix, i = b * G.S + c, mi = b * G.ms + c;
    const float lam = A.m.lam[mi], mu = A.m.mu[mi], l2m = lam + 2.f * mu;
    const bool surf = FS && iz == G.z0;
    if (surf) A.a[SZZ][i] = 0.f;   // the surface row's adjoint szz (its forward value is zeroed)
    const float bsxx = A.a[SXX][i], bsyy = A.a[SYY][i], bszz = surf ? 0.f : A.a[SZZ][i];
    const float bsxy = A.a[SXY][i], bsxz = A.a[SXZ][i], bsyz = A.a[SYZ][i];
    if (in_box(G, ix, iy, iz)) {
        float* const* f = A.f;
        const float fvx_x = dm(f[VX], i, 1, G.idx), fvx_y = dp(f[VX], i, sy, G.idy);
        const float fvx_z = dz_fs<FS, true>(G, f[VX], i, iz, false, false);
        const float fvy_x = dp(f[VY], i, 1, G.idx), fvy_y = dm(f[VY], i, sy, G.idy);
        const float fvy_z = dz_fs<FS, true>(G, f[VY], i, iz, false, false);
        const float fvz_x = dp(f[VZ], i, 1, G.idx), fvz_y = dp(f[VZ], i, sy, G.idy);
        const float fvz_z = dz_fs<FS, false>(G, f[VZ], i, iz, true, true);
        const float rho = A.m.rho[mi], vp = A.m.vp[mi], vs = A.m.vs[mi];
        float gl, gm;
        if (surf) {
            // the surface row's corrected sxx / syy updates (kernels.cuh:1440-1452)
            const float vp2 = vp * vp, vs2 = vs * vs, vp4 = vp2 * vp2;
            const float dcl = 4.f * vs2 * vs2 / vp4;
            const float dcm = 4.f * (vp4 - 2.f * vp2 * vs2 + 2.f * vs2 * vs2) / vp4;
            const float dc2m = 2.f * (vp2 - 2.f * vs2) * (vp2 - 2.f * vs2) / vp4;
            gl = dcl * (bsxx + bsyy) * (fvx_x + fvy_y);
            gm = bsxx * (dcm * fvx_x + dc2m * fvy_y) + bsyy * (dc2m * fvx_x + dcm * fvy_y) + bsxz * (fvx_z + fvz_x) +
                 bsxy * (fvx_y + fvy_x) + bsyz * (fvy_z + fvz_y);
        } else {
            gl = (bsxx + bsyy + bszz) * (fvx_x + fvy_y + fvz_z);
            gm = 2.f * (bsxx * fvx_x + bsyy * fvy_y + bszz * fvz_z) + bsxz * (fvx_z + fvz_x) +
                 bsxy * (fvx_y + fvy_x) + bsyz * (fvy_z + fvz_y);
        }
        A.gvp[i] += -2.f * rho * vp * gl * G.dt;
        A.gvs[i] += -(-4.f * rho * vs * gl + 2.f * rho * vs * gm) * G.dt;
        float gr = (A.a[VX][i] * (f[VX][i] - A.cv[0][i]) + A.a[VY][i] * (f[VY][i] - A.cv[1][i]) +
                    A.a[VZ][i] * (f[VZ][i] - A.cv[2][i])) / rho;
        gr -= gl * (vp * vp - 2.f * vs * vs) * G.dt + gm * (vs * vs) * G.dt;
        A.grho[i] += gr;
    }
    float qxx, qyy, qzz;
    if (surf) {   // transposes of the corrected surface updates
        const float coef = 4.f * mu * (lam + mu) / l2m, coef2 = 2.f * lam * mu / l2m;
        qxx = G.dt * (coef * bsxx + coef2 * bsyy);
        qyy = G.dt * (coef2 * bsxx + coef * bsyy);
        qzz = 0.f;
    } else {
        qxx = G.dt * (l2m * bsxx + lam * bsyy + lam * bszz);
        qyy = G.dt * (lam * bsxx + l2m * bsyy + lam * bszz);
        qzz = G.dt * (lam * bsxx + lam * bsyy + l2m * bszz);
    }
    float qxy = G.dt * mu * bsxy, qxz = G.dt * mu * bsxz;
    float qyx = G.dt * mu * bsxy, qyz = G.dt * mu * bsyz;
    float qzx = G.dt * mu * bsxz, qzy = G.dt * mu * bsyz;
    if (!interior(G, ix, iy, iz)) {
        const long long xo = xsl(G, b, iz, iy, ix), yo = ysl(G, b, iz, iy, ix), zo = zsl(G, b, iz, iy, ix);
        qxx = amem(A.am.x[MX_VX], xo, G.ax[ix], G.bx[ix], qxx);
        qyx = amem(A.am.x[MX_VY], xo, G.axh[ix], G.bxh[ix], qyx);
        qzx = amem(A.am.x[MX_VZ], xo, G.axh[ix], G.bxh[ix], qzx);
        qxy = amem(A.am.y[MY_VX], yo, G.ayh[iy], G.byh[iy], qxy);
        qyy = amem(A.am.y[MY_VY], yo, G.ay[iy], G.by[iy], qyy);
        qzy = amem(A.am.y[MY_VZ], yo, G.ayh[iy], G.byh[iy], qzy);
        qxz = amem(A.am.z[MZ_VX], zo, G.azh[iz], G.bzh[iz], qxz);
        qyz = amem(A.am.z[MZ_VY], zo, G.azh[iz], G.bzh[iz], qyz);
        qzz = amem(A.am.z[MZ_VZ], zo, G.az[iz], G.bz[iz], qzz);
    }
    A.q[0][i] = qxx; A.q[1][i] = qxy; A.q[2][i] = qxz;
    A.q[3][i] = qyx; A.q[4][i] = qyy; A.q[5][i] = qyz;
    A.q[6][i] = qzx; A.q[7][i] = qzy; A.q[8][i] = qzz;
}

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) sapp3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !in_core(G, ix, iy, iz)) return;
    const long long sy = G.nx;
    const long long i = b * G.S + (iz * (long long)G.ny + iy) * G.nx + ix;
    float* const* q = A.q;
    A.a[VX][i] += dp(q[0], i, 1, G.idx) + dm(q[1], i, sy, G.idy) + adz_fs<FS, true>(G, q[2], i, iz, false, false);
    A.a[VY][i] += dm(q[3], i, 1, G.idx) + dp(q[4], i, sy, G.idy) + adz_fs<FS, true>(G, q[5], i, iz, false, false);
    A.a[VZ][i] += dm(q[6], i, 1, G.idx) + dm(q[7], i, sy, G.idy) + adz_fs<FS, false>(G, q[8], i, iz, true, true);
}

__global__ void __launch_bounds__(NTHX * NTHY) vprep3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix)) return;
    const long long c = (iz * (long long)G.ny + iy) * G.nx + ix, i = b * G.S + c;
    const float k = A.m.kv[b * G.ms + c];
    const float bx_ = k * A.a[VX][i], by_ = k * A.a[VY][i], bz_ = k * A.a[VZ][i];
    float pxx = bx_, pxy = bx_, pxz = bx_, pyx = by_, pyy = by_, pyz = by_, pzx = bz_, pzy = bz_, pzz = bz_;
    if (!interior(G, ix, iy, iz)) {
        const long long xo = xsl(G, b, iz, iy, ix), yo = ysl(G, b, iz, iy, ix), zo = zsl(G, b, iz, iy, ix);
        pxx = amem(A.am.x[MX_SXX], xo, G.axh[ix], G.bxh[ix], pxx);
        pyx = amem(A.am.x[MX_SXY], xo, G.ax[ix], G.bx[ix], pyx);
        pzx = amem(A.am.x[MX_SXZ], xo, G.ax[ix], G.bx[ix], pzx);
        pxy = amem(A.am.y[MY_SXY], yo, G.ay[iy], G.by[iy], pxy);
        pyy = amem(A.am.y[MY_SYY], yo, G.ayh[iy], G.byh[iy], pyy);
        pzy = amem(A.am.y[MY_SYZ], yo, G.ay[iy], G.by[iy], pzy);
        pxz = amem(A.am.z[MZ_SXZ], zo, G.az[iz], G.bz[iz], pxz);
        pyz = amem(A.am.z[MZ_SYZ], zo, G.az[iz], G.bz[iz], pyz);
        pzz = amem(A.am.z[MZ_SZZ], zo, G.azh[iz], G.bzh[iz], pzz);
    }
    A.q[0][i] = pxx; A.q[1][i] = pxy; A.q[2][i] = pxz;
    A.q[3][i] = pyx; A.q[4][i] = pyy; A.q[5][i] = pyz;
    A.q[6][i] = pzx; A.q[7][i] = pzy; A.q[8][i] = pzz;
}

template <bool FS>
__global__ void __launch_bounds__(NTHX * NTHY) vapp3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !in_core(G, ix, iy, iz)) return;
    const long long sy = G.nx;
    const long long i = b * G.S + (iz * (long long)G.ny + iy) * G.nx + ix;
    float* const* p = A.q;
    A.a[SXX][i] += dm(p[0], i, 1, G.idx);
    A.a[SXY][i] += dp(p[1], i, sy, G.idy) + dp(p[3], i, 1, G.idx);
    A.a[SXZ][i] += adz_fs<FS, false>(G, p[2], i, iz, true, true) + dp(p[6], i, 1, G.idx);
    A.a[SYY][i] += dm(p[4], i, sy, G.idy);
    A.a[SYZ][i] += adz_fs<FS, false>(G, p[5], i, iz, true, true) + dp(p[7], i, sy, G.idy);
    A.a[SZZ][i] += adz_fs<FS, true>(G, p[8], i, iz, true, false);
}

// v(it) carriers on the box (they hold v(it + 1) for the next reverse step)
__global__ void __launch_bounds__(NTHX * NTHY) cap3(Rev A)
{
    const Geo& G = A.G;
    int b, iz, iy, ix;
    if (!cell_of(G, b, iz, iy, ix) || !in_box(G, ix, iy, iz)) return;
    const long long i = b * G.S + (iz * (long long)G.ny + iy) * G.nx + ix;
    for (int k = 0; k < 3; ++k) A.cv[k][i] = A.f[k][i];
}

__global__ void prep3(const float* __restrict__ vp, const float* __restrict__ vs, const float* __restrict__ rho,
                      long long n, float dt, float* olam, float* omu, float* okv)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const float v = vp[k], s = vs[k], r = rho[k];
        omu[k] = __fmul_rn(__fmul_rn(r, s), s);
        olam[k] = __fmul_rn(r, __fsub_rn(__fmul_rn(v, v), __fmul_rn(__fmul_rn(2.0f, s), s)));
        okv[k] = dt * (1.f / r);
    }
}

// Gradient output: the shots' slots summed in shot order (shared model) or
// copied (per-shot models) on the physical box, zero elsewhere.
__global__ void finalize3(const float* __restrict__ slots, int B, int per_shot, Geo G, float* out)
{
    const int nout = per_shot ? B : 1;
    const long long n = (long long)nout * G.S;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long b = k / G.S, c = k - b * G.S;
        const int iz = (int)(c / ((long long)G.ny * G.nx));
        const int iy = (int)((c / G.nx) % G.ny), ix = (int)(c % G.nx);
        float v = 0.f;
        if (in_box(G, ix, iy, iz)) {
            if (per_shot) v = slots[k];
            else
                for (int s = 0; s < B; ++s) v += slots[s * G.S + c];
        }
        out[k] = v;
    }
}

// ------------------------------------------------------------------- host
struct Plan {
    Geo G;
    int nm;                      // model copies
    std::vector<int> cells;      // strip cells
};

static Plan make_plan(const sweep_elastic3d_desc* d, int mem_mode)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->M == M, "elastic3d: only spatial order 8 (M = 4) is built (got M = %d)", d->M);
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY,
                  "elastic3d: boundary saving with fp32 strips in device memory is built (mem_mode %d)", mem_mode);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1, "elastic3d: B and nt must be >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "elastic3d: negative source/receiver count");
    SWEEP_REQUIRE(d->nsrc_fields >= 1 && d->nsrc_fields <= 9, "elastic3d: 1 to 9 source fields (got %d)",
                  d->nsrc_fields);
    for (int k = 0; k < d->nsrc_fields; ++k) {
        SWEEP_REQUIRE(d->src_fields[k] >= 0 && d->src_fields[k] < NFLD, "elastic3d: bad source field %d",
                      d->src_fields[k]);
        for (int j = 0; j < k; ++j)
            SWEEP_REQUIRE(d->src_fields[j] != d->src_fields[k], "elastic3d: source field %d repeated",
                          d->src_fields[k]);
    }
    SWEEP_REQUIRE(d->nrec_fields >= 1 && d->nrec_fields <= 9, "elastic3d: 1 to 9 receiver fields (got %d)",
                  d->nrec_fields);
    for (int k = 0; k < d->nrec_fields; ++k)
        SWEEP_REQUIRE(d->rec_fields[k] >= 0 && d->rec_fields[k] < NFLD, "elastic3d: bad receiver field %d",
                      d->rec_fields[k]);
    if (d->free_surface)
        SWEEP_REQUIRE(d->pad[0] == 0, "elastic3d: a free top face has no PML pad (got %d)", d->pad[0]);
    for (int f = d->free_surface ? 1 : 0; f < 6; ++f)
        SWEEP_REQUIRE(d->pad[f] >= 1, "elastic3d: every absorbing face needs a PML pad >= 1 (face %d has %d)", f,
                      d->pad[f]);
    Plan pl{};
    Geo& G = pl.G;
    G.fst = d->free_surface ? 1 : 0;
    G.B = d->B; G.nz = d->nz; G.ny = d->ny; G.nx = d->nx; G.nt = d->nt;
    G.S = (long long)d->nz * d->ny * d->nx;
    SWEEP_REQUIRE(G.S < (1LL << 31), "elastic3d: one shot's grid must hold < 2^31 cells");
    G.z0 = d->pad[0] + M; G.z1 = d->nz - d->pad[1] - M;
    G.y0 = d->pad[2] + M; G.y1 = d->ny - d->pad[3] - M;
    G.x0 = d->pad[4] + M; G.x1 = d->nx - d->pad[5] - M;
    SWEEP_REQUIRE(G.z1 - G.z0 >= 2 && G.y1 - G.y0 >= 2 && G.x1 - G.x0 >= 2,
                  "elastic3d: the physical box must be at least 2 cells along every axis");
    G.SZL = std::min(G.z0 + 1, d->nz); G.SZH = std::min(d->nz - (G.z1 - 1), d->nz - G.SZL);
    G.SYL = std::min(G.y0 + 1, d->ny); G.SYH = std::min(d->ny - (G.y1 - 1), d->ny - G.SYL);
    G.SXL = std::min(G.x0 + 1, d->nx); G.SXH = std::min(d->nx - (G.x1 - 1), d->nx - G.SXL);
    G.WX = G.SXL + G.SXH; G.WY = G.SYL + G.SYH; G.WZ = G.SZL + G.SZH;
    G.dt = d->dt; G.idx = 1.f / d->dx; G.idy = 1.f / d->dy; G.idz = 1.f / d->dz;
    G.az = d->az; G.bz = d->bz; G.azh = d->azh; G.bzh = d->bzh;
    G.ay = d->ay; G.by = d->by; G.ayh = d->ayh; G.byh = d->byh;
    G.ax = d->ax; G.bx = d->bx; G.axh = d->axh; G.bxh = d->bxh;
    G.nsrc = d->nsrc; G.nrec = d->nrec;
    G.nsf = d->nsrc_fields; G.nrf = d->nrec_fields;
    for (int k = 0; k < 9; ++k) { G.sf[k] = d->src_fields[k]; G.rf[k] = d->rec_fields[k]; }
    G.src_loc = d->src_loc; G.rec_loc = d->rec_loc; G.wavelet = d->wavelet;
    const bool per_shot = d->model_stride != 0;
    SWEEP_REQUIRE(!per_shot || d->model_stride == G.S, "elastic3d: model_stride must be 0 or nz * ny * nx");
    G.ms = per_shot ? G.S : 0;
    pl.nm = per_shot ? d->B : 1;
    // strip cells: per face a band M + 1 wide from M cells outside the box,
    // spanning the box along the other two axes (each cell once)
    std::vector<char> mark((size_t)G.S, 0);
    auto put = [&](int z, int y, int x) { mark[((size_t)z * G.ny + y) * G.nx + x] = 1; };
    for (int z = G.z0 - M; z <= G.z0; ++z)
        for (int y = G.y0; y < G.y1; ++y)
            for (int x = G.x0; x < G.x1; ++x) { put(z, y, x); put(G.z1 - 1 + (G.z0 - z), y, x); }
    for (int z = G.z0; z < G.z1; ++z) {
        for (int y = G.y0 - M; y <= G.y0; ++y)
            for (int x = G.x0; x < G.x1; ++x) { put(z, y, x); put(z, G.y1 - 1 + (G.y0 - y), x); }
        for (int y = G.y0; y < G.y1; ++y)
            for (int x = G.x0 - M; x <= G.x0; ++x) { put(z, y, x); put(z, y, G.x1 - 1 + (G.x0 - x)); }
    }
    for (size_t c = 0; c < mark.size(); ++c)
        if (mark[c]) pl.cells.push_back((int)c);
    G.ns = (int)pl.cells.size();
    return pl;
}

struct Common {
    float *lam, *mu, *kv;
    int* cells;
};

static void carve_common(Carve& c, const Plan& pl, Common& w)
{
    const long long mc = (long long)pl.nm * pl.G.S;
    w.lam = c.take<float>(mc); w.mu = c.take<float>(mc); w.kv = c.take<float>(mc);
    w.cells = c.take<int>(std::max(pl.G.ns, 1));
}

static void carve_slabs(Carve& c, const Geo& G, Slabs& s)
{
    for (int k = 0; k < 6; ++k) s.x[k] = c.take<float>((long long)G.B * G.nz * G.ny * G.WX);
    for (int k = 0; k < 6; ++k) s.y[k] = c.take<float>((long long)G.B * G.nz * G.WY * G.nx);
    for (int k = 0; k < 6; ++k) s.z[k] = c.take<float>((long long)G.B * G.WZ * G.ny * G.nx);
}

struct FwdWs {
    Common cm;
    float* f[NFLD];
    Slabs mem;
    char *zero0, *zero1;
};

static void carve_fwd(Carve& c, const Plan& pl, FwdWs& w)
{
    carve_common(c, pl, w.cm);
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    for (int k = 0; k < NFLD; ++k) w.f[k] = c.take<float>((long long)pl.G.B * pl.G.S);
    carve_slabs(c, pl.G, w.mem);
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
}

struct RevWs {
    Common cm;
    float* f[NFLD];
    float* a[NFLD];
    float* cv[3];
    float* q[9];
    Slabs am;
    float *gvp, *gvs, *grho;
    char *zero0, *zero1;
};

static void carve_rev(Carve& c, const Plan& pl, RevWs& w)
{
    carve_common(c, pl, w.cm);
    const Geo& G = pl.G;
    const long long n = (long long)G.B * G.S;
    for (int k = 0; k < NFLD; ++k) w.f[k] = c.take<float>(n);
    for (int k = 0; k < 9; ++k) w.q[k] = c.take<float>(n);
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    for (int k = 0; k < NFLD; ++k) w.a[k] = c.take<float>(n);
    for (int k = 0; k < 3; ++k) w.cv[k] = c.take<float>(n);
    carve_slabs(c, G, w.am);
    w.gvp = c.take<float>(n); w.gvs = c.take<float>(n); w.grho = c.take<float>(n);
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
}

static long long step_floats(const Plan& pl) { return (long long)pl.G.B * NFLD * pl.G.ns; }
static int64_t tape_bytes_of(const Plan& pl)
{
    return ((long long)pl.G.nt * step_floats(pl) + (long long)NFLD * pl.G.B * pl.G.S) * 4;
}

void sizes(const sweep_elastic3d_desc* d, int mem_mode, int, int64_t* ws_bytes, int64_t* tape_bytes)
{
    const Plan pl = make_plan(d, mem_mode);
    Carve f(nullptr), r(nullptr);
    FwdWs fw{};
    RevWs rw{};
    carve_fwd(f, pl, fw);
    carve_rev(r, pl, rw);
    *ws_bytes = std::max(f.off, r.off);
    *tape_bytes = tape_bytes_of(pl);
}

static void setup_common(const sweep_elastic3d_desc* d, const Plan& pl, const Common& w, cudaStream_t st)
{
    const long long n = (long long)pl.nm * pl.G.S;
    prep3<<<592, 256, 0, st>>>(d->vp, d->vs, d->rho, n, d->dt, w.lam, w.mu, w.kv);
    SWEEP_LAUNCH_CHECK();
    if (pl.G.ns > 0)
        SWEEP_CUDA(cudaMemcpyAsync(w.cells, pl.cells.data(), sizeof(int) * pl.G.ns, cudaMemcpyHostToDevice, st));
}

static Models models_of(const sweep_elastic3d_desc* d, const Common& w)
{
    return Models{w.lam, w.mu, w.kv, d->vp, d->vs, d->rho};
}

static dim3 rec_grid(const Geo& G)
{
    return dim3((unsigned)std::min((G.nrec + 127) / 128, 64), (unsigned)G.B);
}

static dim3 cell_grid(const Geo& G)
{
    return dim3((G.nx + NTHX - 1) / NTHX, (G.ny + NTHY - 1) / NTHY, (unsigned)(G.nz * G.B));
}

void forward(const sweep_elastic3d_desc* d, int mem_mode, int, float* record, void* tape, void* ws, int64_t ws_bytes,
             cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
    Carve c(ws);
    FwdWs w{};
    carve_fwd(c, pl, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic3d forward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    Geo& G = pl.G;
    G.cells = w.cm.cells;
    setup_common(d, pl, w.cm, st);
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
    if (record && G.nrec > 0)
        SWEEP_CUDA(cudaMemsetAsync(record, 0, sizeof(float) * (size_t)G.B * G.nt * G.nrec * G.nrf, st));
    Fwd A{};
    A.G = G;
    A.m = models_of(d, w.cm);
    for (int k = 0; k < NFLD; ++k) A.f[k] = w.f[k];
    A.mem = w.mem;
    Fields F{};
    for (int k = 0; k < NFLD; ++k) F.f[k] = w.f[k];
    const dim3 grid = cell_grid(G), block(NTHX, NTHY);
    float* slots = static_cast<float*>(tape);
    const unsigned sblocks = (unsigned)std::min<long long>(((long long)G.B * G.ns + 255) / 256, 4096);
    for (int it = 0; it < G.nt; ++it) {
        if (G.fst) {
            vel3<true><<<grid, block, 0, st>>>(A);
            str3<true><<<grid, block, 0, st>>>(A);
        } else {
            vel3<false><<<grid, block, 0, st>>>(A);
            str3<false><<<grid, block, 0, st>>>(A);
        }
        if (G.nsrc > 0) src3<<<G.B, 128, 0, st>>>(G, F, it, 1.f);
        if (slots && G.ns > 0)
            strips3<<<sblocks, 256, 0, st>>>(G, F, slots + (long long)it * step_floats(pl), 0, NFLD, 0);
        if (record && G.nrec > 0) rec3<<<rec_grid(G), 128, 0, st>>>(G, F, record, it);
        SWEEP_LAUNCH_CHECK();
    }
    if (slots) {
        float* fin = slots + (long long)G.nt * step_floats(pl);
        for (int k = 0; k < NFLD; ++k)
            SWEEP_CUDA(cudaMemcpyAsync(fin + (long long)k * G.B * G.S, w.f[k], sizeof(float) * G.B * G.S,
                                       cudaMemcpyDeviceToDevice, st));
    }
}

void backward(const sweep_elastic3d_desc* d, int mem_mode, int, const float* adj, const void* tape, float* grad_vp,
              float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
    SWEEP_REQUIRE(tape != nullptr, "elastic3d backward: the forward's tape is required");
    Carve c(ws);
    RevWs w{};
    carve_rev(c, pl, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic3d backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    Geo& G = pl.G;
    G.cells = w.cm.cells;
    setup_common(d, pl, w.cm, st);
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
    const float* slots = static_cast<const float*>(tape);
    const float* fin = slots + (long long)G.nt * step_floats(pl);
    for (int k = 0; k < NFLD; ++k)
        SWEEP_CUDA(cudaMemcpyAsync(w.f[k], fin + (long long)k * G.B * G.S, sizeof(float) * G.B * G.S,
                                   cudaMemcpyDeviceToDevice, st));
    Rev A{};
    A.G = G;
    A.m = models_of(d, w.cm);
    for (int k = 0; k < NFLD; ++k) { A.f[k] = w.f[k]; A.a[k] = w.a[k]; }
    for (int k = 0; k < 3; ++k) A.cv[k] = w.cv[k];
    for (int k = 0; k < 9; ++k) A.q[k] = w.q[k];
    A.am = w.am;
    A.gvp = w.gvp; A.gvs = w.gvs; A.grho = w.grho;
    A.adj = adj;
    Fields F{};
    for (int k = 0; k < NFLD; ++k) F.f[k] = w.f[k];
    const dim3 grid = cell_grid(G), block(NTHX, NTHY);
    const unsigned sblocks = (unsigned)std::min<long long>(((long long)G.B * G.ns + 255) / 256, 4096);
    bool vsrc = false;
    for (int k = 0; k < G.nsf; ++k) vsrc |= G.sf[k] <= VZ;
    for (int it = G.nt - 1; it >= 1; --it) {
        A.it = it;
        float* prev = const_cast<float*>(slots) + (long long)(it - 1) * step_floats(pl);
        if (vsrc && G.nsrc > 0) vsrc3<<<G.B, 128, 0, st>>>(A);
        if (G.nrec > 0) res3<<<rec_grid(G), 128, 0, st>>>(A);
        if (G.nsrc > 0) src3<<<G.B, 128, 0, st>>>(G, F, it, -1.f);
        if (G.fst) srev3<true><<<grid, block, 0, st>>>(A);
        else srev3<false><<<grid, block, 0, st>>>(A);
        if (G.ns > 0) strips3<<<sblocks, 256, 0, st>>>(G, F, prev, SXX, NFLD, 1);
        if (G.fst) sprep3<true><<<grid, block, 0, st>>>(A);
        else sprep3<false><<<grid, block, 0, st>>>(A);
        if (G.nrec > 0) rrho3<<<rec_grid(G), 128, 0, st>>>(A);
        if (G.fst) sapp3<true><<<grid, block, 0, st>>>(A);
        else sapp3<false><<<grid, block, 0, st>>>(A);
        vprep3<<<grid, block, 0, st>>>(A);
        if (G.fst) vapp3<true><<<grid, block, 0, st>>>(A);
        else vapp3<false><<<grid, block, 0, st>>>(A);
        cap3<<<grid, block, 0, st>>>(A);
        if (G.fst) vrev3<true><<<grid, block, 0, st>>>(A);
        else vrev3<false><<<grid, block, 0, st>>>(A);
        if (G.ns > 0) strips3<<<sblocks, 256, 0, st>>>(G, F, prev, VX, SXX, 1);
        SWEEP_LAUNCH_CHECK();
    }
    const int per_shot = d->model_stride != 0;
    finalize3<<<592, 256, 0, st>>>(w.gvp, G.B, per_shot, G, grad_vp);
    finalize3<<<592, 256, 0, st>>>(w.gvs, G.B, per_shot, G, grad_vs);
    finalize3<<<592, 256, 0, st>>>(w.grho, G.B, per_shot, G, grad_rho);
    SWEEP_LAUNCH_CHECK();
}

}  // namespace el3d
}  // namespace sweep
