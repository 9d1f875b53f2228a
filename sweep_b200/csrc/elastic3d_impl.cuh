// elastic3d_impl.cuh -- the body of the 3-D isotropic elastic path (see
// elastic3d.cu), compiled once per spatial order: the including file defines
// EL3D_M (the stencil half-width, 1..4) and EL3D_NS (the namespace of that
// order's kernels and entry points).  No include guard: one translation unit
// may include it for several orders.
#ifndef EL3D_M
#error "define EL3D_M (the stencil half-width) before including elastic3d_impl.cuh"
#endif
#ifndef EL3D_NS
#error "define EL3D_NS (the namespace of this order) before including elastic3d_impl.cuh"
#endif

namespace sweep {
namespace EL3D_NS {

constexpr int M = EL3D_M;
constexpr int NTHX = 32, NTHY = 4, NTHZ = 2;

// Staggered first-derivative weight k of order 2M (reference
// operators/staggered.cuh:146-147 order 4, 248-250 order 6, 351-354 order 8;
// order 2: the plain difference)
__host__ __device__ constexpr float wt(int k)
{
    return M == 1   ? 1.f
           : M == 2 ? (k == 1 ? 9.f / 8.f : -1.f / 24.f)
           : M == 3 ? (k == 1 ? 75.f / 64.f : k == 2 ? -25.f / 384.f : 3.f / 640.f)
                    : (k == 1 ? 1225.f / 1024.f : k == 2 ? -245.f / 3072.f : k == 3 ? 49.f / 5120.f : -5.f / 7168.f);
}

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

// Boundary-strip storage of the boundary-saving tape.  fp32 and bf16 keep the
// strip set (B, 9, ns), each cell once; fp16 and int8 keep the reference's six
// faces per field -- bands M + 1 wide starting M cells outside the box (z faces
// across the box, y and x faces over its z range, so edge cells sit in two or
// three faces) -- each quantised per field and shot in blocks of kQB cells
// against the block's max |value| (reference boundarysaver.cu:207-460 face
// layout, boundary/strip.cuh:136-175 bands with offset -M and width M + 1,
// boundary/runtime.cuh:313-330 and boundarysaver.cu:925-1095 quantisation).
enum StripFmt { SF_F32 = 0, SF_F16 = 1, SF_BF16 = 2, SF_I8 = 3 };
constexpr int kQB = 256;
constexpr int BW = M + 1;           // face band width

struct StripStore {
    int fmt;                        // StripFmt
    int cells[6], blocks[6];        // per field and shot, per face (top, bottom, front, back, left, right)
    long long pay[6], scl[6];       // byte offsets of each face's codes (9, B, cells) and scales (9, B, blocks)
    long long step;                 // bytes of one step slot
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
    StripStore st;
};

struct Models {
    const float *lam, *mu, *kv;     // kv = dt * (1 / rho)
    const float *vp, *vs, *rho;     // the caller's models (imaging)
};

#if EL3D_M == 4
// order 8 as one expression of the four taps: the form the order-8 kernels
// were tuned in (a loop over wt(k) changes their register allocation and runs
// the step 10 % slower)
__device__ __forceinline__ float dp(const float* __restrict__ u, long long i, long long s, float inv)
{
    return (wt(1) * (__ldg(u + i + s) - __ldg(u + i)) + wt(2) * (__ldg(u + i + 2 * s) - __ldg(u + i - s)) +
            wt(3) * (__ldg(u + i + 3 * s) - __ldg(u + i - 2 * s)) +
            wt(4) * (__ldg(u + i + 4 * s) - __ldg(u + i - 3 * s))) *
           inv;
}
__device__ __forceinline__ float dm(const float* __restrict__ u, long long i, long long s, float inv)
{
    return (wt(1) * (__ldg(u + i) - __ldg(u + i - s)) + wt(2) * (__ldg(u + i + s) - __ldg(u + i - 2 * s)) +
            wt(3) * (__ldg(u + i + 2 * s) - __ldg(u + i - 3 * s)) +
            wt(4) * (__ldg(u + i + 3 * s) - __ldg(u + i - 4 * s))) *
           inv;
}
#else
__device__ __forceinline__ float dp(const float* __restrict__ u, long long i, long long s, float inv)
{
    float g = wt(1) * (__ldg(u + i + s) - __ldg(u + i));
#pragma unroll
    for (int k = 2; k <= M; ++k) g = g + wt(k) * (__ldg(u + i + k * s) - __ldg(u + i - (k - 1) * s));
    return g * inv;
}
__device__ __forceinline__ float dm(const float* __restrict__ u, long long i, long long s, float inv)
{
    float g = wt(1) * (__ldg(u + i) - __ldg(u + i - s));
#pragma unroll
    for (int k = 2; k <= M; ++k) g = g + wt(k) * (__ldg(u + i + (k - 1) * s) - __ldg(u + i - k * s));
    return g * inv;
}
#endif

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
    float w[M];
#pragma unroll
    for (int m = 0; m < M; ++m) w[m] = wt(m + 1);
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
    float w[M];
#pragma unroll
    for (int m = 0; m < M; ++m) w[m] = wt(m + 1);
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

// thread -> (b, iz, iy, ix) on NTHX x NTHY x NTHZ blocks (NTHZ z planes of a
// shot per grid row); false past the grid
__device__ __forceinline__ bool cell_of(const Geo& G, int& b, int& iz, int& iy, int& ix)
{
    const int zb = (G.nz + NTHZ - 1) / NTHZ;
    ix = blockIdx.x * NTHX + threadIdx.x;
    iy = blockIdx.y * NTHY + threadIdx.y;
    b = blockIdx.z / zb;
    iz = (blockIdx.z - b * zb) * NTHZ + threadIdx.z;
    return ix < G.nx && iy < G.ny && iz < G.nz;
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) vel3(Fwd A)
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) str3(Fwd A)
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

// Face f cell idx (of one field and shot) of the scaled formats -> grid cell:
// z faces (band, box y, box x), y faces (box z, band, box x), x faces (box z,
// box y, band).
__device__ __forceinline__ void face_cell(const Geo& G, int f, int idx, int& iz, int& iy, int& ix)
{
    const int bx = G.x1 - G.x0, by = G.y1 - G.y0;
    if (f < 2) {
        ix = G.x0 + idx % bx; idx /= bx;
        iy = G.y0 + idx % by;
        iz = (f == 0 ? G.z0 - M : G.z1 - 1) + idx / by;
    } else if (f < 4) {
        ix = G.x0 + idx % bx; idx /= bx;
        iy = (f == 2 ? G.y0 - M : G.y1 - 1) + idx % BW;
        iz = G.z0 + idx / BW;
    } else {
        ix = (f == 4 ? G.x0 - M : G.x1 - 1) + idx % BW; idx /= BW;
        iy = G.y0 + idx % by;
        iz = G.z0 + idx / by;
    }
}

// The face a scaled-format restore reads strip cell (iz, iy, ix) from: the
// last of the faces holding it in the reference's write order (top, bottom,
// front, back, left, right), and the cell's index in that face.
__device__ __forceinline__ int face_index(const Geo& G, int iz, int iy, int ix, int& f)
{
    const int bx = G.x1 - G.x0, by = G.y1 - G.y0;
    const bool zin = iz >= G.z0 && iz < G.z1, yin = iy >= G.y0 && iy < G.y1, xin = ix >= G.x0 && ix < G.x1;
    if (zin && yin && ix >= G.x1 - 1 && ix < G.x1 - 1 + BW) { f = 5; return ((iz - G.z0) * by + iy - G.y0) * BW + ix - (G.x1 - 1); }
    if (zin && yin && ix >= G.x0 - M && ix <= G.x0) { f = 4; return ((iz - G.z0) * by + iy - G.y0) * BW + ix - (G.x0 - M); }
    if (zin && xin && iy >= G.y1 - 1 && iy < G.y1 - 1 + BW) { f = 3; return ((iz - G.z0) * BW + iy - (G.y1 - 1)) * bx + ix - G.x0; }
    if (zin && xin && iy >= G.y0 - M && iy <= G.y0) { f = 2; return ((iz - G.z0) * BW + iy - (G.y0 - M)) * bx + ix - G.x0; }
    if (iz >= G.z1 - 1) { f = 1; return ((iz - (G.z1 - 1)) * by + iy - G.y0) * bx + ix - G.x0; }
    f = 0;
    return ((iz - (G.z0 - M)) * by + iy - G.y0) * bx + ix - G.x0;
}

// a[f] of a per-face parameter array without a local-memory copy of the array
template <class T>
__device__ __forceinline__ T pick6(const T (&a)[6], int f)
{
    T v = a[0];
#pragma unroll
    for (int k = 1; k < 6; ++k)
        if (f == k) v = a[k];
    return v;
}

// Saved value of field fl at grid cell c of shot b in a scaled-format slot
// (dequantised as the reference does: fp16 code x scale; int8
// (code - 128) x scale / 127).
__device__ __forceinline__ float face_val(const Geo& G, const void* slot, int fl, int b, int c)
{
    const int ix = c % G.nx, r = c / G.nx, iy = r % G.ny, iz = r / G.ny;
    int f;
    const int i = face_index(G, iz, iy, ix, f);
    const StripStore& S = G.st;
    const char* base = static_cast<const char*>(slot);
    const long long row = (long long)fl * G.B + b;
    const float scale = reinterpret_cast<const float*>(base + pick6(S.scl, f))[row * pick6(S.blocks, f) + i / kQB];
    const long long q = row * pick6(S.cells, f) + i;
    const char* pay = base + pick6(S.pay, f);
    if (S.fmt == SF_F16) return __half2float(reinterpret_cast<const __half*>(pay)[q]) * scale;
    return ((float)reinterpret_cast<const uint8_t*>(pay)[q] - 128.0f) * (scale * (1.0f / 127.0f));
}

// Strip save (restore = 0) of fields [f0, f1) into / restore out of one step
// slot in format fmt: fp32 / bf16 slots hold the strip set (B, 9, ns); a
// scaled slot (written by quant3) is read from the field's faces.
__global__ void strips3(const Geo G, const Fields F, void* slot, int fmt, int f0, int f1, int restore)
{
    float* const* f = F.f;
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(e / G.ns), k = (int)(e - (long long)b * G.ns);
        const int c = G.cells[k];
        const long long i = b * G.S + c;
        for (int fl = f0; fl < f1; ++fl) {
            const long long t = ((long long)b * NFLD + fl) * G.ns + k;
            if (fmt == SF_F32) {
                float* p = static_cast<float*>(slot) + t;
                if (restore) f[fl][i] = *p;
                else *p = f[fl][i];
            } else if (fmt == SF_BF16) {
                __nv_bfloat16* p = static_cast<__nv_bfloat16*>(slot) + t;
                if (restore) f[fl][i] = __bfloat162float(*p);
                else *p = __float2bfloat16(f[fl][i]);
            } else if (restore) {
                f[fl][i] = face_val(G, slot, fl, b, c);
            }
        }
    }
}

// One step's nine fields into the scaled faces of a step slot: one CTA per
// (field, shot, face, block of kQB cells) -- the block's max |value| (its
// scale), then the codes (reference boundarysaver.cu:957-990, 1040-1075: int8
// round(v 127 / max) + 128 clamped to [0, 255]; fp16 v (1 / max)).
__global__ void __launch_bounds__(kQB) quant3(const Geo G, const Fields F, void* slot)
{
    const StripStore& S = G.st;
    int per = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) per += S.blocks[f];
    const int row = blockIdx.x / per;                 // field * B + shot
    const int fl = row / G.B, b = row - fl * G.B;
    int j = blockIdx.x - row * per, f = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k)
        if (f == k && j >= S.blocks[k]) { j -= S.blocks[k]; f = k + 1; }
    const int idx = j * kQB + threadIdx.x;
    const int cells = pick6(S.cells, f), blocks = pick6(S.blocks, f);
    const bool in = idx < cells;
    float v = 0.f;
    if (in) {
        int iz, iy, ix;
        face_cell(G, f, idx, iz, iy, ix);
        v = F.f[fl][b * G.S + ((long long)iz * G.ny + iy) * G.nx + ix];
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
    if (threadIdx.x == 0) reinterpret_cast<float*>(base + pick6(S.scl, f))[(long long)row * blocks + j] = m;
    if (!in) return;
    const long long q = (long long)row * cells + idx;
    char* pay = base + pick6(S.pay, f);
    if (S.fmt == SF_F16) {
        const float inv = m > 0.0f ? 1.0f / m : 0.0f;
        reinterpret_cast<__half*>(pay)[q] = __float2half(v * inv);
    } else {
        const float qs = m > 0.0f ? 127.0f / m : 0.0f;
        int c = __float2int_rn(v * qs) + 128;
        c = c < 0 ? 0 : (c > 255 ? 255 : c);
        reinterpret_cast<uint8_t*>(pay)[q] = (uint8_t)c;
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) srev3(Rev A)
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) vrev3(Rev A)
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) sprep3(Rev A)
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) sapp3(Rev A)
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

__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) vprep3(Rev A)
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) vapp3(Rev A)
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
__global__ void __launch_bounds__(NTHX * NTHY * NTHZ) cap3(Rev A)
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
    bool host_tape;              // boundary-saving tape in pinned host memory (SWEEP_MEM_HOST_TAPE)
    std::vector<int> cells;      // strip cells
};

static void check_mode(int mem_mode, int ckpt_every)
{
    if (mem_mode & SWEEP_MEM_HOST_TAPE) {
        mem_mode &= ~SWEEP_MEM_HOST_TAPE;
        SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT && mem_mode != SWEEP_MEM_RECURSIVE,
                      "elastic3d: a host tape goes with boundary saving only");
    }
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY || mem_mode == SWEEP_MEM_CHECKPOINT ||
                      mem_mode == SWEEP_MEM_BOUNDARY_FP16 || mem_mode == SWEEP_MEM_BOUNDARY_BF16 ||
                      mem_mode == SWEEP_MEM_BOUNDARY_INT8 || mem_mode == SWEEP_MEM_RECURSIVE,
                  "elastic3d: unknown memory mode %d", mem_mode);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT || ckpt_every >= 1,
                  "elastic3d: checkpoint interval must be >= 1 (got %d)", ckpt_every);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_RECURSIVE || ckpt_every >= 1,
                  "elastic3d: the recursive checkpoint budget must be >= 1 (got %d)", ckpt_every);
}

static Plan make_plan(const sweep_elastic3d_desc* d)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->M == M, "elastic3d: this build holds order %d (got order %d)", 2 * M, 2 * d->M);
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

// Strip storage of a memory mode: the step-slot layout of the boundary-saving
// tape (the checkpoint modes keep their chunk strips as fp32).
static void set_store(Plan& pl, int mem_mode)
{
    pl.host_tape = (mem_mode & SWEEP_MEM_HOST_TAPE) != 0;
    mem_mode &= ~SWEEP_MEM_HOST_TAPE;
    Geo& G = pl.G;
    StripStore& S = G.st;
    S = StripStore{};
    S.fmt = mem_mode == SWEEP_MEM_BOUNDARY_FP16 ? SF_F16
          : mem_mode == SWEEP_MEM_BOUNDARY_BF16 ? SF_BF16
          : mem_mode == SWEEP_MEM_BOUNDARY_INT8 ? SF_I8 : SF_F32;
    auto up = [](long long v, long long a) { return (v + a - 1) / a * a; };
    const long long per = (long long)G.B * NFLD * G.ns;
    if (S.fmt == SF_F32 || S.fmt == SF_BF16) {
        S.step = up(per * (S.fmt == SF_F32 ? 4 : 2), 256);
        return;
    }
    const long long bx = G.x1 - G.x0, by = G.y1 - G.y0, bz = G.z1 - G.z0;
    const long long cells[6] = {BW * by * bx, BW * by * bx, bz * BW * bx, bz * BW * bx, bz * by * BW, bz * by * BW};
    const int esz = S.fmt == SF_F16 ? 2 : 1;
    long long off = 0;
    for (int f = 0; f < 6; ++f) {
        SWEEP_REQUIRE(cells[f] * NFLD * G.B < (1LL << 31), "elastic3d: a strip face holds too many cells");
        S.cells[f] = (int)cells[f];
        S.blocks[f] = (int)((cells[f] + kQB - 1) / kQB);
        S.pay[f] = off;
        off = up(off + (long long)NFLD * G.B * cells[f] * esz, 16);
    }
    for (int f = 0; f < 6; ++f) {
        S.scl[f] = off;
        off = up(off + (long long)NFLD * G.B * S.blocks[f] * 4, 16);
    }
    S.step = up(off, 256);
}

static unsigned quant_blocks(const Geo& G)
{
    long long per = 0;
    for (int f = 0; f < 6; ++f) per += G.st.blocks[f];
    return (unsigned)(per * NFLD * G.B);
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

static long long slab_count(const Geo& G, int axis)
{
    return axis == 0 ? (long long)G.B * G.nz * G.ny * G.WX
         : axis == 1 ? (long long)G.B * G.nz * G.WY * G.nx : (long long)G.B * G.WZ * G.ny * G.nx;
}

static void carve_slabs(Carve& c, const Geo& G, Slabs& s)
{
    for (int k = 0; k < 6; ++k) s.x[k] = c.take<float>(slab_count(G, 0));
    for (int k = 0; k < 6; ++k) s.y[k] = c.take<float>(slab_count(G, 1));
    for (int k = 0; k < 6; ++k) s.z[k] = c.take<float>(slab_count(G, 2));
}

static float* slab_ptr(const Slabs& s, int k) { return k < 6 ? s.x[k] : k < 12 ? s.y[k - 6] : s.z[k - 12]; }

struct FwdWs {
    Common cm;
    float* f[NFLD];
    Slabs mem;
    char *zero0, *zero1;
    char* ring;                  // host tape: HostRing::R device strip slots
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
    if (pl.host_tape) w.ring = c.take<char>((long long)HostRing::R * pl.G.st.step);
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
    char* ring;                  // host tape: HostRing::R device strip slots
    Slabs fmem;                  // checkpoint modes: forward CPML memories of the replay
    float* chunk;                // checkpoint modes: fp32 strips of one chunk, (k + 1, B, 9, ns)
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
    if (pl.host_tape) w.ring = c.take<char>((long long)HostRing::R * G.st.step);
}

static long long chunk_floats(const Plan& pl) { return (long long)pl.G.B * NFLD * pl.G.ns; }

static void carve_rev_ckpt(Carve& c, const Plan& pl, int k, RevWs& w)
{
    carve_rev(c, pl, w);
    carve_slabs(c, pl.G, w.fmem);
    w.chunk = c.take<float>((long long)(k + 1) * chunk_floats(pl));
}

// Boundary-saving tape: one strip slot per step (G.st.step bytes), then the
// final nine-field state (9, B, nz, ny, nx).
static int64_t tape_bytes_of(const Plan& pl)
{
    return (int64_t)pl.G.nt * pl.G.st.step + (int64_t)NFLD * pl.G.B * pl.G.S * 4;
}

static void* tape_slot(const void* tape, const Plan& pl, int it)
{
    return const_cast<char*>(static_cast<const char*>(tape)) + (long long)it * pl.G.st.step;
}

static float* tape_last(const void* tape, const Plan& pl)
{
    return reinterpret_cast<float*>(static_cast<char*>(tape_slot(tape, pl, pl.G.nt)));
}

// Checkpointed boundary saving (SWEEP_MEM_CHECKPOINT, chunk length k): for
// every chunk c >= 1 the tape holds the state after step c k - 1 -- the nine
// fields and the 18 forward CPML memories -- and the fp32 strips of that step;
// the backward replays each chunk from its checkpoint into the strips of that
// chunk and runs the boundary-saving reverse steps over it (the reference's
// staggered driver replays chunks as well, sg_driver.cuh:911-925).  The
// recursive mode (SWEEP_MEM_RECURSIVE) keeps snapshots of the same layout.
static long long slab_floats(const Geo& G) { return 6 * (slab_count(G, 0) + slab_count(G, 1) + slab_count(G, 2)); }

static long long ckpt_stride(const Plan& pl)
{
    Carve c(nullptr);
    c.take<float>((long long)NFLD * pl.G.B * pl.G.S);
    c.take<float>(slab_floats(pl.G));
    c.take<float>(chunk_floats(pl));
    return (c.off + 255) & ~255LL;
}

static int nchunks(const Plan& pl, int k)
{
    SWEEP_REQUIRE(k >= 1, "elastic3d: checkpoint interval must be >= 1 (got %d)", k);
    return (pl.G.nt + k - 1) / k;
}

struct Ckpt {
    float* f[NFLD];
    float* mem;           // the 18 slabs, x then y then z, in carve_slabs order
    float* strips;
};

static Ckpt ckpt_at(void* tape, const Plan& pl, int ch)
{
    Carve c(static_cast<char*>(tape) + (long long)(ch - 1) * ckpt_stride(pl));
    Ckpt k{};
    for (int f = 0; f < NFLD; ++f) k.f[f] = c.take<float>((long long)pl.G.B * pl.G.S);
    k.mem = c.take<float>(slab_floats(pl.G));
    k.strips = c.take<float>(chunk_floats(pl));
    return k;
}

// Copy the 18 slabs between a Slabs set and a packed checkpoint range.
static void slabs_copy(const Slabs& s, float* packed, const Geo& G, bool to_packed, cudaStream_t st)
{
    long long o = 0;
    for (int k = 0; k < 18; ++k) {
        float* p = slab_ptr(s, k);
        const long long cnt = slab_count(G, k / 6);
        if (to_packed) SWEEP_CUDA(cudaMemcpyAsync(packed + o, p, cnt * 4, cudaMemcpyDeviceToDevice, st));
        else SWEEP_CUDA(cudaMemcpyAsync(p, packed + o, cnt * 4, cudaMemcpyDeviceToDevice, st));
        o += cnt;
    }
}

static void slabs_zero(const Slabs& s, const Geo& G, cudaStream_t st)
{
    for (int k = 0; k < 18; ++k) SWEEP_CUDA(cudaMemsetAsync(slab_ptr(s, k), 0, slab_count(G, k / 6) * 4, st));
}

void sizes(const sweep_elastic3d_desc* d, int mem_mode, int ckpt_every, int64_t* ws_bytes, int64_t* tape_bytes)
{
    check_mode(mem_mode, ckpt_every);
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    const int mode = mem_mode & ~SWEEP_MEM_HOST_TAPE;
    Carve f(nullptr), r(nullptr);
    FwdWs fw{};
    RevWs rw{};
    carve_fwd(f, pl, fw);
    if (mode == SWEEP_MEM_CHECKPOINT) {
        carve_rev_ckpt(r, pl, ckpt_every, rw);
        *tape_bytes = (int64_t)std::max(nchunks(pl, ckpt_every) - 1, 1) * ckpt_stride(pl);
    } else if (mode == SWEEP_MEM_RECURSIVE) {
        carve_rev_ckpt(r, pl, SWEEP_RECURSIVE_LEAF, rw);
        r.take<char>((long long)ckpt_every * ckpt_stride(pl));          // the snapshot slots
        *tape_bytes = 256;                                               // nothing is kept
    } else {
        carve_rev(r, pl, rw);
        *tape_bytes = tape_bytes_of(pl);
    }
    *ws_bytes = std::max(f.off, r.off);
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
    return dim3((G.nx + NTHX - 1) / NTHX, (G.ny + NTHY - 1) / NTHY, (unsigned)((G.nz + NTHZ - 1) / NTHZ * G.B));
}

static unsigned strip_blocks(const Geo& G)
{
    return (unsigned)std::max<long long>(std::min<long long>(((long long)G.B * G.ns + 255) / 256, 4096), 1);
}

// Forward steps [it0, it1) on the fields / memories of A; strips_of(it) is
// the slot (format fmt) that takes the strips of step it, or null.
template <class StripsOf>
static void forward_steps(const Fwd& A, int it0, int it1, StripsOf strips_of, int fmt, float* record, cudaStream_t st,
                          HostRing* hr = nullptr)
{
    const Geo& G = A.G;
    Fields F{};
    for (int k = 0; k < NFLD; ++k) F.f[k] = A.f[k];
    const dim3 grid = cell_grid(G), block(NTHX, NTHY, NTHZ);
    const bool scaled = fmt == SF_F16 || fmt == SF_I8;
    for (int it = it0; it < it1; ++it) {
        if (G.fst) {
            vel3<true><<<grid, block, 0, st>>>(A);
            str3<true><<<grid, block, 0, st>>>(A);
        } else {
            vel3<false><<<grid, block, 0, st>>>(A);
            str3<false><<<grid, block, 0, st>>>(A);
        }
        if (G.nsrc > 0) src3<<<G.B, 128, 0, st>>>(G, F, it, 1.f);
        if (void* slot = strips_of(it)) {
            if (hr) hr->before_write(it);
            if (scaled) quant3<<<quant_blocks(G), kQB, 0, st>>>(G, F, slot);
            else if (G.ns > 0) strips3<<<strip_blocks(G), 256, 0, st>>>(G, F, slot, fmt, 0, NFLD, 0);
            if (hr) hr->after_write(it);
        }
        if (record && G.nrec > 0) rec3<<<rec_grid(G), 128, 0, st>>>(G, F, record, it);
        SWEEP_LAUNCH_CHECK();
    }
}

void forward(const sweep_elastic3d_desc* d, int mem_mode, int ckpt_every, float* record, void* tape, void* ws,
             int64_t ws_bytes, cudaStream_t st)
{
    check_mode(mem_mode, ckpt_every);
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    const int mode = mem_mode & ~SWEEP_MEM_HOST_TAPE;
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
    const long long n = (long long)G.B * G.S;
    if (mode == SWEEP_MEM_RECURSIVE) tape = nullptr;     // the backward replays from the initial state
    if (mode != SWEEP_MEM_CHECKPOINT) {
        HostRing hr;
        const bool host = tape && pl.host_tape;
        if (host) hr.open(w.ring, tape, G.st.step, st);
        forward_steps(A, 0, G.nt,
                      [&](int it) -> void* { return !tape ? nullptr : host ? hr.slot(it) : tape_slot(tape, pl, it); },
                      G.st.fmt, record, st, host ? &hr : nullptr);
        if (host) hr.close();
        if (tape) {
            float* last = tape_last(tape, pl);
            for (int k = 0; k < NFLD; ++k)
                SWEEP_CUDA(cudaMemcpyAsync(last + k * n, w.f[k], sizeof(float) * n, cudaMemcpyDefault, st));
        }
        return;
    }
    const int k = ckpt_every, C = nchunks(pl, k);
    for (int ch = 0; ch < C; ++ch) {
        const int it0 = ch * k, it1 = std::min(G.nt, it0 + k);
        if (tape && ch >= 1) {
            const Ckpt cp = ckpt_at(tape, pl, ch);
            for (int f = 0; f < NFLD; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(cp.f[f], w.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
            slabs_copy(w.mem, cp.mem, G, true, st);
        }
        // the last step of a chunk keeps its strips with the next checkpoint
        forward_steps(A, it0, it1,
                      [&](int it) -> void* {
                          return (tape && it == it1 - 1 && ch + 1 < C) ? ckpt_at(tape, pl, ch + 1).strips : nullptr;
                      },
                      SF_F32, record, st);
    }
}

void backward(const sweep_elastic3d_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
              float* grad_vp, float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    check_mode(mem_mode, ckpt_every);
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    const int mode = mem_mode & ~SWEEP_MEM_HOST_TAPE;
    const bool ckpt = mode == SWEEP_MEM_CHECKPOINT, recursive = mode == SWEEP_MEM_RECURSIVE;
    SWEEP_REQUIRE(recursive || tape != nullptr, "elastic3d backward: the forward's tape is required");
    Carve c(ws);
    RevWs w{};
    char* snaps = nullptr;
    if (ckpt) carve_rev_ckpt(c, pl, ckpt_every, w);
    else if (recursive) {
        carve_rev_ckpt(c, pl, SWEEP_RECURSIVE_LEAF, w);
        snaps = c.take<char>((long long)ckpt_every * ckpt_stride(pl));
    } else carve_rev(c, pl, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic3d backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    Geo& G = pl.G;
    G.cells = w.cm.cells;
    setup_common(d, pl, w.cm, st);
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
    const long long n = (long long)G.B * G.S;
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
    const dim3 grid = cell_grid(G), block(NTHX, NTHY, NTHZ);
    bool vsrc = false;
    for (int k = 0; k < G.nsf; ++k) vsrc |= G.sf[k] <= VZ;
    HostRing hr;
    const bool host = pl.host_tape && !ckpt && !recursive;
    // Reverse steps it1 - 1 .. max(it0, 1) (the staggered reverse has no
    // it = 0 step) on the reconstruction state after step it1 - 1;
    // strips_of(t) holds the strips (format fmt) of the state after step t.
    auto reverse = [&](int it0, int it1, auto strips_of, int fmt) {
        for (int it = it1 - 1; it >= std::max(it0, 1); --it) {
            A.it = it;
            void* prev = strips_of(it - 1);
            if (host) hr.before_read(it - 1);
            if (vsrc && G.nsrc > 0) vsrc3<<<G.B, 128, 0, st>>>(A);
            if (G.nrec > 0) res3<<<rec_grid(G), 128, 0, st>>>(A);
            if (G.nsrc > 0) src3<<<G.B, 128, 0, st>>>(G, F, it, -1.f);
            if (G.fst) srev3<true><<<grid, block, 0, st>>>(A);
            else srev3<false><<<grid, block, 0, st>>>(A);
            if (G.ns > 0) strips3<<<strip_blocks(G), 256, 0, st>>>(G, F, prev, fmt, SXX, NFLD, 1);
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
            if (G.ns > 0) strips3<<<strip_blocks(G), 256, 0, st>>>(G, F, prev, fmt, VX, SXX, 1);
            if (host) {
                hr.after_read(it - 1);
                if (it - 1 - HostRing::R >= std::max(it0 - 1, 0)) hr.fetch(it - 1 - HostRing::R, true);
            }
            SWEEP_LAUNCH_CHECK();
        }
    };
    // the replay of the checkpoint modes runs straight into the reconstruction
    // fields, with its own forward CPML memories
    Fwd R{};
    R.G = G;
    R.m = A.m;
    for (int k = 0; k < NFLD; ++k) R.f[k] = w.f[k];
    R.mem = w.fmem;
    const long long cs = chunk_floats(pl);
    auto chunk_slot = [&](int j) -> void* { return w.chunk + (long long)j * cs; };
    if (recursive) {
        // Recursive checkpointing: the bisection of the acoustic drivers; a
        // snapshot slot has the checkpoint layout (nine fields, 18 CPML slabs,
        // strips of the step before), leaves are SWEEP_RECURSIVE_LEAF steps.
        const int L = SWEEP_RECURSIVE_LEAF, count = ckpt_every;
        auto restore = [&](int k) {
            if (k < 0) {
                for (int f = 0; f < NFLD; ++f) SWEEP_CUDA(cudaMemsetAsync(w.f[f], 0, sizeof(float) * n, st));
                slabs_zero(w.fmem, G, st);
            } else {
                const Ckpt cp = ckpt_at(snaps, pl, k + 1);
                for (int f = 0; f < NFLD; ++f)
                    SWEEP_CUDA(cudaMemcpyAsync(w.f[f], cp.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
                slabs_copy(w.fmem, cp.mem, G, false, st);
            }
        };
        auto save = [&](int k) {
            const Ckpt cp = ckpt_at(snaps, pl, k + 1);
            for (int f = 0; f < NFLD; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(cp.f[f], w.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
            slabs_copy(w.fmem, cp.mem, G, true, st);
        };
        auto strips_from = [&](int k) {        // strips of the step before snapshot k into chunk slot 0
            SWEEP_CUDA(cudaMemcpyAsync(w.chunk, ckpt_at(snaps, pl, k + 1).strips, sizeof(float) * cs,
                                       cudaMemcpyDeviceToDevice, st));
        };
        auto leaf = [&](int a, int e) {
            forward_steps(R, a, e, [&](int it) { return chunk_slot(it - a + 1); }, SF_F32, nullptr, st);
            reverse(a, e, [&](int t) { return chunk_slot(t - (a - 1)); }, SF_F32);
        };
        std::function<void(int, int, int, int)> process = [&](int a, int b, int ka, int free) {
            const int nleaf = (b - a + L - 1) / L;
            if (nleaf <= 1) {
                restore(ka);
                if (a > 0) strips_from(ka);
                leaf(a, b);
                return;
            }
            if (free > 0) {
                const int k = count - free, m = a + L * ((nleaf + 1) / 2);
                restore(ka);
                float* ks = ckpt_at(snaps, pl, k + 1).strips;
                forward_steps(R, a, m, [&](int it) -> void* { return it == m - 1 ? ks : nullptr; }, SF_F32, nullptr,
                              st);
                save(k);
                process(m, b, k, free - 1);
                process(a, m, ka, free);
                return;
            }
            for (int c0 = a + (nleaf - 1) * L; c0 >= a; c0 -= L) {
                restore(ka);
                if (c0 > a)
                    forward_steps(R, a, c0, [&](int it) -> void* { return it == c0 - 1 ? w.chunk : nullptr; },
                                  SF_F32, nullptr, st);
                else if (a > 0)
                    strips_from(ka);
                leaf(c0, std::min(b, c0 + L));
            }
        };
        process(0, G.nt, -1, count);
    } else if (!ckpt) {
        const float* last = tape_last(tape, pl);
        for (int k = 0; k < NFLD; ++k)
            SWEEP_CUDA(cudaMemcpyAsync(w.f[k], last + k * n, sizeof(float) * n, cudaMemcpyDefault, st));
        if (host) {
            hr.open(w.ring, const_cast<void*>(tape), G.st.step, st);
            for (int t = G.nt - 2; t >= 0 && t > G.nt - 2 - HostRing::R; --t) hr.fetch(t, false);
            reverse(0, G.nt, [&](int t) { return hr.slot(t); }, G.st.fmt);
            hr.close();
        } else {
            reverse(0, G.nt, [&](int t) { return tape_slot(tape, pl, t); }, G.st.fmt);
        }
    } else {
        const int k = ckpt_every, C = nchunks(pl, k);
        void* tp = const_cast<void*>(tape);
        for (int ch = C - 1; ch >= 0; --ch) {
            const int it0 = ch * k, it1 = std::min(G.nt, it0 + k);
            if (ch == 0) {
                for (int f = 0; f < NFLD; ++f) SWEEP_CUDA(cudaMemsetAsync(w.f[f], 0, sizeof(float) * n, st));
                slabs_zero(w.fmem, G, st);
            } else {
                const Ckpt cp = ckpt_at(tp, pl, ch);
                for (int f = 0; f < NFLD; ++f)
                    SWEEP_CUDA(cudaMemcpyAsync(w.f[f], cp.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
                slabs_copy(w.fmem, cp.mem, G, false, st);
                SWEEP_CUDA(cudaMemcpyAsync(w.chunk, cp.strips, sizeof(float) * cs, cudaMemcpyDeviceToDevice, st));
            }
            // replay: chunk slot j holds the strips after step it0 - 1 + j
            forward_steps(R, it0, it1, [&](int it) { return chunk_slot(it - it0 + 1); }, SF_F32, nullptr, st);
            reverse(it0, it1, [&](int t) { return chunk_slot(t - (it0 - 1)); }, SF_F32);
        }
    }
    const int per_shot = d->model_stride != 0;
    finalize3<<<592, 256, 0, st>>>(w.gvp, G.B, per_shot, G, grad_vp);
    finalize3<<<592, 256, 0, st>>>(w.gvs, G.B, per_shot, G, grad_vs);
    finalize3<<<592, 256, 0, st>>>(w.grho, G.B, per_shot, G, grad_rho);
    SWEEP_LAUNCH_CHECK();
}

}  // namespace EL3D_NS
}  // namespace sweep
