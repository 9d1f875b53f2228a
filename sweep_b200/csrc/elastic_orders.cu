// elastic_orders.cu -- the 2-D isotropic elastic forward and boundary-saving
// adjoint at every spatial order but 8 (M = 1..7: orders 2, 4, 6, 10, 12,
// 14), for sm_100a.  Order 8 runs the tiled kernels of elastic2d.cu; the
// reference's Elastic defaults to order 4, so a drop-in caller lands here
// unless it asks for order 8.
//
// Restates the reference's templated elastic2d path (src/sweep/csrc/cuda/
// equations/elastic2d/kernels.cuh, common/sg_driver.cuh step order,
// common/elastic_free_surface.cuh for traction-free faces), order by order,
// with the staggered weights of that order (operators/staggered.cuh):
//   forward, per step: velocity step (four stress derivatives, CPML memories
//     outside the physical box), stress step (Robertsson corrections and
//     zeroing on free faces), source injection per source field, the five
//     fields' boundary bands (width M + 1 from M cells outside the box),
//     receivers;
//   reverse, per step it = nt - 1 .. 1: body-force rho correction, signed
//     residuals (stress -1, velocity +1), source removal, stress
//     reconstruction on the box minus one cell, stress bands restored,
//     stress-adjoint prepare with the fused vp / vs / rho imaging, receiver
//     rho correction, stress-adjoint apply, velocity-adjoint prepare and
//     apply, v(it) carriers, velocity reconstruction, velocity bands restored.
// One thread per cell on 32 x 8 tiles, shots on the grid's last axis,
// stencils through the read-only path.  Memory: boundary saving with fp32
// bands in device memory (SWEEP_MEM_BOUNDARY).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "elastic_orders.cuh"

namespace sweep {
namespace eord {

constexpr int MAXM = 7;
enum { VX = 0, VZ = 1, SXX = 2, SZZ = 3, SXZ = 4 };
// CPML memories: the field differenced and the axis
enum { M_VXX, M_VZZ, M_VXZ, M_VZX, M_SXXX, M_SZZZ, M_SXZX, M_SXZZ, NMEM };

struct Geo {
    int B, nz, nx, nt, M;
    long long S;                    // cells per shot
    int pad[4];                     // z_lo, z_hi, x_lo, x_hi
    int fs;                         // bit f: traction-free face f (pad 0)
    int z0, z1, x0, x1;             // physical box
    float dt, dz, dx;
    float c[MAXM + 1];              // staggered weights c[1..M]
    const float *az, *bz, *azh, *bzh, *ax, *bx, *axh, *bxh;
    const float *vp, *vs, *rho;     // the caller's models
    const float *lam, *mu, *kv;     // derived, kv = dt (1 / rho)
    long long ms;                   // model stride between shots (0 or S)
    int nsrc, nrec, nsf, nrf;
    int sf[5], rf[5];
    const int *src, *rec;           // (B, n, 2) runtime (x, z)
    const float* wavelet;           // (B, nsrc, nt)
    const int* cells;               // band cells of a shot grid (cells of two bands listed twice)
    int ns;
};

struct Fields {
    float* f[5];
};
struct Mems {
    float* m[NMEM];
};

__device__ __forceinline__ float ld(const float* p) { return __ldg(p); }

// D+ / D- along stride s: sum_k c_k (u[i + k s] - u[i - (k - 1) s]) (1 / h)
// and sum_k c_k (u[i + (k - 1) s] - u[i - k s]) (1 / h)
template <int M>
__device__ __forceinline__ float dplus(const float* __restrict__ u, long long i, long long s, const Geo& G, float inv)
{
    float g = G.c[1] * (ld(u + i + s) - ld(u + i));
#pragma unroll
    for (int k = 2; k <= M; ++k) g = g + G.c[k] * (ld(u + i + k * s) - ld(u + i - (k - 1) * s));
    return g * inv;
}
template <int M>
__device__ __forceinline__ float dminus(const float* __restrict__ u, long long i, long long s, const Geo& G, float inv)
{
    float g = G.c[1] * (ld(u + i) - ld(u + i - s));
#pragma unroll
    for (int k = 2; k <= M; ++k) g = g + G.c[k] * (ld(u + i + (k - 1) * s) - ld(u + i - k * s));
    return g * inv;
}

// ---------------------------------------------- traction-free faces
// Per axis (0 = z, 1 = x) the low surface is the first physical row / column
// and the high surface the last; cells past them are air, read by a
// derivative along the axis as the image of the cell mirrored about the
// surface (about the node for integer fields, the half cell next to it for
// half fields), negated for odd fields; the M cells from a surface inwards
// take a unit-weight 2nd-order difference (elastic_free_surface.cuh:200-720).
struct FsAx {
    int lo_on, hi_on, lo, hi, n;
    long long s;
    float h;
};

__device__ __forceinline__ FsAx fs_axis(const Geo& G, int a)
{
    FsAx x;
    if (a == 0) {
        x.lo_on = G.fs & 1; x.hi_on = (G.fs >> 1) & 1;
        x.lo = G.pad[0] + G.M; x.hi = G.nz - G.pad[1] - G.M - 1;
        x.n = G.nz; x.s = G.nx; x.h = G.dz;
    } else {
        x.lo_on = (G.fs >> 2) & 1; x.hi_on = (G.fs >> 3) & 1;
        x.lo = G.pad[2] + G.M; x.hi = G.nx - G.pad[3] - G.M - 1;
        x.n = G.nx; x.s = 1; x.h = G.dx;
    }
    return x;
}

__device__ __forceinline__ float fs_at(const FsAx& x, const float* u, long long base, int j, bool odd, bool half)
{
    int m;
    if (x.lo_on && j < x.lo) m = half ? 2 * x.lo - 1 - j : 2 * x.lo - j;
    else if (x.hi_on && j >= (half ? x.hi : x.hi + 1)) m = half ? 2 * x.hi - 1 - j : 2 * x.hi - j;
    else return ld(u + base + (long long)j * x.s);
    const float v = ld(u + base + (long long)m * x.s);
    return odd ? -v : v;
}

template <int M>
__device__ __forceinline__ bool fs_band(const FsAx& x, int j)
{
    return (x.lo_on && j >= x.lo && j < x.lo + M) || (x.hi_on && j > x.hi - M && j <= x.hi);
}

// derivative along axis a at (ix, iz): fwd the D+ form, else the D- form
template <int M>
__device__ float dd(const Geo& G, const float* __restrict__ u, int a, int ix, int iz, bool fwd, bool odd, bool half)
{
    const FsAx x = fs_axis(G, a);
    const long long i = (long long)iz * G.nx + ix;
    if (!x.lo_on && !x.hi_on) return fwd ? dplus<M>(u, i, x.s, G, 1.f / x.h) : dminus<M>(u, i, x.s, G, 1.f / x.h);
    const int j = a == 0 ? iz : ix;
    const long long base = i - (long long)j * x.s;
    if (fs_band<M>(x, j)) {
        const float g = fwd ? fs_at(x, u, base, j + 1, odd, half) - fs_at(x, u, base, j, odd, half)
                            : fs_at(x, u, base, j, odd, half) - fs_at(x, u, base, j - 1, odd, half);
        return g / x.h;
    }
    float g = 0.f;
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        const float up = fwd ? fs_at(x, u, base, j + k, odd, half) : fs_at(x, u, base, j + k - 1, odd, half);
        const float um = fwd ? fs_at(x, u, base, j - k + 1, odd, half) : fs_at(x, u, base, j - k, odd, half);
        g = g + G.c[k] * (up - um);
    }
    return g / x.h;
}

// transpose of dd without the images at input index m: an output cell in a
// band contributes with weight 1, one outside with the full weight
template <int M>
__device__ float adj_plain(const FsAx& x, const Geo& G, const float* q, long long base, int m, bool fwd)
{
    float acc = 0.f;
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        const int jp = fwd ? m + k - 1 : m + k;
        const int jm = fwd ? m - k : m - k + 1;
        if (jp >= 0 && jp < x.n && !fs_band<M>(x, jp)) acc = acc + G.c[k] * ld(q + base + (long long)jp * x.s);
        if (jm >= 0 && jm < x.n && !fs_band<M>(x, jm)) acc = acc - G.c[k] * ld(q + base + (long long)jm * x.s);
    }
    if (fwd) {
        if (fs_band<M>(x, m)) acc = acc + ld(q + base + (long long)m * x.s);
        if (fs_band<M>(x, m - 1)) acc = acc - ld(q + base + (long long)(m - 1) * x.s);
    } else {
        if (fs_band<M>(x, m + 1)) acc = acc + ld(q + base + (long long)(m + 1) * x.s);
        if (fs_band<M>(x, m)) acc = acc - ld(q + base + (long long)m * x.s);
    }
    return acc / x.h;
}

// adjoint of dd (the plain one: D- for a D+ forward and vice versa): zero on
// air cells; else the plain transpose plus each free face's image of this
// cell in the air folded back with the field's parity
template <int M>
__device__ float da(const Geo& G, const float* __restrict__ q, int a, int ix, int iz, bool fwd, bool odd, bool half)
{
    const FsAx x = fs_axis(G, a);
    const long long i = (long long)iz * G.nx + ix;
    if (!x.lo_on && !x.hi_on) return fwd ? dminus<M>(q, i, x.s, G, 1.f / x.h) : dplus<M>(q, i, x.s, G, 1.f / x.h);
    const int j = a == 0 ? iz : ix;
    const long long base = i - (long long)j * x.s;
    if ((x.lo_on && j < x.lo) || (x.hi_on && j > x.hi)) return 0.f;
    const float parity = odd ? -1.f : 1.f;
    float g = adj_plain<M>(x, G, q, base, j, fwd);
    if (x.lo_on) {
        const int mj = half ? 2 * x.lo - 1 - j : 2 * x.lo - j;
        if (mj < x.lo) g = g + parity * adj_plain<M>(x, G, q, base, mj, fwd);
    }
    if (x.hi_on) {
        const int mj = half ? 2 * x.hi - 1 - j : 2 * x.hi - j;
        if (mj >= (half ? x.hi : x.hi + 1)) g = g + parity * adj_plain<M>(x, G, q, base, mj, fwd);
    }
    return g;
}

__device__ __forceinline__ bool fs_zrow(const Geo& G, int iz)
{
    return ((G.fs & 1) && iz == G.pad[0] + G.M) || ((G.fs & 2) && iz == G.nz - G.pad[1] - G.M - 1);
}
__device__ __forceinline__ bool fs_xcol(const Geo& G, int ix)
{
    return ((G.fs & 4) && ix == G.pad[2] + G.M) || ((G.fs & 8) && ix == G.nx - G.pad[3] - G.M - 1);
}
__device__ __forceinline__ bool fs_zero_shear(const Geo& G, int ix, int iz)
{
    return ((G.fs & 2) && iz == G.nz - G.pad[1] - G.M - 1) || ((G.fs & 8) && ix == G.nx - G.pad[3] - G.M - 1);
}
// CPML test of the velocity step and the adjoint prepares: PML pad plus halo
__device__ __forceinline__ bool in_pml(const Geo& G, int ix, int iz)
{
    return ix < G.pad[2] + G.M || ix >= G.nx - G.pad[3] - G.M || iz < G.pad[0] + G.M || iz >= G.nz - G.pad[1] - G.M;
}
// the stress step's: a free surface row / column stays in the CPML branch
__device__ __forceinline__ bool in_pml_stress(const Geo& G, int ix, int iz)
{
    const int M = G.M;
    const int zlo = (G.fs & 1) ? G.pad[0] + M + 1 : G.pad[0] + M;
    const int zhi = (G.fs & 2) ? G.nz - G.pad[1] - M - 1 : G.nz - G.pad[1] - M;
    const int xlo = (G.fs & 4) ? G.pad[2] + M + 1 : G.pad[2] + M;
    const int xhi = (G.fs & 8) ? G.nx - G.pad[3] - M - 1 : G.nx - G.pad[3] - M;
    return ix < xlo || ix >= xhi || iz < zlo || iz >= zhi;
}

// ----------------------------------------------------------------- kernels
__device__ __forceinline__ bool cell2(const Geo& G, int& b, int& iz, int& ix)
{
    ix = blockIdx.x * 32 + threadIdx.x;
    iz = blockIdx.y * 8 + threadIdx.y;
    b = blockIdx.z;
    return ix < G.nx && iz < G.nz;
}
__device__ __forceinline__ bool core(const Geo& G, int ix, int iz)
{
    return ix >= G.M && ix < G.nx - G.M && iz >= G.M && iz < G.nz - G.M;
}

// Lame parameters and dt / rho per model copy (reference
// derived_models.cu:27-37 rounding)
__global__ void prep(const float* __restrict__ vp, const float* __restrict__ vs, const float* __restrict__ rho,
                     long long n, float dt, float* lam, float* mu, float* kv)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const float v = vp[k], s = vs[k], r = rho[k];
        mu[k] = (r * s) * s;
        lam[k] = r * ((v * v) - ((2.f * s) * s));
        kv[k] = dt * (1.f / r);
    }
}

__device__ __forceinline__ void cpml(float* m, long long i, float a, float b, float& d)
{
    const float v = a * m[i] + b * d;
    m[i] = v;
    d = d + v;
}

// velocity step (reference elastic2d/kernels.cuh:48-138)
template <int M>
__global__ void __launch_bounds__(256) vel(const Geo G, Fields F, Mems W)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    float dsxx_dx = dd<M>(G, F.f[SXX] + o, 1, ix, iz, true, true, false);
    float dsxz_dz = dd<M>(G, F.f[SXZ] + o, 0, ix, iz, false, true, true);
    float dsxz_dx = dd<M>(G, F.f[SXZ] + o, 1, ix, iz, false, true, true);
    float dszz_dz = dd<M>(G, F.f[SZZ] + o, 0, ix, iz, true, true, false);
    if (in_pml(G, ix, iz)) {
        cpml(W.m[M_SZZZ] + o, i, G.azh[iz], G.bzh[iz], dszz_dz);
        cpml(W.m[M_SXZX] + o, i, G.ax[ix], G.bx[ix], dsxz_dx);
        cpml(W.m[M_SXZZ] + o, i, G.az[iz], G.bz[iz], dsxz_dz);
        cpml(W.m[M_SXXX] + o, i, G.axh[ix], G.bxh[ix], dsxx_dx);
    }
    const float k = G.kv[b * G.ms + i];
    F.f[VX][o + i] = F.f[VX][o + i] + k * (dsxx_dx + dsxz_dz);
    F.f[VZ][o + i] = F.f[VZ][o + i] + k * (dsxz_dx + dszz_dz);
}

// stress step with the free faces' Robertsson corrections, then the zeroing
// (reference elastic2d/kernels.cuh:182-311)
template <int M>
__global__ void __launch_bounds__(256) str(const Geo G, Fields F, Mems W)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    float dvx_dx = dd<M>(G, F.f[VX] + o, 1, ix, iz, false, true, true);
    float dvz_dz = dd<M>(G, F.f[VZ] + o, 0, ix, iz, false, true, true);
    float dvx_dz = dd<M>(G, F.f[VX] + o, 0, ix, iz, true, false, false);
    float dvz_dx = dd<M>(G, F.f[VZ] + o, 1, ix, iz, true, false, false);
    const long long mi = b * G.ms + i;
    const float lam = G.lam[mi], mu = G.mu[mi];
    const bool pml = in_pml_stress(G, ix, iz);
    if (pml) {
        cpml(W.m[M_VZZ] + o, i, G.az[iz], G.bz[iz], dvz_dz);
        cpml(W.m[M_VXX] + o, i, G.ax[ix], G.bx[ix], dvx_dx);
    }
    float* sxx = F.f[SXX] + o;
    float* szz = F.f[SZZ] + o;
    sxx[i] = sxx[i] + G.dt * ((lam + 2.f * mu) * dvx_dx + lam * dvz_dz);
    szz[i] = szz[i] + G.dt * ((lam + 2.f * mu) * dvz_dz + lam * dvx_dx);
    if (pml) {
        cpml(W.m[M_VXZ] + o, i, G.azh[iz], G.bzh[iz], dvx_dz);
        cpml(W.m[M_VZX] + o, i, G.axh[ix], G.bxh[ix], dvz_dx);
    }
    F.f[SXZ][o + i] = F.f[SXZ][o + i] + (G.dt * mu) * (dvx_dz + dvz_dx);
    if (G.fs) {
        const bool zs = fs_zrow(G, iz), xs = fs_xcol(G, ix);
        if (zs) sxx[i] = sxx[i] + (-G.dt) * lam * ((lam / (lam + 2.f * mu)) * dvx_dx + dvz_dz);
        if (xs) szz[i] = szz[i] + (-G.dt) * lam * ((lam / (lam + 2.f * mu)) * dvz_dz + dvx_dx);
        if (zs) szz[i] = 0.f;
        if (xs) sxx[i] = 0.f;
        if (fs_zero_shear(G, ix, iz)) F.f[SXZ][o + i] = 0.f;
    }
}

// grid offset of location (x, z), or -1 off the grid
__device__ __forceinline__ long long loc(const Geo& G, const int* l)
{
    if (l[0] < 0 || l[0] >= G.nx || l[1] < 0 || l[1] >= G.nz) return -1;
    return (long long)l[1] * G.nx + l[0];
}

// the wavelet of step it, times sign, into every source field
__global__ void inject(const Geo G, Fields F, int it, float sign)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nsrc) return;
    const int b = e / G.nsrc;
    const long long c = loc(G, G.src + 2LL * e);
    if (c < 0) return;
    const float w = sign * G.wavelet[(long long)e * G.nt + it];
    for (int k = 0; k < G.nsf; ++k) atomicAdd(F.f[G.sf[k]] + b * G.S + c, w);
}

// record[b, it, r, k] = field rf[k] at receiver r
__global__ void gather(const Geo G, Fields F, float* record, int it)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const long long c = loc(G, G.rec + 2LL * e);
    if (c < 0) return;
    float* out = record + (((long long)b * G.nt + it) * G.nrec + r) * G.nrf;
    for (int k = 0; k < G.nrf; ++k) out[k] = F.f[G.rf[k]][b * G.S + c];
}

// band save (restore = 0) of fields [f0, f1) into one step slot (B, 5, ns), or restore
__global__ void bands(const Geo G, Fields F, float* slot, int f0, int f1, int restore)
{
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long b = e / G.ns, k = e - b * G.ns;
        const long long i = b * G.S + G.cells[k];
        for (int f = f0; f < f1; ++f) {
            float* t = slot + (b * 5 + f) * G.ns + k;
            if (restore) F.f[f][i] = *t;
            else *t = F.f[f][i];
        }
    }
}

// ---------------------------------------------------------------- reverse
struct Rev {
    float* f[5];                    // reconstructed forward fields
    float* a[5];                    // adjoint fields
    float* am[NMEM];                // adjoint CPML memories
    float* q[4];                    // prepare -> apply scratch (q, then p)
    float *vxn, *vzn;               // v(it + 1) carriers on the box
    float *gvp, *gvs, *grho;        // per-shot gradient slots (B, S)
    const float* adj;               // (B, nt, nrec, nrf)
    int it;
};

// body-force rho correction at velocity sources, before the residuals
__global__ void vsrc_rho(const Geo G, Rev R)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nsrc) return;
    const int b = e / G.nsrc;
    const long long c = loc(G, G.src + 2LL * e);
    if (c < 0) return;
    const float w = G.wavelet[(long long)e * G.nt + R.it];
    for (int k = 0; k < G.nsf; ++k) {
        if (G.sf[k] > VZ) continue;
        atomicAdd(R.grho + b * G.S + c, (R.a[G.sf[k]][b * G.S + c] * w) / G.rho[b * G.ms + c]);
    }
}

// signed residuals into the adjoint fields (stress -1, velocity +1)
__global__ void residual(const Geo G, Rev R)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const long long c = loc(G, G.rec + 2LL * e);
    if (c < 0) return;
    const float* res = R.adj + (((long long)b * G.nt + R.it) * G.nrec + r) * G.nrf;
    for (int k = 0; k < G.nrf; ++k) {
        const int f = G.rf[k];
        atomicAdd(R.a[f] + b * G.S + c, f >= SXX ? -res[k] : res[k]);
    }
}

// receiver rho correction (velocity receivers in the core), after the image
__global__ void rec_rho(const Geo G, Rev R)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const int* l = G.rec + 2LL * e;
    if (!core(G, l[0], l[1])) return;
    const long long c = (long long)l[1] * G.nx + l[0];
    const float* res = R.adj + (((long long)b * G.nt + R.it) * G.nrec + r) * G.nrf;
    for (int k = 0; k < G.nrf; ++k) {
        const int f = G.rf[k];
        if (f > VZ) continue;
        const float now = R.f[f][b * G.S + c], nxt = (f == VX ? R.vxn : R.vzn)[b * G.S + c];
        atomicAdd(R.grho + b * G.S + c, ((-res[k]) * (now - nxt)) / G.rho[b * G.ms + c]);
    }
}

// the reverse box: the physical box minus one cell per face; a free face
// reaches the halo M (reference kernels.cuh:405-535)
__device__ __forceinline__ bool in_rev(const Geo& G, int ix, int iz)
{
    const int M = G.M;
    const int zlo = (G.fs & 1) ? M : G.pad[0] + M + 1, zhi = G.nz - ((G.fs & 2) ? M : G.pad[1] + M + 1);
    const int xlo = (G.fs & 4) ? M : G.pad[2] + M + 1, xhi = G.nx - ((G.fs & 8) ? M : G.pad[3] + M + 1);
    return ix >= xlo && ix < xhi && iz >= zlo && iz < zhi;
}

template <int M>
__global__ void __launch_bounds__(256) srev(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !in_rev(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const float dvx_dx = dd<M>(G, R.f[VX] + o, 1, ix, iz, false, true, true);
    const float dvz_dz = dd<M>(G, R.f[VZ] + o, 0, ix, iz, false, true, true);
    const float dvx_dz = dd<M>(G, R.f[VX] + o, 0, ix, iz, true, false, false);
    const float dvz_dx = dd<M>(G, R.f[VZ] + o, 1, ix, iz, true, false, false);
    const long long mi = b * G.ms + i;
    const float lam = G.lam[mi], mu = G.mu[mi];
    R.f[SXX][o + i] = R.f[SXX][o + i] - G.dt * ((lam + 2.f * mu) * dvx_dx + lam * dvz_dz);
    R.f[SZZ][o + i] = R.f[SZZ][o + i] - G.dt * ((lam + 2.f * mu) * dvz_dz + lam * dvx_dx);
    R.f[SXZ][o + i] = R.f[SXZ][o + i] - (G.dt * mu) * (dvx_dz + dvz_dx);
}

template <int M>
__global__ void __launch_bounds__(256) vrev(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !in_rev(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const float dsxx_dx = dd<M>(G, R.f[SXX] + o, 1, ix, iz, true, true, false);
    const float dsxz_dz = dd<M>(G, R.f[SXZ] + o, 0, ix, iz, false, true, true);
    const float dsxz_dx = dd<M>(G, R.f[SXZ] + o, 1, ix, iz, false, true, true);
    const float dszz_dz = dd<M>(G, R.f[SZZ] + o, 0, ix, iz, true, true, false);
    const float k = G.kv[b * G.ms + i];
    R.f[VX][o + i] = R.f[VX][o + i] - k * (dsxx_dx + dsxz_dz);
    R.f[VZ][o + i] = R.f[VZ][o + i] - k * (dsxz_dx + dszz_dz);
}

// stress-adjoint prepare over every cell with the fused imaging inside the
// physical box (reference kernels.cuh:548-750)
template <int M>
__global__ void __launch_bounds__(256) sprep(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, k = o + i, mi = b * G.ms + i;
    const float lam = G.lam[mi], mu = G.mu[mi], dt = G.dt;
    float bsxx = R.a[SXX][k], bszz = R.a[SZZ][k], bsxz = R.a[SXZ][k];
    const bool zs = G.fs && fs_zrow(G, iz), xs = G.fs && fs_xcol(G, ix);
    if (zs) { bszz = 0.f; R.a[SZZ][k] = 0.f; }
    if (xs) { bsxx = 0.f; R.a[SXX][k] = 0.f; }
    if (G.fs && fs_zero_shear(G, ix, iz)) { bsxz = 0.f; R.a[SXZ][k] = 0.f; }
    if (ix >= G.x0 && ix < G.x1 && iz >= G.z0 && iz < G.z1) {
        const float fvx_x = dd<M>(G, R.f[VX] + o, 1, ix, iz, false, true, true);
        const float fvz_z = dd<M>(G, R.f[VZ] + o, 0, ix, iz, false, true, true);
        const float fvx_z = dd<M>(G, R.f[VX] + o, 0, ix, iz, true, false, false);
        const float fvz_x = dd<M>(G, R.f[VZ] + o, 1, ix, iz, true, false, false);
        const float vp = G.vp[mi], vs = G.vs[mi], rho = G.rho[mi];
        float gl, gm;
        if (zs && xs) {
            gl = 0.f; gm = 0.f;
        } else if (zs || xs) {
            const float vp2 = vp * vp, vs2 = vs * vs, vp4 = vp2 * vp2;
            const float a = zs ? bsxx * fvx_x : bszz * fvz_z;
            gl = a * 4.f * vs2 * vs2 / vp4;
            gm = a * 4.f * (vp4 - 2.f * vp2 * vs2 + 2.f * vs2 * vs2) / vp4;
        } else {
            gl = (bsxx + bszz) * (fvx_x + fvz_z);
            gm = 2.f * (bsxx * fvx_x + bszz * fvz_z);
        }
        gm = gm + bsxz * (fvx_z + fvz_x);
        R.gvp[k] = R.gvp[k] + ((-2.f * rho) * vp) * gl * dt;
        R.gvs[k] = R.gvs[k] + (-((((-4.f * rho) * vs) * gl) + (((2.f * rho) * vs) * gm))) * dt;
        const float gr = R.grho[k] + (R.a[VX][k] * (R.f[VX][k] - R.vxn[k]) + R.a[VZ][k] * (R.f[VZ][k] - R.vzn[k])) / rho;
        R.grho[k] = gr - ((gl * ((vp * vp) - ((2.f * vs) * vs))) * dt + (gm * (vs * vs)) * dt);
    }
    float bvx_x, bvz_z;
    if (zs && xs) {
        bvx_x = 0.f; bvz_z = 0.f;
    } else if (zs) {
        const float c_surf = 4.f * mu * (lam + mu) / (lam + 2.f * mu);
        bvx_x = dt * c_surf * bsxx;
        bvz_z = 0.f;
    } else if (xs) {
        const float c_surf = 4.f * mu * (lam + mu) / (lam + 2.f * mu);
        bvz_z = dt * c_surf * bszz;
        bvx_x = 0.f;
    } else {
        bvx_x = dt * ((lam + 2.f * mu) * bsxx + lam * bszz);
        bvz_z = dt * ((lam + 2.f * mu) * bszz + lam * bsxx);
    }
    const float bvx_z = (dt * mu) * bsxz, bvz_x = (dt * mu) * bsxz;
    if (!in_pml(G, ix, iz)) {
        R.q[0][k] = bvx_x; R.q[1][k] = bvz_z; R.q[2][k] = bvx_z; R.q[3][k] = bvz_x;
        return;
    }
    const float t_vxx = R.am[M_VXX][k] + bvx_x, t_vzz = R.am[M_VZZ][k] + bvz_z;
    const float t_vxz = R.am[M_VXZ][k] + bvx_z, t_vzx = R.am[M_VZX][k] + bvz_x;
    R.q[0][k] = bvx_x + G.bx[ix] * t_vxx;
    R.q[1][k] = bvz_z + G.bz[iz] * t_vzz;
    R.q[2][k] = bvx_z + G.bzh[iz] * t_vxz;
    R.q[3][k] = bvz_x + G.bxh[ix] * t_vzx;
    R.am[M_VXX][k] = G.ax[ix] * t_vxx;
    R.am[M_VZX][k] = G.axh[ix] * t_vzx;
    R.am[M_VZZ][k] = G.az[iz] * t_vzz;
    R.am[M_VXZ][k] = G.azh[iz] * t_vxz;
}

// stress-adjoint apply: adjoint velocities gather the transposed stencils of q
template <int M>
__global__ void __launch_bounds__(256) sapp(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, k = o + (long long)iz * G.nx + ix;
    const float dqxx_dx = da<M>(G, R.q[0] + o, 1, ix, iz, false, true, true);
    const float dqxz_dz = da<M>(G, R.q[2] + o, 0, ix, iz, true, false, false);
    const float dqzx_dx = da<M>(G, R.q[3] + o, 1, ix, iz, true, false, false);
    const float dqzz_dz = da<M>(G, R.q[1] + o, 0, ix, iz, false, true, true);
    R.a[VX][k] = R.a[VX][k] + (dqxx_dx + dqxz_dz);
    R.a[VZ][k] = R.a[VZ][k] + (dqzx_dx + dqzz_dz);
}

// velocity-adjoint prepare over every cell (reference kernels.cuh:873-958)
__global__ void __launch_bounds__(256) vprep(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, k = o + i;
    const float kv = G.kv[b * G.ms + i];
    const float b_sxx_x = kv * R.a[VX][k], b_sxz_z = kv * R.a[VX][k];
    const float b_sxz_x = kv * R.a[VZ][k], b_szz_z = kv * R.a[VZ][k];
    if (!in_pml(G, ix, iz)) {
        R.q[0][k] = b_sxx_x; R.q[2][k] = b_sxz_z; R.q[3][k] = b_sxz_x; R.q[1][k] = b_szz_z;
        return;
    }
    const float t_sxxx = R.am[M_SXXX][k] + b_sxx_x, t_sxzz = R.am[M_SXZZ][k] + b_sxz_z;
    const float t_sxzx = R.am[M_SXZX][k] + b_sxz_x, t_szzz = R.am[M_SZZZ][k] + b_szz_z;
    R.q[0][k] = b_sxx_x + G.bxh[ix] * t_sxxx;
    R.q[2][k] = b_sxz_z + G.bz[iz] * t_sxzz;
    R.q[3][k] = b_sxz_x + G.bx[ix] * t_sxzx;
    R.q[1][k] = b_szz_z + G.bzh[iz] * t_szzz;
    R.am[M_SXXX][k] = G.axh[ix] * t_sxxx;
    R.am[M_SXZX][k] = G.ax[ix] * t_sxzx;
    R.am[M_SXZZ][k] = G.az[iz] * t_sxzz;
    R.am[M_SZZZ][k] = G.azh[iz] * t_szzz;
}

// velocity-adjoint apply (reference kernels.cuh:989-1019)
template <int M>
__global__ void __launch_bounds__(256) vapp(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, k = o + (long long)iz * G.nx + ix;
    const float dpxx_dx = da<M>(G, R.q[0] + o, 1, ix, iz, true, true, false);
    const float dpzz_dz = da<M>(G, R.q[1] + o, 0, ix, iz, true, true, false);
    const float dpxz_dz = da<M>(G, R.q[2] + o, 0, ix, iz, false, true, true);
    const float dpzx_dx = da<M>(G, R.q[3] + o, 1, ix, iz, false, true, true);
    R.a[SXX][k] = R.a[SXX][k] + dpxx_dx;
    R.a[SZZ][k] = R.a[SZZ][k] + dpzz_dz;
    R.a[SXZ][k] = R.a[SXZ][k] + (dpxz_dz + dpzx_dx);
}

// v(it) carriers on the physical box (they hold v(it + 1) for the next step)
__global__ void carriers(const Geo G, Rev R)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || ix < G.x0 || ix >= G.x1 || iz < G.z0 || iz >= G.z1) return;
    const long long k = b * G.S + (long long)iz * G.nx + ix;
    R.vxn[k] = R.f[VX][k];
    R.vzn[k] = R.f[VZ][k];
}

// per-shot slots (B, S) -> out on the physical box, zero elsewhere: (B, S)
// for per-shot models, else the sum over shots in shot order
__global__ void finalize(const Geo G, const float* __restrict__ slots, float* out)
{
    const bool per_shot = G.ms != 0;
    const long long n = per_shot ? (long long)G.B * G.S : G.S;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long c = k % G.S;
        const int iz = (int)(c / G.nx), ix = (int)(c % G.nx);
        float v = 0.f;
        if (ix >= G.x0 && ix < G.x1 && iz >= G.z0 && iz < G.z1) {
            v = slots[k];
            if (!per_shot)
                for (int b = 1; b < G.B; ++b) v += slots[(long long)b * G.S + k];
        }
        out[k] = v;
    }
}

// ------------------------------------------------------------------- host
struct Plan {
    Geo G;
    int nm;                         // model copies
    std::vector<int> cells;
};

// staggered first-derivative weights of half-width M (the closed form
// a_m = (-1)^(m+1) / (2m - 1) prod_{n != m} |(2n-1)^2 / ((2n-1)^2 - (2m-1)^2)|,
// reference operators/staggered.cuh), each rounded from the exact ratio
static void staggered_weights(int M, float* c)
{
    for (int m = 1; m <= M; ++m) {
        long long num = 1, den = 2 * m - 1;
        for (int n = 1; n <= M; ++n) {
            if (n == m) continue;
            const long long a = (long long)(2 * n - 1) * (2 * n - 1), q = (long long)(2 * m - 1) * (2 * m - 1);
            num *= a;
            den *= a > q ? a - q : q - a;
        }
        const double v = (double)num / (double)den;
        c[m] = (float)((m % 2 == 1) ? v : -v);
    }
}

static Plan make_plan(const sweep_elastic_desc* d, int mem_mode)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->M >= 1 && d->M <= MAXM, "elastic: spatial orders 2 to %d are built (got order %d)", 2 * MAXM,
                  2 * d->M);
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY,
                  "elastic order %d: boundary saving with fp32 strips in device memory is built for orders other "
                  "than 8 (mem_mode %d; checkpoints, reduced strip formats and the host tape run at order 8)",
                  2 * d->M, mem_mode);
    SWEEP_REQUIRE(d->B >= 1 && d->B <= 65535 && d->nt >= 1, "elastic: 1 to 65535 shots and nt >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "elastic: negative source/receiver count");
    SWEEP_REQUIRE(d->nsrc_fields >= 1 && d->nsrc_fields <= 5, "elastic: 1 to 5 source fields");
    SWEEP_REQUIRE(d->nrec_fields >= 1 && d->nrec_fields <= 5, "elastic: 1 to 5 receiver fields");
    for (int k = 0; k < d->nsrc_fields; ++k) {
        SWEEP_REQUIRE(d->src_fields[k] >= 0 && d->src_fields[k] < 5, "elastic: bad source field %d", d->src_fields[k]);
        for (int j = 0; j < k; ++j)
            SWEEP_REQUIRE(d->src_fields[j] != d->src_fields[k], "elastic: source field %d repeated", d->src_fields[k]);
    }
    for (int k = 0; k < d->nrec_fields; ++k)
        SWEEP_REQUIRE(d->rec_fields[k] >= 0 && d->rec_fields[k] < 5, "elastic: bad receiver field %d",
                      d->rec_fields[k]);
    Plan pl{};
    Geo& G = pl.G;
    const int M = d->M;
    G.B = d->B; G.nz = d->nz; G.nx = d->nx; G.nt = d->nt; G.M = M;
    G.S = (long long)d->nz * d->nx;
    SWEEP_REQUIRE(G.S < (1LL << 31), "elastic: one shot's grid must hold < 2^31 cells");
    G.fs = 0;
    for (int f = 0; f < 4; ++f) {
        G.pad[f] = d->pad[f];
        if (d->free_surface[f]) {
            SWEEP_REQUIRE(d->pad[f] == 0, "elastic: a free face has no PML pad (face %d has %d)", f, d->pad[f]);
            G.fs |= 1 << f;
        } else {
            SWEEP_REQUIRE(d->pad[f] >= 1, "elastic: every absorbing face needs a PML pad >= 1 (face %d has %d)", f,
                          d->pad[f]);
        }
    }
    G.z0 = G.pad[0] + M; G.z1 = G.nz - G.pad[1] - M;
    G.x0 = G.pad[2] + M; G.x1 = G.nx - G.pad[3] - M;
    SWEEP_REQUIRE(G.z1 - G.z0 >= 2 && G.x1 - G.x0 >= 2, "elastic: the physical box must be at least 2 cells per axis");
    G.dt = d->dt; G.dz = d->dz; G.dx = d->dx;
    for (int k = 0; k <= MAXM; ++k) G.c[k] = 0.f;
    staggered_weights(M, G.c);
    G.az = d->az; G.bz = d->bz; G.azh = d->azh; G.bzh = d->bzh;
    G.ax = d->ax; G.bx = d->bx; G.axh = d->axh; G.bxh = d->bxh;
    G.vp = d->vp; G.vs = d->vs; G.rho = d->rho;
    const bool per_shot = d->model_stride != 0;
    SWEEP_REQUIRE(!per_shot || d->model_stride == G.S, "elastic: model_stride must be 0 or nz * nx");
    G.ms = per_shot ? G.S : 0;
    pl.nm = per_shot ? G.B : 1;
    G.nsrc = d->nsrc; G.nrec = d->nrec; G.nsf = d->nsrc_fields; G.nrf = d->nrec_fields;
    for (int k = 0; k < 5; ++k) { G.sf[k] = d->src_fields[k]; G.rf[k] = d->rec_fields[k]; }
    G.src = d->src_loc; G.rec = d->rec_loc; G.wavelet = d->wavelet;
    // the boundary bands (boundary/strip.cuh:46-123: width M + 1 from M cells
    // outside the box, each band over the box tangentially; a band that would
    // leave the grid slides back inside)
    const int w = M + 1, off = -M;
    auto band_lo = [](int p0, int of, int wd, int n) { int s = p0 + of; if (s + wd > n) s = n - wd; return s < 0 ? 0 : s; };
    auto band_hi = [](int p1, int of, int wd, int n) { int e = p1 - of; if (e - wd < 0) e = wd; return e > n ? n : e; };
    const int ts = band_lo(G.z0, off, w, G.nz), be = band_hi(G.z1, off, w, G.nz);
    const int ls = band_lo(G.x0, off, w, G.nx), re = band_hi(G.x1, off, w, G.nx);
    for (int z = ts; z < ts + w; ++z) for (int x = G.x0; x < G.x1; ++x) pl.cells.push_back(z * G.nx + x);
    for (int z = be - w; z < be; ++z) for (int x = G.x0; x < G.x1; ++x) pl.cells.push_back(z * G.nx + x);
    for (int z = G.z0; z < G.z1; ++z) for (int x = ls; x < ls + w; ++x) pl.cells.push_back(z * G.nx + x);
    for (int z = G.z0; z < G.z1; ++z) for (int x = re - w; x < re; ++x) pl.cells.push_back(z * G.nx + x);
    G.ns = (int)pl.cells.size();
    return pl;
}

struct Ws {
    float *lam, *mu, *kv;
    int* cells;
    float* f[5];
    float* m[NMEM];                 // forward memories / adjoint memories
    float* a[5];
    float* q[4];
    float *vxn, *vzn, *gvp, *gvs, *grho;
    char *zero0, *zero1;
};

static void carve(Carve& c, const Plan& pl, bool rev, Ws& w)
{
    const Geo& G = pl.G;
    const long long n = (long long)G.B * G.S, mc = (long long)pl.nm * G.S;
    w = Ws{};
    w.lam = c.take<float>(mc); w.mu = c.take<float>(mc); w.kv = c.take<float>(mc);
    w.cells = c.take<int>(std::max(G.ns, 1));
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    for (int k = 0; k < 5; ++k) w.f[k] = c.take<float>(n);
    for (int k = 0; k < NMEM; ++k) w.m[k] = c.take<float>(n);
    if (rev) {
        for (int k = 0; k < 5; ++k) w.a[k] = c.take<float>(n);
        w.vxn = c.take<float>(n); w.vzn = c.take<float>(n);
        w.gvp = c.take<float>(n); w.gvs = c.take<float>(n); w.grho = c.take<float>(n);
    }
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
    if (rev)
        for (int k = 0; k < 4; ++k) w.q[k] = c.take<float>(n);
}

static long long slot_floats(const Plan& pl) { return (long long)pl.G.B * 5 * pl.G.ns; }

void sizes(const sweep_elastic_desc* d, int mem_mode, int, int64_t* ws_bytes, int64_t* tape_bytes)
{
    const Plan pl = make_plan(d, mem_mode);
    Carve f(nullptr), r(nullptr);
    Ws w;
    carve(f, pl, false, w);
    carve(r, pl, true, w);
    *ws_bytes = std::max(f.off, r.off);
    *tape_bytes = ((long long)pl.G.nt * slot_floats(pl) + 5LL * pl.G.B * pl.G.S) * 4;
}

static void setup(const sweep_elastic_desc* d, Plan& pl, const Ws& w, cudaStream_t st)
{
    Geo& G = pl.G;
    G.lam = w.lam; G.mu = w.mu; G.kv = w.kv; G.cells = w.cells;
    const long long mc = (long long)pl.nm * G.S;
    prep<<<(unsigned)std::min<long long>((mc + 255) / 256, 4096), 256, 0, st>>>(d->vp, d->vs, d->rho, mc, d->dt,
                                                                                 w.lam, w.mu, w.kv);
    SWEEP_LAUNCH_CHECK();
    if (G.ns > 0)
        SWEEP_CUDA(cudaMemcpyAsync(w.cells, pl.cells.data(), sizeof(int) * G.ns, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
}

static dim3 grid_of(const Geo& G) { return dim3((G.nx + 31) / 32, (G.nz + 7) / 8, (unsigned)G.B); }
static unsigned blocks(long long n) { return (unsigned)std::max<long long>(std::min<long long>((n + 255) / 256, 8192), 1); }

template <int M>
static void forward_m(const sweep_elastic_desc* d, Plan& pl, float* record, void* tape, void* ws, int64_t ws_bytes,
                      cudaStream_t st)
{
    Carve c(ws);
    Ws w;
    carve(c, pl, false, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic forward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    setup(d, pl, w, st);
    const Geo& G = pl.G;
    if (record && G.nrec > 0)
        SWEEP_CUDA(cudaMemsetAsync(record, 0, sizeof(float) * (size_t)G.B * G.nt * G.nrec * G.nrf, st));
    Fields F{};
    Mems W{};
    for (int k = 0; k < 5; ++k) F.f[k] = w.f[k];
    for (int k = 0; k < NMEM; ++k) W.m[k] = w.m[k];
    float* tp = static_cast<float*>(tape);
    const dim3 grid = grid_of(G), block(32, 8);
    for (int it = 0; it < G.nt; ++it) {
        vel<M><<<grid, block, 0, st>>>(G, F, W);
        str<M><<<grid, block, 0, st>>>(G, F, W);
        if (G.nsrc > 0) inject<<<(G.B * G.nsrc + 127) / 128, 128, 0, st>>>(G, F, it, 1.f);
        if (tp) bands<<<blocks((long long)G.B * G.ns), 256, 0, st>>>(G, F, tp + it * slot_floats(pl), 0, 5, 0);
        if (record && G.nrec > 0) gather<<<(G.B * G.nrec + 127) / 128, 128, 0, st>>>(G, F, record, it);
        SWEEP_LAUNCH_CHECK();
    }
    if (tp) {
        // the final state, (B, 5, S)
        float* last = tp + (long long)G.nt * slot_floats(pl);
        for (int b = 0; b < G.B; ++b)
            for (int f = 0; f < 5; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(last + ((long long)b * 5 + f) * G.S, w.f[f] + b * G.S,
                                           sizeof(float) * G.S, cudaMemcpyDeviceToDevice, st));
    }
}

template <int M>
static void backward_m(const sweep_elastic_desc* d, Plan& pl, const float* adj, const void* tape, float* grad_vp,
                       float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    SWEEP_REQUIRE(tape != nullptr, "elastic backward: the forward's tape is required");
    Carve c(ws);
    Ws w;
    carve(c, pl, true, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    setup(d, pl, w, st);
    const Geo& G = pl.G;
    const float* tp = static_cast<const float*>(tape);
    const float* last = tp + (long long)G.nt * slot_floats(pl);
    for (int b = 0; b < G.B; ++b)
        for (int f = 0; f < 5; ++f)
            SWEEP_CUDA(cudaMemcpyAsync(w.f[f] + b * G.S, last + ((long long)b * 5 + f) * G.S, sizeof(float) * G.S,
                                       cudaMemcpyDeviceToDevice, st));
    Fields F{};
    Rev R{};
    for (int k = 0; k < 5; ++k) { F.f[k] = w.f[k]; R.f[k] = w.f[k]; R.a[k] = w.a[k]; }
    for (int k = 0; k < NMEM; ++k) R.am[k] = w.m[k];
    for (int k = 0; k < 4; ++k) R.q[k] = w.q[k];
    R.vxn = w.vxn; R.vzn = w.vzn; R.gvp = w.gvp; R.gvs = w.gvs; R.grho = w.grho;
    R.adj = adj;
    bool vsrc = false;
    for (int k = 0; k < G.nsf; ++k) vsrc |= G.sf[k] <= VZ;
    const dim3 grid = grid_of(G), block(32, 8);
    const unsigned srcb = (unsigned)(G.B * G.nsrc + 127) / 128, recb = (unsigned)(G.B * G.nrec + 127) / 128;
    const unsigned bb = blocks((long long)G.B * G.ns);
    for (int it = G.nt - 1; it >= 1; --it) {
        R.it = it;
        float* prev = const_cast<float*>(tp) + (long long)(it - 1) * slot_floats(pl);
        if (vsrc && G.nsrc > 0) vsrc_rho<<<srcb, 128, 0, st>>>(G, R);
        if (G.nrec > 0) residual<<<recb, 128, 0, st>>>(G, R);
        if (G.nsrc > 0) inject<<<srcb, 128, 0, st>>>(G, F, it, -1.f);
        srev<M><<<grid, block, 0, st>>>(G, R);
        bands<<<bb, 256, 0, st>>>(G, F, prev, SXX, 5, 1);
        sprep<M><<<grid, block, 0, st>>>(G, R);
        if (G.nrec > 0) rec_rho<<<recb, 128, 0, st>>>(G, R);
        sapp<M><<<grid, block, 0, st>>>(G, R);
        vprep<<<grid, block, 0, st>>>(G, R);
        vapp<M><<<grid, block, 0, st>>>(G, R);
        carriers<<<grid, block, 0, st>>>(G, R);
        vrev<M><<<grid, block, 0, st>>>(G, R);
        bands<<<bb, 256, 0, st>>>(G, F, prev, VX, SXX, 1);
        SWEEP_LAUNCH_CHECK();
    }
    const unsigned fb = blocks((long long)pl.nm * G.S);
    finalize<<<fb, 256, 0, st>>>(G, w.gvp, grad_vp);
    finalize<<<fb, 256, 0, st>>>(G, w.gvs, grad_vs);
    finalize<<<fb, 256, 0, st>>>(G, w.grho, grad_rho);
    SWEEP_LAUNCH_CHECK();
}

#define SWEEP_EORD_DISPATCH(M_, CALL) \
    switch (M_) {                     \
    case 1: CALL(1); break;           \
    case 2: CALL(2); break;           \
    case 3: CALL(3); break;           \
    case 4: CALL(4); break;           \
    case 5: CALL(5); break;           \
    case 6: CALL(6); break;           \
    default: CALL(7); break;          \
    }

void forward(const sweep_elastic_desc* d, int mem_mode, int, float* record, void* tape, void* ws, int64_t ws_bytes,
             cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
#define SWEEP_EORD_FWD(m) forward_m<m>(d, pl, record, tape, ws, ws_bytes, st)
    SWEEP_EORD_DISPATCH(d->M, SWEEP_EORD_FWD)
#undef SWEEP_EORD_FWD
}

void backward(const sweep_elastic_desc* d, int mem_mode, int, const float* adj, const void* tape, float* grad_vp,
              float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
#define SWEEP_EORD_BWD(m) backward_m<m>(d, pl, adj, tape, grad_vp, grad_vs, grad_rho, ws, ws_bytes, st)
    SWEEP_EORD_DISPATCH(d->M, SWEEP_EORD_BWD)
#undef SWEEP_EORD_BWD
}

}  // namespace eord
}  // namespace sweep
