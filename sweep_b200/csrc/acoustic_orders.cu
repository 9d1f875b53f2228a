// acoustic_orders.cu -- the acoustic forward and boundary-saving adjoint at
// every spatial order but 8 (M = 1..7: orders 2, 4, 6, 10, 12, 14), 2-D and
// 3-D, for sm_100a.  Order 8 runs the TMA-tiled kernels of acoustic2d.cu /
// acoustic3d.cu; the reference's Acoustic / Acoustic3D default to order 4, so
// a drop-in caller lands here unless it asks for order 8.
//
// Restates the reference's templated acoustic path (src/sweep/csrc/cuda/
// equations/acoustic2d/forward_split.cu:40-250, adjoint_split.cu:27-300,
// acoustic3d/forward_split.cu:79-372, adjoint_split.cu:14-320,
// driver_traits.cuh step order), order by order:
//   * forward and reconstruction Laplacian in difference form
//     sum_k c_k ((u_k - u0) + (u_-k - u0)) / h^2, except order 4, which keeps
//     the summed form (c1 (u_1 + u_-1) + c2 (u_2 + u_-2) - 5/2 u0) / h^2
//     (operators/laplace.cuh:68-100, 145-200); the adjoint in difference
//     form at every order;
//   * CPML per axis in the compute band: 2-D with the fused d(a psi) term
//     (pad + 2M band), 3-D with the product-rule split a d(psi) + d(a) psi on
//     the band plus one cell; the exact transposes in the adjoint;
//   * boundary saving: the strip cells (width M + 1 inside the physical box)
//     of u(it) every step, the last two states at the end; the reverse
//     reconstructs the box minus the strips, restores the strips, takes the
//     source back out of a strip cell, images, re-injects.
// One thread per cell on 32 x 8 tiles (x, z in 2-D; x, y per z plane in
// 3-D), shots on the grid's last axis, stencils through the read-only path.
// Memory: boundary saving with fp32 strips in device memory (SWEEP_MEM_BOUNDARY).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "acoustic_orders.cuh"

namespace sweep {
namespace aord {

constexpr int MAXM = 7;

struct Geo {
    int nd, B, nz, ny, nx, nt;      // ny = 1 in 2-D
    long long S;                    // cells per shot
    int pad[6];                     // z_lo, z_hi, y_lo, y_hi, x_lo, x_hi
    int z0, z1, y0, y1, x0, x1;     // physical box
    int rz0, rz1, ry0, ry1, rx0, rx1;   // reconstruction box (physical box minus the strips)
    float dt, dz, dy, dx;
    float lc[MAXM + 1], gc[MAXM + 1];
    const float *az, *bz, *dbz, *ay, *by, *dby, *ax, *bx, *dbx;
    const float* vp;
    long long vps;                  // model stride between shots (0 or S)
    int nsrc, nrec;
    const int *src, *rec;           // (B, n, nd): x[, y], z
    const float* wavelet;           // (B, nsrc, nt)
    const int* cells;               // strip cells of a shot grid
    int ns;
};

__device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
__device__ __forceinline__ float tap(float uk, float u0) { return __fsub_rn(uk, u0); }

// forward / reconstruction Laplacian along one axis (stride s, spacing h)
template <int M>
__device__ __forceinline__ float lap_f(const float* __restrict__ u, long long i, long long s, const Geo& G, float h)
{
    const float u0 = ld(u + i);
    if (M == 2)
        return ((G.lc[1] * (ld(u + i - s) + ld(u + i + s)) + G.lc[2] * (ld(u + i - 2 * s) + ld(u + i + 2 * s))) -
                2.5f * u0) /
               (h * h);
    float acc = G.lc[1] * (tap(ld(u + i - s), u0) + tap(ld(u + i + s), u0));
#pragma unroll
    for (int k = 2; k <= M; ++k) acc = acc + G.lc[k] * (tap(ld(u + i - k * s), u0) + tap(ld(u + i + k * s), u0));
    return acc / (h * h);
}

// centred first derivative sum_k g_k (u_k - u_-k) / h
template <int M>
__device__ __forceinline__ float grad_c(const float* __restrict__ u, long long i, long long s, const Geo& G, float h)
{
    float acc = G.gc[1] * (ld(u + i + s) - ld(u + i - s));
#pragma unroll
    for (int k = 2; k <= M; ++k) acc = acc + G.gc[k] * (ld(u + i + k * s) - ld(u + i - k * s));
    return acc / h;
}

// the fused d(a psi) / dx tap form of the 2-D forward
template <int M>
__device__ __forceinline__ float grad_apsi(const float* __restrict__ a, int ia, const float* __restrict__ psi,
                                           long long i, long long s, const Geo& G, float h)
{
    float acc = G.gc[1] * (ld(a + ia + 1) * ld(psi + i + s) - ld(a + ia - 1) * ld(psi + i - s));
#pragma unroll
    for (int k = 2; k <= M; ++k)
        acc = acc + G.gc[k] * (ld(a + ia + k) * ld(psi + i + k * s) - ld(a + ia - k) * ld(psi + i - k * s));
    return acc / h;
}

// ------------------------------------------------------------------- 2-D
struct Step2 {
    const float *un, *up;
    float* unx;
    const float *psx, *psz;         // CPML psi (read)
    float *psxn, *pszn;             // (written)
    float *zx, *zz;                 // zeta, in place
};

// u_next = (2 u - u_prev) + v^2 dt^2 w on [M, n - M)^2 (reference
// acoustic2d/forward_split.cu:86-168)
template <int M>
__global__ void __launch_bounds__(256) fwd2(const Geo G, Step2 A)
{
    const int ix = blockIdx.x * 32 + threadIdx.x, iz = blockIdx.y * 8 + threadIdx.y, b = blockIdx.z;
    if (ix < M || ix >= G.nx - M || iz < M || iz >= G.nz - M) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const float* un = A.un + o;
    const float* vp = G.vp + b * G.vps;
    const float lx = lap_f<M>(un, i, 1, G, G.dx), lz = lap_f<M>(un, i, G.nx, G, G.dz);
    const float v = ld(vp + i);
    const float v2dt2 = ((v * v) * G.dt) * G.dt;
    const int pml_x0 = G.pad[4] + M, pml_x1 = G.nx - (G.pad[5] + M);
    const int pml_z0 = G.pad[0] + M, pml_z1 = G.nz - (G.pad[1] + M);
    const bool cx = ix < pml_x0 + M || ix >= pml_x1 - M;
    const bool cz = iz < pml_z0 + M || iz >= pml_z1 - M;
    float w;
    if (!cx && !cz) {
        w = lx + lz;
    } else {
        w = 0.f;
        if (cx) {
            const float* ps = A.psx + o;
            float* zt = A.zx + o;
            const float a = G.ax[ix], bb = G.bx[ix], db = G.dbx[ix];
            const float du = grad_c<M>(un, i, 1, G, G.dx);
            const float dap = grad_apsi<M>(G.ax, ix, ps, i, 1, G, G.dx);
            const float tmp = ((1.f + bb) * lx + db * du) + dap;
            const float z = zt[i];
            w = w + ((1.f + bb) * tmp + a * z);
            A.psxn[o + i] = bb * du + a * ps[i];
            zt[i] = bb * tmp + a * z;
        } else {
            w = w + lx;
        }
        if (cz) {
            const float* ps = A.psz + o;
            float* zt = A.zz + o;
            const float a = G.az[iz], bb = G.bz[iz], db = G.dbz[iz];
            const float du = grad_c<M>(un, i, G.nx, G, G.dz);
            const float dap = grad_apsi<M>(G.az, iz, ps, i, G.nx, G, G.dz);
            const float tmp = ((1.f + bb) * lz + db * du) + dap;
            const float z = zt[i];
            w = w + ((1.f + bb) * tmp + a * z);
            A.pszn[o + i] = bb * du + a * ps[i];
            zt[i] = bb * tmp + a * z;
        } else {
            w = w + lz;
        }
    }
    A.unx[o + i] = (2.f * un[i] - ld(A.up + o + i)) + v2dt2 * w;
}

struct Adj2 {
    const float *ln, *lp;
    float* lnx;
    const float *psx, *psz, *zx, *zz;       // adjoint CPML memories (read)
    float *psxo, *pszo, *zxo, *zzo;         // (written)
};

// exact adjoint step (reference acoustic2d/adjoint_split.cu:27-196): the pure
// interior in difference form around gw = ((v v) dt^2) lambda; elsewhere the
// transposed CPML terms along both axes
template <int M>
__global__ void __launch_bounds__(256) adj2(const Geo G, Adj2 A)
{
    const int ix = blockIdx.x * 32 + threadIdx.x, iz = blockIdx.y * 8 + threadIdx.y, b = blockIdx.z;
    if (ix < M || ix >= G.nx - M || iz < M || iz >= G.nz - M) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const int nx = G.nx;
    const float* vp = G.vp + b * G.vps;
    const float* ln = A.ln + o;
    const float dt2 = G.dt * G.dt;
    const float invdx2 = 1.f / (G.dx * G.dx), invdz2 = 1.f / (G.dz * G.dz);
    const float invdx = 1.f / G.dx, invdz = 1.f / G.dz;
    const int ix_in0 = G.pad[4] + 2 * M + 1, ix_in1 = nx - (G.pad[5] + 2 * M + 1);
    const int iz_in0 = G.pad[0] + 2 * M + 1, iz_in1 = G.nz - (G.pad[1] + 2 * M + 1);
    auto gwat = [&](long long n) { const float v = ld(vp + n); return ((v * v) * dt2) * ld(ln + n); };
    const float gun = ld(ln + i);
    float c0c = ld(vp + i);
    c0c = (c0c * c0c) * dt2;
    const float gw = c0c * gun;
    const bool pure = ix >= ix_in0 && ix < ix_in1 && iz >= iz_in0 && iz < iz_in1;
    if (pure) {
        float lx = 0.f, lz = 0.f;
#pragma unroll
        for (int k = 1; k <= M; ++k) {
            lx = lx + G.lc[k] * (tap(gwat(i + k), gw) + tap(gwat(i - k), gw));
            lz = lz + G.lc[k] * (tap(gwat(i + (long long)k * nx), gw) + tap(gwat(i - (long long)k * nx), gw));
        }
        A.lnx[o + i] = ((2.f * gun - ld(A.lp + o + i)) + lx * invdx2) + lz * invdz2;
        return;
    }
    const float *psx = A.psx + o, *psz = A.psz + o, *zx = A.zx + o, *zz = A.zz + o;
    const float ax_ = G.ax[ix], az_ = G.az[iz], bx_ = G.bx[ix], bz_ = G.bz[iz];
    const float gtx0 = bx_ * zx[i] + (1.f + bx_) * gw;
    const float gtz0 = bz_ * zz[i] + (1.f + bz_) * gw;
    auto gtx = [&](long long n, int c) {
        const float v = ld(vp + n);
        return G.bx[c] * zx[n] + ((1.f + G.bx[c]) * ((v * v) * dt2)) * ld(ln + n);
    };
    auto gtz = [&](long long n, int c) {
        const float v = ld(vp + n);
        return G.bz[c] * zz[n] + ((1.f + G.bz[c]) * ((v * v) * dt2)) * ld(ln + n);
    };
    const float lx0 = (1.f + bx_) * gtx0;
    float Lx = 0.f, Dgx = 0.f, Dqx = 0.f;
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        const long long np = i + k, nm = i - k;
        const int cp = ix + k, cm = ix - k;
        const float tp = gtx(np, cp), tm = gtx(nm, cm);
        const float bp = G.bx[cp], bm = G.bx[cm];
        Lx = Lx + G.lc[k] * (tap((1.f + bp) * tp, lx0) + tap((1.f + bm) * tm, lx0));
        Dgx = Dgx + G.gc[k] * ((bp * psx[np] + G.dbx[cp] * tp) - (bm * psx[nm] + G.dbx[cm] * tm));
        Dqx = Dqx + G.gc[k] * (tp - tm);
    }
    Lx = Lx * invdx2; Dgx = Dgx * invdx; Dqx = Dqx * invdx;
    const float lz0 = (1.f + bz_) * gtz0;
    float Lz = 0.f, Dgz = 0.f, Dqz = 0.f;
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        const long long np = i + (long long)k * nx, nm = i - (long long)k * nx;
        const int cp = iz + k, cm = iz - k;
        const float tp = gtz(np, cp), tm = gtz(nm, cm);
        const float bp = G.bz[cp], bm = G.bz[cm];
        Lz = Lz + G.lc[k] * (tap((1.f + bp) * tp, lz0) + tap((1.f + bm) * tm, lz0));
        Dgz = Dgz + G.gc[k] * ((bp * psz[np] + G.dbz[cp] * tp) - (bm * psz[nm] + G.dbz[cm] * tm));
        Dqz = Dqz + G.gc[k] * (tp - tm);
    }
    Lz = Lz * invdz2; Dgz = Dgz * invdz; Dqz = Dqz * invdz;
    A.lnx[o + i] = (2.f * gun - ld(A.lp + o + i)) + (((Lx + Lz) - Dgx) - Dgz);
    A.psxo[o + i] = ax_ * (psx[i] - Dqx);
    A.pszo[o + i] = az_ * (psz[i] - Dqz);
    A.zxo[o + i] = ax_ * (zx[i] + gw);
    A.zzo[o + i] = az_ * (zz[i] + gw);
}

// ------------------------------------------------------------------- 3-D
struct Step3 {
    const float *un, *up;
    float* unx;
    const float* ps[3];             // CPML psi per axis (x, y, z), read
    float* psn[3];                  // written
    float* zt[3];                   // zeta per axis, in place
};

__device__ __forceinline__ bool cell3(const Geo& G, int M, int& b, int& iz, int& iy, int& ix)
{
    ix = blockIdx.x * 32 + threadIdx.x;
    iy = blockIdx.y * 8 + threadIdx.y;
    b = blockIdx.z / G.nz;
    iz = blockIdx.z - b * G.nz;
    return ix >= M && ix < G.nx - M && iy >= M && iy < G.ny - M && iz >= M && iz < G.nz - M;
}

// one axis of the 3-D forward's CPML shell: tmp = (((1 + b) lap + db du) +
// a d(psi)) + d(a) psi; w += (1 + b) tmp + a zeta; psi' = b du + a psi;
// zeta = b tmp + a zeta (reference acoustic3d/forward_split.cu:120-215)
template <int M>
__device__ __forceinline__ float shell3(const Geo& G, const float* __restrict__ un, long long i, long long s, int c,
                                        const float* __restrict__ A_, const float* __restrict__ B_,
                                        const float* __restrict__ DB_, const float* __restrict__ ps, float* psn,
                                        float* zt, float l, float h)
{
    const float du = grad_c<M>(un, i, s, G, h);
    const float dps = grad_c<M>(ps, i, s, G, h);
    const float a = A_[c], bb = B_[c], db = DB_[c];
    const float da = grad_c<M>(A_, c, 1, G, h);
    const float p = ps[i];
    const float tmp = ((((1.f + bb) * l + db * du) + a * dps) + da * p);
    const float z = zt[i];
    psn[i] = bb * du + a * p;
    zt[i] = bb * tmp + a * z;
    return (1.f + bb) * tmp + a * z;
}

template <int M>
__global__ void __launch_bounds__(256) fwd3(const Geo G, Step3 A)
{
    int b, iz, iy, ix;
    if (!cell3(G, M, b, iz, iy, ix)) return;
    const long long sy = G.nx, sz = (long long)G.nx * G.ny;
    const long long o = b * G.S, i = iz * sz + iy * sy + ix;
    const float* un = A.un + o;
    const float lx = lap_f<M>(un, i, 1, G, G.dx), ly = lap_f<M>(un, i, sy, G, G.dy),
                lz = lap_f<M>(un, i, sz, G, G.dz);
    const int px0 = G.pad[4] + M, px1 = G.nx - G.pad[5] - M;
    const int py0 = G.pad[2] + M, py1 = G.ny - G.pad[3] - M;
    const int pz0 = G.pad[0] + M, pz1 = G.nz - G.pad[1] - M;
    const bool inx = ix < px0 + 1 || ix >= px1 - 1;
    const bool iny = iy < py0 + 1 || iy >= py1 - 1;
    const bool inz = iz < pz0 + 1 || iz >= pz1 - 1;
    float w;
    if (!inx && !iny && !inz) {
        w = (lx + ly) + lz;
    } else {
        w = 0.f;
        w = w + (inx ? shell3<M>(G, un, i, 1, ix, G.ax, G.bx, G.dbx, A.ps[0] + o, A.psn[0] + o, A.zt[0] + o, lx, G.dx)
                     : lx);
        w = w + (iny ? shell3<M>(G, un, i, sy, iy, G.ay, G.by, G.dby, A.ps[1] + o, A.psn[1] + o, A.zt[1] + o, ly, G.dy)
                     : ly);
        w = w + (inz ? shell3<M>(G, un, i, sz, iz, G.az, G.bz, G.dbz, A.ps[2] + o, A.psn[2] + o, A.zt[2] + o, lz, G.dz)
                     : lz);
    }
    const float v = ld(G.vp + b * G.vps + i);
    A.unx[o + i] = (2.f * un[i] - ld(A.up + o + i)) + (((v * v) * G.dt) * G.dt) * w;
}

// gw = ((v v) dt^2) lambda on every cell (the 3-D adjoint's taps read it)
__global__ void gw3(const Geo G, const float* __restrict__ ln, float* __restrict__ gw)
{
    const long long n = (long long)G.B * G.S;
    const float dt2 = G.dt * G.dt;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long b = k / G.S;
        const float v = ld(G.vp + b * G.vps + (k - b * G.S));
        gw[k] = ((v * v) * dt2) * ln[k];
    }
}

struct Adj3 {
    const float *ln, *lp, *gw;
    float* lnx;
    const float *ps[3], *zt[3];     // adjoint CPML memories (read)
    float *pso[3], *zto[3];         // (written)
};

// exact 3-D adjoint step (reference acoustic3d/adjoint_split.cu:14-320)
template <int M>
__global__ void __launch_bounds__(256) adj3(const Geo G, Adj3 A)
{
    int b, iz, iy, ix;
    if (!cell3(G, M, b, iz, iy, ix)) return;
    const long long sy = G.nx, sz = (long long)G.nx * G.ny;
    const long long o = b * G.S, i = iz * sz + iy * sy + ix;
    const float* vp = G.vp + b * G.vps;
    const float* ln = A.ln + o;
    const float* gwb = A.gw + o;
    const float dt2 = G.dt * G.dt;
    const int c[3] = {ix, iy, iz};
    const long long st[3] = {1, sy, sz};
    const float h[3] = {G.dx, G.dy, G.dz};
    const int lo[3] = {G.pad[4] + 2 * M + 1, G.pad[2] + 2 * M + 1, G.pad[0] + 2 * M + 1};
    const int hi[3] = {G.nx - (G.pad[5] + 2 * M + 1), G.ny - (G.pad[3] + 2 * M + 1), G.nz - (G.pad[1] + 2 * M + 1)};
    const float gun = ld(ln + i);
    float c0c = ld(vp + i);
    c0c = (c0c * c0c) * dt2;
    const float gw = c0c * gun;
    bool in[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) in[a] = c[a] < lo[a] || c[a] >= hi[a];
    float L[3], Dg[3] = {0.f, 0.f, 0.f};
    if (!in[0] && !in[1] && !in[2]) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float acc = 0.f;
#pragma unroll
            for (int k = 1; k <= M; ++k)
                acc = acc + G.lc[k] * (tap(ld(gwb + i + k * st[a]), gw) + tap(ld(gwb + i - k * st[a]), gw));
            L[a] = acc;
        }
        A.lnx[o + i] = (((2.f * gun - ld(A.lp + o + i)) + L[0] * (1.f / (h[0] * h[0]))) + L[1] * (1.f / (h[1] * h[1]))) +
                       L[2] * (1.f / (h[2] * h[2]));
        return;
    }
    const float* av[3] = {G.ax, G.ay, G.az};
    const float* bv[3] = {G.bx, G.by, G.bz};
    const float* dbv[3] = {G.dbx, G.dby, G.dbz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float invh2 = 1.f / (h[a] * h[a]), invh = 1.f / h[a];
        if (in[a]) {
            const float *Av = av[a], *Bv = bv[a], *DB = dbv[a];
            const float* Z = A.zt[a] + o;
            const float* PS = A.ps[a] + o;
            const float a_ = Av[c[a]], b_ = Bv[c[a]];
            const float da = grad_c<M>(Av, c[a], 1, G, h[a]);
            const float gt0 = b_ * Z[i] + (1.f + b_) * gw;
            const float l0 = (1.f + b_) * gt0;
            float Lq = 0.f, Dq = 0.f, Dgg = 0.f;
#pragma unroll
            for (int k = 1; k <= M; ++k) {
                const long long np = i + k * st[a], nm = i - k * st[a];
                const int cp = c[a] + k, cm = c[a] - k;
                const float vpp = ld(vp + np), vpm = ld(vp + nm);
                const float tp = Bv[cp] * Z[np] + ((1.f + Bv[cp]) * ((vpp * vpp) * dt2)) * ld(ln + np);
                const float tm = Bv[cm] * Z[nm] + ((1.f + Bv[cm]) * ((vpm * vpm) * dt2)) * ld(ln + nm);
                Lq = Lq + G.lc[k] * (tap((1.f + Bv[cp]) * tp, l0) + tap((1.f + Bv[cm]) * tm, l0));
                Dgg = Dgg + G.gc[k] * ((Bv[cp] * PS[np] + DB[cp] * tp) - (Bv[cm] * PS[nm] + DB[cm] * tm));
                Dq = Dq + G.gc[k] * (Av[cp] * tp - Av[cm] * tm);
            }
            L[a] = Lq * invh2;
            Dg[a] = Dgg * invh;
            Dq = Dq * invh;
            A.pso[a][o + i] = (a_ * PS[i] + da * gt0) - Dq;
            A.zto[a][o + i] = a_ * (Z[i] + gw);
        } else {
            float acc = 0.f;
#pragma unroll
            for (int k = 1; k <= M; ++k)
                acc = acc + G.lc[k] * (tap(ld(gwb + i + k * st[a]), gw) + tap(ld(gwb + i - k * st[a]), gw));
            L[a] = acc * invh2;
        }
    }
    A.lnx[o + i] = (2.f * gun - ld(A.lp + o + i)) + (((((L[0] + L[1]) + L[2]) - Dg[0]) - Dg[1]) - Dg[2]);
}

// ------------------------------------------------------- per-step helpers
// grid offset of location l (x[, y], z) of shot b, or -1 off the grid
__device__ __forceinline__ long long loc_cell(const Geo& G, const int* l)
{
    const int x = l[0], y = G.nd == 3 ? l[1] : 0, z = l[G.nd - 1];
    if (x < 0 || x >= G.nx || y < 0 || y >= G.ny || z < 0 || z >= G.nz) return -1;
    return ((long long)z * G.ny + y) * G.nx + x;
}

__device__ __forceinline__ bool in_phys(const Geo& G, long long c)
{
    const int x = (int)(c % G.nx), r = (int)(c / G.nx), y = r % G.ny, z = r / G.ny;
    return x >= G.x0 && x < G.x1 && y >= G.y0 && y < G.y1 && z >= G.z0 && z < G.z1;
}

__device__ __forceinline__ bool in_recon(const Geo& G, long long c)
{
    const int x = (int)(c % G.nx), r = (int)(c / G.nx), y = r % G.ny, z = r / G.ny;
    return x >= G.rx0 && x < G.rx1 && y >= G.ry0 && y < G.ry1 && z >= G.rz0 && z < G.rz1;
}

// u(cell) += sign * wavelet[b, s, it] at every source (one thread per (shot, source))
__global__ void inject_src(const Geo G, float* u, int it, float sign, int only_strip)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nsrc) return;
    const int b = e / G.nsrc;
    const long long c = loc_cell(G, G.src + (long long)e * G.nd);
    if (c < 0) return;
    if (only_strip && !(in_phys(G, c) && !in_recon(G, c))) return;
    atomicAdd(u + b * G.S + c, sign * G.wavelet[(long long)e * G.nt + it]);
}

// lambda(cell) += adj[b, it, r] at every receiver
__global__ void inject_res(const Geo G, float* l, const float* __restrict__ adj, int it)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const long long c = loc_cell(G, G.rec + (long long)e * G.nd);
    if (c < 0) return;
    atomicAdd(l + b * G.S + c, adj[((long long)b * G.nt + it) * G.nrec + r]);
}

// record[b, it, r] = u(cell) (records start zeroed: off-grid receivers stay 0)
__global__ void gather_rec(const Geo G, const float* __restrict__ u, float* record, int it)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const long long c = loc_cell(G, G.rec + (long long)e * G.nd);
    if (c < 0) return;
    record[((long long)b * G.nt + it) * G.nrec + r] = u[b * G.S + c];
}

// grad_wavelet[b, s, it] = lambda(cell) at every source
__global__ void gather_src(const Geo G, const float* __restrict__ l, float* gwav, int it)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nsrc) return;
    const int b = e / G.nsrc;
    const long long c = loc_cell(G, G.src + (long long)e * G.nd);
    if (c < 0) return;
    gwav[(long long)e * G.nt + it] = l[b * G.S + c];
}

// strip save (restore = 0) of u into one step slot (B, ns), or restore
__global__ void strips(const Geo G, float* u, float* slot, int restore)
{
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long b = e / G.ns;
        const long long i = b * G.S + G.cells[e - b * G.ns];
        if (restore) u[i] = slot[e];
        else slot[e] = u[i];
    }
}

// image 2 dt^2 u_tt lambda / v, u_tt = ((u(it-1) - 2 u(it)) + u(it+1)) / dt^2
__device__ __forceinline__ void image(const Geo& G, long long b, long long c, const float* rx, const float* rn,
                                      const float* rp, const float* ln, float* g)
{
    const long long i = b * G.S + c;
    const float dt2 = G.dt * G.dt;
    const float utt = ((rx[i] - 2.f * rn[i]) + rp[i]) / dt2;
    g[i] = g[i] + ((((2.f * G.dt) * G.dt) * utt) * ln[i]) / ld(G.vp + b * G.vps + c);
}

__global__ void strip_image(const Geo G, const float* rx, const float* rn, const float* rp, const float* ln,
                            float* g)
{
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long b = e / G.ns;
        image(G, b, G.cells[e - b * G.ns], rx, rn, rp, ln, g);
    }
}

// u(it-1) = (2 u(it) - u(it+1)) + v^2 dt^2 Lap u(it) on the reconstruction box,
// with the fused image (reference acoustic2d/kernels.cuh:474-528,
// acoustic3d/forward_split.cu:292-372)
template <int M>
__global__ void __launch_bounds__(256) recon(const Geo G, const float* rn, const float* rp, float* rx,
                                             const float* ln, float* g)
{
    int ix, iy, iz, b;
    if (G.nd == 2) {
        ix = blockIdx.x * 32 + threadIdx.x; iz = blockIdx.y * 8 + threadIdx.y; iy = 0; b = blockIdx.z;
    } else {
        ix = blockIdx.x * 32 + threadIdx.x; iy = blockIdx.y * 8 + threadIdx.y;
        b = blockIdx.z / G.nz; iz = blockIdx.z - b * G.nz;
    }
    if (ix < G.rx0 || ix >= G.rx1 || iz < G.rz0 || iz >= G.rz1 || (G.nd == 3 && (iy < G.ry0 || iy >= G.ry1))) return;
    const long long sy = G.nx, sz = (long long)G.nx * G.ny;
    const long long o = (long long)b * G.S, c = iz * sz + iy * sy + ix;
    const float* u = rn + o;
    float w;
    if (G.nd == 2) w = lap_f<M>(u, c, 1, G, G.dx) + lap_f<M>(u, c, sz, G, G.dz);
    else w = (lap_f<M>(u, c, 1, G, G.dx) + lap_f<M>(u, c, sy, G, G.dy)) + lap_f<M>(u, c, sz, G, G.dz);
    const float v = ld(G.vp + b * G.vps + c);
    const float u0 = u[c], up = rp[o + c];
    const float un = (2.f * u0 - up) + (((v * v) * G.dt) * G.dt) * w;
    rx[o + c] = un;
    const float dt2 = G.dt * G.dt;
    const float utt = ((un - 2.f * u0) + up) / dt2;
    g[o + c] = g[o + c] + ((((2.f * G.dt) * G.dt) * utt) * ln[o + c]) / v;
}

// illumination on the physical box: ir += lambda^2; is += u_tt^2 (is null:
// the it = 0 tail, lambda only)
__global__ void illum(const Geo G, const float* rx, const float* rn, const float* rp, const float* ln, float* is,
                      float* ir)
{
    const long long n = (long long)G.B * G.S;
    const float dt2 = G.dt * G.dt;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long c = k % G.S;
        if (!in_phys(G, c)) continue;
        ir[k] += ln[k] * ln[k];
        if (is) {
            const float utt = ((rx[k] - 2.f * rn[k]) + rp[k]) / dt2;
            is[k] += utt * utt;
        }
    }
}

// per-shot slots (B, S) -> out: (B, S) for per-shot models, else the sum over
// shots in shot order
__global__ void finalize(const Geo G, const float* __restrict__ slots, int per_shot, float* out)
{
    const long long n = per_shot ? (long long)G.B * G.S : G.S;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        float v = slots[k];
        if (!per_shot)
            for (int b = 1; b < G.B; ++b) v += slots[(long long)b * G.S + k];
        out[k] = v;
    }
}

// ------------------------------------------------------------------- host
struct Plan {
    Geo G;
    std::vector<int> cells;
};

static Plan make_plan(const sweep_acoustic_desc* d, int mem_mode)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
    SWEEP_REQUIRE(d->M >= 1 && d->M <= MAXM, "acoustic: spatial orders 2 to %d are built (got order %d)", 2 * MAXM,
                  2 * d->M);
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY,
                  "acoustic order %d: boundary saving with fp32 strips in device memory is built for orders other "
                  "than 8 (mem_mode %d; checkpoints, reduced strip formats and the host tape run at order 8)",
                  2 * d->M, mem_mode);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1, "acoustic: B and nt must be >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "acoustic: negative source/receiver count");
    const int nf = d->ndim == 2 ? 4 : 6;
    for (int f = 0; f < 6; ++f)
        SWEEP_REQUIRE(d->pad[f] >= 0, "acoustic: negative PML pad on face %d", f);
    (void)nf;
    Plan pl{};
    Geo& G = pl.G;
    const int M = d->M;
    G.nd = d->ndim; G.B = d->B; G.nz = d->nz; G.nx = d->nx; G.nt = d->nt;
    G.ny = d->ndim == 3 ? d->ny : 1;
    G.S = (long long)G.nz * G.ny * G.nx;
    SWEEP_REQUIRE(G.S < (1LL << 31), "acoustic: one shot's grid must hold < 2^31 cells");
    SWEEP_REQUIRE(d->ndim == 2 || (long long)G.nz * G.B <= 65535, "acoustic: nz x shots must be <= 65535");
    SWEEP_REQUIRE(d->ndim == 3 || G.B <= 65535, "acoustic: at most 65535 shots per call");
    for (int f = 0; f < 6; ++f) G.pad[f] = d->pad[f];
    if (d->ndim == 2) { G.pad[2] = G.pad[3] = 0; }
    G.z0 = G.pad[0] + M; G.z1 = G.nz - G.pad[1] - M;
    G.x0 = G.pad[4] + M; G.x1 = G.nx - G.pad[5] - M;
    if (d->ndim == 3) { G.y0 = G.pad[2] + M; G.y1 = G.ny - G.pad[3] - M; }
    else { G.y0 = 0; G.y1 = 1; }
    SWEEP_REQUIRE(G.z1 > G.z0 && G.x1 > G.x0 && G.y1 > G.y0, "acoustic: the physical box is empty");
    G.rz0 = G.pad[0] + 2 * M + 1; G.rz1 = G.nz - (G.pad[1] + 2 * M + 1);
    G.rx0 = G.pad[4] + 2 * M + 1; G.rx1 = G.nx - (G.pad[5] + 2 * M + 1);
    if (d->ndim == 3) { G.ry0 = G.pad[2] + 2 * M + 1; G.ry1 = G.ny - (G.pad[3] + 2 * M + 1); }
    else { G.ry0 = 0; G.ry1 = 1; }
    G.dt = d->dt; G.dz = d->dz; G.dy = d->dy; G.dx = d->dx;
    for (int k = 0; k <= MAXM; ++k) { G.lc[k] = k <= M ? d->lap[k] : 0.f; G.gc[k] = k <= M ? d->grad[k] : 0.f; }
    G.az = d->az; G.bz = d->bz; G.dbz = d->dbz;
    G.ay = d->ay; G.by = d->by; G.dby = d->dby;
    G.ax = d->ax; G.bx = d->bx; G.dbx = d->dbx;
    G.vp = d->vp;
    SWEEP_REQUIRE(d->vp_stride == 0 || d->vp_stride == G.S, "acoustic: vp_stride must be 0 or the cells per shot");
    G.vps = d->vp_stride;
    G.nsrc = d->nsrc; G.nrec = d->nrec;
    G.src = d->src_loc; G.rec = d->rec_loc; G.wavelet = d->wavelet;
    // strip cells: the physical box within M + 1 of its faces (widths clipped
    // on a thin box: boundary/strip.cuh:63-67)
    const int w = M + 1;
    auto widths = [&](int e, int& lo, int& hi) {
        lo = std::min(w, std::max(e, 0));
        hi = std::min(w, std::max(e - lo, 0));
    };
    int wzl, wzh, wyl, wyh, wxl, wxh;
    widths(G.z1 - G.z0, wzl, wzh);
    widths(G.y1 - G.y0, wyl, wyh);
    widths(G.x1 - G.x0, wxl, wxh);
    if (d->ndim == 2) { wyl = wyh = 0; }
    for (int iz = G.z0; iz < G.z1; ++iz)
        for (int iy = G.y0; iy < G.y1; ++iy)
            for (int ix = G.x0; ix < G.x1; ++ix) {
                const bool zs = iz < G.z0 + wzl || iz >= G.z1 - wzh;
                const bool ys = iy < G.y0 + wyl || iy >= G.y1 - wyh;
                const bool xs = ix < G.x0 + wxl || ix >= G.x1 - wxh;
                if (zs || ys || xs) pl.cells.push_back((int)(((long long)iz * G.ny + iy) * G.nx + ix));
            }
    G.ns = (int)pl.cells.size();
    return pl;
}

struct Ws {
    int* cells;
    float* u[3];                    // forward: u_prev, u, u_next; backward: reconstruction
    float* l[3];                    // backward: adjoint
    float* ps[2][3];                // CPML psi (forward) / adjoint psi, double-buffered
    float* zt[2][3];                // zeta (forward: [0] only) / adjoint zeta, double-buffered
    float *g, *gw, *is, *ir;        // backward: per-shot image, gw buffer, illumination slots
    char *zero0, *zero1;
};

static void carve(Carve& c, const Plan& pl, bool rev, Ws& w)
{
    const Geo& G = pl.G;
    const long long n = (long long)G.B * G.S;
    w = Ws{};
    w.cells = c.take<int>(std::max(G.ns, 1));
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    for (int k = 0; k < 3; ++k) w.u[k] = c.take<float>(n);
    for (int s = 0; s < 2; ++s)
        for (int a = 0; a < G.nd; ++a) w.ps[s][a] = c.take<float>(n);
    for (int s = 0; s < (rev ? 2 : 1); ++s)
        for (int a = 0; a < G.nd; ++a) w.zt[s][a] = c.take<float>(n);
    if (rev) {
        for (int k = 0; k < 3; ++k) w.l[k] = c.take<float>(n);
        w.g = c.take<float>(n);
        w.is = c.take<float>(n);
        w.ir = c.take<float>(n);
    }
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
    if (rev && G.nd == 3) w.gw = c.take<float>(n);
}

static long long slot_floats(const Plan& pl) { return (long long)pl.G.B * pl.G.ns; }

void sizes(const sweep_acoustic_desc* d, int mem_mode, int, int64_t* ws_bytes, int64_t* tape_bytes)
{
    const Plan pl = make_plan(d, mem_mode);
    Carve f(nullptr), r(nullptr);
    Ws w;
    carve(f, pl, false, w);
    carve(r, pl, true, w);
    *ws_bytes = std::max(f.off, r.off);
    *tape_bytes = ((long long)pl.G.nt * slot_floats(pl) + 2LL * pl.G.B * pl.G.S) * 4;
}

static dim3 cell_grid(const Geo& G)
{
    if (G.nd == 2) return dim3((G.nx + 31) / 32, (G.nz + 7) / 8, (unsigned)G.B);
    return dim3((G.nx + 31) / 32, (G.ny + 7) / 8, (unsigned)(G.nz * G.B));
}

static unsigned blocks_of(long long n, int per) { return (unsigned)std::max<long long>(std::min<long long>((n + per - 1) / per, 8192), 1); }

template <int M>
static void fwd_step(const Geo& G, const Ws& w, float* un, float* up, float* unx, int cur, cudaStream_t st)
{
    const dim3 grid = cell_grid(G), block(32, 8);
    if (G.nd == 2) {
        Step2 A{un, up, unx, w.ps[cur][0], w.ps[cur][1], w.ps[cur ^ 1][0], w.ps[cur ^ 1][1], w.zt[0][0], w.zt[0][1]};
        fwd2<M><<<grid, block, 0, st>>>(G, A);
    } else {
        Step3 A{};
        A.un = un; A.up = up; A.unx = unx;
        for (int a = 0; a < 3; ++a) { A.ps[a] = w.ps[cur][a]; A.psn[a] = w.ps[cur ^ 1][a]; A.zt[a] = w.zt[0][a]; }
        fwd3<M><<<grid, block, 0, st>>>(G, A);
    }
}

template <int M>
static void adj_step(const Geo& G, const Ws& w, float* ln, float* lp, float* lnx, int cur, cudaStream_t st)
{
    const dim3 grid = cell_grid(G), block(32, 8);
    if (G.nd == 2) {
        // the 2-D axes are x (slot 0) and z (slot 1)
        Adj2 A{ln, lp, lnx, w.ps[cur][0], w.ps[cur][1], w.zt[cur][0], w.zt[cur][1],
               w.ps[cur ^ 1][0], w.ps[cur ^ 1][1], w.zt[cur ^ 1][0], w.zt[cur ^ 1][1]};
        adj2<M><<<grid, block, 0, st>>>(G, A);
    } else {
        gw3<<<blocks_of((long long)G.B * G.S, 256), 256, 0, st>>>(G, ln, w.gw);
        Adj3 A{};
        A.ln = ln; A.lp = lp; A.gw = w.gw; A.lnx = lnx;
        for (int a = 0; a < 3; ++a) {
            A.ps[a] = w.ps[cur][a]; A.zt[a] = w.zt[cur][a];
            A.pso[a] = w.ps[cur ^ 1][a]; A.zto[a] = w.zt[cur ^ 1][a];
        }
        adj3<M><<<grid, block, 0, st>>>(G, A);
    }
}

template <int M>
static void forward_m(Plan& pl, float* record, void* tape, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Carve c(ws);
    Ws w;
    carve(c, pl, false, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "acoustic forward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    Geo& G = pl.G;
    G.cells = w.cells;
    if (G.ns > 0)
        SWEEP_CUDA(cudaMemcpyAsync(w.cells, pl.cells.data(), sizeof(int) * G.ns, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
    if (record && G.nrec > 0)
        SWEEP_CUDA(cudaMemsetAsync(record, 0, sizeof(float) * (size_t)G.B * G.nt * G.nrec, st));
    float* tp = static_cast<float*>(tape);
    const long long n = (long long)G.B * G.S;
    float *up = w.u[0], *un = w.u[1], *unx = w.u[2];
    int cur = 0;
    const unsigned sb = blocks_of(slot_floats(pl), 256);
    for (int it = 0; it < G.nt; ++it) {
        fwd_step<M>(G, w, un, up, unx, cur, st);
        if (tp && G.ns > 0) strips<<<sb, 256, 0, st>>>(G, un, tp + (long long)it * slot_floats(pl), 0);
        if (G.nsrc > 0) inject_src<<<(G.B * G.nsrc + 127) / 128, 128, 0, st>>>(G, unx, it, 1.f, 0);
        if (record && G.nrec > 0) gather_rec<<<(G.B * G.nrec + 127) / 128, 128, 0, st>>>(G, unx, record, it);
        SWEEP_LAUNCH_CHECK();
        float* t = up; up = un; un = unx; unx = t;
        cur ^= 1;
    }
    if (tp) {
        float* tail = tp + (long long)G.nt * slot_floats(pl);
        SWEEP_CUDA(cudaMemcpyAsync(tail, up, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        SWEEP_CUDA(cudaMemcpyAsync(tail + n, un, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    }
}

template <int M>
static void backward_m(Plan& pl, const float* adj, const void* tape, float* grad_vp, float* grad_wavelet,
                       float* illum_src, float* illum_rec, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Carve c(ws);
    Ws w;
    carve(c, pl, true, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "acoustic backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    SWEEP_REQUIRE(tape != nullptr, "acoustic backward: the forward's tape is required");
    Geo& G = pl.G;
    G.cells = w.cells;
    if (G.ns > 0)
        SWEEP_CUDA(cudaMemcpyAsync(w.cells, pl.cells.data(), sizeof(int) * G.ns, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
    if (grad_wavelet && G.nsrc > 0)
        SWEEP_CUDA(cudaMemsetAsync(grad_wavelet, 0, sizeof(float) * (size_t)G.B * G.nsrc * G.nt, st));
    const float* tp = static_cast<const float*>(tape);
    const long long n = (long long)G.B * G.S;
    const bool il = illum_src || illum_rec;
    float *rp = w.u[0], *rn = w.u[1], *rx = w.u[2];
    const float* tail = tp + (long long)G.nt * slot_floats(pl);
    SWEEP_CUDA(cudaMemcpyAsync(rp, tail + n, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    SWEEP_CUDA(cudaMemcpyAsync(rn, tail, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    float *lp = w.l[0], *ln = w.l[1], *lx = w.l[2];
    int cur = 0;
    const dim3 grid = cell_grid(G), block(32, 8);
    const unsigned sb = blocks_of(slot_floats(pl), 256), cb = blocks_of(n, 256);
    const unsigned srcb = (unsigned)(G.B * G.nsrc + 127) / 128, recb = (unsigned)(G.B * G.nrec + 127) / 128;
    for (int it = G.nt - 1; it >= 0; --it) {
        adj_step<M>(G, w, ln, lp, lx, cur, st);
        if (G.nrec > 0) inject_res<<<recb, 128, 0, st>>>(G, lx, adj, it);
        { float* t = lp; lp = ln; ln = lx; lx = t; }
        cur ^= 1;
        if (grad_wavelet && G.nsrc > 0) gather_src<<<srcb, 128, 0, st>>>(G, ln, grad_wavelet, it);
        if (it == 0) {
            if (il) illum<<<cb, 256, 0, st>>>(G, rx, rn, rp, ln, nullptr, w.ir);
            SWEEP_LAUNCH_CHECK();
            break;
        }
        recon<M><<<grid, block, 0, st>>>(G, rn, rp, rx, ln, w.g);
        if (G.ns > 0) strips<<<sb, 256, 0, st>>>(G, rx, const_cast<float*>(tp) + (long long)(it - 1) * slot_floats(pl), 1);
        if (G.nsrc > 0) inject_src<<<srcb, 128, 0, st>>>(G, rx, it, -1.f, 1);
        if (G.ns > 0) strip_image<<<sb, 256, 0, st>>>(G, rx, rn, rp, ln, w.g);
        if (il) illum<<<cb, 256, 0, st>>>(G, rx, rn, rp, ln, w.is, w.ir);
        if (G.nsrc > 0) inject_src<<<srcb, 128, 0, st>>>(G, rx, it, 1.f, 0);
        SWEEP_LAUNCH_CHECK();
        { float* t = rp; rp = rn; rn = rx; rx = t; }
    }
    const int per_shot = G.vps != 0;
    finalize<<<cb, 256, 0, st>>>(G, w.g, per_shot, grad_vp);
    if (illum_src) finalize<<<cb, 256, 0, st>>>(G, w.is, per_shot, illum_src);
    if (illum_rec) finalize<<<cb, 256, 0, st>>>(G, w.ir, per_shot, illum_rec);
    SWEEP_LAUNCH_CHECK();
}

#define SWEEP_AORD_DISPATCH(M_, CALL)                                              \
    switch (M_) {                                                                  \
    case 1: CALL(1); break;                                                        \
    case 2: CALL(2); break;                                                        \
    case 3: CALL(3); break;                                                        \
    case 4: CALL(4); break;                                                        \
    case 5: CALL(5); break;                                                        \
    case 6: CALL(6); break;                                                        \
    default: CALL(7); break;                                                       \
    }

void forward(const sweep_acoustic_desc* d, int mem_mode, int, float* record, void* tape, void* ws, int64_t ws_bytes,
             cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
#define SWEEP_AORD_FWD(m) forward_m<m>(pl, record, tape, ws, ws_bytes, st)
    SWEEP_AORD_DISPATCH(d->M, SWEEP_AORD_FWD)
#undef SWEEP_AORD_FWD
}

void backward(const sweep_acoustic_desc* d, int mem_mode, int, const float* adj, const void* tape, float* grad_vp,
              float* grad_wavelet, float* illum_src, float* illum_rec, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
#define SWEEP_AORD_BWD(m) backward_m<m>(pl, adj, tape, grad_vp, grad_wavelet, illum_src, illum_rec, ws, ws_bytes, st)
    SWEEP_AORD_DISPATCH(d->M, SWEEP_AORD_BWD)
#undef SWEEP_AORD_BWD
}

}  // namespace aord
}  // namespace sweep
