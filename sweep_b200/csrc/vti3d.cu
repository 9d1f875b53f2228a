// vti3d.cu -- 3-D first-order acoustic VTI (Duveneck et al. 2008: vx, vy, vz
// and the horizontal / vertical stresses sH = s11 = s22, sV = s33 on a
// staggered grid) forward and boundary-saving adjoint with vp / epsilon /
// delta / rho gradients, at every even spatial order 2..14, for sm_100a.
//
// Restates the reference's compiled path (src/sweep/csrc/cuda/equations/
// acoustic_vti_1st_3d/kernels.cuh, forward.cu, backward.cu;
// common/derived_models.cu:40-53 for the stiffness):
//   forward, per step: velocity step (D+ of sH along x and y, of sV along z;
//     CPML memories m_sHx / m_sHy / m_sVz on the half-cell profiles outside
//     the physical box), stress step (D- of vx / vy / vz, memories m_vxx /
//     m_vyy / m_vzz; dh = dvx/dx + dvy/dy, sH += dt (c11 dh + c13 dvz/dz),
//     sV += dt (c13 dh + c33 dvz/dz)), the source into every source field,
//     the five fields' boundary bands, receivers;
//   reverse, per step it = nt - 1 .. 1: the residuals (unsigned), the source
//     taken back out, stress reconstruction on the box minus one cell, stress
//     bands, adjoint half-step A (p = (ph, ph, pv), ph = c11 lsH + c13 lsV,
//     pv = c13 lsH + c33 lsV, through the stress step's transposed CPML;
//     lambda_v += -dt D+ p), the gradient (forward velocities at the end of
//     the step, stresses at its start), half-step B (q = lambda_v / rho
//     through the velocity step's transposed CPML; lambda_sH += -dt (D-x qx +
//     D-y qy), lambda_sV += -dt D-z qz), velocity reconstruction, velocity
//     bands.
// One thread per cell on 32 x 4 x 2 (x, y, z) blocks, two z planes of a shot
// per grid row; stencils through the read-only path.
// Layout: every field and memory (B, nz, ny, nx), x fastest; models and the
// derived stiffness (B|1, nz, ny, nx).  Boundary bands: per face a band M + 1
// wide from M cells outside the box, spanning the box along the other two
// axes (boundary/strip.cuh:136-175), each cell kept once; tape slot of a step
// (B, 5, ns) after the final state (B, 5, S) at the end.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "vti3d.cuh"

namespace sweep {
namespace vti3 {

constexpr int MAXM = 7;
constexpr int NF = 5;
enum { VX = 0, VY = 1, VZ = 2, SH = 3, SV = 4 };
enum { M_SHX, M_SHY, M_SVZ, M_VXX, M_VYY, M_VZZ, NMEM };

struct Geo {
    int B, nz, ny, nx, nt, M;
    long long S;                    // cells per shot
    int pad[6];                     // z_lo, z_hi, y_lo, y_hi, x_lo, x_hi
    int z0, z1, y0, y1, x0, x1;     // physical box
    float dt, dz, dy, dx;
    float c[MAXM + 1];              // staggered weights c[1..M]
    const float *az, *bz, *azh, *bzh, *ay, *by, *ayh, *byh, *ax, *bx, *axh, *bxh;
    const float *vp, *eps, *dlt, *rho;   // the caller's models
    const float *c11, *c33, *c13, *irho; // derived per model copy
    long long ms;                   // model stride between shots (0 or S)
    int nsrc, nrec, nsf, nrf;
    int sf[NF], rf[NF];
    const int *src, *rec;           // (B, n, 3) runtime (x, y, z)
    const float* wavelet;           // (B, nsrc, nt)
    const int* cells;               // band cells of a shot grid, each once
    int ns;
};

struct Fields {
    float* f[NMEM];
};

__device__ __forceinline__ float ld(const float* p) { return __ldg(p); }

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

// the thread's cell (32 x 4 x 2 blocks: two z planes of a shot per grid row);
// o = the shot's offset, i = the cell within the shot
__device__ __forceinline__ bool cell3(const Geo& G, int& b, int& iz, int& iy, int& ix, long long& o, long long& i)
{
    const int zb = (G.nz + 1) >> 1;
    ix = blockIdx.x * 32 + threadIdx.x;
    iy = blockIdx.y * 4 + threadIdx.y;
    b = blockIdx.z / zb;
    iz = (blockIdx.z - b * zb) * 2 + threadIdx.z;
    o = b * G.S;
    i = ((long long)iz * G.ny + iy) * G.nx + ix;
    return ix < G.nx && iy < G.ny && iz < G.nz;
}
__device__ __forceinline__ bool core(const Geo& G, int ix, int iy, int iz)
{
    return ix >= G.M && ix < G.nx - G.M && iy >= G.M && iy < G.ny - G.M && iz >= G.M && iz < G.nz - G.M;
}
// outside the physical box (PML pad plus the stencil halo) on any axis
__device__ __forceinline__ bool in_pml(const Geo& G, int ix, int iy, int iz)
{
    return ix < G.x0 || ix >= G.x1 || iy < G.y0 || iy >= G.y1 || iz < G.z0 || iz >= G.z1;
}
// the reverse box: the physical box minus one cell per face
__device__ __forceinline__ bool in_rev(const Geo& G, int ix, int iy, int iz)
{
    return ix > G.x0 && ix < G.x1 - 1 && iy > G.y0 && iy < G.y1 - 1 && iz > G.z0 && iz < G.z1 - 1;
}

// stiffness per model copy, each operation rounded once (reference
// derived_models.cu:40-53)
__global__ void prep(const float* __restrict__ vp, const float* __restrict__ eps, const float* __restrict__ dlt,
                     const float* __restrict__ rho, long long n, float* c11, float* c33, float* c13, float* irho)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const float v = vp[k], r = rho[k];
        const float rv2 = __fmul_rn(r, __fmul_rn(v, v));
        c33[k] = rv2;
        c11[k] = __fmul_rn(rv2, __fadd_rn(1.0f, __fmul_rn(2.0f, eps[k])));
        c13[k] = __fmul_rn(rv2, __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(2.0f, dlt[k]))));
        irho[k] = __fdiv_rn(1.0f, r);
    }
}

// velocity step (reference kernels.cuh:150-210)
template <int M>
__global__ void __launch_bounds__(256) vel(const Geo G, Fields F, Fields W)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || !core(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx;
    float dsx = dplus<M>(F.f[SH] + o, i, 1, G, 1.f / G.dx);
    float dsy = dplus<M>(F.f[SH] + o, i, sy, G, 1.f / G.dy);
    float dsz = dplus<M>(F.f[SV] + o, i, sz, G, 1.f / G.dz);
    if (in_pml(G, ix, iy, iz)) {
        float* mx = W.f[M_SHX] + o;
        float* my = W.f[M_SHY] + o;
        float* mz = W.f[M_SVZ] + o;
        mx[i] = G.axh[ix] * mx[i] + G.bxh[ix] * dsx;
        dsx = dsx + mx[i];
        my[i] = G.ayh[iy] * my[i] + G.byh[iy] * dsy;
        dsy = dsy + my[i];
        mz[i] = G.azh[iz] * mz[i] + G.bzh[iz] * dsz;
        dsz = dsz + mz[i];
    }
    const float k = G.dt * G.irho[b * G.ms + i];
    F.f[VX][o + i] = F.f[VX][o + i] + k * dsx;
    F.f[VY][o + i] = F.f[VY][o + i] + k * dsy;
    F.f[VZ][o + i] = F.f[VZ][o + i] + k * dsz;
}

// stress step (reference kernels.cuh:275-333)
template <int M>
__global__ void __launch_bounds__(256) str(const Geo G, Fields F, Fields W)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || !core(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx, mi = b * G.ms + i;
    float dvx = dminus<M>(F.f[VX] + o, i, 1, G, 1.f / G.dx);
    float dvy = dminus<M>(F.f[VY] + o, i, sy, G, 1.f / G.dy);
    float dvz = dminus<M>(F.f[VZ] + o, i, sz, G, 1.f / G.dz);
    if (in_pml(G, ix, iy, iz)) {
        float* mx = W.f[M_VXX] + o;
        float* my = W.f[M_VYY] + o;
        float* mz = W.f[M_VZZ] + o;
        mx[i] = G.ax[ix] * mx[i] + G.bx[ix] * dvx;
        dvx = dvx + mx[i];
        my[i] = G.ay[iy] * my[i] + G.by[iy] * dvy;
        dvy = dvy + my[i];
        mz[i] = G.az[iz] * mz[i] + G.bz[iz] * dvz;
        dvz = dvz + mz[i];
    }
    const float dh = dvx + dvy;
    const float c11 = G.c11[mi], c33 = G.c33[mi], c13 = G.c13[mi];
    F.f[SH][o + i] = F.f[SH][o + i] + G.dt * (c11 * dh + c13 * dvz);
    F.f[SV][o + i] = F.f[SV][o + i] + G.dt * (c13 * dh + c33 * dvz);
}

__device__ __forceinline__ long long loc(const Geo& G, const int* l)
{
    if (l[0] < 0 || l[0] >= G.nx || l[1] < 0 || l[1] >= G.ny || l[2] < 0 || l[2] >= G.nz) return -1;
    return ((long long)l[2] * G.ny + l[1]) * G.nx + l[0];
}

// the wavelet of step it, times sign, into every source field
__global__ void inject(const Geo G, Fields F, int it, float sign)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nsrc) return;
    const int b = e / G.nsrc;
    const long long c = loc(G, G.src + 3LL * e);
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
    const long long c = loc(G, G.rec + 3LL * e);
    if (c < 0) return;
    float* out = record + (((long long)b * G.nt + it) * G.nrec + r) * G.nrf;
    for (int k = 0; k < G.nrf; ++k) out[k] = F.f[G.rf[k]][b * G.S + c];
}

// the residuals of step it into the adjoint fields, unsigned
__global__ void residual(const Geo G, Fields A, const float* __restrict__ adj, int it)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const long long c = loc(G, G.rec + 3LL * e);
    if (c < 0) return;
    const float* res = adj + (((long long)b * G.nt + it) * G.nrec + r) * G.nrf;
    for (int k = 0; k < G.nrf; ++k) atomicAdd(A.f[G.rf[k]] + b * G.S + c, res[k]);
}

// band save (restore = 0) of fields [f0, f1) into one step slot (B, 5, ns), or restore
__global__ void bands(const Geo G, Fields F, float* slot, int f0, int f1, int restore)
{
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long b = e / G.ns, k = e - b * G.ns;
        const long long i = b * G.S + G.cells[k];
        for (int f = f0; f < f1; ++f) {
            float* t = slot + (b * NF + f) * G.ns + k;
            if (restore) F.f[f][i] = *t;
            else *t = F.f[f][i];
        }
    }
}

// stress reconstruction (reference kernels.cuh:462-490)
template <int M>
__global__ void __launch_bounds__(256) srev(const Geo G, Fields F)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || !in_rev(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx, mi = b * G.ms + i;
    const float dvx = dminus<M>(F.f[VX] + o, i, 1, G, 1.f / G.dx);
    const float dvy = dminus<M>(F.f[VY] + o, i, sy, G, 1.f / G.dy);
    const float dvz = dminus<M>(F.f[VZ] + o, i, sz, G, 1.f / G.dz);
    const float dh = dvx + dvy;
    const float c11 = G.c11[mi], c33 = G.c33[mi], c13 = G.c13[mi];
    F.f[SH][o + i] = F.f[SH][o + i] - G.dt * (c11 * dh + c13 * dvz);
    F.f[SV][o + i] = F.f[SV][o + i] - G.dt * (c13 * dh + c33 * dvz);
}

// velocity reconstruction (reference kernels.cuh:400-425)
template <int M>
__global__ void __launch_bounds__(256) vrev(const Geo G, Fields F)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || !in_rev(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx;
    const float dsx = dplus<M>(F.f[SH] + o, i, 1, G, 1.f / G.dx);
    const float dsy = dplus<M>(F.f[SH] + o, i, sy, G, 1.f / G.dy);
    const float dsz = dplus<M>(F.f[SV] + o, i, sz, G, 1.f / G.dz);
    const float k = G.dt * G.irho[b * G.ms + i];
    F.f[VX][o + i] = F.f[VX][o + i] - k * dsx;
    F.f[VY][o + i] = F.f[VY][o + i] - k * dsy;
    F.f[VZ][o + i] = F.f[VZ][o + i] - k * dsz;
}

struct Scratch {
    float* s[3];
};

// adjoint half-step A, pre-multiply on every cell (kernels.cuh:606-645):
// p = (ph, ph, pv) with the stress step's CPML transposed where that step
// keeps memories (core cells outside the box)
__global__ void __launch_bounds__(256) premA(const Geo G, Fields A, Fields W, Scratch P)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i)) return;
    const long long k = o + i, mi = b * G.ms + i;
    const float lsh = A.f[SH][k], lsv = A.f[SV][k];
    const float ph = G.c11[mi] * lsh + G.c13[mi] * lsv;
    const float pv = G.c13[mi] * lsh + G.c33[mi] * lsv;
    float p_x = ph, p_y = ph, p_z = pv;
    if (core(G, ix, iy, iz) && in_pml(G, ix, iy, iz)) {
        const float tx = W.f[M_VXX][k] + p_x, ty = W.f[M_VYY][k] + p_y, tz = W.f[M_VZZ][k] + p_z;
        p_x += G.bx[ix] * tx;
        p_y += G.by[iy] * ty;
        p_z += G.bz[iz] * tz;
        W.f[M_VXX][k] = G.ax[ix] * tx;
        W.f[M_VYY][k] = G.ay[iy] * ty;
        W.f[M_VZZ][k] = G.az[iz] * tz;
    }
    P.s[0][k] = p_x;
    P.s[1][k] = p_y;
    P.s[2][k] = p_z;
}

// half-step A, apply on the core: lambda_v += -dt D+(p) (kernels.cuh:760-775)
template <int M>
__global__ void __launch_bounds__(256) appA(const Geo G, Fields A, Scratch P)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || !core(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx;
    const float dpx = dplus<M>(P.s[0] + o, i, 1, G, 1.f / G.dx);
    const float dpy = dplus<M>(P.s[1] + o, i, sy, G, 1.f / G.dy);
    const float dpz = dplus<M>(P.s[2] + o, i, sz, G, 1.f / G.dz);
    A.f[VX][o + i] += -G.dt * dpx;
    A.f[VY][o + i] += -G.dt * dpy;
    A.f[VZ][o + i] += -G.dt * dpz;
}

// half-step B, pre-multiply on every cell (kernels.cuh:690-725):
// q = inv_rho lambda_v with the velocity step's transposed CPML
__global__ void __launch_bounds__(256) premB(const Geo G, Fields A, Fields W, Scratch Q)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i)) return;
    const long long k = o + i;
    const float ir = G.irho[b * G.ms + i];
    float q_x = ir * A.f[VX][k], q_y = ir * A.f[VY][k], q_z = ir * A.f[VZ][k];
    if (core(G, ix, iy, iz) && in_pml(G, ix, iy, iz)) {
        const float tx = W.f[M_SHX][k] + q_x, ty = W.f[M_SHY][k] + q_y, tz = W.f[M_SVZ][k] + q_z;
        q_x += G.bxh[ix] * tx;
        q_y += G.byh[iy] * ty;
        q_z += G.bzh[iz] * tz;
        W.f[M_SHX][k] = G.axh[ix] * tx;
        W.f[M_SHY][k] = G.ayh[iy] * ty;
        W.f[M_SVZ][k] = G.azh[iz] * tz;
    }
    Q.s[0][k] = q_x;
    Q.s[1][k] = q_y;
    Q.s[2][k] = q_z;
}

// half-step B, apply on the core (kernels.cuh:800-815):
// lambda_sH += -dt (D-x qx + D-y qy), lambda_sV += -dt D-z qz
template <int M>
__global__ void __launch_bounds__(256) appB(const Geo G, Fields A, Scratch Q)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || !core(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx;
    const float dqx = dminus<M>(Q.s[0] + o, i, 1, G, 1.f / G.dx);
    const float dqy = dminus<M>(Q.s[1] + o, i, sy, G, 1.f / G.dy);
    const float dqz = dminus<M>(Q.s[2] + o, i, sz, G, 1.f / G.dz);
    A.f[SH][o + i] += -G.dt * (dqx + dqy);
    A.f[SV][o + i] += -G.dt * dqz;
}

struct Grads {
    float *vp, *eps, *dlt, *rho;    // per-shot slots (B, S)
};

// the gradient of one step on the physical box (kernels.cuh:940-1000): the
// stiffness gradients from the forward velocities at the end of the step, the
// 1 / rho gradient from the stresses at its start, chained to the models
template <int M>
__global__ void __launch_bounds__(256) grad(const Geo G, Fields F, Fields A, Grads g)
{
    int b, iz, iy, ix;
    long long o, i;
    if (!cell3(G, b, iz, iy, ix, o, i) || in_pml(G, ix, iy, iz) || !core(G, ix, iy, iz)) return;
    const long long sy = G.nx, sz = (long long)G.ny * G.nx, k = o + i, mi = b * G.ms + i;
    const float dvx = dminus<M>(F.f[VX] + o, i, 1, G, 1.f / G.dx);
    const float dvy = dminus<M>(F.f[VY] + o, i, sy, G, 1.f / G.dy);
    const float dvz = dminus<M>(F.f[VZ] + o, i, sz, G, 1.f / G.dz);
    const float dsx = dplus<M>(F.f[SH] + o, i, 1, G, 1.f / G.dx);
    const float dsy = dplus<M>(F.f[SH] + o, i, sy, G, 1.f / G.dy);
    const float dsz = dplus<M>(F.f[SV] + o, i, sz, G, 1.f / G.dz);
    const float lsh = A.f[SH][k], lsv = A.f[SV][k];
    const float lvx = A.f[VX][k], lvy = A.f[VY][k], lvz = A.f[VZ][k];
    const float dh = dvx + dvy;
    const float dt = G.dt;
    const float g11 = dt * lsh * dh;
    const float g33 = dt * lsv * dvz;
    const float g13 = dt * (lsh * dvz + lsv * dh);
    const float gir = dt * (lvx * dsx + lvy * dsy + lvz * dsz);
    const float v = G.vp[mi], e = G.eps[mi], d = G.dlt[mi], r = G.rho[mi];
    const float ope = 1.f + 2.f * e, opd = 1.f + 2.f * d;
    const float sd = sqrtf(opd);
    const float v2 = v * v;
    const float common = g11 * ope + g33 + g13 * sd;
    g.vp[k] += 2.f * r * v * common;
    g.eps[k] += g11 * 2.f * r * v2;
    g.dlt[k] += g13 * r * v2 / fmaxf(sd, 1e-12f);
    g.rho[k] += v2 * common - gir / (r * r);
}

// per-shot slots -> out on the physical box, zero elsewhere: (B, S) for
// per-shot models, else the sum over shots in shot order
__global__ void finalize(const Geo G, const float* __restrict__ slots, float* out)
{
    const bool per_shot = G.ms != 0;
    const long long n = per_shot ? (long long)G.B * G.S : G.S;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long c = k % G.S;
        const int ix = (int)(c % G.nx), iy = (int)((c / G.nx) % G.ny), iz = (int)(c / ((long long)G.nx * G.ny));
        float v = 0.f;
        if (!in_pml(G, ix, iy, iz)) {
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

static Plan make_plan(const sweep_vti3d_desc* d, int mem_mode)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->M >= 1 && d->M <= MAXM, "vti3d: spatial orders 2 to %d are built (got order %d)", 2 * MAXM,
                  2 * d->M);
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY,
                  "vti3d: boundary saving with fp32 strips in device memory is built (mem_mode %d)", mem_mode);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1 && d->nz >= 1 && (long long)d->B * d->nz <= 65535,
                  "vti3d: B * nz must be 1 to 65535 (one grid row per z plane and shot) and nt >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "vti3d: negative source/receiver count");
    SWEEP_REQUIRE(d->nsrc_fields >= 1 && d->nsrc_fields <= NF, "vti3d: 1 to 5 source fields");
    SWEEP_REQUIRE(d->nrec_fields >= 1 && d->nrec_fields <= NF, "vti3d: 1 to 5 receiver fields");
    for (int k = 0; k < d->nsrc_fields; ++k) {
        SWEEP_REQUIRE(d->src_fields[k] >= 0 && d->src_fields[k] < NF, "vti3d: bad source field %d", d->src_fields[k]);
        for (int j = 0; j < k; ++j)
            SWEEP_REQUIRE(d->src_fields[j] != d->src_fields[k], "vti3d: source field %d repeated", d->src_fields[k]);
    }
    for (int k = 0; k < d->nrec_fields; ++k)
        SWEEP_REQUIRE(d->rec_fields[k] >= 0 && d->rec_fields[k] < NF, "vti3d: bad receiver field %d",
                      d->rec_fields[k]);
    for (int f = 0; f < 6; ++f)
        SWEEP_REQUIRE(d->pad[f] >= 1, "vti3d: every face needs a PML pad >= 1 (face %d has %d)", f, d->pad[f]);
    Plan pl{};
    Geo& G = pl.G;
    const int M = d->M;
    G.B = d->B; G.nz = d->nz; G.ny = d->ny; G.nx = d->nx; G.nt = d->nt; G.M = M;
    G.S = (long long)d->nz * d->ny * d->nx;
    SWEEP_REQUIRE(G.S < (1LL << 31), "vti3d: one shot's grid must hold < 2^31 cells");
    for (int f = 0; f < 6; ++f) G.pad[f] = d->pad[f];
    G.z0 = G.pad[0] + M; G.z1 = G.nz - G.pad[1] - M;
    G.y0 = G.pad[2] + M; G.y1 = G.ny - G.pad[3] - M;
    G.x0 = G.pad[4] + M; G.x1 = G.nx - G.pad[5] - M;
    SWEEP_REQUIRE(G.z1 - G.z0 >= 2 && G.y1 - G.y0 >= 2 && G.x1 - G.x0 >= 2,
                  "vti3d: the physical box must be at least 2 cells per axis");
    G.dt = d->dt; G.dz = d->dz; G.dy = d->dy; G.dx = d->dx;
    for (int k = 0; k <= MAXM; ++k) G.c[k] = 0.f;
    staggered_weights(M, G.c);
    G.az = d->az; G.bz = d->bz; G.azh = d->azh; G.bzh = d->bzh;
    G.ay = d->ay; G.by = d->by; G.ayh = d->ayh; G.byh = d->byh;
    G.ax = d->ax; G.bx = d->bx; G.axh = d->axh; G.bxh = d->bxh;
    G.vp = d->vp; G.eps = d->epsilon; G.dlt = d->delta; G.rho = d->rho;
    const bool per_shot = d->model_stride != 0;
    SWEEP_REQUIRE(!per_shot || d->model_stride == G.S, "vti3d: model_stride must be 0 or nz * ny * nx");
    G.ms = per_shot ? G.S : 0;
    pl.nm = per_shot ? G.B : 1;
    G.nsrc = d->nsrc; G.nrec = d->nrec; G.nsf = d->nsrc_fields; G.nrf = d->nrec_fields;
    for (int k = 0; k < NF; ++k) { G.sf[k] = d->src_fields[k]; G.rf[k] = d->rec_fields[k]; }
    G.src = d->src_loc; G.rec = d->rec_loc; G.wavelet = d->wavelet;
    // band cells: per face a band M + 1 wide from M cells outside the box,
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

struct Ws {
    float *c11, *c33, *c13, *irho;
    int* cells;
    float* f[NF];
    float* m[NMEM];                 // forward memories / adjoint memories
    float* a[NF];
    float* s[3];                    // pre-multiply scratch
    float *gvp, *geps, *gdlt, *grho;
    char *zero0, *zero1;
};

static void carve(Carve& c, const Plan& pl, bool rev, Ws& w)
{
    const Geo& G = pl.G;
    const long long n = (long long)G.B * G.S, mc = (long long)pl.nm * G.S;
    w = Ws{};
    w.c11 = c.take<float>(mc); w.c33 = c.take<float>(mc); w.c13 = c.take<float>(mc); w.irho = c.take<float>(mc);
    w.cells = c.take<int>(std::max(G.ns, 1));
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    for (int k = 0; k < NF; ++k) w.f[k] = c.take<float>(n);
    for (int k = 0; k < NMEM; ++k) w.m[k] = c.take<float>(n);
    if (rev) {
        for (int k = 0; k < NF; ++k) w.a[k] = c.take<float>(n);
        w.gvp = c.take<float>(n); w.geps = c.take<float>(n); w.gdlt = c.take<float>(n); w.grho = c.take<float>(n);
    }
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
    if (rev)
        for (int k = 0; k < 3; ++k) w.s[k] = c.take<float>(n);
}

static long long slot_floats(const Plan& pl) { return (long long)pl.G.B * NF * pl.G.ns; }

void sizes(const sweep_vti3d_desc* d, int mem_mode, int, int64_t* ws_bytes, int64_t* tape_bytes)
{
    const Plan pl = make_plan(d, mem_mode);
    Carve f(nullptr), r(nullptr);
    Ws w;
    carve(f, pl, false, w);
    carve(r, pl, true, w);
    *ws_bytes = std::max(f.off, r.off);
    *tape_bytes = ((long long)pl.G.nt * slot_floats(pl) + (long long)NF * pl.G.B * pl.G.S) * 4;
}

static void setup(const sweep_vti3d_desc* d, Plan& pl, const Ws& w, cudaStream_t st)
{
    Geo& G = pl.G;
    G.c11 = w.c11; G.c33 = w.c33; G.c13 = w.c13; G.irho = w.irho; G.cells = w.cells;
    const long long mc = (long long)pl.nm * G.S;
    prep<<<(unsigned)std::min<long long>((mc + 255) / 256, 4096), 256, 0, st>>>(d->vp, d->epsilon, d->delta, d->rho,
                                                                                 mc, w.c11, w.c33, w.c13, w.irho);
    SWEEP_LAUNCH_CHECK();
    if (G.ns > 0)
        SWEEP_CUDA(cudaMemcpyAsync(w.cells, pl.cells.data(), sizeof(int) * G.ns, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
}

static dim3 grid_of(const Geo& G) { return dim3((G.nx + 31) / 32, (G.ny + 3) / 4, (unsigned)(G.B * ((G.nz + 1) / 2))); }
static unsigned blocks(long long n) { return (unsigned)std::max<long long>(std::min<long long>((n + 255) / 256, 8192), 1); }

template <int M>
static void forward_m(const sweep_vti3d_desc* d, Plan& pl, float* record, void* tape, void* ws, int64_t ws_bytes,
                      cudaStream_t st)
{
    Carve c(ws);
    Ws w;
    carve(c, pl, false, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "vti3d forward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    setup(d, pl, w, st);
    const Geo& G = pl.G;
    if (record && G.nrec > 0)
        SWEEP_CUDA(cudaMemsetAsync(record, 0, sizeof(float) * (size_t)G.B * G.nt * G.nrec * G.nrf, st));
    Fields F{}, W{};
    for (int k = 0; k < NF; ++k) F.f[k] = w.f[k];
    for (int k = 0; k < NMEM; ++k) W.f[k] = w.m[k];
    float* tp = static_cast<float*>(tape);
    const dim3 grid = grid_of(G), block(32, 4, 2);
    for (int it = 0; it < G.nt; ++it) {
        vel<M><<<grid, block, 0, st>>>(G, F, W);
        str<M><<<grid, block, 0, st>>>(G, F, W);
        if (G.nsrc > 0) inject<<<(G.B * G.nsrc + 127) / 128, 128, 0, st>>>(G, F, it, 1.f);
        if (tp) bands<<<blocks((long long)G.B * G.ns), 256, 0, st>>>(G, F, tp + it * slot_floats(pl), 0, NF, 0);
        if (record && G.nrec > 0) gather<<<(G.B * G.nrec + 127) / 128, 128, 0, st>>>(G, F, record, it);
        SWEEP_LAUNCH_CHECK();
    }
    if (tp) {
        float* last = tp + (long long)G.nt * slot_floats(pl);
        for (int b = 0; b < G.B; ++b)
            for (int f = 0; f < NF; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(last + ((long long)b * NF + f) * G.S, w.f[f] + b * G.S,
                                           sizeof(float) * G.S, cudaMemcpyDeviceToDevice, st));
    }
}

template <int M>
static void backward_m(const sweep_vti3d_desc* d, Plan& pl, const float* adj, const void* tape, float* const out[4],
                       void* ws, int64_t ws_bytes, cudaStream_t st)
{
    SWEEP_REQUIRE(tape != nullptr, "vti3d backward: the forward's tape is required");
    Carve c(ws);
    Ws w;
    carve(c, pl, true, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "vti3d backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    setup(d, pl, w, st);
    const Geo& G = pl.G;
    const float* tp = static_cast<const float*>(tape);
    const float* last = tp + (long long)G.nt * slot_floats(pl);
    for (int b = 0; b < G.B; ++b)
        for (int f = 0; f < NF; ++f)
            SWEEP_CUDA(cudaMemcpyAsync(w.f[f] + b * G.S, last + ((long long)b * NF + f) * G.S, sizeof(float) * G.S,
                                       cudaMemcpyDeviceToDevice, st));
    Fields F{}, A{}, W{};
    for (int k = 0; k < NF; ++k) { F.f[k] = w.f[k]; A.f[k] = w.a[k]; }
    for (int k = 0; k < NMEM; ++k) W.f[k] = w.m[k];
    const Scratch S{{w.s[0], w.s[1], w.s[2]}};
    const Grads g{w.gvp, w.geps, w.gdlt, w.grho};
    const dim3 grid = grid_of(G), block(32, 4, 2);
    const unsigned srcb = (unsigned)(G.B * G.nsrc + 127) / 128, recb = (unsigned)(G.B * G.nrec + 127) / 128;
    const unsigned bb = blocks((long long)G.B * G.ns);
    for (int it = G.nt - 1; it >= 1; --it) {
        float* prev = const_cast<float*>(tp) + (long long)(it - 1) * slot_floats(pl);
        if (G.nrec > 0) residual<<<recb, 128, 0, st>>>(G, A, adj, it);
        if (G.nsrc > 0) inject<<<srcb, 128, 0, st>>>(G, F, it, -1.f);
        srev<M><<<grid, block, 0, st>>>(G, F);
        bands<<<bb, 256, 0, st>>>(G, F, prev, SH, NF, 1);
        premA<<<grid, block, 0, st>>>(G, A, W, S);
        appA<M><<<grid, block, 0, st>>>(G, A, S);
        grad<M><<<grid, block, 0, st>>>(G, F, A, g);
        premB<<<grid, block, 0, st>>>(G, A, W, S);
        appB<M><<<grid, block, 0, st>>>(G, A, S);
        vrev<M><<<grid, block, 0, st>>>(G, F);
        bands<<<bb, 256, 0, st>>>(G, F, prev, VX, SH, 1);
        SWEEP_LAUNCH_CHECK();
    }
    const unsigned fb = blocks((long long)pl.nm * G.S);
    const float* slots[4] = {w.gvp, w.geps, w.gdlt, w.grho};
    for (int k = 0; k < 4; ++k) finalize<<<fb, 256, 0, st>>>(G, slots[k], out[k]);
    SWEEP_LAUNCH_CHECK();
}

#define SWEEP_VTI3_DISPATCH(M_, CALL) \
    switch (M_) {                     \
    case 1: CALL(1); break;           \
    case 2: CALL(2); break;           \
    case 3: CALL(3); break;           \
    case 4: CALL(4); break;           \
    case 5: CALL(5); break;           \
    case 6: CALL(6); break;           \
    default: CALL(7); break;          \
    }

void forward(const sweep_vti3d_desc* d, int mem_mode, int, float* record, void* tape, void* ws, int64_t ws_bytes,
             cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
#define SWEEP_VTI3_FWD(m) forward_m<m>(d, pl, record, tape, ws, ws_bytes, st)
    SWEEP_VTI3_DISPATCH(d->M, SWEEP_VTI3_FWD)
#undef SWEEP_VTI3_FWD
}

void backward(const sweep_vti3d_desc* d, int mem_mode, int, const float* adj, const void* tape, float* grad_vp,
              float* grad_eps, float* grad_dlt, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
    float* const out[4] = {grad_vp, grad_eps, grad_dlt, grad_rho};
#define SWEEP_VTI3_BWD(m) backward_m<m>(d, pl, adj, tape, out, ws, ws_bytes, st)
    SWEEP_VTI3_DISPATCH(d->M, SWEEP_VTI3_BWD)
#undef SWEEP_VTI3_BWD
}

}  // namespace vti3
}  // namespace sweep
