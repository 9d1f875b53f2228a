// vti2d.cu -- 2-D first-order acoustic VTI (Duveneck et al. 2008: vx, vz and
// the horizontal / vertical stresses sH, sV on a staggered grid) forward and
// boundary-saving adjoint with vp / epsilon / delta / rho gradients, at every
// even spatial order 2..14, for sm_100a.
//
// Restates the reference's compiled path (src/sweep/csrc/cuda/equations/
// acoustic_vti_1st_2d/kernels.cuh, forward.cu, backward.cu:469-742;
// common/derived_models.cu:40-53 for the stiffness):
//   forward, per step: velocity step (D+ of sH / sV, CPML memories on the
//     half-cell profiles outside the physical box), stress step (D- of
//     vx / vz, integer profiles), the source into every source field, the
//     four fields' bands (width M + 1 from M cells outside the box), receivers;
//   reverse, per step it = nt - 1 .. 1: the residuals (unsigned), the source
//     taken back out, stress reconstruction on the box minus one cell, stress
//     bands, adjoint half-step A (p = C lambda_s with the stress step's
//     transposed CPML, lambda_v += -dt D+ p), the gradient (forward
//     velocities at the end of the step, stresses at its start), half-step B
//     (q = lambda_v / rho with the velocity step's transposed CPML,
//     lambda_s += -dt D- q), velocity reconstruction, velocity bands.
// One thread per cell on 32 x 8 tiles, shots on the grid's last axis,
// stencils through the read-only path.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "vti2d.cuh"

namespace sweep {
namespace vti {

constexpr int MAXM = 7;
enum { VX = 0, VZ = 1, SH = 2, SV = 3 };
enum { M_SHX, M_SVZ, M_VXX, M_VZZ, NMEM };

struct Geo {
    int B, nz, nx, nt, M;
    long long S;                    // cells per shot
    int pad[4];                     // z_lo, z_hi, x_lo, x_hi
    int z0, z1, x0, x1;             // physical box
    float dt, dz, dx;
    float c[MAXM + 1];              // staggered weights c[1..M]
    const float *az, *bz, *azh, *bzh, *ax, *bx, *axh, *bxh;
    const float *vp, *eps, *dlt, *rho;   // the caller's models
    const float *c11, *c33, *c13, *irho; // derived per model copy
    long long ms;                   // model stride between shots (0 or S)
    int nsrc, nrec, nsf, nrf;
    int sf[4], rf[4];
    const int *src, *rec;           // (B, n, 2) runtime (x, z)
    const float* wavelet;           // (B, nsrc, nt)
    const int* cells;               // band cells of a shot grid (cells of two bands listed twice)
    int ns;
};

struct Fields {
    float* f[4];
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
// outside the physical box (PML pad plus the stencil halo)
__device__ __forceinline__ bool in_pml(const Geo& G, int ix, int iz)
{
    return ix < G.pad[2] + G.M || ix >= G.nx - G.pad[3] - G.M || iz < G.pad[0] + G.M || iz >= G.nz - G.pad[1] - G.M;
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

// velocity step (reference kernels.cuh:104-163)
template <int M>
__global__ void __launch_bounds__(256) vel(const Geo G, Fields F, Fields W)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    float dsH = dplus<M>(F.f[SH] + o, i, 1, G, 1.f / G.dx);
    float dsV = dplus<M>(F.f[SV] + o, i, G.nx, G, 1.f / G.dz);
    if (in_pml(G, ix, iz)) {
        float* mx = W.f[M_SHX] + o;
        float* mz = W.f[M_SVZ] + o;
        mx[i] = G.axh[ix] * mx[i] + G.bxh[ix] * dsH;
        dsH = dsH + mx[i];
        mz[i] = G.azh[iz] * mz[i] + G.bzh[iz] * dsV;
        dsV = dsV + mz[i];
    }
    const float k = G.dt * G.irho[b * G.ms + i];
    F.f[VX][o + i] = F.f[VX][o + i] + k * dsH;
    F.f[VZ][o + i] = F.f[VZ][o + i] + k * dsV;
}

// stress step (reference kernels.cuh:209-272)
template <int M>
__global__ void __launch_bounds__(256) str(const Geo G, Fields F, Fields W)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, mi = b * G.ms + i;
    float dvx = dminus<M>(F.f[VX] + o, i, 1, G, 1.f / G.dx);
    float dvz = dminus<M>(F.f[VZ] + o, i, G.nx, G, 1.f / G.dz);
    if (in_pml(G, ix, iz)) {
        float* mx = W.f[M_VXX] + o;
        float* mz = W.f[M_VZZ] + o;
        mx[i] = G.ax[ix] * mx[i] + G.bx[ix] * dvx;
        dvx = dvx + mx[i];
        mz[i] = G.az[iz] * mz[i] + G.bz[iz] * dvz;
        dvz = dvz + mz[i];
    }
    const float c11 = G.c11[mi], c33 = G.c33[mi], c13 = G.c13[mi];
    F.f[SH][o + i] = F.f[SH][o + i] + G.dt * (c11 * dvx + c13 * dvz);
    F.f[SV][o + i] = F.f[SV][o + i] + G.dt * (c13 * dvx + c33 * dvz);
}

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

// the residuals of step it into the adjoint fields, unsigned (backward.cu:632-641)
__global__ void residual(const Geo G, Fields A, const float* __restrict__ adj, int it)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= G.B * G.nrec) return;
    const int b = e / G.nrec, r = e - b * G.nrec;
    const long long c = loc(G, G.rec + 2LL * e);
    if (c < 0) return;
    const float* res = adj + (((long long)b * G.nt + it) * G.nrec + r) * G.nrf;
    for (int k = 0; k < G.nrf; ++k) atomicAdd(A.f[G.rf[k]] + b * G.S + c, res[k]);
}

// band save (restore = 0) of fields [f0, f1) into one step slot (B, 4, ns), or restore
__global__ void bands(const Geo G, Fields F, float* slot, int f0, int f1, int restore)
{
    const long long n = (long long)G.B * G.ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long b = e / G.ns, k = e - b * G.ns;
        const long long i = b * G.S + G.cells[k];
        for (int f = f0; f < f1; ++f) {
            float* t = slot + (b * 4 + f) * G.ns + k;
            if (restore) F.f[f][i] = *t;
            else *t = F.f[f][i];
        }
    }
}

// the reverse box: the physical box minus one cell per face (kernels.cuh:320-420)
__device__ __forceinline__ bool in_rev(const Geo& G, int ix, int iz)
{
    const int M = G.M;
    return ix >= G.pad[2] + M + 1 && ix < G.nx - (G.pad[3] + M + 1) && iz >= G.pad[0] + M + 1 &&
           iz < G.nz - (G.pad[1] + M + 1);
}

template <int M>
__global__ void __launch_bounds__(256) srev(const Geo G, Fields F)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !in_rev(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, mi = b * G.ms + i;
    const float dvx = dminus<M>(F.f[VX] + o, i, 1, G, 1.f / G.dx);
    const float dvz = dminus<M>(F.f[VZ] + o, i, G.nx, G, 1.f / G.dz);
    const float c11 = G.c11[mi], c33 = G.c33[mi], c13 = G.c13[mi];
    F.f[SH][o + i] = F.f[SH][o + i] - G.dt * (c11 * dvx + c13 * dvz);
    F.f[SV][o + i] = F.f[SV][o + i] - G.dt * (c13 * dvx + c33 * dvz);
}

template <int M>
__global__ void __launch_bounds__(256) vrev(const Geo G, Fields F)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !in_rev(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const float dsH = dplus<M>(F.f[SH] + o, i, 1, G, 1.f / G.dx);
    const float dsV = dplus<M>(F.f[SV] + o, i, G.nx, G, 1.f / G.dz);
    const float k = G.dt * G.irho[b * G.ms + i];
    F.f[VX][o + i] = F.f[VX][o + i] - k * dsH;
    F.f[VZ][o + i] = F.f[VZ][o + i] - k * dsV;
}

// adjoint half-step A, pre-multiply on every cell (kernels.cuh:536-603):
// p = (c11 lsH + c13 lsV, c13 lsH + c33 lsV), with the stress step's CPML
// transposed where that step keeps memories (core cells outside the box)
__global__ void __launch_bounds__(256) premA(const Geo G, Fields A, Fields W, float* px, float* pz)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, k = o + i, mi = b * G.ms + i;
    const float lsh = A.f[SH][k], lsv = A.f[SV][k];
    float p_x = G.c11[mi] * lsh + G.c13[mi] * lsv;
    float p_z = G.c13[mi] * lsh + G.c33[mi] * lsv;
    if (core(G, ix, iz) && in_pml(G, ix, iz)) {
        const float tx = W.f[M_VXX][k] + p_x, tz = W.f[M_VZZ][k] + p_z;
        p_x += G.bx[ix] * tx;
        p_z += G.bz[iz] * tz;
        W.f[M_VXX][k] = G.ax[ix] * tx;
        W.f[M_VZZ][k] = G.az[iz] * tz;
    }
    px[k] = p_x;
    pz[k] = p_z;
}

// half-step A, apply on the core: lambda_v += -dt D+(p) (kernels.cuh:667-690)
template <int M>
__global__ void __launch_bounds__(256) appA(const Geo G, Fields A, const float* px, const float* pz)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const float dpx = dplus<M>(px + o, i, 1, G, 1.f / G.dx);
    const float dpz = dplus<M>(pz + o, i, G.nx, G, 1.f / G.dz);
    A.f[VX][o + i] += -G.dt * dpx;
    A.f[VZ][o + i] += -G.dt * dpz;
}

// half-step B, pre-multiply on every cell (kernels.cuh:605-640):
// q = inv_rho lambda_v with the velocity step's transposed CPML
__global__ void __launch_bounds__(256) premB(const Geo G, Fields A, Fields W, float* qx, float* qz)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, k = o + i;
    const float ir = G.irho[b * G.ms + i];
    float q_x = ir * A.f[VX][k];
    float q_z = ir * A.f[VZ][k];
    if (core(G, ix, iz) && in_pml(G, ix, iz)) {
        const float tx = W.f[M_SHX][k] + q_x, tz = W.f[M_SVZ][k] + q_z;
        q_x += G.bxh[ix] * tx;
        q_z += G.bzh[iz] * tz;
        W.f[M_SHX][k] = G.axh[ix] * tx;
        W.f[M_SVZ][k] = G.azh[iz] * tz;
    }
    qx[k] = q_x;
    qz[k] = q_z;
}

// half-step B, apply on the core: lambda_s += -dt D-(q) (kernels.cuh:726-750)
template <int M>
__global__ void __launch_bounds__(256) appB(const Geo G, Fields A, const float* qx, const float* qz)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix;
    const float dqx = dminus<M>(qx + o, i, 1, G, 1.f / G.dx);
    const float dqz = dminus<M>(qz + o, i, G.nx, G, 1.f / G.dz);
    A.f[SH][o + i] += -G.dt * dqx;
    A.f[SV][o + i] += -G.dt * dqz;
}

struct Grads {
    float *vp, *eps, *dlt, *rho;    // per-shot slots (B, S)
};

// the gradient of one step on the physical box (kernels.cuh:822-912): the
// stiffness gradients from the forward velocities at the end of the step, the
// 1 / rho gradient from the stresses at its start, chained to the models
template <int M>
__global__ void __launch_bounds__(256) grad(const Geo G, Fields F, Fields A, Grads g)
{
    int b, iz, ix;
    if (!cell2(G, b, iz, ix) || ix < G.x0 || ix >= G.x1 || iz < G.z0 || iz >= G.z1 || !core(G, ix, iz)) return;
    const long long o = b * G.S, i = (long long)iz * G.nx + ix, k = o + i, mi = b * G.ms + i;
    const float dvx = dminus<M>(F.f[VX] + o, i, 1, G, 1.f / G.dx);
    const float dvz = dminus<M>(F.f[VZ] + o, i, G.nx, G, 1.f / G.dz);
    const float dsH = dplus<M>(F.f[SH] + o, i, 1, G, 1.f / G.dx);
    const float dsV = dplus<M>(F.f[SV] + o, i, G.nx, G, 1.f / G.dz);
    const float lsh = A.f[SH][k], lsv = A.f[SV][k], lvx = A.f[VX][k], lvz = A.f[VZ][k];
    const float dt = G.dt;
    const float g11 = dt * lsh * dvx;
    const float g33 = dt * lsv * dvz;
    const float g13 = dt * (lsh * dvz + lsv * dvx);
    const float gir = dt * (lvx * dsH + lvz * dsV);
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

static Plan make_plan(const sweep_vti_desc* d, int mem_mode)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->M >= 1 && d->M <= MAXM, "vti: spatial orders 2 to %d are built (got order %d)", 2 * MAXM,
                  2 * d->M);
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY,
                  "vti: boundary saving with fp32 strips in device memory is built (mem_mode %d)", mem_mode);
    SWEEP_REQUIRE(d->B >= 1 && d->B <= 65535 && d->nt >= 1, "vti: 1 to 65535 shots and nt >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "vti: negative source/receiver count");
    SWEEP_REQUIRE(d->nsrc_fields >= 1 && d->nsrc_fields <= 4, "vti: 1 to 4 source fields");
    SWEEP_REQUIRE(d->nrec_fields >= 1 && d->nrec_fields <= 4, "vti: 1 to 4 receiver fields");
    for (int k = 0; k < d->nsrc_fields; ++k) {
        SWEEP_REQUIRE(d->src_fields[k] >= 0 && d->src_fields[k] < 4, "vti: bad source field %d", d->src_fields[k]);
        for (int j = 0; j < k; ++j)
            SWEEP_REQUIRE(d->src_fields[j] != d->src_fields[k], "vti: source field %d repeated", d->src_fields[k]);
    }
    for (int k = 0; k < d->nrec_fields; ++k)
        SWEEP_REQUIRE(d->rec_fields[k] >= 0 && d->rec_fields[k] < 4, "vti: bad receiver field %d", d->rec_fields[k]);
    for (int f = 0; f < 4; ++f)
        SWEEP_REQUIRE(d->pad[f] >= 1, "vti: every face needs a PML pad >= 1 (face %d has %d)", f, d->pad[f]);
    Plan pl{};
    Geo& G = pl.G;
    const int M = d->M;
    G.B = d->B; G.nz = d->nz; G.nx = d->nx; G.nt = d->nt; G.M = M;
    G.S = (long long)d->nz * d->nx;
    SWEEP_REQUIRE(G.S < (1LL << 31), "vti: one shot's grid must hold < 2^31 cells");
    for (int f = 0; f < 4; ++f) G.pad[f] = d->pad[f];
    G.z0 = G.pad[0] + M; G.z1 = G.nz - G.pad[1] - M;
    G.x0 = G.pad[2] + M; G.x1 = G.nx - G.pad[3] - M;
    SWEEP_REQUIRE(G.z1 - G.z0 >= 2 && G.x1 - G.x0 >= 2, "vti: the physical box must be at least 2 cells per axis");
    G.dt = d->dt; G.dz = d->dz; G.dx = d->dx;
    for (int k = 0; k <= MAXM; ++k) G.c[k] = 0.f;
    staggered_weights(M, G.c);
    G.az = d->az; G.bz = d->bz; G.azh = d->azh; G.bzh = d->bzh;
    G.ax = d->ax; G.bx = d->bx; G.axh = d->axh; G.bxh = d->bxh;
    G.vp = d->vp; G.eps = d->epsilon; G.dlt = d->delta; G.rho = d->rho;
    const bool per_shot = d->model_stride != 0;
    SWEEP_REQUIRE(!per_shot || d->model_stride == G.S, "vti: model_stride must be 0 or nz * nx");
    G.ms = per_shot ? G.S : 0;
    pl.nm = per_shot ? G.B : 1;
    G.nsrc = d->nsrc; G.nrec = d->nrec; G.nsf = d->nsrc_fields; G.nrf = d->nrec_fields;
    for (int k = 0; k < 4; ++k) { G.sf[k] = d->src_fields[k]; G.rf[k] = d->rec_fields[k]; }
    G.src = d->src_loc; G.rec = d->rec_loc; G.wavelet = d->wavelet;
    // the reference's four bands (boundary/strip.cuh:46-123), cells of two bands listed twice
    const int w = M + 1;
    const int ts = G.z0 - M, be = G.z1 + M, ls = G.x0 - M, re = G.x1 + M;
    for (int z = ts; z < ts + w; ++z) for (int x = G.x0; x < G.x1; ++x) pl.cells.push_back(z * G.nx + x);
    for (int z = be - w; z < be; ++z) for (int x = G.x0; x < G.x1; ++x) pl.cells.push_back(z * G.nx + x);
    for (int z = G.z0; z < G.z1; ++z) for (int x = ls; x < ls + w; ++x) pl.cells.push_back(z * G.nx + x);
    for (int z = G.z0; z < G.z1; ++z) for (int x = re - w; x < re; ++x) pl.cells.push_back(z * G.nx + x);
    G.ns = (int)pl.cells.size();
    return pl;
}

struct Ws {
    float *c11, *c33, *c13, *irho;
    int* cells;
    float* f[4];
    float* m[NMEM];                 // forward memories / adjoint memories
    float* a[4];
    float *sx, *sz;                 // pre-multiply scratch
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
    for (int k = 0; k < 4; ++k) w.f[k] = c.take<float>(n);
    for (int k = 0; k < NMEM; ++k) w.m[k] = c.take<float>(n);
    if (rev) {
        for (int k = 0; k < 4; ++k) w.a[k] = c.take<float>(n);
        w.gvp = c.take<float>(n); w.geps = c.take<float>(n); w.gdlt = c.take<float>(n); w.grho = c.take<float>(n);
    }
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
    if (rev) { w.sx = c.take<float>(n); w.sz = c.take<float>(n); }
}

static long long slot_floats(const Plan& pl) { return (long long)pl.G.B * 4 * pl.G.ns; }

void sizes(const sweep_vti_desc* d, int mem_mode, int, int64_t* ws_bytes, int64_t* tape_bytes)
{
    const Plan pl = make_plan(d, mem_mode);
    Carve f(nullptr), r(nullptr);
    Ws w;
    carve(f, pl, false, w);
    carve(r, pl, true, w);
    *ws_bytes = std::max(f.off, r.off);
    *tape_bytes = ((long long)pl.G.nt * slot_floats(pl) + 4LL * pl.G.B * pl.G.S) * 4;
}

static void setup(const sweep_vti_desc* d, Plan& pl, const Ws& w, cudaStream_t st)
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

static dim3 grid_of(const Geo& G) { return dim3((G.nx + 31) / 32, (G.nz + 7) / 8, (unsigned)G.B); }
static unsigned blocks(long long n) { return (unsigned)std::max<long long>(std::min<long long>((n + 255) / 256, 8192), 1); }

template <int M>
static void forward_m(const sweep_vti_desc* d, Plan& pl, float* record, void* tape, void* ws, int64_t ws_bytes,
                      cudaStream_t st)
{
    Carve c(ws);
    Ws w;
    carve(c, pl, false, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "vti forward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    setup(d, pl, w, st);
    const Geo& G = pl.G;
    if (record && G.nrec > 0)
        SWEEP_CUDA(cudaMemsetAsync(record, 0, sizeof(float) * (size_t)G.B * G.nt * G.nrec * G.nrf, st));
    Fields F{}, W{};
    for (int k = 0; k < 4; ++k) { F.f[k] = w.f[k]; W.f[k] = w.m[k]; }
    float* tp = static_cast<float*>(tape);
    const dim3 grid = grid_of(G), block(32, 8);
    for (int it = 0; it < G.nt; ++it) {
        vel<M><<<grid, block, 0, st>>>(G, F, W);
        str<M><<<grid, block, 0, st>>>(G, F, W);
        if (G.nsrc > 0) inject<<<(G.B * G.nsrc + 127) / 128, 128, 0, st>>>(G, F, it, 1.f);
        if (tp) bands<<<blocks((long long)G.B * G.ns), 256, 0, st>>>(G, F, tp + it * slot_floats(pl), 0, 4, 0);
        if (record && G.nrec > 0) gather<<<(G.B * G.nrec + 127) / 128, 128, 0, st>>>(G, F, record, it);
        SWEEP_LAUNCH_CHECK();
    }
    if (tp) {
        float* last = tp + (long long)G.nt * slot_floats(pl);
        for (int b = 0; b < G.B; ++b)
            for (int f = 0; f < 4; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(last + ((long long)b * 4 + f) * G.S, w.f[f] + b * G.S,
                                           sizeof(float) * G.S, cudaMemcpyDeviceToDevice, st));
    }
}

template <int M>
static void backward_m(const sweep_vti_desc* d, Plan& pl, const float* adj, const void* tape, float* const out[4],
                       void* ws, int64_t ws_bytes, cudaStream_t st)
{
    SWEEP_REQUIRE(tape != nullptr, "vti backward: the forward's tape is required");
    Carve c(ws);
    Ws w;
    carve(c, pl, true, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "vti backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    setup(d, pl, w, st);
    const Geo& G = pl.G;
    const float* tp = static_cast<const float*>(tape);
    const float* last = tp + (long long)G.nt * slot_floats(pl);
    for (int b = 0; b < G.B; ++b)
        for (int f = 0; f < 4; ++f)
            SWEEP_CUDA(cudaMemcpyAsync(w.f[f] + b * G.S, last + ((long long)b * 4 + f) * G.S, sizeof(float) * G.S,
                                       cudaMemcpyDeviceToDevice, st));
    Fields F{}, A{}, W{};
    for (int k = 0; k < 4; ++k) { F.f[k] = w.f[k]; A.f[k] = w.a[k]; W.f[k] = w.m[k]; }
    const Grads g{w.gvp, w.geps, w.gdlt, w.grho};
    const dim3 grid = grid_of(G), block(32, 8);
    const unsigned srcb = (unsigned)(G.B * G.nsrc + 127) / 128, recb = (unsigned)(G.B * G.nrec + 127) / 128;
    const unsigned bb = blocks((long long)G.B * G.ns);
    for (int it = G.nt - 1; it >= 1; --it) {
        float* prev = const_cast<float*>(tp) + (long long)(it - 1) * slot_floats(pl);
        if (G.nrec > 0) residual<<<recb, 128, 0, st>>>(G, A, adj, it);
        if (G.nsrc > 0) inject<<<srcb, 128, 0, st>>>(G, F, it, -1.f);
        srev<M><<<grid, block, 0, st>>>(G, F);
        bands<<<bb, 256, 0, st>>>(G, F, prev, SH, 4, 1);
        premA<<<grid, block, 0, st>>>(G, A, W, w.sx, w.sz);
        appA<M><<<grid, block, 0, st>>>(G, A, w.sx, w.sz);
        grad<M><<<grid, block, 0, st>>>(G, F, A, g);
        premB<<<grid, block, 0, st>>>(G, A, W, w.sx, w.sz);
        appB<M><<<grid, block, 0, st>>>(G, A, w.sx, w.sz);
        vrev<M><<<grid, block, 0, st>>>(G, F);
        bands<<<bb, 256, 0, st>>>(G, F, prev, VX, SH, 1);
        SWEEP_LAUNCH_CHECK();
    }
    const unsigned fb = blocks((long long)pl.nm * G.S);
    const float* slots[4] = {w.gvp, w.geps, w.gdlt, w.grho};
    for (int k = 0; k < 4; ++k) finalize<<<fb, 256, 0, st>>>(G, slots[k], out[k]);
    SWEEP_LAUNCH_CHECK();
}

#define SWEEP_VTI_DISPATCH(M_, CALL) \
    switch (M_) {                    \
    case 1: CALL(1); break;          \
    case 2: CALL(2); break;          \
    case 3: CALL(3); break;          \
    case 4: CALL(4); break;          \
    case 5: CALL(5); break;          \
    case 6: CALL(6); break;          \
    default: CALL(7); break;         \
    }

void forward(const sweep_vti_desc* d, int mem_mode, int, float* record, void* tape, void* ws, int64_t ws_bytes,
             cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
#define SWEEP_VTI_FWD(m) forward_m<m>(d, pl, record, tape, ws, ws_bytes, st)
    SWEEP_VTI_DISPATCH(d->M, SWEEP_VTI_FWD)
#undef SWEEP_VTI_FWD
}

void backward(const sweep_vti_desc* d, int mem_mode, int, const float* adj, const void* tape, float* grad_vp,
              float* grad_eps, float* grad_dlt, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    Plan pl = make_plan(d, mem_mode);
    float* const out[4] = {grad_vp, grad_eps, grad_dlt, grad_rho};
#define SWEEP_VTI_BWD(m) backward_m<m>(d, pl, adj, tape, out, ws, ws_bytes, st)
    SWEEP_VTI_DISPATCH(d->M, SWEEP_VTI_BWD)
#undef SWEEP_VTI_BWD
}

}  // namespace vti
}  // namespace sweep
