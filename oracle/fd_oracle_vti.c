/*
 * fd_oracle_vti.c -- CPU restatement of the reference's compiled (impl='c')
 * 2-D first-order acoustic VTI path (Duveneck et al. 2008: vx, vz and the
 * horizontal / vertical stresses sH, sV on a staggered grid), used ONLY as
 * test infrastructure: the parity checker of the CUDA library.  It is never
 * linked into, loaded by or called from the product library.
 *
 * Built with REAL=float and REAL=double by oracle/Makefile, -ffp-contract=off.
 * Layout: every field is (B, nz, nx), x fastest, on the runtime grid; runtime
 * (x, z) coordinates, off-grid ones skipped.  Field indices: 0 vx, 1 vz,
 * 2 sH, 3 sV.  Records and their cotangents are (B, nt, nrec, nfield).
 *
 * What each function restates (reference paths, relative to the project root):
 *   stiffness         src/sweep/csrc/cuda/common/derived_models.cu:40-53
 *                     (c33 = rho vp^2, c11 = c33 (1 + 2 eps),
 *                     c13 = c33 sqrt(1 + 2 delta), inv_rho = 1 / rho)
 *   velocity step     src/sweep/csrc/cuda/equations/acoustic_vti_1st_2d/
 *                     kernels.cuh:104-163 (D+ of sH / sV, CPML memories on the
 *                     half-cell profiles outside the physical box)
 *   stress step       kernels.cuh:209-272 (D- of vx / vz, integer profiles)
 *   reverse (NOPML)   kernels.cuh:320-420 (box pad + M + 1 per face)
 *   adjoint           kernels.cuh:505-760: the stress pre-multiply
 *                     p = (c11 lsH + c13 lsV, c13 lsH + c33 lsV) with the
 *                     transposed CPML of the stress step, then
 *                     lv += -dt D+(p); the velocity pre-multiply
 *                     q = inv_rho lv with the velocity step's transposed CPML,
 *                     then ls += -dt D-(q)
 *   gradient          kernels.cuh:770-915 (c11 / c33 / c13 / inv_rho gradients
 *                     on the physical box, chained to vp, epsilon, delta, rho)
 *   step order        acoustic_vti_1st_2d/forward.cu (velocity, stress, source,
 *                     band save, record), backward.cu:631-740 (residual, source
 *                     removal, stress reverse, stress bands, adjoint A,
 *                     gradient, adjoint B, velocity reverse, velocity bands;
 *                     it = nt - 1 .. 1)
 *   bands             src/sweep/csrc/cuda/common/boundary/strip.cuh:46-123
 *                     (width M+1 at offset -M, physical box tangentially)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#endif
#define R(x) ((REAL)(x))

typedef long long i64;

typedef struct {
    int B, nz, nx, nt, M;
    int pad[4];                 /* zlo, zhi, xlo, xhi PML widths */
    REAL dt, dz, dx;
    const REAL* c;              /* c[1..M] staggered coefficients */
    const REAL *az, *bz, *azh, *bzh, *ax, *bx, *axh, *bxh;
    const REAL *vp, *eps, *dlt, *rho;
    i64 ms;                     /* model stride between shots (0 = shared) */
    int nsrc; const int* src; const REAL* wavelet; int nsf; const int* sf;
    int nrec; const int* rec; int nrf; const int* rf;
} VTI;

enum { VX, VZ, SH, SV, M_SHX, M_SVZ, M_VXX, M_VZZ, NF };

static inline REAL dplus(const REAL* u, i64 i, i64 s, int M, const REAL* c, REAL inv)
{
    REAL g = c[1] * (u[i + s] - u[i]);
    for (int k = 2; k <= M; ++k) g = g + c[k] * (u[i + k * s] - u[i - (k - 1) * s]);
    return g * inv;
}

static inline REAL dminus(const REAL* u, i64 i, i64 s, int M, const REAL* c, REAL inv)
{
    REAL g = c[1] * (u[i] - u[i - s]);
    for (int k = 2; k <= M; ++k) g = g + c[k] * (u[i + (k - 1) * s] - u[i - k * s]);
    return g * inv;
}

static int in_grid(int ix, int iz, int nx, int nz) { return ix >= 0 && ix < nx && iz >= 0 && iz < nz; }

/* outside the physical box (PML pad plus the stencil halo) */
static inline int in_pml(const VTI* p, int ix, int iz)
{
    const int h = p->M;
    return ix < p->pad[2] + h || ix >= p->nx - p->pad[3] - h || iz < p->pad[0] + h || iz >= p->nz - p->pad[1] - h;
}

static inline int in_core(const VTI* p, int ix, int iz)
{
    return ix >= p->M && ix < p->nx - p->M && iz >= p->M && iz < p->nz - p->M;
}

static void stiffness(const VTI* p, int b, REAL* c11, REAL* c33, REAL* c13, REAL* irho)
{
    const i64 n = (i64)p->nz * p->nx;
    const REAL *v = p->vp + b * p->ms, *e = p->eps + b * p->ms, *d = p->dlt + b * p->ms, *r = p->rho + b * p->ms;
    for (i64 i = 0; i < n; ++i) {
        const REAL rv2 = r[i] * (v[i] * v[i]);
        c33[i] = rv2;
        c11[i] = rv2 * (R(1) + R(2) * e[i]);
        c13[i] = rv2 * (REAL)sqrt((double)(R(1) + R(2) * d[i]));
        irho[i] = R(1) / r[i];
    }
}

static void velocity_step(const VTI* p, REAL** F, const REAL* irho)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz)
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dsH = dplus(F[SH], i, 1, M, p->c, R(1) / p->dx);
            REAL dsV = dplus(F[SV], i, nx, M, p->c, R(1) / p->dz);
            if (in_pml(p, ix, iz)) {
                F[M_SHX][i] = p->axh[ix] * F[M_SHX][i] + p->bxh[ix] * dsH;
                dsH = dsH + F[M_SHX][i];
                F[M_SVZ][i] = p->azh[iz] * F[M_SVZ][i] + p->bzh[iz] * dsV;
                dsV = dsV + F[M_SVZ][i];
            }
            F[VX][i] = F[VX][i] + (p->dt * irho[i]) * dsH;
            F[VZ][i] = F[VZ][i] + (p->dt * irho[i]) * dsV;
        }
}

static void stress_step(const VTI* p, REAL** F, const REAL* c11, const REAL* c33, const REAL* c13)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz)
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dvx = dminus(F[VX], i, 1, M, p->c, R(1) / p->dx);
            REAL dvz = dminus(F[VZ], i, nx, M, p->c, R(1) / p->dz);
            if (in_pml(p, ix, iz)) {
                F[M_VXX][i] = p->ax[ix] * F[M_VXX][i] + p->bx[ix] * dvx;
                dvx = dvx + F[M_VXX][i];
                F[M_VZZ][i] = p->az[iz] * F[M_VZZ][i] + p->bz[iz] * dvz;
                dvz = dvz + F[M_VZZ][i];
            }
            F[SH][i] = F[SH][i] + p->dt * (c11[i] * dvx + c13[i] * dvz);
            F[SV][i] = F[SV][i] + p->dt * (c13[i] * dvx + c33[i] * dvz);
        }
}

static void inject(const VTI* p, int b, REAL* u, int it, REAL sign)
{
    for (int s = 0; s < p->nsrc; ++s) {
        int ix = p->src[(b * p->nsrc + s) * 2], iz = p->src[(b * p->nsrc + s) * 2 + 1];
        if (!in_grid(ix, iz, p->nx, p->nz)) continue;
        u[(i64)iz * p->nx + ix] += sign * p->wavelet[((i64)b * p->nsrc + s) * p->nt + it];
    }
}

static int band_lo(int p0, int off, int w, int n) { int s = p0 + off; if (s + w > n) s = n - w; return s < 0 ? 0 : s; }
static int band_hi(int p1, int off, int w, int n) { int e = p1 - off; if (e - w < 0) e = w; return e > n ? n : e; }

/* the reference's four bands (cells of two bands listed twice) */
static int band_cells(const VTI* p, int* out)
{
    const int nz = p->nz, nx = p->nx, M = p->M, w = M + 1, off = -M;
    const int z0 = p->pad[0] + M, z1 = nz - p->pad[1] - M, x0 = p->pad[2] + M, x1 = nx - p->pad[3] - M;
    const int ts = band_lo(z0, off, w, nz), be = band_hi(z1, off, w, nz);
    const int ls = band_lo(x0, off, w, nx), re = band_hi(x1, off, w, nx);
    int n = 0;
    for (int z = ts; z < ts + w; ++z) for (int x = x0; x < x1; ++x) { if (out) out[n] = z * nx + x; ++n; }
    for (int z = be - w; z < be; ++z) for (int x = x0; x < x1; ++x) { if (out) out[n] = z * nx + x; ++n; }
    for (int z = z0; z < z1; ++z) for (int x = ls; x < ls + w; ++x) { if (out) out[n] = z * nx + x; ++n; }
    for (int z = z0; z < z1; ++z) for (int x = re - w; x < re; ++x) { if (out) out[n] = z * nx + x; ++n; }
    return n;
}

long long oracle_vti2d_tape_len(int B, int nz, int nx, int nt, int M, const int* pad)
{
    VTI p; memset(&p, 0, sizeof p);
    p.B = B; p.nz = nz; p.nx = nx; p.nt = nt; p.M = M;
    for (int k = 0; k < 4; ++k) p.pad[k] = pad[k];
    return (long long)nt * B * 4 * band_cells(&p, NULL) + 4LL * B * nz * nx;
}

#define SETUP_VTI                                                                         \
    VTI p = {B, nz, nx, nt, M, {pad[0], pad[1], pad[2], pad[3]}, dt, dz, dx, coef,          \
             prof, prof + nz, prof + 2 * nz, prof + 3 * nz,                                 \
             prof + 4 * nz, prof + 4 * nz + nx, prof + 4 * nz + 2 * nx, prof + 4 * nz + 3 * nx, \
             vp, eps, dlt, rho, m_stride, nsrc, src, wavelet, nsf, sfields, nrec, rec, nrf, rfields}

int oracle_vti2d_forward(
    int B, int nz, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dx,
    const REAL* coef, const REAL* prof,
    const REAL* vp, const REAL* eps, const REAL* dlt, const REAL* rho, i64 m_stride,
    int nsrc, const int* src, const REAL* wavelet, int nsf, const int* sfields,
    int nrec, const int* rec, int nrf, const int* rfields,
    REAL* record, REAL* tape)
{
    SETUP_VTI;
    const i64 n = (i64)nz * nx;
    const int ns = band_cells(&p, NULL);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    REAL* buf = (REAL*)calloc((size_t)n * (NF + 4), sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    band_cells(&p, cells);
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * (NF + 4));
        REAL* F[NF];
        for (int f = 0; f < NF; ++f) F[f] = buf + f * n;
        REAL *c11 = buf + NF * n, *c33 = buf + (NF + 1) * n, *c13 = buf + (NF + 2) * n, *irho = buf + (NF + 3) * n;
        stiffness(&p, b, c11, c33, c13, irho);
        for (int it = 0; it < nt; ++it) {
            velocity_step(&p, F, irho);
            stress_step(&p, F, c11, c33, c13);
            for (int k = 0; k < nsf; ++k) inject(&p, b, F[sfields[k]], it, R(1));
            if (tape)
                for (int f = 0; f < 4; ++f) {
                    REAL* dst = tape + (((i64)it * B + b) * 4 + f) * ns;
                    for (int c = 0; c < ns; ++c) dst[c] = F[f][cells[c]];
                }
            for (int r = 0; r < nrec; ++r) {
                int ix = rec[(b * nrec + r) * 2], iz = rec[(b * nrec + r) * 2 + 1];
                if (!in_grid(ix, iz, nx, nz)) continue;
                for (int k = 0; k < nrf; ++k)
                    record[(((i64)b * nt + it) * nrec + r) * nrf + k] = F[rfields[k]][(i64)iz * nx + ix];
            }
        }
        if (tape)
            for (int f = 0; f < 4; ++f)
                memcpy(tape + (i64)nt * B * 4 * ns + ((i64)b * 4 + f) * n, F[f], sizeof(REAL) * n);
    }
    free(buf); free(cells);
    return 0;
}

/* reverse (NOPML) steps on the box pad + M + 1 per face (kernels.cuh:320-420) */
static void reverse_box(const VTI* p, int lo[2], int hi[2])
{
    const int M = p->M;
    lo[0] = p->pad[0] + M + 1; hi[0] = p->nz - (p->pad[1] + M + 1);
    lo[1] = p->pad[2] + M + 1; hi[1] = p->nx - (p->pad[3] + M + 1);
}

static void stress_reverse(const VTI* p, REAL** F, const REAL* c11, const REAL* c33, const REAL* c13)
{
    const int nx = p->nx, M = p->M;
    int lo[2], hi[2];
    reverse_box(p, lo, hi);
    #pragma omp parallel for schedule(static)
    for (int iz = lo[0]; iz < hi[0]; ++iz)
        for (int ix = lo[1]; ix < hi[1]; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            const REAL dvx = dminus(F[VX], i, 1, M, p->c, R(1) / p->dx);
            const REAL dvz = dminus(F[VZ], i, nx, M, p->c, R(1) / p->dz);
            F[SH][i] = F[SH][i] - p->dt * (c11[i] * dvx + c13[i] * dvz);
            F[SV][i] = F[SV][i] - p->dt * (c13[i] * dvx + c33[i] * dvz);
        }
}

static void velocity_reverse(const VTI* p, REAL** F, const REAL* irho)
{
    const int nx = p->nx, M = p->M;
    int lo[2], hi[2];
    reverse_box(p, lo, hi);
    #pragma omp parallel for schedule(static)
    for (int iz = lo[0]; iz < hi[0]; ++iz)
        for (int ix = lo[1]; ix < hi[1]; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            const REAL dsH = dplus(F[SH], i, 1, M, p->c, R(1) / p->dx);
            const REAL dsV = dplus(F[SV], i, nx, M, p->c, R(1) / p->dz);
            F[VX][i] = F[VX][i] - (p->dt * irho[i]) * dsH;
            F[VZ][i] = F[VZ][i] - (p->dt * irho[i]) * dsV;
        }
}

/* adjoint half-step A (kernels.cuh:505-715): p = C lambda_s with the stress
 * step's transposed CPML on every cell, then lambda_v += -dt D+(p) */
static void adjoint_A(const VTI* p, REAL** A, REAL* px, REAL* pz, const REAL* c11, const REAL* c33, const REAL* c13)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
        for (int ix = 0; ix < nx; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL qx = c11[i] * A[SH][i] + c13[i] * A[SV][i];
            REAL qz = c13[i] * A[SH][i] + c33[i] * A[SV][i];
            if (in_core(p, ix, iz) && in_pml(p, ix, iz)) {
                const REAL tx = A[M_VXX][i] + qx, tz = A[M_VZZ][i] + qz;
                qx = qx + p->bx[ix] * tx;
                qz = qz + p->bz[iz] * tz;
                A[M_VXX][i] = p->ax[ix] * tx;
                A[M_VZZ][i] = p->az[iz] * tz;
            }
            px[i] = qx;
            pz[i] = qz;
        }
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz)
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            A[VX][i] = A[VX][i] + (-p->dt) * dplus(px, i, 1, M, p->c, R(1) / p->dx);
            A[VZ][i] = A[VZ][i] + (-p->dt) * dplus(pz, i, nx, M, p->c, R(1) / p->dz);
        }
}

/* adjoint half-step B (kernels.cuh:595-760): q = inv_rho lambda_v with the
 * velocity step's transposed CPML, then lambda_s += -dt D-(q) */
static void adjoint_B(const VTI* p, REAL** A, REAL* qx_, REAL* qz_, const REAL* irho)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
        for (int ix = 0; ix < nx; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL qx = irho[i] * A[VX][i];
            REAL qz = irho[i] * A[VZ][i];
            if (in_core(p, ix, iz) && in_pml(p, ix, iz)) {
                const REAL tx = A[M_SHX][i] + qx, tz = A[M_SVZ][i] + qz;
                qx = qx + p->bxh[ix] * tx;
                qz = qz + p->bzh[iz] * tz;
                A[M_SHX][i] = p->axh[ix] * tx;
                A[M_SVZ][i] = p->azh[iz] * tz;
            }
            qx_[i] = qx;
            qz_[i] = qz;
        }
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz)
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            A[SH][i] = A[SH][i] + (-p->dt) * dminus(qx_, i, 1, M, p->c, R(1) / p->dx);
            A[SV][i] = A[SV][i] + (-p->dt) * dminus(qz_, i, nx, M, p->c, R(1) / p->dz);
        }
}

/* gradient of one step on the physical box (kernels.cuh:770-915): forward
 * velocities at the end of the step, stresses at its start, the adjoint
 * between half-steps A and B */
static void gradient(const VTI* p, int b, REAL** F, REAL** A, REAL* gvp, REAL* geps, REAL* gdlt, REAL* grho)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL *vp = p->vp + b * p->ms, *ep = p->eps + b * p->ms, *dl = p->dlt + b * p->ms, *rh = p->rho + b * p->ms;
    const int z0 = p->pad[0] + M, z1 = nz - p->pad[1] - M, x0 = p->pad[2] + M, x1 = nx - p->pad[3] - M;
    const REAL dt = p->dt;
    #pragma omp parallel for schedule(static)
    for (int iz = z0; iz < z1; ++iz)
        for (int ix = x0; ix < x1; ++ix) {
            if (!in_core(p, ix, iz)) continue;
            const i64 i = (i64)iz * nx + ix;
            const REAL dvx = dminus(F[VX], i, 1, M, p->c, R(1) / p->dx);
            const REAL dvz = dminus(F[VZ], i, nx, M, p->c, R(1) / p->dz);
            const REAL dsH = dplus(F[SH], i, 1, M, p->c, R(1) / p->dx);
            const REAL dsV = dplus(F[SV], i, nx, M, p->c, R(1) / p->dz);
            const REAL lsh = A[SH][i], lsv = A[SV][i], lvx = A[VX][i], lvz = A[VZ][i];
            const REAL g11 = dt * lsh * dvx;
            const REAL g33 = dt * lsv * dvz;
            const REAL g13 = dt * (lsh * dvz + lsv * dvx);
            const REAL gir = dt * (lvx * dsH + lvz * dsV);
            const REAL v = vp[i], e = ep[i], d = dl[i], r = rh[i];
            const REAL ope = R(1) + R(2) * e, opd = R(1) + R(2) * d;
            const REAL sd = (REAL)sqrt((double)opd);
            const REAL v2 = v * v;
            const REAL common = g11 * ope + g33 + g13 * sd;
            gvp[i] = gvp[i] + R(2) * r * v * common;
            geps[i] = geps[i] + g11 * R(2) * r * v2;
            gdlt[i] = gdlt[i] + g13 * r * v2 / (sd > R(1e-12) ? sd : R(1e-12));
            grho[i] = grho[i] + (v2 * common - gir / (r * r));
        }
}

int oracle_vti2d_backward(
    int B, int nz, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dx,
    const REAL* coef, const REAL* prof,
    const REAL* vp, const REAL* eps, const REAL* dlt, const REAL* rho, i64 m_stride,
    int nsrc, const int* src, const REAL* wavelet, int nsf, const int* sfields,
    int nrec, const int* rec, int nrf, const int* rfields,
    const REAL* adj, const REAL* tape, REAL* grad_vp, REAL* grad_eps, REAL* grad_dlt, REAL* grad_rho)
{
    SETUP_VTI;
    const i64 n = (i64)nz * nx;
    const int ns = band_cells(&p, NULL);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    const int nbuf = 4 + NF + 4 + 4;
    REAL* buf = (REAL*)calloc((size_t)n * nbuf, sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    band_cells(&p, cells);
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * nbuf);
        REAL *F[4], *A[NF];
        for (int f = 0; f < 4; ++f) F[f] = buf + f * n;
        for (int f = 0; f < NF; ++f) A[f] = buf + (4 + f) * n;
        REAL *sx = buf + (4 + NF) * n, *sz = buf + (5 + NF) * n;
        REAL *c11 = buf + (6 + NF) * n, *c33 = buf + (7 + NF) * n, *c13 = buf + (8 + NF) * n, *irho = buf + (9 + NF) * n;
        stiffness(&p, b, c11, c33, c13, irho);
        REAL *gvp = grad_vp + b * m_stride, *geps = grad_eps + b * m_stride;
        REAL *gdlt = grad_dlt + b * m_stride, *grho = grad_rho + b * m_stride;
        for (int f = 0; f < 4; ++f)
            memcpy(F[f], tape + (i64)nt * B * 4 * ns + ((i64)b * 4 + f) * n, sizeof(REAL) * n);
        for (int it = nt - 1; it >= 1; --it) {
            /* residuals into the adjoint fields, unsigned (backward.cu:632-641:
               the adjoint stresses are not negated here) */
            for (int k = 0; k < nrf; ++k)
                for (int r = 0; r < nrec; ++r) {
                    int ix = rec[(b * nrec + r) * 2], iz = rec[(b * nrec + r) * 2 + 1];
                    if (!in_grid(ix, iz, nx, nz)) continue;
                    A[rfields[k]][(i64)iz * nx + ix] += adj[(((i64)b * nt + it) * nrec + r) * nrf + k];
                }
            for (int k = 0; k < nsf; ++k) inject(&p, b, F[sfields[k]], it, R(-1));
            stress_reverse(&p, F, c11, c33, c13);
            for (int f = SH; f <= SV; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 4 + f) * ns;
                for (int c = 0; c < ns; ++c) F[f][cells[c]] = s[c];
            }
            adjoint_A(&p, A, sx, sz, c11, c33, c13);
            gradient(&p, b, F, A, gvp, geps, gdlt, grho);
            adjoint_B(&p, A, sx, sz, irho);
            velocity_reverse(&p, F, irho);
            for (int f = VX; f <= VZ; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 4 + f) * ns;
                for (int c = 0; c < ns; ++c) F[f][cells[c]] = s[c];
            }
        }
    }
    free(buf); free(cells);
    return 0;
}
