/*
 * fd_oracle_vti3d.c -- CPU restatement of the reference's compiled (impl='c')
 * 3-D first-order acoustic VTI path (Duveneck et al. 2008: vx, vy, vz and the
 * horizontal / vertical stresses sH = s11 = s22, sV = s33 on a staggered
 * grid), used ONLY as test infrastructure: the parity checker of the CUDA
 * library.  It is never linked into, loaded by or called from the product
 * library.
 *
 * Built with REAL=float and REAL=double by oracle/Makefile, -ffp-contract=off.
 * Layout: every field is (B, nz, ny, nx), x fastest, on the runtime grid;
 * runtime (x, y, z) coordinates, off-grid ones skipped.  Field indices: 0 vx,
 * 1 vy, 2 vz, 3 sH, 4 sV.  Records and their cotangents are
 * (B, nt, nrec, nfield).
 *
 * What each function restates (reference paths, relative to the project root):
 *   stiffness         src/sweep/csrc/cuda/common/derived_models.cu:40-53
 *   velocity step     src/sweep/csrc/cuda/equations/acoustic_vti_1st_3d/
 *                     kernels.cuh:150-210 (D+ of sH along x and y, of sV along
 *                     z; the memories m_sHx / m_sHy / m_sVz on the half-cell
 *                     profiles outside the physical box)
 *   stress step       kernels.cuh:275-333 (D- of vx / vy / vz, memories
 *                     m_vxx / m_vyy / m_vzz; dh = dvx/dx + dvy/dy,
 *                     sH += dt (c11 dh + c13 dvz/dz), sV += dt (c13 dh + c33 dvz/dz))
 *   reverse (NOPML)   kernels.cuh:400-490 (box pad + M + 1 per face)
 *   adjoint           kernels.cuh:606-760: p = (ph, ph, pv) with
 *                     ph = c11 lsH + c13 lsV, pv = c13 lsH + c33 lsV, through
 *                     the stress step's transposed CPML, then lv += -dt D+(p);
 *                     q = inv_rho lv through the velocity step's transposed
 *                     CPML, then lsH += -dt (D-x qx + D-y qy), lsV += -dt D-z qz
 *   gradient          kernels.cuh:940-1000 (c11 / c33 / c13 / inv_rho
 *                     gradients on the physical box, chained to vp, epsilon,
 *                     delta, rho)
 *   step order        acoustic_vti_1st_3d/forward.cu (velocity, stress, source,
 *                     band save, record), backward.cu (residual, source
 *                     removal, stress reverse, stress bands, adjoint A,
 *                     gradient, adjoint B, velocity reverse, velocity bands;
 *                     it = nt - 1 .. 1)
 *   bands             src/sweep/csrc/cuda/common/boundary/strip.cuh:136-175
 *                     (per face a band M + 1 wide from M cells outside the
 *                     box, spanning the box along the other two axes; each
 *                     cell restored once, which writes the same values as the
 *                     reference's face-by-face restore)
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
    int B, nz, ny, nx, nt, M;
    int pad[6];                 /* z_lo, z_hi, y_lo, y_hi, x_lo, x_hi PML widths */
    REAL dt, dz, dy, dx;
    const REAL* c;              /* c[1..M] staggered coefficients */
    const REAL *az, *bz, *azh, *bzh, *ay, *by, *ayh, *byh, *ax, *bx, *axh, *bxh;
    const REAL *vp, *eps, *dlt, *rho;
    i64 ms;                     /* model stride between shots (0 = shared) */
    int nsrc; const int* src; const REAL* wavelet; int nsf; const int* sf;
    int nrec; const int* rec; int nrf; const int* rf;
} VTI3;

enum { VX, VY, VZ, SH, SV, M_SHX, M_SHY, M_SVZ, M_VXX, M_VYY, M_VZZ, NF };

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

static i64 at(const VTI3* p, const int* l)
{
    if (l[0] < 0 || l[0] >= p->nx || l[1] < 0 || l[1] >= p->ny || l[2] < 0 || l[2] >= p->nz) return -1;
    return ((i64)l[2] * p->ny + l[1]) * p->nx + l[0];
}

/* outside the physical box (PML pad plus the stencil halo) on any axis */
static inline int in_pml(const VTI3* p, int ix, int iy, int iz)
{
    const int h = p->M;
    return ix < p->pad[4] + h || ix >= p->nx - p->pad[5] - h || iy < p->pad[2] + h || iy >= p->ny - p->pad[3] - h ||
           iz < p->pad[0] + h || iz >= p->nz - p->pad[1] - h;
}

static inline int in_core(const VTI3* p, int ix, int iy, int iz)
{
    const int M = p->M;
    return ix >= M && ix < p->nx - M && iy >= M && iy < p->ny - M && iz >= M && iz < p->nz - M;
}

static void stiffness(const VTI3* p, int b, REAL* c11, REAL* c33, REAL* c13, REAL* irho)
{
    const i64 n = (i64)p->nz * p->ny * p->nx;
    const REAL *v = p->vp + b * p->ms, *e = p->eps + b * p->ms, *d = p->dlt + b * p->ms, *r = p->rho + b * p->ms;
    for (i64 i = 0; i < n; ++i) {
        const REAL rv2 = r[i] * (v[i] * v[i]);
        c33[i] = rv2;
        c11[i] = rv2 * (R(1) + R(2) * e[i]);
        c13[i] = rv2 * (REAL)sqrt((double)(R(1) + R(2) * d[i]));
        irho[i] = R(1) / r[i];
    }
}

#define FOR_CORE(p)                                          \
    for (int iz = (p)->M; iz < (p)->nz - (p)->M; ++iz)        \
        for (int iy = (p)->M; iy < (p)->ny - (p)->M; ++iy)    \
            for (int ix = (p)->M; ix < (p)->nx - (p)->M; ++ix)

static void velocity_step(const VTI3* p, REAL** F, const REAL* irho)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    #pragma omp parallel for schedule(static)
    FOR_CORE(p) {
        const i64 i = iz * sz + iy * sy + ix;
        REAL dsx = dplus(F[SH], i, 1, M, p->c, R(1) / p->dx);
        REAL dsy = dplus(F[SH], i, sy, M, p->c, R(1) / p->dy);
        REAL dsz = dplus(F[SV], i, sz, M, p->c, R(1) / p->dz);
        if (in_pml(p, ix, iy, iz)) {
            F[M_SHX][i] = p->axh[ix] * F[M_SHX][i] + p->bxh[ix] * dsx;
            dsx = dsx + F[M_SHX][i];
            F[M_SHY][i] = p->ayh[iy] * F[M_SHY][i] + p->byh[iy] * dsy;
            dsy = dsy + F[M_SHY][i];
            F[M_SVZ][i] = p->azh[iz] * F[M_SVZ][i] + p->bzh[iz] * dsz;
            dsz = dsz + F[M_SVZ][i];
        }
        const REAL k = p->dt * irho[i];
        F[VX][i] = F[VX][i] + k * dsx;
        F[VY][i] = F[VY][i] + k * dsy;
        F[VZ][i] = F[VZ][i] + k * dsz;
    }
}

static void stress_step(const VTI3* p, REAL** F, const REAL* c11, const REAL* c33, const REAL* c13)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    #pragma omp parallel for schedule(static)
    FOR_CORE(p) {
        const i64 i = iz * sz + iy * sy + ix;
        REAL dvx = dminus(F[VX], i, 1, M, p->c, R(1) / p->dx);
        REAL dvy = dminus(F[VY], i, sy, M, p->c, R(1) / p->dy);
        REAL dvz = dminus(F[VZ], i, sz, M, p->c, R(1) / p->dz);
        if (in_pml(p, ix, iy, iz)) {
            F[M_VXX][i] = p->ax[ix] * F[M_VXX][i] + p->bx[ix] * dvx;
            dvx = dvx + F[M_VXX][i];
            F[M_VYY][i] = p->ay[iy] * F[M_VYY][i] + p->by[iy] * dvy;
            dvy = dvy + F[M_VYY][i];
            F[M_VZZ][i] = p->az[iz] * F[M_VZZ][i] + p->bz[iz] * dvz;
            dvz = dvz + F[M_VZZ][i];
        }
        const REAL dh = dvx + dvy;
        F[SH][i] = F[SH][i] + p->dt * (c11[i] * dh + c13[i] * dvz);
        F[SV][i] = F[SV][i] + p->dt * (c13[i] * dh + c33[i] * dvz);
    }
}

static void inject(const VTI3* p, int b, REAL* u, int it, REAL sign)
{
    for (int s = 0; s < p->nsrc; ++s) {
        const i64 c = at(p, p->src + (b * p->nsrc + s) * 3);
        if (c < 0) continue;
        u[c] += sign * p->wavelet[((i64)b * p->nsrc + s) * p->nt + it];
    }
}

/* the band cells of one shot grid, each once, in grid order */
static int band_cells(const VTI3* p, int* out)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const int z0 = p->pad[0] + M, z1 = nz - p->pad[1] - M, y0 = p->pad[2] + M, y1 = ny - p->pad[3] - M;
    const int x0 = p->pad[4] + M, x1 = nx - p->pad[5] - M;
    int n = 0;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const int zin = z >= z0 && z < z1, yin = y >= y0 && y < y1, xin = x >= x0 && x < x1;
                const int zb = (z >= z0 - M && z <= z0) || (z >= z1 - 1 && z <= z1 - 1 + M);
                const int yb = (y >= y0 - M && y <= y0) || (y >= y1 - 1 && y <= y1 - 1 + M);
                const int xb = (x >= x0 - M && x <= x0) || (x >= x1 - 1 && x <= x1 - 1 + M);
                if ((zb && yin && xin) || (zin && yb && xin) || (zin && yin && xb)) {
                    if (out) out[n] = (z * ny + y) * nx + x;
                    ++n;
                }
            }
    return n;
}

long long oracle_vti3d_tape_len(int B, int nz, int ny, int nx, int nt, int M, const int* pad)
{
    VTI3 p; memset(&p, 0, sizeof p);
    p.B = B; p.nz = nz; p.ny = ny; p.nx = nx; p.nt = nt; p.M = M;
    for (int k = 0; k < 6; ++k) p.pad[k] = pad[k];
    return (long long)nt * B * 5 * band_cells(&p, NULL) + 5LL * B * nz * ny * nx;
}

static VTI3 setup(int B, int nz, int ny, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dy, REAL dx,
                  const REAL* coef, const REAL* prof, const REAL* vp, const REAL* eps, const REAL* dlt,
                  const REAL* rho, i64 m_stride, int nsrc, const int* src, const REAL* wavelet, int nsf,
                  const int* sfields, int nrec, const int* rec, int nrf, const int* rfields)
{
    VTI3 p;
    memset(&p, 0, sizeof p);
    p.B = B; p.nz = nz; p.ny = ny; p.nx = nx; p.nt = nt; p.M = M;
    for (int k = 0; k < 6; ++k) p.pad[k] = pad[k];
    p.dt = dt; p.dz = dz; p.dy = dy; p.dx = dx; p.c = coef;
    const REAL* q = prof;
    p.az = q; p.bz = q + nz; p.azh = q + 2 * nz; p.bzh = q + 3 * nz; q += 4 * nz;
    p.ay = q; p.by = q + ny; p.ayh = q + 2 * ny; p.byh = q + 3 * ny; q += 4 * ny;
    p.ax = q; p.bx = q + nx; p.axh = q + 2 * nx; p.bxh = q + 3 * nx;
    p.vp = vp; p.eps = eps; p.dlt = dlt; p.rho = rho; p.ms = m_stride;
    p.nsrc = nsrc; p.src = src; p.wavelet = wavelet; p.nsf = nsf; p.sf = sfields;
    p.nrec = nrec; p.rec = rec; p.nrf = nrf; p.rf = rfields;
    return p;
}

#define VTI3_ARGS                                                                                     \
    int B, int nz, int ny, int nx, int nt, int M, const int *pad, REAL dt, REAL dz, REAL dy, REAL dx,  \
        const REAL *coef, const REAL *prof, const REAL *vp, const REAL *eps, const REAL *dlt,          \
        const REAL *rho, i64 m_stride, int nsrc, const int *src, const REAL *wavelet, int nsf,         \
        const int *sfields, int nrec, const int *rec, int nrf, const int *rfields
#define VTI3_SETUP                                                                                     \
    VTI3 p = setup(B, nz, ny, nx, nt, M, pad, dt, dz, dy, dx, coef, prof, vp, eps, dlt, rho, m_stride, \
                   nsrc, src, wavelet, nsf, sfields, nrec, rec, nrf, rfields)

int oracle_vti3d_forward(VTI3_ARGS, REAL* record, REAL* tape)
{
    VTI3_SETUP;
    const i64 n = (i64)nz * ny * nx;
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
                for (int f = 0; f < 5; ++f) {
                    REAL* dst = tape + (((i64)it * B + b) * 5 + f) * ns;
                    for (int c = 0; c < ns; ++c) dst[c] = F[f][cells[c]];
                }
            for (int r = 0; r < nrec; ++r) {
                const i64 c = at(&p, rec + (b * nrec + r) * 3);
                if (c < 0) continue;
                for (int k = 0; k < nrf; ++k) record[(((i64)b * nt + it) * nrec + r) * nrf + k] = F[rfields[k]][c];
            }
        }
        if (tape)
            for (int f = 0; f < 5; ++f)
                memcpy(tape + (i64)nt * B * 5 * ns + ((i64)b * 5 + f) * n, F[f], sizeof(REAL) * n);
    }
    free(buf); free(cells);
    return 0;
}

/* reverse (NOPML) steps on the box pad + M + 1 per face (kernels.cuh:400-490) */
#define FOR_REV(p)                                                                    \
    for (int iz = (p)->pad[0] + (p)->M + 1; iz < (p)->nz - ((p)->pad[1] + (p)->M + 1); ++iz)     \
        for (int iy = (p)->pad[2] + (p)->M + 1; iy < (p)->ny - ((p)->pad[3] + (p)->M + 1); ++iy) \
            for (int ix = (p)->pad[4] + (p)->M + 1; ix < (p)->nx - ((p)->pad[5] + (p)->M + 1); ++ix)

static void stress_reverse(const VTI3* p, REAL** F, const REAL* c11, const REAL* c33, const REAL* c13)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    #pragma omp parallel for schedule(static)
    FOR_REV(p) {
        const i64 i = iz * sz + iy * sy + ix;
        const REAL dvx = dminus(F[VX], i, 1, M, p->c, R(1) / p->dx);
        const REAL dvy = dminus(F[VY], i, sy, M, p->c, R(1) / p->dy);
        const REAL dvz = dminus(F[VZ], i, sz, M, p->c, R(1) / p->dz);
        const REAL dh = dvx + dvy;
        F[SH][i] = F[SH][i] - p->dt * (c11[i] * dh + c13[i] * dvz);
        F[SV][i] = F[SV][i] - p->dt * (c13[i] * dh + c33[i] * dvz);
    }
}

static void velocity_reverse(const VTI3* p, REAL** F, const REAL* irho)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    #pragma omp parallel for schedule(static)
    FOR_REV(p) {
        const i64 i = iz * sz + iy * sy + ix;
        const REAL k = p->dt * irho[i];
        F[VX][i] = F[VX][i] - k * dplus(F[SH], i, 1, M, p->c, R(1) / p->dx);
        F[VY][i] = F[VY][i] - k * dplus(F[SH], i, sy, M, p->c, R(1) / p->dy);
        F[VZ][i] = F[VZ][i] - k * dplus(F[SV], i, sz, M, p->c, R(1) / p->dz);
    }
}

/* adjoint half-step A: p = (ph, ph, pv) through the stress step's
 * transposed CPML on every cell, then lambda_v += -dt D+(p) on the core */
static void adjoint_A(const VTI3* p, REAL** A, REAL* px, REAL* py, REAL* pz, const REAL* c11, const REAL* c33,
                      const REAL* c13)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < p->nz; ++iz)
        for (int iy = 0; iy < p->ny; ++iy)
            for (int ix = 0; ix < p->nx; ++ix) {
                const i64 i = iz * sz + iy * sy + ix;
                const REAL ph = c11[i] * A[SH][i] + c13[i] * A[SV][i];
                const REAL pv = c13[i] * A[SH][i] + c33[i] * A[SV][i];
                REAL qx = ph, qy = ph, qz = pv;
                if (in_core(p, ix, iy, iz) && in_pml(p, ix, iy, iz)) {
                    const REAL tx = A[M_VXX][i] + qx, ty = A[M_VYY][i] + qy, tz = A[M_VZZ][i] + qz;
                    qx = qx + p->bx[ix] * tx;
                    qy = qy + p->by[iy] * ty;
                    qz = qz + p->bz[iz] * tz;
                    A[M_VXX][i] = p->ax[ix] * tx;
                    A[M_VYY][i] = p->ay[iy] * ty;
                    A[M_VZZ][i] = p->az[iz] * tz;
                }
                px[i] = qx;
                py[i] = qy;
                pz[i] = qz;
            }
    #pragma omp parallel for schedule(static)
    FOR_CORE(p) {
        const i64 i = iz * sz + iy * sy + ix;
        A[VX][i] = A[VX][i] + (-p->dt) * dplus(px, i, 1, M, p->c, R(1) / p->dx);
        A[VY][i] = A[VY][i] + (-p->dt) * dplus(py, i, sy, M, p->c, R(1) / p->dy);
        A[VZ][i] = A[VZ][i] + (-p->dt) * dplus(pz, i, sz, M, p->c, R(1) / p->dz);
    }
}

/* adjoint half-step B: q = inv_rho lambda_v through the velocity step's
 * transposed CPML, then lambda_sH += -dt (D-x qx + D-y qy),
 * lambda_sV += -dt D-z qz on the core */
static void adjoint_B(const VTI3* p, REAL** A, REAL* qx_, REAL* qy_, REAL* qz_, const REAL* irho)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < p->nz; ++iz)
        for (int iy = 0; iy < p->ny; ++iy)
            for (int ix = 0; ix < p->nx; ++ix) {
                const i64 i = iz * sz + iy * sy + ix;
                REAL qx = irho[i] * A[VX][i], qy = irho[i] * A[VY][i], qz = irho[i] * A[VZ][i];
                if (in_core(p, ix, iy, iz) && in_pml(p, ix, iy, iz)) {
                    const REAL tx = A[M_SHX][i] + qx, ty = A[M_SHY][i] + qy, tz = A[M_SVZ][i] + qz;
                    qx = qx + p->bxh[ix] * tx;
                    qy = qy + p->byh[iy] * ty;
                    qz = qz + p->bzh[iz] * tz;
                    A[M_SHX][i] = p->axh[ix] * tx;
                    A[M_SHY][i] = p->ayh[iy] * ty;
                    A[M_SVZ][i] = p->azh[iz] * tz;
                }
                qx_[i] = qx;
                qy_[i] = qy;
                qz_[i] = qz;
            }
    #pragma omp parallel for schedule(static)
    FOR_CORE(p) {
        const i64 i = iz * sz + iy * sy + ix;
        const REAL dqx = dminus(qx_, i, 1, M, p->c, R(1) / p->dx);
        const REAL dqy = dminus(qy_, i, sy, M, p->c, R(1) / p->dy);
        A[SH][i] = A[SH][i] + (-p->dt) * (dqx + dqy);
        A[SV][i] = A[SV][i] + (-p->dt) * dminus(qz_, i, sz, M, p->c, R(1) / p->dz);
    }
}

/* gradient of one step on the physical box: forward velocities at the end
 * of the step, stresses at its start, the adjoint between half-steps A and B */
static void gradient(const VTI3* p, int b, REAL** F, REAL** A, REAL* gvp, REAL* geps, REAL* gdlt, REAL* grho)
{
    const i64 sy = p->nx, sz = (i64)p->ny * p->nx;
    const int M = p->M;
    const REAL *vp = p->vp + b * p->ms, *ep = p->eps + b * p->ms, *dl = p->dlt + b * p->ms, *rh = p->rho + b * p->ms;
    const int z0 = p->pad[0] + M, z1 = p->nz - p->pad[1] - M, y0 = p->pad[2] + M, y1 = p->ny - p->pad[3] - M;
    const int x0 = p->pad[4] + M, x1 = p->nx - p->pad[5] - M;
    const REAL dt = p->dt;
    #pragma omp parallel for schedule(static)
    for (int iz = z0; iz < z1; ++iz)
        for (int iy = y0; iy < y1; ++iy)
            for (int ix = x0; ix < x1; ++ix) {
                if (!in_core(p, ix, iy, iz)) continue;
                const i64 i = iz * sz + iy * sy + ix;
                const REAL dvx = dminus(F[VX], i, 1, M, p->c, R(1) / p->dx);
                const REAL dvy = dminus(F[VY], i, sy, M, p->c, R(1) / p->dy);
                const REAL dvz = dminus(F[VZ], i, sz, M, p->c, R(1) / p->dz);
                const REAL dsx = dplus(F[SH], i, 1, M, p->c, R(1) / p->dx);
                const REAL dsy = dplus(F[SH], i, sy, M, p->c, R(1) / p->dy);
                const REAL dsz = dplus(F[SV], i, sz, M, p->c, R(1) / p->dz);
                const REAL lsh = A[SH][i], lsv = A[SV][i];
                const REAL dh = dvx + dvy;
                const REAL g11 = dt * lsh * dh;
                const REAL g33 = dt * lsv * dvz;
                const REAL g13 = dt * (lsh * dvz + lsv * dh);
                const REAL gir = dt * (A[VX][i] * dsx + A[VY][i] * dsy + A[VZ][i] * dsz);
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

int oracle_vti3d_backward(VTI3_ARGS, const REAL* adj, const REAL* tape, REAL* grad_vp, REAL* grad_eps,
                          REAL* grad_dlt, REAL* grad_rho)
{
    VTI3_SETUP;
    const i64 n = (i64)nz * ny * nx;
    const int ns = band_cells(&p, NULL);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    const int nbuf = 5 + NF + 3 + 4;
    REAL* buf = (REAL*)calloc((size_t)n * nbuf, sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    band_cells(&p, cells);
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * nbuf);
        REAL *F[5], *A[NF];
        for (int f = 0; f < 5; ++f) F[f] = buf + f * n;
        for (int f = 0; f < NF; ++f) A[f] = buf + (5 + f) * n;
        REAL *s0 = buf + (5 + NF) * n, *s1 = buf + (6 + NF) * n, *s2 = buf + (7 + NF) * n;
        REAL *c11 = buf + (8 + NF) * n, *c33 = buf + (9 + NF) * n, *c13 = buf + (10 + NF) * n;
        REAL* irho = buf + (11 + NF) * n;
        stiffness(&p, b, c11, c33, c13, irho);
        REAL *gvp = grad_vp + b * m_stride, *geps = grad_eps + b * m_stride;
        REAL *gdlt = grad_dlt + b * m_stride, *grho = grad_rho + b * m_stride;
        for (int f = 0; f < 5; ++f)
            memcpy(F[f], tape + (i64)nt * B * 5 * ns + ((i64)b * 5 + f) * n, sizeof(REAL) * n);
        for (int it = nt - 1; it >= 1; --it) {
            /* residuals into the adjoint fields, unsigned */
            for (int k = 0; k < nrf; ++k)
                for (int r = 0; r < nrec; ++r) {
                    const i64 c = at(&p, rec + (b * nrec + r) * 3);
                    if (c < 0) continue;
                    A[rfields[k]][c] += adj[(((i64)b * nt + it) * nrec + r) * nrf + k];
                }
            for (int k = 0; k < nsf; ++k) inject(&p, b, F[sfields[k]], it, R(-1));
            stress_reverse(&p, F, c11, c33, c13);
            for (int f = SH; f <= SV; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 5 + f) * ns;
                for (int c = 0; c < ns; ++c) F[f][cells[c]] = s[c];
            }
            adjoint_A(&p, A, s0, s1, s2, c11, c33, c13);
            gradient(&p, b, F, A, gvp, geps, gdlt, grho);
            adjoint_B(&p, A, s0, s1, s2, irho);
            velocity_reverse(&p, F, irho);
            for (int f = VX; f <= VZ; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 5 + f) * ns;
                for (int c = 0; c < ns; ++c) F[f][cells[c]] = s[c];
            }
        }
    }
    free(buf); free(cells);
    return 0;
}
