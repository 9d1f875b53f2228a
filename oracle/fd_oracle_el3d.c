/*
 * fd_oracle_el3d.c -- CPU restatement of the reference's compiled (impl='c')
 * 3-D isotropic elastic path (velocity-stress, staggered grid), used ONLY as
 * test infrastructure: the parity checker of the CUDA library.  It is never
 * linked into, loaded by or called from the product library.
 *
 * Built with REAL=float and REAL=double by oracle/Makefile, -ffp-contract=off.
 *
 * Layout: every field is (B, nz, ny, nx), x fastest, on the runtime grid
 * (physical + PML pad + stencil halo M per face).  Coordinates are runtime
 * (x, y, z) int32 triples; off-grid ones are skipped.  Records and their
 * cotangents are (B, nt, nrec, nfield).  Field indices: 0 vx, 1 vy, 2 vz,
 * 3 sxx, 4 syy, 5 szz, 6 sxy, 7 sxz, 8 syz (reference
 * src/sweep/csrc/cuda/common/elastic.h:736-749).
 *
 * What each function restates (reference paths, relative to the project root,
 * under src/sweep/csrc/cuda/):
 *   velocity step     equations/elastic3d/kernels.cuh:104-248 (the CPML branch
 *                     outside the physical box shrunk by one cell)
 *   stress step       equations/elastic3d/kernels.cuh:290-483
 *   reverse (NOPML)   equations/elastic3d/kernels.cuh:536-768 (band pad+M+1)
 *   velocity adjoint  equations/elastic3d/kernels.cuh:959-1236 (prepare, apply)
 *   stress adjoint    equations/elastic3d/kernels.cuh:1367-1780 (prepare with
 *                     the fused vp / vs / rho imaging, apply)
 *   strips            equations/elastic3d/driver_traits.cuh:265-290 (nine
 *                     fields, width M+1 at offset -M per face)
 *   reverse order     equations/elastic3d/driver_traits.cuh:680-905,
 *                     524-640 (source and receiver rho corrections, signed
 *                     residuals: stress -1, velocity +1)
 *   free top face     common/elastic_free_surface.cuh:723-952 (the full
 *                     stencil over image values, its exact transpose), and
 *                     elastic3d/kernels.cuh:360-372, 1421-1470, 1489-1499
 *                     (Robertsson sxx / syy, szz = 0, their transposes and
 *                     the surface row's image)
 */
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
    const REAL *vp, *vs, *rho;
    i64 ms;                     /* model stride between shots (0 = shared) */
    int nsrc; const int* src; const REAL* wavelet; int nsf; const int* sf;
    int nrec; const int* rec; int nrf; const int* rf;
    int fs;                     /* 1: traction-free top face (pad[0] == 0) */
} EL3;

enum { VX, VY, VZ, SXX, SYY, SZZ, SXY, SXZ, SYZ,
       M_VXX, M_VXY, M_VXZ, M_VYX, M_VYY, M_VYZ, M_VZX, M_VZY, M_VZZ,
       M_SXXX, M_SZZZ, M_SXYX, M_SXYY, M_SXZX, M_SXZZ, M_SYYY, M_SYZY, M_SYZZ, NF };

/* D+ / D- along stride s: sum_k c_k (u[i+k s] - u[i-(k-1) s]) and
 * sum_k c_k (u[i+(k-1) s] - u[i-k s]), times 1/h. */
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

/* ---- traction-free top face -----------------------------------------------
 * The surface is the first physical row top = pad[0] + M; the rows above it
 * are air, read by z-derivatives as the image of the row mirrored about the
 * surface (about top for integer fields, top - 1/2 for fields half a cell
 * below, negated for odd fields).  In 3-D the full stencil runs over those
 * images (no reduced rows near the surface). */
static inline REAL fs_at3(const EL3* p, const REAL* u, i64 base, i64 sz, int k, int odd, int half)
{
    const int top = p->pad[0] + p->M;
    if (k < top) {
        const int m = half ? 2 * top - 1 - k : 2 * top - k;
        const REAL v = u[base + (i64)m * sz];
        return odd ? -v : v;
    }
    return u[base + (i64)k * sz];
}

/* z-derivative at row iz of the column through `base` (row 0): fwd = 1 the
 * D+ form, 0 the D- form; the plain stencil without a free surface. */
static REAL dz3(const EL3* p, const REAL* u, i64 base, int iz, int fwd, int odd, int half)
{
    const i64 sz = (i64)p->nx * p->ny;
    const i64 i = base + (i64)iz * sz;
    if (!p->fs) return fwd ? dplus(u, i, sz, p->M, p->c, R(1) / p->dz) : dminus(u, i, sz, p->M, p->c, R(1) / p->dz);
    REAL g = R(0);
    for (int k = 1; k <= p->M; ++k) {
        const REAL up = fwd ? fs_at3(p, u, base, sz, iz + k, odd, half) : fs_at3(p, u, base, sz, iz + k - 1, odd, half);
        const REAL um = fwd ? fs_at3(p, u, base, sz, iz - k + 1, odd, half) : fs_at3(p, u, base, sz, iz - k, odd, half);
        g = g + p->c[k] * (up - um);
    }
    return g / p->dz;
}

/* Exact transpose of dz3 (negated: the D- form for a D+ forward and vice
 * versa): the direct taps from rows at or below the surface, and each air
 * row's image folded back with the field's parity. */
static REAL adz3(const EL3* p, const REAL* q, i64 base, int iz, int fwd, int odd, int half)
{
    const i64 sz = (i64)p->nx * p->ny;
    const i64 i = base + (i64)iz * sz;
    if (!p->fs) return fwd ? dminus(q, i, sz, p->M, p->c, R(1) / p->dz) : dplus(q, i, sz, p->M, p->c, R(1) / p->dz);
    const int top = p->pad[0] + p->M, lo = half ? top - 1 : top;
    const REAL parity = odd ? R(-1) : R(1);
    REAL g = R(0);
    for (int k = 1; k <= p->M; ++k) {
        const int m = k - 1;
        const int jp = fwd ? iz + m : iz + m + 1;
        const int jm = fwd ? iz - m - 1 : iz - m;
        const int jg = fwd ? (half ? 2 * top - 1 + m - iz : 2 * top + m - iz)
                           : (half ? 2 * top + m - iz : 2 * top + m + 1 - iz);
        if (jp >= top && jp < p->nz) g = g + p->c[k] * q[base + (i64)jp * sz];
        if (jm >= top) g = g - p->c[k] * q[base + (i64)jm * sz];
        if (iz > lo && jg >= top) g = g + p->c[k] * parity * q[base + (i64)jg * sz];
    }
    return g / p->dz;
}

static inline int surf_row(const EL3* p, int iz) { return p->fs && iz == p->pad[0] + p->M; }

typedef struct { int z0, z1, y0, y1, x0, x1; } BOX;

static BOX box_of(const EL3* p)
{
    BOX b;
    b.z0 = p->pad[0] + p->M; b.z1 = p->nz - p->pad[1] - p->M;
    b.y0 = p->pad[2] + p->M; b.y1 = p->ny - p->pad[3] - p->M;
    b.x0 = p->pad[4] + p->M; b.x1 = p->nx - p->pad[5] - p->M;
    return b;
}

/* The cells that skip the CPML branch: the physical box shrunk by one cell
 * (kernels.cuh:159-166); also the reverse (NOPML) region (band pad + M + 1). */
static inline int interior(const BOX* b, int ix, int iy, int iz)
{
    return ix >= b->x0 + 1 && ix < b->x1 - 1 && iy >= b->y0 + 1 && iy < b->y1 - 1 && iz >= b->z0 + 1 &&
           iz < b->z1 - 1;
}

static void lame(const EL3* p, int b, REAL* lam, REAL* mu)
{
    const i64 n = (i64)p->nz * p->ny * p->nx;
    const REAL *v = p->vp + b * p->ms, *s = p->vs + b * p->ms, *r = p->rho + b * p->ms;
    for (i64 i = 0; i < n; ++i) {
        mu[i] = (r[i] * s[i]) * s[i];
        lam[i] = r[i] * ((v[i] * v[i]) - ((R(2) * s[i]) * s[i]));
    }
}

#define LOOP_CORE                                                               \
    _Pragma("omp parallel for collapse(2) schedule(static)")                    \
    for (int iz = M; iz < nz - M; ++iz)                                        \
        for (int iy = M; iy < ny - M; ++iy)                                    \
            for (int ix = M; ix < nx - M; ++ix)

static void velocity_step(const EL3* p, int b, REAL** F)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL* rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy;
    const BOX bx_ = box_of(p);
    LOOP_CORE {
        const i64 i = iz * sz + iy * sy + ix;
        const i64 col = i - iz * sz;
        REAL dsxx_dx = dplus(F[SXX], i, 1, M, p->c, ix_);
        REAL dsxy_dy = dminus(F[SXY], i, sy, M, p->c, iy_);
        REAL dsxz_dz = dz3(p, F[SXZ], col, iz, 0, 1, 1);
        REAL dsxy_dx = dminus(F[SXY], i, 1, M, p->c, ix_);
        REAL dsyy_dy = dplus(F[SYY], i, sy, M, p->c, iy_);
        REAL dsyz_dz = dz3(p, F[SYZ], col, iz, 0, 1, 1);
        REAL dsxz_dx = dminus(F[SXZ], i, 1, M, p->c, ix_);
        REAL dsyz_dy = dminus(F[SYZ], i, sy, M, p->c, iy_);
        REAL dszz_dz = dz3(p, F[SZZ], col, iz, 1, 1, 0);
        const REAL inv_rho = R(1) / rho[i];
        if (!interior(&bx_, ix, iy, iz)) {
            REAL m;
#define MEM(slot, a, bb, d) m = (a) * F[slot][i] + (bb) * d; F[slot][i] = m; d = d + m
            MEM(M_SZZZ, p->azh[iz], p->bzh[iz], dszz_dz);
            MEM(M_SXZX, p->ax[ix], p->bx[ix], dsxz_dx);
            MEM(M_SXZZ, p->az[iz], p->bz[iz], dsxz_dz);
            MEM(M_SXXX, p->axh[ix], p->bxh[ix], dsxx_dx);
            MEM(M_SXYY, p->ay[iy], p->by[iy], dsxy_dy);
            MEM(M_SXYX, p->ax[ix], p->bx[ix], dsxy_dx);
            MEM(M_SYYY, p->ayh[iy], p->byh[iy], dsyy_dy);
            MEM(M_SYZZ, p->az[iz], p->bz[iz], dsyz_dz);
            MEM(M_SYZY, p->ay[iy], p->by[iy], dsyz_dy);
        }
        F[VX][i] = F[VX][i] + (p->dt * inv_rho) * ((dsxx_dx + dsxy_dy) + dsxz_dz);
        F[VY][i] = F[VY][i] + (p->dt * inv_rho) * ((dsxy_dx + dsyy_dy) + dsyz_dz);
        F[VZ][i] = F[VZ][i] + (p->dt * inv_rho) * ((dsxz_dx + dsyz_dy) + dszz_dz);
    }
}

static void stress_step(const EL3* p, REAL** F, const REAL* lam_, const REAL* mu_)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy;
    const BOX bx_ = box_of(p);
    LOOP_CORE {
        const i64 i = iz * sz + iy * sy + ix, col = i - iz * sz;
        REAL dvx_dx = dminus(F[VX], i, 1, M, p->c, ix_);
        REAL dvx_dy = dplus(F[VX], i, sy, M, p->c, iy_);
        REAL dvx_dz = dz3(p, F[VX], col, iz, 1, 0, 0);
        REAL dvy_dx = dplus(F[VY], i, 1, M, p->c, ix_);
        REAL dvy_dy = dminus(F[VY], i, sy, M, p->c, iy_);
        REAL dvy_dz = dz3(p, F[VY], col, iz, 1, 0, 0);
        REAL dvz_dx = dplus(F[VZ], i, 1, M, p->c, ix_);
        REAL dvz_dy = dplus(F[VZ], i, sy, M, p->c, iy_);
        REAL dvz_dz = dz3(p, F[VZ], col, iz, 0, 1, 1);
        const REAL lam = lam_[i], mu = mu_[i];
        if (!interior(&bx_, ix, iy, iz)) {
            REAL m;
            MEM(M_VZZ, p->az[iz], p->bz[iz], dvz_dz);
            MEM(M_VYY, p->ay[iy], p->by[iy], dvy_dy);
            MEM(M_VXX, p->ax[ix], p->bx[ix], dvx_dx);
            MEM(M_VXZ, p->azh[iz], p->bzh[iz], dvx_dz);
            MEM(M_VZX, p->axh[ix], p->bxh[ix], dvz_dx);
            MEM(M_VXY, p->ayh[iy], p->byh[iy], dvx_dy);
            MEM(M_VYX, p->axh[ix], p->bxh[ix], dvy_dx);
            MEM(M_VYZ, p->azh[iz], p->bzh[iz], dvy_dz);
            MEM(M_VZY, p->ayh[iy], p->byh[iy], dvz_dy);
#undef MEM
        }
        const REAL div = (dvx_dx + dvy_dy) + dvz_dz;
        F[SXX][i] = F[SXX][i] + p->dt * (lam * div + (R(2) * mu) * dvx_dx);
        F[SYY][i] = F[SYY][i] + p->dt * (lam * div + (R(2) * mu) * dvy_dy);
        F[SZZ][i] = F[SZZ][i] + p->dt * (lam * div + (R(2) * mu) * dvz_dz);
        F[SXY][i] = F[SXY][i] + (p->dt * mu) * (dvx_dy + dvy_dx);
        F[SXZ][i] = F[SXZ][i] + (p->dt * mu) * (dvx_dz + dvz_dx);
        F[SYZ][i] = F[SYZ][i] + (p->dt * mu) * (dvy_dz + dvz_dy);
        if (surf_row(p, iz)) {   /* Robertsson sxx / syy, then szz = 0 (kernels.cuh:360-372) */
            const REAL rob = (-p->dt) * lam * ((lam / (lam + R(2) * mu)) * (dvx_dx + dvy_dy) + dvz_dz);
            F[SXX][i] = F[SXX][i] + rob;
            F[SYY][i] = F[SYY][i] + rob;
            F[SZZ][i] = R(0);
        }
    }
}

static inline int on_grid(const EL3* p, const int* loc, i64* cell)
{
    const int ix = loc[0], iy = loc[1], iz = loc[2];
    if (ix < 0 || ix >= p->nx || iy < 0 || iy >= p->ny || iz < 0 || iz >= p->nz) return 0;
    *cell = ((i64)iz * p->ny + iy) * p->nx + ix;
    return 1;
}

static void inject(const EL3* p, int b, REAL* u, int it, REAL sign)
{
    for (int s = 0; s < p->nsrc; ++s) {
        i64 c;
        if (!on_grid(p, p->src + ((i64)b * p->nsrc + s) * 3, &c)) continue;
        u[c] += sign * p->wavelet[((i64)b * p->nsrc + s) * p->nt + it];
    }
}

/* Boundary-saving band cells: per face a band M+1 wide starting M cells
 * outside the physical box, spanning the box along the other two axes.
 * Cells of two bands are listed twice (their saved values agree). */
static int band_cells(const EL3* p, int* out)
{
    const BOX b = box_of(p);
    const int w = p->M + 1, M = p->M, nx = p->nx, ny = p->ny;
    int n = 0;
#define PUT(z, y, x) do { if (out) out[n] = ((z) * ny + (y)) * nx + (x); ++n; } while (0)
    for (int z = b.z0 - M; z < b.z0 - M + w; ++z) for (int y = b.y0; y < b.y1; ++y) for (int x = b.x0; x < b.x1; ++x) PUT(z, y, x);
    for (int z = b.z1 + M - w; z < b.z1 + M; ++z) for (int y = b.y0; y < b.y1; ++y) for (int x = b.x0; x < b.x1; ++x) PUT(z, y, x);
    for (int z = b.z0; z < b.z1; ++z) for (int y = b.y0 - M; y < b.y0 - M + w; ++y) for (int x = b.x0; x < b.x1; ++x) PUT(z, y, x);
    for (int z = b.z0; z < b.z1; ++z) for (int y = b.y1 + M - w; y < b.y1 + M; ++y) for (int x = b.x0; x < b.x1; ++x) PUT(z, y, x);
    for (int z = b.z0; z < b.z1; ++z) for (int y = b.y0; y < b.y1; ++y) for (int x = b.x0 - M; x < b.x0 - M + w; ++x) PUT(z, y, x);
    for (int z = b.z0; z < b.z1; ++z) for (int y = b.y0; y < b.y1; ++y) for (int x = b.x1 + M - w; x < b.x1 + M; ++x) PUT(z, y, x);
#undef PUT
    return n;
}

long long oracle_el3d_tape_len(int B, int nz, int ny, int nx, int nt, int M, const int* pad)
{
    EL3 p; memset(&p, 0, sizeof p);
    p.B = B; p.nz = nz; p.ny = ny; p.nx = nx; p.nt = nt; p.M = M;
    for (int k = 0; k < 6; ++k) p.pad[k] = pad[k];
    const int ns = band_cells(&p, NULL);
    return (long long)nt * B * 9 * ns + 9LL * B * nz * ny * nx;
}

#define SETUP_EL3                                                                              \
    EL3 p = {B, nz, ny, nx, nt, M, {pad[0], pad[1], pad[2], pad[3], pad[4], pad[5]}, dt, dz, dy, dx, coef, \
             prof, prof + nz, prof + 2 * nz, prof + 3 * nz,                                          \
             prof + 4 * nz, prof + 4 * nz + ny, prof + 4 * nz + 2 * ny, prof + 4 * nz + 3 * ny,       \
             prof + 4 * nz + 4 * ny, prof + 4 * nz + 4 * ny + nx, prof + 4 * nz + 4 * ny + 2 * nx,    \
             prof + 4 * nz + 4 * ny + 3 * nx,                                                          \
             vp, vs, rho, m_stride, nsrc, src, wavelet, nsf, sfields, nrec, rec, nrf, rfields, fs}

/* Forward: velocity step, stress step, source injection per source field,
 * band save of the 9 fields (tape non-NULL), record per receiver field; the
 * final 9-field state closes the tape. */
int oracle_el3d_forward(
    int B, int nz, int ny, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dy, REAL dx,
    const REAL* coef, const REAL* prof,
    const REAL* vp, const REAL* vs, const REAL* rho, i64 m_stride,
    int nsrc, const int* src, const REAL* wavelet, int nsf, const int* sfields,
    int nrec, const int* rec, int nrf, const int* rfields, int fs,
    REAL* record, REAL* tape)
{
    SETUP_EL3;
    const i64 n = (i64)nz * ny * nx;
    const int ns = band_cells(&p, NULL);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    REAL* buf = (REAL*)calloc((size_t)n * (NF + 2), sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    band_cells(&p, cells);
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * (NF + 2));
        REAL* F[NF];
        for (int f = 0; f < NF; ++f) F[f] = buf + f * n;
        REAL *lam = buf + NF * n, *mu = buf + (NF + 1) * n;
        lame(&p, b, lam, mu);
        for (int it = 0; it < nt; ++it) {
            velocity_step(&p, b, F);
            stress_step(&p, F, lam, mu);
            for (int k = 0; k < nsf; ++k) inject(&p, b, F[sfields[k]], it, R(1));
            if (tape)
                for (int f = 0; f < 9; ++f) {
                    REAL* dst = tape + (((i64)it * B + b) * 9 + f) * ns;
                    for (int c = 0; c < ns; ++c) dst[c] = F[f][cells[c]];
                }
            for (int r = 0; r < nrec; ++r) {
                i64 c;
                if (!on_grid(&p, rec + ((i64)b * nrec + r) * 3, &c)) continue;
                for (int k = 0; k < nrf; ++k)
                    record[(((i64)b * nt + it) * nrec + r) * nrf + k] = F[rfields[k]][c];
            }
        }
        if (tape)
            for (int f = 0; f < 9; ++f)
                memcpy(tape + (i64)nt * B * 9 * ns + ((i64)b * 9 + f) * n, F[f], sizeof(REAL) * n);
    }
    free(buf); free(cells);
    return 0;
}

#define LOOP_REV                                                                \
    _Pragma("omp parallel for collapse(2) schedule(static)")                    \
    for (int iz = p->fs ? p->M : bx_.z0 + 1; iz < bx_.z1 - 1; ++iz)             \
        for (int iy = bx_.y0 + 1; iy < bx_.y1 - 1; ++iy)                       \
            for (int ix = bx_.x0 + 1; ix < bx_.x1 - 1; ++ix)

static void stress_reverse(const EL3* p, REAL** F, const REAL* lam_, const REAL* mu_)
{
    const int ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy;
    const BOX bx_ = box_of(p);
    LOOP_REV {
        const i64 i = iz * sz + iy * sy + ix, col = i - iz * sz;
        const REAL dvx_dx = dminus(F[VX], i, 1, M, p->c, ix_);
        const REAL dvx_dy = dplus(F[VX], i, sy, M, p->c, iy_);
        const REAL dvx_dz = dz3(p, F[VX], col, iz, 1, 0, 0);
        const REAL dvy_dx = dplus(F[VY], i, 1, M, p->c, ix_);
        const REAL dvy_dy = dminus(F[VY], i, sy, M, p->c, iy_);
        const REAL dvy_dz = dz3(p, F[VY], col, iz, 1, 0, 0);
        const REAL dvz_dx = dplus(F[VZ], i, 1, M, p->c, ix_);
        const REAL dvz_dy = dplus(F[VZ], i, sy, M, p->c, iy_);
        const REAL dvz_dz = dz3(p, F[VZ], col, iz, 0, 1, 1);
        const REAL lam = lam_[i], mu = mu_[i];
        const REAL div = (dvx_dx + dvy_dy) + dvz_dz;
        F[SXX][i] = F[SXX][i] - p->dt * (lam * div + (R(2) * mu) * dvx_dx);
        F[SYY][i] = F[SYY][i] - p->dt * (lam * div + (R(2) * mu) * dvy_dy);
        F[SZZ][i] = F[SZZ][i] - p->dt * (lam * div + (R(2) * mu) * dvz_dz);
        F[SXY][i] = F[SXY][i] - (p->dt * mu) * (dvx_dy + dvy_dx);
        F[SXZ][i] = F[SXZ][i] - (p->dt * mu) * (dvx_dz + dvz_dx);
        F[SYZ][i] = F[SYZ][i] - (p->dt * mu) * (dvy_dz + dvz_dy);
    }
}

static void velocity_reverse(const EL3* p, int b, REAL** F)
{
    const int ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL* rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy;
    const BOX bx_ = box_of(p);
    LOOP_REV {
        const i64 i = iz * sz + iy * sy + ix, col = i - iz * sz;
        const REAL dsxx_dx = dplus(F[SXX], i, 1, M, p->c, ix_);
        const REAL dsxy_dy = dminus(F[SXY], i, sy, M, p->c, iy_);
        const REAL dsxz_dz = dz3(p, F[SXZ], col, iz, 0, 1, 1);
        const REAL dsxy_dx = dminus(F[SXY], i, 1, M, p->c, ix_);
        const REAL dsyy_dy = dplus(F[SYY], i, sy, M, p->c, iy_);
        const REAL dsyz_dz = dz3(p, F[SYZ], col, iz, 0, 1, 1);
        const REAL dsxz_dx = dminus(F[SXZ], i, 1, M, p->c, ix_);
        const REAL dsyz_dy = dminus(F[SYZ], i, sy, M, p->c, iy_);
        const REAL dszz_dz = dz3(p, F[SZZ], col, iz, 1, 1, 0);
        const REAL inv_rho = R(1) / rho[i];
        F[VX][i] = F[VX][i] - (p->dt * inv_rho) * ((dsxx_dx + dsxy_dy) + dsxz_dz);
        F[VY][i] = F[VY][i] - (p->dt * inv_rho) * ((dsxy_dx + dsyy_dy) + dsyz_dz);
        F[VZ][i] = F[VZ][i] - (p->dt * inv_rho) * ((dsxz_dx + dsyz_dy) + dszz_dz);
    }
}

/* Stress-adjoint prepare over every cell with the fused imaging inside the
 * physical box: A = adjoint fields + memories, Fw = reconstructed forward
 * fields (v at it), vn = v at it + 1. */
static void stress_adjoint_prepare(const EL3* p, int b, REAL** A, REAL** Q, const REAL* lam_, const REAL* mu_,
                                   REAL** Fw, REAL** vn, REAL* gvp, REAL* gvs, REAL* grho)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const BOX bx_ = box_of(p);
    const REAL *vp = p->vp + b * p->ms, *vs = p->vs + b * p->ms, *rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy, dt = p->dt;
    _Pragma("omp parallel for collapse(2) schedule(static)")
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const i64 i = iz * sz + iy * sy + ix, col = i - iz * sz;
                const REAL lam = lam_[i], mu = mu_[i], l2m = lam + R(2) * mu;
                const int surf = surf_row(p, iz);
                if (surf) A[SZZ][i] = R(0);
                const REAL bsxx = A[SXX][i], bsyy = A[SYY][i], bszz = A[SZZ][i];
                const REAL bsxy = A[SXY][i], bsxz = A[SXZ][i], bsyz = A[SYZ][i];
                if (gvp && ix >= bx_.x0 && ix < bx_.x1 && iy >= bx_.y0 && iy < bx_.y1 && iz >= bx_.z0 &&
                    iz < bx_.z1) {
                    const REAL fvx_x = dminus(Fw[VX], i, 1, M, p->c, ix_);
                    const REAL fvx_y = dplus(Fw[VX], i, sy, M, p->c, iy_);
                    const REAL fvx_z = dz3(p, Fw[VX], col, iz, 1, 0, 0);
                    const REAL fvy_x = dplus(Fw[VY], i, 1, M, p->c, ix_);
                    const REAL fvy_y = dminus(Fw[VY], i, sy, M, p->c, iy_);
                    const REAL fvy_z = dz3(p, Fw[VY], col, iz, 1, 0, 0);
                    const REAL fvz_x = dplus(Fw[VZ], i, 1, M, p->c, ix_);
                    const REAL fvz_y = dplus(Fw[VZ], i, sy, M, p->c, iy_);
                    const REAL fvz_z = dz3(p, Fw[VZ], col, iz, 0, 1, 1);
                    REAL gl, gm;
                    if (surf) {   /* the surface row's corrected sxx / syy updates (kernels.cuh:1440-1452) */
                        const REAL vp2 = vp[i] * vp[i], vs2 = vs[i] * vs[i], vp4 = vp2 * vp2;
                        const REAL dcl = R(4) * vs2 * vs2 / vp4;
                        const REAL dcm = R(4) * (vp4 - R(2) * vp2 * vs2 + R(2) * vs2 * vs2) / vp4;
                        const REAL dc2m = R(2) * (vp2 - R(2) * vs2) * (vp2 - R(2) * vs2) / vp4;
                        gl = dcl * (bsxx + bsyy) * (fvx_x + fvy_y);
                        gm = bsxx * (dcm * fvx_x + dc2m * fvy_y) + bsyy * (dc2m * fvx_x + dcm * fvy_y) +
                             bsxz * (fvx_z + fvz_x) + bsxy * (fvx_y + fvy_x) + bsyz * (fvy_z + fvz_y);
                    } else {
                        gl = ((bsxx + bsyy) + bszz) * ((fvx_x + fvy_y) + fvz_z);
                        gm = R(2) * ((bsxx * fvx_x + bsyy * fvy_y) + bszz * fvz_z) + bsxz * (fvx_z + fvz_x) +
                             bsxy * (fvx_y + fvy_x) + bsyz * (fvy_z + fvz_y);
                    }
                    gvp[i] = gvp[i] + ((R(-2) * rho[i]) * vp[i]) * gl * dt;
                    gvs[i] = gvs[i] + (-((((R(-4) * rho[i]) * vs[i]) * gl) + (((R(2) * rho[i]) * vs[i]) * gm))) * dt;
                    grho[i] = grho[i] + ((A[VX][i] * (Fw[VX][i] - vn[0][i]) + A[VY][i] * (Fw[VY][i] - vn[1][i])) +
                                         A[VZ][i] * (Fw[VZ][i] - vn[2][i])) / rho[i];
                    grho[i] = grho[i] - ((gl * ((vp[i] * vp[i]) - ((R(2) * vs[i]) * vs[i]))) * dt +
                                         (gm * (vs[i] * vs[i])) * dt);
                }
                REAL bvx_x, bvy_y, bvz_z;
                if (surf) {   /* transposes of the corrected surface updates */
                    const REAL coef = R(4) * mu * (lam + mu) / l2m, coef2 = R(2) * lam * mu / l2m;
                    bvx_x = dt * (coef * bsxx + coef2 * bsyy);
                    bvy_y = dt * (coef2 * bsxx + coef * bsyy);
                    bvz_z = R(0);
                } else {
                    bvx_x = dt * ((l2m * bsxx + lam * bsyy) + lam * bszz);
                    bvy_y = dt * ((lam * bsxx + l2m * bsyy) + lam * bszz);
                    bvz_z = dt * ((lam * bsxx + lam * bsyy) + l2m * bszz);
                }
                const REAL bvx_y = (dt * mu) * bsxy, bvx_z = (dt * mu) * bsxz;
                const REAL bvy_x = (dt * mu) * bsxy, bvy_z = (dt * mu) * bsyz;
                const REAL bvz_x = (dt * mu) * bsxz, bvz_y = (dt * mu) * bsyz;
                if (interior(&bx_, ix, iy, iz)) {
                    Q[0][i] = bvx_x; Q[1][i] = bvx_y; Q[2][i] = bvx_z;
                    Q[3][i] = bvy_x; Q[4][i] = bvy_y; Q[5][i] = bvy_z;
                    Q[6][i] = bvz_x; Q[7][i] = bvz_y; Q[8][i] = bvz_z;
                    continue;
                }
                const REAL t_vxx = A[M_VXX][i] + bvx_x, t_vxy = A[M_VXY][i] + bvx_y, t_vxz = A[M_VXZ][i] + bvx_z;
                const REAL t_vyx = A[M_VYX][i] + bvy_x, t_vyy = A[M_VYY][i] + bvy_y, t_vyz = A[M_VYZ][i] + bvy_z;
                const REAL t_vzx = A[M_VZX][i] + bvz_x, t_vzy = A[M_VZY][i] + bvz_y, t_vzz = A[M_VZZ][i] + bvz_z;
                Q[0][i] = bvx_x + p->bx[ix] * t_vxx;
                Q[1][i] = bvx_y + p->byh[iy] * t_vxy;
                Q[2][i] = bvx_z + p->bzh[iz] * t_vxz;
                Q[3][i] = bvy_x + p->bxh[ix] * t_vyx;
                Q[4][i] = bvy_y + p->by[iy] * t_vyy;
                Q[5][i] = bvy_z + p->bzh[iz] * t_vyz;
                Q[6][i] = bvz_x + p->bxh[ix] * t_vzx;
                Q[7][i] = bvz_y + p->byh[iy] * t_vzy;
                Q[8][i] = bvz_z + p->bz[iz] * t_vzz;
                A[M_VXX][i] = p->ax[ix] * t_vxx; A[M_VYX][i] = p->axh[ix] * t_vyx; A[M_VZX][i] = p->axh[ix] * t_vzx;
                A[M_VXY][i] = p->ayh[iy] * t_vxy; A[M_VYY][i] = p->ay[iy] * t_vyy; A[M_VZY][i] = p->ayh[iy] * t_vzy;
                A[M_VXZ][i] = p->azh[iz] * t_vxz; A[M_VYZ][i] = p->azh[iz] * t_vyz; A[M_VZZ][i] = p->az[iz] * t_vzz;
            }
}

/* Stress-adjoint apply: the adjoint velocities gather the transposed
 * stencils of q (D+ of a D- forward and vice versa). */
static void stress_adjoint_apply(const EL3* p, REAL** A, REAL** Q)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy;
    LOOP_CORE {
        const i64 i = iz * sz + iy * sy + ix, col = i - iz * sz;
        const REAL qxx = dplus(Q[0], i, 1, M, p->c, ix_), qxy = dminus(Q[1], i, sy, M, p->c, iy_);
        const REAL qxz = adz3(p, Q[2], col, iz, 1, 0, 0);
        const REAL qyx = dminus(Q[3], i, 1, M, p->c, ix_), qyy = dplus(Q[4], i, sy, M, p->c, iy_);
        const REAL qyz = adz3(p, Q[5], col, iz, 1, 0, 0);
        const REAL qzx = dminus(Q[6], i, 1, M, p->c, ix_), qzy = dminus(Q[7], i, sy, M, p->c, iy_);
        const REAL qzz = adz3(p, Q[8], col, iz, 0, 1, 1);
        A[VX][i] = A[VX][i] + ((qxx + qxy) + qxz);
        A[VY][i] = A[VY][i] + ((qyx + qyy) + qyz);
        A[VZ][i] = A[VZ][i] + ((qzx + qzy) + qzz);
    }
}

/* Velocity-adjoint prepare (every cell) and apply: p = dt / rho * adjoint v
 * with the CPML memories outside the interior. */
static void velocity_adjoint(const EL3* p, int b, REAL** A, REAL** P)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const BOX bx_ = box_of(p);
    const REAL* rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iy_ = R(1) / p->dy, dt = p->dt;
    _Pragma("omp parallel for collapse(2) schedule(static)")
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const i64 i = iz * sz + iy * sy + ix;
                const REAL k = dt * (R(1) / rho[i]);
                const REAL bx_v = k * A[VX][i], by_v = k * A[VY][i], bz_v = k * A[VZ][i];
                if (interior(&bx_, ix, iy, iz)) {
                    P[0][i] = bx_v; P[1][i] = bx_v; P[2][i] = bx_v;
                    P[3][i] = by_v; P[4][i] = by_v; P[5][i] = by_v;
                    P[6][i] = bz_v; P[7][i] = bz_v; P[8][i] = bz_v;
                    continue;
                }
                const REAL t_sxxx = A[M_SXXX][i] + bx_v, t_sxyy = A[M_SXYY][i] + bx_v, t_sxzz = A[M_SXZZ][i] + bx_v;
                const REAL t_sxyx = A[M_SXYX][i] + by_v, t_syyy = A[M_SYYY][i] + by_v, t_syzz = A[M_SYZZ][i] + by_v;
                const REAL t_sxzx = A[M_SXZX][i] + bz_v, t_syzy = A[M_SYZY][i] + bz_v, t_szzz = A[M_SZZZ][i] + bz_v;
                P[0][i] = bx_v + p->bxh[ix] * t_sxxx;   /* pxx */
                P[1][i] = bx_v + p->by[iy] * t_sxyy;    /* pxy */
                P[2][i] = bx_v + p->bz[iz] * t_sxzz;    /* pxz */
                P[3][i] = by_v + p->bx[ix] * t_sxyx;    /* pyx */
                P[4][i] = by_v + p->byh[iy] * t_syyy;   /* pyy */
                P[5][i] = by_v + p->bz[iz] * t_syzz;    /* pyz */
                P[6][i] = bz_v + p->bx[ix] * t_sxzx;    /* pzx */
                P[7][i] = bz_v + p->by[iy] * t_syzy;    /* pzy */
                P[8][i] = bz_v + p->bzh[iz] * t_szzz;   /* pzz */
                A[M_SXXX][i] = p->axh[ix] * t_sxxx; A[M_SXYX][i] = p->ax[ix] * t_sxyx; A[M_SXZX][i] = p->ax[ix] * t_sxzx;
                A[M_SXYY][i] = p->ay[iy] * t_sxyy; A[M_SYYY][i] = p->ayh[iy] * t_syyy; A[M_SYZY][i] = p->ay[iy] * t_syzy;
                A[M_SXZZ][i] = p->az[iz] * t_sxzz; A[M_SYZZ][i] = p->az[iz] * t_syzz; A[M_SZZZ][i] = p->azh[iz] * t_szzz;
            }
    LOOP_CORE {
        const i64 i = iz * sz + iy * sy + ix, col = i - iz * sz;
        const REAL pxx = dminus(P[0], i, 1, M, p->c, ix_), pxy = dplus(P[1], i, sy, M, p->c, iy_);
        const REAL pxz = adz3(p, P[2], col, iz, 0, 1, 1);
        const REAL pyx = dplus(P[3], i, 1, M, p->c, ix_), pyy = dminus(P[4], i, sy, M, p->c, iy_);
        const REAL pyz = adz3(p, P[5], col, iz, 0, 1, 1);
        const REAL pzx = dplus(P[6], i, 1, M, p->c, ix_), pzy = dplus(P[7], i, sy, M, p->c, iy_);
        const REAL pzz = adz3(p, P[8], col, iz, 1, 1, 0);
        A[SXX][i] = A[SXX][i] + pxx;
        A[SXY][i] = A[SXY][i] + (pxy + pyx);
        A[SXZ][i] = A[SXZ][i] + (pxz + pzx);
        A[SYY][i] = A[SYY][i] + pyy;
        A[SYZ][i] = A[SYZ][i] + (pyz + pzy);
        A[SZZ][i] = A[SZZ][i] + pzz;
    }
}

/* Boundary-saving backward, reverse steps nt-1 .. 1 (the staggered reverse
 * has no it = 0 step).  adj: (B, nt, nrec, nrf); grad_* accumulate
 * (B|1, nz, ny, nx) with the model stride; tape: from oracle_el3d_forward. */
int oracle_el3d_backward(
    int B, int nz, int ny, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dy, REAL dx,
    const REAL* coef, const REAL* prof,
    const REAL* vp, const REAL* vs, const REAL* rho, i64 m_stride,
    int nsrc, const int* src, const REAL* wavelet, int nsf, const int* sfields,
    int nrec, const int* rec, int nrf, const int* rfields, int fs,
    const REAL* adj, const REAL* tape, REAL* grad_vp, REAL* grad_vs, REAL* grad_rho)
{
    SETUP_EL3;
    const i64 n = (i64)nz * ny * nx;
    const int ns = band_cells(&p, NULL);
    const BOX bx_ = box_of(&p);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    const int nbuf = 9 + NF + 18 + 3 + 2;
    REAL* buf = (REAL*)calloc((size_t)n * nbuf, sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    band_cells(&p, cells);
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * nbuf);
        REAL *Fw[9], *A[NF], *Q[9], *P[9], *vn[3];
        for (int f = 0; f < 9; ++f) Fw[f] = buf + f * n;
        for (int f = 0; f < NF; ++f) A[f] = buf + (9 + f) * n;
        for (int f = 0; f < 9; ++f) { Q[f] = buf + (9 + NF + f) * n; P[f] = buf + (9 + NF + 9 + f) * n; }
        for (int f = 0; f < 3; ++f) vn[f] = buf + (9 + NF + 18 + f) * n;
        REAL *lam = buf + (9 + NF + 21) * n, *mu = buf + (9 + NF + 22) * n;
        lame(&p, b, lam, mu);
        REAL *gvp = grad_vp + b * m_stride, *gvs = grad_vs + b * m_stride, *grho = grad_rho + b * m_stride;
        const REAL* rb = rho + b * m_stride;
        for (int f = 0; f < 9; ++f)
            memcpy(Fw[f], tape + (i64)nt * B * 9 * ns + ((i64)b * 9 + f) * n, sizeof(REAL) * n);
        for (int it = nt - 1; it >= 1; --it) {
            /* body-force rho correction at velocity sources, before the residuals */
            for (int k = 0; k < nsf; ++k) {
                if (sfields[k] > 2) continue;
                for (int s = 0; s < nsrc; ++s) {
                    i64 c;
                    if (!on_grid(&p, src + ((i64)b * nsrc + s) * 3, &c)) continue;
                    grho[c] = grho[c] + (A[sfields[k]][c] * wavelet[((i64)b * nsrc + s) * nt + it]) / rb[c];
                }
            }
            /* signed residuals: stress -1, velocity +1 */
            for (int k = 0; k < nrf; ++k) {
                const REAL sign = rfields[k] >= 3 ? R(-1) : R(1);
                for (int r = 0; r < nrec; ++r) {
                    i64 c;
                    if (!on_grid(&p, rec + ((i64)b * nrec + r) * 3, &c)) continue;
                    A[rfields[k]][c] += sign * adj[(((i64)b * nt + it) * nrec + r) * nrf + k];
                }
            }
            for (int k = 0; k < nsf; ++k) inject(&p, b, Fw[sfields[k]], it, R(-1));
            /* stress half */
            stress_reverse(&p, Fw, lam, mu);
            for (int f = 3; f < 9; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 9 + f) * ns;
                for (int c = 0; c < ns; ++c) Fw[f][cells[c]] = s[c];
            }
            stress_adjoint_prepare(&p, b, A, Q, lam, mu, Fw, vn, gvp, gvs, grho);
            for (int k = 0; k < nrf; ++k) {
                const int fld = rfields[k];
                if (fld > 2) continue;
                for (int r = 0; r < nrec; ++r) {
                    const int* l = rec + ((i64)b * nrec + r) * 3;
                    if (l[0] < M || l[0] >= nx - M || l[1] < M || l[1] >= ny - M || l[2] < M || l[2] >= nz - M)
                        continue;
                    const i64 c = ((i64)l[2] * ny + l[1]) * nx + l[0];
                    const REAL a = adj[(((i64)b * nt + it) * nrec + r) * nrf + k];
                    grho[c] = grho[c] + ((-a) * (Fw[fld][c] - vn[fld][c])) / rb[c];
                }
            }
            stress_adjoint_apply(&p, A, Q);
            /* velocity half */
            velocity_adjoint(&p, b, A, P);
            for (int iz = bx_.z0; iz < bx_.z1; ++iz)
                for (int iy = bx_.y0; iy < bx_.y1; ++iy)
                    for (int ix = bx_.x0; ix < bx_.x1; ++ix) {
                        const i64 i = ((i64)iz * ny + iy) * nx + ix;
                        vn[0][i] = Fw[VX][i]; vn[1][i] = Fw[VY][i]; vn[2][i] = Fw[VZ][i];
                    }
            velocity_reverse(&p, b, Fw);
            for (int f = 0; f < 3; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 9 + f) * ns;
                for (int c = 0; c < ns; ++c) Fw[f][cells[c]] = s[c];
            }
        }
    }
    free(buf); free(cells);
    return 0;
}
