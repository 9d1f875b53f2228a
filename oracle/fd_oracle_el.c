/*
 * fd_oracle_el.c -- CPU restatement of the reference's compiled (impl='c')
 * 2-D isotropic elastic path (velocity-stress, staggered grid, Virieux), used
 * ONLY as test infrastructure: the parity checker of the CUDA library.  It is
 * never linked into, loaded by or called from the product library.
 *
 * Built with REAL=float and REAL=double by oracle/Makefile, -ffp-contract=off
 * (every operation rounds once, in the reference's expression order).
 *
 * Layout: every field is (B, nz, nx), x fastest, on the runtime grid
 * (physical + PML pad + stencil halo M per face).  Coordinates are runtime
 * (x, z) int32 pairs; off-grid ones are skipped (reference
 * src/sweep/csrc/cuda/common/common.cu:24-28, 137-138).  Records and their
 * cotangents are (B, nt, nrec, nfield).  Field indices: 0 vx, 1 vz, 2 sxx,
 * 3 szz, 4 sxz (src/sweep/csrc/cuda/common/elastic.h:715-725).
 *
 * What each function restates (reference paths, relative to the project root):
 *   staggered D+/D-   src/sweep/csrc/cuda/operators/staggered.cuh:332-430
 *   Lame parameters   src/sweep/csrc/cuda/common/derived_models.cu:27-37
 *   velocity step     src/sweep/csrc/cuda/equations/elastic2d/kernels.cuh:48-138
 *   stress step       kernels.cuh:182-311
 *   reverse (NOPML)   kernels.cuh:365-535
 *   stress adjoint    kernels.cuh:548-750 (prepare, fused vp/vs/rho imaging
 *                     601-663), 807-837 (apply)
 *   velocity adjoint  kernels.cuh:873-958 (prepare), 989-1019 (apply)
 *   adjoint stencils  src/sweep/csrc/cuda/common/elastic_free_surface.cuh:
 *                     395-415, 655-675 (transpose of D- is D+ and vice versa,
 *                     no sign: the adjoint stresses carry the negated adjoint)
 *   source / receiver src/sweep/csrc/cuda/common/common.cu:11-160 (add_source,
 *                     add_body_force_rho_grad_correction,
 *                     sub_receiver_rho_grad_correction, record_kernel)
 *   residual signs    src/sweep/csrc/cuda/common/elastic.h:696-713 (stress -1,
 *                     velocity +1)
 *   step order        src/sweep/csrc/cuda/common/sg_driver.cuh:291-340
 *                     (forward), 760-806 (boundary-saving reverse, floor it=1);
 *                     src/sweep/csrc/cuda/equations/elastic2d/driver_traits.cuh:
 *                     222-318, 387-490, 659-826
 *   strip geometry    src/sweep/csrc/cuda/common/boundary/strip.cuh:46-123
 *                     (width M+1 at offset -M, physical box tangentially)
 *   free top face     src/sweep/csrc/cuda/common/elastic_free_surface.cuh:
 *                     200-465 (image values, order-2 band, reduced transpose
 *                     and folds); elastic2d/kernels.cuh:216-234, 293-303
 *                     (surface row in the CPML branch, Robertsson sxx
 *                     correction, szz = 0), 592-700 (adjoint zeroing, surface
 *                     imaging, transposed correction), 365-535 (reverse rows
 *                     from M on a free face)
 */
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
    const REAL* c;              /* c[1..M] staggered coefficients (c[0] unused) */
    const REAL *az, *bz, *azh, *bzh, *ax, *bx, *axh, *bxh;
    const REAL *vp, *vs, *rho;
    i64 ms;                     /* model stride between shots (0 = shared) */
    int nsrc; const int* src; const REAL* wavelet; int nsf; const int* sf;
    int nrec; const int* rec; int nrf; const int* rf;
    int fs;                     /* bit 0: traction-free top face (pad[0] == 0) */
} EL;

/* D+ along stride s: sum_k c_k (u[i+k s] - u[i-(k-1) s]) * (1/h). */
static inline REAL dplus(const REAL* u, i64 i, i64 s, int M, const REAL* c, REAL inv)
{
    REAL g = c[1] * (u[i + s] - u[i]);
    for (int k = 2; k <= M; ++k) g = g + c[k] * (u[i + k * s] - u[i - (k - 1) * s]);
    return g * inv;
}

/* D- along stride s: sum_k c_k (u[i+(k-1) s] - u[i-k s]) * (1/h). */
static inline REAL dminus(const REAL* u, i64 i, i64 s, int M, const REAL* c, REAL inv)
{
    REAL g = c[1] * (u[i] - u[i - s]);
    for (int k = 2; k <= M; ++k) g = g + c[k] * (u[i + (k - 1) * s] - u[i - k * s]);
    return g * inv;
}

static int in_grid(int ix, int iz, int nx, int nz) { return ix >= 0 && ix < nx && iz >= 0 && iz < nz; }

/* ---- traction-free top face (image method) -------------------------------
 * The surface is the first physical row, top = pad[0] + M = M (a free face
 * has no PML pad); rows above it are air.  z-derivatives read an air row as
 * the image of the row mirrored about the surface: about `top` for fields on
 * integer rows (szz, vx), about top - 1/2 for fields half a cell below them
 * (sxz, vz), negated for the odd fields.  The M rows from the surface down
 * take a 2nd-order (unit-weight) difference instead of the full stencil. */
static inline int fs_top_row(const EL* p) { return p->pad[0] + p->M; }

static inline REAL fs_at(const EL* p, const REAL* u, int ix, int iz, int odd, int half)
{
    const int top = fs_top_row(p);
    if (iz < top) {
        const int m = half ? 2 * top - 1 - iz : 2 * top - iz;
        const REAL v = u[(i64)m * p->nx + ix];
        return odd ? -v : v;
    }
    return u[(i64)iz * p->nx + ix];
}

/* z-derivative at (ix, iz) on a free top face: fwd = 1 the D+ form (taps
 * iz+k and iz-k+1), fwd = 0 the D- form (taps iz+k-1 and iz-k). */
static REAL fs_dz(const EL* p, const REAL* u, int ix, int iz, int fwd, int odd, int half)
{
    const int top = fs_top_row(p), M = p->M;
    if (iz - top >= 0 && iz - top < M) {
        const REAL g = fwd ? fs_at(p, u, ix, iz + 1, odd, half) - fs_at(p, u, ix, iz, odd, half)
                           : fs_at(p, u, ix, iz, odd, half) - fs_at(p, u, ix, iz - 1, odd, half);
        return g / p->dz;
    }
    REAL g = R(0);
    for (int k = 1; k <= M; ++k) {
        const REAL up = fwd ? fs_at(p, u, ix, iz + k, odd, half) : fs_at(p, u, ix, iz + k - 1, odd, half);
        const REAL um = fwd ? fs_at(p, u, ix, iz - k + 1, odd, half) : fs_at(p, u, ix, iz - k, odd, half);
        g = g + p->c[k] * (up - um);
    }
    return g / p->dz;
}

static inline int fs_band(const EL* p, int j)
{
    const int top = fs_top_row(p);
    return j >= top && j < top + p->M;
}

/* Transpose of fs_dz without the image (negated, in the sign convention of
 * the plain adjoint stencils: D- for a D+ forward and vice versa) at input
 * row m: each output row j contributes with the full weight if it lies below
 * the order-2 band, with weight 1 if it lies in it; reads outside the grid
 * are skipped. */
static REAL fs_adj_plain(const EL* p, const REAL* q, int ix, int m, int fwd)
{
    const int M = p->M, nz = p->nz, nx = p->nx;
    REAL acc = R(0);
    for (int k = 1; k <= M; ++k) {
        const int jp = fwd ? m + k - 1 : m + k;
        const int jm = fwd ? m - k : m - k + 1;
        if (jp >= 0 && jp < nz && !fs_band(p, jp)) acc = acc + p->c[k] * q[(i64)jp * nx + ix];
        if (jm >= 0 && jm < nz && !fs_band(p, jm)) acc = acc - p->c[k] * q[(i64)jm * nx + ix];
    }
    if (fwd) {
        if (fs_band(p, m)) acc = acc + q[(i64)m * nx + ix];
        if (fs_band(p, m - 1)) acc = acc - q[(i64)(m - 1) * nx + ix];
    } else {
        if (fs_band(p, m + 1)) acc = acc + q[(i64)(m + 1) * nx + ix];
        if (fs_band(p, m)) acc = acc - q[(i64)m * nx + ix];
    }
    return acc / p->dz;
}

/* Adjoint of fs_dz at row iz: zero on air rows (the forward overwrites them
 * with images); else the plain transpose plus, where the row's mirror lies in
 * the air, the transpose at that air row folded back with the field's
 * parity. */
static REAL fs_adj_dz(const EL* p, const REAL* q, int ix, int iz, int fwd, int odd, int half)
{
    const int top = fs_top_row(p);
    if (iz < top) return R(0);
    REAL g = fs_adj_plain(p, q, ix, iz, fwd);
    const int miz = half ? 2 * top - 1 - iz : 2 * top - iz;
    if (miz < top) g = g + (odd ? R(-1) : R(1)) * fs_adj_plain(p, q, ix, miz, fwd);
    return g;
}

/* CPML test shared by the velocity step, the stress step (no free surface)
 * and both adjoint prepares: the PML pad plus the stencil halo, per face. */
static inline int in_pml(const EL* p, int ix, int iz)
{
    const int h = p->M;
    return ix < p->pad[2] + h || ix >= p->nx - p->pad[3] - h ||
           iz < p->pad[0] + h || iz >= p->nz - p->pad[1] - h;
}

/* Per-shot field bundle: 5 wavefields then 8 CPML memories. */
enum { VX, VZ, SXX, SZZ, SXZ, M_VXX, M_VZZ, M_VXZ, M_VZX, M_SXXX, M_SZZZ, M_SXZX, M_SXZZ, NF };

static void lame(const EL* p, int b, REAL* lam, REAL* mu)
{
    const i64 n = (i64)p->nz * p->nx;
    const REAL *v = p->vp + b * p->ms, *s = p->vs + b * p->ms, *r = p->rho + b * p->ms;
    for (i64 i = 0; i < n; ++i) {
        mu[i] = (r[i] * s[i]) * s[i];
        lam[i] = r[i] * ((v[i] * v[i]) - ((R(2) * s[i]) * s[i]));
    }
}

static void velocity_step(const EL* p, int b, REAL** F)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL* rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz;
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dsxx_dx = dplus(F[SXX], i, 1, M, p->c, ix_);
            REAL dsxz_dz = p->fs ? fs_dz(p, F[SXZ], ix, iz, 0, 1, 1) : dminus(F[SXZ], i, nx, M, p->c, iz_);
            REAL dsxz_dx = dminus(F[SXZ], i, 1, M, p->c, ix_);
            REAL dszz_dz = p->fs ? fs_dz(p, F[SZZ], ix, iz, 1, 1, 0) : dplus(F[SZZ], i, nx, M, p->c, iz_);
            REAL inv_rho = R(1) / rho[i];
            if (in_pml(p, ix, iz)) {
                REAL m;
                m = p->azh[iz] * F[M_SZZZ][i] + p->bzh[iz] * dszz_dz; F[M_SZZZ][i] = m; dszz_dz = dszz_dz + m;
                m = p->ax[ix] * F[M_SXZX][i] + p->bx[ix] * dsxz_dx; F[M_SXZX][i] = m; dsxz_dx = dsxz_dx + m;
                m = p->az[iz] * F[M_SXZZ][i] + p->bz[iz] * dsxz_dz; F[M_SXZZ][i] = m; dsxz_dz = dsxz_dz + m;
                m = p->axh[ix] * F[M_SXXX][i] + p->bxh[ix] * dsxx_dx; F[M_SXXX][i] = m; dsxx_dx = dsxx_dx + m;
            }
            F[VX][i] = F[VX][i] + (p->dt * inv_rho) * (dsxx_dx + dsxz_dz);
            F[VZ][i] = F[VZ][i] + (p->dt * inv_rho) * (dsxz_dx + dszz_dz);
        }
    }
}

static void stress_step(const EL* p, REAL** F, const REAL* lam_, const REAL* mu_)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz;
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dvx_dx = dminus(F[VX], i, 1, M, p->c, ix_);
            REAL dvz_dz = p->fs ? fs_dz(p, F[VZ], ix, iz, 0, 1, 1) : dminus(F[VZ], i, nx, M, p->c, iz_);
            REAL dvx_dz = p->fs ? fs_dz(p, F[VX], ix, iz, 1, 0, 0) : dplus(F[VX], i, nx, M, p->c, iz_);
            REAL dvz_dx = dplus(F[VZ], i, 1, M, p->c, ix_);
            REAL lam = lam_[i], mu = mu_[i];
            /* a free surface row takes the CPML branch (kernels.cuh:216-234) */
            const int surf = p->fs && iz == fs_top_row(p);
            const int pml = in_pml(p, ix, iz) || surf;
            if (pml) {
                REAL m;
                m = p->az[iz] * F[M_VZZ][i] + p->bz[iz] * dvz_dz; F[M_VZZ][i] = m; dvz_dz = dvz_dz + m;
                m = p->ax[ix] * F[M_VXX][i] + p->bx[ix] * dvx_dx; F[M_VXX][i] = m; dvx_dx = dvx_dx + m;
            }
            F[SXX][i] = F[SXX][i] + p->dt * ((lam + R(2) * mu) * dvx_dx + lam * dvz_dz);
            F[SZZ][i] = F[SZZ][i] + p->dt * ((lam + R(2) * mu) * dvz_dz + lam * dvx_dx);
            if (pml) {
                REAL m;
                m = p->azh[iz] * F[M_VXZ][i] + p->bzh[iz] * dvx_dz; F[M_VXZ][i] = m; dvx_dz = dvx_dz + m;
                m = p->axh[ix] * F[M_VZX][i] + p->bxh[ix] * dvz_dx; F[M_VZX][i] = m; dvz_dx = dvz_dx + m;
            }
            F[SXZ][i] = F[SXZ][i] + (p->dt * mu) * (dvx_dz + dvz_dx);
            if (surf) {   /* Robertsson correction, then szz = 0 (kernels.cuh:293-303) */
                F[SXX][i] = F[SXX][i] + (-p->dt) * lam * ((lam / (lam + R(2) * mu)) * dvx_dx + dvz_dz);
                F[SZZ][i] = R(0);
            }
        }
    }
}

/* Point injection of the (B, nsrc, nt) wavelet into one field. */
static void inject(const EL* p, int b, REAL* u, int it, REAL sign)
{
    for (int s = 0; s < p->nsrc; ++s) {
        int ix = p->src[(b * p->nsrc + s) * 2], iz = p->src[(b * p->nsrc + s) * 2 + 1];
        if (!in_grid(ix, iz, p->nx, p->nz)) continue;
        u[(i64)iz * p->nx + ix] += sign * p->wavelet[((i64)b * p->nsrc + s) * p->nt + it];
    }
}

/* Boundary-saving band cells (strip.cuh:81-114, width M+1, offset -M): top and
 * bottom bands over the box width, left and right bands over the box height.
 * Cells of two bands are listed twice (their saved values agree). */
static int band_lo(int p0, int off, int w, int n) { int s = p0 + off; if (s + w > n) s = n - w; return s < 0 ? 0 : s; }
static int band_hi(int p1, int off, int w, int n) { int e = p1 - off; if (e - w < 0) e = w; return e > n ? n : e; }

static int band_cells(const EL* p, int* out)
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

long long oracle_el2d_tape_len(int B, int nz, int nx, int nt, int M, const int* pad)
{
    EL p; memset(&p, 0, sizeof p);
    p.B = B; p.nz = nz; p.nx = nx; p.nt = nt; p.M = M;
    for (int k = 0; k < 4; ++k) p.pad[k] = pad[k];
    const int ns = band_cells(&p, NULL);
    return (long long)nt * B * 5 * ns + 5LL * B * nz * nx;
}

#define SETUP_EL                                                                         \
    EL p = {B, nz, nx, nt, M, {pad[0], pad[1], pad[2], pad[3]}, dt, dz, dx, coef,          \
            prof, prof + nz, prof + 2 * nz, prof + 3 * nz,                                 \
            prof + 4 * nz, prof + 4 * nz + nx, prof + 4 * nz + 2 * nx, prof + 4 * nz + 3 * nx, \
            vp, vs, rho, m_stride, nsrc, src, wavelet, nsf, sfields, nrec, rec, nrf, rfields, fs}

/* Forward (sg_driver.cuh:291-340): velocity step, stress step, source
 * injection per source field, band save of the 5 fields (tape non-NULL),
 * record per receiver field; the final 5-field state closes the tape. */
int oracle_el2d_forward(
    int B, int nz, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dx,
    const REAL* coef, const REAL* prof,
    const REAL* vp, const REAL* vs, const REAL* rho, i64 m_stride,
    int nsrc, const int* src, const REAL* wavelet, int nsf, const int* sfields,
    int nrec, const int* rec, int nrf, const int* rfields, int fs,
    REAL* record, REAL* tape)
{
    SETUP_EL;
    const i64 n = (i64)nz * nx;
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
                for (int f = 0; f < 5; ++f) {
                    REAL* dst = tape + (((i64)it * B + b) * 5 + f) * ns;
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
            for (int f = 0; f < 5; ++f)
                memcpy(tape + (i64)nt * B * 5 * ns + ((i64)b * 5 + f) * n, F[f], sizeof(REAL) * n);
    }
    free(buf); free(cells);
    return 0;
}

/* Reverse (NOPML) stress and velocity steps on the box minus one cell per
 * face (kernels.cuh:405-535, band pad + M + 1). */
static void stress_reverse(const EL* p, REAL** F, const REAL* lam_, const REAL* mu_)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz;
    const int zlo = p->fs ? M : p->pad[0] + M + 1;   /* a free face narrows to the halo */
    #pragma omp parallel for schedule(static)
    for (int iz = zlo; iz < nz - (p->pad[1] + M + 1); ++iz) {
        for (int ix = p->pad[2] + M + 1; ix < nx - (p->pad[3] + M + 1); ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dvx_dx = dminus(F[VX], i, 1, M, p->c, ix_);
            REAL dvz_dz = p->fs ? fs_dz(p, F[VZ], ix, iz, 0, 1, 1) : dminus(F[VZ], i, nx, M, p->c, iz_);
            REAL dvx_dz = p->fs ? fs_dz(p, F[VX], ix, iz, 1, 0, 0) : dplus(F[VX], i, nx, M, p->c, iz_);
            REAL dvz_dx = dplus(F[VZ], i, 1, M, p->c, ix_);
            REAL lam = lam_[i], mu = mu_[i];
            F[SXX][i] = F[SXX][i] - p->dt * ((lam + R(2) * mu) * dvx_dx + lam * dvz_dz);
            F[SZZ][i] = F[SZZ][i] - p->dt * ((lam + R(2) * mu) * dvz_dz + lam * dvx_dx);
            F[SXZ][i] = F[SXZ][i] - (p->dt * mu) * (dvx_dz + dvz_dx);
        }
    }
}

static void velocity_reverse(const EL* p, int b, REAL** F)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL* rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz;
    const int zlo = p->fs ? M : p->pad[0] + M + 1;
    #pragma omp parallel for schedule(static)
    for (int iz = zlo; iz < nz - (p->pad[1] + M + 1); ++iz) {
        for (int ix = p->pad[2] + M + 1; ix < nx - (p->pad[3] + M + 1); ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dsxx_dx = dplus(F[SXX], i, 1, M, p->c, ix_);
            REAL dsxz_dz = p->fs ? fs_dz(p, F[SXZ], ix, iz, 0, 1, 1) : dminus(F[SXZ], i, nx, M, p->c, iz_);
            REAL dsxz_dx = dminus(F[SXZ], i, 1, M, p->c, ix_);
            REAL dszz_dz = p->fs ? fs_dz(p, F[SZZ], ix, iz, 1, 1, 0) : dplus(F[SZZ], i, nx, M, p->c, iz_);
            REAL inv_rho = R(1) / rho[i];
            F[VX][i] = F[VX][i] - (p->dt * inv_rho) * (dsxx_dx + dsxz_dz);
            F[VZ][i] = F[VZ][i] - (p->dt * inv_rho) * (dsxz_dx + dszz_dz);
        }
    }
}

/* Stress-adjoint prepare over every cell (kernels.cuh:548-750) with the fused
 * imaging inside the physical box (601-663): A = adjoint fields + memories,
 * Fw = reconstructed forward fields (v at it), vxn/vzn = v at it+1. */
static void stress_adjoint_prepare(const EL* p, int b, REAL** A, REAL** Q, const REAL* lam_, const REAL* mu_,
                                   REAL** Fw, const REAL* vxn, const REAL* vzn,
                                   REAL* gvp, REAL* gvs, REAL* grho)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const int z0 = p->pad[0] + M, z1 = nz - p->pad[1] - M, x0 = p->pad[2] + M, x1 = nx - p->pad[3] - M;
    const REAL *vp = p->vp + b * p->ms, *vs = p->vs + b * p->ms, *rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz, dt = p->dt;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz) {
        for (int ix = 0; ix < nx; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL lam = lam_[i], mu = mu_[i];
            REAL bsxx = A[SXX][i], bszz = A[SZZ][i], bsxz = A[SXZ][i];
            const int surf = p->fs && iz == fs_top_row(p);
            if (surf) { bszz = R(0); A[SZZ][i] = R(0); }
            if (gvp && ix >= x0 && ix < x1 && iz >= z0 && iz < z1) {
                REAL fvx_x = dminus(Fw[VX], i, 1, M, p->c, ix_);
                REAL fvz_z = p->fs ? fs_dz(p, Fw[VZ], ix, iz, 0, 1, 1) : dminus(Fw[VZ], i, nx, M, p->c, iz_);
                REAL fvx_z = p->fs ? fs_dz(p, Fw[VX], ix, iz, 1, 0, 0) : dplus(Fw[VX], i, nx, M, p->c, iz_);
                REAL fvz_x = dplus(Fw[VZ], i, 1, M, p->c, ix_);
                REAL gl, gm;
                if (surf) {
                    /* d/d(lam, mu) of the surface row's sxx update,
                     * dt C dvx_dx with C = 4 mu (lam + mu) / (lam + 2 mu) */
                    const REAL vp2 = vp[i] * vp[i], vs2 = vs[i] * vs[i], vp4 = vp2 * vp2;
                    const REAL a = bsxx * fvx_x;
                    gl = a * R(4) * vs2 * vs2 / vp4;
                    gm = a * R(4) * (vp4 - R(2) * vp2 * vs2 + R(2) * vs2 * vs2) / vp4;
                } else {
                    gl = (bsxx + bszz) * (fvx_x + fvz_z);
                    gm = R(2) * (bsxx * fvx_x + bszz * fvz_z);
                }
                gm = gm + bsxz * (fvx_z + fvz_x);
                gvp[i] = gvp[i] + ((R(-2) * rho[i]) * vp[i]) * gl * dt;
                gvs[i] = gvs[i] + (-((((R(-4) * rho[i]) * vs[i]) * gl) + (((R(2) * rho[i]) * vs[i]) * gm))) * dt;
                grho[i] = grho[i] + (A[VX][i] * (Fw[VX][i] - vxn[i]) + A[VZ][i] * (Fw[VZ][i] - vzn[i])) / rho[i];
                grho[i] = grho[i] - ((gl * ((vp[i] * vp[i]) - ((R(2) * vs[i]) * vs[i]))) * dt +
                                     (gm * (vs[i] * vs[i])) * dt);
            }
            REAL bvx_x, bvz_z;
            if (surf) {   /* transpose of the corrected surface update */
                const REAL c_surf = R(4) * mu * (lam + mu) / (lam + R(2) * mu);
                bvx_x = dt * c_surf * bsxx;
                bvz_z = R(0);
            } else {
                bvx_x = dt * ((lam + R(2) * mu) * bsxx + lam * bszz);
                bvz_z = dt * ((lam + R(2) * mu) * bszz + lam * bsxx);
            }
            REAL bvx_z = (dt * mu) * bsxz;
            REAL bvz_x = (dt * mu) * bsxz;
            if (!in_pml(p, ix, iz)) {
                Q[0][i] = bvx_x; Q[1][i] = bvz_z; Q[2][i] = bvx_z; Q[3][i] = bvz_x;
                continue;
            }
            REAL t_vxx = A[M_VXX][i] + bvx_x, t_vzz = A[M_VZZ][i] + bvz_z;
            REAL t_vxz = A[M_VXZ][i] + bvx_z, t_vzx = A[M_VZX][i] + bvz_x;
            Q[0][i] = bvx_x + p->bx[ix] * t_vxx;
            Q[1][i] = bvz_z + p->bz[iz] * t_vzz;
            Q[2][i] = bvx_z + p->bzh[iz] * t_vxz;
            Q[3][i] = bvz_x + p->bxh[ix] * t_vzx;
            A[M_VXX][i] = p->ax[ix] * t_vxx;
            A[M_VZX][i] = p->axh[ix] * t_vzx;
            A[M_VZZ][i] = p->az[iz] * t_vzz;
            A[M_VXZ][i] = p->azh[iz] * t_vxz;
        }
    }
}

/* Stress-adjoint apply (kernels.cuh:807-837): adjoint velocities gather the
 * transposed stencils of q (qxx, qzz, qxz, qzx). */
static void stress_adjoint_apply(const EL* p, REAL** A, REAL** Q)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz;
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dqxx_dx = dplus(Q[0], i, 1, M, p->c, ix_);
            REAL dqxz_dz = p->fs ? fs_adj_dz(p, Q[2], ix, iz, 1, 0, 0) : dminus(Q[2], i, nx, M, p->c, iz_);
            REAL dqzx_dx = dminus(Q[3], i, 1, M, p->c, ix_);
            REAL dqzz_dz = p->fs ? fs_adj_dz(p, Q[1], ix, iz, 0, 1, 1) : dplus(Q[1], i, nx, M, p->c, iz_);
            A[VX][i] = A[VX][i] + (dqxx_dx + dqxz_dz);
            A[VZ][i] = A[VZ][i] + (dqzx_dx + dqzz_dz);
        }
    }
}

/* Velocity-adjoint prepare (kernels.cuh:873-958) and apply (989-1019):
 * p = (pxx, pzz, pxz, pzx). */
static void velocity_adjoint(const EL* p, int b, REAL** A, REAL** P)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL* rho = p->rho + b * p->ms;
    const REAL ix_ = R(1) / p->dx, iz_ = R(1) / p->dz, dt = p->dt;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz) {
        for (int ix = 0; ix < nx; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL inv_rho = R(1) / rho[i];
            REAL b_sxx_x = (dt * inv_rho) * A[VX][i];
            REAL b_sxz_z = (dt * inv_rho) * A[VX][i];
            REAL b_sxz_x = (dt * inv_rho) * A[VZ][i];
            REAL b_szz_z = (dt * inv_rho) * A[VZ][i];
            if (!in_pml(p, ix, iz)) {
                P[0][i] = b_sxx_x; P[2][i] = b_sxz_z; P[3][i] = b_sxz_x; P[1][i] = b_szz_z;
                continue;
            }
            REAL t_sxxx = A[M_SXXX][i] + b_sxx_x, t_sxzz = A[M_SXZZ][i] + b_sxz_z;
            REAL t_sxzx = A[M_SXZX][i] + b_sxz_x, t_szzz = A[M_SZZZ][i] + b_szz_z;
            P[0][i] = b_sxx_x + p->bxh[ix] * t_sxxx;
            P[2][i] = b_sxz_z + p->bz[iz] * t_sxzz;
            P[3][i] = b_sxz_x + p->bx[ix] * t_sxzx;
            P[1][i] = b_szz_z + p->bzh[iz] * t_szzz;
            A[M_SXXX][i] = p->axh[ix] * t_sxxx;
            A[M_SXZX][i] = p->ax[ix] * t_sxzx;
            A[M_SXZZ][i] = p->az[iz] * t_sxzz;
            A[M_SZZZ][i] = p->azh[iz] * t_szzz;
        }
    }
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dpxx_dx = dminus(P[0], i, 1, M, p->c, ix_);
            REAL dpzz_dz = p->fs ? fs_adj_dz(p, P[1], ix, iz, 1, 1, 0) : dminus(P[1], i, nx, M, p->c, iz_);
            REAL dpxz_dz = p->fs ? fs_adj_dz(p, P[2], ix, iz, 0, 1, 1) : dplus(P[2], i, nx, M, p->c, iz_);
            REAL dpzx_dx = dplus(P[3], i, 1, M, p->c, ix_);
            A[SXX][i] = A[SXX][i] + dpxx_dx;
            A[SZZ][i] = A[SZZ][i] + dpzz_dz;
            A[SXZ][i] = A[SXZ][i] + (dpxz_dz + dpzx_dx);
        }
    }
}

/* Boundary-saving backward (sg_driver.cuh:760-806, driver_traits.cuh:387-490,
 * 659-826), reverse steps nt-1 .. 1 (the staggered reverse has no it = 0
 * step).  adj: (B, nt, nrec, nrf) record cotangent; grad_* accumulate
 * (B|1, nz, nx) with the model stride (a shared model sums the shots in
 * order).  tape: from oracle_el2d_forward. */
int oracle_el2d_backward(
    int B, int nz, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dx,
    const REAL* coef, const REAL* prof,
    const REAL* vp, const REAL* vs, const REAL* rho, i64 m_stride,
    int nsrc, const int* src, const REAL* wavelet, int nsf, const int* sfields,
    int nrec, const int* rec, int nrf, const int* rfields, int fs,
    const REAL* adj, const REAL* tape, REAL* grad_vp, REAL* grad_vs, REAL* grad_rho)
{
    SETUP_EL;
    const i64 n = (i64)nz * nx;
    const int ns = band_cells(&p, NULL);
    const int z0 = pad[0] + M, z1 = nz - pad[1] - M, x0 = pad[2] + M, x1 = nx - pad[3] - M;
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    const int nbuf = 5 + NF + 8 + 2 + 2;
    REAL* buf = (REAL*)calloc((size_t)n * nbuf, sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    band_cells(&p, cells);
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * nbuf);
        REAL *Fw[5], *A[NF], *Q[4], *P[4];
        for (int f = 0; f < 5; ++f) Fw[f] = buf + f * n;
        for (int f = 0; f < NF; ++f) A[f] = buf + (5 + f) * n;
        for (int f = 0; f < 4; ++f) { Q[f] = buf + (5 + NF + f) * n; P[f] = buf + (5 + NF + 4 + f) * n; }
        REAL *vxn = buf + (5 + NF + 8) * n, *vzn = buf + (5 + NF + 9) * n;
        REAL *lam = buf + (5 + NF + 10) * n, *mu = buf + (5 + NF + 11) * n;
        lame(&p, b, lam, mu);
        REAL *gvp = grad_vp + b * m_stride, *gvs = grad_vs + b * m_stride, *grho = grad_rho + b * m_stride;
        const REAL* rb = rho + b * m_stride;
        for (int f = 0; f < 5; ++f)
            memcpy(Fw[f], tape + (i64)nt * B * 5 * ns + ((i64)b * 5 + f) * n, sizeof(REAL) * n);
        for (int it = nt - 1; it >= 1; --it) {
            /* body-force rho correction at velocity sources, before the residuals */
            for (int k = 0; k < nsf; ++k) {
                if (sfields[k] > 1) continue;
                for (int s = 0; s < nsrc; ++s) {
                    int ix = src[(b * nsrc + s) * 2], iz = src[(b * nsrc + s) * 2 + 1];
                    if (!in_grid(ix, iz, nx, nz)) continue;
                    i64 i = (i64)iz * nx + ix;
                    grho[i] = grho[i] + (A[sfields[k]][i] * wavelet[((i64)b * nsrc + s) * nt + it]) / rb[i];
                }
            }
            /* signed residuals: stress -1, velocity +1 */
            for (int k = 0; k < nrf; ++k) {
                REAL sign = rfields[k] >= 2 ? R(-1) : R(1);
                for (int r = 0; r < nrec; ++r) {
                    int ix = rec[(b * nrec + r) * 2], iz = rec[(b * nrec + r) * 2 + 1];
                    if (!in_grid(ix, iz, nx, nz)) continue;
                    A[rfields[k]][(i64)iz * nx + ix] += sign * adj[(((i64)b * nt + it) * nrec + r) * nrf + k];
                }
            }
            for (int k = 0; k < nsf; ++k) inject(&p, b, Fw[sfields[k]], it, R(-1));
            /* stress half */
            stress_reverse(&p, Fw, lam, mu);
            for (int f = 2; f < 5; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 5 + f) * ns;
                for (int c = 0; c < ns; ++c) Fw[f][cells[c]] = s[c];
            }
            stress_adjoint_prepare(&p, b, A, Q, lam, mu, Fw, vxn, vzn, gvp, gvs, grho);
            for (int k = 0; k < nrf; ++k) {
                const int fld = rfields[k];
                if (fld > 1) continue;
                const REAL* now = Fw[fld];
                const REAL* nxt = fld == 0 ? vxn : vzn;
                for (int r = 0; r < nrec; ++r) {
                    int ix = rec[(b * nrec + r) * 2], iz = rec[(b * nrec + r) * 2 + 1];
                    if (ix < M || ix >= nx - M || iz < M || iz >= nz - M) continue;
                    i64 i = (i64)iz * nx + ix;
                    REAL a = adj[(((i64)b * nt + it) * nrec + r) * nrf + k];
                    grho[i] = grho[i] + ((-a) * (now[i] - nxt[i])) / rb[i];
                }
            }
            stress_adjoint_apply(&p, A, Q);
            /* velocity half */
            velocity_adjoint(&p, b, A, P);
            for (int iz = z0; iz < z1; ++iz)
                for (int ix = x0; ix < x1; ++ix) {
                    i64 i = (i64)iz * nx + ix;
                    vxn[i] = Fw[VX][i]; vzn[i] = Fw[VZ][i];
                }
            velocity_reverse(&p, b, Fw);
            for (int f = 0; f < 2; ++f) {
                const REAL* s = tape + (((i64)(it - 1) * B + b) * 5 + f) * ns;
                for (int c = 0; c < ns; ++c) Fw[f][cells[c]] = s[c];
            }
        }
    }
    free(buf); free(cells);
    return 0;
}
