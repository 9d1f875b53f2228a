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
    int fs;                     /* bit f: traction-free face f (z_lo, z_hi, x_lo, x_hi; pad 0) */
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

/* ---- traction-free faces (image method) ---------------------------------
 * Bit f of `fs` (0 z_lo, 1 z_hi, 2 x_lo, 3 x_hi) makes face f traction free;
 * a free face has no PML pad.  Per axis (0 = z, 1 = x) the low surface is the
 * first physical row / column and the high surface the last; the cells past
 * them are air.  Derivatives along the axis read an air cell as the image of
 * the cell mirrored about the surface -- about the surface node for fields
 * on integer nodes, about the half cell next to it for fields half a cell
 * along the axis ("half") -- negated for odd fields.  On the high side a
 * half field's surface node is itself air.  The M cells from a surface
 * inwards take a unit-weight 2nd-order difference instead of the full
 * stencil.  (elastic_free_surface.cuh:200-465, 466-720.) */
typedef struct { int lo_on, hi_on, lo, hi, n, M; i64 s; REAL h; } FSAX;

static FSAX fs_axis(const EL* p, int a)
{
    FSAX x;
    x.M = p->M;
    if (a == 0) {
        x.lo_on = p->fs & 1; x.hi_on = (p->fs >> 1) & 1;
        x.lo = p->pad[0] + p->M; x.hi = p->nz - p->pad[1] - p->M - 1;
        x.n = p->nz; x.s = p->nx; x.h = p->dz;
    } else {
        x.lo_on = (p->fs >> 2) & 1; x.hi_on = (p->fs >> 3) & 1;
        x.lo = p->pad[2] + p->M; x.hi = p->nx - p->pad[3] - p->M - 1;
        x.n = p->nx; x.s = 1; x.h = p->dx;
    }
    return x;
}

/* u at index j along the axis of the line through `base` (index 0) */
static inline REAL fs_at(const FSAX* x, const REAL* u, i64 base, int j, int odd, int half)
{
    int m;
    if (x->lo_on && j < x->lo) m = half ? 2 * x->lo - 1 - j : 2 * x->lo - j;
    else if (x->hi_on && j >= (half ? x->hi : x->hi + 1)) m = half ? 2 * x->hi - 1 - j : 2 * x->hi - j;
    else return u[base + (i64)j * x->s];
    const REAL v = u[base + (i64)m * x->s];
    return odd ? -v : v;
}

static inline int fs_band(const FSAX* x, int j)
{
    return (x->lo_on && j >= x->lo && j < x->lo + x->M) || (x->hi_on && j > x->hi - x->M && j <= x->hi);
}

/* Derivative along axis a at (ix, iz): fwd = 1 the D+ form (taps j+k and
 * j-k+1), fwd = 0 the D- form (taps j+k-1 and j-k); the plain stencil when
 * neither face of the axis is free. */
static REAL fs_d(const EL* p, const REAL* u, int a, int ix, int iz, int fwd, int odd, int half)
{
    const FSAX x = fs_axis(p, a);
    const int M = p->M;
    const i64 i = (i64)iz * p->nx + ix;
    if (!x.lo_on && !x.hi_on)
        return fwd ? dplus(u, i, x.s, M, p->c, R(1) / x.h) : dminus(u, i, x.s, M, p->c, R(1) / x.h);
    const int j = a == 0 ? iz : ix;
    const i64 base = i - (i64)j * x.s;
    if (fs_band(&x, j)) {
        const REAL g = fwd ? fs_at(&x, u, base, j + 1, odd, half) - fs_at(&x, u, base, j, odd, half)
                           : fs_at(&x, u, base, j, odd, half) - fs_at(&x, u, base, j - 1, odd, half);
        return g / x.h;
    }
    REAL g = R(0);
    for (int k = 1; k <= M; ++k) {
        const REAL up = fwd ? fs_at(&x, u, base, j + k, odd, half) : fs_at(&x, u, base, j + k - 1, odd, half);
        const REAL um = fwd ? fs_at(&x, u, base, j - k + 1, odd, half) : fs_at(&x, u, base, j - k, odd, half);
        g = g + p->c[k] * (up - um);
    }
    return g / x.h;
}

/* Transpose of fs_d without the images (negated, in the sign convention of
 * the plain adjoint stencils: D- for a D+ forward and vice versa) at input
 * index m: an output cell in a band contributes with weight 1, one outside
 * with the full weight; reads outside the grid are skipped. */
static REAL fs_adj_plain(const FSAX* x, const REAL* c, const REAL* q, i64 base, int m, int fwd)
{
    REAL acc = R(0);
    for (int k = 1; k <= x->M; ++k) {
        const int jp = fwd ? m + k - 1 : m + k;
        const int jm = fwd ? m - k : m - k + 1;
        if (jp >= 0 && jp < x->n && !fs_band(x, jp)) acc = acc + c[k] * q[base + (i64)jp * x->s];
        if (jm >= 0 && jm < x->n && !fs_band(x, jm)) acc = acc - c[k] * q[base + (i64)jm * x->s];
    }
    if (fwd) {
        if (fs_band(x, m)) acc = acc + q[base + (i64)m * x->s];
        if (fs_band(x, m - 1)) acc = acc - q[base + (i64)(m - 1) * x->s];
    } else {
        if (fs_band(x, m + 1)) acc = acc + q[base + (i64)(m + 1) * x->s];
        if (fs_band(x, m)) acc = acc - q[base + (i64)m * x->s];
    }
    return acc / x->h;
}

/* Adjoint of fs_d at (ix, iz): zero on air cells (the forward overwrites them
 * with images); else the plain transpose plus, for each free face whose image
 * of this cell lies in the air, the transpose at that air cell folded back
 * with the field's parity. */
static REAL fs_adj(const EL* p, const REAL* q, int a, int ix, int iz, int fwd, int odd, int half)
{
    const FSAX x = fs_axis(p, a);
    const int M = p->M;
    const i64 i = (i64)iz * p->nx + ix;
    if (!x.lo_on && !x.hi_on)
        return fwd ? dminus(q, i, x.s, M, p->c, R(1) / x.h) : dplus(q, i, x.s, M, p->c, R(1) / x.h);
    const int j = a == 0 ? iz : ix;
    const i64 base = i - (i64)j * x.s;
    if ((x.lo_on && j < x.lo) || (x.hi_on && j > x.hi)) return R(0);
    const REAL parity = odd ? R(-1) : R(1);
    REAL g = fs_adj_plain(&x, p->c, q, base, j, fwd);
    if (x.lo_on) {
        const int mj = half ? 2 * x.lo - 1 - j : 2 * x.lo - j;
        if (mj < x.lo) g = g + parity * fs_adj_plain(&x, p->c, q, base, mj, fwd);
    }
    if (x.hi_on) {
        const int mj = half ? 2 * x.hi - 1 - j : 2 * x.hi - j;
        if (mj >= (half ? x.hi : x.hi + 1)) g = g + parity * fs_adj_plain(&x, p->c, q, base, mj, fwd);
    }
    return g;
}

/* Surface rows / columns: the normal-stress conditions (z row: Robertsson
 * sxx, szz = 0; x column: Robertsson szz, sxx = 0) and the shear zeroing of
 * the high-side faces (kernels.cuh:293-303, elastic_free_surface.cuh:485-500). */
static inline int fs_zrow(const EL* p, int iz)
{
    return ((p->fs & 1) && iz == p->pad[0] + p->M) || ((p->fs & 2) && iz == p->nz - p->pad[1] - p->M - 1);
}
static inline int fs_xcol(const EL* p, int ix)
{
    return ((p->fs & 4) && ix == p->pad[2] + p->M) || ((p->fs & 8) && ix == p->nx - p->pad[3] - p->M - 1);
}
static inline int fs_zero_shear(const EL* p, int ix, int iz)
{
    return ((p->fs & 2) && iz == p->nz - p->pad[1] - p->M - 1) || ((p->fs & 8) && ix == p->nx - p->pad[3] - p->M - 1);
}

/* The stress kernel's CPML test: a free surface row / column stays in the
 * CPML branch (kernels.cuh:216-234). */
static inline int in_pml_stress(const EL* p, int ix, int iz)
{
    const int M = p->M;
    const int zlo = (p->fs & 1) ? p->pad[0] + M + 1 : p->pad[0] + M;
    const int zhi = (p->fs & 2) ? p->nz - p->pad[1] - M - 1 : p->nz - p->pad[1] - M;
    const int xlo = (p->fs & 4) ? p->pad[2] + M + 1 : p->pad[2] + M;
    const int xhi = (p->fs & 8) ? p->nx - p->pad[3] - M - 1 : p->nx - p->pad[3] - M;
    return ix < xlo || ix >= xhi || iz < zlo || iz >= zhi;
}

#define DZ(u, fwd, odd, half) fs_d(p, (u), 0, ix, iz, (fwd), (odd), (half))
#define DX(u, fwd, odd, half) fs_d(p, (u), 1, ix, iz, (fwd), (odd), (half))
#define AZ(q, fwd, odd, half) fs_adj(p, (q), 0, ix, iz, (fwd), (odd), (half))
#define AX(q, fwd, odd, half) fs_adj(p, (q), 1, ix, iz, (fwd), (odd), (half))

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
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dsxx_dx = DX(F[SXX], 1, 1, 0);
            REAL dsxz_dz = DZ(F[SXZ], 0, 1, 1);
            REAL dsxz_dx = DX(F[SXZ], 0, 1, 1);
            REAL dszz_dz = DZ(F[SZZ], 1, 1, 0);
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
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dvx_dx = DX(F[VX], 0, 1, 1);
            REAL dvz_dz = DZ(F[VZ], 0, 1, 1);
            REAL dvx_dz = DZ(F[VX], 1, 0, 0);
            REAL dvz_dx = DX(F[VZ], 1, 0, 0);
            REAL lam = lam_[i], mu = mu_[i];
            const int pml = in_pml_stress(p, ix, iz);
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
            /* Robertsson corrections first, then the zeroing (kernels.cuh:293-303) */
            const int zs = fs_zrow(p, iz), xs = fs_xcol(p, ix);
            if (zs) F[SXX][i] = F[SXX][i] + (-p->dt) * lam * ((lam / (lam + R(2) * mu)) * dvx_dx + dvz_dz);
            if (xs) F[SZZ][i] = F[SZZ][i] + (-p->dt) * lam * ((lam / (lam + R(2) * mu)) * dvz_dz + dvx_dx);
            if (zs) F[SZZ][i] = R(0);
            if (xs) F[SXX][i] = R(0);
            if (fs_zero_shear(p, ix, iz)) F[SXZ][i] = R(0);
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
 * face (kernels.cuh:405-535, band pad + M + 1); a free face narrows to the
 * halo M. */
static void reverse_box(const EL* p, int lo[2], int hi[2])
{
    const int M = p->M;
    lo[0] = (p->fs & 1) ? M : p->pad[0] + M + 1;
    hi[0] = p->nz - ((p->fs & 2) ? M : p->pad[1] + M + 1);
    lo[1] = (p->fs & 4) ? M : p->pad[2] + M + 1;
    hi[1] = p->nx - ((p->fs & 8) ? M : p->pad[3] + M + 1);
}

static void stress_reverse(const EL* p, REAL** F, const REAL* lam_, const REAL* mu_)
{
    const int nx = p->nx;
    int lo[2], hi[2];
    reverse_box(p, lo, hi);
    #pragma omp parallel for schedule(static)
    for (int iz = lo[0]; iz < hi[0]; ++iz) {
        for (int ix = lo[1]; ix < hi[1]; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dvx_dx = DX(F[VX], 0, 1, 1);
            REAL dvz_dz = DZ(F[VZ], 0, 1, 1);
            REAL dvx_dz = DZ(F[VX], 1, 0, 0);
            REAL dvz_dx = DX(F[VZ], 1, 0, 0);
            REAL lam = lam_[i], mu = mu_[i];
            F[SXX][i] = F[SXX][i] - p->dt * ((lam + R(2) * mu) * dvx_dx + lam * dvz_dz);
            F[SZZ][i] = F[SZZ][i] - p->dt * ((lam + R(2) * mu) * dvz_dz + lam * dvx_dx);
            F[SXZ][i] = F[SXZ][i] - (p->dt * mu) * (dvx_dz + dvz_dx);
        }
    }
}

static void velocity_reverse(const EL* p, int b, REAL** F)
{
    const int nx = p->nx;
    const REAL* rho = p->rho + b * p->ms;
    int lo[2], hi[2];
    reverse_box(p, lo, hi);
    #pragma omp parallel for schedule(static)
    for (int iz = lo[0]; iz < hi[0]; ++iz) {
        for (int ix = lo[1]; ix < hi[1]; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dsxx_dx = DX(F[SXX], 1, 1, 0);
            REAL dsxz_dz = DZ(F[SXZ], 0, 1, 1);
            REAL dsxz_dx = DX(F[SXZ], 0, 1, 1);
            REAL dszz_dz = DZ(F[SZZ], 1, 1, 0);
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
    const REAL dt = p->dt;
    #pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz) {
        for (int ix = 0; ix < nx; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL lam = lam_[i], mu = mu_[i];
            REAL bsxx = A[SXX][i], bszz = A[SZZ][i], bsxz = A[SXZ][i];
            const int zs = fs_zrow(p, iz), xs = fs_xcol(p, ix);
            if (zs) { bszz = R(0); A[SZZ][i] = R(0); }
            if (xs) { bsxx = R(0); A[SXX][i] = R(0); }
            if (fs_zero_shear(p, ix, iz)) { bsxz = R(0); A[SXZ][i] = R(0); }
            if (gvp && ix >= x0 && ix < x1 && iz >= z0 && iz < z1) {
                REAL fvx_x = DX(Fw[VX], 0, 1, 1);
                REAL fvz_z = DZ(Fw[VZ], 0, 1, 1);
                REAL fvx_z = DZ(Fw[VX], 1, 0, 0);
                REAL fvz_x = DX(Fw[VZ], 1, 0, 0);
                REAL gl, gm;
                if (zs && xs) {
                    gl = R(0); gm = R(0);     /* a corner: every stress zeroed */
                } else if (zs || xs) {
                    /* d/d(lam, mu) of the surface update of the tangential
                     * normal stress, dt C d(tangential v) with
                     * C = 4 mu (lam + mu) / (lam + 2 mu) (kernels.cuh:633-646) */
                    const REAL vp2 = vp[i] * vp[i], vs2 = vs[i] * vs[i], vp4 = vp2 * vp2;
                    const REAL a = zs ? bsxx * fvx_x : bszz * fvz_z;
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
            if (zs && xs) {
                bvx_x = R(0); bvz_z = R(0);
            } else if (zs) {   /* transposes of the corrected surface updates */
                const REAL c_surf = R(4) * mu * (lam + mu) / (lam + R(2) * mu);
                bvx_x = dt * c_surf * bsxx;
                bvz_z = R(0);
            } else if (xs) {
                const REAL c_surf = R(4) * mu * (lam + mu) / (lam + R(2) * mu);
                bvz_z = dt * c_surf * bszz;
                bvx_x = R(0);
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
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            const i64 i = (i64)iz * nx + ix;
            REAL dqxx_dx = AX(Q[0], 0, 1, 1);
            REAL dqxz_dz = AZ(Q[2], 1, 0, 0);
            REAL dqzx_dx = AX(Q[3], 1, 0, 0);
            REAL dqzz_dz = AZ(Q[1], 0, 1, 1);
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
    const REAL dt = p->dt;
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
            REAL dpxx_dx = AX(P[0], 1, 1, 0);
            REAL dpzz_dz = AZ(P[1], 1, 1, 0);
            REAL dpxz_dz = AZ(P[2], 0, 1, 1);
            REAL dpzx_dx = AX(P[3], 0, 1, 1);
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
