/*
 * fd_oracle.c -- CPU restatement of the reference's compiled (impl='c')
 * finite-difference path, used ONLY as test infrastructure: the parity
 * checker of the CUDA library and the timed CPU baseline.  It is never linked
 * into, loaded by or called from the product library.
 *
 * Built twice by oracle/Makefile: REAL=float (liboracle_f32.so, the float32
 * restatement that is pinned against the reference's own outputs in
 * tests/golden/) and REAL=double (liboracle_f64.so, the FP64 oracle the
 * CUDA results are also measured against).  Compiled with -ffp-contract=off,
 * like the reference's host core (src/sweep/backend/c/hostcore.py:74-80), so
 * every operation rounds once, in the reference's expression order.
 *
 * Layout: every field is (B, nz, nx) or (B, nz, ny, nx), x fastest, on the
 * runtime grid (physical + PML pad + stencil halo M per face).  Coordinates
 * are runtime-grid (x, [y,] z) int32 triples; off-grid ones are skipped
 * (reference src/sweep/csrc/cuda/common/common.cu:24-28,137-138).
 *
 * What each function restates (reference paths, relative to the project root):
 *   forward step      src/sweep/csrc/cuda/equations/acoustic2d/forward_split.cu:40-168
 *                     (interior fast path and CPML ring, one expression tree)
 *   Laplacian         src/sweep/csrc/cuda/operators/laplace.cuh:93-100, 327-380
 *                     (difference form, minus tap first)
 *   first derivative  src/sweep/csrc/cuda/operators/gradient.cuh:49-88
 *   fused d(a psi)    src/sweep/csrc/cuda/equations/acoustic2d/kernels.cuh:30-77
 *   adjoint step      src/sweep/csrc/cuda/equations/acoustic2d/adjoint_split.cu:27-196
 *   reconstruction    src/sweep/csrc/cuda/equations/acoustic2d/kernels.cuh:474-574
 *   strip imaging     src/sweep/csrc/cuda/equations/acoustic2d/kernels.cu:83-131
 *   step order        src/sweep/csrc/cuda/common/eq_driver.cuh:377-434 (forward),
 *                     814-880 (boundary-saving reverse), and
 *                     src/sweep/csrc/cuda/equations/acoustic2d/driver_traits.cuh:529-635
 *   strip geometry    src/sweep/csrc/cuda/common/boundary/strip.cuh:45-118
 */
#include <stdlib.h>
#include <string.h>
#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
#endif

#ifndef REAL
#define REAL float
#endif
#define R(x) ((REAL)(x))

typedef long long i64;

/* ------------------------------------------------------ subnormals as zero */
/* oracle_ftz(1) sets flush-to-zero and denormals-are-zero in every thread of
 * the OpenMP team (the caller's included), oracle_ftz(0) restores each
 * thread's previous mode.  The device flushes float subnormals (the CUDA
 * path's -ftz=true) and so does the reference's host core
 * (src/sweep/csrc/host/launch.h:45-83): on x86 every subnormal operand or
 * result otherwise takes a microcode assist, which slows a decaying
 * wavefield several times over.  The Python wrapper brackets every oracle
 * call with the pair. */
static unsigned ftz_saved;
static int ftz_held;
#pragma omp threadprivate(ftz_saved, ftz_held)

void oracle_ftz(int on)
{
#if defined(__x86_64__) || defined(__i386__)
    #pragma omp parallel
    {
        if (on) {
            if (!ftz_held) { ftz_saved = _mm_getcsr(); ftz_held = 1; }
            _mm_setcsr(ftz_saved | 0x8040u);
        } else if (ftz_held) {
            _mm_setcsr(ftz_saved);
            ftz_held = 0;
        }
    }
#else
    (void)on;
#endif
}

/* ------------------------------------------------------------------ helpers */

/* Half-open physical box of one axis on the runtime grid. */
static void phys_range(int n, int M, int pad_lo, int pad_hi, int* p0, int* p1)
{
    *p0 = pad_lo + M;
    *p1 = n - pad_hi - M;
}

/* Strip widths of the boundary-saving shell (driver_traits.cuh:188 save_width,
 * clipped like boundary/strip.cuh:63-67 bs_strip_widths). */
static void strip_widths(int extent, int w, int* lo, int* hi)
{
    int l = w < (extent > 0 ? extent : 0) ? w : (extent > 0 ? extent : 0);
    int rem = extent - l; if (rem < 0) rem = 0;
    int h = w < rem ? w : rem;
    *lo = l; *hi = h;
}

/* Number of strip cells of a 2-D physical box and their flat indices, in the
 * band-imaging order: top rows, bottom rows (full box width), then left and
 * right columns over the inner rows (kernels.cu:95-107). */
static int strip_cells_2d(int nz, int nx, int M, const int* pad, int w, int* out)
{
    int z0, z1, x0, x1;
    phys_range(nz, M, pad[0], pad[1], &z0, &z1);
    phys_range(nx, M, pad[2], pad[3], &x0, &x1);
    int wzl, wzh, wxl, wxh;
    strip_widths(z1 - z0, w, &wzl, &wzh);
    strip_widths(x1 - x0, w, &wxl, &wxh);
    int bw = x1 - x0, zi0 = z0 + wzl, zi1 = z1 - wzh, bh = zi1 - zi0;
    if (bh < 0) bh = 0;
    int n = 0;
    for (int t = 0; t < wzl * bw; ++t) { if (out) out[n] = (z0 + t / bw) * nx + x0 + t % bw; ++n; }
    for (int t = 0; t < wzh * bw; ++t) { if (out) out[n] = (zi1 + t / bw) * nx + x0 + t % bw; ++n; }
    for (int t = 0; t < wxl * bh; ++t) { if (out) out[n] = (zi0 + t / wxl) * nx + x0 + t % wxl; ++n; }
    for (int t = 0; t < wxh * bh; ++t) { if (out) out[n] = (zi0 + t / wxh) * nx + (x1 - wxh) + t % wxh; ++n; }
    return n;
}

/* Laplacian along one axis as the forward and the reconstruction take it
 * (laplace.cuh:68-100, 327-445): the difference form
 * sum_k c_k ((u_-k - u0) + (u_+k - u0)) / h^2, minus tap first, at every order
 * but 4; order 4 (M = 2) keeps the summed form
 * (c1 (u_-1 + u_1) + c2 (u_-2 + u_2) - c0 u0) / h^2 with c0 = 5/2
 * (laplace.cuh:145-200).  The adjoint takes the difference form everywhere. */
static inline REAL lap_axis(const REAL* u, i64 i, i64 s, int M, const REAL* lc, REAL h)
{
    REAL u0 = u[i];
    if (M == 2)
        return ((lc[1] * (u[i - s] + u[i + s]) + lc[2] * (u[i - 2 * s] + u[i + 2 * s])) - R(2.5) * u0) / (h * h);
    REAL acc = R(0);
    for (int k = 1; k <= M; ++k) {
        REAL t = lc[k] * ((u[i - k * s] - u0) + (u[i + k * s] - u0));
        acc = (k == 1) ? t : acc + t;
    }
    return acc / (h * h);
}

/* Centered first derivative (gradient.cuh:49-88): sum_k g_k (u_k - u_-k) / h. */
static inline REAL grad_axis(const REAL* u, i64 i, i64 s, int M, const REAL* gc, REAL h)
{
    REAL acc = R(0);
    for (int k = 1; k <= M; ++k) {
        REAL t = gc[k] * (u[i + k * s] - u[i - k * s]);
        acc = (k == 1) ? t : acc + t;
    }
    return acc / h;
}

/* Fused d(a psi)/dx tap form (kernels.cuh:30-77). */
static inline REAL grad_apsi(const REAL* a, int ia, const REAL* psi, i64 i, i64 s,
                             int M, const REAL* gc, REAL h)
{
    REAL acc = R(0);
    for (int k = 1; k <= M; ++k) {
        REAL t = gc[k] * (a[ia + k] * psi[i + k * s] - a[ia - k] * psi[i - k * s]);
        acc = (k == 1) ? t : acc + t;
    }
    return acc / h;
}

/* ----------------------------------------------------------- acoustic 2-D */

typedef struct {
    int B, nz, nx, nt, M;
    int pad[4];              /* PML pad per face: z_lo, z_hi, x_lo, x_hi */
    REAL dt, dz, dx;
    const REAL* lap;         /* [M+1], lap[1..M] */
    const REAL* gco;         /* [M+1], gco[1..M] */
    const REAL *az, *bz, *dbz, *ax, *bx, *dbx;
    const REAL* vp; i64 vp_stride;   /* 0 = one model shared by every shot */
    int nsrc; const int* src; const REAL* wavelet;   /* (B,nsrc,2), (B,nsrc,nt) */
    int nrec; const int* rec;                         /* (B,nrec,2) */
} A2D;

static int in_grid2(int ix, int iz, int nx, int nz) { return ix >= 0 && ix < nx && iz >= 0 && iz < nz; }

/* One forward step of shot b: u_next from u_now / u_prev, CPML memories
 * updated (psi written to psin, zeta in place: forward_split.cu:86-168). */
static void a2d_step(const A2D* p, int b, const REAL* un, const REAL* up, REAL* unext,
                     const REAL* psix, const REAL* psiz, REAL* psixn, REAL* psizn,
                     REAL* zetax, REAL* zetaz)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL* vp = p->vp + b * p->vp_stride;
    const int pml_x0 = p->pad[2] + M, pml_x1 = nx - (p->pad[3] + M);
    const int pml_z0 = p->pad[0] + M, pml_z1 = nz - (p->pad[1] + M);
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            i64 i = (i64)iz * nx + ix;
            REAL lx = lap_axis(un, i, 1, M, p->lap, p->dx);
            REAL lz = lap_axis(un, i, nx, M, p->lap, p->dz);
            REAL v = vp[i];
            REAL v2dt2 = ((v * v) * p->dt) * p->dt;
            int cx = (ix < pml_x0 + M) || (ix >= pml_x1 - M);
            int cz = (iz < pml_z0 + M) || (iz >= pml_z1 - M);
            REAL w;
            if (!cx && !cz) {
                w = lx + lz;
            } else {
                w = R(0);
                if (cx) {
                    REAL a = p->ax[ix], bb = p->bx[ix], db = p->dbx[ix];
                    REAL du = grad_axis(un, i, 1, M, p->gco, p->dx);
                    REAL dap = grad_apsi(p->ax, ix, psix, i, 1, M, p->gco, p->dx);
                    REAL tmp = ((R(1) + bb) * lx + db * du) + dap;
                    w = w + ((R(1) + bb) * tmp + a * zetax[i]);
                    psixn[i] = bb * du + a * psix[i];
                    zetax[i] = bb * tmp + a * zetax[i];
                } else {
                    w = w + lx;
                }
                if (cz) {
                    REAL a = p->az[iz], bb = p->bz[iz], db = p->dbz[iz];
                    REAL du = grad_axis(un, i, nx, M, p->gco, p->dz);
                    REAL dap = grad_apsi(p->az, iz, psiz, i, nx, M, p->gco, p->dz);
                    REAL tmp = ((R(1) + bb) * lz + db * du) + dap;
                    w = w + ((R(1) + bb) * tmp + a * zetaz[i]);
                    psizn[i] = bb * du + a * psiz[i];
                    zetaz[i] = bb * tmp + a * zetaz[i];
                } else {
                    w = w + lz;
                }
            }
            unext[i] = (R(2) * un[i] - up[i]) + v2dt2 * w;
        }
    }
}

/* Tape: per step the strip cells of u_now (U[it]) for every shot, then the
 * last two states (U[nt-1], U[nt]) of every shot. */
long long oracle_a2d_tape_len(int B, int nz, int nx, int nt, int M, const int* pad)
{
    int w = M + 1;
    int ns = strip_cells_2d(nz, nx, M, pad, w, NULL);
    return (long long)nt * B * ns + 2LL * B * nz * nx;
}

static void inject2(const A2D* p, int b, REAL* u, const REAL* amp, int n, const int* loc, int it, REAL sign)
{
    for (int s = 0; s < n; ++s) {
        int ix = loc[(b * n + s) * 2], iz = loc[(b * n + s) * 2 + 1];
        if (!in_grid2(ix, iz, p->nx, p->nz)) continue;
        u[(i64)iz * p->nx + ix] += sign * amp[((i64)b * n + s) * p->nt + it];
    }
}

/* Forward: records (B, nrec, nt); tape filled when non-NULL.
 * Step order (eq_driver.cuh:377-434): stencil -> save strips of u_now ->
 * add source to u_next -> record u_next -> rotate. */
int oracle_a2d_forward(
    int B, int nz, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dx,
    const REAL* lap, const REAL* gco,
    const REAL* az, const REAL* bz, const REAL* dbz, const REAL* ax, const REAL* bx, const REAL* dbx,
    const REAL* vp, i64 vp_stride,
    int nsrc, const int* src, const REAL* wavelet, int nrec, const int* rec,
    REAL* record, REAL* tape)
{
    A2D p = {B, nz, nx, nt, M, {pad[0], pad[1], pad[2], pad[3]}, dt, dz, dx, lap, gco,
             az, bz, dbz, ax, bx, dbx, vp, vp_stride, nsrc, src, wavelet, nrec, rec};
    const i64 n = (i64)nz * nx;
    const int w = M + 1;
    int ns = strip_cells_2d(nz, nx, M, pad, w, NULL);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    strip_cells_2d(nz, nx, M, pad, w, cells);
    REAL* buf = (REAL*)calloc((size_t)n * 7, sizeof(REAL));
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * 7);
        REAL *u0 = buf, *u1 = buf + n, *u2 = buf + 2 * n;
        REAL *psix = buf + 3 * n, *psiz = buf + 4 * n, *zx = buf + 5 * n, *zz = buf + 6 * n;
        REAL* psin = (REAL*)calloc((size_t)n * 2, sizeof(REAL));
        REAL *psixn = psin, *psizn = psin + n;
        REAL *up = u0, *un = u1, *unx = u2;
        for (int it = 0; it < nt; ++it) {
            a2d_step(&p, b, un, up, unx, psix, psiz, psixn, psizn, zx, zz);
            if (tape) {
                REAL* dst = tape + ((i64)it * B + b) * ns;
                for (int c = 0; c < ns; ++c) dst[c] = un[cells[c]];
            }
            inject2(&p, b, unx, wavelet, nsrc, src, it, R(1));
            for (int r = 0; r < nrec; ++r) {
                int ix = rec[(b * nrec + r) * 2], iz = rec[(b * nrec + r) * 2 + 1];
                if (!in_grid2(ix, iz, nx, nz)) continue;
                record[((i64)b * nrec + r) * nt + it] = unx[(i64)iz * nx + ix];
            }
            REAL* t = up; up = un; un = unx; unx = t;
            t = psix; psix = psixn; psixn = t;
            t = psiz; psiz = psizn; psizn = t;
        }
        if (tape) {
            REAL* last = tape + (i64)nt * B * ns + (i64)b * 2 * n;
            memcpy(last, up, sizeof(REAL) * n);       /* U[nt-1] */
            memcpy(last + n, un, sizeof(REAL) * n);   /* U[nt]   */
        }
        free(psin);
    }
    free(buf); free(cells);
    return 0;
}

/* One exact adjoint step of shot b (adjoint_split.cu:27-196): l_next from
 * l_now / l_prev, adjoint CPML memories read from (psi, zeta) and written to
 * (psi_o, zeta_o). */
static void a2d_adjoint(const A2D* p, int b, const REAL* ln, const REAL* lp, REAL* lnext,
                        const REAL* psix, const REAL* psiz, const REAL* zx, const REAL* zz,
                        REAL* psix_o, REAL* psiz_o, REAL* zx_o, REAL* zz_o)
{
    const int nz = p->nz, nx = p->nx, M = p->M;
    const REAL* vp = p->vp + b * p->vp_stride;
    const REAL dt2 = p->dt * p->dt;
    const REAL* lc = p->lap;
    const REAL* gc = p->gco;
    const REAL invdx2 = R(1) / (p->dx * p->dx), invdz2 = R(1) / (p->dz * p->dz);
    const REAL invdx = R(1) / p->dx, invdz = R(1) / p->dz;
    const int ix_in0 = p->pad[2] + 2 * M + 1, ix_in1 = nx - (p->pad[3] + 2 * M + 1);
    const int iz_in0 = p->pad[0] + 2 * M + 1, iz_in1 = nz - (p->pad[1] + 2 * M + 1);
#define GW_AT(n) ((((vp[n] * vp[n]) * dt2)) * ln[n])
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz) {
        for (int ix = M; ix < nx - M; ++ix) {
            i64 i = (i64)iz * nx + ix;
            REAL gun = ln[i];
            REAL c0c = vp[i]; c0c = (c0c * c0c) * dt2;
            REAL gw = c0c * gun;
            int pure = ix >= ix_in0 && ix < ix_in1 && iz >= iz_in0 && iz < iz_in1;
            if (pure) {
                REAL lx = R(0), lz = R(0);
                for (int k = 1; k <= M; ++k) {
                    lx = lx + lc[k] * ((GW_AT(i + k) - gw) + (GW_AT(i - k) - gw));
                    lz = lz + lc[k] * ((GW_AT(i + (i64)k * nx) - gw) + (GW_AT(i - (i64)k * nx) - gw));
                }
                lnext[i] = ((R(2) * gun - lp[i]) + lx * invdx2) + lz * invdz2;
                continue;
            }
            REAL ax_ = p->ax[ix], az_ = p->az[iz], bx_ = p->bx[ix], bz_ = p->bz[iz];
            REAL gtx0 = bx_ * zx[i] + (R(1) + bx_) * gw;
            REAL gtz0 = bz_ * zz[i] + (R(1) + bz_) * gw;
#define GTX(n, c) (p->bx[c] * zx[n] + ((R(1) + p->bx[c]) * ((vp[n] * vp[n]) * dt2)) * ln[n])
#define GTZ(n, c) (p->bz[c] * zz[n] + ((R(1) + p->bz[c]) * ((vp[n] * vp[n]) * dt2)) * ln[n])
            REAL lx0 = (R(1) + bx_) * gtx0;
            REAL Lx = R(0), Dgx = R(0), Dqx = R(0);
            for (int k = 1; k <= M; ++k) {
                i64 np = i + k, nm = i - k; int cp = ix + k, cm = ix - k;
                REAL tp = GTX(np, cp), tm = GTX(nm, cm);
                REAL bp = p->bx[cp], bm = p->bx[cm];
                Lx = Lx + lc[k] * ((((R(1) + bp) * tp) - lx0) + (((R(1) + bm) * tm) - lx0));
                Dgx = Dgx + gc[k] * ((bp * psix[np] + p->dbx[cp] * tp) - (bm * psix[nm] + p->dbx[cm] * tm));
                Dqx = Dqx + gc[k] * (tp - tm);
            }
            Lx = Lx * invdx2; Dgx = Dgx * invdx; Dqx = Dqx * invdx;
            REAL lz0 = (R(1) + bz_) * gtz0;
            REAL Lz = R(0), Dgz = R(0), Dqz = R(0);
            for (int k = 1; k <= M; ++k) {
                i64 np = i + (i64)k * nx, nm = i - (i64)k * nx; int cp = iz + k, cm = iz - k;
                REAL tp = GTZ(np, cp), tm = GTZ(nm, cm);
                REAL bp = p->bz[cp], bm = p->bz[cm];
                Lz = Lz + lc[k] * ((((R(1) + bp) * tp) - lz0) + (((R(1) + bm) * tm) - lz0));
                Dgz = Dgz + gc[k] * ((bp * psiz[np] + p->dbz[cp] * tp) - (bm * psiz[nm] + p->dbz[cm] * tm));
                Dqz = Dqz + gc[k] * (tp - tm);
            }
            Lz = Lz * invdz2; Dgz = Dgz * invdz; Dqz = Dqz * invdz;
            lnext[i] = (R(2) * gun - lp[i]) + (((Lx + Lz) - Dgx) - Dgz);
            psix_o[i] = ax_ * (psix[i] - Dqx);
            psiz_o[i] = az_ * (psiz[i] - Dqz);
            zx_o[i] = ax_ * (zx[i] + gw);
            zz_o[i] = az_ * (zz[i] + gw);
#undef GTX
#undef GTZ
        }
    }
#undef GW_AT
}

/* Boundary-saving backward (eq_driver.cuh:814-880, driver_traits.cuh:490-635).
 * adj: (B, nrec, nt) record cotangent; grad_vp accumulates (B|1, nz, nx) with
 * the model's stride (a shared model sums the per-shot images in shot order);
 * grad_wavelet (B, nsrc, nt) or NULL. */
int oracle_a2d_backward(
    int B, int nz, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dx,
    const REAL* lap, const REAL* gco,
    const REAL* az, const REAL* bz, const REAL* dbz, const REAL* ax, const REAL* bx, const REAL* dbx,
    const REAL* vp, i64 vp_stride,
    int nsrc, const int* src, const REAL* wavelet, int nrec, const int* rec,
    const REAL* adj, const REAL* tape, REAL* grad_vp, REAL* grad_wavelet,
    REAL* illum_s, REAL* illum_r)
{
    A2D p = {B, nz, nx, nt, M, {pad[0], pad[1], pad[2], pad[3]}, dt, dz, dx, lap, gco,
             az, bz, dbz, ax, bx, dbx, vp, vp_stride, nsrc, src, wavelet, nrec, rec};
    const i64 n = (i64)nz * nx;
    const int w = M + 1;
    int ns = strip_cells_2d(nz, nx, M, pad, w, NULL);
    int* cells = (int*)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    char* in_strip = (char*)calloc((size_t)n, 1);
    strip_cells_2d(nz, nx, M, pad, w, cells);
    for (int c = 0; c < ns; ++c) in_strip[cells[c]] = 1;
    /* adjoint: 3 lambda + psi/zeta double buffers; reconstruction: 3 u; per-shot gradient */
    REAL* buf = (REAL*)malloc(sizeof(REAL) * n * 15);
    if (!buf || !cells || !in_strip) { free(buf); free(cells); free(in_strip); return 1; }
    int z0, z1, x0, x1;
    phys_range(nz, M, pad[0], pad[1], &z0, &z1);
    phys_range(nx, M, pad[2], pad[3], &x0, &x1);
    const int rz0 = pad[0] + 2 * M + 1, rz1 = nz - (pad[1] + 2 * M + 1);
    const int rx0 = pad[2] + 2 * M + 1, rx1 = nx - (pad[3] + 2 * M + 1);
    const REAL dt2 = dt * dt;
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * 15);
        REAL *l0 = buf, *l1 = buf + n, *l2 = buf + 2 * n;
        REAL *aps[2] = {buf + 3 * n, buf + 4 * n}, *apz[2] = {buf + 5 * n, buf + 6 * n};
        REAL *azx[2] = {buf + 7 * n, buf + 8 * n}, *azz[2] = {buf + 9 * n, buf + 10 * n};
        REAL *r0 = buf + 11 * n, *r1 = buf + 12 * n, *r2 = buf + 13 * n;
        REAL* g = buf + 14 * n;
        const REAL* vpb = vp + b * vp_stride;
        REAL *lp = l0, *ln = l1, *lnx = l2;
        int cur = 0;
        /* seed (driver_traits.cuh:493-505): prev = U[nt], now = U[nt-1], rim zeroed */
        const REAL* last = tape + (i64)nt * B * ns + (i64)b * 2 * n;
        REAL *rp = r0, *rn = r1, *rnx = r2;
        memcpy(rp, last + n, sizeof(REAL) * n);
        memcpy(rn, last, sizeof(REAL) * n);
        for (int iz = 0; iz < nz; ++iz)
            for (int ix = 0; ix < nx; ++ix)
                if (iz < z0 || iz >= z1 || ix < x0 || ix >= x1) {
                    rp[(i64)iz * nx + ix] = R(0);
                    rn[(i64)iz * nx + ix] = R(0);
                }
        for (int it = nt - 1; it >= 0; --it) {
            a2d_adjoint(&p, b, ln, lp, lnx, aps[cur], apz[cur], azx[cur], azz[cur],
                        aps[1 - cur], apz[1 - cur], azx[1 - cur], azz[1 - cur]);
            inject2(&p, b, lnx, adj, nrec, rec, it, R(1));
            { REAL* t = lp; lp = ln; ln = lnx; lnx = t; }
            cur = 1 - cur;
            if (grad_wavelet) {
                for (int s = 0; s < nsrc; ++s) {
                    int ix = src[(b * nsrc + s) * 2], iz = src[(b * nsrc + s) * 2 + 1];
                    if (!in_grid2(ix, iz, nx, nz)) continue;
                    grad_wavelet[((i64)b * nsrc + s) * nt + it] += ln[(i64)iz * nx + ix];
                }
            }
            if (it == 0) {
                /* the it == 0 tail: no reconstruction, no imaging; the receiver
                   illumination still takes lambda(0)^2 (driver_traits.cuh:515-527) */
                if (illum_r)
                    for (int iz = z0; iz < z1; ++iz)
                        for (int ix = x0; ix < x1; ++ix) {
                            const i64 i = (i64)iz * nx + ix;
                            illum_r[i] += ln[i] * ln[i];
                        }
                break;
            }
            /* NOPML reconstruction + fused imaging (kernels.cuh:474-528) */
            #pragma omp parallel for schedule(static)
            for (int iz = rz0; iz < rz1; ++iz) {
                for (int ix = rx0; ix < rx1; ++ix) {
                    i64 i = (i64)iz * nx + ix;
                    REAL wsum = lap_axis(rn, i, 1, M, lap, dx) + lap_axis(rn, i, nx, M, lap, dz);
                    REAL v = vpb[i];
                    REAL u0 = rn[i], up = rp[i];
                    REAL un = (R(2) * u0 - up) + (((v * v) * dt) * dt) * wsum;
                    rnx[i] = un;
                    REAL utt = ((un - R(2) * u0) + up) / dt2;
                    g[i] = g[i] + ((((R(2) * dt) * dt) * utt) * ln[i]) / v;
                }
            }
            /* restore the strips with the saved U[it-1] (runtime.cuh:1157-1201) */
            const REAL* saved = tape + ((i64)(it - 1) * B + b) * ns;
            for (int c = 0; c < ns; ++c) rnx[cells[c]] = saved[c];
            /* take s^it back out of a source cell the restore overwrote (common.cu:252-290) */
            for (int s = 0; s < nsrc; ++s) {
                int ix = src[(b * nsrc + s) * 2], iz = src[(b * nsrc + s) * 2 + 1];
                if (!in_grid2(ix, iz, nx, nz)) continue;
                i64 i = (i64)iz * nx + ix;
                if (in_strip[i]) rnx[i] -= wavelet[((i64)b * nsrc + s) * nt + it];
            }
            /* strip imaging (kernels.cu:83-131) */
            for (int c = 0; c < ns; ++c) {
                i64 i = cells[c];
                REAL utt = ((rnx[i] - R(2) * rn[i]) + rp[i]) / dt2;
                g[i] = g[i] + ((((R(2) * dt) * dt) * utt) * ln[i]) / vpb[i];
            }
            /* illumination on the physical box, the three time levels the
               imaging used, before the source injection (kernels.cu:133-182,
               driver_traits.cuh:610-626): sum_t u_tt^2 and sum_t lambda^2,
               summed over shots */
            if (illum_s)
                for (int iz = z0; iz < z1; ++iz)
                    for (int ix = x0; ix < x1; ++ix) {
                        const i64 i = (i64)iz * nx + ix;
                        illum_r[i] += ln[i] * ln[i];
                        const REAL utt = ((rnx[i] - R(2) * rn[i]) + rp[i]) / dt2;
                        illum_s[i] += utt * utt;
                    }
            inject2(&p, b, rnx, wavelet, nsrc, src, it, R(1));
            { REAL* t = rp; rp = rn; rn = rnx; rnx = t; }
        }
        REAL* gout = grad_vp + b * vp_stride;
        for (i64 i = 0; i < n; ++i) gout[i] += g[i];
    }
    free(buf); free(cells); free(in_strip);
    return 0;
}
