/*
 * fd_oracle3d.c -- CPU restatement of the reference's compiled 3-D acoustic
 * path (impl='c'), test infrastructure only (see fd_oracle.c for the build and
 * the rules).
 *
 *   forward step     src/sweep/csrc/cuda/equations/acoustic3d/forward_split.cu:79-290
 *                    (interior; per-axis CPML shell with the product-rule split
 *                    a * d(psi) + d(a) * psi; branch on the band plus one cell)
 *   adjoint step     src/sweep/csrc/cuda/equations/acoustic3d/adjoint_split.cu:14-320
 *   reconstruction   src/sweep/csrc/cuda/equations/acoustic3d/forward_split.cu:292-372
 *   step order       src/sweep/csrc/cuda/equations/acoustic3d/driver_traits.cuh:481-590
 *                    (same as 2-D: reconstruct + image, restore, un-inject in
 *                    the strip, strip imaging, re-inject)
 *   strip geometry   src/sweep/csrc/cuda/common/boundary/strip.cuh:125-
 *
 * Fields are (B, nz, ny, nx), x fastest; coordinates (x, y, z).
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
    int pad[6];              /* z_lo, z_hi, y_lo, y_hi, x_lo, x_hi */
    REAL dt, dz, dy, dx;
    const REAL *lap, *gco;
    const REAL *az, *bz, *dbz, *ay, *by, *dby, *ax, *bx, *dbx;
    const REAL* vp; i64 vp_stride;
    int nsrc; const int* src; const REAL* wavelet;
    int nrec; const int* rec;
} A3D;

/* forward / reconstruction Laplacian along one axis: the difference form,
 * order 4 in the summed form (laplace.cuh:68-100, 145-200; see fd_oracle.c) */
static inline REAL lap1(const REAL* u, i64 i, i64 s, int M, const REAL* lc, REAL h)
{
    REAL u0 = u[i], acc = R(0);
    if (M == 2)
        return ((lc[1] * (u[i - s] + u[i + s]) + lc[2] * (u[i - 2 * s] + u[i + 2 * s])) - R(2.5) * u0) / (h * h);
    for (int k = 1; k <= M; ++k) {
        REAL t = lc[k] * ((u[i - k * s] - u0) + (u[i + k * s] - u0));
        acc = (k == 1) ? t : acc + t;
    }
    return acc / (h * h);
}

static inline REAL grad1(const REAL* u, i64 i, i64 s, int M, const REAL* gc, REAL h)
{
    REAL acc = R(0);
    for (int k = 1; k <= M; ++k) {
        REAL t = gc[k] * (u[i + k * s] - u[i - k * s]);
        acc = (k == 1) ? t : acc + t;
    }
    return acc / h;
}

static int in_grid3(const A3D* p, int ix, int iy, int iz)
{
    return ix >= 0 && ix < p->nx && iy >= 0 && iy < p->ny && iz >= 0 && iz < p->nz;
}

/* strip cells of the physical box (width w): z faces (full x-y), y faces over
 * the inner z rows, x faces over the inner z and y rows */
static int strip_cells_3d(const A3D* p, int w, i64* out)
{
    const int M = p->M;
    int z0 = p->pad[0] + M, z1 = p->nz - p->pad[1] - M;
    int y0 = p->pad[2] + M, y1 = p->ny - p->pad[3] - M;
    int x0 = p->pad[4] + M, x1 = p->nx - p->pad[5] - M;
    int lo, hi;
#define WID(ext, L, H) do { int e_ = (ext) > 0 ? (ext) : 0; L = w < e_ ? w : e_; \
        int r_ = e_ - L; H = w < r_ ? w : r_; } while (0)
    int wzl, wzh, wyl, wyh, wxl, wxh;
    WID(z1 - z0, wzl, wzh);
    WID(y1 - y0, wyl, wyh);
    WID(x1 - x0, wxl, wxh);
#undef WID
    (void)lo; (void)hi;
    int n = 0;
    for (int iz = z0; iz < z1; ++iz)
        for (int iy = y0; iy < y1; ++iy)
            for (int ix = x0; ix < x1; ++ix) {
                int zs = iz < z0 + wzl || iz >= z1 - wzh;
                int ys = iy < y0 + wyl || iy >= y1 - wyh;
                int xs = ix < x0 + wxl || ix >= x1 - wxh;
                if (zs || ys || xs) {
                    if (out) out[n] = ((i64)iz * p->ny + iy) * p->nx + ix;
                    ++n;
                }
            }
    return n;
}

long long oracle_a3d_tape_len(int B, int nz, int ny, int nx, int nt, int M, const int* pad)
{
    A3D p; memset(&p, 0, sizeof p);
    p.B = B; p.nz = nz; p.ny = ny; p.nx = nx; p.nt = nt; p.M = M;
    for (int i = 0; i < 6; ++i) p.pad[i] = pad[i];
    int ns = strip_cells_3d(&p, M + 1, NULL);
    return (long long)nt * B * ns + 2LL * B * nz * ny * nx;
}

/* forward step of shot b; psi written to psin, zeta in place */
static void a3d_step(const A3D* p, int b, const REAL* un, const REAL* up, REAL* unx,
                     const REAL* psx, const REAL* psy, const REAL* psz,
                     REAL* psxn, REAL* psyn, REAL* pszn, REAL* zx, REAL* zy, REAL* zz)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL* vp = p->vp + b * p->vp_stride;
    const int px0 = p->pad[4] + M, px1 = nx - p->pad[5] - M;
    const int py0 = p->pad[2] + M, py1 = ny - p->pad[3] - M;
    const int pz0 = p->pad[0] + M, pz1 = nz - p->pad[1] - M;
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz)
        for (int iy = M; iy < ny - M; ++iy)
            for (int ix = M; ix < nx - M; ++ix) {
                i64 i = iz * sz + iy * sy + ix;
                REAL lx = lap1(un, i, 1, M, p->lap, p->dx);
                REAL ly = lap1(un, i, sy, M, p->lap, p->dy);
                REAL lz = lap1(un, i, sz, M, p->lap, p->dz);
                int inx = ix < px0 + 1 || ix >= px1 - 1;
                int iny = iy < py0 + 1 || iy >= py1 - 1;
                int inz = iz < pz0 + 1 || iz >= pz1 - 1;
                REAL w;
                if (!inx && !iny && !inz) {
                    w = (lx + ly) + lz;
                } else {
                    w = R(0);
                    if (inx) {
                        REAL du = grad1(un, i, 1, M, p->gco, p->dx);
                        REAL dps = grad1(psx, i, 1, M, p->gco, p->dx);
                        REAL a = p->ax[ix], bb = p->bx[ix], db = p->dbx[ix];
                        REAL da = grad1(p->ax, ix, 1, M, p->gco, p->dx);
                        REAL tmp = ((((R(1) + bb) * lx + db * du) + a * dps) + da * psx[i]);
                        w = w + ((R(1) + bb) * tmp + a * zx[i]);
                        psxn[i] = bb * du + a * psx[i];
                        zx[i] = bb * tmp + a * zx[i];
                    } else {
                        w = w + lx;
                    }
                    if (iny) {
                        REAL du = grad1(un, i, sy, M, p->gco, p->dy);
                        REAL dps = grad1(psy, i, sy, M, p->gco, p->dy);
                        REAL a = p->ay[iy], bb = p->by[iy], db = p->dby[iy];
                        REAL da = grad1(p->ay, iy, 1, M, p->gco, p->dy);
                        REAL tmp = ((((R(1) + bb) * ly + db * du) + a * dps) + da * psy[i]);
                        w = w + ((R(1) + bb) * tmp + a * zy[i]);
                        psyn[i] = bb * du + a * psy[i];
                        zy[i] = bb * tmp + a * zy[i];
                    } else {
                        w = w + ly;
                    }
                    if (inz) {
                        REAL du = grad1(un, i, sz, M, p->gco, p->dz);
                        REAL dps = grad1(psz, i, sz, M, p->gco, p->dz);
                        REAL a = p->az[iz], bb = p->bz[iz], db = p->dbz[iz];
                        REAL da = grad1(p->az, iz, 1, M, p->gco, p->dz);
                        REAL tmp = ((((R(1) + bb) * lz + db * du) + a * dps) + da * psz[i]);
                        w = w + ((R(1) + bb) * tmp + a * zz[i]);
                        pszn[i] = bb * du + a * psz[i];
                        zz[i] = bb * tmp + a * zz[i];
                    } else {
                        w = w + lz;
                    }
                }
                REAL v = vp[i];
                unx[i] = (R(2) * un[i] - up[i]) + (((v * v) * p->dt) * p->dt) * w;
            }
}

static void inject3(const A3D* p, int b, REAL* u, const REAL* amp, int n, const int* loc, int it, REAL sign)
{
    for (int s = 0; s < n; ++s) {
        const int* c = loc + (b * n + s) * 3;
        if (!in_grid3(p, c[0], c[1], c[2])) continue;
        u[((i64)c[2] * p->ny + c[1]) * p->nx + c[0]] += sign * amp[((i64)b * n + s) * p->nt + it];
    }
}

#define A3D_ARGS \
    int B, int nz, int ny, int nx, int nt, int M, const int* pad, REAL dt, REAL dz, REAL dy, REAL dx, \
    const REAL* lap, const REAL* gco, \
    const REAL* az, const REAL* bz, const REAL* dbz, const REAL* ay, const REAL* by, const REAL* dby, \
    const REAL* ax, const REAL* bx, const REAL* dbx, const REAL* vp, i64 vp_stride, \
    int nsrc, const int* src, const REAL* wavelet, int nrec, const int* rec
#define A3D_INIT(p) \
    A3D p = {B, nz, ny, nx, nt, M, {pad[0], pad[1], pad[2], pad[3], pad[4], pad[5]}, dt, dz, dy, dx, \
             lap, gco, az, bz, dbz, ay, by, dby, ax, bx, dbx, vp, vp_stride, nsrc, src, wavelet, nrec, rec}

int oracle_a3d_forward(A3D_ARGS, REAL* record, REAL* tape)
{
    A3D_INIT(p);
    const i64 n = (i64)nz * ny * nx;
    int ns = strip_cells_3d(&p, M + 1, NULL);
    i64* cells = (i64*)malloc(sizeof(i64) * (ns > 0 ? ns : 1));
    strip_cells_3d(&p, M + 1, cells);
    REAL* buf = (REAL*)malloc(sizeof(REAL) * n * 12);
    if (!buf || !cells) { free(buf); free(cells); return 1; }
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * 12);
        REAL *up = buf, *un = buf + n, *ux = buf + 2 * n;
        REAL *ps[3] = {buf + 3 * n, buf + 4 * n, buf + 5 * n}, *psn[3] = {buf + 6 * n, buf + 7 * n, buf + 8 * n};
        REAL *zx = buf + 9 * n, *zy = buf + 10 * n, *zz = buf + 11 * n;
        for (int it = 0; it < nt; ++it) {
            a3d_step(&p, b, un, up, ux, ps[0], ps[1], ps[2], psn[0], psn[1], psn[2], zx, zy, zz);
            if (tape) {
                REAL* dst = tape + ((i64)it * B + b) * ns;
                for (int c = 0; c < ns; ++c) dst[c] = un[cells[c]];
            }
            inject3(&p, b, ux, wavelet, nsrc, src, it, R(1));
            for (int r = 0; r < nrec; ++r) {
                const int* c = rec + (b * nrec + r) * 3;
                if (!in_grid3(&p, c[0], c[1], c[2])) continue;
                record[((i64)b * nrec + r) * nt + it] = ux[((i64)c[2] * ny + c[1]) * nx + c[0]];
            }
            REAL* t = up; up = un; un = ux; ux = t;
            for (int a = 0; a < 3; ++a) { t = ps[a]; ps[a] = psn[a]; psn[a] = t; }
        }
        if (tape) {
            REAL* last = tape + (i64)nt * B * ns + (i64)b * 2 * n;
            memcpy(last, up, sizeof(REAL) * n);
            memcpy(last + n, un, sizeof(REAL) * n);
        }
    }
    free(buf); free(cells);
    return 0;
}

/* exact adjoint step of shot b (adjoint_split.cu:14-320) */
static void a3d_adjoint(const A3D* p, int b, const REAL* ln, const REAL* lp, REAL* lx_,
                        REAL* const ps[3], REAL* const zt[3], REAL* const pso[3], REAL* const zto[3],
                        REAL* gwb)
{
    const int nz = p->nz, ny = p->ny, nx = p->nx, M = p->M;
    const i64 sy = nx, sz = (i64)nx * ny;
    const REAL* vp = p->vp + b * p->vp_stride;
    const REAL dt2 = p->dt * p->dt;
    const REAL* lc = p->lap;
    const REAL* gc = p->gco;
    const REAL h[3] = {p->dx, p->dy, p->dz};
    const i64 st[3] = {1, sy, sz};
    const REAL* av[3] = {p->ax, p->ay, p->az};
    const REAL* bv[3] = {p->bx, p->by, p->bz};
    const REAL* dbv[3] = {p->dbx, p->dby, p->dbz};
    const int lo[3] = {p->pad[4] + 2 * M + 1, p->pad[2] + 2 * M + 1, p->pad[0] + 2 * M + 1};
    const int hi[3] = {nx - (p->pad[5] + 2 * M + 1), ny - (p->pad[3] + 2 * M + 1), nz - (p->pad[1] + 2 * M + 1)};
    /* gw = ((vp * vp) * dt^2) * lambda once per cell (the taps below read it) */
    #pragma omp parallel for schedule(static)
    for (i64 i = 0; i < (i64)nz * sz; ++i) gwb[i] = ((vp[i] * vp[i]) * dt2) * ln[i];
#define GW(n) (gwb[n])
    #pragma omp parallel for schedule(static)
    for (int iz = M; iz < nz - M; ++iz)
        for (int iy = M; iy < ny - M; ++iy)
            for (int ix = M; ix < nx - M; ++ix) {
                i64 i = iz * sz + iy * sy + ix;
                const int c[3] = {ix, iy, iz};
                REAL gun = ln[i];
                REAL c0c = vp[i]; c0c = (c0c * c0c) * dt2;
                REAL gw = c0c * gun;
                int in[3];
                for (int a = 0; a < 3; ++a) in[a] = c[a] < lo[a] || c[a] >= hi[a];
                if (!in[0] && !in[1] && !in[2]) {
                    REAL L[3];
                    for (int a = 0; a < 3; ++a) {
                        REAL acc = R(0);
                        for (int k = 1; k <= M; ++k)
                            acc = acc + lc[k] * ((GW(i + k * st[a]) - gw) + (GW(i - k * st[a]) - gw));
                        L[a] = acc;
                    }
                    lx_[i] = (((R(2) * gun - lp[i]) + L[0] * (R(1) / (h[0] * h[0]))) +
                              L[1] * (R(1) / (h[1] * h[1]))) + L[2] * (R(1) / (h[2] * h[2]));
                    continue;
                }
                REAL L[3], Dg[3];
                for (int a = 0; a < 3; ++a) {
                    const REAL invh2 = R(1) / (h[a] * h[a]), invh = R(1) / h[a];
                    Dg[a] = R(0);
                    if (in[a]) {
                        const REAL* A = av[a]; const REAL* Bv = bv[a]; const REAL* DB = dbv[a];
                        const REAL* Z = zt[a]; const REAL* PS = ps[a];
                        REAL a_ = A[c[a]], b_ = Bv[c[a]];
                        REAL da = grad1(A, c[a], 1, M, gc, h[a]);
                        REAL gt0 = b_ * Z[i] + (R(1) + b_) * gw;
                        REAL l0 = (R(1) + b_) * gt0;
                        REAL Lq = R(0), Dq = R(0), Dgg = R(0);
                        for (int k = 1; k <= M; ++k) {
                            i64 np = i + k * st[a], nm = i - k * st[a];
                            int cp = c[a] + k, cm = c[a] - k;
                            REAL tp = Bv[cp] * Z[np] + ((R(1) + Bv[cp]) * ((vp[np] * vp[np]) * dt2)) * ln[np];
                            REAL tm = Bv[cm] * Z[nm] + ((R(1) + Bv[cm]) * ((vp[nm] * vp[nm]) * dt2)) * ln[nm];
                            Lq = Lq + lc[k] * ((((R(1) + Bv[cp]) * tp) - l0) + (((R(1) + Bv[cm]) * tm) - l0));
                            Dgg = Dgg + gc[k] * ((Bv[cp] * PS[np] + DB[cp] * tp) - (Bv[cm] * PS[nm] + DB[cm] * tm));
                            Dq = Dq + gc[k] * (A[cp] * tp - A[cm] * tm);
                        }
                        L[a] = Lq * invh2; Dg[a] = Dgg * invh; Dq = Dq * invh;
                        pso[a][i] = (a_ * PS[i] + da * gt0) - Dq;
                        zto[a][i] = a_ * (Z[i] + gw);
                    } else {
                        REAL acc = R(0);
                        for (int k = 1; k <= M; ++k)
                            acc = acc + lc[k] * ((GW(i + k * st[a]) - gw) + (GW(i - k * st[a]) - gw));
                        L[a] = acc * invh2;
                    }
                }
                lx_[i] = (R(2) * gun - lp[i]) + (((((L[0] + L[1]) + L[2]) - Dg[0]) - Dg[1]) - Dg[2]);
            }
#undef GW
}

int oracle_a3d_backward(A3D_ARGS, const REAL* adj, const REAL* tape, REAL* grad_vp, REAL* grad_wavelet,
                        REAL* illum_s, REAL* illum_r)
{
    A3D_INIT(p);
    const i64 n = (i64)nz * ny * nx;
    const i64 sy = nx, sz = (i64)nx * ny;
    int ns = strip_cells_3d(&p, M + 1, NULL);
    i64* cells = (i64*)malloc(sizeof(i64) * (ns > 0 ? ns : 1));
    char* in_strip = (char*)calloc((size_t)n, 1);
    strip_cells_3d(&p, M + 1, cells);
    for (int c = 0; c < ns; ++c) in_strip[cells[c]] = 1;
    REAL* buf = (REAL*)malloc(sizeof(REAL) * n * 20);
    if (!buf || !cells || !in_strip) { free(buf); free(cells); free(in_strip); return 1; }
    int z0 = pad[0] + M, z1 = nz - pad[1] - M, y0 = pad[2] + M, y1 = ny - pad[3] - M;
    int x0 = pad[4] + M, x1 = nx - pad[5] - M;
    const int rz0 = pad[0] + 2 * M + 1, rz1 = nz - (pad[1] + 2 * M + 1);
    const int ry0 = pad[2] + 2 * M + 1, ry1 = ny - (pad[3] + 2 * M + 1);
    const int rx0 = pad[4] + 2 * M + 1, rx1 = nx - (pad[5] + 2 * M + 1);
    const REAL dt2 = dt * dt;
    for (int b = 0; b < B; ++b) {
        memset(buf, 0, sizeof(REAL) * n * 20);
        REAL *lp = buf, *ln = buf + n, *lx = buf + 2 * n;
        REAL* aps[2][3] = {{buf + 3 * n, buf + 4 * n, buf + 5 * n}, {buf + 6 * n, buf + 7 * n, buf + 8 * n}};
        REAL* azt[2][3] = {{buf + 9 * n, buf + 10 * n, buf + 11 * n}, {buf + 12 * n, buf + 13 * n, buf + 14 * n}};
        REAL *rp = buf + 15 * n, *rn = buf + 16 * n, *rx = buf + 17 * n;
        REAL* g = buf + 18 * n;
        REAL* gwb = buf + 19 * n;
        const REAL* vpb = vp + b * vp_stride;
        int cur = 0;
        const REAL* last = tape + (i64)nt * B * ns + (i64)b * 2 * n;
        memcpy(rp, last + n, sizeof(REAL) * n);
        memcpy(rn, last, sizeof(REAL) * n);
        for (int it = nt - 1; it >= 0; --it) {
            a3d_adjoint(&p, b, ln, lp, lx, aps[cur], azt[cur], aps[1 - cur], azt[1 - cur], gwb);
            inject3(&p, b, lx, adj, nrec, rec, it, R(1));
            { REAL* t = lp; lp = ln; ln = lx; lx = t; }
            cur = 1 - cur;
            if (grad_wavelet) {
                for (int s = 0; s < nsrc; ++s) {
                    const int* c = src + (b * nsrc + s) * 3;
                    if (!in_grid3(&p, c[0], c[1], c[2])) continue;
                    grad_wavelet[((i64)b * nsrc + s) * nt + it] += ln[((i64)c[2] * ny + c[1]) * nx + c[0]];
                }
            }
            if (it == 0) {
                /* receiver illumination of the it == 0 tail
                   (acoustic3d/driver_traits.cuh:467-478) */
                if (illum_r)
                    for (int iz = z0; iz < z1; ++iz)
                        for (int iy = y0; iy < y1; ++iy)
                            for (int ix = x0; ix < x1; ++ix) {
                                const i64 i = iz * sz + iy * sy + ix;
                                illum_r[i] += ln[i] * ln[i];
                            }
                break;
            }
            #pragma omp parallel for schedule(static)
            for (int iz = rz0; iz < rz1; ++iz)
                for (int iy = ry0; iy < ry1; ++iy)
                    for (int ix = rx0; ix < rx1; ++ix) {
                        i64 i = iz * sz + iy * sy + ix;
                        REAL w = (lap1(rn, i, 1, M, lap, dx) + lap1(rn, i, sy, M, lap, dy)) + lap1(rn, i, sz, M, lap, dz);
                        REAL v = vpb[i], u0 = rn[i], up = rp[i];
                        REAL un = (R(2) * u0 - up) + (((v * v) * dt) * dt) * w;
                        rx[i] = un;
                        REAL utt = ((un - R(2) * u0) + up) / dt2;
                        g[i] = g[i] + ((((R(2) * dt) * dt) * utt) * ln[i]) / v;
                    }
            const REAL* saved = tape + ((i64)(it - 1) * B + b) * ns;
            for (int c = 0; c < ns; ++c) rx[cells[c]] = saved[c];
            for (int s = 0; s < nsrc; ++s) {
                const int* c = src + (b * nsrc + s) * 3;
                if (!in_grid3(&p, c[0], c[1], c[2])) continue;
                i64 i = ((i64)c[2] * ny + c[1]) * nx + c[0];
                if (in_strip[i]) rx[i] -= wavelet[((i64)b * nsrc + s) * nt + it];
            }
            for (int c = 0; c < ns; ++c) {
                i64 i = cells[c];
                REAL utt = ((rx[i] - R(2) * rn[i]) + rp[i]) / dt2;
                g[i] = g[i] + ((((R(2) * dt) * dt) * utt) * ln[i]) / vpb[i];
            }
            /* illumination on the physical box after the strip imaging, before
               the source injection (acoustic3d/driver_traits.cuh:556-575,
               kernels.cu:150-200), summed over shots */
            if (illum_s)
                for (int iz = z0; iz < z1; ++iz)
                    for (int iy = y0; iy < y1; ++iy)
                        for (int ix = x0; ix < x1; ++ix) {
                            const i64 i = iz * sz + iy * sy + ix;
                            illum_r[i] += ln[i] * ln[i];
                            const REAL utt = ((rx[i] - R(2) * rn[i]) + rp[i]) / dt2;
                            illum_s[i] += utt * utt;
                        }
            inject3(&p, b, rx, wavelet, nsrc, src, it, R(1));
            { REAL* t = rp; rp = rn; rn = rx; rx = t; }
        }
        REAL* gout = grad_vp + b * vp_stride;
        for (i64 i = 0; i < n; ++i) gout[i] += g[i];
    }
    free(buf); free(cells); free(in_strip);
    return 0;
}
