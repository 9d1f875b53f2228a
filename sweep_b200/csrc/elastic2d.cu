// elastic2d.cu -- 2-D isotropic elastic (velocity-stress, staggered grid)
// forward and boundary-saving adjoint for sm_100a.
//
// Restates the reference's elastic2d path (src/sweep/csrc/cuda/equations/
// elastic2d/, common/sg_driver.cuh) with a different kernel structure:
//
//   forward, per step (reference: velocity kernel, stress kernel, add_source
//   per field, 5 boundary saves, record per field = 2 + 2 + 5 + 2 launches):
//     fwd_vel   velocity update with its 4 CPML memories   kernels.cuh:48-138
//     fwd_str   stress update with its 4 CPML memories     kernels.cuh:182-311
//               + source injection, the 5-field boundary-strip save and the
//               receiver gather of the same step, done by the CTA that owns
//               the cell                                   sg_driver.cuh:291-340
//   reverse, per step (reference: 8-13 launches, sg_driver.cuh:786-806):
//     rev_str   stress reconstruction (NOPML) + strip restore, the residual
//               injection, the vp/vs/rho imaging and the receiver rho fix,
//               sharing the velocity derivatives between reconstruction and
//               imaging                                    kernels.cuh:455-535,
//                                                          601-663; common.cu:77-117
//     rev_sadj  stress-adjoint apply; the four q fields (stress-adjoint
//               prepare, kernels.cuh:548-750) are built in shared memory for
//               the tile and its halo instead of a global round trip
//     rev_vadj  velocity-adjoint apply with p built the same way
//               (kernels.cuh:873-1019) + carrier capture, velocity
//               reconstruction (NOPML) and strip restore  kernels.cuh:365-450,
//                                                          driver_traits.cuh:758-826
//
// Building q / p in shared memory lets every CTA recompute them for its halo,
// so the adjoint CPML memories are double-buffered (read the old set, write
// the new one) and neighbouring CTAs never race on them.
//
// Layout: fields are pitched (B, nz, P), P = nx rounded up to 32 floats.
// CPML memories live in per-axis slabs (x: (B, nz, WX), z: (B, WZ, P)) that
// cover the PML band plus one cell (the half-cell profile reaches one cell
// further inward on the high side; reference context.h:359-400 keeps wider
// slabs for the same reason).  Tiles are 32 x 32 cells, 256 threads, 4 rows
// per thread.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <vector>

#include "common.cuh"
#include "elastic2d.cuh"
#include "tma.cuh"

namespace sweep {
namespace el2d {

constexpr int M = 4;
constexpr int TX = 32, TZ = 32, NTH = 256, RPT = TZ / 8;
constexpr int HX = TX + 2 * M, HZ = TZ + 2 * M, HN = HX * HZ;

// Staggered first-derivative weights of order 8 (reference
// operators/staggered.cuh:351-354; scalars.py:25-49).
#define C1 (1225.f / 1024.f)
#define C2 (-245.f / 3072.f)
#define C3 (49.f / 5120.f)
#define C4 (-5.f / 7168.f)

enum { VX = 0, VZ = 1, SXX = 2, SZZ = 3, SXZ = 4 };

// Boundary-strip storage of the boundary-saving tape.  fp32 and bf16 keep the
// strip set (B, 5, nstrip); fp16 and int8 keep the reference's four bands per
// field (top and bottom: M + 1 rows from M outside the box over its width;
// left and right: M + 1 columns down the box), each quantised per field and
// shot in blocks of kQB cells against the block's max |value| (reference
// boundarysaver.cu:906-1100, elastic2d/driver_traits.cuh:270-291).
enum StripFmt { SF_F32 = 0, SF_F16 = 1, SF_BF16 = 2, SF_I8 = 3 };
constexpr int kQB = 256;

struct StripStore {
    int fmt;                        // StripFmt
    int cells[4], blocks[4];        // per field and shot, per band (top, bottom, left, right)
    long long pay[4], scl[4];       // byte offsets of each band's codes (5, B, cells) and scales (5, B, blocks)
    long long step;                 // bytes of one step slot
};

struct Geo {
    int B, nz, nx, nt, P;
    long long S;                    // pitched cells per shot
    int z0, z1, x0, x1;             // physical box
    int XL, XH, ZL, ZH;             // CPML band (pad + M) per face
    int SXL, SXH, SZL, SZH;         // slab side widths (band + 1)
    int WX, WZ;                     // slab widths
    int ntx, ntz;
    int bw, bh, nstrip;             // strip geometry
    float dt, idx, idz;
    const float *az, *bz, *azh, *bzh, *ax, *bx, *axh, *bxh;
    int nsrc, nrec, nsf, nrf;
    int sf[5], rf[5];               // stress source fields (nsf), receiver fields (nrf)
    int nvf, vf[2];                 // velocity (body-force) source fields
    const int *src_loc, *rec_loc;   // (B, nsrc, 2), (B, nrec, 2) runtime (x, z)
    long long ms;                   // model stride between shots (0 or S)
    EventTable src, rec;
    const float* wavelet;           // (B, nsrc, nt)
    int gf;                         // shots per CTA of the forward kernels
    int* err;                       // bounded-wait failure flag (0 = none)
    StripStore st;
    int fs;                         // bit f: traction-free face f (z_lo, z_hi, x_lo, x_hi), pad 0
};

enum { ERR_WAIT_FWD = 1, ERR_WAIT_REV = 2 };
constexpr int CN = TX * TZ;         // floats of a centre tile

// Models on the pitched grid, one copy (shared) or B copies (per shot).
struct Models {
    const float *rho, *lam, *mu, *bv, *vp, *vs;   // bv = dt * (1 / rho)
};

// Memory-variable slabs of one wavefield set: x slab m_x[k] (B, nz, WX) and
// z slab m_z[k] (B, WZ, P).
struct Slabs {
    float* x[4];
    float* z[4];
};

__device__ __forceinline__ int xslab(const Geo& G, int ix)
{
    return ix < G.SXL ? ix : (ix >= G.nx - G.SXH ? G.SXL + ix - (G.nx - G.SXH) : -1);
}
__device__ __forceinline__ int zslab(const Geo& G, int iz)
{
    return iz < G.SZL ? iz : (iz >= G.nz - G.SZH ? G.SZL + iz - (G.nz - G.SZH) : -1);
}
__device__ __forceinline__ bool in_pml(const Geo& G, int ix, int iz)
{
    return ix < G.XL || ix >= G.nx - G.XH || iz < G.ZL || iz >= G.nz - G.ZH;
}
__device__ __forceinline__ bool in_core(const Geo& G, int ix, int iz)
{
    return ix >= M && ix < G.nx - M && iz >= M && iz < G.nz - M;
}
// Reverse (NOPML) reconstruction region: the box minus one cell per face
// (reference kernels.cuh:430-440, band abcn + M + 1).
__device__ __forceinline__ bool in_recon(const Geo& G, int ix, int iz)
{
    return ix > G.x0 && ix < G.x1 - 1 && iz > G.z0 && iz < G.z1 - 1;
}
__device__ __forceinline__ bool in_box(const Geo& G, int ix, int iz)
{
    return ix >= G.x0 && ix < G.x1 && iz >= G.z0 && iz < G.z1;
}

// Index of (iz, ix) in the boundary-strip set, or -1.  The set is the union
// of the reference's four bands, width M + 1 at offset -M around the physical
// box (reference boundary/strip.cuh:81-114): M rows above and below the box
// over its width, the box's first and last rows over the box width plus M
// cells each side, and the M + 1 cells each side of the inner box rows.  Every
// cell is stored once.
__device__ __forceinline__ int strip_index(const Geo& G, int iz, int ix)
{
    constexpr int W = M + 1;
    if (iz >= G.z0 - M && iz < G.z0) {
        return (ix >= G.x0 && ix < G.x1) ? (iz - (G.z0 - M)) * G.bw + ix - G.x0 : -1;
    }
    if (iz >= G.z1 && iz < G.z1 + M) {
        return (ix >= G.x0 && ix < G.x1) ? (M + iz - G.z1) * G.bw + ix - G.x0 : -1;
    }
    if (iz < G.z0 || iz >= G.z1 || ix < G.x0 - M || ix >= G.x1 + M) return -1;
    const int row = G.bw + 2 * M, base = 2 * M * G.bw;
    if (iz == G.z0) return base + ix - (G.x0 - M);
    if (iz == G.z1 - 1) return base + row + ix - (G.x0 - M);
    const int r = base + 2 * row + (iz - G.z0 - 1) * 2 * W;
    if (ix <= G.x0) return r + ix - (G.x0 - M);
    if (ix >= G.x1 - 1) return r + W + ix - (G.x1 - 1);
    return -1;
}

// Band f (0 top, 1 bottom, 2 left, 3 right; width M + 1 at offset -M) cell
// `idx` of the scaled formats -> grid cell.
__device__ __forceinline__ void band_cell(const Geo& G, int f, int idx, int& iz, int& ix)
{
    constexpr int W = M + 1;
    if (f < 2) {
        const int r = idx / G.bw;
        iz = (f == 0 ? G.z0 - M : G.z1 - 1) + r;
        ix = G.x0 + (idx - r * G.bw);
    } else {
        const int r = idx / W;
        iz = G.z0 + r;
        ix = (f == 2 ? G.x0 - M : G.x1 - 1) + (idx - r * W);
    }
}

// The band a scaled-format restore reads strip cell (iz, ix) from: the last
// of the bands holding it in the reference's restore order top, bottom,
// left, right.
__device__ __forceinline__ int band_index(const Geo& G, int iz, int ix, int& f)
{
    constexpr int W = M + 1;
    const bool rows = iz >= G.z0 && iz < G.z1;
    if (rows && ix >= G.x1 - 1) { f = 3; return (iz - G.z0) * W + (ix - (G.x1 - 1)); }
    if (rows && ix <= G.x0) { f = 2; return (iz - G.z0) * W + (ix - (G.x0 - M)); }
    if (iz >= G.z1 - 1) { f = 1; return (iz - (G.z1 - 1)) * G.bw + (ix - G.x0); }
    f = 0;
    return (iz - (G.z0 - M)) * G.bw + (ix - G.x0);
}

// Saved value of field k at strip cell (iz, ix) (strip index si) of shot b
// (dequantised as the reference does: fp16 code x scale; int8
// (code - 128) x scale / 127).
__device__ __forceinline__ float strip_val(const Geo& G, const void* slot, int b, int k, int iz, int ix, int si)
{
    const StripStore& S = G.st;
    const long long e = ((long long)b * 5 + k) * G.nstrip + si;
    if (S.fmt == SF_F32) return static_cast<const float*>(slot)[e];
    if (S.fmt == SF_BF16) return __bfloat162float(static_cast<const __nv_bfloat16*>(slot)[e]);
    int f;
    const int i = band_index(G, iz, ix, f);
    const char* base = static_cast<const char*>(slot);
    const long long row = (long long)k * G.B + b;
    const float scale = reinterpret_cast<const float*>(base + S.scl[f])[row * S.blocks[f] + i / kQB];
    const long long q = row * S.cells[f] + i;
    if (S.fmt == SF_F16) return __half2float(reinterpret_cast<const __half*>(base + S.pay[f])[q]) * scale;
    return ((float)reinterpret_cast<const uint8_t*>(base + S.pay[f])[q] - 128.0f) * (scale * (1.0f / 127.0f));
}

// Does tile (tz0, tx0) hold any strip cell?  The strips lie within M cells
// of the physical box's edges; a tile strictly inside the reconstruction
// region or strictly outside the box plus M has none.
__device__ __forceinline__ bool tile_has_strips(const Geo& G, int tz0, int tx0)
{
    const bool outside = tx0 + TX <= G.x0 - M || tx0 >= G.x1 + M || tz0 + TZ <= G.z0 - M || tz0 >= G.z1 + M;
    const bool inside = tx0 > G.x0 && tx0 + TX < G.x1 - 1 && tz0 > G.z0 && tz0 + TZ < G.z1 - 1;
    return !outside && !inside;
}

// ---------------------------------------------------------------- stencils
// D+ / D- on a shared tile (pitch HX) at flat index c (reference
// operators/staggered.cuh:356-430, same term order).
__device__ __forceinline__ float dpx(const float* t, int c, float inv)
{
    return (C1 * (t[c + 1] - t[c]) + C2 * (t[c + 2] - t[c - 1]) + C3 * (t[c + 3] - t[c - 2]) +
            C4 * (t[c + 4] - t[c - 3])) * inv;
}
__device__ __forceinline__ float dmx(const float* t, int c, float inv)
{
    return (C1 * (t[c] - t[c - 1]) + C2 * (t[c + 1] - t[c - 2]) + C3 * (t[c + 2] - t[c - 3]) +
            C4 * (t[c + 3] - t[c - 4])) * inv;
}
__device__ __forceinline__ float dpz(const float* t, int c, float inv)
{
    return (C1 * (t[c + HX] - t[c]) + C2 * (t[c + 2 * HX] - t[c - HX]) +
            C3 * (t[c + 3 * HX] - t[c - 2 * HX]) + C4 * (t[c + 4 * HX] - t[c - 3 * HX])) * inv;
}
__device__ __forceinline__ float dmz(const float* t, int c, float inv)
{
    return (C1 * (t[c] - t[c - HX]) + C2 * (t[c + HX] - t[c - 2 * HX]) +
            C3 * (t[c + 2 * HX] - t[c - 3 * HX]) + C4 * (t[c + 3 * HX] - t[c - 4 * HX])) * inv;
}

// ------------------------------------------------------ traction-free faces
// Image method of the reference (common/elastic_free_surface.cuh:200-720,
// elastic2d/kernels.cuh:216-303, 592-700).  Bit f of G.fs (z_lo, z_hi, x_lo,
// x_hi) makes face f free; a free face has no PML pad, its surface is the
// first / last physical row or column and the M halo cells past it are air.
// Along an axis with a free face the M cells from the surface inwards take a
// unit-weight 2nd-order difference, and a difference that reaches into the
// air reads the image of the cell mirrored about the surface (about the node
// for fields on integer nodes, about the half cell next to it for fields half
// a cell along the axis; on the high side a half field's surface node is
// itself air), negated for odd fields.  Below the band every stencil stays in
// the medium: the D+ forms are only applied to integer fields and the D-
// forms to half fields.  After the stress update a surface row's sxx (a
// surface column's szz) takes the Robertsson correction, its szz (sxx) is
// zeroed, and a high-side face zeroes sxz on its surface row / column.
struct FsAx {
    bool lo_on, hi_on;
    int lo, hi;              // surface cells
};
__device__ __forceinline__ FsAx fs_zax(const Geo& G) { return {(G.fs & 1) != 0, (G.fs & 2) != 0, G.z0, G.z1 - 1}; }
__device__ __forceinline__ FsAx fs_xax(const Geo& G) { return {(G.fs & 4) != 0, (G.fs & 8) != 0, G.x0, G.x1 - 1}; }

__device__ __forceinline__ bool fs_band(const FsAx& a, int j)
{
    return (a.lo_on && j >= a.lo && j < a.lo + M) || (a.hi_on && j > a.hi - M && j <= a.hi);
}
__device__ __forceinline__ bool fs_air(const FsAx& a, int j)
{
    return (a.lo_on && j < a.lo) || (a.hi_on && j > a.hi);
}
// a cell whose adjoint stencil reaches a band or an image
__device__ __forceinline__ bool fs_near(const FsAx& a, int j)
{
    return (a.lo_on && j < a.lo + 2 * M) || (a.hi_on && j > a.hi - 2 * M);
}
__device__ __forceinline__ bool fs_zrow(const Geo& G, int iz)
{
    return ((G.fs & 1) && iz == G.z0) || ((G.fs & 2) && iz == G.z1 - 1);
}
__device__ __forceinline__ bool fs_xcol(const Geo& G, int ix)
{
    return ((G.fs & 4) && ix == G.x0) || ((G.fs & 8) && ix == G.x1 - 1);
}
__device__ __forceinline__ bool fs_zero_shear(const Geo& G, int ix, int iz)
{
    return ((G.fs & 2) && iz == G.z1 - 1) || ((G.fs & 8) && ix == G.x1 - 1);
}
// does the tile hold a surface row or column?
__device__ __forceinline__ bool fs_tile(const Geo& G, int tz0, int tx0)
{
    auto in = [](int j, int t0, int w) { return j >= t0 && j < t0 + w; };
    return ((G.fs & 1) && in(G.z0, tz0, TZ)) || ((G.fs & 2) && in(G.z1 - 1, tz0, TZ)) ||
           ((G.fs & 4) && in(G.x0, tx0, TX)) || ((G.fs & 8) && in(G.x1 - 1, tx0, TX));
}

// Value at index j along the axis (stride S in the tile) of the line through
// tile cell c, which sits at index j0, with the images of the free faces.
template <int S>
__device__ __forceinline__ float fs_val(const FsAx& a, const float* t, int c, int j0, int j, bool odd, bool half)
{
    int m;
    if (a.lo_on && j < a.lo) m = half ? 2 * a.lo - 1 - j : 2 * a.lo - j;
    else if (a.hi_on && j >= (half ? a.hi : a.hi + 1)) m = half ? 2 * a.hi - 1 - j : 2 * a.hi - j;
    else return t[c + (j - j0) * S];
    const float v = t[c + (m - j0) * S];
    return odd ? -v : v;
}

template <int S, bool FWD>
__device__ __forceinline__ float d_plain(const float* t, int c, float inv)
{
    if constexpr (S == 1) return FWD ? dpx(t, c, inv) : dmx(t, c, inv);
    else return FWD ? dpz(t, c, inv) : dmz(t, c, inv);
}

// Forward derivative along an axis: D+ (FWD) or D-, at tile cell c, index j.
template <bool FS, int S, bool FWD>
__device__ __forceinline__ float d_fs(const FsAx& a, const float* t, int c, int j, bool odd, bool half, float inv)
{
    if (!FS || !fs_band(a, j)) return d_plain<S, FWD>(t, c, inv);
    return (FWD ? fs_val<S>(a, t, c, j, j + 1, odd, half) - fs_val<S>(a, t, c, j, j, odd, half)
                : fs_val<S>(a, t, c, j, j, odd, half) - fs_val<S>(a, t, c, j, j - 1, odd, half)) * inv;
}

// Transposed reduced stencil at index m, read from the tile line through
// cell c (index j0): output cells in a band contribute with weight 1, the
// others with the full weight; air cells hold no adjoint (sources and
// receivers beyond a free surface are off the grid).  Every cell it reads
// lies within M of j0; the range test only guards the tile.
template <int S, bool FWD>
__device__ __forceinline__ float adj_red(const FsAx& a, const float* q, int c, int j0, int m, int n)
{
    auto live = [&](int j) { return j >= 0 && j < n && !fs_band(a, j) && !fs_air(a, j) && j - j0 >= -M && j - j0 <= M; };
    auto at = [&](int j) { return (j - j0 >= -M && j - j0 <= M) ? q[c + (j - j0) * S] : 0.f; };
    const float w[M] = {C1, C2, C3, C4};
    float acc = 0.f;
#pragma unroll
    for (int k = 1; k <= M; ++k) {
        const int jp = FWD ? m + k - 1 : m + k;
        const int jm = FWD ? m - k : m - k + 1;
        if (live(jp)) acc += w[k - 1] * at(jp);
        if (live(jm)) acc -= w[k - 1] * at(jm);
    }
    if (FWD) {
        if (fs_band(a, m)) acc += at(m);
        if (fs_band(a, m - 1)) acc -= at(m - 1);
    } else {
        if (fs_band(a, m + 1)) acc += at(m + 1);
        if (fs_band(a, m)) acc -= at(m);
    }
    return acc;
}

// Adjoint of d_fs (negated transpose; the plain one is D- for a D+ forward
// and D+ for a D- forward): the reduced transpose plus, for each free face
// whose image of this cell lies in the air, the transpose there folded back
// with the field's parity.
template <bool FS, int S, bool FWD>
__device__ __forceinline__ float adj_fs(const FsAx& a, const float* q, int c, int j, int n, bool odd, bool half,
                                        float inv)
{
    if (!FS || !fs_near(a, j)) return d_plain<S, !FWD>(q, c, inv);
    if (fs_air(a, j)) return 0.f;
    float g = adj_red<S, FWD>(a, q, c, j, j, n);
    const float par = odd ? -1.f : 1.f;
    if (a.lo_on) {
        const int mj = half ? 2 * a.lo - 1 - j : 2 * a.lo - j;
        if (mj < a.lo) g += par * adj_red<S, FWD>(a, q, c, j, mj, n);
    }
    if (a.hi_on) {
        const int mj = half ? 2 * a.hi - 1 - j : 2 * a.hi - j;
        if (mj >= (half ? a.hi : a.hi + 1)) g += par * adj_red<S, FWD>(a, q, c, j, mj, n);
    }
    return g * inv;
}

// Cooperative load of NF fields' tiles plus an M-cell halo (zero outside the
// grid) into shared memory: every thread issues all its global loads before
// its first shared store, so the loads of a CTA are in flight together.
constexpr int NLD = (HN + NTH - 1) / NTH;   // loads per thread per field

template <int NF>
__device__ __forceinline__ void load_tiles(float* const (&t)[NF], const float* const (&g)[NF], const Geo& G,
                                           int tz0, int tx0)
{
    const int tid = threadIdx.x + threadIdx.y * TX;
    float v[NF][NLD];
    long long off[NLD];
    bool ok[NLD];
#pragma unroll
    for (int j = 0; j < NLD; ++j) {
        const int k = tid + j * NTH;
        const int lz = k / HX, lx = k - lz * HX;
        const int iz = tz0 - M + lz, ix = tx0 - M + lx;
        ok[j] = k < HN && (unsigned)iz < (unsigned)G.nz && (unsigned)ix < (unsigned)G.nx;
        off[j] = (long long)iz * G.P + ix;
    }
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < NLD; ++j) v[f][j] = ok[j] ? __ldg(g[f] + off[j]) : 0.f;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < NLD; ++j) {
            const int k = tid + j * NTH;
            if (k < HN) t[f][k] = v[f][j];
        }
}

// Add w to the stress field `fld` (one of SXX, SZZ, SXZ) held in registers.
__device__ __forceinline__ void add_to(int fld, float w, float& sxx, float& szz, float& sxz)
{
    if (fld == SXX) sxx += w;
    else if (fld == SZZ) szz += w;
    else sxz += w;
}

__device__ __forceinline__ void tile_origin(const Geo& G, int tile, int& tz0, int& tx0)
{
    tz0 = (tile / G.ntx) * TZ;
    tx0 = (tile % G.ntx) * TX;
}

// ------------------------------------------------------------------ forward
struct FwdArgs {
    Geo G;
    Models m;
    float* f[5];          // vx, vz, sxx, szz, sxz
    Slabs mem;            // forward memories: x {vxx, vzx, sxxx, sxzx}, z {vzz, vxz, szzz, sxzz}
    void* strips;         // this step's strips (B, 5, nstrip): float, or bf16 when G.st.fmt is bf16; or null
    float* record;        // (B, nt, nrec, nrf)
    int it;
};
// memory slot names
enum { XM_VXX = 0, XM_VZX = 1, XM_SXXX = 2, XM_SXZX = 3 };
enum { ZM_VZZ = 0, ZM_VXZ = 1, ZM_SZZZ = 2, ZM_SXZZ = 3 };

// Does tile (tz0, tx0) reach the CPML band (pad + M per face)?
__device__ __forceinline__ bool tile_in_pml(const Geo& G, int tz0, int tx0)
{
    return tx0 < G.XL || tx0 + TX > G.nx - G.XH || tz0 < G.ZL || tz0 + TZ > G.nz - G.ZH;
}

// Two CPML memories of one axis at one cell: their slab offset (-1: the cell
// has no memory on that axis) and old values.
struct MemPair {
    long long at;
    float a, b;
};

__device__ __forceinline__ MemPair load_mem_z(const Geo& G, const Slabs& m, int k0, int k1, int b, int iz, int ix,
                                              bool surf = false)
{
    MemPair p{-1, 0.f, 0.f};
    if (iz >= G.nz || ix >= G.nx || !(surf || in_pml(G, ix, iz))) return p;
    const int zs = zslab(G, iz);
    if (zs < 0) return p;
    p.at = ((long long)b * G.WZ + zs) * G.P + ix;
    p.a = m.z[k0][p.at];
    p.b = m.z[k1][p.at];
    return p;
}

__device__ __forceinline__ MemPair load_mem_x(const Geo& G, const Slabs& m, int k0, int k1, int b, int iz, int ix,
                                              bool surf = false)
{
    MemPair p{-1, 0.f, 0.f};
    if (iz >= G.nz || ix >= G.nx || !(surf || in_pml(G, ix, iz))) return p;
    const int xs = xslab(G, ix);
    if (xs < 0) return p;
    p.at = ((long long)b * G.nz + iz) * G.WX + xs;
    p.a = m.x[k0][p.at];
    p.b = m.x[k1][p.at];
    return p;
}

// TMA tensor maps of the five wavefields: (HX x HZ) boxes for the stencil
// inputs with their halo, (TX x TZ) boxes for the centre tiles.
struct FwdMaps {
    CUtensorMap halo[5];
    CUtensorMap tile[5];
};

// Shared memory of the forward kernels: two pipeline stages, each holding
// one shot's halo'd stencil inputs and centre tiles.
template <int NH, int NC>
struct StageSmem {
    float h[2][NH][HN];
    float c[2][NC][CN];
    uint64_t bar[2];
    int bad[2];      // a thread's wait for shot g failed: bad[g & 1] (read after the shot's barrier)
};
using VelSmem = StageSmem<3, 2>;   // sxx, szz, sxz halos; vx, vz centres
using StrSmem = StageSmem<2, 3>;   // vx, vz halos; sxx, szz, sxz centres

// One CTA = one tile for G shots.  Thread 0 issues each shot's TMA loads into
// a 2-stage mbarrier pipeline, so shot g+1's tiles are in flight while shot g
// computes; every wait is bounded and sets the call's error flag.
template <int NH, int NC, class Issue>
__device__ __forceinline__ void pipeline_start(StageSmem<NH, NC>& sm, int nloc, int b0, Issue issue)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        tma::mbar_init(&sm.bar[0], 1);
        tma::mbar_init(&sm.bar[1], 1);
        tma::fence_barrier_init();
        sm.bad[0] = sm.bad[1] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        issue(0, b0);
        if (nloc > 1) issue(1, b0 + 1);
    }
}

// After a failed wait on shot g's stage: wait (bounded) for the copies this
// CTA still has in flight -- shot g's and, if issued, shot g+1's -- then exit.
template <int NH, int NC>
__device__ __forceinline__ void drain(StageSmem<NH, NC>& sm, int g, int nloc, int* err, int code)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        tma::mbar_wait(&sm.bar[g & 1], (g >> 1) & 1, err, code);
        if (g + 1 < nloc) tma::mbar_wait(&sm.bar[(g + 1) & 1], ((g + 1) >> 1) & 1, err, code);
    }
}

// Velocity step (reference kernels.cuh:48-138).
template <bool FS>
__global__ void __launch_bounds__(NTH, 4) fwd_vel(const __grid_constant__ FwdMaps MP, FwdArgs A)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    VelSmem& sm = *reinterpret_cast<VelSmem*>(smem_raw);
    const Geo& G = A.G;
    int tz0, tx0;
    tile_origin(G, blockIdx.x, tz0, tx0);
    const int b0 = blockIdx.y * G.gf, nloc = min(G.gf, G.B - b0);
    constexpr uint32_t kBytes = (3 * HN + 2 * CN) * 4;
    auto issue = [&](int s, int b) {
        tma::mbar_expect_tx(&sm.bar[s], kBytes);
        for (int f = 0; f < 3; ++f) tma::load_3d(sm.h[s][f], &MP.halo[SXX + f], &sm.bar[s], tx0 - M, tz0 - M, b);
        for (int f = 0; f < 2; ++f) tma::load_3d(sm.c[s][f], &MP.tile[VX + f], &sm.bar[s], tx0, tz0, b);
    };
    pipeline_start(sm, nloc, b0, issue);
    const int lx = threadIdx.x, ix = tx0 + lx;
    // dt / rho of this thread's cells (a shared model: once for every shot)
    float bvr[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int iz = tz0 + threadIdx.y + 8 * r;
        bvr[r] = in_core(G, ix, iz) ? A.m.bv[(long long)b0 * G.ms + (long long)iz * G.P + ix] : 0.f;
    }
    const bool ring = tile_in_pml(G, tz0, tx0);
    bool bad = false;
    for (int g = 0; g < nloc; ++g) {
        const int b = b0 + g, s = g & 1;
        // the CPML memories of this thread's cells, loaded while the tiles arrive
        MemPair mz[RPT], mx[RPT];
        if (ring) {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int iz = tz0 + threadIdx.y + 8 * r;
                mz[r] = load_mem_z(G, A.mem, ZM_SZZZ, ZM_SXZZ, b, iz, ix);
                mx[r] = load_mem_x(G, A.mem, XM_SXZX, XM_SXXX, b, iz, ix);
            }
        }
        // each thread waits for the stage itself; a failed wait leaves at the
        // barrier that ends the shot (after drain)
        if (!tma::mbar_wait(&sm.bar[s], (g >> 1) & 1, G.err, ERR_WAIT_FWD)) bad = true;
        const float *tsxx = sm.h[s][0], *tszz = sm.h[s][1], *tsxz = sm.h[s][2];
        const long long so = (long long)b * G.S;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int lz = threadIdx.y + 8 * r, iz = tz0 + lz;
            if (!in_core(G, ix, iz)) continue;
            const int c = (lz + M) * HX + lx + M;
            const FsAx az = fs_zax(G), ax = fs_xax(G);
            float dsxx_dx = d_fs<FS, 1, true>(ax, tsxx, c, ix, true, false, G.idx);
            float dsxz_dz = d_fs<FS, HX, false>(az, tsxz, c, iz, true, true, G.idz);
            float dsxz_dx = d_fs<FS, 1, false>(ax, tsxz, c, ix, true, true, G.idx);
            float dszz_dz = d_fs<FS, HX, true>(az, tszz, c, iz, true, false, G.idz);
            const long long i = (long long)iz * G.P + ix;
            if (ring && in_pml(G, ix, iz)) {
                if (mz[r].at >= 0) {
                    float m0 = G.azh[iz] * mz[r].a + G.bzh[iz] * dszz_dz;
                    dszz_dz += m0;
                    float m1 = G.az[iz] * mz[r].b + G.bz[iz] * dsxz_dz;
                    dsxz_dz += m1;
                    A.mem.z[ZM_SZZZ][mz[r].at] = m0;
                    A.mem.z[ZM_SXZZ][mz[r].at] = m1;
                }
                if (mx[r].at >= 0) {
                    float m0 = G.ax[ix] * mx[r].a + G.bx[ix] * dsxz_dx;
                    dsxz_dx += m0;
                    float m1 = G.axh[ix] * mx[r].b + G.bxh[ix] * dsxx_dx;
                    dsxx_dx += m1;
                    A.mem.x[XM_SXZX][mx[r].at] = m0;
                    A.mem.x[XM_SXXX][mx[r].at] = m1;
                }
            }
            const int cc = lz * TX + lx;
            A.f[VX][so + i] = sm.c[s][0][cc] + bvr[r] * (dsxx_dx + dsxz_dz);
            A.f[VZ][so + i] = sm.c[s][1][cc] + bvr[r] * (dsxz_dx + dszz_dz);
        }
        if (__syncthreads_or(bad)) {           // every thread is done with stage s
            drain(sm, g, nloc, G.err, ERR_WAIT_FWD);
            return;
        }
        if (threadIdx.x == 0 && threadIdx.y == 0 && g + 2 < nloc) issue(s, b + 2);
    }
}

// Stress step (reference kernels.cuh:182-311, with the free top face), then the
// step's point work for the cells this CTA owns: source injection into the
// stress source fields, the 5-field strip save and the receiver gather
// (reference sg_driver.cuh:300-340 order: inject, save, record).
template <bool FS>
__global__ void __launch_bounds__(NTH, 4) fwd_str(const __grid_constant__ FwdMaps MP, FwdArgs A)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    StrSmem& sm = *reinterpret_cast<StrSmem*>(smem_raw);
    const Geo& G = A.G;
    const int tile = blockIdx.x;
    int tz0, tx0;
    tile_origin(G, tile, tz0, tx0);
    const int b0 = blockIdx.y * G.gf, nloc = min(G.gf, G.B - b0);
    constexpr uint32_t kBytes = (2 * HN + 3 * CN) * 4;
    auto issue = [&](int s, int b) {
        tma::mbar_expect_tx(&sm.bar[s], kBytes);
        for (int f = 0; f < 2; ++f) tma::load_3d(sm.h[s][f], &MP.halo[VX + f], &sm.bar[s], tx0 - M, tz0 - M, b);
        for (int f = 0; f < 3; ++f) tma::load_3d(sm.c[s][f], &MP.tile[SXX + f], &sm.bar[s], tx0, tz0, b);
    };
    pipeline_start(sm, nloc, b0, issue);
    const int lx = threadIdx.x, ix = tx0 + lx;
    float lamr[RPT], mur[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int iz = tz0 + threadIdx.y + 8 * r;
        const bool in = in_core(G, ix, iz);
        const long long i = (long long)b0 * G.ms + (long long)iz * G.P + ix;
        lamr[r] = in ? A.m.lam[i] : 0.f;
        mur[r] = in ? A.m.mu[i] : 0.f;
    }
    const int ntl = G.ntx * G.ntz;
    const bool ring = tile_in_pml(G, tz0, tx0) || (FS && fs_tile(G, tz0, tx0));
    const bool stile = A.strips != nullptr && tile_has_strips(G, tz0, tx0);
    for (int g = 0; g < nloc; ++g) {
        const int b = b0 + g, s = g & 1;
        // each thread waits for the stage itself; a failed wait leaves at the
        // barrier that ends the shot (after drain).  The flag is in shared
        // memory, by parity, so shot g + 1's write cannot meet a slower
        // thread's read for shot g (a register kept across the loop spills).
        if (!tma::mbar_wait(&sm.bar[s], (g >> 1) & 1, G.err, ERR_WAIT_FWD)) sm.bad[s] = 1;
        const float *tvx = sm.h[s][0], *tvz = sm.h[s][1];
        const long long so = (long long)b * G.S;
        const int key = b * ntl + tile;
        MemPair mz[RPT], mx[RPT];
        if (ring) {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int iz = tz0 + threadIdx.y + 8 * r;
                // a free surface row / column takes the CPML branch at every
                // cell (reference kernels.cuh:216-234): the high sides'
                // half-cell profiles are nonzero one cell inside their band
                const bool surf = FS && (fs_zrow(G, iz) || fs_xcol(G, ix));
                mz[r] = load_mem_z(G, A.mem, ZM_VZZ, ZM_VXZ, b, iz, ix, surf);
                mx[r] = load_mem_x(G, A.mem, XM_VXX, XM_VZX, b, iz, ix, surf);
            }
        }
        const int s0 = G.src.off[key], s1 = G.src.off[key + 1];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int lz = threadIdx.y + 8 * r, iz = tz0 + lz;
            if (iz >= G.nz || ix >= G.nx) continue;
            const int c = (lz + M) * HX + lx + M;
            const int cell = lz * TX + lx;
            const long long i = (long long)iz * G.P + ix;
            float sxx = sm.c[s][0][cell], szz = sm.c[s][1][cell], sxz = sm.c[s][2][cell];
            if (in_core(G, ix, iz)) {
                const FsAx az = fs_zax(G), ax = fs_xax(G);
                float dvx_dx = d_fs<FS, 1, false>(ax, tvx, c, ix, true, true, G.idx);
                float dvz_dz = d_fs<FS, HX, false>(az, tvz, c, iz, true, true, G.idz);
                float dvx_dz = d_fs<FS, HX, true>(az, tvx, c, iz, false, false, G.idz);
                float dvz_dx = d_fs<FS, 1, true>(ax, tvz, c, ix, false, false, G.idx);
                const float lam = lamr[r], mu = mur[r];
                const bool zs = FS && fs_zrow(G, iz), xs = FS && fs_xcol(G, ix);
                const bool pml = ring && (in_pml(G, ix, iz) || zs || xs);
                if (pml && mz[r].at >= 0) {
                    float m = G.az[iz] * mz[r].a + G.bz[iz] * dvz_dz;
                    A.mem.z[ZM_VZZ][mz[r].at] = m; dvz_dz += m;
                }
                if (pml && mx[r].at >= 0) {
                    float m = G.ax[ix] * mx[r].a + G.bx[ix] * dvx_dx;
                    A.mem.x[XM_VXX][mx[r].at] = m; dvx_dx += m;
                }
                sxx += G.dt * ((lam + 2.f * mu) * dvx_dx + lam * dvz_dz);
                szz += G.dt * ((lam + 2.f * mu) * dvz_dz + lam * dvx_dx);
                if (pml && mz[r].at >= 0) {
                    float m = G.azh[iz] * mz[r].b + G.bzh[iz] * dvx_dz;
                    A.mem.z[ZM_VXZ][mz[r].at] = m; dvx_dz += m;
                }
                if (pml && mx[r].at >= 0) {
                    float m = G.axh[ix] * mx[r].b + G.bxh[ix] * dvz_dx;
                    A.mem.x[XM_VZX][mx[r].at] = m; dvz_dx += m;
                }
                sxz += G.dt * mu * (dvx_dz + dvz_dx);
                if (FS) {   // Robertsson corrections first, then the zeroing
                    if (zs) sxx += -G.dt * lam * (lam / (lam + 2.f * mu) * dvx_dx + dvz_dz);
                    if (xs) szz += -G.dt * lam * (lam / (lam + 2.f * mu) * dvz_dz + dvx_dx);
                    if (zs) szz = 0.f;
                    if (xs) sxx = 0.f;
                    if (fs_zero_shear(G, ix, iz)) sxz = 0.f;
                }
            }
            // point sources of this cell (usually none in the tile)
            for (int e = s0; e < s1; ++e) {
                const int2 ev = G.src.ev[e];
                if (ev.x != cell) continue;
                const float w = G.wavelet[(long long)ev.y * G.nt + A.it];
                for (int k = 0; k < G.nsf; ++k) add_to(G.sf[k], w, sxx, szz, sxz);
            }
            A.f[SXX][so + i] = sxx;
            A.f[SZZ][so + i] = szz;
            A.f[SXZ][so + i] = sxz;
            if (stile) {
                const int si = strip_index(G, iz, ix);
                if (si >= 0) {
                    const long long e = (long long)b * 5 * G.nstrip + si;
                    if (G.st.fmt == SF_BF16) {
                        __nv_bfloat16* st = static_cast<__nv_bfloat16*>(A.strips) + e;
                        st[0] = __float2bfloat16(tvx[c]);
                        st[G.nstrip] = __float2bfloat16(tvz[c]);
                        st[2 * G.nstrip] = __float2bfloat16(sxx);
                        st[3 * G.nstrip] = __float2bfloat16(szz);
                        st[4 * G.nstrip] = __float2bfloat16(sxz);
                    } else {
                        float* st = static_cast<float*>(A.strips) + e;
                        st[0] = tvx[c];
                        st[G.nstrip] = tvz[c];
                        st[2 * G.nstrip] = sxx;
                        st[3 * G.nstrip] = szz;
                        st[4 * G.nstrip] = sxz;
                    }
                }
            }
        }
        // receivers of this (shot, tile): read back the final values of the step
        const int r0 = G.rec.off[key], r1 = G.rec.off[key + 1];
        __syncthreads();                       // stage s consumed; this shot's stores visible
        if (sm.bad[s]) {
            drain(sm, g, nloc, G.err, ERR_WAIT_FWD);
            return;
        }
        if (A.record && r1 > r0) {
            for (int e = r0 + threadIdx.x + threadIdx.y * TX; e < r1; e += NTH) {
                const int2 ev = G.rec.ev[e];
                const int iz = tz0 + ev.x / TX, jx = tx0 + ev.x % TX;
                const long long i = so + (long long)iz * G.P + jx;
                float* out = A.record + ((long long)(b * G.nt + A.it) * G.nrec + (ev.y - b * G.nrec)) * G.nrf;
                for (int k = 0; k < G.nrf; ++k) out[k] = A.f[G.rf[k]][i];
            }
        }
        if (threadIdx.x == 0 && threadIdx.y == 0 && g + 2 < nloc) issue(s, b + 2);
    }
}

// Body-force (velocity) sources, forward (reference sg_driver inject_source on
// a velocity field, common.cu:11-36): after the stress step, add the wavelet to
// vx / vz at each source cell of shot blockIdx.x, then -- that cell's step
// outputs having been written before the injection by fwd_str -- store the
// injected value again into the step's boundary strips (fp32 or bf16 here;
// the scaled formats are quantised from this fp32 slot afterwards) and into
// the record of any receiver on the cell.  A separate launch: every fwd_str
// CTA reads the velocities of its halo, which the injection must not race.
__global__ void vsrc_forward(const Geo G, float* vx, float* vz, void* strips, float* record, int it)
{
    const int b = blockIdx.x;
    const long long so = (long long)b * G.S;
    float* const vf[2] = {vx, vz};
    for (int s = threadIdx.x; s < G.nsrc; s += blockDim.x) {
        const int ix = G.src_loc[2 * ((long long)b * G.nsrc + s)], iz = G.src_loc[2 * ((long long)b * G.nsrc + s) + 1];
        if (ix < 0 || ix >= G.nx || iz < 0 || iz >= G.nz) continue;
        const float w = G.wavelet[((long long)b * G.nsrc + s) * G.nt + it];
        for (int k = 0; k < G.nvf; ++k) atomicAdd(vf[G.vf[k]] + so + (long long)iz * G.P + ix, w);
    }
    __syncthreads();                          // the injected values are visible to the block
    for (int s = threadIdx.x; strips && s < G.nsrc; s += blockDim.x) {
        const int ix = G.src_loc[2 * ((long long)b * G.nsrc + s)], iz = G.src_loc[2 * ((long long)b * G.nsrc + s) + 1];
        if (ix < 0 || ix >= G.nx || iz < 0 || iz >= G.nz) continue;
        const int si = strip_index(G, iz, ix);
        if (si < 0) continue;
        for (int k = 0; k < G.nvf; ++k) {
            const int fld = G.vf[k];
            const float v = vf[fld][so + (long long)iz * G.P + ix];
            const long long e = ((long long)b * 5 + fld) * G.nstrip + si;
            if (G.st.fmt == SF_BF16) static_cast<__nv_bfloat16*>(strips)[e] = __float2bfloat16(v);
            else static_cast<float*>(strips)[e] = v;
        }
    }
    for (int r = threadIdx.x; record && r < G.nrec; r += blockDim.x) {
        const int ix = G.rec_loc[2 * ((long long)b * G.nrec + r)], iz = G.rec_loc[2 * ((long long)b * G.nrec + r) + 1];
        if (ix < 0 || ix >= G.nx || iz < 0 || iz >= G.nz) continue;
        bool on_source = false;
        for (int s = 0; s < G.nsrc && !on_source; ++s)
            on_source = G.src_loc[2 * ((long long)b * G.nsrc + s)] == ix && G.src_loc[2 * ((long long)b * G.nsrc + s) + 1] == iz;
        if (!on_source) continue;
        float* out = record + ((long long)(b * G.nt + it) * G.nrec + r) * G.nrf;
        for (int k = 0; k < G.nrf; ++k)
            if (G.rf[k] <= VZ) out[k] = vf[G.rf[k]][so + (long long)iz * G.P + ix];
    }
}

// Body-force sources, reverse step it (reference fix_rho_grad_at_sources,
// common.cu:40-75, then uninject_forward_source; elastic2d/driver_traits.cuh
// 380-410): before this step's residuals enter the adjoint, add
// (adjoint v * w) / rho to the rho-gradient slot of the shot at each source
// cell, and take the wavelet back out of the reconstructed vx / vz there.
__global__ void vsrc_reverse(const Geo G, const float* avx, const float* avz, float* vx, float* vz,
                             float* grho, const float* rho, int g_shots, int it)
{
    const int b = blockIdx.x;
    const long long so = (long long)b * G.S;
    const float* const av[2] = {avx, avz};
    float* const vf[2] = {vx, vz};
    float* const gslot = grho + (long long)(b / g_shots) * G.S;
    for (int s = threadIdx.x; s < G.nsrc; s += blockDim.x) {
        const int ix = G.src_loc[2 * ((long long)b * G.nsrc + s)], iz = G.src_loc[2 * ((long long)b * G.nsrc + s) + 1];
        if (ix < 0 || ix >= G.nx || iz < 0 || iz >= G.nz) continue;
        const long long c = (long long)iz * G.P + ix;
        const float w = G.wavelet[((long long)b * G.nsrc + s) * G.nt + it];
        for (int k = 0; k < G.nvf; ++k) {
            const int fld = G.vf[k];
            atomicAdd(gslot + c, (av[fld][so + c] * w) / rho[(long long)b * G.ms + c]);
            atomicAdd(vf[fld] + so + c, -w);
        }
    }
}

// ------------------------------------------------------------------ reverse
struct RevArgs {
    Geo G;
    Models m;
    float* f[5];          // reconstructed forward fields
    float* cvx;           // carriers: v of the next step (box cells)
    float* cvz;
    float* a[5];          // adjoint fields (stress ones hold the negated adjoint)
    Slabs mo, mn;         // adjoint memories: read set (old), write set (new)
    const void* strips;   // step slot holding the strips of step it - 1 (format G.st)
    const float* adj;     // (B, nt, nrec, nrf) residuals
    float* gvp;           // gradient slots (nslot, S)
    float* gvs;
    float* grho;
    int G_shots;          // shots per CTA of rev_str (shared models)
    int it;
};
// adjoint memory slots: x {vxx, vzx, sxxx, sxzx}, z {vzz, vxz, szzz, sxzz}

// Reverse stress half for shots [g*G_shots, ...): residual injection
// (reference inject_residuals, signs: stress -1, velocity +1), stress
// reconstruction on the NOPML region with the forward source removed
// (kernels.cuh:455-493 after uninject_forward_source) or strip restore, the
// fused vp / vs / rho imaging on the physical box (kernels.cuh:601-663) and
// the receiver rho correction (common.cu:77-117).  The gradient contributions
// of the CTA's shots are summed in registers and added to slot blockIdx.y.
template <bool FS>
__global__ void __launch_bounds__(NTH, 4) rev_str(RevArgs A)
{
    extern __shared__ float sm[];
    float *tvx = sm, *tvz = sm + HN;
    const Geo& G = A.G;
    const int tile = blockIdx.x, grp = blockIdx.y;
    int tz0, tx0;
    tile_origin(G, tile, tz0, tx0);
    const int lx = threadIdx.x, ix = tx0 + lx;
    const int b_lo = grp * A.G_shots, b_hi = min(G.B, b_lo + A.G_shots);
    float gvp[RPT], gvs[RPT], grho[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) gvp[r] = gvs[r] = grho[r] = 0.f;
    const int tid = threadIdx.x + threadIdx.y * TX;

    for (int b = b_lo; b < b_hi; ++b) {
        const long long so = (long long)b * G.S;
        const int key = b * G.ntx * G.ntz + tile;
        const int r0 = G.rec.off[key], r1 = G.rec.off[key + 1];
        const int s0 = G.src.off[key], s1 = G.src.off[key + 1];
        __syncthreads();                       // previous shot's tiles consumed
        {
            float* const t[2] = {tvx, tvz};
            const float* const g[2] = {A.f[VX] + so, A.f[VZ] + so};
            load_tiles<2>(t, g, G, tz0, tx0);
        }
        // residuals of step it into the adjoint fields of this tile's receivers
        for (int e = r0 + tid; e < r1; e += NTH) {
            const int2 ev = G.rec.ev[e];
            const long long i = so + (long long)(tz0 + ev.x / TX) * G.P + tx0 + ev.x % TX;
            const float* res = A.adj + ((long long)(b * G.nt + A.it) * G.nrec + (ev.y - b * G.nrec)) * G.nrf;
            for (int k = 0; k < G.nrf; ++k) {
                const int fld = G.rf[k];
                atomicAdd(A.a[fld] + i, fld >= SXX ? -res[k] : res[k]);
            }
        }
        __syncthreads();
        const float* __restrict__ lam_ = A.m.lam + (long long)b * G.ms;
        const float* __restrict__ mu_ = A.m.mu + (long long)b * G.ms;
        const float* __restrict__ rho_ = A.m.rho + (long long)b * G.ms;
        const float* __restrict__ vp_ = A.m.vp + (long long)b * G.ms;
        const float* __restrict__ vs_ = A.m.vs + (long long)b * G.ms;
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int lz = threadIdx.y + 8 * r, iz = tz0 + lz;
            if (iz >= G.nz || ix >= G.nx) continue;
            const long long i = (long long)iz * G.P + ix;
            if (!in_core(G, ix, iz)) {
                const int si = strip_index(G, iz, ix);
                if (si >= 0) {
                    A.f[SXX][so + i] = strip_val(G, A.strips, b, SXX, iz, ix, si);
                    A.f[SZZ][so + i] = strip_val(G, A.strips, b, SZZ, iz, ix, si);
                    A.f[SXZ][so + i] = strip_val(G, A.strips, b, SXZ, iz, ix, si);
                }
                continue;
            }
            const int c = (lz + M) * HX + lx + M;
            const FsAx az = fs_zax(G), ax = fs_xax(G);
            const float dvx_dx = d_fs<FS, 1, false>(ax, tvx, c, ix, true, true, G.idx);
            const float dvz_dz = d_fs<FS, HX, false>(az, tvz, c, iz, true, true, G.idz);
            const float dvx_dz = d_fs<FS, HX, true>(az, tvx, c, iz, false, false, G.idz);
            const float dvz_dx = d_fs<FS, 1, true>(ax, tvz, c, ix, false, false, G.idx);
            if (in_recon(G, ix, iz)) {
                float sxx = A.f[SXX][so + i], szz = A.f[SZZ][so + i], sxz = A.f[SXZ][so + i];
                const int cell = lz * TX + lx;
                for (int e = s0; e < s1; ++e) {
                    const int2 ev = G.src.ev[e];
                    if (ev.x != cell) continue;
                    const float w = G.wavelet[(long long)ev.y * G.nt + A.it];
                    for (int k = 0; k < G.nsf; ++k) add_to(G.sf[k], -w, sxx, szz, sxz);
                }
                const float lam = lam_[i], mu = mu_[i];
                A.f[SXX][so + i] = sxx - G.dt * ((lam + 2.f * mu) * dvx_dx + lam * dvz_dz);
                A.f[SZZ][so + i] = szz - G.dt * ((lam + 2.f * mu) * dvz_dz + lam * dvx_dx);
                A.f[SXZ][so + i] = sxz - G.dt * mu * (dvx_dz + dvz_dx);
            } else {
                const int si = strip_index(G, iz, ix);
                if (si >= 0) {
                    A.f[SXX][so + i] = strip_val(G, A.strips, b, SXX, iz, ix, si);
                    A.f[SZZ][so + i] = strip_val(G, A.strips, b, SZZ, iz, ix, si);
                    A.f[SXZ][so + i] = strip_val(G, A.strips, b, SXZ, iz, ix, si);
                }
            }
            if (in_box(G, ix, iz)) {
                // the stresses a surface zeroes carry no adjoint there
                const bool zs = FS && fs_zrow(G, iz), xs = FS && fs_xcol(G, ix);
                const float bsxx = xs ? 0.f : A.a[SXX][so + i];
                const float bszz = zs ? 0.f : A.a[SZZ][so + i];
                const float bsxz = FS && fs_zero_shear(G, ix, iz) ? 0.f : A.a[SXZ][so + i];
                const float rho = rho_[i], vp = vp_[i], vs = vs_[i];
                float gl, gm;
                if (zs && xs) {
                    gl = gm = 0.f;           // a corner: every stress is zeroed
                } else if (zs || xs) {
                    // d / d(lam, mu) of the corrected surface update dt C d(v
                    // along the surface), C = 4 mu (lam + mu) / (lam + 2 mu)
                    // (kernels.cuh:633-646)
                    const float vp2 = vp * vp, vs2 = vs * vs, vp4 = vp2 * vp2;
                    const float a = zs ? bsxx * dvx_dx : bszz * dvz_dz;
                    gl = a * 4.f * vs2 * vs2 / vp4;
                    gm = a * 4.f * (vp4 - 2.f * vp2 * vs2 + 2.f * vs2 * vs2) / vp4;
                } else {
                    gl = (bsxx + bszz) * (dvx_dx + dvz_dz);
                    gm = 2.f * (bsxx * dvx_dx + bszz * dvz_dz);
                }
                gm += bsxz * (dvx_dz + dvz_dx);
                gvp[r] += -2.f * rho * vp * gl * G.dt;
                gvs[r] += -(-4.f * rho * vs * gl + 2.f * rho * vs * gm) * G.dt;
                float gr = (A.a[VX][so + i] * (tvx[c] - A.cvx[so + i]) + A.a[VZ][so + i] * (tvz[c] - A.cvz[so + i])) / rho;
                gr -= gl * (vp * vp - 2.f * vs * vs) * G.dt + gm * (vs * vs) * G.dt;
                grho[r] += gr;
            }
        }
    }
    // add the group's image to its slot
    const long long slot = (long long)grp * G.S;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int iz = tz0 + threadIdx.y + 8 * r;
        if (!in_box(G, ix, iz)) continue;
        const long long i = slot + (long long)iz * G.P + ix;
        A.gvp[i] += gvp[r];
        A.gvs[i] += gvs[r];
        A.grho[i] += grho[r];
    }
    // receiver rho correction after the image (velocity receivers in the box)
    bool any = false;
    for (int b = b_lo; b < b_hi; ++b) {
        const int key = b * G.ntx * G.ntz + tile;
        any |= G.rec.off[key + 1] > G.rec.off[key];
    }
    if (!any) return;
    __syncthreads();
    for (int b = b_lo; b < b_hi; ++b) {
        const long long so = (long long)b * G.S;
        const int key = b * G.ntx * G.ntz + tile;
        const float* __restrict__ rho_ = A.m.rho + (long long)b * G.ms;
        for (int e = G.rec.off[key] + tid; e < G.rec.off[key + 1]; e += NTH) {
            const int2 ev = G.rec.ev[e];
            const int iz = tz0 + ev.x / TX, jx = tx0 + ev.x % TX;
            if (!in_box(G, jx, iz)) continue;
            const long long i = (long long)iz * G.P + jx;
            const float* res = A.adj + ((long long)(b * G.nt + A.it) * G.nrec + (ev.y - b * G.nrec)) * G.nrf;
            for (int k = 0; k < G.nrf; ++k) {
                const int fld = G.rf[k];
                if (fld > VZ) continue;
                const float now = A.f[fld][so + i];
                const float nxt = (fld == VX ? A.cvx : A.cvz)[so + i];
                atomicAdd(A.grho + slot + i, -res[k] * (now - nxt) / rho_[i]);
            }
        }
    }
}

__device__ __forceinline__ bool owns(int lz, int lx)
{
    return lz >= M && lz < M + TZ && lx >= M && lx < M + TX;
}

// Stress-adjoint apply (reference kernels.cuh:807-837) with q = (qxx, qzz,
// qxz, qzx) of the stress-adjoint prepare (kernels.cuh:676-750) built in
// shared memory for the tile and its halo.  The owner of a cell writes its new
// adjoint CPML memories.
template <bool FS>
__global__ void __launch_bounds__(NTH, 4) rev_sadj(RevArgs A)
{
    extern __shared__ float sm[];
    float* tq[4] = {sm, sm + HN, sm + 2 * HN, sm + 3 * HN};
    const Geo& G = A.G;
    const int b = blockIdx.y;
    int tz0, tx0;
    tile_origin(G, blockIdx.x, tz0, tx0);
    const long long so = (long long)b * G.S;
    const float* __restrict__ lam_ = A.m.lam + (long long)b * G.ms;
    const float* __restrict__ mu_ = A.m.mu + (long long)b * G.ms;
    const int tid = threadIdx.x + threadIdx.y * TX;
    const float* __restrict__ mo_vxx = A.mo.x[XM_VXX];
    const float* __restrict__ mo_vzx = A.mo.x[XM_VZX];
    const float* __restrict__ mo_vzz = A.mo.z[ZM_VZZ];
    const float* __restrict__ mo_vxz = A.mo.z[ZM_VXZ];
    float* __restrict__ mn_vxx = A.mn.x[XM_VXX];
    float* __restrict__ mn_vzx = A.mn.x[XM_VZX];
    float* __restrict__ mn_vzz = A.mn.z[ZM_VZZ];
    float* __restrict__ mn_vxz = A.mn.z[ZM_VXZ];
    float rs[NLD][5];
#pragma unroll
    for (int j = 0; j < NLD; ++j) {
        const int k = tid + j * NTH;
        const int lz = k / HX, lx = k - lz * HX;
        const int iz = tz0 - M + lz, ix = tx0 - M + lx;
        const bool ok = k < HN && (unsigned)iz < (unsigned)G.nz && (unsigned)ix < (unsigned)G.nx;
        const long long i = (long long)iz * G.P + ix;
        rs[j][0] = ok ? A.a[SXX][so + i] : 0.f;
        rs[j][1] = ok ? A.a[SZZ][so + i] : 0.f;
        rs[j][2] = ok ? A.a[SXZ][so + i] : 0.f;
        rs[j][3] = ok ? lam_[i] : 0.f;
        rs[j][4] = ok ? mu_[i] : 0.f;
    }
#pragma unroll
    for (int j = 0; j < NLD; ++j) {
        const int k = tid + j * NTH;
        if (k >= HN) continue;
        const int lz = k / HX, lx = k - lz * HX;
        const int iz = tz0 - M + lz, ix = tx0 - M + lx;
        const bool ing = (unsigned)iz < (unsigned)G.nz && (unsigned)ix < (unsigned)G.nx;
        const bool zs = FS && ing && fs_zrow(G, iz), xs = FS && ing && fs_xcol(G, ix);
        const float bsxx = xs ? 0.f : rs[j][0], bszz = zs ? 0.f : rs[j][1];
        const float bsxz = FS && ing && fs_zero_shear(G, ix, iz) ? 0.f : rs[j][2];
        const float lam = rs[j][3], mu = rs[j][4];
        float q0, q1;
        if (zs || xs) {
            // transposes of the corrected surface updates (a corner: none)
            const float cs = zs && xs ? 0.f : G.dt * (4.f * mu * (lam + mu) / (lam + 2.f * mu));
            q0 = zs ? cs * bsxx : 0.f;
            q1 = xs ? cs * bszz : 0.f;
        } else {
            q0 = G.dt * ((lam + 2.f * mu) * bsxx + lam * bszz);
            q1 = G.dt * ((lam + 2.f * mu) * bszz + lam * bsxx);
        }
        float q2 = G.dt * mu * bsxz;
        float q3 = G.dt * mu * bsxz;
        if ((unsigned)iz < (unsigned)G.nz && (unsigned)ix < (unsigned)G.nx && in_pml(G, ix, iz)) {
            const bool own = owns(lz, lx);
            const int xs = xslab(G, ix), zs = zslab(G, iz);
            if (xs >= 0) {
                const long long xi = ((long long)b * G.nz + iz) * G.WX + xs;
                const float t0 = mo_vxx[xi] + q0, t3 = mo_vzx[xi] + q3;
                if (own) {
                    mn_vxx[xi] = G.ax[ix] * t0;
                    mn_vzx[xi] = G.axh[ix] * t3;
                }
                q0 = q0 + G.bx[ix] * t0;
                q3 = q3 + G.bxh[ix] * t3;
            }
            if (zs >= 0) {
                const long long zi = ((long long)b * G.WZ + zs) * G.P + ix;
                const float t1 = mo_vzz[zi] + q1, t2 = mo_vxz[zi] + q2;
                if (own) {
                    mn_vzz[zi] = G.az[iz] * t1;
                    mn_vxz[zi] = G.azh[iz] * t2;
                }
                q1 = q1 + G.bz[iz] * t1;
                q2 = q2 + G.bzh[iz] * t2;
            }
        }
        tq[0][k] = q0; tq[1][k] = q1; tq[2][k] = q2; tq[3][k] = q3;
    }
    __syncthreads();
    const int lx = threadIdx.x, ix = tx0 + lx;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int lz = threadIdx.y + 8 * r, iz = tz0 + lz;
        if (!in_core(G, ix, iz)) continue;
        const int c = (lz + M) * HX + lx + M;
        const long long i = so + (long long)iz * G.P + ix;
        const FsAx az = fs_zax(G), ax = fs_xax(G);
        A.a[VX][i] += adj_fs<FS, 1, false>(ax, tq[0], c, ix, G.nx, true, true, G.idx) +
                      adj_fs<FS, HX, true>(az, tq[2], c, iz, G.nz, false, false, G.idz);
        A.a[VZ][i] += adj_fs<FS, 1, true>(ax, tq[3], c, ix, G.nx, false, false, G.idx) +
                      adj_fs<FS, HX, false>(az, tq[1], c, iz, G.nz, true, true, G.idz);
    }
}

// Velocity-adjoint apply (reference kernels.cuh:989-1019) with p = (pxx,
// pzz, pxz, pzx) of the velocity-adjoint prepare (kernels.cuh:873-958) built
// in shared memory, then the reverse velocity half of the forward
// reconstruction: carrier capture of v(it) on the box, the NOPML velocity
// step (kernels.cuh:365-401) and the velocity strip restore of step it - 1.
template <bool FS>
__global__ void __launch_bounds__(NTH, 4) rev_vadj(RevArgs A)
{
    extern __shared__ float sm[];
    float* tp[4] = {sm, sm + HN, sm + 2 * HN, sm + 3 * HN};
    float *tsxx = sm + 4 * HN, *tszz = sm + 5 * HN, *tsxz = sm + 6 * HN;
    const Geo& G = A.G;
    const int b = blockIdx.y;
    int tz0, tx0;
    tile_origin(G, blockIdx.x, tz0, tx0);
    const long long so = (long long)b * G.S;
    const float* __restrict__ bv_ = A.m.bv + (long long)b * G.ms;
    const int tid = threadIdx.x + threadIdx.y * TX;
    const float* __restrict__ mo_sxxx = A.mo.x[XM_SXXX];
    const float* __restrict__ mo_sxzx = A.mo.x[XM_SXZX];
    const float* __restrict__ mo_sxzz = A.mo.z[ZM_SXZZ];
    const float* __restrict__ mo_szzz = A.mo.z[ZM_SZZZ];
    float* __restrict__ mn_sxxx = A.mn.x[XM_SXXX];
    float* __restrict__ mn_sxzx = A.mn.x[XM_SXZX];
    float* __restrict__ mn_sxzz = A.mn.z[ZM_SXZZ];
    float* __restrict__ mn_szzz = A.mn.z[ZM_SZZZ];
    float rv[NLD][3];
#pragma unroll
    for (int j = 0; j < NLD; ++j) {
        const int k = tid + j * NTH;
        const int lz = k / HX, lx = k - lz * HX;
        const int iz = tz0 - M + lz, ix = tx0 - M + lx;
        const bool ok = k < HN && (unsigned)iz < (unsigned)G.nz && (unsigned)ix < (unsigned)G.nx;
        const long long i = (long long)iz * G.P + ix;
        rv[j][0] = ok ? A.a[VX][so + i] : 0.f;
        rv[j][1] = ok ? A.a[VZ][so + i] : 0.f;
        rv[j][2] = ok ? bv_[i] : 0.f;
    }
#pragma unroll
    for (int j = 0; j < NLD; ++j) {
        const int k = tid + j * NTH;
        if (k >= HN) continue;
        const int lz = k / HX, lx = k - lz * HX;
        const int iz = tz0 - M + lz, ix = tx0 - M + lx;
        const float avx = rv[j][0], avz = rv[j][1], k_ = rv[j][2];
        float p0 = k_ * avx;      // pxx
        float p2 = k_ * avx;      // pxz
        float p3 = k_ * avz;      // pzx
        float p1 = k_ * avz;      // pzz
        if ((unsigned)iz < (unsigned)G.nz && (unsigned)ix < (unsigned)G.nx && in_pml(G, ix, iz)) {
            const bool own = owns(lz, lx);
            const int xs = xslab(G, ix), zs = zslab(G, iz);
            if (xs >= 0) {
                const long long xi = ((long long)b * G.nz + iz) * G.WX + xs;
                const float t0 = mo_sxxx[xi] + p0, t3 = mo_sxzx[xi] + p3;
                if (own) {
                    mn_sxxx[xi] = G.axh[ix] * t0;
                    mn_sxzx[xi] = G.ax[ix] * t3;
                }
                p0 = p0 + G.bxh[ix] * t0;
                p3 = p3 + G.bx[ix] * t3;
            }
            if (zs >= 0) {
                const long long zi = ((long long)b * G.WZ + zs) * G.P + ix;
                const float t2 = mo_sxzz[zi] + p2, t1 = mo_szzz[zi] + p1;
                if (own) {
                    mn_sxzz[zi] = G.az[iz] * t2;
                    mn_szzz[zi] = G.azh[iz] * t1;
                }
                p2 = p2 + G.bz[iz] * t2;
                p1 = p1 + G.bzh[iz] * t1;
            }
        }
        tp[0][k] = p0; tp[1][k] = p1; tp[2][k] = p2; tp[3][k] = p3;
    }
    {
        float* const t[3] = {tsxx, tszz, tsxz};
        const float* const g[3] = {A.f[SXX] + so, A.f[SZZ] + so, A.f[SXZ] + so};
        load_tiles<3>(t, g, G, tz0, tx0);
    }
    __syncthreads();
    const int lx = threadIdx.x, ix = tx0 + lx;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int lz = threadIdx.y + 8 * r, iz = tz0 + lz;
        if (!in_core(G, ix, iz)) continue;
        const int c = (lz + M) * HX + lx + M;
        const long long i = (long long)iz * G.P + ix;
        // the stresses a surface zeroes had their adjoint zeroed by this
        // step's stress half
        const FsAx az = fs_zax(G), ax = fs_xax(G);
        const float sxx0 = FS && fs_xcol(G, ix) ? 0.f : A.a[SXX][so + i];
        const float szz0 = FS && fs_zrow(G, iz) ? 0.f : A.a[SZZ][so + i];
        const float sxz0 = FS && fs_zero_shear(G, ix, iz) ? 0.f : A.a[SXZ][so + i];
        A.a[SXX][so + i] = sxx0 + adj_fs<FS, 1, true>(ax, tp[0], c, ix, G.nx, true, false, G.idx);
        A.a[SZZ][so + i] = szz0 + adj_fs<FS, HX, true>(az, tp[1], c, iz, G.nz, true, false, G.idz);
        A.a[SXZ][so + i] = sxz0 + (adj_fs<FS, HX, false>(az, tp[2], c, iz, G.nz, true, true, G.idz) +
                                   adj_fs<FS, 1, false>(ax, tp[3], c, ix, G.nx, true, true, G.idx));
        if (!in_box(G, ix, iz)) continue;
        const float vx = A.f[VX][so + i], vz = A.f[VZ][so + i];
        A.cvx[so + i] = vx;
        A.cvz[so + i] = vz;
        if (in_recon(G, ix, iz)) {
            const float k_ = bv_[i];
            A.f[VX][so + i] = vx - k_ * (d_fs<FS, 1, true>(ax, tsxx, c, ix, true, false, G.idx) +
                                         d_fs<FS, HX, false>(az, tsxz, c, iz, true, true, G.idz));
            A.f[VZ][so + i] = vz - k_ * (d_fs<FS, 1, false>(ax, tsxz, c, ix, true, true, G.idx) +
                                         d_fs<FS, HX, true>(az, tszz, c, iz, true, false, G.idz));
        }
    }
    // strips (box ring and the M cells outside it) of step it - 1
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int lz = threadIdx.y + 8 * r, iz = tz0 + lz;
        if (iz >= G.nz || ix >= G.nx || in_recon(G, ix, iz)) continue;
        const int si = strip_index(G, iz, ix);
        if (si < 0) continue;
        const long long i = so + (long long)iz * G.P + ix;
        A.f[VX][i] = strip_val(G, A.strips, b, VX, iz, ix, si);
        A.f[VZ][i] = strip_val(G, A.strips, b, VZ, iz, ix, si);
    }
}

// One step's strips (fp32 strip set (B, 5, nstrip) in `scratch`) into the
// scaled bands of a step slot: one CTA per (field, shot, band, block of kQB
// cells) -- max |value| of the block, its scale, the codes (reference
// boundarysaver.cu:957-990, 1050-1080).
__global__ void __launch_bounds__(kQB) quantize_strips(const Geo G, const float* __restrict__ scratch, void* slot)
{
    const StripStore& S = G.st;
    const int per = S.blocks[0] + S.blocks[1] + S.blocks[2] + S.blocks[3];
    const int row = blockIdx.x / per;                 // field k * B + shot b
    const int k = row / G.B, b = row - k * G.B;
    int j = blockIdx.x - row * per, f = 0;
    while (f < 3 && j >= S.blocks[f]) { j -= S.blocks[f]; ++f; }
    const int idx = j * kQB + threadIdx.x;
    const bool in = idx < S.cells[f];
    float v = 0.f;
    if (in) {
        int iz, ix;
        band_cell(G, f, idx, iz, ix);
        v = scratch[((long long)b * 5 + k) * G.nstrip + strip_index(G, iz, ix)];
    }
    float m = fabsf(v);
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wmax[kQB / 32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    m = wmax[0];
#pragma unroll
    for (int i = 1; i < kQB / 32; ++i) m = fmaxf(m, wmax[i]);
    char* base = static_cast<char*>(slot);
    if (threadIdx.x == 0) reinterpret_cast<float*>(base + S.scl[f])[(long long)row * S.blocks[f] + j] = m;
    if (!in) return;
    const long long q = (long long)row * S.cells[f] + idx;
    if (S.fmt == SF_F16) {
        const float inv = m > 0.0f ? 1.0f / m : 0.0f;
        reinterpret_cast<__half*>(base + S.pay[f])[q] = __float2half(v * inv);
    } else {
        const float qs = m > 0.0f ? 127.0f / m : 0.0f;
        int c = __float2int_rn(v * qs) + 128;
        c = c < 0 ? 0 : (c > 255 ? 255 : c);
        reinterpret_cast<uint8_t*>(base + S.pay[f])[q] = (uint8_t)c;
    }
}

// Models onto the pitched grid: rho, Lame parameters (reference
// derived_models.cu:27-37, same rounding), bv = dt * (1 / rho) (the velocity
// kernels' dt * inv_rho, kernels.cuh:73, 389, 901), vp and vs for the imaging.
__global__ void prep_kernel(const float* __restrict__ vp, const float* __restrict__ vs,
                            const float* __restrict__ rho, int nm, int nz, int nx, int P, float dt,
                            float* orho, float* olam, float* omu, float* obv, float* ovp, float* ovs)
{
    const long long n = (long long)nm * nz * nx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long b = k / ((long long)nz * nx), rem = k - b * nz * nx;
        const int iz = (int)(rem / nx), ix = (int)(rem - (long long)iz * nx);
        const long long o = (b * nz + iz) * P + ix;
        const float v = vp[k], s = vs[k], r = rho[k];
        orho[o] = r;
        omu[o] = __fmul_rn(__fmul_rn(r, s), s);
        olam[o] = __fmul_rn(r, __fsub_rn(__fmul_rn(v, v), __fmul_rn(__fmul_rn(2.0f, s), s)));
        obv[o] = dt * (1.f / r);
        ovp[o] = v;
        ovs[o] = s;
    }
}

// Gradient output: sum of the slots in slot order on the physical box, zero
// elsewhere, unpitched (nout, nz, nx); slot s of a per-shot model is shot s.
__global__ void finalize_kernel(const float* __restrict__ slots, int nslot, int per_shot, Geo G, float* out)
{
    const int nout = per_shot ? nslot : 1;
    const long long n = (long long)nout * G.nz * G.nx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long b = k / ((long long)G.nz * G.nx), rem = k - b * G.nz * G.nx;
        const int iz = (int)(rem / G.nx), ix = (int)(rem - (long long)iz * G.nx);
        float v = 0.f;
        if (in_box(G, ix, iz)) {
            const long long o = (long long)iz * G.P + ix;
            if (per_shot) {
                v = slots[b * G.S + o];
            } else {
                for (int s = 0; s < nslot; ++s) v += slots[s * G.S + o];
            }
        }
        out[k] = v;
    }
}

// ------------------------------------------------------------------- host
struct Plan {
    Geo G;
    int nm;          // model copies
    int gshots;      // shots per rev_str CTA
    int graph_steps; // time steps per captured CUDA graph (0: stream launches)
    int nslot;       // gradient slots
    bool host_tape;  // boundary-saving tape in pinned host memory (SWEEP_MEM_HOST_TAPE)
};

static int env_int(const char* name, int dflt)
{
    if (const char* e = getenv(name)) {
        const int v = atoi(e);
        if (v >= 1) return v;
    }
    return dflt;
}

static Plan make_plan(const sweep_elastic_desc* d)
{
    SWEEP_REQUIRE(d != nullptr, "null descriptor");
    SWEEP_REQUIRE(d->M == M, "elastic2d: only spatial order 8 (M = 4) is built (got M = %d)", d->M);
    SWEEP_REQUIRE(d->B >= 1 && d->nt >= 1, "elastic2d: B and nt must be >= 1");
    SWEEP_REQUIRE(d->nsrc >= 0 && d->nrec >= 0, "elastic2d: negative source/receiver count");
    SWEEP_REQUIRE(d->nsrc_fields >= 1 && d->nsrc_fields <= 5, "elastic2d: 1 to 5 source fields (got %d)", d->nsrc_fields);
    for (int k = 0; k < d->nsrc_fields; ++k) {
        SWEEP_REQUIRE(d->src_fields[k] >= VX && d->src_fields[k] <= SXZ, "elastic2d: bad source field %d",
                      d->src_fields[k]);
        for (int j = 0; j < k; ++j)
            SWEEP_REQUIRE(d->src_fields[j] != d->src_fields[k], "elastic2d: source field %d repeated", d->src_fields[k]);
    }
    SWEEP_REQUIRE(d->nrec_fields >= 1 && d->nrec_fields <= 5, "elastic2d: 1 to 5 receiver fields (got %d)", d->nrec_fields);
    for (int k = 0; k < d->nrec_fields; ++k)
        SWEEP_REQUIRE(d->rec_fields[k] >= 0 && d->rec_fields[k] <= SXZ, "elastic2d: bad receiver field %d", d->rec_fields[k]);
    for (int f = 0; f < 4; ++f) {
        if (d->free_surface[f])
            SWEEP_REQUIRE(d->pad[f] == 0, "elastic2d: a free face has no PML pad (face %d has %d)", f, d->pad[f]);
        else
            SWEEP_REQUIRE(d->pad[f] >= 1, "elastic2d: every absorbing face needs a PML pad >= 1 (face %d has %d)", f,
                          d->pad[f]);
    }
    Plan pl{};
    Geo& G = pl.G;
    G.fs = 0;
    for (int f = 0; f < 4; ++f)
        if (d->free_surface[f]) G.fs |= 1 << f;
    G.B = d->B; G.nz = d->nz; G.nx = d->nx; G.nt = d->nt;
    G.P = (d->nx + 31) / 32 * 32;
    G.S = (long long)d->nz * G.P;
    SWEEP_REQUIRE(G.S < (1LL << 31), "elastic2d: one shot's grid must hold < 2^31 cells");
    G.z0 = d->pad[0] + M; G.z1 = d->nz - d->pad[1] - M;
    G.x0 = d->pad[2] + M; G.x1 = d->nx - d->pad[3] - M;
    G.bw = G.x1 - G.x0; G.bh = G.z1 - G.z0;
    SWEEP_REQUIRE(G.bw >= 2 && G.bh >= 2, "elastic2d: the physical box must be at least 2 x 2 cells");
    G.ZL = d->pad[0] + M; G.ZH = d->pad[1] + M; G.XL = d->pad[2] + M; G.XH = d->pad[3] + M;
    G.SZL = std::min(G.ZL + 1, d->nz); G.SZH = std::min(G.ZH + 1, d->nz - G.SZL);
    G.SXL = std::min(G.XL + 1, d->nx); G.SXH = std::min(G.XH + 1, d->nx - G.SXL);
    G.WX = G.SXL + G.SXH; G.WZ = G.SZL + G.SZH;
    G.ntx = (d->nx + TX - 1) / TX; G.ntz = (d->nz + TZ - 1) / TZ;
    G.nstrip = 2 * M * G.bw + 2 * (G.bw + 2 * M) + (G.bh - 2) * 2 * (M + 1);
    G.dt = d->dt; G.idx = 1.f / d->dx; G.idz = 1.f / d->dz;
    G.az = d->az; G.bz = d->bz; G.azh = d->azh; G.bzh = d->bzh;
    G.ax = d->ax; G.bx = d->bx; G.axh = d->axh; G.bxh = d->bxh;
    G.nsrc = d->nsrc; G.nrec = d->nrec; G.nrf = d->nrec_fields;
    for (int k = 0; k < 5; ++k) G.rf[k] = d->rec_fields[k];
    // stress sources are added inside the stress kernels; velocity (body-force)
    // sources by vsrc_forward / vsrc_reverse around them
    G.nsf = G.nvf = 0;
    for (int k = 0; k < d->nsrc_fields; ++k) {
        if (d->src_fields[k] >= SXX) G.sf[G.nsf++] = d->src_fields[k];
        else G.vf[G.nvf++] = d->src_fields[k];
    }
    G.src_loc = d->src_loc; G.rec_loc = d->rec_loc;
    const bool per_shot = d->model_stride != 0;
    SWEEP_REQUIRE(!per_shot || d->model_stride == (int64_t)d->nz * d->nx,
                  "elastic2d: model_stride must be 0 or nz * nx");
    G.ms = per_shot ? G.S : 0;
    G.wavelet = d->wavelet;
    pl.nm = per_shot ? d->B : 1;
    // shots per CTA: the shape's recorded schedule value if any, else the
    // environment, else the measured default (the forward's capped to keep at
    // least two waves of CTAs)
    const sweep_b200_schedule sc = recorded_schedule(d);
    pl.gshots = per_shot ? 1
                         : std::min(sc.shots_rev >= 1 ? sc.shots_rev : env_int("SWEEP_B200_EL_SHOTS_PER_CTA", 4), d->B);
    const long long ntl = (long long)G.ntx * G.ntz;
    int gf = per_shot ? 1 : std::min(env_int("SWEEP_B200_EL_SHOTS_PER_CTA_FWD", 4), d->B);
    while (gf > 1 && ntl * ((d->B + gf - 1) / gf) < 2LL * 148 * 4) --gf;
    if (!per_shot && sc.shots_fwd >= 1) gf = std::min(sc.shots_fwd, d->B);
    G.gf = gf;
    pl.graph_steps = resolve_graph_steps(sc.graph_steps);
    pl.nslot = (d->B + pl.gshots - 1) / pl.gshots;
    return pl;
}

struct Common {
    float *rho, *lam, *mu, *bv, *vp, *vs;
    int32_t *src_off, *rec_off;
    int2 *src_ev, *rec_ev;
    int* err;
};

static void carve_common(Carve& c, const Plan& pl, Common& w)
{
    const Geo& G = pl.G;
    const long long mc = (long long)pl.nm * G.S;
    w.rho = c.take<float>(mc); w.lam = c.take<float>(mc); w.mu = c.take<float>(mc);
    w.bv = c.take<float>(mc); w.vp = c.take<float>(mc); w.vs = c.take<float>(mc);
    const long long nkey = (long long)G.B * G.ntx * G.ntz + 1;
    w.src_off = c.take<int32_t>(nkey);
    w.rec_off = c.take<int32_t>(nkey);
    w.src_ev = c.take<int2>((long long)G.B * G.nsrc + 1);
    w.rec_ev = c.take<int2>((long long)G.B * G.nrec + 1);
    w.err = c.take<int>(1);
}

static void carve_slabs(Carve& c, const Geo& G, Slabs& s)
{
    for (int k = 0; k < 4; ++k) s.x[k] = c.take<float>((long long)G.B * G.nz * G.WX);
    for (int k = 0; k < 4; ++k) s.z[k] = c.take<float>((long long)G.B * G.WZ * G.P);
}

struct FwdWs {
    Common cm;
    float* f[5];
    Slabs mem;
    char* zero0;          // [zero0, zero1) cleared before the time loop
    char* zero1;
    float* scratch;       // one step's fp32 strips ahead of their quantisation (scaled formats)
    char* ring;           // host tape: HostRing::R device strip slots
};

static void carve_fwd(Carve& c, const Plan& pl, FwdWs& w)
{
    carve_common(c, pl, w.cm);
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    for (int k = 0; k < 5; ++k) w.f[k] = c.take<float>((long long)pl.G.B * pl.G.S);
    carve_slabs(c, pl.G, w.mem);
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
    if (pl.G.st.fmt == SF_F16 || pl.G.st.fmt == SF_I8) w.scratch = c.take<float>(5LL * pl.G.B * pl.G.nstrip);
    if (pl.host_tape) w.ring = c.take<char>((long long)HostRing::R * pl.G.st.step);
}

struct RevWs {
    Common cm;
    float* f[5];
    float *cvx, *cvz;
    float* a[5];
    Slabs m[2];
    float *gvp, *gvs, *grho;
    char* zero0;
    char* zero1;
    Slabs fmem;           // checkpoint mode: forward CPML memories of the replay
    float* chunk;         // checkpoint mode: strips of one chunk, (k + 1, B, 5, nstrip)
    char* ring;           // host tape: HostRing::R device strip slots
};

static void carve_rev(Carve& c, const Plan& pl, RevWs& w)
{
    carve_common(c, pl, w.cm);
    const Geo& G = pl.G;
    for (int k = 0; k < 5; ++k) w.f[k] = c.take<float>((long long)G.B * G.S);
    c.take<char>(0);
    w.zero0 = c.base ? c.base + c.off : nullptr;
    w.cvx = c.take<float>((long long)G.B * G.S);
    w.cvz = c.take<float>((long long)G.B * G.S);
    for (int k = 0; k < 5; ++k) w.a[k] = c.take<float>((long long)G.B * G.S);
    carve_slabs(c, G, w.m[0]);
    carve_slabs(c, G, w.m[1]);
    w.gvp = c.take<float>((long long)pl.nslot * G.S);
    w.gvs = c.take<float>((long long)pl.nslot * G.S);
    w.grho = c.take<float>((long long)pl.nslot * G.S);
    c.take<char>(0);
    w.zero1 = c.base ? c.base + c.off : nullptr;
    if (pl.host_tape) w.ring = c.take<char>((long long)HostRing::R * G.st.step);
}

static void carve_rev_ckpt(Carve& c, const Plan& pl, int k, RevWs& w)
{
    carve_rev(c, pl, w);
    carve_slabs(c, pl.G, w.fmem);
    w.chunk = c.take<float>((long long)(k + 1) * pl.G.B * 5 * pl.G.nstrip);
}

// Checkpointed boundary saving (SWEEP_MEM_CHECKPOINT, chunk length k): for
// every chunk c >= 1 the tape holds the state after step c k - 1 -- the five
// fields and the eight forward CPML memories -- and the strips of that step;
// the backward replays each chunk from its checkpoint into the strips of that
// chunk and runs the boundary-saving reverse steps over it (the reference's
// staggered driver replays chunks as well, sg_driver.cuh:911-925).
static long long slab_floats(const Geo& G)
{
    return 4LL * G.B * G.nz * G.WX + 4LL * G.B * G.WZ * G.P;
}

static long long ckpt_stride(const Plan& pl)
{
    Carve c(nullptr);
    c.take<float>(5LL * pl.G.B * pl.G.S);
    c.take<float>(slab_floats(pl.G));
    c.take<float>((long long)pl.G.B * 5 * pl.G.nstrip);
    return (c.off + 255) & ~255LL;
}

static int nchunks(const Plan& pl, int k)
{
    SWEEP_REQUIRE(k >= 1, "elastic2d: checkpoint interval must be >= 1 (got %d)", k);
    return (pl.G.nt + k - 1) / k;
}

struct Ckpt {
    float* f[5];
    float* mem;           // the 8 slabs, x then z, in carve_slabs order
    float* strips;
};

static Ckpt ckpt_at(void* tape, const Plan& pl, int ch)
{
    Carve c(static_cast<char*>(tape) + (long long)(ch - 1) * ckpt_stride(pl));
    Ckpt k{};
    for (int f = 0; f < 5; ++f) k.f[f] = c.take<float>((long long)pl.G.B * pl.G.S);
    k.mem = c.take<float>(slab_floats(pl.G));
    k.strips = c.take<float>((long long)pl.G.B * 5 * pl.G.nstrip);
    return k;
}

// Copy the 8 slabs between a Slabs set and a packed checkpoint range.
static void slabs_copy(const Slabs& s, float* packed, const Geo& G, bool to_packed, cudaStream_t st)
{
    long long o = 0;
    for (int k = 0; k < 8; ++k) {
        float* p = k < 4 ? s.x[k] : s.z[k - 4];
        const long long cnt = k < 4 ? (long long)G.B * G.nz * G.WX : (long long)G.B * G.WZ * G.P;
        if (to_packed) SWEEP_CUDA(cudaMemcpyAsync(packed + o, p, cnt * 4, cudaMemcpyDeviceToDevice, st));
        else SWEEP_CUDA(cudaMemcpyAsync(p, packed + o, cnt * 4, cudaMemcpyDeviceToDevice, st));
        o += cnt;
    }
}

// Strip storage of a memory mode: the step-slot layout of the boundary-saving
// tape (the checkpoint mode keeps its chunk strips as fp32).
static void set_store(Plan& pl, int mem_mode)
{
    pl.host_tape = (mem_mode & SWEEP_MEM_HOST_TAPE) != 0;
    mem_mode &= ~SWEEP_MEM_HOST_TAPE;
    Geo& G = pl.G;
    StripStore& S = G.st;
    S = StripStore{};
    S.fmt = mem_mode == SWEEP_MEM_BOUNDARY_FP16 ? SF_F16
          : mem_mode == SWEEP_MEM_BOUNDARY_BF16 ? SF_BF16
          : mem_mode == SWEEP_MEM_BOUNDARY_INT8 ? SF_I8 : SF_F32;
    auto up = [](long long v, long long a) { return (v + a - 1) / a * a; };
    const long long per = (long long)G.B * 5 * G.nstrip;
    if (S.fmt == SF_F32 || S.fmt == SF_BF16) {
        S.step = up(per * (S.fmt == SF_F32 ? 4 : 2), 256);
        return;
    }
    const int cells[4] = {(M + 1) * G.bw, (M + 1) * G.bw, G.bh * (M + 1), G.bh * (M + 1)};
    const int esz = S.fmt == SF_F16 ? 2 : 1;
    long long off = 0;
    for (int f = 0; f < 4; ++f) {
        S.cells[f] = cells[f];
        S.blocks[f] = (cells[f] + kQB - 1) / kQB;
        S.pay[f] = off;
        off = up(off + 5LL * G.B * cells[f] * esz, 16);
    }
    for (int f = 0; f < 4; ++f) {
        S.scl[f] = off;
        off = up(off + 5LL * G.B * S.blocks[f] * 4, 16);
    }
    S.step = up(off, 256);
}

// tape: one strip slot per step (G.st.step bytes), then the final 5-field
// state (5, B, nz, P)
static int64_t tape_bytes(const Plan& pl)
{
    return (int64_t)pl.G.nt * pl.G.st.step + 5LL * pl.G.B * pl.G.S * 4;
}

static void* tape_slot(const void* tape, const Plan& pl, int it)
{
    return const_cast<char*>(static_cast<const char*>(tape)) + (long long)it * pl.G.st.step;
}

static float* tape_last(void* tape, const Plan& pl)
{
    return static_cast<float*>(tape_slot(tape, pl, pl.G.nt));
}

// CSR of the point events of (shot, tile), like the 2-D acoustic path: the
// tile-local cell and the global event id b * n + s.  Every in-grid cell
// counts (the reference skips only off-grid coordinates, common.cu:24-28).
static int build_events(const Geo& G, const int32_t* loc, int n, int32_t* off, int2* ev, std::vector<int32_t>& fill)
{
    const int ntiles = G.ntx * G.ntz, nkey = G.B * ntiles;
    for (int i = 0; i <= nkey; ++i) off[i] = 0;
    auto key_of = [&](int e) -> int {
        const int ix = loc[2 * e], iz = loc[2 * e + 1];
        if (ix < 0 || ix >= G.nx || iz < 0 || iz >= G.nz) return -1;
        return (e / n) * ntiles + (iz / TZ) * G.ntx + ix / TX;
    };
    for (int e = 0; e < G.B * n; ++e) {
        const int k = key_of(e);
        if (k >= 0) off[k + 1]++;
    }
    for (int i = 1; i <= nkey; ++i) off[i] += off[i - 1];
    fill.assign(off, off + nkey);
    for (int e = 0; e < G.B * n; ++e) {
        const int k = key_of(e);
        if (k < 0) continue;
        const int ix = loc[2 * e], iz = loc[2 * e + 1];
        ev[fill[k]++] = make_int2((iz % TZ) * TX + ix % TX, e);
    }
    return off[nkey];
}

static void setup_common(const sweep_elastic_desc* d, Plan& pl, const Common& w, cudaStream_t st)
{
    Geo& G = pl.G;
    SWEEP_REQUIRE(d->vp && d->vs && d->rho, "elastic2d: null model pointer");
    prep_kernel<<<592, 256, 0, st>>>(d->vp, d->vs, d->rho, pl.nm, d->nz, d->nx, G.P, d->dt,
                                     w.rho, w.lam, w.mu, w.bv, w.vp, w.vs);
    SWEEP_LAUNCH_CHECK();
    std::vector<int32_t> ls((size_t)d->B * d->nsrc * 2 + 1), lr((size_t)d->B * d->nrec * 2 + 1);
    const size_t ns = (size_t)d->B * d->nsrc * 2, nr = (size_t)d->B * d->nrec * 2;
    if (ns) SWEEP_CUDA(cudaMemcpyAsync(ls.data(), d->src_loc, ns * 4, cudaMemcpyDeviceToHost, st));
    if (nr) SWEEP_CUDA(cudaMemcpyAsync(lr.data(), d->rec_loc, nr * 4, cudaMemcpyDeviceToHost, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    const size_t nkey = (size_t)G.B * G.ntx * G.ntz + 1;
    std::vector<int32_t> os(nkey), orr(nkey), fill;
    std::vector<int2> es((size_t)d->B * d->nsrc + 1), er((size_t)d->B * d->nrec + 1);
    const int nsev = build_events(G, ls.data(), d->nsrc, os.data(), es.data(), fill);
    const int nrev = build_events(G, lr.data(), d->nrec, orr.data(), er.data(), fill);
    SWEEP_CUDA(cudaMemcpyAsync(w.src_off, os.data(), nkey * 4, cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaMemcpyAsync(w.rec_off, orr.data(), nkey * 4, cudaMemcpyHostToDevice, st));
    if (nsev) SWEEP_CUDA(cudaMemcpyAsync(w.src_ev, es.data(), nsev * sizeof(int2), cudaMemcpyHostToDevice, st));
    if (nrev) SWEEP_CUDA(cudaMemcpyAsync(w.rec_ev, er.data(), nrev * sizeof(int2), cudaMemcpyHostToDevice, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));   // host staging released on return
    G.src.off = w.src_off; G.src.ev = w.src_ev;
    G.rec.off = w.rec_off; G.rec.ev = w.rec_ev;
    SWEEP_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    G.err = w.err;
}

static void check_err(const Common& w, cudaStream_t st, const char* what)
{
    int h = 0;
    SWEEP_CUDA(cudaMemcpyAsync(&h, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SWEEP_CUDA(cudaStreamSynchronize(st));
    SWEEP_REQUIRE(h == 0, "elastic2d %s: a tile load did not complete in time (code %d); results are invalid", what, h);
}

static CUtensorMap field_map(const float* base, const Geo& G, bool halo)
{
    const uint64_t dims[3] = {(uint64_t)G.nx, (uint64_t)G.nz, (uint64_t)G.B};
    const uint64_t strides[2] = {(uint64_t)G.P, (uint64_t)G.S};
    const uint32_t box[3] = {(uint32_t)(halo ? HX : TX), (uint32_t)(halo ? HZ : TZ), 1u};
    return tma::make_map(base, 3, dims, strides, box);
}

static FwdMaps fwd_maps(float* const* f, const Geo& G)
{
    FwdMaps m;
    for (int k = 0; k < 5; ++k) {
        m.halo[k] = field_map(f[k], G, true);
        m.tile[k] = field_map(f[k], G, false);
    }
    return m;
}

static Models models_of(const Common& w)
{
    return Models{w.rho, w.lam, w.mu, w.bv, w.vp, w.vs};
}

constexpr size_t SM_FWD_VEL = sizeof(VelSmem);
constexpr size_t SM_FWD_STR = sizeof(StrSmem);

static void set_attrs()
{
    static bool done = false;
    if (done) return;
    SWEEP_CUDA(cudaFuncSetAttribute(fwd_vel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_FWD_VEL));
    SWEEP_CUDA(cudaFuncSetAttribute(fwd_str<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_FWD_STR));
    SWEEP_CUDA(cudaFuncSetAttribute(fwd_vel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_FWD_VEL));
    SWEEP_CUDA(cudaFuncSetAttribute(fwd_str<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_FWD_STR));
    done = true;
}
constexpr size_t SM_REV_STR = 2 * HN * sizeof(float);
constexpr size_t SM_REV_SADJ = 4 * HN * sizeof(float);
constexpr size_t SM_REV_VADJ = 7 * HN * sizeof(float);

static void check_mode(int mem_mode, int ckpt_every)
{
    if (mem_mode & SWEEP_MEM_HOST_TAPE) {
        mem_mode &= ~SWEEP_MEM_HOST_TAPE;
        SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT && mem_mode != SWEEP_MEM_RECURSIVE,
                      "elastic2d: a host tape goes with boundary saving only");
    }
    SWEEP_REQUIRE(mem_mode == SWEEP_MEM_BOUNDARY || mem_mode == SWEEP_MEM_CHECKPOINT ||
                      mem_mode == SWEEP_MEM_BOUNDARY_FP16 || mem_mode == SWEEP_MEM_BOUNDARY_BF16 ||
                      mem_mode == SWEEP_MEM_BOUNDARY_INT8 || mem_mode == SWEEP_MEM_RECURSIVE,
                  "elastic2d: unknown memory mode %d", mem_mode);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_CHECKPOINT || ckpt_every >= 1,
                  "elastic2d: checkpoint interval must be >= 1 (got %d)", ckpt_every);
    SWEEP_REQUIRE(mem_mode != SWEEP_MEM_RECURSIVE || ckpt_every >= 1,
                  "elastic2d: the recursive checkpoint budget must be >= 1 (got %d)", ckpt_every);
}

void schedule_of(const sweep_elastic_desc* d, sweep_b200_schedule* out)
{
    const Plan pl = make_plan(d);
    out->shots_fwd = pl.G.gf;
    out->shots_rev = pl.gshots;
    out->z_chunks = 0;
    out->graph_steps = pl.graph_steps;
    out->tile_y = 0;
}

void sizes(const sweep_elastic_desc* d, int mem_mode, int ckpt_every, int64_t* ws, int64_t* tape)
{
    check_mode(mem_mode, ckpt_every);
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    Carve cf(nullptr);
    FwdWs fw{};
    carve_fwd(cf, pl, fw);
    Carve cr(nullptr);
    RevWs rw{};
    if (mem_mode == SWEEP_MEM_CHECKPOINT) {
        carve_rev_ckpt(cr, pl, ckpt_every, rw);
        *tape = (int64_t)std::max(nchunks(pl, ckpt_every) - 1, 1) * ckpt_stride(pl);
    } else if (mem_mode == SWEEP_MEM_RECURSIVE) {
        carve_rev_ckpt(cr, pl, SWEEP_RECURSIVE_LEAF, rw);
        cr.take<char>((long long)ckpt_every * ckpt_stride(pl));         // the snapshot slots
        *tape = 256;                                                     // nothing is kept
    } else {
        carve_rev(cr, pl, rw);
        *tape = tape_bytes(pl);
    }
    *ws = std::max(cf.off, cr.off);
}

// Forward steps [it0, it1) on the fields / memories of A; strips_of(it) is
// the strip slot of step it (null: none).
template <class StripsOf>
static void forward_steps(FwdArgs& A, int it0, int it1, StripsOf strips_of, float* scratch, cudaStream_t st,
                          int graph_steps, HostRing* hr = nullptr)
{
    StepGraphs gs(st, hr ? 0 : graph_steps);
    const Geo& G = A.G;
    set_attrs();
    const FwdMaps maps = fwd_maps(A.f, G);
    const dim3 grid(G.ntx * G.ntz, (G.B + G.gf - 1) / G.gf), block(TX, 8);
    const bool scaled = G.st.fmt == SF_F16 || G.st.fmt == SF_I8;
    const unsigned qblocks = (unsigned)(5 * G.B * (G.st.blocks[0] + G.st.blocks[1] + G.st.blocks[2] + G.st.blocks[3]));
    for (int it = it0; it < it1; ++it) {
        A.it = it;
        void* slot = strips_of(it);
        A.strips = (slot && scaled) ? static_cast<void*>(scratch) : slot;
        const cudaStream_t ls = gs.stream();
        if (G.fs) fwd_vel<true><<<grid, block, SM_FWD_VEL, ls>>>(maps, A);
        else fwd_vel<false><<<grid, block, SM_FWD_VEL, ls>>>(maps, A);
        if (slot && hr) hr->before_write(it);
        if (G.fs) fwd_str<true><<<grid, block, SM_FWD_STR, ls>>>(maps, A);
        else fwd_str<false><<<grid, block, SM_FWD_STR, ls>>>(maps, A);
        if (G.nvf) vsrc_forward<<<G.B, 128, 0, ls>>>(G, A.f[VX], A.f[VZ], A.strips, A.record, it);
        if (slot && scaled) quantize_strips<<<qblocks, kQB, 0, ls>>>(G, scratch, slot);
        if (slot && hr) hr->after_write(it);
        SWEEP_LAUNCH_CHECK();
        gs.step_done();
    }
    gs.flush();
}

static void forward_with(const sweep_elastic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape,
                         void* ws, int64_t ws_bytes, cudaStream_t st, StepState* seg, int seg0, int seg1)
{
    // a stepped run covers [seg0, seg1) of the time axis (the fields and CPML
    // memories are updated in place: nothing rotates between segments)
    const bool stepped = seg != nullptr;
    const int a = stepped ? seg0 : 0;
    check_mode(mem_mode, ckpt_every);
    SWEEP_REQUIRE(!stepped || (mem_mode != SWEEP_MEM_CHECKPOINT && mem_mode != SWEEP_MEM_RECURSIVE),
                  "elastic2d stepped forward: boundary saving only");
    SWEEP_REQUIRE(record != nullptr || d->nrec == 0, "elastic2d forward: null record");
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    Carve c(ws);
    FwdWs w{};
    carve_fwd(c, pl, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic2d forward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    if (a == 0) {
        SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
        if (record && d->nrec)
            SWEEP_CUDA(cudaMemsetAsync(record, 0, sizeof(float) * (size_t)d->B * d->nt * d->nrec * d->nrec_fields,
                                       st));
    }
    setup_common(d, pl, w.cm, st);
    FwdArgs A{};
    A.G = pl.G;
    A.m = models_of(w.cm);
    for (int k = 0; k < 5; ++k) A.f[k] = w.f[k];
    A.mem = w.mem;
    A.record = record;
    const Geo& G = pl.G;
    const long long n = (long long)G.B * G.S;
    if (mem_mode == SWEEP_MEM_RECURSIVE) tape = nullptr;     // the backward replays from the initial state
    if (mem_mode != SWEEP_MEM_CHECKPOINT) {
        HostRing hr;
        const bool host = tape && pl.host_tape;
        const int b = stepped ? seg1 : G.nt;
        if (host) hr.open(w.ring, tape, G.st.step, st);
        forward_steps(A, a, b,
                      [&](int it) { return !tape ? nullptr : host ? hr.slot(it) : tape_slot(tape, pl, it); },
                      w.scratch, st, pl.graph_steps, host ? &hr : nullptr);
        if (host) hr.close();
        if (tape && b == G.nt) {
            float* last = tape_last(tape, pl);
            for (int k = 0; k < 5; ++k)
                SWEEP_CUDA(cudaMemcpyAsync(last + k * n, w.f[k], sizeof(float) * n, cudaMemcpyDefault, st));
        }
        check_err(w.cm, st, "forward");
        return;
    }
    const int k = ckpt_every, C = nchunks(pl, k);
    for (int ch = 0; ch < C; ++ch) {
        const int it0 = ch * k, it1 = std::min(G.nt, it0 + k);
        if (tape && ch >= 1) {
            const Ckpt cp = ckpt_at(tape, pl, ch);
            for (int f = 0; f < 5; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(cp.f[f], w.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
            slabs_copy(w.mem, cp.mem, G, true, st);
        }
        // the last step of a chunk keeps its strips with the next checkpoint
        forward_steps(A, it0, it1,
                      [&](int it) { return (tape && it == it1 - 1 && ch + 1 < C) ? ckpt_at(tape, pl, ch + 1).strips : nullptr; },
                      nullptr, st, pl.graph_steps);
    }
    check_err(w.cm, st, "forward");
}

static void backward_with(const sweep_elastic_desc* d, int mem_mode, int ckpt_every, const float* adj,
                          const void* tape, float* grad_vp, float* grad_vs, float* grad_rho, void* ws,
                          int64_t ws_bytes, cudaStream_t st, StepState* seg, int bw0, int bw1)
{
    // a stepped run reverses [bw1, bw0) top down, continuing seg's state
    const bool stepped = seg != nullptr;
    const int top = stepped ? bw0 : d->nt, bottom = stepped ? bw1 : 0;
    const bool first = top == d->nt;
    check_mode(mem_mode, ckpt_every);
    SWEEP_REQUIRE(tape != nullptr, "elastic2d backward: null tape");
    SWEEP_REQUIRE(grad_vp && grad_vs && grad_rho, "elastic2d backward: null gradient output");
    SWEEP_REQUIRE(adj != nullptr || d->nrec == 0, "elastic2d backward: null adjoint source");
    const bool ckpt = mem_mode == SWEEP_MEM_CHECKPOINT;
    const bool recursive = mem_mode == SWEEP_MEM_RECURSIVE;
    SWEEP_REQUIRE(!stepped || (!ckpt && !recursive), "elastic2d stepped backward: boundary saving only");
    Plan pl = make_plan(d);
    set_store(pl, mem_mode);
    Carve c(ws);
    RevWs w{};
    char* snaps = nullptr;
    if (ckpt) carve_rev_ckpt(c, pl, ckpt_every, w);
    else if (recursive) {
        carve_rev_ckpt(c, pl, SWEEP_RECURSIVE_LEAF, w);
        snaps = c.take<char>((long long)ckpt_every * ckpt_stride(pl));
    } else carve_rev(c, pl, w);
    SWEEP_REQUIRE(ws != nullptr && c.off <= ws_bytes, "elastic2d backward: workspace too small (%lld < %lld bytes)",
                  (long long)ws_bytes, (long long)c.off);
    if (first) SWEEP_CUDA(cudaMemsetAsync(w.zero0, 0, w.zero1 - w.zero0, st));
    setup_common(d, pl, w.cm, st);
    const Geo& G = pl.G;
    const long long n = (long long)G.B * G.S;
    RevArgs A{};
    A.G = G;
    A.m = models_of(w.cm);
    for (int k = 0; k < 5; ++k) { A.f[k] = w.f[k]; A.a[k] = w.a[k]; }
    A.cvx = w.cvx; A.cvz = w.cvz;
    A.adj = adj;
    A.gvp = w.gvp; A.gvs = w.gvs; A.grho = w.grho;
    A.G_shots = pl.gshots;
    const dim3 block(TX, 8);
    const dim3 grid_s(G.ntx * G.ntz, pl.nslot), grid_b(G.ntx * G.ntz, G.B);
    int cur = stepped && !first ? seg->idx[0] : 0;
    // Reverse steps it1 - 1 .. max(it0, 1) (the staggered reverse has no
    // it = 0 step) on the reconstruction state after step it1 - 1;
    // strips_of(t) holds the strips of the state after step t.
    HostRing hr;
    const bool host = pl.host_tape && !ckpt && !recursive;
    auto reverse = [&](int it0, int it1, auto strips_of) {
        StepGraphs gs(st, host ? 0 : pl.graph_steps);
        for (int it = it1 - 1; it >= std::max(it0, 1); --it) {
            A.it = it;
            A.strips = strips_of(it - 1);
            A.mo = w.m[cur];
            A.mn = w.m[cur ^ 1];
            if (host) hr.before_read(it - 1);
            const cudaStream_t ls = gs.stream();
            if (G.nvf)
                vsrc_reverse<<<G.B, 128, 0, ls>>>(G, A.a[VX], A.a[VZ], A.f[VX], A.f[VZ], A.grho, A.m.rho, A.G_shots, it);
            if (G.fs) {
                rev_str<true><<<grid_s, block, SM_REV_STR, ls>>>(A);
                rev_sadj<true><<<grid_b, block, SM_REV_SADJ, ls>>>(A);
                rev_vadj<true><<<grid_b, block, SM_REV_VADJ, ls>>>(A);
            } else {
                rev_str<false><<<grid_s, block, SM_REV_STR, ls>>>(A);
                rev_sadj<false><<<grid_b, block, SM_REV_SADJ, ls>>>(A);
                rev_vadj<false><<<grid_b, block, SM_REV_VADJ, ls>>>(A);
            }
            if (host) {
                hr.after_read(it - 1);
                if (it - 1 - HostRing::R >= std::max(it0 - 1, 0)) hr.fetch(it - 1 - HostRing::R, true);
            }
            SWEEP_LAUNCH_CHECK();
            gs.step_done();
            cur ^= 1;
        }
        gs.flush();
    };
    if (recursive) {
        // Recursive checkpointing (SWEEP_MEM_RECURSIVE): the bisection of the
        // acoustic drivers (acoustic2d.cu backward_recursive); a snapshot slot
        // is the checkpoint layout (five fields, eight CPML slabs, strips of the
        // step before), the replay runs straight into the reconstruction fields
        // as in the checkpoint mode, leaves are SWEEP_RECURSIVE_LEAF steps.
        const int L = SWEEP_RECURSIVE_LEAF, count = ckpt_every;
        const long long cs = (long long)G.B * 5 * G.nstrip;
        FwdArgs F{};
        F.G = G;
        F.m = A.m;
        for (int f = 0; f < 5; ++f) F.f[f] = w.f[f];
        F.mem = w.fmem;
        F.record = nullptr;
        auto restore = [&](int k) {
            if (k < 0) {
                for (int f = 0; f < 5; ++f) SWEEP_CUDA(cudaMemsetAsync(w.f[f], 0, sizeof(float) * n, st));
                for (int s2 = 0; s2 < 4; ++s2) {
                    SWEEP_CUDA(cudaMemsetAsync(w.fmem.x[s2], 0, sizeof(float) * G.B * G.nz * G.WX, st));
                    SWEEP_CUDA(cudaMemsetAsync(w.fmem.z[s2], 0, sizeof(float) * G.B * G.WZ * G.P, st));
                }
            } else {
                const Ckpt cp = ckpt_at(snaps, pl, k + 1);
                for (int f = 0; f < 5; ++f)
                    SWEEP_CUDA(cudaMemcpyAsync(w.f[f], cp.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
                slabs_copy(w.fmem, cp.mem, G, false, st);
            }
        };
        auto save = [&](int k) {
            const Ckpt cp = ckpt_at(snaps, pl, k + 1);
            for (int f = 0; f < 5; ++f)
                SWEEP_CUDA(cudaMemcpyAsync(cp.f[f], w.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
            slabs_copy(w.fmem, cp.mem, G, true, st);
        };
        auto strips_from = [&](int k) {        // strips of the step before snapshot k into chunk slot 0
            SWEEP_CUDA(cudaMemcpyAsync(w.chunk, ckpt_at(snaps, pl, k + 1).strips, sizeof(float) * cs,
                                       cudaMemcpyDeviceToDevice, st));
        };
        auto leaf = [&](int a, int e) {
            forward_steps(F, a, e, [&](int it) { return w.chunk + (long long)(it - a + 1) * cs; }, nullptr, st,
                          pl.graph_steps);
            reverse(a, e, [&](int t) { return (const float*)w.chunk + (long long)(t - (a - 1)) * cs; });
        };
        std::function<void(int, int, int, int)> process = [&](int a, int b, int ka, int free) {
            const int nleaf = (b - a + L - 1) / L;
            if (nleaf <= 1) {
                restore(ka);
                if (a > 0) strips_from(ka);
                leaf(a, b);
                return;
            }
            if (free > 0) {
                const int k = count - free, m = a + L * ((nleaf + 1) / 2);
                restore(ka);
                float* ks = ckpt_at(snaps, pl, k + 1).strips;
                forward_steps(F, a, m, [&](int it) { return it == m - 1 ? ks : nullptr; }, nullptr, st,
                              pl.graph_steps);
                save(k);
                process(m, b, k, free - 1);
                process(a, m, ka, free);
                return;
            }
            for (int c0 = a + (nleaf - 1) * L; c0 >= a; c0 -= L) {
                restore(ka);
                if (c0 > a)
                    forward_steps(F, a, c0, [&](int it) { return it == c0 - 1 ? w.chunk : nullptr; }, nullptr, st,
                                  pl.graph_steps);
                else if (a > 0)
                    strips_from(ka);
                leaf(c0, std::min(b, c0 + L));
            }
        };
        process(0, G.nt, -1, count);
    } else if (!ckpt) {
        if (first) {
            const float* last = tape_last(const_cast<void*>(tape), pl);
            for (int k = 0; k < 5; ++k)
                SWEEP_CUDA(cudaMemcpyAsync(w.f[k], last + k * n, sizeof(float) * n, cudaMemcpyDefault, st));
        }
        if (host) {
            hr.open(w.ring, const_cast<void*>(tape), G.st.step, st);
            for (int t = top - 2; t >= std::max(bottom - 1, 0) && t > top - 2 - HostRing::R; --t) hr.fetch(t, false);
            reverse(bottom, top, [&](int t) { return hr.slot(t); });
            hr.close();
        } else {
            reverse(bottom, top, [&](int t) { return tape_slot(tape, pl, t); });
        }
    } else {
        const int k = ckpt_every, C = nchunks(pl, k);
        void* tp = const_cast<void*>(tape);
        const long long cs = (long long)G.B * 5 * G.nstrip;
        FwdArgs F{};
        F.G = G;
        F.m = A.m;
        for (int f = 0; f < 5; ++f) F.f[f] = w.f[f];     // replay straight into the reconstruction fields
        F.mem = w.fmem;
        F.record = nullptr;
        for (int ch = C - 1; ch >= 0; --ch) {
            const int it0 = ch * k, it1 = std::min(G.nt, it0 + k);
            if (ch == 0) {
                for (int f = 0; f < 5; ++f) SWEEP_CUDA(cudaMemsetAsync(w.f[f], 0, sizeof(float) * n, st));
                for (int s2 = 0; s2 < 4; ++s2) {
                    SWEEP_CUDA(cudaMemsetAsync(w.fmem.x[s2], 0, sizeof(float) * G.B * G.nz * G.WX, st));
                    SWEEP_CUDA(cudaMemsetAsync(w.fmem.z[s2], 0, sizeof(float) * G.B * G.WZ * G.P, st));
                }
            } else {
                const Ckpt cp = ckpt_at(tp, pl, ch);
                for (int f = 0; f < 5; ++f)
                    SWEEP_CUDA(cudaMemcpyAsync(w.f[f], cp.f[f], sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
                slabs_copy(w.fmem, cp.mem, G, false, st);
                SWEEP_CUDA(cudaMemcpyAsync(w.chunk, cp.strips, sizeof(float) * cs, cudaMemcpyDeviceToDevice, st));
            }
            // replay: chunk slot j holds the strips after step it0 - 1 + j
            forward_steps(F, it0, it1, [&](int it) { return w.chunk + (long long)(it - it0 + 1) * cs; }, nullptr, st,
                          pl.graph_steps);
            reverse(it0, it1, [&](int t) { return (const float*)w.chunk + (long long)(t - (it0 - 1)) * cs; });
        }
    }
    if (stepped) seg->idx[0] = cur;
    const int per_shot = G.ms != 0;
    finalize_kernel<<<592, 256, 0, st>>>(w.gvp, pl.nslot, per_shot, G, grad_vp);
    finalize_kernel<<<592, 256, 0, st>>>(w.gvs, pl.nslot, per_shot, G, grad_vs);
    finalize_kernel<<<592, 256, 0, st>>>(w.grho, pl.nslot, per_shot, G, grad_rho);
    SWEEP_LAUNCH_CHECK();
    check_err(w.cm, st, "backward");
}

void forward(const sweep_elastic_desc* d, int mem_mode, int ckpt_every, float* record, void* tape,
             void* ws, int64_t ws_bytes, cudaStream_t st)
{
    forward_with(d, mem_mode, ckpt_every, record, tape, ws, ws_bytes, st, nullptr, 0, 0);
}

void backward(const sweep_elastic_desc* d, int mem_mode, int ckpt_every, const float* adj, const void* tape,
              float* grad_vp, float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st)
{
    backward_with(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_vs, grad_rho, ws, ws_bytes, st, nullptr, 0, 0);
}

void forward_segment(const sweep_elastic_desc* d, int mem_mode, float* record, void* tape, void* ws,
                     int64_t ws_bytes, cudaStream_t st, StepState& seg, int it0, int it1)
{
    forward_with(d, mem_mode, 0, record, tape, ws, ws_bytes, st, &seg, it0, it1);
}

void backward_segment(const sweep_elastic_desc* d, int mem_mode, const float* adj, const void* tape,
                      float* grad_vp, float* grad_vs, float* grad_rho, void* ws, int64_t ws_bytes, cudaStream_t st,
                      StepState& seg, int bw0, int bw1)
{
    backward_with(d, mem_mode, 0, adj, tape, grad_vp, grad_vs, grad_rho, ws, ws_bytes, st, &seg, bw0, bw1);
}

}  // namespace el2d
}  // namespace sweep
