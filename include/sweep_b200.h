/*
 * sweep_b200.h -- C ABI of libsweep_b200.so, the B200 (sm_100a) finite-difference
 * core behind sweep_b200.PropTorch.
 *
 * This boundary replaces the reference's compiled-core entry
 *     int sweep_call(int entry, const void* in, void* out, char* err, int err_cap)
 * (reference src/sweep/csrc/core/capi.h:225) for the entries of the hot path:
 *     acoustic2d 0 forward, 2 backward_bs, 3 backward_ckpt, 4 backward_recursive_ckpt  (capi.h:39-45)
 *     acoustic3d 5 forward, 7 backward_bs, 8 backward_ckpt, 9 backward_recursive_ckpt  (capi.h:46-52)
 *     elastic2d 60 forward, 62 backward_bs, 63 backward_ckpt, 64 backward_recursive_ckpt (capi.h:96-103)
 * with one plain function per (equation family, pass) instead of an entry
 * number, and one POD descriptor instead of the reference's ForwardInputCore /
 * BackwardInputCore Buf structs (reference src/sweep/csrc/core/input_core.h).
 *
 * Conventions shared by every entry point (same as the reference's ABI:
 * capi.h:2-7, buf.h:13-17, capi.cu:578-580):
 *   - the caller allocates EVERY buffer, outputs included; pointers are device
 *     pointers unless stated otherwise; nothing here owns memory;
 *   - fields are float32, shot-major, x fastest: (B, nz, nx) / (B, nz, ny, nx)
 *     on the runtime grid (physical + PML pad + stencil halo M per face);
 *   - coordinates are runtime-grid int32 (x, z) / (x, y, z) per shot; a
 *     coordinate outside the grid is skipped (reference common.cu:24-28);
 *   - records are (B, nt, nrec) -- the canonical (B, nt, nrec, nfield) layout
 *     of the reference's Python API with nfield folded -- and record cotangents
 *     are read in the same layout;
 *   - work is enqueued on `stream` (a cudaStream_t, NULL = legacy default) and
 *     is asynchronous; results are valid in stream order;
 *   - return 0 on success, else non-zero with a NUL-terminated message copied
 *     into err[0..err_cap); nothing is thrown across the boundary.
 */
#ifndef SWEEP_B200_H
#define SWEEP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWEEP_B200_ABI_VERSION 8

#if defined(__GNUC__)
#define SWEEP_B200_API __attribute__((visibility("default")))
#else
#define SWEEP_B200_API
#endif

/* Scalar-wave (acoustic, constant density) problem: 2-D when ndim == 2
 * (ny == 1, the y entries unused), 3-D when ndim == 3.  Replaces the geometry,
 * model and source/receiver fields of the reference's ForwardInputCore
 * (reference src/sweep/backend/c/abi.py:108-166). */
typedef struct sweep_acoustic_desc {
    int32_t ndim;            /* 2 or 3 */
    int32_t B;               /* shots advanced together */
    int32_t nz, ny, nx;      /* runtime grid */
    int32_t nt;              /* time steps */
    int32_t M;               /* stencil half-width (spatial order / 2); 4 */
    int32_t pad[6];          /* PML pad per face: z_lo, z_hi, y_lo, y_hi, x_lo, x_hi */
    float dt, dz, dy, dx;
    float lap[8];            /* lap[1..M]: second-derivative taps (lap[0] unused) */
    float grad[8];           /* grad[1..M]: centred first-derivative taps */
    const float *az, *bz, *dbz;   /* CPML profiles per axis: a, b, d b / d axis */
    const float *ay, *by, *dby;   /* (length nz / ny / nx); y unused in 2-D */
    const float *ax, *bx, *dbx;
    const float* vp;         /* (B|1, cells) velocity on the runtime grid */
    int64_t vp_stride;       /* 0: one model shared by every shot; else cells per shot */
    int32_t nsrc;            /* sources per shot */
    const int32_t* src_loc;  /* (B, nsrc, ndim) */
    const float* wavelet;    /* (B, nsrc, nt) raw amplitudes added to the field */
    int32_t nrec;            /* receivers per shot (padded to a rectangle) */
    const int32_t* rec_loc;  /* (B, nrec, ndim) */
} sweep_acoustic_desc;

/* Memory modes of the backward (reference src/sweep/propagator/options.py:186-246). */
#define SWEEP_MEM_BOUNDARY   0   /* save boundary strips each step; replay them in reverse */
#define SWEEP_MEM_CHECKPOINT 1   /* save state every `ckpt_every` steps; re-run each chunk */
/* Boundary saving with the strips held in fewer bytes (reference
 * BoundarySaving(storage_dtype=...), options.py:194-212; boundarysaver.cu:
 * 906-1100).  Compute stays FP32.  fp16 and int8 quantise each face of the
 * strip set per shot in blocks of 256 cells against the block's max |value|
 * (one FP32 scale per block; elastic: per field); bf16 rounds each value. */
#define SWEEP_MEM_BOUNDARY_FP16 2
#define SWEEP_MEM_BOUNDARY_BF16 3
#define SWEEP_MEM_BOUNDARY_INT8 4
/* OR'ed into a boundary-saving mode (0, 2, 3, 4): `tape` is pinned HOST
 * memory (reference BoundarySaving(storage='cpu'), boundary/runtime.cuh:
 * 91-620); the strips pass through a small device ring in the workspace and a
 * copy stream.  Every equation. */
#define SWEEP_MEM_HOST_TAPE 0x100
/* Recursive checkpointing with a fixed snapshot budget (reference
 * Ckpt(mode='recursive', count=N), options.py:348-370; entries 4 / 9 / 64,
 * capi.h:39-103): the forward keeps no tape; the backward bisects the time
 * axis, holding at most `ckpt_every` = N forward states at once, replays each
 * leaf of SWEEP_RECURSIVE_LEAF steps into its boundary strips and runs the
 * boundary-saving reverse over it.  Leaves fall on multiples of the leaf
 * length, so the gradient equals SWEEP_MEM_CHECKPOINT's with that interval. */
#define SWEEP_MEM_RECURSIVE 5
#define SWEEP_RECURSIVE_LEAF 64

/* Bytes the caller must allocate: `workspace` (scratch, reusable between calls
 * once the previous call has finished on its stream) and `tape` (written by
 * the forward, read by the backward; keep it between the two).  `mem_mode` is
 * one of the SWEEP_MEM_* modes above; `ckpt_every` the checkpoint interval
 * (SWEEP_MEM_CHECKPOINT), the snapshot budget (SWEEP_MEM_RECURSIVE), else
 * ignored.  Host-side only, no device work. */
SWEEP_B200_API int sweep_b200_acoustic_sizes(const sweep_acoustic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                              int64_t* workspace_bytes, int64_t* tape_bytes,
                              char* err, int32_t err_cap);

/* Forward propagation (reference entry 0 / 5: eq_driver.cuh:357-453).
 * record: (B, nt, nrec) out.  tape: NULL for a forward without a later
 * backward, else `tape_bytes` of device memory the backward will read. */
SWEEP_B200_API int sweep_b200_acoustic_forward(const sweep_acoustic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                float* record, void* tape,
                                void* workspace, int64_t workspace_bytes,
                                void* stream, char* err, int32_t err_cap);

/* Adjoint propagation and gradient accumulation (reference entries 2/3/4 and
 * 7/8/9: eq_driver.cuh:721-1135).  adj: (B, nt, nrec) record cotangent.
 * grad_vp: (B|1, cells) on the runtime grid, same stride rule as vp,
 * OVERWRITTEN with d loss / d vp (zero outside the physical box).
 * grad_wavelet: (B, nsrc, nt) overwritten, or NULL.  illum_src / illum_rec:
 * (B|1, cells) overwritten with sum_t u_tt^2 and sum_t lambda^2 over the
 * physical box (reference acoustic2d/kernels.cu:133), or NULL. */
SWEEP_B200_API int sweep_b200_acoustic_backward(const sweep_acoustic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                 const float* adj, const void* tape,
                                 float* grad_vp, float* grad_wavelet,
                                 float* illum_src, float* illum_rec,
                                 void* workspace, int64_t workspace_bytes,
                                 void* stream, char* err, int32_t err_cap);

/* Allocation-free forward (records only) for callers that cannot allocate
 * device memory -- code running where cudaMalloc is not allowed or not wanted
 * (inside another library's memory manager, a loop that must not allocate, a
 * process whose device memory is already handed out).  No counterpart in the
 * reference: it is the 2-D acoustic forward of sweep_b200_acoustic_forward
 * (no tape, no backward) with its scratch in a static 64 MiB array that every
 * GPU loading this library holds until exit.  The caller passes the inputs
 * (d) and the output (record, (B, nt, nrec)).  A problem needing more scratch
 * than the array, or more than 65536 shot-tiles or 32768 sources / receivers,
 * is rejected with an error.  Every call synchronizes its stream (the
 * source / receiver tables go through host memory and the error word is read
 * back), so no call can run under stream capture.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress) with that device
 * current.  The address is kept for the life of the
 * process: cudaDeviceReset after the entry point has been used is not
 * supported.  Every call shares the array: calls that overlap on the GPU
 * race; calls of one process are serialised by one process-wide lock (on
 * every device); each call clears what must start at zero.  Calls no cudaMalloc,
 * cudaFree or other allocating routine on the device. */
SWEEP_B200_API int sweep_b200_acoustic_forward_noalloc(const sweep_acoustic_desc* d, float* record,
                                                       void* stream, char* err, int32_t err_cap);

/* 2-D isotropic elastic problem (velocity-stress, staggered grid).  Replaces
 * the geometry, model and source/receiver fields of the reference's
 * ForwardInputCore for the elastic2d entries (reference
 * src/sweep/backend/c/abi.py:108-166, elastic2d/driver_traits.cuh:110-150).
 * Wavefield indices: 0 vx, 1 vz, 2 sxx, 3 szz, 4 sxz (reference
 * src/sweep/csrc/cuda/common/elastic.h:715-725). */
typedef struct sweep_elastic_desc {
    int32_t B;               /* shots advanced together */
    int32_t nz, nx;          /* runtime grid */
    int32_t nt;              /* time steps */
    int32_t M;               /* stencil half-width (spatial order / 2); 4 */
    int32_t pad[4];          /* PML pad per face: z_lo, z_hi, x_lo, x_hi */
    float dt, dz, dx;
    const float *az, *bz, *azh, *bzh;   /* staggered CPML profiles (length nz): */
    const float *ax, *bx, *axh, *bxh;   /* integer and half-cell positions (nx) */
    const float *vp, *vs, *rho;  /* (B|1, nz, nx) models on the runtime grid */
    int64_t model_stride;    /* 0: models shared by every shot; else nz * nx */
    int32_t nsrc;            /* sources per shot */
    const int32_t* src_loc;  /* (B, nsrc, 2) runtime (x, z) */
    const float* wavelet;    /* (B, nsrc, nt) amplitude added to every source field */
    int32_t nsrc_fields;     /* 1..3 */
    int32_t src_fields[5];   /* wavefield indices the wavelet is added to */
    int32_t nrec;            /* receivers per shot (padded to a rectangle) */
    const int32_t* rec_loc;  /* (B, nrec, 2) */
    int32_t nrec_fields;     /* 1..5 */
    int32_t rec_fields[5];   /* wavefield indices recorded, in record order */
    /* Traction-free faces z_lo, z_hi, x_lo, x_hi (reference PropTorch(
     * free_surface=...) for Elastic: the image method of
     * elastic_free_surface.cuh, the Robertsson sxx correction and szz = 0 on
     * the surface row, elastic2d/kernels.cuh:293-303; the x <-> z swap on a
     * free column, zeroed sxz on a high-side face).  1 = free; a free face
     * has pad 0. */
    int32_t free_surface[4];
} sweep_elastic_desc;

/* Sizes of the elastic workspace and tape (as sweep_b200_acoustic_sizes). */
SWEEP_B200_API int sweep_b200_elastic_sizes(const sweep_elastic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                            int64_t* workspace_bytes, int64_t* tape_bytes,
                                            char* err, int32_t err_cap);

/* Elastic forward (reference entry 60: sg_driver.cuh:291-340).  record:
 * (B, nt, nrec, nrec_fields) out.  tape: NULL (no backward to follow) or
 * `tape_bytes` of device memory for the backward. */
SWEEP_B200_API int sweep_b200_elastic_forward(const sweep_elastic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                              float* record, void* tape,
                                              void* workspace, int64_t workspace_bytes,
                                              void* stream, char* err, int32_t err_cap);

/* Elastic adjoint and vp / vs / rho gradients (reference entry 62:
 * sg_driver.cuh:760-806).  adj: (B, nt, nrec, nrec_fields) record cotangent.
 * grad_vp / grad_vs / grad_rho: (B|1, nz, nx), same stride rule as the
 * models, OVERWRITTEN (zero outside the physical box).  The wavelet gradient
 * is not produced, as in the reference (src/sweep/propagator/_c.py:2368-2374). */
SWEEP_B200_API int sweep_b200_elastic_backward(const sweep_elastic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                               const float* adj, const void* tape,
                                               float* grad_vp, float* grad_vs, float* grad_rho,
                                               void* workspace, int64_t workspace_bytes,
                                               void* stream, char* err, int32_t err_cap);

/* 2-D first-order acoustic VTI problem (reference
 * sweep.equations.AcousticVTI1st, Duveneck et al. 2008; equations/
 * acoustic_vti_1st_2d/): velocities vx, vz and the horizontal / vertical
 * stresses sH, sV on a staggered grid, stiffness c33 = rho vp^2,
 * c11 = c33 (1 + 2 epsilon), c13 = c33 sqrt(1 + 2 delta).  Wavefield
 * indices: 0 vx, 1 vz, 2 sH, 3 sV.  Every even spatial order 2..14; memory:
 * boundary saving with fp32 strips in device memory (SWEEP_MEM_BOUNDARY). */
typedef struct sweep_vti_desc {
    int32_t B;               /* shots advanced together */
    int32_t nz, nx;          /* runtime grid */
    int32_t nt;              /* time steps */
    int32_t M;               /* stencil half-width (spatial order / 2) */
    int32_t pad[4];          /* PML pad per face: z_lo, z_hi, x_lo, x_hi (>= 1) */
    float dt, dz, dx;
    const float *az, *bz, *azh, *bzh;   /* staggered CPML profiles (length nz): */
    const float *ax, *bx, *axh, *bxh;   /* integer and half-cell positions (nx) */
    const float *vp, *epsilon, *delta, *rho;  /* (B|1, nz, nx) models on the runtime grid */
    int64_t model_stride;    /* 0: models shared by every shot; else nz * nx */
    int32_t nsrc;            /* sources per shot */
    const int32_t* src_loc;  /* (B, nsrc, 2) runtime (x, z) */
    const float* wavelet;    /* (B, nsrc, nt) amplitude added to every source field */
    int32_t nsrc_fields;     /* 1..4 */
    int32_t src_fields[4];   /* wavefield indices the wavelet is added to */
    int32_t nrec;            /* receivers per shot (padded to a rectangle) */
    const int32_t* rec_loc;  /* (B, nrec, 2) */
    int32_t nrec_fields;     /* 1..4 */
    int32_t rec_fields[4];   /* wavefield indices recorded, in record order */
} sweep_vti_desc;

/* Sizes of the VTI workspace and tape (as sweep_b200_acoustic_sizes). */
SWEEP_B200_API int sweep_b200_vti_sizes(const sweep_vti_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                        int64_t* workspace_bytes, int64_t* tape_bytes, char* err, int32_t err_cap);

/* VTI forward (reference acoustic_vti_1st_2d/forward.cu).  record:
 * (B, nt, nrec, nrec_fields) out; tape: NULL or `tape_bytes` of device memory. */
SWEEP_B200_API int sweep_b200_vti_forward(const sweep_vti_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                          float* record, void* tape, void* workspace, int64_t workspace_bytes,
                                          void* stream, char* err, int32_t err_cap);

/* VTI adjoint and vp / epsilon / delta / rho gradients (reference
 * acoustic_vti_1st_2d/backward.cu:469-742, boundary saving).  adj:
 * (B, nt, nrec, nrec_fields) record cotangent; the four gradients (B|1, nz, nx),
 * same stride rule as the models, OVERWRITTEN (zero outside the physical box). */
SWEEP_B200_API int sweep_b200_vti_backward(const sweep_vti_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                           const float* adj, const void* tape, float* grad_vp, float* grad_epsilon,
                                           float* grad_delta, float* grad_rho, void* workspace,
                                           int64_t workspace_bytes, void* stream, char* err, int32_t err_cap);

/* 3-D first-order acoustic VTI problem (reference
 * sweep.equations.AcousticVTI1st3D, Duveneck et al. 2008; equations/
 * acoustic_vti_1st_3d/): velocities vx, vy, vz and the horizontal / vertical
 * stresses sH = s11 = s22, sV = s33 on a staggered grid, the 2-D problem's
 * stiffness.  Wavefield indices: 0 vx, 1 vy, 2 vz, 3 sH, 4 sV.  Every even
 * spatial order 2..14; memory: boundary saving with fp32 strips in device
 * memory (SWEEP_MEM_BOUNDARY).  B * nz <= 65535. */
typedef struct sweep_vti3d_desc {
    int32_t B;               /* shots advanced together */
    int32_t nz, ny, nx;      /* runtime grid */
    int32_t nt;              /* time steps */
    int32_t M;               /* stencil half-width (spatial order / 2) */
    int32_t pad[6];          /* PML pad per face: z_lo, z_hi, y_lo, y_hi, x_lo, x_hi (>= 1) */
    float dt, dz, dy, dx;
    const float *az, *bz, *azh, *bzh;   /* staggered CPML profiles per axis: */
    const float *ay, *by, *ayh, *byh;   /* integer and half-cell positions */
    const float *ax, *bx, *axh, *bxh;
    const float *vp, *epsilon, *delta, *rho;  /* (B|1, nz, ny, nx) models on the runtime grid */
    int64_t model_stride;    /* 0: models shared by every shot; else nz * ny * nx */
    int32_t nsrc;            /* sources per shot */
    const int32_t* src_loc;  /* (B, nsrc, 3) runtime (x, y, z) */
    const float* wavelet;    /* (B, nsrc, nt) amplitude added to every source field */
    int32_t nsrc_fields;     /* 1..5 */
    int32_t src_fields[5];   /* wavefield indices the wavelet is added to */
    int32_t nrec;            /* receivers per shot (padded to a rectangle) */
    const int32_t* rec_loc;  /* (B, nrec, 3) */
    int32_t nrec_fields;     /* 1..5 */
    int32_t rec_fields[5];   /* wavefield indices recorded, in record order */
} sweep_vti3d_desc;

/* Sizes, forward (reference acoustic_vti_1st_3d/forward.cu) and backward
 * (acoustic_vti_1st_3d/backward.cu, boundary saving) of the 3-D VTI problem,
 * as the 2-D VTI entries: record (B, nt, nrec, nrec_fields); the four
 * gradients (B|1, nz, ny, nx), OVERWRITTEN, zero outside the physical box. */
SWEEP_B200_API int sweep_b200_vti3d_sizes(const sweep_vti3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                          int64_t* workspace_bytes, int64_t* tape_bytes, char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_vti3d_forward(const sweep_vti3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                            float* record, void* tape, void* workspace, int64_t workspace_bytes,
                                            void* stream, char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_vti3d_backward(const sweep_vti3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                             const float* adj, const void* tape, float* grad_vp, float* grad_epsilon,
                                             float* grad_delta, float* grad_rho, void* workspace,
                                             int64_t workspace_bytes, void* stream, char* err, int32_t err_cap);

/* 3-D isotropic elastic problem (velocity-stress, staggered grid; reference
 * sweep.equations.Elastic3D, entries 66-70: capi.h:105-109,
 * elastic3d/driver_traits.cuh).  Wavefield indices: 0 vx, 1 vy, 2 vz, 3 sxx,
 * 4 syy, 5 szz, 6 sxy, 7 sxz, 8 syz (reference common/elastic.h:736-749).
 * Memory: every SWEEP_MEM_* mode -- boundary saving with fp32 / fp16 / bf16 /
 * int8 strips (entry 67; fp16 and int8 in the reference's per-face layout),
 * the host tape, SWEEP_MEM_CHECKPOINT (entry 68, nine fields and 18 CPML
 * memories per checkpoint) and SWEEP_MEM_RECURSIVE (entry 69). */
typedef struct sweep_elastic3d_desc {
    int32_t B;               /* shots advanced together */
    int32_t nz, ny, nx;      /* runtime grid */
    int32_t nt;              /* time steps */
    int32_t M;               /* stencil half-width (spatial order / 2); 4 */
    int32_t pad[6];          /* PML pad per face: z_lo, z_hi, y_lo, y_hi, x_lo, x_hi */
    float dt, dz, dy, dx;
    const float *az, *bz, *azh, *bzh;   /* staggered CPML profiles per axis: */
    const float *ay, *by, *ayh, *byh;   /* integer and half-cell positions */
    const float *ax, *bx, *axh, *bxh;
    const float *vp, *vs, *rho;  /* (B|1, nz, ny, nx) models on the runtime grid */
    int64_t model_stride;    /* 0: models shared by every shot; else nz * ny * nx */
    int32_t nsrc;            /* sources per shot */
    const int32_t* src_loc;  /* (B, nsrc, 3) runtime (x, y, z) */
    const float* wavelet;    /* (B, nsrc, nt) amplitude added to every source field */
    int32_t nsrc_fields;     /* 1..9 */
    int32_t src_fields[9];   /* wavefield indices the wavelet is added to */
    int32_t nrec;            /* receivers per shot (padded to a rectangle) */
    const int32_t* rec_loc;  /* (B, nrec, 3) */
    int32_t nrec_fields;     /* 1..9 */
    int32_t rec_fields[9];   /* wavefield indices recorded, in record order */
    /* 1: traction-free top face (reference Elastic3D with free_surface=True:
     * the full stencil over image values, Robertsson sxx / syy and szz = 0 on
     * the surface row; common/elastic_free_surface.cuh:723-952); pad[0] = 0. */
    int32_t free_surface;
} sweep_elastic3d_desc;

/* Sizes, forward and backward of the 3-D elastic problem, as the 2-D
 * elastic entries (record (B, nt, nrec, nrec_fields); gradients (B|1, nz, ny,
 * nx), OVERWRITTEN, zero outside the physical box). */
SWEEP_B200_API int sweep_b200_elastic3d_sizes(const sweep_elastic3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                              int64_t* workspace_bytes, int64_t* tape_bytes,
                                              char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_elastic3d_forward(const sweep_elastic3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                                float* record, void* tape,
                                                void* workspace, int64_t workspace_bytes,
                                                void* stream, char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_elastic3d_backward(const sweep_elastic3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                                 const float* adj, const void* tape,
                                                 float* grad_vp, float* grad_vs, float* grad_rho,
                                                 void* workspace, int64_t workspace_bytes,
                                                 void* stream, char* err, int32_t err_cap);

/* BF16 3x3 convolution (stride 1, zero padding 1) as an implicit GEMM on the
 * tensor cores with FP32 accumulation, for the learned FWI preconditioner.
 * No counterpart in the reference (it has no learned component).
 * Activations are NHWC bf16 with c a multiple of 8; 16-byte aligned.
 *   out[p, j] = sum_{t, ch} act[p + sign * off(t), ch] * bt[j, t * c + ch] (+ bias[j])
 * out: (n, h, w, nout) float32.  sign +1 is the forward pass with
 * bt = weights (nout, 3, 3, c); sign -1 is the data gradient with act = the
 * output gradient and bt = the weights transposed per tap to (c_in, 3, 3, c). */
SWEEP_B200_API int sweep_b200_conv3x3_gemm(const void* act, const void* bt, const float* bias, float* out,
                                           int32_t n, int32_t h, int32_t w, int32_t c, int32_t nout,
                                           int32_t sign, void* stream, char* err, int32_t err_cap);

/* Weight gradient of the same convolution: dw (co, 3, 3, c) float32,
 * OVERWRITTEN with sum_p dy[p, o] x[p + off(t), ch]; x (n, h, w, c) and
 * dy (n, h, w, co) bf16, c and co multiples of 8. */
SWEEP_B200_API int sweep_b200_conv3x3_wgrad(const void* x, const void* dy, float* dw, int32_t n, int32_t h,
                                            int32_t w, int32_t c, int32_t co, void* stream, char* err,
                                            int32_t err_cap);

/* Waits for `stream` and reports (then clears) a timed-out tensor-core wait
 * in any convolution launched since the last call: the convolution entries
 * return at launch, so their device-side failures surface here. */
SWEEP_B200_API int sweep_b200_conv3x3_status(void* stream, char* err, int32_t err_cap);

/* Launch schedule of one problem shape.  No counterpart in the reference: its
 * launch shapes are fixed per kernel (reference
 * src/sweep/csrc/cuda/launch/config.h:65-70) and its time loop issues every
 * launch from the host (eq_driver.cuh:357-453).  A schedule is recorded per
 * shape -- equation family, ndim, shots B, runtime grid, PML pads and whether
 * models are per shot; nt, sources and receivers are not part of it -- in a
 * process-wide table behind a mutex, read by every later call of that shape.
 * The autotuner (sweep_b200.autotune) times candidates and records the
 * fastest.  A field left at its "built-in" value keeps the library's default;
 * a per-shot-model problem always runs one shot per CTA. */
typedef struct sweep_b200_schedule {
    int32_t shots_fwd;    /* shots per CTA of the forward step kernels (2-D acoustic
                           * fwd_kernel, elastic fwd_vel / fwd_str); 0 = built-in */
    int32_t shots_rev;    /* shots per CTA of the reverse kernels that sum the image
                           * (2-D acoustic rev_kernel, elastic rev_str); 0 = built-in */
    int32_t z_chunks;     /* 3-D acoustic: z chunks each column block is cut into
                           * (grid depth per shot); 0 = built-in */
    int32_t graph_steps;  /* time steps per captured CUDA graph in the step loops
                           * (0: plain stream launches; < 0: built-in); host-tape
                           * loops always use plain launches */
    int32_t tile_y;       /* 3-D acoustic: rows of the 32-column block a CTA of the
                           * stencil kernels covers, 8 or 16 (0 = built-in 8) */
} sweep_b200_schedule;

#define SWEEP_FAMILY_ACOUSTIC 0   /* desc is a sweep_acoustic_desc (2-D or 3-D) */
#define SWEEP_FAMILY_ELASTIC  1   /* desc is a sweep_elastic_desc */

/* Record `s` as the schedule of the shape of `desc` (replacing any earlier
 * one).  Host-side only, no device work. */
SWEEP_B200_API int sweep_b200_schedule_set(int32_t family, const void* desc, const sweep_b200_schedule* s,
                                           char* err, int32_t err_cap);

/* The schedule a call with `desc` would run, every field resolved (recorded
 * value, else environment override, else built-in default).  Host-side only. */
SWEEP_B200_API int sweep_b200_schedule_get(int32_t family, const void* desc, sweep_b200_schedule* out,
                                           char* err, int32_t err_cap);

/* Forget every recorded schedule.  Host-side only. */
SWEEP_B200_API int sweep_b200_schedule_clear(void);

/* Stepped runners: a pass advanced segment by segment over the time axis
 * (reference src/sweep/csrc/core/capi.h:236-243, sweep_forward_runner_* /
 * sweep_backward_runner_*; eq_driver.cuh:199-453 and 715-925).  A runner is
 * created over a problem and its caller-owned buffers -- descriptor (copied;
 * the arrays it points at), record or gradients, tape, workspace (sized by the
 * *_sizes query) -- which stay valid until destroy; nothing is allocated on
 * the device.  Boundary saving only (every strip format, device or host
 * tape), as the reference's runners.
 *
 * Forward runner: run(it_begin, it_end) advances steps [it_begin, it_end),
 * segments in order from 0 to nt; the record holds every step run so far; the
 * tape is complete once a segment ends at nt.  Backward runner (over that
 * tape and the record cotangent): run(bw_it_begin, bw_it_end) reverses the
 * steps [bw_it_end, bw_it_begin), segments in order from nt down to 0; the
 * gradients (and illuminations) are overwritten after every segment with the
 * contribution of every step reversed so far.  Segments compute what one call
 * computes: the same kernels, in the same order, on the same state.
 * step_phase must be 0: the reference's 1 / 2 split a step around a
 * domain-decomposition halo exchange, which has no counterpart here.  A
 * runner's calls run on its creation device. */
SWEEP_B200_API int sweep_b200_acoustic_forward_runner_create(const sweep_acoustic_desc* d, int32_t mem_mode,
                                                             float* record, void* tape, void* workspace,
                                                             int64_t workspace_bytes, void** handle,
                                                             char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_acoustic_backward_runner_create(const sweep_acoustic_desc* d, int32_t mem_mode,
                                                              const float* adj, const void* tape,
                                                              float* grad_vp, float* grad_wavelet,
                                                              float* illum_src, float* illum_rec,
                                                              void* workspace, int64_t workspace_bytes,
                                                              void** handle, char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_elastic_forward_runner_create(const sweep_elastic_desc* d, int32_t mem_mode,
                                                            float* record, void* tape, void* workspace,
                                                            int64_t workspace_bytes, void** handle,
                                                            char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_elastic_backward_runner_create(const sweep_elastic_desc* d, int32_t mem_mode,
                                                             const float* adj, const void* tape,
                                                             float* grad_vp, float* grad_vs, float* grad_rho,
                                                             void* workspace, int64_t workspace_bytes,
                                                             void** handle, char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_forward_runner_run(void* handle, int32_t it_begin, int32_t it_end,
                                                 int32_t step_phase, void* stream, char* err, int32_t err_cap);
SWEEP_B200_API int sweep_b200_backward_runner_run(void* handle, int32_t bw_it_begin, int32_t bw_it_end,
                                                  int32_t step_phase, void* stream, char* err, int32_t err_cap);
/* The device a runner was created on (-1 for a null handle). */
SWEEP_B200_API int sweep_b200_runner_device_index(void* handle);
/* Releases a runner of either kind (null: no-op). */
SWEEP_B200_API void sweep_b200_runner_destroy(void* handle);

/* Runs the bounded-wait failure path on purpose.  No counterpart in the
 * reference, whose kernels do not wait on barriers.  Every mbarrier wait of
 * this library's step kernels gives up after a fixed budget (about 2 s of SM
 * clock), raises the call's error word and returns, so that a tile load that
 * never lands surfaces as an error return instead of a hung GPU.  This entry
 * launches one CTA that waits, with `budget_cycles` (1 .. that budget), on an
 * mbarrier nothing arrives at (no copy in flight), then reads its error word
 * as the step loops do: it returns non-zero with a "did not complete in time"
 * message.  With `arrive` non-zero the CTA arrives first and the call
 * succeeds.  Allocates nothing; synchronises `stream`. */
SWEEP_B200_API int sweep_b200_wait_selftest(int64_t budget_cycles, int32_t arrive, void* stream,
                                            char* err, int32_t err_cap);

/* ABI version (SWEEP_B200_ABI_VERSION) -- checked by the Python loader, like
 * the reference's sweep_core_abi_version() (reference loader.py:92-138). */
SWEEP_B200_API int sweep_b200_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SWEEP_B200_H */
