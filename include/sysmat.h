/* sysmat: B200-native SPECT system-matrix generator — public C ABI.
 *
 * Two layers of entry points:
 *
 * 1. Reference-compatible entry points.  Same names (where C allows), same argument
 *    meaning, same host-buffer ownership and output layout as the reference programs.
 *    A reference CLI re-linked against libsysmat.so runs unchanged: the C++-mangled
 *    names it links against (PESysMatGen and the three `scatter` overloads) are exported
 *    by csrc/cxx_abi.cpp of the package as aliases of the C entry points below.
 *
 * 2. A native, handle-based API on device pointers and a caller-supplied CUDA stream,
 *    used by the reference-compatible layer, the tests and the benchmark.  It never
 *    calls cudaSetDevice behind the caller's back and never exits the process.
 *
 * Matrix layout everywhere: float dst[detector][voxel], voxel v = ix + Nx*(iy + Ny*iz)
 * (reference PESysMatGen.cu:1025, :1031-1034).  Parameter arrays: float32, 80000
 * (collimator), 80000 (detector), 100 (image), 100 (physics) values, laid out as in the
 * reference (PESysMatGen.cu:961-1075, scatter.cu:1144-1167).
 *
 * Errors: every function returns an int; negative values are SYSMAT_ERR_* codes.
 */
#ifndef SYSMAT_H
#define SYSMAT_H

#if defined(SYSMAT_BUILD)
#define SYSMAT_API __attribute__((visibility("default")))
#else
#define SYSMAT_API
#endif

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SYSMAT_OK 0
#define SYSMAT_ERR_ARG (-1)        /* invalid argument or parameter array */
#define SYSMAT_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define SYSMAT_ERR_CAPACITY (-3)   /* a geometry exceeds a documented capacity */
#define SYSMAT_ERR_IO (-4)         /* a relationship-bitmap file could not be read/written */
#define SYSMAT_ERR_NOMEM (-5)      /* device or host allocation failed */
#define SYSMAT_ERR_TIMEOUT (-6)    /* a bounded device wait gave up */

/* Summation modes of the photoelectric kernel. */
#define SYSMAT_MODE_REFERENCE 0    /* sub-element sum as one float chain in reference order */
#define SYSMAT_MODE_PRECISE 1      /* sub-element sum accumulated in FP64 */
/* The reference's element program evaluated in FP64 from the float parameters (geometry,
 * chords, attenuation, exponentials, solid angle; elliptical holes included); no reference
 * counterpart.  Taken by sysmat_pe, sysmat_pe_csr_file and batched launches. */
#define SYSMAT_MODE_FP64 2
/* The reference's element program in FP32 arithmetic that stays within 1e-5 of its FP64
 * evaluation: large and shared quantities (voxel, crystal and hole positions relative to the
 * ray) are formed in double once per element, hole chords are y-extents in the hole's own
 * frame, the septal length is (T - sum of extents) / cos, crystal and self-attenuation chords
 * are measured from the sub-element, and the sub-element contributions are summed with
 * compensated (Neumaier) summation; an elliptical hole's extent is the unit circle's in its
 * frame scaled by the semi-axes.  No reference counterpart.  Taken by sysmat_pe,
 * sysmat_pe_sampled_mode and sysmat_pe_csr_file. */
#define SYSMAT_MODE_LOCAL 3

/* Scatter parts (bit mask) and collimator solid-angle models. */
#define SYSMAT_SCATTER_CRYSTAL 1
#define SYSMAT_SCATTER_COLLIMATOR 2
#define SYSMAT_HOLE_MODEL_COMBINED 0   /* ScatterGen_RayTracing_CircularHole/scatter.cu:1711-1716 */
#define SYSMAT_HOLE_MODEL_VARIANT 1    /* ScatterGen_Collimator/scatter.cu:1212-1215 */
/* Native collimator scatter (no reference counterpart; see sysmat_scatter_prepare_native). */
#define SYSMAT_HOLE_MODEL_NATIVE 2

/* ---------------------------------------------------------------------------------- */
/* Reference-compatible entry points (host buffers in, host buffers out, synchronous). */

/* Replaces PESysMatGen (PEGen_RayTracing_CircularHole/PESysMatGen.h:4-5, defined at
 * PESysMatGen.cu:1368).  Reads 80000/80000/100 floats; writes D*V floats of the rotation
 * parameter_Image[20] into dst.  Returns V (the number of voxels) or a SYSMAT_ERR_* code.
 * The reference computes in one float chain per element; so does this entry point. */
SYSMAT_API int PESysMatGen(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
                float* dst, int cuda_id);

/* Replaces scatter of the combined program (ScatterGen_RayTracing_CircularHole/scatter.h:4-5,
 * scatter.cu:2013).  PE_SysMat: the D*V photoelectric matrix read from offset 0.  The
 * bitmaps are computed and written to the named files when parameter_Physics[8] / [9]
 * equal 1, else read from them (scatter.cu:2116-2164, :2246-2296).  A file shorter than
 * its bitmap reads its missing words as 0, with a warning on stderr, as the reference's
 * zero-filled buffer does.  Files are read by up to 12 threads through pinned staging
 * memory (32 MB per thread), allocated on the first read on a device and kept for the
 * process.  Writes D*V floats = collimator scatter + crystal scatter.  Returns V or a
 * SYSMAT_ERR_* code. */
SYSMAT_API int scatter(float* parameter_Collimator, float* parameter_Detector, float* parameter_Image,
            float* parameter_Physics, float* PE_SysMat, const char* FnameGeoCrystal,
            const char* FnameGeoCollimator, float* dst, int cuda_id);

/* Replaces scatter of the collimator-only program (ScatterGen_Collimator/scatter.h:4-5,
 * scatter.cu:1511): collimator scatter with that program's hole solid angle. */
SYSMAT_API int scatter_collimator(float* parameter_Collimator, float* parameter_Detector,
                       float* parameter_Image, float* parameter_Physics, float* PE_SysMat,
                       const char* FnameGeo, float* dst, int cuda_id);

/* Replaces scatter of the crystal-only program (ScatterGen_Crystal/scatter.h:4-5,
 * scatter.cu:1528): inter-crystal scatter only. */
SYSMAT_API int scatter_crystal(float* parameter_Detector, float* parameter_Image, float* parameter_Physics,
                    float* PE_SysMat, const char* FnameGeo, float* dst, int cuda_id);

/* ---------------------------------------------------------------------------------- */
/* Native API.  The caller makes `device` current before every call that takes a ctx.   */

typedef struct sysmat_ctx sysmat_ctx;

/* Parse and upload one system.  pC/pD/pI/pP are host arrays of 80000/80000/100/100
 * floats (pC may be NULL for crystal-only use, pP may be NULL for PE-only use).  Derived
 * per-crystal and per-hole tables are computed on the device. */
SYSMAT_API int sysmat_create(sysmat_ctx** out, int device, const float* pC, const float* pD,
                  const float* pI, const float* pP);
SYSMAT_API int sysmat_destroy(sysmat_ctx* ctx);

/* Geometry sizes: D, V (all voxels), holes of layer 0, total holes, layers. */
SYSMAT_API int sysmat_dims(const sysmat_ctx* ctx, int* n_det, long long* n_vox, int* n_holes0,
                int* n_holes, int* n_layers);

/* Photoelectric matrix block for one rotation index: detectors [det_begin,
 * det_begin+det_count) x voxels [vox_begin, vox_begin+vox_count), written to d_out with
 * row stride ld (floats).  mode: SYSMAT_MODE_*.  Asynchronous on `stream`
 * (cudaStream_t; NULL = legacy default stream). */
SYSMAT_API int sysmat_pe(sysmat_ctx* ctx, float rotation, int det_begin, int det_count, long long vox_begin,
              long long vox_count, float* d_out, long long ld, int mode, void* stream);

/* Photoelectric block in the sampled form.  No reference counterpart: the reference divides
 * every crystal into 8 x 16 x 8 sub-elements and uses one source point, the voxel centre
 * (PESysMatGen.cu:1196-1217, :1031-1034).  crystal_div[3]: sub-elements along x, depth (y)
 * and z (each 1..SYSMAT_SAMPLED_MAX_DIV, product <= SYSMAT_SAMPLED_MAX_SUBELEMENTS);
 * voxel_sub[3]: source points along x, y and z on the centres of a grid over the voxel (each
 * 1..SYSMAT_SAMPLED_MAX_SUB, product <= SYSMAT_SAMPLED_MAX_POINTS).  The element is the mean
 * over the source points of the reference's element at that point with that division, every
 * sub-element contribution summed in FP64; {8,16,8} with {1,1,1} runs SYSMAT_MODE_PRECISE's
 * float program, compiled separately (measured within 1.5e-5 relative of it, the largest
 * differences on heavily attenuated elements).  Blocks, strides and errors as sysmat_pe. */
#define SYSMAT_SAMPLED_MAX_DIV 64
#define SYSMAT_SAMPLED_MAX_SUBELEMENTS 4096
#define SYSMAT_SAMPLED_MAX_SUB 8
#define SYSMAT_SAMPLED_MAX_POINTS 64
SYSMAT_API int sysmat_pe_sampled(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                 long long vox_begin, long long vox_count, const int* crystal_div,
                                 const int* voxel_sub, float* d_out, long long ld, void* stream);

/* The sampled form in a chosen arithmetic: SYSMAT_MODE_PRECISE (the reference's float program,
 * exactly what sysmat_pe_sampled computes) or SYSMAT_MODE_LOCAL (the local-coordinate FP32 form
 * of SYSMAT_MODE_LOCAL at each source point, contributions summed with compensation: within 1e-5
 * of the sampled form's FP64 evaluation).  Other arguments and errors as sysmat_pe_sampled. */
SYSMAT_API int sysmat_pe_sampled_mode(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                      long long vox_begin, long long vox_count, const int* crystal_div,
                                      const int* voxel_sub, int mode, float* d_out, long long ld, void* stream);

/* Relationship bitmaps in the reference's word layout (scatter.cu:1040-1074).
 * Word counts: crystal ceil(D(D+1)/2*D/32), collimator ceil(H0*D*D/32). */
SYSMAT_API long long sysmat_bitmap_crystal_words(const sysmat_ctx* ctx);
SYSMAT_API long long sysmat_bitmap_collimator_words(const sysmat_ctx* ctx);
SYSMAT_API int sysmat_bitmap_crystal(sysmat_ctx* ctx, uint32_t* d_words, void* stream);
SYSMAT_API int sysmat_bitmap_collimator(sysmat_ctx* ctx, uint32_t* d_words, void* stream);

/* Build the scatter path's per-(scatterer, detector) pair tables from relationship bitmaps
 * (as produced above or loaded from the reference's files).  parts: SYSMAT_SCATTER_* mask;
 * the bitmap of a part that is not requested may be NULL.  Synchronises `stream` once.
 * The tables stay valid until the next prepare or sysmat_destroy. */
SYSMAT_API int sysmat_scatter_prepare(sysmat_ctx* ctx, int parts, const uint32_t* d_bm_crystal,
                                      const uint32_t* d_bm_collimator, void* stream);

/* Pair tables of the native scatter model, which fixes three simplifications of the reference's
 * collimator scatter (scatter.cu:1544-1936): the holes of every layer are scatter points (the
 * reference uses layer 0 only, H0 = Params_Collimator[10]), each weighted with its own layer's
 * mu_C / mu_total (the reference uses layer 0's, scatter.cu:1716), and the scattered photon is
 * attenuated by the tungsten between the hole and the crystal (plate chords minus hole chords
 * per layer, mu_pe and mu_C rescaled to the scattered energy as for crystals; the reference
 * ignores it).  The crystal part is the reference's.  The collimator-scatter attenuators come
 * from the reference's relationship predicate evaluated for every hole (no bitmap file).
 * Use with hole_model SYSMAT_HOLE_MODEL_NATIVE; synchronises `stream` once. */
SYSMAT_API int sysmat_scatter_prepare_native(sysmat_ctx* ctx, int parts, const uint32_t* d_bm_crystal, void* stream);

/* Primary Compton scatter with scatter points on a grid (no reference counterpart; the
 * reference scatters at one point per crystal centre and one per layer-0 hole centre,
 * ScatterGen_RayTracing_CircularHole/scatter.cu:1218-1223, :1707-1716).  Scatter points are
 * the centres of cells of side `cell` mm (0.25 for the configurations here) inside every
 * crystal (parts bit SYSMAT_SCATTER_CRYSTAL; weight = the cell's photoelectric contribution
 * from the voxel in the local-coordinate FP32 form times mu_C / mu_pe) and inside the
 * tungsten of every collimator layer (bit SYSMAT_SCATTER_COLLIMATOR; weight = V / (4 pi r^2)
 * exp(-attenuation to the cell) mu_C).  Each item is the reference's scatter item with that
 * scatter point, every crystal on the way (and the tungsten, for septal points) as
 * attenuator at the scattered energy, and the exact Klein-Nishina fraction; each element
 * sums its ~10^6 items in FP64.  Every crystal must have the same cell division.  Elliptical
 * holes (sysmat_set_hole_shapes) bound the septal cells and the hole media by their ellipses.
 * Needs no PE matrix or bitmaps.  Synchronous on `stream` (it allocates and frees its
 * scratch). */
/* Batched scatter (no reference counterpart; the reference computes one geometry per call,
 * scatter.cu:2169-2194, :2303-2329): many scatter tasks, each what one sysmat_scatter call
 * takes, in one persistent launch over a work queue, replayed as a CUDA graph.  Every element
 * equals the per-task sysmat_scatter element bit for bit.  The plan keeps pointers to the
 * contexts' pair tables, PE matrices and outputs: keep them alive and prepared as they were at
 * creation while the plan is used.  Creation may synchronise `stream` once (Klein-Nishina
 * tables); runs are asynchronous on `stream`. */
typedef struct sysmat_scatter_item {
    int ctx;                 /* index into the ctxs array */
    int parts;               /* SYSMAT_SCATTER_* bits */
    int hole_model;          /* SYSMAT_HOLE_MODEL_* (as prepared) */
    float rotation;
    const float* d_pe;       /* the rotation's PE matrix (D x V), for the crystal part */
    int det_begin, det_count;
    long long vox_begin, vox_count;
    float* d_out;
    long long ld;
} sysmat_scatter_item;

typedef struct sysmat_scatter_plan sysmat_scatter_plan;

SYSMAT_API int sysmat_scatter_batch_create(sysmat_scatter_plan** plan, sysmat_ctx* const* ctxs, int n_ctx,
                                           const sysmat_scatter_item* items, int n_items, void* stream);
SYSMAT_API int sysmat_scatter_batch_run(sysmat_scatter_plan* plan, void* stream);
SYSMAT_API int sysmat_scatter_batch_destroy(sysmat_scatter_plan* plan);

SYSMAT_API int sysmat_scatter_grid(sysmat_ctx* ctx, int parts, float cell, float rotation, int det_begin,
                                   int det_count, long long vox_begin, long long vox_count, float* d_out,
                                   long long ld, void* stream);

/* Primary-Compton scatter block (parts must have been prepared).  d_pe: the D x V
 * photoelectric matrix (row stride V) the crystal part reads.  hole_model:
 * SYSMAT_HOLE_MODEL_*.  With both parts the result is float(collimator) + float(crystal),
 * as the reference sums on the host (scatter.cu:2354-2357). */
SYSMAT_API int sysmat_scatter(sysmat_ctx* ctx, int parts, int hole_model, float rotation,
                              const float* d_pe, int det_begin, int det_count, long long vox_begin,
                              long long vox_count, float* d_out, long long ld, void* stream);

/* Elliptical holes (an extension: the reference defines length_ellipticalcylinder_ray,
 * PESysMatGen.cu:801-947, but its kernels never call it and its parameter files have no
 * field for it).  Host arrays of n_holes values: hole h is the cylinder
 * ((x'-x)/rho_x)^2 + ((z'-z)/rho_z)^2 <= 1 in its frame rotated by theta[h] (radians), with
 * the reference's chord; rho_x[h] <= 0 keeps it circular.  The hole's radius field in
 * Params_Collimator must bound both semi-axes (the reference cone test and the kernel's
 * filters use it).  rho_x = NULL restores circular holes.  Applies to sysmat_pe (and the
 * entry points built on it), to the projection entry points and their vector-Jacobian
 * product, and to batch plans created afterwards. */
SYSMAT_API int sysmat_set_hole_shapes(sysmat_ctx* ctx, const float* rho_x, const float* rho_z, const float* theta);

/* Whole photoelectric matrix of rotation `rotation` written to `path` in compressed form
 * (entries > threshold), computed and compressed on the device in blocks of rows_per_block
 * detector rows (0: about 1 GB of dense block) and streamed to the file.  The reference CLI
 * writes the dense D*V floats instead (PEGen_CircularHole.cpp:141-147).  File layout:
 * "SMCSR001", int64 rows, int64 cols, float threshold, int32 mode, int64 reserved; then
 * blocks of (int64 first_row, int64 n_rows, int64 nnz, int64 row_ptr[n_rows+1], int64
 * col[nnz], float val[nnz]).  *nnz_total (may be NULL) receives the total.  Synchronous on
 * `stream`; allocates its block buffers for the duration of the call. */
SYSMAT_API int sysmat_pe_csr_file(sysmat_ctx* ctx, float rotation, const char* path, float threshold, int mode,
                                  int rows_per_block, long long* nnz_total, void* stream);

/* ---- Batched photoelectric launches --------------------------------------------------------
 * Many (system, rotation, block) tasks in one persistent launch over a device work queue.
 * No reference counterpart: the reference computes one rotation of one system per call
 * (PESysMatGen.cu:1368-1437).  Every context of a plan must live on the current device. */
typedef struct sysmat_batch_item {
    int ctx;                    /* index into the context array of the plan */
    float rotation;             /* rotation index, as Params_Image[20] */
    int det_begin, det_count;   /* detector rows */
    long long vox_begin, vox_count;   /* voxels (flat index ix + Nx*(iy + Ny*iz)) */
    float* d_out;               /* device block of det_count rows, row stride ld floats */
    long long ld;
} sysmat_batch_item;

typedef struct sysmat_batch_plan sysmat_batch_plan;

/* Validate the items (each block as sysmat_pe checks it) and upload the work queue.  The
 * plan keeps pointers to the contexts' device tables: destroy it before them.  It takes each
 * context's hole shapes (sysmat_set_hole_shapes) as they are when the plan is created. */
SYSMAT_API int sysmat_batch_create(sysmat_batch_plan** plan, sysmat_ctx* const* ctxs, int n_ctx,
                                   const sysmat_batch_item* items, int n_items);
/* Voxel brick of one work item (bx*by*bz <= 512) and resident blocks per SM (0 = all that fit). */
SYSMAT_API int sysmat_batch_set_tiles(sysmat_batch_plan* plan, int bx, int by, int bz, int blocks_per_sm);
/* tiles[4] = bx, by, bz, blocks_per_sm currently in use. */
SYSMAT_API int sysmat_batch_get_tiles(const sysmat_batch_plan* plan, int* tiles);
/* Time candidate bricks on a probe subset of the batch (synchronises `stream`), keep the
 * fastest and return it in tiles[4] (may be NULL). */
SYSMAT_API int sysmat_batch_tune(sysmat_batch_plan* plan, int mode, void* stream, int* tiles);
/* Run the whole batch on `stream` (asynchronous) in `mode` (SYSMAT_MODE_REFERENCE, _PRECISE,
 * _FP64 or _LOCAL; every element equals sysmat_pe's in that mode).  The first run per mode
 * captures the launch into a CUDA graph on a plan-owned stream; later runs replay it. */
SYSMAT_API int sysmat_batch_run(sysmat_batch_plan* plan, int mode, void* stream);
SYSMAT_API int sysmat_batch_destroy(sysmat_batch_plan* plan);
/* One-shot: create, run once without a graph, synchronise `stream`, destroy. */
SYSMAT_API int sysmat_batch(sysmat_ctx* const* ctxs, int n_ctx, const sysmat_batch_item* items, int n_items,
                            int mode, void* stream);

/* ---- Forward projection and its adjoint -----------------------------------------------------
 * No reference counterpart: the reference only writes the dense matrix.  Both functions cover
 * every voxel of rotation `rotation` and detector rows [det_begin, +det_count), recompute A
 * brick by brick (nothing of A is stored) and skip voxels with x = 0.  Asynchronous on
 * `stream`; calls on one context share its work counter, so issue them on one stream.
 *
 * theta, the parameters of the derivative, in this order:
 *   0 mu_W        total attenuation of every collimator layer (Params_Collimator[(m+1)*10+5])
 *   1 mu_crystal  total attenuation of every crystal (Params_Detector[12d+7]; mu_pe held fixed)
 *   2 radius      radius of every hole (Params_Collimator[100+9h+4])
 *   3 dx          shift of every hole centre along x
 *   4 dy          shift of every hole's caps and every layer plane along y
 *   5 dz          shift of every hole centre along z
 *   6 tilt        rotation of the hole pattern about the y axis, radians
 *                 (x' = x cos t - z sin t, z' = x sin t + z cos t); it turns the frame of an
 *                 elliptical hole with the pattern (theta[h] + t)
 * Thresholds of the reference's program (plate penalty, eps cut-offs) are piecewise constant
 * and contribute nothing to the derivative.  An elliptical hole's chord does not read the
 * radius field (which only bounds the ellipse), so such holes add nothing to the radius
 * partial. */
#define SYSMAT_THETA_N 7

/* d_p[i] = sum_v A[det_begin + i, v] * d_x[v] in double (precise-mode elements).
 * d_x: n_vox floats; d_p: det_count doubles, overwritten. */
SYSMAT_API int sysmat_project(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                              const float* d_x, double* d_p, void* stream);

/* Vector-Jacobian product of the projection: with u = d_u (det_count floats, the cotangent of
 * d_p), d_grad[k] = sum_{i,v} u[i] x[v] dA[det_begin + i, v]/dtheta_k for k < SYSMAT_THETA_N,
 * and d_grad[SYSMAT_THETA_N] = u^T A x.  d_grad: SYSMAT_THETA_N + 1 doubles, overwritten.
 * For loss = |A x - y|^2 pass u = 2 (A x - y). */
SYSMAT_API int sysmat_vjp(sysmat_ctx* ctx, float rotation, int det_begin, int det_count, const float* d_x,
                          const float* d_u, double* d_grad, void* stream);

/* Back projection d_q[v] = sum_i A[det_begin + i, v] * d_u[i] (the gradient of u^T A x with
 * respect to x).  d_u: det_count floats; d_q: n_vox doubles, overwritten. */
SYSMAT_API int sysmat_backproject(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                  const float* d_u, double* d_q, void* stream);

/* Photoelectric block like sysmat_pe, for callers that cannot allocate device memory when
 * they call (for example a host that gives all device memory to its own pool at start-up,
 * or a plug-in host that forbids allocation after initialisation).  No counterpart in the
 * reference.  pC/pD/pI are host arrays of 80000/80000/100 floats; d_out is device memory
 * of det_count rows with stride ld.  Nothing is allocated: the parameter copies, derived
 * tables, work counter and status word live in a static device array of about 1.6 MB
 * (each GPU that loads the library holds it until exit), limited to 6666 crystals and 8877
 * holes (larger systems return SYSMAT_ERR_CAPACITY).  The first call on a device looks
 * up that array's device address and should come before any stream capture; the address
 * is looked up again when the current CUDA context of the device changes (after
 * cudaDeviceReset, or under another context the caller made current).  Calls share the
 * array: calls that overlap on the GPU race.  Synchronous on `stream`. */
SYSMAT_API int sysmat_pe_noalloc(const float* pC, const float* pD, const float* pI, float rotation,
                                 int det_begin, int det_count, long long vox_begin,
                                 long long vox_count, float* d_out, long long ld, int mode,
                                 void* stream);

/* ---------------------------------------------------------------------------------- */
/* Compressed output.  A dense block (rows x cols, row stride ld) becomes CSR with the      */
/* entries whose value is > threshold (1e-9 for production matrices), in column order.      */

/* Pass 1: d_row_nnz[rows] receives the per-row counts, d_row_ptr[rows + 1] their exclusive
 * prefix sum (d_row_ptr[rows] = total).  Asynchronous on `stream`. */
SYSMAT_API int sysmat_csr_count(const float* d_dense, int rows, long long cols, long long ld,
                                float threshold, long long* d_row_nnz, long long* d_row_ptr,
                                void* stream);

/* Pass 2: writes column indices (+ col_offset, e.g. the block's first voxel) and values at
 * the row pointers of pass 1; d_col_idx and d_val hold d_row_ptr[rows] entries. */
SYSMAT_API int sysmat_csr_fill(const float* d_dense, int rows, long long cols, long long ld,
                               float threshold, long long col_offset, const long long* d_row_ptr,
                               long long* d_col_idx, float* d_val, void* stream);

/* ---------------------------------------------------------------------------------- */
/* Diagnostics (benchmark roofline).                                                     */

/* Same block as sysmat_pe (reference summation) with work counters (12 values):
 * counts[0] sub-elements evaluated, [1] hole chords that are non-zero, [2] crystal chords
 * that are non-zero, [3] elements, [4] sub-elements stopped by the plate-bypass penalty,
 * [5] elements walked in several chunks, [6] kept candidate objects, [7] round sub-list
 * entries, [8] work items whose candidate superset overflowed shared memory, [9] summed
 * superset sizes, [10] hole chords evaluated, [11] crystal chords evaluated.  Synchronous. */
SYSMAT_API int sysmat_pe_work(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                              long long vox_begin, long long vox_count, float* d_out, long long ld,
                              unsigned long long* counts, void* stream);

/* Measured FP32 FMA throughput (TFLOP/s, FMA = 2 flops) and MUFU throughput (Tops/s) of
 * the current device, from two short calibration kernels. */
SYSMAT_API int sysmat_measure_peaks(double* fp32_tflops, double* mufu_tops);

/* Diagnostic: the elliptical-cylinder chord used for elliptical holes, on n device items of
 * 13 floats (x_in, y_in, z_in, x_out, y_out, z_out, x, y1, y2, z, rho_x, rho_z, theta), in
 * the argument order of the reference's length_ellipticalcylinder_ray (PESysMatGen.cu:801). */
SYSMAT_API int sysmat_ell_chords(const float* d_args, float* d_out, int n, void* stream);

/* Text for a SYSMAT_ERR_* code. */
SYSMAT_API const char* sysmat_error_string(int code);

/* Library build identification (for logs): returns a static string. */
SYSMAT_API const char* sysmat_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SYSMAT_H */
