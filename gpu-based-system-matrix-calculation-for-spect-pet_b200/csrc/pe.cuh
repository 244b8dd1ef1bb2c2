// Launch interface of the photoelectric kernel (pe.cu).
#pragma once

#include <cuda_runtime.h>

#include "geom.cuh"

namespace sysmat {

// Per-element capacities of the shared-memory candidate lists (after cone culling and
// the ray-bundle filter).  An element that exceeds them raises kStatusCapacity.
constexpr int kPeEffCrystals = 96;
constexpr int kPeEffHoles = 192;

// Bits of the device status word.
constexpr int kStatusCapacity = 1;

// Sampled form of the photoelectric element (no reference counterpart): crystal sub-elements
// along x, depth and z, and source points per voxel along x, y and z.  The reference fixes
// 8 x 16 x 8 and 1 x 1 x 1 (PESysMatGen.cu:1196-1217, :1031-1034).
struct Sampling {
    int nx = 8, ny = 16, nz = 8;
    int sx = 1, sy = 1, sz = 1;
};

struct PeLaunch {
    int det_begin, det_count;
    long long vox_begin, vox_count;
    long long ld;                          // row stride of out, in floats
    float rotation;                        // rotation index, as Params_Image[20]
    float* out;
    unsigned long long* work_counter;      // zeroed before the launch
    int* status;                           // zeroed before the launch
    // optional work counters (nullptr in timed runs): [0] sub-elements evaluated,
    // [1] non-zero hole chords, [2] non-zero crystal chords, [3] elements, [4] plate-blocked
    // sub-elements, [5] cone-test candidates (holes + crystals)
    unsigned long long* counters;
    Sampling smp;                          // read by the sampled instances only
    // local sampled instance only (optional): per-sub-element contributions, written at
    // ((v - vox_begin) * det_count + (d - det_begin)) * n_sub + (iz * ny + iy) * nx + ix
    float* sub_out = nullptr;
};

// One (geometry, rotation, detector x voxel block) task of a batched launch.  The host fills
// the brick grid of the block (nbx x nby x nbz bricks over z-planes iz0..iz1) and the first
// global item number of the task; items are (row, brick) pairs, row-major.
struct BatchTask {
    int geom;                              // index into the launch's geometry array
    float rotation;                        // rotation index, as Params_Image[20]
    int det_begin, det_count;
    long long vox_begin, vox_count;
    float* out;
    long long ld;
    long long item_begin;
    int nbx, nby, nbz, iz0, iz1;
};

struct BatchLaunch {
    const DevGeom* geoms;                  // device array
    const BatchTask* tasks;                // device array, item_begin ascending
    int n_tasks;
    long long total_items;
    int bx, by, bz;
    unsigned long long* work_counter;      // zeroed before the launch
};

// Forward projection and its vector-Jacobian product over all voxels of one rotation and a
// range of detector rows (pe_adjoint.cuh).
struct AdjLaunch {
    int det_begin, det_count;
    float rotation;
    int bx = 4, by = 4, bz = 2;
    const float* x;                        // n_vox activity values
    const float* u;                        // det_count cotangent values (vjp only)
    double* p;                             // det_count projections (project only), zeroed
    double* grad;                          // 8 values (vjp only), zeroed
    double* q;                             // n_vox back projections (back projection only), zeroed
    unsigned long long* work_counter;      // zeroed
};

int launch_pe(const DevGeom& g, const PeLaunch& L, int mode, int num_sms, cudaStream_t stream);
// The sampled form (L.smp), accumulated in FP64.
int launch_pe_sampled(const DevGeom& g, const PeLaunch& L, int num_sms, cudaStream_t stream);
// The local-coordinate FP32 form with the crystal division of L.smp (voxel centres only),
// optionally writing every sub-element's contribution to L.sub_out.
int launch_pe_local_sampled(const DevGeom& g, const PeLaunch& L, int num_sms, cudaStream_t stream);
// kind 0: projection, kind 1: vector-Jacobian product, kind 2: back projection.
int launch_pe_adjoint(const DevGeom& g, const AdjLaunch& L, int kind, int num_sms, cudaStream_t stream);
// Sets the batched kernel's shared-memory attribute on the current device (once) and returns
// how many of its blocks fit on one SM.  Call before capturing a launch into a graph.
// ell: some system of the launch has elliptical holes (the elliptical instance; it also
// computes circular holes, bit-identically).
int configure_pe_batch(int mode, bool ell, int* blocks_per_sm);
int launch_pe_batch(const BatchLaunch& B, int mode, bool ell, int grid, cudaStream_t stream);

__global__ void derive_crystals(const float* __restrict__ det, float fov, int n, float4* pos,
                                float4* size, float4* mu, float4* trig);
__global__ void derive_holes(const float* __restrict__ col, float fov, int n, float4* a, float4* b,
                             float4* raw);
__global__ void derive_shapes(const float* __restrict__ s, int n, float4* out);
__global__ void derive_shapes64(const float* __restrict__ s, int n, D4* out);
__global__ void derive_tables64(const float* __restrict__ det, const float* __restrict__ col, float fov, int n_det,
                                int n_holes, D4* cry_pos, D4* cry_size, D4* cry_trig, D4* hole_a, D4* hole_b);

}  // namespace sysmat
