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
};

int launch_pe(const DevGeom& g, const PeLaunch& L, int mode, int num_sms, cudaStream_t stream);

__global__ void derive_crystals(const float* __restrict__ det, float fov, int n, float4* pos,
                                float4* size, float4* mu, float4* trig);
__global__ void derive_holes(const float* __restrict__ col, float fov, int n, float4* a, float4* b,
                             float4* raw);

}  // namespace sysmat
