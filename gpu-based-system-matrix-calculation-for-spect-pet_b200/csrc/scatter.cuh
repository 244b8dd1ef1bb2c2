// Launch interface of the primary-Compton scatter kernels and the relationship-bitmap
// kernels (scatter.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "geom.cuh"

namespace sysmat {

// Device scratch owned by a context for the scatter path: per-(scatterer, detector) pair
// records and the attenuator lists they index.
struct ScatterScratch {
    void* base = nullptr;
    size_t bytes = 0;
};

inline void scatter_scratch_free(ScatterScratch& s)
{
    if (s.base) cudaFree(s.base);
    s.base = nullptr;
    s.bytes = 0;
}

// Pair record of scatterer s (crystal k = s, or hole h = s - D) and detector crystal d,
// stored at index d * (D + H0) + s (reference hole models: layer-0 holes) or d * (D + H) + s
// (native model: the holes of every layer).
struct PairRec {
    float xss, yss, zss;   // scatter point in crystal d's frame
    float lsd;             // |scatter point - crystal d centre| (world)
    float labs;            // chord of the absorption ray inside crystal d
    int att_begin;         // first entry in the attenuator list, counted from the first
                           // entry of detector row d (the row's 64-bit offset is kept apart)
    int att_count;         // number of attenuators with a non-zero chord
    int valid;             // 0 for the excluded pair s == d
};

// Native model only, beside each PairRec: tungsten on the way from a hole scatter point to d,
// sum_m mu_pe,m L_m and sum_m mu_C,m L_m at the photopeak, and the scatter hole's layer
// mu_total and mu_C (its interaction weight); zero for crystal scatterers.
struct PairNative {
    float w_pe, w_c, mu_tot_h, mu_c_h;
};

// Attenuator entry: chord length and the attenuator's photoelectric and Compton
// coefficients at the photopeak energy.
struct AttEntry {
    float len, mu_pe, mu_c;
};

struct ScatterPhysics {
    int use_compton;       // (int)floor(P[0] + 0.5f) == 1
    int same_window;       // (int)floor(P[4] + 0.5f) > 0
    float lo, hi;          // P[5], P[6]
    float e0;              // P[7]
    float integ;           // KN normalisation over [0, pi] (FP64 sum, rounded)
    float col_mu_tot0;     // C[15]
    float col_mu_c0;       // C[17]
};

struct ScatterLaunch {
    int parts;             // bit 0 crystal, bit 1 collimator
    int hole_model;        // 0 combined program, 1 collimator-only program, 2 native
    int det_begin, det_count;
    long long vox_begin, vox_count, ld;
    float rotation;
    const float* pe;       // D x V photoelectric matrix (crystal part)
    const PairRec* pairs;
    const PairNative* native;   // hole_model 2 only
    const AttEntry* att;
    const long long* att_offsets;   // 64-bit list offset of pair p; row d starts at [d * ns]
    const double* kn_tab;  // Klein-Nishina table (kn_table_build), kKnTable + 1 nodes on [0, pi]
    float* out;
};

// FP64 table of the Klein-Nishina shape on [0, pi]: nodes theta_i = i * pi / kKnTable;
// [0 .. N] integral from 0, [N+1 .. 2N+1] F = KN(theta) sin(theta), [2N+2 .. 3N+2] dF/dtheta.
constexpr int kKnTable = 4096;
void kn_table_build(double e0, double* host_tab);   // host buffer of 3 * (kKnTable + 1) doubles

// The Klein-Nishina table at angle th: G (integral from 0) and F by cubic Hermite
// interpolation (error ~1e-14), F' linearly.
__device__ __forceinline__ void kn_tab_eval(const double* __restrict__ tab, double th, double& G,
                                            double& F, double& Fp)
{
    const double hc = 3.14159265358979323846 / kKnTable;
    double x = th * (kKnTable / 3.14159265358979323846);   // cell coordinate (no double division)
    int i = (int)x;
    i = i < 0 ? 0 : (i > kKnTable - 1 ? kKnTable - 1 : i);
    const double t = x - (double)i;
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
    const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    const double* Gt = tab;
    const double* Ft = tab + (kKnTable + 1);
    const double* Pt = tab + 2 * (kKnTable + 1);
    const double g0 = __ldg(&Gt[i]), g1 = __ldg(&Gt[i + 1]);
    const double f0 = __ldg(&Ft[i]), f1 = __ldg(&Ft[i + 1]);
    const double p0 = __ldg(&Pt[i]), p1 = __ldg(&Pt[i + 1]);
    G = h00 * g0 + h10 * hc * f0 + h01 * g1 + h11 * hc * f1;
    F = h00 * f0 + h10 * hc * p0 + h01 * f1 + h11 * hc * p1;
    Fp = (1.0 - t) * p0 + t * p1;
}

// Energy-window probability of a Gaussian of resolution res (FWHM fraction) at energy e
// (calculategaussianIntegral, ScatterGen_RayTracing_CircularHole/scatter.cu:1025-1038).
__device__ __forceinline__ float window_prob(float e, float res, float lo, float hi)
{
    const float sigma = res / 2.35482f * e;
    const float s2 = (float)((double)sigma * 1.4142135623730951);   // sigma * sqrt(2.0)
    const float z1 = (lo - e) / s2;
    const float z2 = (hi - e) / s2;
    return 0.5f * (erff(z2) - erff(z1));
}

// Word counts of the reference bitmap layouts (scatter.cu:2053-2056, :2234-2237).
long long bitmap_crystal_words(int n_det);
long long bitmap_collimator_words(int n_det, int n_holes0);

int launch_bitmap_crystal(const DevGeom& g, uint32_t* words, cudaStream_t s);
int launch_bitmap_collimator(const DevGeom& g, uint32_t* words, cudaStream_t s);

// Build pair records and attenuator lists.  Allocates/grows `scratch` as needed (synchronises
// `s` once to size the attenuator list).  parts selects which pairs are built.  The lists are
// indexed with 64-bit offsets (*att_offsets, one per pair plus the total): a production system
// can hold more than 2^31 attenuator entries.
int build_scatter_pairs(const DevGeom& g, int parts, const uint32_t* bm_crystal,
                        const uint32_t* bm_collimator, ScatterScratch& scratch, PairRec** pairs,
                        AttEntry** att, long long** att_offsets, cudaStream_t s);

// Native model: scatter points at the holes of every layer, each with its layer's mu; the
// collimator-scatter attenuators from the relationship predicate evaluated directly (no
// bitmap); tungsten attenuation of the scattered photon on its way to the crystal.
int build_scatter_pairs_native(const DevGeom& g, int parts, const uint32_t* bm_crystal,
                               ScatterScratch& scratch, PairRec** pairs, PairNative** native, AttEntry** att,
                               long long** att_offsets, cudaStream_t s);

int launch_scatter(const DevGeom& g, const ScatterPhysics& ph, const ScatterLaunch& L,
                   cudaStream_t s);

// Voxels per scatter block (one thread per voxel) and the batched launch: one task per
// (system, rotation, detector x voxel block); items are (row, voxel block) pairs, row-major.
constexpr int kScatterBlockVoxels = 128;
struct ScatterTask {
    ScatterLaunch L;
    ScatterPhysics ph;
    int geom;                  // index into the launch's geometry array
    int n_vblocks;             // voxel blocks of the task
    long long item_begin;
};
struct ScatterBatchLaunch {
    const DevGeom* geoms;
    const ScatterTask* tasks;  // item_begin ascending
    int n_tasks;
    long long total_items;
    unsigned long long* work_counter;   // zeroed before the launch
};
int scatter_batch_blocks_per_sm();
int launch_scatter_batch(const ScatterBatchLaunch& B, int grid, cudaStream_t s);

// Klein-Nishina normalisation of the reference, sum over theta_i = float(i * 0.01f),
// i = 0..floor(float(pi)/0.01f), evaluated in double (scatter.cu:980-993, :1169).
double kn_normalisation(double e0);

}  // namespace sysmat
