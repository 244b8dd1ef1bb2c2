// The native API's context (one uploaded system on one device), shared by the library's
// host translation units.
#pragma once

#include <vector>

#include "geom.cuh"
#include "scatter.cuh"

struct sysmat_ctx {
    int device = -1;
    int num_sms = 0;
    sysmat::DevGeom g{};
    int n_holes0_host = 0;
    // raw parameter arrays on the device (bitmap kernels read them like the reference)
    float* d_col = nullptr;
    float* d_det = nullptr;
    float* d_img = nullptr;
    float* d_phys = nullptr;
    std::vector<float> h_phys;
    std::vector<float> h_img;
    std::vector<float> h_det;       // detector parameters (grid scatter: crystal cell divisions)
    float h_col15 = 0.0f, h_col17 = 0.0f;   // layer-0 mu_total and mu_compton (scatter.cu:1716)
    // derived tables
    float4* d_tables = nullptr;
    // launch bookkeeping
    unsigned long long* d_counter = nullptr;
    int* d_status = nullptr;
    // scatter pair tables (sysmat_scatter_prepare)
    sysmat::ScatterScratch scratch{};
    int prepared_parts = 0;
    int prepared_native = 0;        // the pair tables are the native model's
    sysmat::PairRec* pairs = nullptr;
    sysmat::PairNative* pairs_native = nullptr;   // native model's extra pair fields
    sysmat::AttEntry* att = nullptr;
    long long* att_offsets = nullptr;             // 64-bit attenuator-list offset per pair
    double* d_kn_tab = nullptr;     // Klein-Nishina table for kn_e0
    float4* d_shapes = nullptr;     // elliptical holes (sysmat_set_hole_shapes), or nullptr
    void* d_tables64 = nullptr;     // FP64 mode tables (DevGeom::t64)
    sysmat::D4* d_shapes64 = nullptr;   // FP64 mode elliptical holes, or nullptr
    float kn_e0 = -1.0f;
};

namespace sysmat {
// SYSMAT_OK when [det_begin, +det_count) x [vox_begin, +vox_count) lies inside the context's
// matrix, ld >= vox_count, d_out is set and the context's device is current.
int check_block(const sysmat_ctx* ctx, int det_begin, int det_count, long long vox_begin,
                long long vox_count, const float* d_out, long long ld);
// Checks a scatter block as sysmat_scatter does and fills its launch (building the context's
// Klein-Nishina table when needed; synchronises `stream` then).
int scatter_setup(sysmat_ctx* ctx, int parts, int hole_model, float rotation, const float* d_pe, int det_begin,
                  int det_count, long long vox_begin, long long vox_count, float* d_out, long long ld,
                  cudaStream_t stream, ScatterPhysics* ph, ScatterLaunch* L);
}  // namespace sysmat
