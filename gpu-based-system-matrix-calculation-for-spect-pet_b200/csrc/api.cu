// Host side of libsysmat: parameter decoding, device tables, the native handle API and the
// reference-compatible entry points.
//
// The reference host wrappers (PESysMatGen.cu:1368-1437, scatter.cu:2013-2378) allocate,
// copy, launch and free on every call.  Here a context holds the uploaded geometry and its
// derived tables; the reference-compatible entry points keep one cached context per device
// keyed by the parameter contents, so a rotation loop re-uses the tables and the output
// buffer.  No function calls exit(); every failure is an error code.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/sysmat.h"
#include "geom.cuh"
#include "pe.cuh"
#include "scatter.cuh"
#include "ctx.cuh"

using namespace sysmat;

#define CUDA_TRY(expr)                                                                     \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess) {                                                           \
            std::fprintf(stderr, "sysmat: %s failed: %s (%s:%d)\n", #expr,                 \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                      \
            return SYSMAT_ERR_CUDA;                                                        \
        }                                                                                  \
    } while (0)


namespace {

int floor_count(float v, float bias) { return (int)std::floor(v + bias); }

bool finite_all(const float* p, size_t n)
{
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// Decode counts and sizes exactly as the reference kernels do and check the documented
// capacities (PESysMatGen.cu:964-1013; the 80000-float tables hold at most 6666 crystals
// and 8877 holes; layer headers 1..9 sit below the hole table at index 100).
int decode(const float* pC, const float* pD, const float* pI, DevGeom& g, int& n_holes0)
{
    if (!pD || !pI) return SYSMAT_ERR_ARG;
    std::memset(&g, 0, sizeof(g));
    g.n_det = floor_count(pD[0], 0.000001f);
    if (g.n_det < 1 || g.n_det > (kNDetector - 1) / 12) return SYSMAT_ERR_CAPACITY;
    if (!finite_all(pD, 1 + 12 * (size_t)g.n_det)) return SYSMAT_ERR_ARG;
    g.nx = (int)std::floor(pI[0]);
    g.ny = (int)std::floor(pI[1]);
    g.nz = (int)std::floor(pI[2]);
    if (g.nx < 1 || g.ny < 1 || g.nz < 1) return SYSMAT_ERR_ARG;
    g.nvox = (long long)g.nx * g.ny * g.nz;
    if (!finite_all(pI, 12) || !std::isfinite(pI[20])) return SYSMAT_ERR_ARG;
    g.wx = pI[3]; g.wy = pI[4]; g.wz = pI[5];
    g.shx = pI[8]; g.shy = pI[9]; g.shz = pI[10];
    g.fov = pI[11];
    g.angle_step = pI[7];
    g.nonneg_mu = 1;
    for (int d = 0; d < g.n_det; ++d)
        for (int k = 7; k <= 9; ++k)
            if (!(pD[12 * d + k] >= 0.0f)) g.nonneg_mu = 0;
    n_holes0 = 0;
    if (pC) {
        g.n_layers = floor_count(pC[0], 0.000001f);
        if (g.n_layers < 0 || g.n_layers > kMaxLayers) return SYSMAT_ERR_CAPACITY;
        int h = 0;
        for (int m = 0; m < g.n_layers; ++m) {
            const float* L = pC + (m + 1) * 10;
            if (!finite_all(L, 8)) return SYSMAT_ERR_ARG;
            const int nh = (int)std::floor(L[0]);
            if (nh < 0) return SYSMAT_ERR_ARG;
            LayerInfo& Ly = g.layer[m];
            // plate box exactly as PESysMatGen.cu:1242-1249 forms it
            Ly.x1 = -L[1] / 2.0f;
            Ly.x2 = L[1] / 2.0f;
            Ly.y1 = -L[2] / 2.0f + g.fov + L[4];
            Ly.y2 = L[2] / 2.0f + g.fov + L[4];
            Ly.z1 = -L[3] / 2.0f;
            Ly.z2 = L[3] / 2.0f;
            Ly.thickness = L[2];
            Ly.mu_total = L[5];
            Ly.mu_pe = L[6];
            Ly.mu_c = L[7];
            if (!(L[5] >= 0.0f)) g.nonneg_mu = 0;
            Ly.hole_begin = h;
            Ly.hole_count = nh;
            h += nh;
            if (h > (kNCollimator - 100) / 9) return SYSMAT_ERR_CAPACITY;
        }
        g.n_holes = h;
        if (!finite_all(pC + 100, 9 * (size_t)h)) return SYSMAT_ERR_ARG;
        for (int i = 0; i < h; ++i)
            if (!(pC[100 + 9 * i + 5] >= 0.0f)) g.nonneg_mu = 0;
        n_holes0 = floor_count(pC[10], 0.000001f);
        if (n_holes0 < 0 || n_holes0 > h) n_holes0 = g.n_layers > 0 ? g.layer[0].hole_count : 0;
        g.n_holes0 = n_holes0;
    }
    return SYSMAT_OK;
}

bool same_device(const sysmat_ctx* ctx)
{
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return false;
    return cur == ctx->device;
}

}  // namespace

// Parameter decoding for other translation units of the library (see noalloc.cu).
namespace sysmat {
int sysmat_decode_geometry(const float* pC, const float* pD, const float* pI, DevGeom& g, int& n_holes0)
{
    return decode(pC, pD, pI, g, n_holes0);
}
}  // namespace sysmat

extern "C" SYSMAT_API const char* sysmat_error_string(int code)
{
    switch (code) {
    case SYSMAT_OK: return "ok";
    case SYSMAT_ERR_ARG: return "invalid argument or parameter array";
    case SYSMAT_ERR_CUDA: return "CUDA runtime error";
    case SYSMAT_ERR_CAPACITY: return "geometry exceeds a documented capacity";
    case SYSMAT_ERR_IO: return "relationship bitmap file could not be read or written";
    case SYSMAT_ERR_NOMEM: return "allocation failed";
    case SYSMAT_ERR_TIMEOUT: return "a bounded device wait gave up";
    default: return "unknown error";
    }
}

extern "C" SYSMAT_API const char* sysmat_version(void) { return "sysmat-b200 0.1 (sm_100a)"; }

extern "C" SYSMAT_API int sysmat_create(sysmat_ctx** out, int device, const float* pC, const float* pD,
                             const float* pI, const float* pP)
{
    if (!out) return SYSMAT_ERR_ARG;
    *out = nullptr;
    DevGeom g;
    int nh0 = 0;
    int rc = decode(pC, pD, pI, g, nh0);
    if (rc) return rc;
    int cur = -1;
    CUDA_TRY(cudaGetDevice(&cur));
    if (cur != device) return SYSMAT_ERR_ARG;
    sysmat_ctx* ctx = new sysmat_ctx();
    ctx->device = device;
    ctx->g = g;
    ctx->n_holes0_host = nh0;
    ctx->h_img.assign(pI, pI + kNImage);
    ctx->h_det.assign(pD, pD + kNDetector);
    if (pC) { ctx->h_col15 = pC[15]; ctx->h_col17 = pC[17]; }
    if (pP) ctx->h_phys.assign(pP, pP + kNPhysics);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete ctx; return SYSMAT_ERR_CUDA; }
    ctx->num_sms = prop.multiProcessorCount;

    const int D = g.n_det, H = g.n_holes;
    const size_t n_tables = 4 * (size_t)D + 3 * (size_t)(H > 0 ? H : 1);
    bool ok = cudaMalloc(&ctx->d_det, sizeof(float) * kNDetector) == cudaSuccess &&
              cudaMalloc(&ctx->d_col, sizeof(float) * kNCollimator) == cudaSuccess &&
              cudaMalloc(&ctx->d_img, sizeof(float) * kNImage) == cudaSuccess &&
              cudaMalloc(&ctx->d_phys, sizeof(float) * kNPhysics) == cudaSuccess &&
              cudaMalloc(&ctx->d_tables, sizeof(float4) * n_tables) == cudaSuccess &&
              cudaMalloc(&ctx->d_counter, sizeof(unsigned long long) * 4) == cudaSuccess &&
              cudaMalloc(&ctx->d_status, sizeof(int) * 4) == cudaSuccess;
    if (!ok) { sysmat_destroy(ctx); return SYSMAT_ERR_NOMEM; }
    ok = cudaMemcpy(ctx->d_det, pD, sizeof(float) * kNDetector, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(ctx->d_col, 0, sizeof(float) * kNCollimator) == cudaSuccess &&
         (!pC || cudaMemcpy(ctx->d_col, pC, sizeof(float) * kNCollimator, cudaMemcpyHostToDevice) == cudaSuccess) &&
         cudaMemcpy(ctx->d_img, pI, sizeof(float) * kNImage, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(ctx->d_phys, 0, sizeof(float) * kNPhysics) == cudaSuccess &&
         (!pP || cudaMemcpy(ctx->d_phys, pP, sizeof(float) * kNPhysics, cudaMemcpyHostToDevice) == cudaSuccess);
    if (!ok) { sysmat_destroy(ctx); return SYSMAT_ERR_CUDA; }

    float4* t = ctx->d_tables;
    ctx->g.raw_det = ctx->d_det;
    ctx->g.cry.pos = t;
    ctx->g.cry.size = t + D;
    ctx->g.cry.mu = t + 2 * D;
    ctx->g.cry.trig = t + 3 * D;
    float4* th = t + 4 * D;
    const int Hs = H > 0 ? H : 1;
    ctx->g.hole.a = th;
    ctx->g.hole.b = th + Hs;
    ctx->g.hole.raw = th + 2 * Hs;
    derive_crystals<<<(D + 127) / 128, 128>>>(ctx->d_det, g.fov, D, t, t + D, t + 2 * D, t + 3 * D);
    if (H > 0) derive_holes<<<(H + 127) / 128, 128>>>(ctx->d_col, g.fov, H, th, th + Hs, th + 2 * Hs);

    // FP64 mode tables: crystals 3 x D4, holes 2 x D4, layers kLayer64 doubles each (from the
    // raw floats in double, as the FP64 restatement forms them: PESysMatGen.cu:1242-1249)
    const size_t n64 = 3 * (size_t)D + 2 * (size_t)Hs;
    const size_t layer_bytes = sizeof(double) * kLayer64 * (size_t)(g.n_layers > 0 ? g.n_layers : 1);
    if (cudaMalloc(&ctx->d_tables64, sizeof(D4) * n64 + layer_bytes) != cudaSuccess) {
        ctx->d_tables64 = nullptr;
        sysmat_destroy(ctx);
        return SYSMAT_ERR_NOMEM;
    }
    D4* t64 = static_cast<D4*>(ctx->d_tables64);
    ctx->g.t64.cry_pos = t64;
    ctx->g.t64.cry_size = t64 + D;
    ctx->g.t64.cry_trig = t64 + 2 * D;
    ctx->g.t64.hole_a = t64 + 3 * D;
    ctx->g.t64.hole_b = t64 + 3 * D + Hs;
    double* lay64 = reinterpret_cast<double*>(t64 + n64);
    ctx->g.t64.layer = lay64;
    {
        std::vector<double> hl(kLayer64 * (size_t)(g.n_layers > 0 ? g.n_layers : 1), 0.0);
        const double fov = (double)g.fov;
        for (int m = 0; m < g.n_layers; ++m) {
            const float* L = pC + (m + 1) * 10;
            double* o = hl.data() + kLayer64 * m;
            o[0] = -(double)L[1] / 2.0;
            o[1] = (double)L[1] / 2.0;
            o[2] = -(double)L[2] / 2.0 + fov + (double)L[4];
            o[3] = (double)L[2] / 2.0 + fov + (double)L[4];
            o[4] = -(double)L[3] / 2.0;
            o[5] = (double)L[3] / 2.0;
            o[6] = (double)L[2];
            o[7] = (double)L[5];
        }
        if (cudaMemcpy(lay64, hl.data(), sizeof(double) * hl.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            sysmat_destroy(ctx);
            return SYSMAT_ERR_CUDA;
        }
    }
    if (D + H > 0)
        derive_tables64<<<(D + H + 127) / 128, 128>>>(ctx->d_det, ctx->d_col, g.fov, D, H, t64, t64 + D, t64 + 2 * D,
                                                      t64 + 3 * D, t64 + 3 * D + Hs);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        sysmat_destroy(ctx);
        return SYSMAT_ERR_CUDA;
    }
    *out = ctx;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_destroy(sysmat_ctx* ctx)
{
    if (!ctx) return SYSMAT_OK;
    scatter_scratch_free(ctx->scratch);
    cudaFree(ctx->d_kn_tab);
    cudaFree(ctx->d_shapes);
    cudaFree(ctx->d_tables64);
    cudaFree(ctx->d_shapes64);
    cudaFree(ctx->d_det);
    cudaFree(ctx->d_col);
    cudaFree(ctx->d_img);
    cudaFree(ctx->d_phys);
    cudaFree(ctx->d_tables);
    cudaFree(ctx->d_counter);
    cudaFree(ctx->d_status);
    delete ctx;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_set_hole_shapes(sysmat_ctx* ctx, const float* rho_x, const float* rho_z,
                                                  const float* theta)
{
    if (!ctx || !same_device(ctx)) return SYSMAT_ERR_ARG;
    if (!rho_x) {                                   // back to circular holes
        // the tables stay allocated until sysmat_destroy: batch plans copy their pointers
        ctx->g.hole_shape = nullptr;
        ctx->g.t64.hole_shape = nullptr;
        return SYSMAT_OK;
    }
    if (!rho_z || !theta) return SYSMAT_ERR_ARG;
    const int n = ctx->g.n_holes;
    std::vector<float> h(3 * (size_t)(n > 0 ? n : 1), 0.0f);
    std::vector<float> col(kNCollimator);
    CUDA_TRY(cudaMemcpy(col.data(), ctx->d_col, sizeof(float) * kNCollimator, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) {
        const float rx = rho_x[i], rz = rho_z[i], th = theta[i];
        if (!std::isfinite(rx) || !std::isfinite(rz) || !std::isfinite(th)) return SYSMAT_ERR_ARG;
        if (rx > 0.0f) {
            // the hole's radius field bounds the ellipse: the cone test and the filters use it
            const float r = col[100 + 9 * i + 4];
            if (!(rz > 0.0f) || rx > r || rz > r) return SYSMAT_ERR_ARG;
        }
        h[3 * i] = rx > 0.0f ? rx : 0.0f;
        h[3 * i + 1] = rz;
        h[3 * i + 2] = th;
    }
    float* d_s = nullptr;
    if (!ctx->d_shapes && cudaMalloc(&ctx->d_shapes, sizeof(float4) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) {
        ctx->d_shapes = nullptr;
        return SYSMAT_ERR_NOMEM;
    }
    if (!ctx->d_shapes64 && cudaMalloc(&ctx->d_shapes64, sizeof(D4) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) {
        ctx->d_shapes64 = nullptr;
        return SYSMAT_ERR_NOMEM;
    }
    if (cudaMalloc(&d_s, sizeof(float) * h.size()) != cudaSuccess) return SYSMAT_ERR_NOMEM;
    cudaError_t e = cudaMemcpy(d_s, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) {
        derive_shapes<<<(n + 255) / 256, 256>>>(d_s, n, ctx->d_shapes);
        derive_shapes64<<<(n + 255) / 256, 256>>>(d_s, n, ctx->d_shapes64);
        e = cudaDeviceSynchronize();
    }
    cudaFree(d_s);
    if (e != cudaSuccess) return SYSMAT_ERR_CUDA;
    ctx->g.hole_shape = ctx->d_shapes;
    ctx->g.t64.hole_shape = ctx->d_shapes64;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_dims(const sysmat_ctx* ctx, int* n_det, long long* n_vox, int* n_holes0,
                           int* n_holes, int* n_layers)
{
    if (!ctx) return SYSMAT_ERR_ARG;
    if (n_det) *n_det = ctx->g.n_det;
    if (n_vox) *n_vox = ctx->g.nvox;
    if (n_holes0) *n_holes0 = ctx->g.n_holes0;
    if (n_holes) *n_holes = ctx->g.n_holes;
    if (n_layers) *n_layers = ctx->g.n_layers;
    return SYSMAT_OK;
}

namespace sysmat {
int check_block(const sysmat_ctx* ctx, int det_begin, int det_count, long long vox_begin,
                long long vox_count, const float* d_out, long long ld)
{
    if (!ctx || !d_out) return SYSMAT_ERR_ARG;
    if (det_begin < 0 || det_count < 0 || det_begin + det_count > ctx->g.n_det) return SYSMAT_ERR_ARG;
    if (vox_begin < 0 || vox_count < 0 || vox_begin + vox_count > ctx->g.nvox) return SYSMAT_ERR_ARG;
    if (ld < vox_count) return SYSMAT_ERR_ARG;
    if (!same_device(ctx)) return SYSMAT_ERR_ARG;
    return SYSMAT_OK;
}
}  // namespace sysmat

namespace {

// The launch record of one photoelectric block, with the context's counter and status word.
PeLaunch pe_block(sysmat_ctx* ctx, float rotation, int det_begin, int det_count, long long vox_begin,
                  long long vox_count, float* d_out, long long ld)
{
    PeLaunch L;
    L.det_begin = det_begin;
    L.det_count = det_count;
    L.vox_begin = vox_begin;
    L.vox_count = vox_count;
    L.ld = ld;
    L.rotation = rotation;
    L.out = d_out;
    L.work_counter = ctx->d_counter;
    L.status = ctx->d_status;
    L.counters = nullptr;
    return L;
}

// Zero the counter and status word, launch (launch(L) returns non-zero on a launch error),
// then wait for the status word: SYSMAT_ERR_CAPACITY if an element overflowed a list.
template <class Launch>
int run_pe_block(sysmat_ctx* ctx, const PeLaunch& L, cudaStream_t s, Launch&& launch)
{
    CUDA_TRY(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), s));
    CUDA_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s));
    if (launch(L)) return SYSMAT_ERR_CUDA;
    int status = 0;
    CUDA_TRY(cudaMemcpyAsync(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return (status & kStatusCapacity) ? SYSMAT_ERR_CAPACITY : SYSMAT_OK;
}

}  // namespace

extern "C" SYSMAT_API int sysmat_pe(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                         long long vox_begin, long long vox_count, float* d_out, long long ld,
                         int mode, void* stream)
{
    int rc = check_block(ctx, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    if (rc) return rc;
    if (mode != SYSMAT_MODE_REFERENCE && mode != SYSMAT_MODE_PRECISE && mode != SYSMAT_MODE_FP64 &&
        mode != SYSMAT_MODE_LOCAL)
        return SYSMAT_ERR_ARG;
    if (det_count == 0 || vox_count == 0) return SYSMAT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const PeLaunch L = pe_block(ctx, rotation, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    return run_pe_block(ctx, L, s, [&](const PeLaunch& l) { return launch_pe(ctx->g, l, mode, ctx->num_sms, s); });
}

extern "C" SYSMAT_API int sysmat_pe_sampled_mode(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                                 long long vox_begin, long long vox_count, const int* crystal_div,
                                                 const int* voxel_sub, int mode, float* d_out, long long ld,
                                                 void* stream)
{
    int rc = check_block(ctx, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    if (rc) return rc;
    if (!crystal_div || !voxel_sub) return SYSMAT_ERR_ARG;
    if (mode != SYSMAT_MODE_PRECISE && mode != SYSMAT_MODE_LOCAL) return SYSMAT_ERR_ARG;
    Sampling smp;
    smp.nx = crystal_div[0]; smp.ny = crystal_div[1]; smp.nz = crystal_div[2];
    smp.sx = voxel_sub[0]; smp.sy = voxel_sub[1]; smp.sz = voxel_sub[2];
    const int div[3] = {smp.nx, smp.ny, smp.nz}, sub[3] = {smp.sx, smp.sy, smp.sz};
    for (int k = 0; k < 3; ++k) {
        if (div[k] < 1 || div[k] > SYSMAT_SAMPLED_MAX_DIV) return SYSMAT_ERR_ARG;
        if (sub[k] < 1 || sub[k] > SYSMAT_SAMPLED_MAX_SUB) return SYSMAT_ERR_ARG;
    }
    if (smp.nx * smp.ny * smp.nz > SYSMAT_SAMPLED_MAX_SUBELEMENTS) return SYSMAT_ERR_ARG;
    if (smp.sx * smp.sy * smp.sz > SYSMAT_SAMPLED_MAX_POINTS) return SYSMAT_ERR_ARG;
    if (det_count == 0 || vox_count == 0) return SYSMAT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    PeLaunch L = pe_block(ctx, rotation, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    L.smp = smp;
    if (mode == SYSMAT_MODE_LOCAL)
        return run_pe_block(ctx, L, s,
                            [&](const PeLaunch& l) { return launch_pe_local_sampled(ctx->g, l, ctx->num_sms, s); });
    return run_pe_block(ctx, L, s, [&](const PeLaunch& l) { return launch_pe_sampled(ctx->g, l, ctx->num_sms, s); });
}

extern "C" SYSMAT_API int sysmat_pe_sampled(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                            long long vox_begin, long long vox_count, const int* crystal_div,
                                            const int* voxel_sub, float* d_out, long long ld, void* stream)
{
    return sysmat_pe_sampled_mode(ctx, rotation, det_begin, det_count, vox_begin, vox_count, crystal_div, voxel_sub,
                                  SYSMAT_MODE_PRECISE, d_out, ld, stream);
}

extern "C" SYSMAT_API long long sysmat_bitmap_crystal_words(const sysmat_ctx* ctx)
{
    return ctx ? bitmap_crystal_words(ctx->g.n_det) : SYSMAT_ERR_ARG;
}

extern "C" SYSMAT_API long long sysmat_bitmap_collimator_words(const sysmat_ctx* ctx)
{
    return ctx ? bitmap_collimator_words(ctx->g.n_det, ctx->g.n_holes0) : SYSMAT_ERR_ARG;
}

extern "C" SYSMAT_API int sysmat_bitmap_crystal(sysmat_ctx* ctx, uint32_t* d_words, void* stream)
{
    if (!ctx || !d_words || !same_device(ctx)) return SYSMAT_ERR_ARG;
    return launch_bitmap_crystal(ctx->g, d_words, (cudaStream_t)stream) ? SYSMAT_ERR_CUDA : SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_bitmap_collimator(sysmat_ctx* ctx, uint32_t* d_words, void* stream)
{
    if (!ctx || !d_words || !same_device(ctx)) return SYSMAT_ERR_ARG;
    return launch_bitmap_collimator(ctx->g, d_words, (cudaStream_t)stream) ? SYSMAT_ERR_CUDA : SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_scatter_prepare(sysmat_ctx* ctx, int parts, const uint32_t* d_bm_crystal,
                                                 const uint32_t* d_bm_collimator, void* stream)
{
    if (!ctx || !same_device(ctx)) return SYSMAT_ERR_ARG;
    if (parts < 1 || parts > 3) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_CRYSTAL) && !d_bm_crystal) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_COLLIMATOR) && (!d_bm_collimator || ctx->g.n_holes0 < 1))
        return SYSMAT_ERR_ARG;
    ctx->prepared_parts = 0;
    const int rc = build_scatter_pairs(ctx->g, parts, d_bm_crystal, d_bm_collimator, ctx->scratch,
                                       &ctx->pairs, &ctx->att, &ctx->att_offsets, (cudaStream_t)stream);
    if (rc == -2) return SYSMAT_ERR_NOMEM;
    if (rc) return SYSMAT_ERR_CUDA;
    ctx->prepared_parts = parts;
    ctx->prepared_native = 0;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_scatter_prepare_native(sysmat_ctx* ctx, int parts, const uint32_t* d_bm_crystal,
                                                        void* stream)
{
    if (!ctx || !same_device(ctx)) return SYSMAT_ERR_ARG;
    if (parts < 1 || parts > 3) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_CRYSTAL) && !d_bm_crystal) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_COLLIMATOR) && (ctx->g.n_holes < 1 || ctx->g.n_layers < 1)) return SYSMAT_ERR_ARG;
    ctx->prepared_parts = 0;
    const int rc = build_scatter_pairs_native(ctx->g, parts, d_bm_crystal, ctx->scratch, &ctx->pairs,
                                              &ctx->pairs_native, &ctx->att, &ctx->att_offsets,
                                              (cudaStream_t)stream);
    if (rc == -2) return SYSMAT_ERR_NOMEM;
    if (rc) return SYSMAT_ERR_CUDA;
    ctx->prepared_parts = parts;
    ctx->prepared_native = 1;
    return SYSMAT_OK;
}

namespace sysmat {

// Checks a scatter block against the context (as sysmat_scatter documents), builds the
// Klein-Nishina table of the context's photopeak if needed, and fills the launch.
int scatter_setup(sysmat_ctx* ctx, int parts, int hole_model, float rotation, const float* d_pe, int det_begin,
                  int det_count, long long vox_begin, long long vox_count, float* d_out, long long ld,
                  cudaStream_t stream, ScatterPhysics* ph_out, ScatterLaunch* L_out)
{
    int rc = check_block(ctx, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    if (rc) return rc;
    if (parts < 1 || parts > 3 || (parts & ~ctx->prepared_parts)) return SYSMAT_ERR_ARG;
    if (hole_model != SYSMAT_HOLE_MODEL_COMBINED && hole_model != SYSMAT_HOLE_MODEL_VARIANT &&
        hole_model != SYSMAT_HOLE_MODEL_NATIVE)
        return SYSMAT_ERR_ARG;
    // the pair tables' layout follows the model they were prepared for
    if ((hole_model == SYSMAT_HOLE_MODEL_NATIVE) != (ctx->prepared_native != 0)) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_CRYSTAL) && !d_pe) return SYSMAT_ERR_ARG;
    if (!std::isfinite(rotation)) return SYSMAT_ERR_ARG;
    if (ctx->h_phys.size() != (size_t)kNPhysics) return SYSMAT_ERR_ARG;
    const float* P = ctx->h_phys.data();
    ScatterPhysics ph;
    ph.use_compton = (int)std::floor(P[0] + 0.5f) == 1;          // scatter.cu:1144
    ph.same_window = (int)std::floor(P[4] + 0.5f) > 0;           // :1145, :1154
    ph.lo = P[5];
    ph.hi = P[6];
    ph.e0 = P[7];
    ph.integ = (float)kn_normalisation((double)P[7]);
    ph.col_mu_tot0 = 0.0f;
    ph.col_mu_c0 = 0.0f;
    if (ctx->g.n_layers > 0) {
        ph.col_mu_tot0 = ctx->h_col15;
        ph.col_mu_c0 = ctx->h_col17;
    }
    ScatterLaunch L;
    L.parts = parts;
    L.hole_model = hole_model;
    L.det_begin = det_begin;
    L.det_count = det_count;
    L.vox_begin = vox_begin;
    L.vox_count = vox_count;
    L.ld = ld;
    L.rotation = rotation;
    L.pe = d_pe;
    L.pairs = ctx->pairs;
    L.native = ctx->pairs_native;
    L.att = ctx->att;
    L.att_offsets = ctx->att_offsets;
    L.out = d_out;
    if (!ctx->d_kn_tab || ctx->kn_e0 != ph.e0) {     // (re)build the FP64 Klein-Nishina table
        std::vector<double> tab(3 * (size_t)(kKnTable + 1));
        kn_table_build((double)ph.e0, tab.data());
        if (!ctx->d_kn_tab &&
            cudaMalloc(&ctx->d_kn_tab, sizeof(double) * tab.size()) != cudaSuccess) {
            ctx->d_kn_tab = nullptr;
            return SYSMAT_ERR_NOMEM;
        }
        CUDA_TRY(cudaMemcpyAsync(ctx->d_kn_tab, tab.data(), sizeof(double) * tab.size(),
                                 cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        ctx->kn_e0 = ph.e0;
    }
    L.kn_tab = ctx->d_kn_tab;
    *ph_out = ph;
    *L_out = L;
    return SYSMAT_OK;
}

}  // namespace sysmat

extern "C" SYSMAT_API int sysmat_scatter(sysmat_ctx* ctx, int parts, int hole_model, float rotation,
                                         const float* d_pe, int det_begin, int det_count,
                                         long long vox_begin, long long vox_count, float* d_out,
                                         long long ld, void* stream)
{
    ScatterPhysics ph;
    ScatterLaunch L;
    const int rc = scatter_setup(ctx, parts, hole_model, rotation, d_pe, det_begin, det_count, vox_begin,
                                 vox_count, d_out, ld, (cudaStream_t)stream, &ph, &L);
    if (rc) return rc;
    return launch_scatter(ctx->g, ph, L, (cudaStream_t)stream) ? SYSMAT_ERR_CUDA : SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_pe_work(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                         long long vox_begin, long long vox_count, float* d_out,
                                         long long ld, unsigned long long* counts, void* stream)
{
    int rc = check_block(ctx, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    if (rc) return rc;
    if (!counts) return SYSMAT_ERR_ARG;
    unsigned long long* d_cnt = nullptr;
    if (cudaMalloc(&d_cnt, 16 * sizeof(unsigned long long)) != cudaSuccess) return SYSMAT_ERR_NOMEM;
    cudaStream_t s = (cudaStream_t)stream;
    PeLaunch L = pe_block(ctx, rotation, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    L.counters = d_cnt;
    rc = SYSMAT_OK;
    if (cudaMemsetAsync(d_cnt, 0, 16 * sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s) != cudaSuccess ||
        launch_pe(ctx->g, L, SYSMAT_MODE_REFERENCE, ctx->num_sms, s) ||
        cudaMemcpyAsync(counts, d_cnt, 12 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        rc = SYSMAT_ERR_CUDA;
    cudaFree(d_cnt);
    return rc;
}

// ------------------------------------------------------------------------------------
// Reference-compatible entry points.

namespace {

uint64_t fnv1a(uint64_t h, const void* p, size_t n)
{
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes)
    {
        if (cap >= bytes && p) return SYSMAT_OK;
        cudaFree(p);
        p = nullptr;
        cap = 0;
        if (cudaMalloc(&p, bytes ? bytes : 4) != cudaSuccess) { p = nullptr; return SYSMAT_ERR_NOMEM; }
        cap = bytes;
        return SYSMAT_OK;
    }
};

// Pinned staging for the bitmap file reader: per reader thread two pieces, a stream and an
// event per piece.  Made on the first file read of a device and kept (32 MB pinned per
// reader), since pinning that much memory costs more than reading a config-3 bitmap file.
// Readers: three quarters of the host threads, at most 12.  Measured on a 16-thread host, a
// legacy scatter() call that reads 9.1 GB of bitmap files from the page cache took 757 ms
// with 4 readers, 609 ms with 8 and 561 ms with 12; one thread reads the files alone in 2.2 s.
struct FileStaging {
    static constexpr int kMaxReaders = 12;
    static constexpr size_t kPiece = 16u << 20;
    unsigned char* piece[kMaxReaders][2] = {};
    cudaEvent_t done[kMaxReaders][2] = {};
    cudaStream_t stream[kMaxReaders] = {};
    int readers = 0;
    bool ready = false;
    int ensure()
    {
        if (ready) return SYSMAT_OK;
        const int hc = (int)std::thread::hardware_concurrency();
        readers = std::max(1, std::min(kMaxReaders, hc - hc / 4));
        for (int t = 0; t < readers; ++t) {
            if (!stream[t] && cudaStreamCreateWithFlags(&stream[t], cudaStreamNonBlocking) != cudaSuccess)
                return SYSMAT_ERR_CUDA;
            for (int b = 0; b < 2; ++b) {
                if (!piece[t][b] && cudaHostAlloc((void**)&piece[t][b], kPiece, cudaHostAllocDefault) != cudaSuccess) {
                    piece[t][b] = nullptr;
                    return SYSMAT_ERR_NOMEM;
                }
                if (!done[t][b] && cudaEventCreateWithFlags(&done[t][b], cudaEventDisableTiming) != cudaSuccess)
                    return SYSMAT_ERR_CUDA;
            }
        }
        ready = true;
        return SYSMAT_OK;
    }
};

struct LegacySlot {
    std::mutex mu;
    uint64_t key = 0;
    sysmat_ctx* ctx = nullptr;
    float* d_out = nullptr;
    size_t out_cap = 0;
    DevBuf pe, bm_crystal, bm_collimator;
    FileStaging staging;
};

LegacySlot& slot_for(int device)
{
    static LegacySlot slots[64];
    return slots[device & 63];
}

// Context for the given parameter contents (image rotation index excluded), re-used
// across calls on the same device.
int legacy_ctx(int device, const float* pC, const float* pD, const float* pI, const float* pP,
               LegacySlot& slot)
{
    float img[kNImage];
    std::memcpy(img, pI, sizeof(img));
    img[20] = 0.0f;
    uint64_t key = 1469598103934665603ull;
    key = fnv1a(key, pD, sizeof(float) * kNDetector);
    key = fnv1a(key, img, sizeof(img));
    if (pC) key = fnv1a(key, pC, sizeof(float) * kNCollimator);
    else key = fnv1a(key, "noC", 3);
    if (pP) key = fnv1a(key, pP, sizeof(float) * kNPhysics);
    else key = fnv1a(key, "noP", 3);
    if (slot.ctx && slot.key == key) return SYSMAT_OK;
    if (slot.ctx) { sysmat_destroy(slot.ctx); slot.ctx = nullptr; }
    int rc = sysmat_create(&slot.ctx, device, pC, pD, pI, pP);
    if (rc) return rc;
    slot.key = key;
    return SYSMAT_OK;
}

int legacy_out(LegacySlot& slot, size_t n)
{
    if (slot.out_cap >= n && slot.d_out) return SYSMAT_OK;
    cudaFree(slot.d_out);
    slot.d_out = nullptr;
    slot.out_cap = 0;
    if (cudaMalloc(&slot.d_out, sizeof(float) * n) != cudaSuccess) return SYSMAT_ERR_NOMEM;
    slot.out_cap = n;
    return SYSMAT_OK;
}

int select_device(int cuda_id)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return SYSMAT_ERR_CUDA;
    // the reference falls back to the current device when cuda_id is out of range
    // (scatter.cu:2034-2042)
    int dev = (cuda_id >= 0 && cuda_id < n) ? cuda_id : 0;
    if (cudaSetDevice(dev) != cudaSuccess) return SYSMAT_ERR_CUDA;
    return dev;
}

}  // namespace

extern "C" SYSMAT_API int PESysMatGen(float* parameter_Collimator, float* parameter_Detector,
                           float* parameter_Image, float* dst, int cuda_id)
{
    if (!parameter_Collimator || !parameter_Detector || !parameter_Image || !dst) return SYSMAT_ERR_ARG;
    const int dev = select_device(cuda_id);
    if (dev < 0) return dev;
    LegacySlot& slot = slot_for(dev);
    std::lock_guard<std::mutex> lock(slot.mu);
    int rc = legacy_ctx(dev, parameter_Collimator, parameter_Detector, parameter_Image, nullptr, slot);
    if (rc) return rc;
    const int D = slot.ctx->g.n_det;
    const long long V = slot.ctx->g.nvox;
    rc = legacy_out(slot, (size_t)D * (size_t)V);
    if (rc) return rc;
    rc = sysmat_pe(slot.ctx, parameter_Image[20], 0, D, 0, V, slot.d_out, V, SYSMAT_MODE_REFERENCE,
                   nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(dst, slot.d_out, sizeof(float) * (size_t)D * (size_t)V, cudaMemcpyDeviceToHost));
    return (int)V;
}

namespace {

// Write a device bitmap to a file the way the reference does (fopen "wb+", raw uint32).
int bitmap_to_file(const char* fname, const uint32_t* d_words, long long n)
{
    if (!fname) return SYSMAT_ERR_ARG;
    std::vector<uint32_t> h((size_t)n);
    if (cudaMemcpy(h.data(), d_words, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return SYSMAT_ERR_CUDA;
    FILE* f = std::fopen(fname, "wb+");
    if (!f) return SYSMAT_ERR_IO;
    const size_t w = std::fwrite(h.data(), sizeof(uint32_t), (size_t)n, f);
    std::fclose(f);
    return w == (size_t)n ? SYSMAT_OK : SYSMAT_ERR_IO;
}

// Read a bitmap file into device memory.  Like the reference (zero-initialised buffer and an
// unchecked fread, scatter.cu:2156-2159), a short file leaves the remaining words zero.  The
// file (gigabytes for a large system) streams through a pipeline: reader threads, each with two
// pinned staging pieces and its own stream, read interleaved pieces with pread and copy each
// to the device while reading the next, so the read, the copy and the other readers overlap.
int bitmap_from_file(const char* fname, uint32_t* d_words, long long n, int device, FileStaging& stg)
{
    if (!fname) return SYSMAT_ERR_ARG;
    const int fd = ::open(fname, O_RDONLY);
    if (fd < 0) return SYSMAT_ERR_IO;
    struct stat st;
    if (::fstat(fd, &st) != 0) {
        ::close(fd);
        return SYSMAT_ERR_IO;
    }
    const size_t want = sizeof(uint32_t) * (size_t)n;
    const size_t have = (size_t)st.st_size < want ? (size_t)st.st_size / sizeof(uint32_t) * sizeof(uint32_t) : want;
    int rc = stg.ensure();
    if (!rc && have < want) {
        std::fprintf(stderr, "sysmat: %s holds %zu of %lld bitmap words; the rest read as 0\n", fname,
                     have / sizeof(uint32_t), n);
        if (cudaMemset((unsigned char*)d_words + have, 0, want - have) != cudaSuccess) rc = SYSMAT_ERR_CUDA;
    }
    if (rc) {
        ::close(fd);
        return rc;
    }
    constexpr size_t kPiece = FileStaging::kPiece;
    const size_t n_pieces = (have + kPiece - 1) / kPiece;
    const int n_readers = (int)std::min<size_t>(n_pieces, (size_t)stg.readers);
    int status[FileStaging::kMaxReaders] = {};
    auto reader = [&](int t) {
        int r = cudaSetDevice(device) == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
        int use = 0;
        for (size_t k = (size_t)t; k < n_pieces && r == SYSMAT_OK; k += (size_t)n_readers, ++use) {
            const int b = use & 1;
            unsigned char* h = stg.piece[t][b];
            const size_t off = k * kPiece, len = std::min(kPiece, have - off);
            if (cudaEventSynchronize(stg.done[t][b]) != cudaSuccess) {   // the piece's last copy is done
                r = SYSMAT_ERR_CUDA;
                break;
            }
            size_t got = 0;
            while (got < len) {
                const ssize_t q = ::pread(fd, h + got, len - got, (off_t)(off + got));
                if (q <= 0) break;
                got += (size_t)q;
            }
            if (got != len) {
                r = SYSMAT_ERR_IO;
                break;
            }
            if (cudaMemcpyAsync((unsigned char*)d_words + off, h, len, cudaMemcpyHostToDevice, stg.stream[t]) != cudaSuccess ||
                cudaEventRecord(stg.done[t][b], stg.stream[t]) != cudaSuccess)
                r = SYSMAT_ERR_CUDA;
        }
        if (cudaStreamSynchronize(stg.stream[t]) != cudaSuccess && r == SYSMAT_OK) r = SYSMAT_ERR_CUDA;
        status[t] = r;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < n_readers; ++t) pool.emplace_back(reader, t);
    if (n_readers > 0) reader(0);
    for (auto& th : pool) th.join();
    ::close(fd);
    for (int t = 0; t < n_readers; ++t)
        if (status[t]) return status[t];
    return SYSMAT_OK;
}

// Compute (flag set) or load a relationship bitmap for the reference-compatible scatter
// programs (scatter.cu:2116-2167, :2246-2301).
int legacy_bitmap(sysmat_ctx* ctx, bool crystal, bool compute, const char* fname, DevBuf& buf,
                  FileStaging& stg)
{
    const long long n = crystal ? sysmat_bitmap_crystal_words(ctx) : sysmat_bitmap_collimator_words(ctx);
    if (n < 0) return (int)n;
    int rc = buf.ensure(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    if (rc) return rc;
    uint32_t* words = (uint32_t*)buf.p;
    if (compute) {
        rc = crystal ? sysmat_bitmap_crystal(ctx, words, nullptr) : sysmat_bitmap_collimator(ctx, words, nullptr);
        if (rc) return rc;
        return bitmap_to_file(fname, words, n);
    }
    return bitmap_from_file(fname, words, n, ctx->device, stg);
}

int legacy_scatter(int cuda_id, float* pC, float* pD, float* pI, float* pP, float* pe,
                   const char* f_crystal, const char* f_collimator, float* dst, int parts,
                   int hole_model, bool comp_crystal, bool comp_collimator)
{
    if (!pD || !pI || !pP || !dst) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_COLLIMATOR) && !pC) return SYSMAT_ERR_ARG;
    if ((parts & SYSMAT_SCATTER_CRYSTAL) && !pe) return SYSMAT_ERR_ARG;
    const int dev = select_device(cuda_id);
    if (dev < 0) return dev;
    LegacySlot& slot = slot_for(dev);
    std::lock_guard<std::mutex> lock(slot.mu);
    int rc = legacy_ctx(dev, (parts & SYSMAT_SCATTER_COLLIMATOR) ? pC : nullptr, pD, pI, pP, slot);
    if (rc) return rc;
    sysmat_ctx* ctx = slot.ctx;
    const int D = ctx->g.n_det;
    const long long V = ctx->g.nvox;
    const size_t nel = (size_t)D * (size_t)V;
    if (parts & SYSMAT_SCATTER_CRYSTAL) {
        rc = legacy_bitmap(ctx, true, comp_crystal, f_crystal, slot.bm_crystal, slot.staging);
        if (rc) return rc;
        rc = slot.pe.ensure(sizeof(float) * nel);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpy(slot.pe.p, pe, sizeof(float) * nel, cudaMemcpyHostToDevice));
    }
    if (parts & SYSMAT_SCATTER_COLLIMATOR) {
        rc = legacy_bitmap(ctx, false, comp_collimator, f_collimator, slot.bm_collimator, slot.staging);
        if (rc) return rc;
    }
    rc = legacy_out(slot, nel);
    if (rc) return rc;
    rc = sysmat_scatter_prepare(ctx, parts, (const uint32_t*)slot.bm_crystal.p,
                                (const uint32_t*)slot.bm_collimator.p, nullptr);
    if (rc) return rc;
    rc = sysmat_scatter(ctx, parts, hole_model, pI[20], (const float*)slot.pe.p, 0, D, 0, V, slot.d_out,
                        V, nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(dst, slot.d_out, sizeof(float) * nel, cudaMemcpyDeviceToHost));
    return (int)V;
}

}  // namespace

extern "C" SYSMAT_API int scatter(float* parameter_Collimator, float* parameter_Detector,
                                  float* parameter_Image, float* parameter_Physics, float* PE_SysMat,
                                  const char* FnameGeoCrystal, const char* FnameGeoCollimator,
                                  float* dst, int cuda_id)
{
    if (!parameter_Physics) return SYSMAT_ERR_ARG;
    const bool cc = (int)std::floor(parameter_Physics[8]) == 1;                 // scatter.cu:2116
    const bool ch = (int)std::floor(parameter_Physics[9] + 0.001f) == 1;        // scatter.cu:2246
    return legacy_scatter(cuda_id, parameter_Collimator, parameter_Detector, parameter_Image,
                          parameter_Physics, PE_SysMat, FnameGeoCrystal, FnameGeoCollimator, dst,
                          SYSMAT_SCATTER_CRYSTAL | SYSMAT_SCATTER_COLLIMATOR,
                          SYSMAT_HOLE_MODEL_COMBINED, cc, ch);
}

extern "C" SYSMAT_API int scatter_collimator(float* parameter_Collimator, float* parameter_Detector,
                                             float* parameter_Image, float* parameter_Physics,
                                             float* PE_SysMat, const char* FnameGeo, float* dst,
                                             int cuda_id)
{
    if (!parameter_Physics) return SYSMAT_ERR_ARG;
    const bool ch = (int)std::floor(parameter_Physics[9]) == 1;   // ScatterGen_Collimator/scatter.cu:1617
    (void)PE_SysMat;   // the collimator part does not read the PE matrix
    return legacy_scatter(cuda_id, parameter_Collimator, parameter_Detector, parameter_Image,
                          parameter_Physics, nullptr, nullptr, FnameGeo, dst, SYSMAT_SCATTER_COLLIMATOR,
                          SYSMAT_HOLE_MODEL_VARIANT, false, ch);
}

extern "C" SYSMAT_API int scatter_crystal(float* parameter_Detector, float* parameter_Image,
                                          float* parameter_Physics, float* PE_SysMat, const char* FnameGeo,
                                          float* dst, int cuda_id)
{
    if (!parameter_Physics) return SYSMAT_ERR_ARG;
    const bool cc = (int)std::floor(parameter_Physics[8]) == 1;   // ScatterGen_Crystal/scatter.cu:1626
    return legacy_scatter(cuda_id, nullptr, parameter_Detector, parameter_Image, parameter_Physics,
                          PE_SysMat, FnameGeo, nullptr, dst, SYSMAT_SCATTER_CRYSTAL,
                          SYSMAT_HOLE_MODEL_COMBINED, cc, false);
}

// Internal C names used by the C++-linkage aliases in cxx_abi.cpp (not in sysmat.h).
extern "C" int sysmat_legacy_pe(float* pC, float* pD, float* pI, float* dst, int cuda_id)
{
    return PESysMatGen(pC, pD, pI, dst, cuda_id);
}
extern "C" int sysmat_legacy_scatter(float* pC, float* pD, float* pI, float* pP, float* pe,
                                     const char* fc, const char* fh, float* dst, int cuda_id)
{
    return scatter(pC, pD, pI, pP, pe, fc, fh, dst, cuda_id);
}
extern "C" int sysmat_legacy_scatter_collimator(float* pC, float* pD, float* pI, float* pP, float* pe,
                                                const char* fh, float* dst, int cuda_id)
{
    return scatter_collimator(pC, pD, pI, pP, pe, fh, dst, cuda_id);
}
extern "C" int sysmat_legacy_scatter_crystal(float* pD, float* pI, float* pP, float* pe, const char* fc,
                                             float* dst, int cuda_id)
{
    return scatter_crystal(pD, pI, pP, pe, fc, dst, cuda_id);
}
