// Photoelectric matrix entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc when they need a matrix block: an application that
// hands all device memory to its own pool at start-up, a host whose plug-in contract
// forbids allocation after initialisation, or a latency-critical loop where the implicit
// synchronisation of cudaMalloc/cudaFree is not acceptable.  sysmat_pe_noalloc serves them:
// the caller passes the parameter arrays (host memory) and the output block (device
// memory); every other buffer the photoelectric kernel needs (the uploaded parameter
// arrays, the derived crystal and hole tables, the work counter and the status word) lives
// in one statically sized device array of this file.
//
// That array is a __device__ variable: each GPU that loads the library holds it (about
// 1.6 MB) until the process exits.  In host code its name is only a host-side stand-in, so
// the device address is obtained with cudaGetSymbolAddress, once per device, with that
// device current, on the first call made on it.  That first call should come before any
// CUDA stream capture.  All calls share the array and it keeps the last call's contents:
// each call re-uploads the parameters, rebuilds the tables and clears the counter and
// status before its launch.  Calls whose work overlaps on the GPU (two streams, two host
// threads on one device) race on the array; serialise them.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda.h>

#include "../../include/sysmat.h"
#include "geom.cuh"
#include "pe.cuh"

namespace sysmat {
int sysmat_decode_geometry(const float* pC, const float* pD, const float* pI, DevGeom& g,
                           int& n_holes0);
}

using namespace sysmat;

namespace {

// Capacities of the static scratch: the reference's own table limits (80000-float
// detector table: 6666 crystals; collimator table: 8877 holes).
constexpr int kNoAllocMaxCrystals = 6666;
constexpr int kNoAllocMaxHoles = 8877;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr size_t kOffDet = 0;                                                  // raw detector
constexpr size_t kOffCol = align256(kOffDet + sizeof(float) * kNDetector);    // raw collimator
constexpr size_t kOffCry = align256(kOffCol + sizeof(float) * kNCollimator);  // 4 float4 / crystal
constexpr size_t kOffHole = align256(kOffCry + sizeof(float4) * 4 * kNoAllocMaxCrystals);
constexpr size_t kOffCounter = align256(kOffHole + sizeof(float4) * 3 * kNoAllocMaxHoles);
constexpr size_t kOffStatus = kOffCounter + 256;
constexpr size_t kScratchBytes = kOffStatus + 256;

static __device__ __align__(256) unsigned char g_pe_scratch[kScratchBytes];

// Device address of g_pe_scratch per device, with the CUDA context it was looked up in.
// A symbol's address belongs to one context: after cudaDeviceReset, or when the caller makes
// another (non-primary) context current on the same device, the address is looked up again.
std::mutex g_setup_mu;
struct ScratchSlot {
    CUcontext ctx;
    unsigned char* ptr;
};
ScratchSlot g_scratch[64] = {};
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn g_ctx_get_current = nullptr;

int current_context(CUcontext* ctx)
{
    if (!g_ctx_get_current) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return SYSMAT_ERR_CUDA;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    return g_ctx_get_current(ctx) == CUDA_SUCCESS ? SYSMAT_OK : SYSMAT_ERR_CUDA;
}

int scratch_for_current_device(unsigned char** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SYSMAT_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    CUcontext ctx = nullptr;
    if (current_context(&ctx)) return SYSMAT_ERR_CUDA;
    if (!ctx || !g_scratch[dev].ptr || g_scratch[dev].ctx != ctx) {
        // the lookup also binds the runtime's context when this thread has none yet
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_pe_scratch) != cudaSuccess || !p) return SYSMAT_ERR_CUDA;
        if (current_context(&ctx) || !ctx) return SYSMAT_ERR_CUDA;
        g_scratch[dev].ctx = ctx;
        g_scratch[dev].ptr = static_cast<unsigned char*>(p);
    }
    *out = g_scratch[dev].ptr;
    return SYSMAT_OK;
}

}  // namespace

extern "C" SYSMAT_API int sysmat_pe_noalloc(const float* pC, const float* pD, const float* pI,
                                            float rotation, int det_begin, int det_count,
                                            long long vox_begin, long long vox_count, float* d_out,
                                            long long ld, int mode, void* stream)
{
    if (!pC || !pD || !pI || !d_out) return SYSMAT_ERR_ARG;
    if (mode != SYSMAT_MODE_REFERENCE && mode != SYSMAT_MODE_PRECISE) return SYSMAT_ERR_ARG;
    // sizes first, against the static scratch, with a message naming the limit
    const double n_det = std::floor((double)(pD[0] + 0.000001f));
    const int n_layers = (int)std::floor(pC[0] + 0.000001f);
    double n_holes = 0;
    for (int m = 0; m < n_layers && m < kMaxLayers; ++m) n_holes += std::floor(pC[(m + 1) * 10]);
    if (n_det > kNoAllocMaxCrystals || n_holes > kNoAllocMaxHoles) {
        std::fprintf(stderr, "sysmat_pe_noalloc: %.0f crystals / %.0f holes exceed the static scratch "
                     "(at most %d crystals and %d holes)\n", n_det, n_holes, kNoAllocMaxCrystals,
                     kNoAllocMaxHoles);
        return SYSMAT_ERR_CAPACITY;
    }
    DevGeom g;
    int nh0 = 0;
    int rc = sysmat_decode_geometry(pC, pD, pI, g, nh0);
    if (rc) return rc;
    if (det_begin < 0 || det_count < 0 || det_begin + det_count > g.n_det) return SYSMAT_ERR_ARG;
    if (vox_begin < 0 || vox_count < 0 || vox_begin + vox_count > g.nvox || ld < vox_count)
        return SYSMAT_ERR_ARG;
    if (det_count == 0 || vox_count == 0) return SYSMAT_OK;

    unsigned char* base = nullptr;
    rc = scratch_for_current_device(&base);
    if (rc) return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return SYSMAT_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;

    float* d_det = reinterpret_cast<float*>(base + kOffDet);
    float* d_col = reinterpret_cast<float*>(base + kOffCol);
    float4* t = reinterpret_cast<float4*>(base + kOffCry);
    float4* th = reinterpret_cast<float4*>(base + kOffHole);
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(base + kOffCounter);
    int* status = reinterpret_cast<int*>(base + kOffStatus);
    const int D = g.n_det, H = g.n_holes, Hs = H > 0 ? H : 1;
    g.raw_det = d_det;
    g.cry.pos = t;
    g.cry.size = t + D;
    g.cry.mu = t + 2 * D;
    g.cry.trig = t + 3 * D;
    g.hole.a = th;
    g.hole.b = th + Hs;
    g.hole.raw = th + 2 * Hs;

    if (cudaMemcpyAsync(d_det, pD, sizeof(float) * kNDetector, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(d_col, pC, sizeof(float) * kNCollimator, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return SYSMAT_ERR_CUDA;
    derive_crystals<<<(D + 127) / 128, 128, 0, s>>>(d_det, g.fov, D, t, t + D, t + 2 * D, t + 3 * D);
    if (H > 0) derive_holes<<<(H + 127) / 128, 128, 0, s>>>(d_col, g.fov, H, th, th + Hs, th + 2 * Hs);
    if (cudaGetLastError() != cudaSuccess) return SYSMAT_ERR_CUDA;
    // counter and status must start at zero: the array keeps the previous call's values
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess)
        return SYSMAT_ERR_CUDA;
    PeLaunch L;
    L.det_begin = det_begin;
    L.det_count = det_count;
    L.vox_begin = vox_begin;
    L.vox_count = vox_count;
    L.ld = ld;
    L.rotation = rotation;
    L.out = d_out;
    L.work_counter = counter;
    L.status = status;
    L.counters = nullptr;
    if (launch_pe(g, L, mode, sms, s)) return SYSMAT_ERR_CUDA;
    int st = 0;
    if (cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return SYSMAT_ERR_CUDA;
    return (st & kStatusCapacity) ? SYSMAT_ERR_CAPACITY : SYSMAT_OK;
}
