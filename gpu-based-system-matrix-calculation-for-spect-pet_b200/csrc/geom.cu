// Geometry setup on the device: derived per-crystal and per-hole tables, and the slow
// (axis-parallel) path of the box chords.
//
// Derived values are computed on the GPU with the same float operations the reference
// kernels use inline (PESysMatGen.cu:1058-1068, :1124-1135, :1159-1166;
// scatter.cu:1465-1479), so they round exactly as the reference's own copies do.
#include "pe.cuh"

namespace sysmat {

// One thread per crystal.
__global__ void derive_crystals(const float* __restrict__ det, float fov, int n, float4* pos,
                                float4* size, float4* mu, float4* trig)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const float* p = det + 12 * d;
    const float w = p[4], t = p[5], h = p[6], rot = p[11];
    pos[d] = make_float4(p[1], p[2] + fov, p[3], rot);
    size[d] = make_float4(w, t, h, sqrtf(w * w + h * h + t * t));
    mu[d] = make_float4(p[7], p[8], p[9], p[10]);
    trig[d] = make_float4(cosf(rot), sinf(rot), cosf(-rot), sinf(-rot));
}

// One thread per hole (all layers, global numbering).
__global__ void derive_holes(const float* __restrict__ col, float fov, int n, float4* a, float4* b,
                             float4* raw)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    const float* p = col + 100 + 9 * h;
    const float y1 = p[1] + fov, y2 = p[2] + fov, r = p[4];
    a[h] = make_float4(p[0], y1, y2, p[3]);
    const float yc = (y1 + y2) / 2.0f;
    const float crit = sqrtf(r * r * 4 + (y1 - y2) * (y1 - y2)) / 2.0f;
    b[h] = make_float4(r, p[5], yc, crit);
    raw[h] = make_float4(p[0], p[1], p[2], p[3]);
}

}  // namespace sysmat
