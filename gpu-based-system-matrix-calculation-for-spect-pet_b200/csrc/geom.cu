// Geometry setup on the device: derived per-crystal and per-hole tables, and the slow
// (axis-parallel) path of the box chords.
//
// Derived values are computed on the GPU with the same float operations the reference
// kernels use inline (PESysMatGen.cu:1058-1068, :1124-1135, :1159-1166;
// scatter.cu:1465-1479), so they round exactly as the reference's own copies do.
#include "pe.cuh"
#include "../../include/sysmat.h"

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

// One thread per hole: (rho_x, rho_z, theta) -> (rho_x, rho_z, cos theta, sin theta), with the
// float cos/sin the reference's elliptical chord evaluates (PESysMatGen.cu:832-836);
// rho_x <= 0 marks a circular hole (stored as 0).
__global__ void derive_shapes(const float* __restrict__ s, int n, float4* out)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    const float rx = s[3 * h], rz = s[3 * h + 1], th = s[3 * h + 2];
    out[h] = rx > 0.0f ? make_float4(rx, rz, cosf(th), sinf(th)) : make_float4(0.0f, 0.0f, 1.0f, 0.0f);
}

// The same shapes for the FP64 mode: cos and sin of the float angle in double, as the FP64
// restatement evaluates them.
__global__ void derive_shapes64(const float* __restrict__ s, int n, D4* out)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    const float rx = s[3 * h], rz = s[3 * h + 1];
    const double th = (double)s[3 * h + 2];
    out[h] = rx > 0.0f ? D4{(double)rx, (double)rz, cos(th), sin(th)} : D4{0.0, 0.0, 1.0, 0.0};
}

// Diagnostic: the elliptical-cylinder chord on arrays of arguments (13 per item, as
// sysmat_ell_chords documents), one thread per item.
__global__ void ell_chords_kernel(const float* __restrict__ a, float* __restrict__ out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* p = a + 13 * (long long)i;
    out[i] = ell_chord(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], p[11], cosf(p[12]),
                       sinf(p[12]));
}

// FP64 tables: one thread per crystal, then one per hole (all layers), with the double
// operations of the FP64 restatement of PESysMatGen.cu:1058-1068, :1124-1135, :1159-1166.
__global__ void derive_tables64(const float* __restrict__ det, const float* __restrict__ col, float fov, int n_det,
                                int n_holes, D4* cry_pos, D4* cry_size, D4* cry_trig, D4* hole_a, D4* hole_b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double f = (double)fov;
    if (i < n_det) {
        const float* p = det + 12 * i;
        const double rot = (double)p[11];
        cry_pos[i] = D4{(double)p[1], (double)p[2] + f, (double)p[3], (double)p[7]};
        cry_size[i] = D4{(double)p[4], (double)p[5], (double)p[6], (double)p[8]};
        cry_trig[i] = D4{cos(rot), sin(rot), cos(-rot), sin(-rot)};
    } else if (i < n_det + n_holes) {
        const int h = i - n_det;
        const float* p = col + 100 + 9 * h;
        const double y1 = (double)p[1] + f, y2 = (double)p[2] + f, r = (double)p[4];
        hole_a[h] = D4{(double)p[0], y1, y2, (double)p[3]};
        hole_b[h] = D4{r, (double)p[5], (y1 + y2) / 2.0, sqrt(r * r * 4.0 + (y1 - y2) * (y1 - y2)) / 2.0};
    }
}

}  // namespace sysmat

extern "C" SYSMAT_API int sysmat_ell_chords(const float* d_args, float* d_out, int n, void* stream)
{
    if (n < 0 || (n > 0 && (!d_args || !d_out))) return SYSMAT_ERR_ARG;
    if (n == 0) return SYSMAT_OK;
    sysmat::ell_chords_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_args, d_out, n);
    return cudaGetLastError() == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
}
