// Test infrastructure only: the reference's elliptical-cylinder chord
// (PEGen_RayTracing_CircularHole/PESysMatGen.cu:801-947, a __device__ function the reference
// kernels never call) evaluated on arrays of arguments, so that golden vectors can pin the
// oracle's restatement.  The unmodified reference source is compiled into this translation
// unit by oracle/Makefile (-I to its directory); nothing of it is copied here.
#include <cuda_runtime.h>

#include "PESysMatGen.cu"

__global__ void ref_ell_kernel(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + 13 * i;
    out[i] = length_ellipticalcylinder_ray(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9],
                                           a[10], a[11], a[12]);
}

// h_in: 13 floats per item (x_in, y_in, z_in, x_out, y_out, z_out, xc, y1, y2, zc, rho_x, rho_z,
// theta); h_out: n floats.  Returns 0 on success.
extern "C" int ref_ell_chords(const float* h_in, float* h_out, int n, int cuda_id)
{
    if (cudaSetDevice(cuda_id) != cudaSuccess) return -1;
    float *d_in = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, sizeof(float) * 13 * (size_t)n) != cudaSuccess) return -2;
    if (cudaMalloc(&d_out, sizeof(float) * (size_t)n) != cudaSuccess) { cudaFree(d_in); return -2; }
    cudaMemcpy(d_in, h_in, sizeof(float) * 13 * (size_t)n, cudaMemcpyHostToDevice);
    ref_ell_kernel<<<(n + 255) / 256, 256>>>(d_in, d_out, n);
    const cudaError_t e = cudaMemcpy(h_out, d_out, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    return e == cudaSuccess ? 0 : -3;
}
