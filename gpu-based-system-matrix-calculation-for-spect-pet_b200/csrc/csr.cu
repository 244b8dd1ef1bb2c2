// Dense block -> CSR on the device (entries with value > threshold), for streaming large
// system matrices to the host in compressed form (production matrices use 1e-9).
//
// Two passes over the dense block: a per-row count (one warp per row, ballot + popc), a
// single-block exclusive scan of the counts into row pointers, then an ordered fill (one
// warp per row; ballot compaction keeps column order).  Column indices are the voxel
// indices of the block's columns plus col_offset.
#include <cuda_runtime.h>

#include "../../include/sysmat.h"

namespace {

constexpr int kWarps = 8;

__global__ void csr_count_kernel(const float* __restrict__ a, int rows, long long cols, long long ld,
                                 float thr, long long* __restrict__ nnz)
{
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (row >= rows) return;
    const float* r = a + (long long)row * ld;
    long long c = 0;
    for (long long j = lane; j < cols; j += 32) c += (__ldg(&r[j]) > thr);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if (lane == 0) nnz[row] = c;
}

// Exclusive scan of rows counts into row_ptr[0..rows]; one block of 1024 threads.
__global__ void csr_scan_kernel(const long long* __restrict__ nnz, int rows, long long* __restrict__ ptr)
{
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const int per = (rows + 1023) / 1024;
    const int b = t * per, e = min(rows, b + per);
    long long s = 0;
    for (int i = b; i < e; ++i) s += nnz[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {          // inclusive Hillis-Steele scan
        const long long v = (t >= off) ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = part[t] - s;                          // exclusive start of this thread
    for (int i = b; i < e; ++i) { ptr[i] = run; run += nnz[i]; }
    if (t == 1023) ptr[rows] = part[1023];
}

__global__ void csr_fill_kernel(const float* __restrict__ a, int rows, long long cols, long long ld,
                                float thr, long long col_offset, const long long* __restrict__ ptr,
                                long long* __restrict__ col_idx, float* __restrict__ val)
{
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (row >= rows) return;
    const float* r = a + (long long)row * ld;
    long long pos = ptr[row];
    for (long long j0 = 0; j0 < cols; j0 += 32) {
        const long long j = j0 + lane;
        const float v = (j < cols) ? __ldg(&r[j]) : 0.0f;
        const bool keep = (j < cols) && v > thr;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const long long p = pos + __popc(m & ((1u << lane) - 1u));
            col_idx[p] = j + col_offset;
            val[p] = v;
        }
        pos += __popc(m);
    }
}

}  // namespace

extern "C" SYSMAT_API int sysmat_csr_count(const float* d_dense, int rows, long long cols, long long ld,
                                           float threshold, long long* d_row_nnz, long long* d_row_ptr,
                                           void* stream)
{
    if (!d_dense || !d_row_nnz || !d_row_ptr || rows < 0 || cols < 0 || ld < cols) return SYSMAT_ERR_ARG;
    if (rows == 0) return cudaMemsetAsync(d_row_ptr, 0, sizeof(long long), (cudaStream_t)stream) == cudaSuccess
                              ? SYSMAT_OK : SYSMAT_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    csr_count_kernel<<<(rows + kWarps - 1) / kWarps, kWarps * 32, 0, s>>>(d_dense, rows, cols, ld, threshold,
                                                                          d_row_nnz);
    csr_scan_kernel<<<1, 1024, 0, s>>>(d_row_nnz, rows, d_row_ptr);
    return cudaGetLastError() == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
}

extern "C" SYSMAT_API int sysmat_csr_fill(const float* d_dense, int rows, long long cols, long long ld,
                                          float threshold, long long col_offset, const long long* d_row_ptr,
                                          long long* d_col_idx, float* d_val, void* stream)
{
    if (!d_dense || !d_row_ptr || rows < 0 || cols < 0 || ld < cols) return SYSMAT_ERR_ARG;
    if (rows == 0) return SYSMAT_OK;
    if (!d_col_idx || !d_val) return SYSMAT_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    csr_fill_kernel<<<(rows + kWarps - 1) / kWarps, kWarps * 32, 0, s>>>(d_dense, rows, cols, ld, threshold,
                                                                         col_offset, d_row_ptr, d_col_idx, d_val);
    return cudaGetLastError() == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
}
