// Whole photoelectric matrix of one rotation -> compressed file, computed and compressed on
// the device block by block so that neither the dense matrix nor its CSR has to fit anywhere
// at once.  The reference writes the dense float matrix (PEGen_CircularHole.cpp:141-147:
// D*V floats per rotation, 4.83 GB for a 4096-crystal, 96x96x32 system); at the production
// threshold (1e-9) most of it is attenuated to nothing.
//
// File layout (little-endian):
//   header  char magic[8] = "SMCSR001"; int64 rows (crystals); int64 cols (voxels);
//           float threshold; int32 mode; int64 reserved
//   blocks  repeated until end of file: int64 first_row; int64 n_rows; int64 nnz;
//           int64 row_ptr[n_rows + 1] (block-relative, row_ptr[0] = 0);
//           int64 col[nnz] (voxel index); float val[nnz]
// Rows appear in ascending order; within a row, columns ascend.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/sysmat.h"
#include "ctx.cuh"

namespace {

struct DevMem {
    void* p = nullptr;
    ~DevMem() { cudaFree(p); }
    bool alloc(size_t n) { return cudaMalloc(&p, n == 0 ? 1 : n) == cudaSuccess; }
};

struct HostMem {
    void* p = nullptr;
    ~HostMem() { cudaFreeHost(p); }
    bool alloc(size_t n) { return cudaMallocHost(&p, n == 0 ? 1 : n) == cudaSuccess; }
};

bool put(FILE* f, const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }

}  // namespace

extern "C" SYSMAT_API int sysmat_pe_csr_file(sysmat_ctx* ctx, float rotation, const char* path, float threshold,
                                             int mode, int rows_per_block, long long* nnz_total, void* stream)
{
    if (!ctx || !path || rows_per_block < 0 || !(threshold >= 0.0f)) return SYSMAT_ERR_ARG;
    if (mode != SYSMAT_MODE_REFERENCE && mode != SYSMAT_MODE_PRECISE && mode != SYSMAT_MODE_FP64 &&
        mode != SYSMAT_MODE_LOCAL)
        return SYSMAT_ERR_ARG;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != ctx->device) return SYSMAT_ERR_ARG;
    const long long D = ctx->g.n_det, V = ctx->g.nvox;
    long long rb = rows_per_block;
    if (rb == 0) rb = (1ll << 28) / (V > 0 ? V : 1);          // about 1 GB of dense block
    if (rb < 1) rb = 1;
    if (rb > D) rb = D > 0 ? D : 1;
    const size_t cells = (size_t)rb * (size_t)V;
    DevMem dense, row_nnz, row_ptr, col, val;
    HostMem h_ptr, h_col, h_val;
    if (!dense.alloc(sizeof(float) * cells) || !row_nnz.alloc(sizeof(long long) * rb) ||
        !row_ptr.alloc(sizeof(long long) * (rb + 1)) || !col.alloc(sizeof(long long) * cells) ||
        !val.alloc(sizeof(float) * cells) || !h_ptr.alloc(sizeof(long long) * (rb + 1)) ||
        !h_col.alloc(sizeof(long long) * cells) || !h_val.alloc(sizeof(float) * cells))
        return SYSMAT_ERR_NOMEM;
    FILE* f = std::fopen(path, "wb");
    if (!f) return SYSMAT_ERR_IO;
    cudaStream_t s = (cudaStream_t)stream;
    char magic[8];
    std::memcpy(magic, "SMCSR001", 8);
    const long long reserved = 0;
    bool ok = put(f, magic, 8) && put(f, &D, 8) && put(f, &V, 8) && put(f, &threshold, 4) && put(f, &mode, 4) &&
              put(f, &reserved, 8);
    long long total = 0;
    int rc = ok ? SYSMAT_OK : SYSMAT_ERR_IO;
    for (long long d0 = 0; rc == SYSMAT_OK && d0 < D; d0 += rb) {
        const long long n = (D - d0 < rb) ? D - d0 : rb;
        rc = sysmat_pe(ctx, rotation, (int)d0, (int)n, 0, V, (float*)dense.p, V, mode, stream);
        if (rc) break;
        rc = sysmat_csr_count((const float*)dense.p, (int)n, V, V, threshold, (long long*)row_nnz.p,
                              (long long*)row_ptr.p, stream);
        if (rc) break;
        if (cudaMemcpyAsync(h_ptr.p, row_ptr.p, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = SYSMAT_ERR_CUDA;
            break;
        }
        const long long nnz = ((const long long*)h_ptr.p)[n];
        rc = sysmat_csr_fill((const float*)dense.p, (int)n, V, V, threshold, 0, (const long long*)row_ptr.p,
                             (long long*)col.p, (float*)val.p, stream);
        if (rc) break;
        if ((nnz && (cudaMemcpyAsync(h_col.p, col.p, sizeof(long long) * nnz, cudaMemcpyDeviceToHost, s) !=
                         cudaSuccess ||
                     cudaMemcpyAsync(h_val.p, val.p, sizeof(float) * nnz, cudaMemcpyDeviceToHost, s) !=
                         cudaSuccess)) ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = SYSMAT_ERR_CUDA;
            break;
        }
        if (!(put(f, &d0, 8) && put(f, &n, 8) && put(f, &nnz, 8) && put(f, h_ptr.p, sizeof(long long) * (n + 1)) &&
              put(f, h_col.p, sizeof(long long) * nnz) && put(f, h_val.p, sizeof(float) * nnz)))
            rc = SYSMAT_ERR_IO;
        total += nnz;
    }
    if (std::fclose(f) != 0 && rc == SYSMAT_OK) rc = SYSMAT_ERR_IO;
    if (nnz_total) *nnz_total = total;
    return rc;
}
