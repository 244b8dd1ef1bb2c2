// Host side of the forward projection and its vector-Jacobian product (pe_adjoint.cuh).
//
// The reference has no adjoint: it writes the dense matrix (PESysMatGen.cu:1368-1437) and a
// reconstruction or calibration code multiplies it.  Here p = A(theta) x and
// g = d(u^T A(theta) x)/d(theta) are computed brick by brick with A recomputed, never stored,
// so a calibration loop over collimator parameters needs no matrix memory.
#include <cstdio>

#include "../../include/sysmat.h"
#include "ctx.cuh"
#include "pe.cuh"

using namespace sysmat;

namespace {

int adjoint_call(sysmat_ctx* ctx, float rotation, int det_begin, int det_count, const float* d_x,
                 const float* d_u, double* d_out, int kind, void* stream)
{
    if (!ctx || det_begin < 0 || det_count < 0 || det_begin + det_count > ctx->g.n_det) return SYSMAT_ERR_ARG;
    const size_t n_out = kind == 0 ? (size_t)det_count
                       : kind == 1 ? (size_t)(SYSMAT_THETA_N + 1) : (size_t)ctx->g.nvox;
    if ((n_out && !d_out) || (det_count && ((kind != 2 && !d_x) || (kind >= 1 && !d_u)))) return SYSMAT_ERR_ARG;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != ctx->device) return SYSMAT_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (n_out && cudaMemsetAsync(d_out, 0, sizeof(double) * n_out, s) != cudaSuccess) return SYSMAT_ERR_CUDA;
    if (det_count == 0) return SYSMAT_OK;
    if (cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return SYSMAT_ERR_CUDA;
    AdjLaunch L;
    L.det_begin = det_begin;
    L.det_count = det_count;
    L.rotation = rotation;
    L.x = d_x;
    L.u = d_u;
    L.p = kind == 0 ? d_out : nullptr;
    L.grad = kind == 1 ? d_out : nullptr;
    L.q = kind == 2 ? d_out : nullptr;
    L.work_counter = ctx->d_counter;
    if (launch_pe_adjoint(ctx->g, L, kind, ctx->num_sms, s)) {
        std::fprintf(stderr, "sysmat: adjoint launch failed: %s\n", cudaGetErrorString(cudaGetLastError()));
        return SYSMAT_ERR_CUDA;
    }
    return SYSMAT_OK;
}

}  // namespace

extern "C" SYSMAT_API int sysmat_project(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                         const float* d_x, double* d_p, void* stream)
{
    return adjoint_call(ctx, rotation, det_begin, det_count, d_x, nullptr, d_p, 0, stream);
}

extern "C" SYSMAT_API int sysmat_vjp(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                     const float* d_x, const float* d_u, double* d_grad, void* stream)
{
    return adjoint_call(ctx, rotation, det_begin, det_count, d_x, d_u, d_grad, 1, stream);
}

extern "C" SYSMAT_API int sysmat_backproject(sysmat_ctx* ctx, float rotation, int det_begin, int det_count,
                                             const float* d_u, double* d_q, void* stream)
{
    return adjoint_call(ctx, rotation, det_begin, det_count, nullptr, d_u, d_q, 2, stream);
}
