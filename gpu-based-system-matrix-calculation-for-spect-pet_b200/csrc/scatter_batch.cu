// Batched primary-Compton scatter: many (system, rotation, detector x voxel block) scatter
// tasks in one persistent launch over a device work queue, replayed as a CUDA graph.
//
// The reference computes the scatter of one geometry per host call, one launch per part
// (ScatterGen_RayTracing_CircularHole/scatter.cu:2169-2194, :2303-2329).  Tasks of a design
// sweep differ in pair-table and attenuator-list lengths (hole count, crystal layout) and in
// how many items survive the energy window, so per-task launches leave the GPU idle in each
// launch's tail and between launches.  A plan queues the (row, voxel block) items of every task
// and one launch drains the queue; each item runs the single launch's block code
// (scatter_rows), so every element is bit-identical to a per-task sysmat_scatter.
#include <cstdio>
#include <vector>

#include "../../include/sysmat.h"
#include "ctx.cuh"
#include "scatter.cuh"

using namespace sysmat;

struct sysmat_scatter_plan {
    int device = -1;
    int num_sms = 0;
    DevGeom* d_geoms = nullptr;
    ScatterTask* d_tasks = nullptr;
    unsigned long long* d_counter = nullptr;
    ScatterBatchLaunch launch{};
    cudaStream_t capture = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" SYSMAT_API int sysmat_scatter_batch_destroy(sysmat_scatter_plan* p)
{
    if (!p) return SYSMAT_ERR_ARG;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->capture) cudaStreamDestroy(p->capture);
    cudaFree(p->d_geoms);
    cudaFree(p->d_tasks);
    cudaFree(p->d_counter);
    delete p;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_scatter_batch_create(sysmat_scatter_plan** out, sysmat_ctx* const* ctxs, int n_ctx,
                                                      const sysmat_scatter_item* items, int n_items, void* stream)
{
    if (!out || !ctxs || n_ctx < 1 || n_items < 0 || (n_items > 0 && !items)) return SYSMAT_ERR_ARG;
    *out = nullptr;
    const int device = ctxs[0] ? ctxs[0]->device : -1;
    for (int c = 0; c < n_ctx; ++c)
        if (!ctxs[c] || ctxs[c]->device != device) return SYSMAT_ERR_ARG;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != device) return SYSMAT_ERR_ARG;
    std::vector<ScatterTask> tasks;
    long long next = 0;
    for (int i = 0; i < n_items; ++i) {
        const sysmat_scatter_item& it = items[i];
        if (it.ctx < 0 || it.ctx >= n_ctx) return SYSMAT_ERR_ARG;
        ScatterTask t{};
        const int rc = scatter_setup(ctxs[it.ctx], it.parts, it.hole_model, it.rotation, it.d_pe, it.det_begin,
                                     it.det_count, it.vox_begin, it.vox_count, it.d_out, it.ld,
                                     (cudaStream_t)stream, &t.ph, &t.L);
        if (rc) return rc;
        if (it.det_count == 0 || it.vox_count == 0) continue;
        t.geom = it.ctx;
        t.n_vblocks = (int)((it.vox_count + kScatterBlockVoxels - 1) / kScatterBlockVoxels);
        t.item_begin = next;
        next += (long long)t.n_vblocks * it.det_count;
        tasks.push_back(t);
    }
    auto* p = new sysmat_scatter_plan();
    p->device = device;
    p->num_sms = ctxs[0]->num_sms;
    std::vector<DevGeom> geoms;
    for (int c = 0; c < n_ctx; ++c) geoms.push_back(ctxs[c]->g);
    const size_t nt = tasks.empty() ? 1 : tasks.size();
    if (cudaMalloc(&p->d_geoms, sizeof(DevGeom) * geoms.size()) != cudaSuccess ||
        cudaMalloc(&p->d_tasks, sizeof(ScatterTask) * nt) != cudaSuccess ||
        cudaMalloc(&p->d_counter, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemcpy(p->d_geoms, geoms.data(), sizeof(DevGeom) * geoms.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        (!tasks.empty() &&
         cudaMemcpy(p->d_tasks, tasks.data(), sizeof(ScatterTask) * tasks.size(), cudaMemcpyHostToDevice) !=
             cudaSuccess) ||
        cudaStreamCreateWithFlags(&p->capture, cudaStreamNonBlocking) != cudaSuccess) {
        sysmat_scatter_batch_destroy(p);
        return SYSMAT_ERR_NOMEM;
    }
    p->launch.geoms = p->d_geoms;
    p->launch.tasks = p->d_tasks;
    p->launch.n_tasks = (int)tasks.size();
    p->launch.total_items = next;
    p->launch.work_counter = p->d_counter;
    *out = p;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_scatter_batch_run(sysmat_scatter_plan* p, void* stream)
{
    if (!p) return SYSMAT_ERR_ARG;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != p->device) return SYSMAT_ERR_ARG;
    if (p->launch.total_items < 1) return SYSMAT_OK;
    if (!p->exec) {                    // capture "zero the counter + launch" once, replay after
        const int grid = p->num_sms * scatter_batch_blocks_per_sm();
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(p->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return SYSMAT_ERR_CUDA;
        const bool ok = cudaMemsetAsync(p->d_counter, 0, sizeof(unsigned long long), p->capture) == cudaSuccess &&
                        launch_scatter_batch(p->launch, grid, p->capture) == 0;
        const cudaError_t end = cudaStreamEndCapture(p->capture, &graph);
        if (!ok || end != cudaSuccess || !graph) {
            if (graph) cudaGraphDestroy(graph);
            std::fprintf(stderr, "sysmat: scatter batch graph capture failed\n");
            return SYSMAT_ERR_CUDA;
        }
        const cudaError_t inst = cudaGraphInstantiate(&p->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (inst != cudaSuccess) {
            p->exec = nullptr;
            return SYSMAT_ERR_CUDA;
        }
    }
    return cudaGraphLaunch(p->exec, (cudaStream_t)stream) == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
}
