// Batched photoelectric launches: many (system, rotation, block) tasks in one persistent
// launch over a device work queue, replayed as a CUDA graph, with the voxel brick of a work
// item chosen by a timing autotuner.
//
// The reference computes one rotation of one system per host call (PESysMatGen.cu:1368-1437:
// allocate, copy, launch, copy back, free).  Sweeping collimator designs and rotations that
// way leaves the GPU idle between calls and in each launch's tail, where a few long elements
// finish alone.  A plan instead puts the items of every task in one queue: blocks move on to
// the next task's items while others finish, and the whole batch is one graph launch.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../include/sysmat.h"
#include "ctx.cuh"
#include "pe.cuh"

using namespace sysmat;

#define BATCH_TRY(expr)                                                                    \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess) {                                                           \
            std::fprintf(stderr, "sysmat: %s failed: %s (%s:%d)\n", #expr,                 \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                      \
            return SYSMAT_ERR_CUDA;                                                        \
        }                                                                                  \
    } while (0)

struct sysmat_batch_plan {
    int device = -1;
    int num_sms = 0;
    std::vector<DevGeom> geoms;            // one per context, as the contexts hold them
    bool ell = false;                      // some context has elliptical holes
    std::vector<sysmat_batch_item> items;  // non-empty items, in the caller's order
    int bx = 4, by = 4, bz = 2, blocks_per_sm = 0;   // 0: as many as fit
    DevGeom* d_geoms = nullptr;
    BatchTask* d_tasks = nullptr;
    int task_capacity = 0;
    unsigned long long* d_counter = nullptr;
    BatchLaunch launch{};                  // current task table
    cudaStream_t capture = nullptr;
    cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};   // one graph per mode
};

namespace {

bool device_is(int device)
{
    int cur = -1;
    return cudaGetDevice(&cur) == cudaSuccess && cur == device;
}

void drop_graphs(sysmat_batch_plan* p)
{
    for (auto& e : p->exec) {
        if (e) cudaGraphExecDestroy(e);
        e = nullptr;
    }
}

// Task table of `items` for brick (bx, by, bz), uploaded to the plan's task array.
int upload_tasks(sysmat_batch_plan* p, const std::vector<sysmat_batch_item>& items, int bx, int by, int bz)
{
    std::vector<BatchTask> t;
    t.reserve(items.size());
    long long next = 0;
    for (const sysmat_batch_item& it : items) {
        const DevGeom& g = p->geoms[it.ctx];
        const long long nxy = (long long)g.nx * g.ny;
        const long long vlast = it.vox_begin + it.vox_count - 1;
        BatchTask k{};
        k.geom = it.ctx;
        k.rotation = it.rotation;
        k.det_begin = it.det_begin;
        k.det_count = it.det_count;
        k.vox_begin = it.vox_begin;
        k.vox_count = it.vox_count;
        k.out = it.d_out;
        k.ld = it.ld;
        k.iz0 = (int)(it.vox_begin / nxy);
        k.iz1 = (int)(vlast / nxy);
        k.nbx = (g.nx + bx - 1) / bx;
        k.nby = (g.ny + by - 1) / by;
        k.nbz = (k.iz1 - k.iz0 + 1 + bz - 1) / bz;
        k.item_begin = next;
        next += (long long)k.nbx * k.nby * k.nbz * it.det_count;
        t.push_back(k);
    }
    if ((int)t.size() > p->task_capacity) return SYSMAT_ERR_CAPACITY;
    if (!t.empty())
        BATCH_TRY(cudaMemcpy(p->d_tasks, t.data(), sizeof(BatchTask) * t.size(), cudaMemcpyHostToDevice));
    p->launch.geoms = p->d_geoms;
    p->launch.tasks = p->d_tasks;
    p->launch.n_tasks = (int)t.size();
    p->launch.total_items = next;
    p->launch.bx = bx;
    p->launch.by = by;
    p->launch.bz = bz;
    p->launch.work_counter = p->d_counter;
    return SYSMAT_OK;
}

int grid_of(const sysmat_batch_plan* p, int mode, int* grid)
{
    int per_sm = 0;
    if (configure_pe_batch(mode, p->ell, &per_sm)) return SYSMAT_ERR_CUDA;
    if (p->blocks_per_sm > 0 && p->blocks_per_sm < per_sm) per_sm = p->blocks_per_sm;
    *grid = p->num_sms * per_sm;
    return SYSMAT_OK;
}

// Launch the current task table directly (no graph) on `s`.
int launch_direct(sysmat_batch_plan* p, int mode, cudaStream_t s)
{
    int grid = 0;
    int rc = grid_of(p, mode, &grid);
    if (rc) return rc;
    BATCH_TRY(cudaMemsetAsync(p->d_counter, 0, sizeof(unsigned long long), s));
    return launch_pe_batch(p->launch, mode, p->ell, grid, s) ? SYSMAT_ERR_CUDA : SYSMAT_OK;
}

}  // namespace

extern "C" SYSMAT_API int sysmat_batch_create(sysmat_batch_plan** out, sysmat_ctx* const* ctxs, int n_ctx,
                                              const sysmat_batch_item* items, int n_items)
{
    if (!out || !ctxs || n_ctx < 1 || n_items < 0 || (n_items > 0 && !items)) return SYSMAT_ERR_ARG;
    *out = nullptr;
    const int device = ctxs[0] ? ctxs[0]->device : -1;
    for (int c = 0; c < n_ctx; ++c)
        if (!ctxs[c] || ctxs[c]->device != device) return SYSMAT_ERR_ARG;
    if (!device_is(device)) return SYSMAT_ERR_ARG;
    auto* p = new sysmat_batch_plan();
    p->device = device;
    p->num_sms = ctxs[0]->num_sms;
    for (int c = 0; c < n_ctx; ++c) {
        p->geoms.push_back(ctxs[c]->g);
        p->ell = p->ell || ctxs[c]->g.hole_shape != nullptr;
    }
    for (int i = 0; i < n_items; ++i) {
        const sysmat_batch_item& it = items[i];
        if (it.ctx < 0 || it.ctx >= n_ctx ||
            check_block(ctxs[it.ctx], it.det_begin, it.det_count, it.vox_begin, it.vox_count, it.d_out, it.ld) ||
            !std::isfinite(it.rotation)) {
            delete p;
            return SYSMAT_ERR_ARG;
        }
        if (it.det_count > 0 && it.vox_count > 0) p->items.push_back(it);
    }
    p->task_capacity = (int)p->items.size() > 32 ? (int)p->items.size() : 32;   // >= the tuner's probe
    if (cudaMalloc(&p->d_geoms, sizeof(DevGeom) * p->geoms.size()) != cudaSuccess ||
        cudaMalloc(&p->d_tasks, sizeof(BatchTask) * p->task_capacity) != cudaSuccess ||
        cudaMalloc(&p->d_counter, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemcpy(p->d_geoms, p->geoms.data(), sizeof(DevGeom) * p->geoms.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaStreamCreateWithFlags(&p->capture, cudaStreamNonBlocking) != cudaSuccess) {
        sysmat_batch_destroy(p);
        return SYSMAT_ERR_NOMEM;
    }
    const int rc = upload_tasks(p, p->items, p->bx, p->by, p->bz);
    if (rc) {
        sysmat_batch_destroy(p);
        return rc;
    }
    *out = p;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_batch_destroy(sysmat_batch_plan* p)
{
    if (!p) return SYSMAT_ERR_ARG;
    drop_graphs(p);
    if (p->capture) cudaStreamDestroy(p->capture);
    cudaFree(p->d_geoms);
    cudaFree(p->d_tasks);
    cudaFree(p->d_counter);
    delete p;
    return SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_batch_set_tiles(sysmat_batch_plan* p, int bx, int by, int bz, int blocks_per_sm)
{
    if (!p || bx < 1 || by < 1 || bz < 1 || bx * by * bz > 512 || blocks_per_sm < 0) return SYSMAT_ERR_ARG;
    if (!device_is(p->device)) return SYSMAT_ERR_ARG;
    drop_graphs(p);
    p->bx = bx;
    p->by = by;
    p->bz = bz;
    p->blocks_per_sm = blocks_per_sm;
    return upload_tasks(p, p->items, bx, by, bz);
}

extern "C" SYSMAT_API int sysmat_batch_get_tiles(const sysmat_batch_plan* p, int* tiles)
{
    if (!p || !tiles) return SYSMAT_ERR_ARG;
    tiles[0] = p->bx;
    tiles[1] = p->by;
    tiles[2] = p->bz;
    tiles[3] = p->blocks_per_sm;
    return SYSMAT_OK;
}

bool plan_mode_ok(const sysmat_batch_plan*, int mode)
{
    return mode == SYSMAT_MODE_REFERENCE || mode == SYSMAT_MODE_PRECISE || mode == SYSMAT_MODE_FP64 ||
           mode == SYSMAT_MODE_LOCAL;
}

extern "C" SYSMAT_API int sysmat_batch_run(sysmat_batch_plan* p, int mode, void* stream)
{
    if (!p || !plan_mode_ok(p, mode)) return SYSMAT_ERR_ARG;
    if (!device_is(p->device)) return SYSMAT_ERR_ARG;
    if (p->launch.total_items < 1) return SYSMAT_OK;
    cudaGraphExec_t& exec = p->exec[mode];
    if (!exec) {
        int grid = 0;
        int rc = grid_of(p, mode, &grid);
        if (rc) return rc;
        cudaGraph_t graph = nullptr;
        BATCH_TRY(cudaStreamBeginCapture(p->capture, cudaStreamCaptureModeThreadLocal));
        const bool ok = cudaMemsetAsync(p->d_counter, 0, sizeof(unsigned long long), p->capture) == cudaSuccess &&
                        launch_pe_batch(p->launch, mode, p->ell, grid, p->capture) == 0;
        const cudaError_t end = cudaStreamEndCapture(p->capture, &graph);
        if (!ok || end != cudaSuccess || !graph) {
            if (graph) cudaGraphDestroy(graph);
            std::fprintf(stderr, "sysmat: batch graph capture failed\n");
            return SYSMAT_ERR_CUDA;
        }
        const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (inst != cudaSuccess) {
            exec = nullptr;
            std::fprintf(stderr, "sysmat: batch graph instantiation failed: %s\n", cudaGetErrorString(inst));
            return SYSMAT_ERR_CUDA;
        }
    }
    BATCH_TRY(cudaGraphLaunch(exec, (cudaStream_t)stream));
    return SYSMAT_OK;
}

// Autotuner: times candidate bricks on a probe subset of the batch (up to 8 tasks spread over
// it, up to 4 detector rows of each, spread over its rows) and keeps the fastest.  The probe
// writes rows of the caller's outputs with the values the batch itself computes there.
extern "C" SYSMAT_API int sysmat_batch_tune(sysmat_batch_plan* p, int mode, void* stream, int* tiles)
{
    if (!p || !plan_mode_ok(p, mode)) return SYSMAT_ERR_ARG;
    if (!device_is(p->device)) return SYSMAT_ERR_ARG;
    if (p->items.empty()) return tiles ? sysmat_batch_get_tiles(p, tiles) : SYSMAT_OK;
    drop_graphs(p);                          // the probe reuses the task array
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<sysmat_batch_item> probe;
    const int n = (int)p->items.size();
    const int n_tasks = n < 8 ? n : 8;
    for (int k = 0; k < n_tasks; ++k) {
        const sysmat_batch_item& it = p->items[(long long)k * n / n_tasks];
        const int rows = it.det_count < 4 ? it.det_count : 4;
        for (int r = 0; r < rows; ++r) {
            sysmat_batch_item q = it;
            const int di = (int)((long long)r * it.det_count / rows);
            q.det_begin = it.det_begin + di;
            q.det_count = 1;
            q.d_out = it.d_out + (long long)di * it.ld;
            probe.push_back(q);
        }
    }
    static const int cand[][3] = {{4, 4, 2}, {4, 4, 1}, {8, 4, 1}, {4, 2, 2}, {2, 2, 2}, {8, 8, 1}, {4, 4, 4}};
    cudaEvent_t e0, e1;
    BATCH_TRY(cudaEventCreate(&e0));
    BATCH_TRY(cudaEventCreate(&e1));
    float best = INFINITY;
    int best_c = 0;
    int rc = SYSMAT_OK;
    for (int c = 0; c < (int)(sizeof(cand) / sizeof(cand[0])) && rc == SYSMAT_OK; ++c) {
        rc = upload_tasks(p, probe, cand[c][0], cand[c][1], cand[c][2]);
        if (rc) break;
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && rc == SYSMAT_OK; ++rep) {   // first run warms caches
            if (cudaEventRecord(e0, s) != cudaSuccess) rc = SYSMAT_ERR_CUDA;
            if (!rc) rc = launch_direct(p, mode, s);
            if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = SYSMAT_ERR_CUDA;
            if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                rc = SYSMAT_ERR_CUDA;
        }
        if (!rc && ms < best) {
            best = ms;
            best_c = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        upload_tasks(p, p->items, p->bx, p->by, p->bz);
        return rc;
    }
    rc = sysmat_batch_set_tiles(p, cand[best_c][0], cand[best_c][1], cand[best_c][2], p->blocks_per_sm);
    if (rc) return rc;
    return tiles ? sysmat_batch_get_tiles(p, tiles) : SYSMAT_OK;
}

extern "C" SYSMAT_API int sysmat_batch(sysmat_ctx* const* ctxs, int n_ctx, const sysmat_batch_item* items,
                                       int n_items, int mode, void* stream)
{
    if (mode != SYSMAT_MODE_REFERENCE && mode != SYSMAT_MODE_PRECISE && mode != SYSMAT_MODE_FP64 &&
        mode != SYSMAT_MODE_LOCAL)
        return SYSMAT_ERR_ARG;
    sysmat_batch_plan* p = nullptr;
    int rc = sysmat_batch_create(&p, ctxs, n_ctx, items, n_items);
    if (rc) return rc;
    rc = launch_direct(p, mode, (cudaStream_t)stream);
    if (!rc && cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) rc = SYSMAT_ERR_CUDA;
    sysmat_batch_destroy(p);
    return rc;
}
