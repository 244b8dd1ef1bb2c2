// Launch interface of the primary-Compton scatter kernels (scatter.cu).
#pragma once

#include <cuda_runtime.h>

#include "geom.cuh"

namespace sysmat {

// Device scratch owned by a context for the scatter path.
struct ScatterScratch {
    void* base = nullptr;
    size_t bytes = 0;
};

inline void scatter_scratch_free(ScatterScratch& s)
{
    if (s.base) cudaFree(s.base);
    s.base = nullptr;
    s.bytes = 0;
}

}  // namespace sysmat
