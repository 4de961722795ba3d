// Launch plan of the tiled confined-solver step kernel. The plan records which tiles of
// the box contain cells the step must visit; tiles that hold only frozen exterior cells are
// skipped (their values never change and are identical in both ping-pong buffers).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ldg_common.cuh"

namespace ldg {

struct TiledPlan {
    bool ok = false;
    long long active_cells = 0;
};

inline int tiled_plan_build(TiledPlan& plan, int Nx, int Ny, int Nz, int, long long, const uint8_t*) {
    plan.ok = false;
    plan.active_cells = (long long)Nx * Ny * Nz;
    return 0;
}

inline int tiled_step(const TiledPlan&, const float*, float*, const uint8_t*, const QsrConst&, bool, bool, bool,
                      cudaStream_t) {
    return 0;
}

inline void tiled_plan_free(TiledPlan& plan) { plan = TiledPlan{}; }

}  // namespace ldg
