// efl_solver.cuh — the red-black Gauss-Seidel pressure sweep
// (projection/shaders/gauss_seidel.wgsl:12-88, host loop gauss_seidel.rs:142-147).
#pragma once

#include <string>

#include "efl_kernels.cuh"

namespace efl {

struct SolverWorkspace {
    int nx = 0, ny = 0;
};

inline efl_status solver_init(SolverWorkspace& ws, int nx, int ny, int /*device*/, std::string* /*err*/) {
    ws.nx = nx;
    ws.ny = ny;
    return EFL_OK;
}
inline void solver_free(SolverWorkspace&) {}

// n red-black iterations at level L (red then black per iteration).
inline efl_status solve_gs_fixed(SolverWorkspace&, const Level& L, const Uniform& U, float weight, uint32_t n,
                                 cudaStream_t stream) {
    const dim3 b(32, 8);
    const dim3 g(((L.nx + 1) / 2 + b.x - 1) / b.x, (L.ny + b.y - 1) / b.y);
    for (uint32_t k = 0; k < n; ++k) {
        k_gs_color<float><<<g, b, 0, stream>>>(L, U.dx, U.rho, U.dt, weight, 1);
        k_gs_color<float><<<g, b, 0, stream>>>(L, U.dx, U.rho, U.dt, weight, 0);
    }
    return EFL_OK;
}

}  // namespace efl
