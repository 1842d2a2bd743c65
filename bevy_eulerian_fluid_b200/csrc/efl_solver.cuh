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

// n red-black iterations at level 0 (red then black per iteration),
// f32 (reference) or f64 (tolerance-driven) iterate.
template <class T>
inline efl_status solve_gs_fixed(SolverWorkspace&, const LevelT<T>& L, const Uniform& U, float weight, uint32_t n,
                                 cudaStream_t stream) {
    const dim3 b(32, 8);
    const dim3 g(((L.nx + 1) / 2 + b.x - 1) / b.x, (L.ny + b.y - 1) / b.y);
    for (uint32_t k = 0; k < n; ++k) {
        k_gs_color<T><<<g, b, count_launch(), stream>>>(L, U.dx, U.rho, U.dt, weight, 1);
        k_gs_color<T><<<g, b, count_launch(), stream>>>(L, U.dx, U.rho, U.dt, weight, 0);
    }
    return EFL_OK;
}

}  // namespace efl
