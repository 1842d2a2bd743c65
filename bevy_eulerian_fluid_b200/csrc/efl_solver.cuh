// efl_solver.cuh — red-black Gauss-Seidel pressure solves
// (projection/shaders/gauss_seidel.wgsl:12-88, host loop gauss_seidel.rs:142-147).
//
// Two forms:
//  * solve_gs_fixed: n red-black iterations as one launch per colour
//    (k_gs_color), f32 (the reference's fixed-count mode) or f64.
//  * solve_gs64_persistent: the tolerance-driven FP64 solve as ONE
//    cooperative launch.  Each CTA owns a tile of the grid and keeps the
//    tile plus a halo of 2k cells in shared memory -- the iterate, the
//    right-hand side, the per-cell diagonal and its reciprocal, the face
//    fractions and the fluid flags -- so that k red-black iterations run
//    from shared memory between two halo exchanges (temporal blocking; the
//    result is identical to k global sweeps because a half-sweep only reads
//    the other colour).  Halos are exchanged through L2 behind a grid
//    barrier whose spin is bounded; the relative residual is reduced and
//    tested on the device every check_interval iterations, so the whole
//    solve needs no host round trip.
#pragma once

#include <algorithm>
#include <string>

#include "efl_kernels.cuh"

namespace efl {

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
    int error;
    int pad;
};

struct SolveResult {
    unsigned int iterations;
    int converged;
    int error;  // 1: a grid barrier timed out
    int pad;
    double r0, r1;  // relative residual before / after
};

struct SolverWorkspace {
    int nx = 0, ny = 0, device = 0;
    int num_sms = 0;
    size_t max_smem = 0;
    GridBarrier* barrier = nullptr;
    SolveResult* result = nullptr;    // device
    SolveResult* h_result = nullptr;  // pinned host
    double2* partials = nullptr;
    int max_blocks = 0;
};

constexpr int PS_THREADS = 512;
constexpr long long kBarrierSpinLimit = 1ll << 22;  // x ~100 ns sleeps: well under a second

// Grid-wide barrier for a cooperative launch (all CTAs co-resident), with a
// bounded spin: a CTA that waits more than kBarrierSpinLimit polls sets
// barrier->error and every CTA leaves the solve.
EFL_DEV bool grid_barrier(GridBarrier* gb, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* vgen = &gb->gen;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&gb->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == gen) {
                if (++spins > kBarrierSpinLimit) {
                    atomicExch(&gb->error, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        if (*(volatile int*)&gb->error) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct PersistentParams {
    Level64 L;  // level 0: x = FP64 iterate (global), b = widened divergence
    int tx, ty, halo, kmax;
    int tiles_x;
    double cdiv;    // ((dx*dx)*rho)/dt (gauss_seidel.wgsl:58)
    double factor;  // dt/rho/dx/dx (residual.wgsl:34)
    double weight;
    double tol;
    unsigned max_iters, check_interval;
    double2* partials;
    GridBarrier* barrier;
    SolveResult* result;
};

constexpr unsigned char M_DOMAIN = 1, M_FLUID = 2, M_COUNTED = 4, M_UPDATE = 8;

struct PsSmem {
    double* p;
    double* b;
    double* den;
    double* inv;
    float* fu;  // (EX+1) x EY: face lx sits between cells lx-1 and lx
    float* fv;  // EX x (EY+1)
    unsigned char* m;
    int EX, EY;
};

EFL_DEV PsSmem ps_carve(unsigned char* base, int EX, int EY) {
    PsSmem s;
    const int n = EX * EY;
    s.EX = EX;
    s.EY = EY;
    s.p = reinterpret_cast<double*>(base);
    s.b = s.p + n;
    s.den = s.b + n;
    s.inv = s.den + n;
    s.fu = reinterpret_cast<float*>(s.inv + n);
    s.fv = s.fu + (EX + 1) * EY;
    s.m = reinterpret_cast<unsigned char*>(s.fv + EX * (EY + 1));
    return s;
}
inline size_t ps_smem_bytes(int EX, int EY) {
    const size_t n = (size_t)EX * EY;
    return n * 4 * sizeof(double) + (size_t)(EX + 1) * EY * 4 + (size_t)EX * (EY + 1) * 4 + n;
}

// One half-sweep of colour `color` ((x+y)&1 == color) over the extended
// tile minus its outer ring.  Update of the tolerance-driven mode:
// p = w * ((cdiv*b + sum w_k p_k) * (1/denom)) + (1-w) * p, neighbour order
// (-x, +x, -y, +y) as gauss_seidel.wgsl:68-79; w_k = 0 for air or
// out-of-domain neighbours.
EFL_DEV void ps_half_sweep(const PsSmem& s, int gx0, int gy0, int color, double cdiv, double w, double omw) {
    const int EX = s.EX, EY = s.EY;
    const int half = (EX - 2 + 1) / 2;
    const int total = half * (EY - 2);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int ly = 1 + i / half;
        const int j = i - (ly - 1) * half;
        const int lx0 = 1 + ((color + gx0 + gy0 + ly + 1) & 1);
        const int lx = lx0 + 2 * j;
        if (lx > EX - 2) continue;
        const int c = ly * EX + lx;
        const unsigned char m = s.m[c];
        if (!(m & M_DOMAIN)) continue;
        if (!(m & M_UPDATE)) {
            s.p[c] = 0.0;
            continue;
        }
        const double w0 = (s.m[c - 1] & M_FLUID) ? (double)s.fu[ly * (EX + 1) + lx] : 0.0;
        const double w1 = (s.m[c + 1] & M_FLUID) ? (double)s.fu[ly * (EX + 1) + lx + 1] : 0.0;
        const double w2 = (s.m[c - EX] & M_FLUID) ? (double)s.fv[ly * EX + lx] : 0.0;
        const double w3 = (s.m[c + EX] & M_FLUID) ? (double)s.fv[(ly + 1) * EX + lx] : 0.0;
        double nume = cdiv * s.b[c];
        nume = nume + w0 * s.p[c - 1];
        nume = nume + w1 * s.p[c + 1];
        nume = nume + w2 * s.p[c - EX];
        nume = nume + w3 * s.p[c + EX];
        s.p[c] = w * (nume * s.inv[c]) + omw * s.p[c];
    }
}

// ||r||^2 and ||b||^2 over the owned cells of this tile (all halo cells
// valid), r = b - factor * (denom * p - sum w_k p_k).
EFL_DEV double2 ps_residual_partial(const PsSmem& s, int H, int tx, int ty, double factor) {
    const int EX = s.EX;
    double ar = 0.0, ab = 0.0;
    for (int i = threadIdx.x; i < tx * ty; i += blockDim.x) {
        const int ly = H + i / tx, lx = H + i % tx;
        const int c = ly * EX + lx;
        const unsigned char m = s.m[c];
        if ((m & (M_DOMAIN | M_COUNTED)) != (M_DOMAIN | M_COUNTED)) continue;
        const double w0 = (s.m[c - 1] & M_FLUID) ? (double)s.fu[ly * (EX + 1) + lx] : 0.0;
        const double w1 = (s.m[c + 1] & M_FLUID) ? (double)s.fu[ly * (EX + 1) + lx + 1] : 0.0;
        const double w2 = (s.m[c - EX] & M_FLUID) ? (double)s.fv[ly * EX + lx] : 0.0;
        const double w3 = (s.m[c + EX] & M_FLUID) ? (double)s.fv[(ly + 1) * EX + lx] : 0.0;
        double sum = w0 * s.p[c - 1];
        sum = sum + w1 * s.p[c + 1];
        sum = sum + w2 * s.p[c - EX];
        sum = sum + w3 * s.p[c + EX];
        const double r = s.b[c] - factor * (s.den[c] * s.p[c] - sum);
        ar += r * r;
        ab += s.b[c] * s.b[c];
    }
    ar = warp_sum(ar);
    ab = warp_sum(ab);
    __shared__ double red_r[32], red_b[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red_r[wid] = ar;
        red_b[wid] = ab;
    }
    __syncthreads();
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            out.x += red_r[k];
            out.y += red_b[k];
        }
    }
    __syncthreads();
    return out;
}

EFL_DEV void ps_load_p(const PsSmem& s, const Level64& L, int gx0, int gy0) {
    const int n = s.EX * s.EY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int ly = i / s.EX, lx = i - ly * s.EX;
        const int gx = gx0 + lx, gy = gy0 + ly;
        s.p[i] = (s.m[i] & M_DOMAIN) ? __ldcg(&L.x.p[(size_t)gy * L.x.P + gx]) : 0.0;
    }
}
EFL_DEV void ps_store_owned(const PsSmem& s, const Level64& L, int gx0, int gy0, int H, int tx, int ty) {
    for (int i = threadIdx.x; i < tx * ty; i += blockDim.x) {
        const int ly = H + i / tx, lx = H + i % tx;
        const int c = ly * s.EX + lx;
        if (s.m[c] & M_DOMAIN) __stcg(&L.x.p[(size_t)(gy0 + ly) * L.x.P + gx0 + lx], s.p[c]);
    }
}
// Sum of all CTAs' partials in CTA order; identical in every CTA.
EFL_DEV double ps_total_relative(const double2* partials, int nblocks) {
    __shared__ double s_rel;
    if (threadIdx.x == 0) {
        double r = 0.0, b = 0.0;
        for (int i = 0; i < nblocks; ++i) {
            double2 v = __ldcg(&partials[i]);
            r += v.x;
            b += v.y;
        }
        s_rel = b > 0.0 ? sqrt(r) / sqrt(b) : (r > 0.0 ? __longlong_as_double(0x7ff0000000000000ll) : 0.0);
    }
    __syncthreads();
    double v = s_rel;
    __syncthreads();
    return v;
}

__global__ void __launch_bounds__(PS_THREADS, 1) k_gs64_persistent(PersistentParams P) {
    extern __shared__ __align__(16) unsigned char ps_raw[];
    const int H = P.halo;
    const int EX = P.tx + 2 * H, EY = P.ty + 2 * H;
    const PsSmem s = ps_carve(ps_raw, EX, EY);
    const Level64& L = P.L;
    const int tile = blockIdx.x;
    const int gx0 = (tile % P.tiles_x) * P.tx - H, gy0 = (tile / P.tiles_x) * P.ty - H;
    const unsigned nblocks = gridDim.x;

    // Per-solve coefficients of the extended tile (gauss_seidel.wgsl:44-80 and
    // residual.wgsl:21-54, neighbour order of the reference).
    const int n = EX * EY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int ly = i / EX, lx = i - ly * EX;
        const int gx = gx0 + lx, gy = gy0 + ly;
        unsigned char m = 0;
        double den = 0.0, inv = 0.0, bb = 0.0;
        if ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
            m |= M_DOMAIN;
            const float phi = L.ls.at(gx, gy);
            bb = L.b.at(gx, gy);
            if (phi < 0.0f) {
                m |= M_FLUID;
                const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
                if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                    m |= M_COUNTED;
                    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int jx = gx + ox[k], jy = gy + oy[k];
                        if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                            const float level = L.ls.at(jx, jy);
                            if (level < 0.0f) den += (double)f[k];
                            else den += (double)f[k] * (1.0 - (double)level / (double)phi);
                        }
                    }
                    if (!(fabs(den) < (double)1.0e-6f)) {
                        m |= M_UPDATE;
                        inv = 1.0 / den;
                    }
                }
            }
        }
        s.m[i] = m;
        s.den[i] = den;
        s.inv[i] = inv;
        s.b[i] = bb;
    }
    for (int i = threadIdx.x; i < (EX + 1) * EY; i += blockDim.x) {
        const int ly = i / (EX + 1), lx = i - ly * (EX + 1);
        s.fu[i] = L.fu.ld(gx0 + lx, gy0 + ly);
    }
    for (int i = threadIdx.x; i < EX * (EY + 1); i += blockDim.x) {
        const int ly = i / EX, lx = i - ly * EX;
        s.fv[i] = L.fv.ld(gx0 + lx, gy0 + ly);
    }
    __syncthreads();
    ps_load_p(s, L, gx0, gy0);
    __syncthreads();

    const double w = P.weight, omw = 1.0 - P.weight;
    unsigned iters = 0;
    double2 part = ps_residual_partial(s, H, P.tx, P.ty, P.factor);
    if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
    bool ok = grid_barrier(P.barrier, nblocks);
    double r = ok ? ps_total_relative(P.partials, nblocks) : 0.0;
    const double r0 = r;
    while (ok && !(r <= P.tol) && iters < P.max_iters) {
        unsigned todo = min(P.check_interval, P.max_iters - iters);
        while (ok && todo > 0) {
            const unsigned kk = min((unsigned)P.kmax, todo);
            for (unsigned it = 0; it < kk; ++it) {
                ps_half_sweep(s, gx0, gy0, 1, P.cdiv, w, omw);  // red: (x+y) odd
                __syncthreads();
                ps_half_sweep(s, gx0, gy0, 0, P.cdiv, w, omw);  // black
                __syncthreads();
            }
            ps_store_owned(s, L, gx0, gy0, H, P.tx, P.ty);
            ok = grid_barrier(P.barrier, nblocks);
            if (!ok) break;
            ps_load_p(s, L, gx0, gy0);
            __syncthreads();
            todo -= kk;
            iters += kk;
        }
        if (!ok) break;
        part = ps_residual_partial(s, H, P.tx, P.ty, P.factor);
        if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
        ok = grid_barrier(P.barrier, nblocks);
        if (!ok) break;
        r = ps_total_relative(P.partials, nblocks);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.result->iterations = iters;
        P.result->converged = (ok && r <= P.tol) ? 1 : 0;
        P.result->error = ok ? 0 : 1;
        P.result->r0 = r0;
        P.result->r1 = r;
    }
}

inline efl_status solver_init(SolverWorkspace& ws, int nx, int ny, int device, std::string* err) {
    ws.nx = nx;
    ws.ny = ny;
    ws.device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        *err = "cudaGetDeviceProperties failed";
        return EFL_ERR_CUDA;
    }
    ws.num_sms = prop.multiProcessorCount;
    ws.max_smem = prop.sharedMemPerBlockOptin;
    ws.max_blocks = 4 * ws.num_sms;
    if (cudaMalloc(&ws.barrier, sizeof(GridBarrier)) != cudaSuccess ||
        cudaMalloc(&ws.result, sizeof(SolveResult)) != cudaSuccess ||
        cudaMalloc(&ws.partials, ws.max_blocks * sizeof(double2)) != cudaSuccess ||
        cudaMallocHost(&ws.h_result, sizeof(SolveResult)) != cudaSuccess) {
        *err = "solver workspace allocation failed";
        return EFL_ERR_OUT_OF_MEMORY;
    }
    return EFL_OK;
}
inline void solver_free(SolverWorkspace& ws) {
    if (ws.barrier) cudaFree(ws.barrier);
    if (ws.result) cudaFree(ws.result);
    if (ws.partials) cudaFree(ws.partials);
    if (ws.h_result) cudaFreeHost(ws.h_result);
    ws = SolverWorkspace{};
}

// n red-black iterations at level L (red then black per iteration),
// f32 (reference) or f64 iterate, one launch per colour.
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

struct PersistentPlan {
    int tx = 0, ty = 0, kmax = 0, tiles_x = 0, tiles_y = 0;
    size_t smem = 0;
    bool ok = false;
};

// Deepest temporal blocking and a tile shape whose CTAs are all co-resident
// (one per SM) and whose extended tile fits in shared memory.
inline PersistentPlan plan_persistent(const SolverWorkspace& ws, int nx, int ny) {
    static const int cand[][3] = {{4, 64, 32}, {4, 32, 32}, {2, 64, 32}, {2, 64, 64}, {4, 32, 16}, {2, 32, 32},
                                  {1, 64, 64}, {1, 128, 64}};
    for (const auto& c : cand) {
        PersistentPlan p;
        p.kmax = c[0];
        p.tx = c[1];
        p.ty = c[2];
        p.tiles_x = (nx + p.tx - 1) / p.tx;
        p.tiles_y = (ny + p.ty - 1) / p.ty;
        const int H = 2 * p.kmax;
        p.smem = ps_smem_bytes(p.tx + 2 * H, p.ty + 2 * H) + 64;
        if (p.smem + 1024 > ws.max_smem) continue;  // room for the kernel's static shared memory
        if (p.tiles_x * p.tiles_y > ws.num_sms || p.tiles_x * p.tiles_y > ws.max_blocks) continue;
        p.ok = true;
        return p;
    }
    return PersistentPlan{};
}

// Tolerance-driven FP64 solve in one cooperative launch.  Returns
// EFL_ERR_STATE if the grid does not fit the persistent scheme (the caller
// then uses the host-driven loop).
inline efl_status solve_gs64_persistent(SolverWorkspace& ws, const Level64& L, const Uniform& U, float weight,
                                        double tol, uint32_t max_iters, uint32_t check_interval,
                                        cudaStream_t stream, SolveResult* out, std::string* err) {
    PersistentPlan plan = plan_persistent(ws, L.nx, L.ny);
    if (!plan.ok) return EFL_ERR_STATE;
    if (cudaFuncSetAttribute(k_gs64_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem) !=
        cudaSuccess) {
        cudaGetLastError();
        return EFL_ERR_STATE;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs64_persistent, PS_THREADS, plan.smem) !=
            cudaSuccess ||
        per_sm < 1 || plan.tiles_x * plan.tiles_y > per_sm * ws.num_sms)
        return EFL_ERR_STATE;
    PersistentParams P;
    P.L = L;
    P.tx = plan.tx;
    P.ty = plan.ty;
    P.kmax = plan.kmax;
    P.halo = 2 * plan.kmax;
    P.tiles_x = plan.tiles_x;
    const double dx = (double)U.dx;
    P.cdiv = dx * dx * (double)U.rho / (double)U.dt;
    P.factor = (double)U.dt / (double)U.rho / dx / dx;
    P.weight = (double)weight;
    P.tol = tol;
    P.max_iters = max_iters;
    P.check_interval = std::max<uint32_t>(1, check_interval);
    P.partials = ws.partials;
    P.barrier = ws.barrier;
    P.result = ws.result;
    if (cudaMemsetAsync(ws.barrier, 0, sizeof(GridBarrier), stream) != cudaSuccess) {
        *err = "barrier reset failed";
        return EFL_ERR_CUDA;
    }
    void* args[] = {&P};
    count_launch();
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_gs64_persistent, dim3(plan.tiles_x * plan.tiles_y),
                                                dim3(PS_THREADS), args, plan.smem, stream);
    if (e != cudaSuccess) {
        *err = std::string("cooperative launch of the persistent solver failed: ") + cudaGetErrorString(e);
        return EFL_ERR_CUDA;
    }
    if (cudaMemcpyAsync(ws.h_result, ws.result, sizeof(SolveResult), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
        *err = std::string("persistent solver failed: ") + cudaGetErrorString(cudaGetLastError());
        return EFL_ERR_CUDA;
    }
    *out = *ws.h_result;
    if (out->error) {
        *err = "persistent solver: a grid barrier timed out";
        return EFL_ERR_CUDA;
    }
    return EFL_OK;
}

}  // namespace efl
