// efl_solver.cuh — red-black Gauss-Seidel pressure solves
// (projection/shaders/gauss_seidel.wgsl:12-88, host loop gauss_seidel.rs:142-147).
//
// Forms:
//  * solve_gs_fixed: n red-black iterations as one launch per colour
//    (k_gs_color), f32 (the reference's fixed-count mode) or f64.
//  * solve_gsmix_persistent: the tolerance-driven solve (mixed-precision
//    iterative refinement, below) as ONE cooperative launch.  Each CTA owns a
//    tile of the grid and keeps the tile plus a halo of 2k cells in shared
//    memory -- FP64 iterate, right-hand side and diagonal, f32 correction,
//    coefficients and residual, the cell modes -- so that k red-black
//    iterations run from shared memory between two halo exchanges (temporal
//    blocking; the result is identical to k global sweeps because a
//    half-sweep only reads the other colour).  Halos are exchanged through
//    L2 behind a grid barrier whose spin is bounded; the relative residual is
//    reduced and tested on the device every check_interval iterations, so the
//    whole solve needs no host round trip.
//  * solve_gsmix_global: the same solve with global-memory kernels and a host
//    loop, for grids the persistent scheme does not cover.
//  * solve_gs32_tiled: fixed-count f32 sweeps through shared-memory tiles
//    (used when the TMA sweep of efl_sweep_tma.cuh is unavailable).
#pragma once

#include <algorithm>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "efl_kernels.cuh"

namespace efl {

struct GridBarrier {
    unsigned int count;
    unsigned int gen;  // unused (layout kept)
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
    long long spin_limit = 0;  // grid-barrier polls before giving up (0: kBarrierSpinLimit)
    bool use_reg = true;       // register-resident form of the persistent solve (else the shared-memory form)
};

constexpr int PS_THREADS = 1024;

constexpr long long kBarrierSpinLimit = 1ll << 25;  // acquire polls (~ 1 s)

// Grid-wide barrier for a cooperative launch (all CTAs co-resident), with a
// bounded spin.  count only grows (it is zeroed before each launch): a CTA's
// acq_rel arrival returns its arrival number, arrivals of barrier e are
// numbers [e * nblocks, (e + 1) * nblocks) because no CTA reaches barrier
// e + 1 before all have arrived at e, so the CTA waits (acquire loads) until
// count reaches the end of its barrier's range; the last arriver leaves at
// once.  One atomic round trip on the way in, none on the way out.  A CTA
// that polls `limit` times (kBarrierSpinLimit unless the caller set a
// shorter limit) sets barrier->error and leaves; the others see the flag
// while they wait (checked every 1024 polls) and leave too.
EFL_DEV bool grid_barrier(GridBarrier* gb, unsigned nblocks, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned arrived, cur;
        asm volatile("atom.acq_rel.gpu.add.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(&gb->count) : "memory");
        const unsigned target = (arrived / nblocks + 1) * nblocks;
        if (arrived + 1 != target) {
            long long spins = 0;
            for (;;) {
                asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(&gb->count) : "memory");
                if ((int)(cur - target) >= 0) break;
                if ((++spins & 1023) == 0 || spins >= limit) {
                    int e;
                    asm volatile("ld.acquire.gpu.s32 %0, [%1];" : "=r"(e) : "l"(&gb->error) : "memory");
                    if (e || spins >= limit) {
                        atomicExch(&gb->error, 1);
                        ok = 0;
                        break;
                    }
                }
            }
        }
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
    long long spin_limit;  // grid-barrier polls before giving up
    PF dbuf2;              // the exchanges alternate between the correction planes dbuf and dbuf2
    float one;             // 1.0f, passed at run time (see x2_add1)
};

constexpr unsigned char MODE_SKIP = 0;     // outside the domain or on the tile's outer ring
constexpr unsigned char MODE_ZERO = 1;     // air, fully solid or |denom| < 1e-6: p = 0
constexpr unsigned char MODE_UPDATE = 2;   // regular update
constexpr unsigned char MODE_COUNTED = 4;  // counted in the residual norms
constexpr unsigned char MODE_STD = 8;      // update cell with w = (1, 1, 1, 1), inv = 0.25 (coefficients implied)

// Sum of all CTAs' partials in CTA order; identical in every CTA.
EFL_DEV double ps_total_relative(const double2* partials, int nblocks) {
    // Warp 0: lane l adds partials l, l + 32, ... in order (independent loads,
    // one round of latency), then a fixed xor-shuffle tree; the same in every CTA.
    __shared__ double s_rel;
    if (threadIdx.x < 32) {
        double r = 0.0, b = 0.0;
        int i = threadIdx.x;
        for (; i + 96 < nblocks; i += 128) {  // four loads in flight, added in the same order
            const double2 v0 = __ldcg(&partials[i]), v1 = __ldcg(&partials[i + 32]);
            const double2 v2 = __ldcg(&partials[i + 64]), v3 = __ldcg(&partials[i + 96]);
            r += v0.x;
            b += v0.y;
            r += v1.x;
            b += v1.y;
            r += v2.x;
            b += v2.y;
            r += v3.x;
            b += v3.y;
        }
        for (; i < nblocks; i += 32) {
            const double2 v = __ldcg(&partials[i]);
            r += v.x;
            b += v.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_xor_sync(0xffffffffu, r, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (threadIdx.x == 0)
            s_rel = b > 0.0 ? sqrt(r) / sqrt(b) : (r > 0.0 ? __longlong_as_double(0x7ff0000000000000ll) : 0.0);
    }
    __syncthreads();
    double v = s_rel;
    __syncthreads();
    return v;
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

// ---------------------------------------------------------------------------
// Tolerance-driven solve in mixed-precision iterative-refinement form.
// Every check block of n iterations: the FP64 residual r of the FP64 iterate
// p (operator of residual.wgsl in factored form) gives the convergence test
// and the f32 right-hand side rc = f32(cdiv * r); n SOR red-black
// iterations then run in f32 on the correction d (starting at 0) with f32
// coefficients w_k (face fraction of fluid in-bounds neighbours, else 0) and
// inv = f32(1/denom); then p += d in FP64, and the cells the reference sets
// to zero (air, fully solid, |denom| < 1e-6) get p = 0.  SOR is affine, so
// in exact arithmetic these are the RBGS iterates themselves: the
// iteration counts are those of red-black Gauss-Seidel, while the sweeps move
// f32 data.
// Shared-memory image of one extended tile (EX x EY cells, EX even), stored
// per colour in checkerboard-compressed form: cell (lx, ly) of colour
// c = (gx + gy) & 1 lives at [c][ly][lx >> 1].  A cell's left / right
// neighbours are the other colour's entries (lx >> 1) - 1 + (lx & 1) and
// (lx >> 1) + (lx & 1) of the same row, up / down are entry lx >> 1 of the
// rows above and below, so a warp reads consecutive words.
template <int EX, int EY>
struct MixTile {
    static constexpr int W2 = EX / 2;
    static constexpr int N2 = W2 * EY;
    double p[2][N2];  // FP64 iterate
    double b[2][N2];
    double den[2][N2];
    float4 w[2][N2];
    float d[2][N2];   // f32 correction
    float rc[2][N2];  // f32 right-hand side of the correction
    float inv[2][N2];
    unsigned char mode[2][N2];
};

// Half-sweep h (0-based within a block of red-black iterations) of colour c
// over the cells of rings >= 1 + h: rows and columns [1 + h, EX - 1 - h), the
// region the remaining half-sweeps of the block still read.  Colour-c cells
// of row ly sit at x = 2 j + odd, so a row has exactly (EX - 2 - 2 h) / 2 of
// them and the work is a dense index range.
template <int EX, int EY, int HH>
EFL_DEV void mix_half_sweep_h(MixTile<EX, EY>& T, int base, int c, float w, float omw) {
    constexpr int W2 = EX / 2, NJ = W2 - 1 - HH, ROWS = EY - 2 - 2 * HH, TOTAL = NJ * ROWS;
    constexpr int X0 = 1 + HH, Y0 = 1 + HH;
    const int o = 1 - c;
    for (int i = threadIdx.x; i < TOTAL; i += PS_THREADS) {
        const int r = i / NJ;
        const int ly = Y0 + r;
        const int odd = (base + ly + c) & 1;
        const int k = ly * W2 + ((X0 - odd + 1) >> 1) + (i - r * NJ);
        const unsigned char m = T.mode[c][k];
        if (m & MODE_STD) {  // 1 * d is d exactly and inv is 0.25: the general update, without its loads
            float nume = T.rc[c][k];
            nume = nume + T.d[o][k - 1 + odd];
            nume = nume + T.d[o][k + odd];
            nume = nume + T.d[o][k - W2];
            nume = nume + T.d[o][k + W2];
            T.d[c][k] = w * (nume * 0.25f) + omw * T.d[c][k];
        } else if (m & MODE_UPDATE) {
            const float4 wk = T.w[c][k];
            float nume = T.rc[c][k];
            nume = nume + wk.x * T.d[o][k - 1 + odd];
            nume = nume + wk.y * T.d[o][k + odd];
            nume = nume + wk.z * T.d[o][k - W2];
            nume = nume + wk.w * T.d[o][k + W2];
            T.d[c][k] = w * (nume * T.inv[c][k]) + omw * T.d[c][k];
        }
    }
}
template <int EX, int EY>
EFL_DEV void mix_half_sweep(MixTile<EX, EY>& T, int base, int c, int h, float w, float omw) {
    switch (h) {  // h < 2 * KMAX <= 8
        case 0: mix_half_sweep_h<EX, EY, 0>(T, base, c, w, omw); break;
        case 1: mix_half_sweep_h<EX, EY, 1>(T, base, c, w, omw); break;
        case 2: mix_half_sweep_h<EX, EY, 2>(T, base, c, w, omw); break;
        case 3: mix_half_sweep_h<EX, EY, 3>(T, base, c, w, omw); break;
        case 4: mix_half_sweep_h<EX, EY, 4>(T, base, c, w, omw); break;
        case 5: mix_half_sweep_h<EX, EY, 5>(T, base, c, w, omw); break;
        case 6: mix_half_sweep_h<EX, EY, 6>(T, base, c, w, omw); break;
        default: mix_half_sweep_h<EX, EY, 7>(T, base, c, w, omw); break;
    }
}

// FP64 residual at every cell of rings >= 1 (rc = f32(cdiv * r) for cells
// that update, d = 0) and the norms over the owned cells.
template <int EX, int EY>
EFL_DEV double2 mix_check(MixTile<EX, EY>& T, int base, int H, int tx, int ty, double cdiv, double factor) {
    constexpr int W2 = EX / 2;
    double ar = 0.0, ab = 0.0;
    for (int i = threadIdx.x; i < EX * EY; i += PS_THREADS) {
        const int ly = i / EX, lx = i - ly * EX;
        const int c = (base + lx + ly) & 1, o = 1 - c, odd = lx & 1;
        const int k = ly * W2 + (lx >> 1);
        const unsigned char m = T.mode[c][k];
        float rcv = 0.0f;
        const bool ring0 = lx == 0 || ly == 0 || lx == EX - 1 || ly == EY - 1;
        if ((m & MODE_COUNTED) && !ring0) {
            const float4 wk = T.w[c][k];
            double sum = (double)wk.x * T.p[o][k - 1 + odd];
            sum = sum + (double)wk.y * T.p[o][k + odd];
            sum = sum + (double)wk.z * T.p[o][k - W2];
            sum = sum + (double)wk.w * T.p[o][k + W2];
            const double bb = T.b[c][k];
            const double r = bb - factor * (T.den[c][k] * T.p[c][k] - sum);
            if (m & MODE_UPDATE) rcv = (float)(cdiv * r);
            if (lx >= H && lx < H + tx && ly >= H && ly < H + ty) {
                ar += r * r;
                ab += bb * bb;
            }
        }
        T.rc[c][k] = rcv;
        T.d[c][k] = 0.0f;
    }
    ar = warp_sum(ar);
    ab = warp_sum(ab);
    __shared__ double red_r[PS_THREADS / 32], red_b[PS_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red_r[wid] = ar;
        red_b[wid] = ab;
    }
    __syncthreads();
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        for (int q = 0; q < PS_THREADS / 32; ++q) {
            out.x += red_r[q];
            out.y += red_b[q];
        }
    }
    __syncthreads();
    return out;
}

// The halo ring of an EX x EY tile image with owned interior [H, EX - H) x [H, EY - H): 2 H rows of EX
// cells (top, then bottom), then 2 H columns of each interior row.  Every thread loads its (at most
// ceil(ring / threads)) cells from global memory before it stores any into the image, so a reload
// costs one round of L2 latency.
template <int EX, int EY, int H, class V>
EFL_DEV void halo_reload(V (*img)[(EX / 2) * EY], const V* src, size_t pitch, int gx0, int gy0, int base, int nx,
                         int ny) {
    constexpr int TY = EY - 2 * H, RING = 2 * H * EX + 2 * H * TY;
    constexpr int PER = (RING + PS_THREADS - 1) / PS_THREADS;
    V v[PER];
    int at[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int i = threadIdx.x + q * PS_THREADS;
        at[q] = -1;
        v[q] = V(0);
        if (i < RING) {
            int lx, ly;
            if (i < 2 * H * EX) {
                const int r = i / EX;
                lx = i - r * EX;
                ly = r < H ? r : TY + r;  // rows [0, H) then [EY - H, EY)
            } else {
                const int j = i - 2 * H * EX, r = j / (2 * H), c = j - r * (2 * H);
                ly = H + r;
                lx = c < H ? c : EX - 2 * H + c;  // columns [0, H) then [EX - H, EX)
            }
            const int gx = gx0 + lx, gy = gy0 + ly;
            if ((unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny) v[q] = __ldcg(&src[(size_t)gy * pitch + gx]);
            at[q] = (((base + lx + ly) & 1) << 24) | (ly * (EX / 2) + (lx >> 1));
        }
    }
#pragma unroll
    for (int q = 0; q < PER; ++q)
        if (at[q] >= 0) img[at[q] >> 24][at[q] & 0xffffff] = v[q];
}

template <int EX, int EY, int KMAX>
__global__ void __launch_bounds__(PS_THREADS, 1) k_gsmix_persistent(PersistentParams P, PF dbuf) {
    static_assert(KMAX >= 1 && KMAX <= 4, "mix_half_sweep dispatches h < 8");
    extern __shared__ __align__(16) unsigned char ps_raw[];
    MixTile<EX, EY>& T = *reinterpret_cast<MixTile<EX, EY>*>(ps_raw);
    constexpr int H = 2 * KMAX;
    constexpr int W2 = EX / 2;
    const int tx = EX - 2 * H, ty = EY - 2 * H;
    const Level64& L = P.L;
    const int tile = blockIdx.x;
    const int gx0 = (tile % P.tiles_x) * tx - H, gy0 = (tile / P.tiles_x) * ty - H;
    const int base = (gx0 + gy0) & 1;
    const unsigned nblocks = gridDim.x;

    for (int i = threadIdx.x; i < EX * EY; i += PS_THREADS) {
        const int ly = i / EX, lx = i - ly * EX;
        const int gx = gx0 + lx, gy = gy0 + ly;
        const int c = (base + lx + ly) & 1, k = ly * W2 + (lx >> 1);
        unsigned char m = MODE_SKIP;
        double den = 0.0, bb = 0.0, pv = 0.0;
        float inv = 0.0f;
        float4 wk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
            const bool ring = lx == 0 || ly == 0 || lx == EX - 1 || ly == EY - 1;
            const float phi = L.ls.at(gx, gy);
            bb = L.b.at(gx, gy);
            pv = __ldcg(&L.x.p[(size_t)gy * L.x.P + gx]);
            bool update = false, counted = false;
            if (phi < 0.0f) {
                const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
                if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                    counted = true;
                    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
                    float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int jx = gx + ox[q], jy = gy + oy[q];
                        if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                            const float level = L.ls.at(jx, jy);
                            if (level < 0.0f) {
                                den += (double)f[q];
                                wv[q] = f[q];
                            } else {
                                den += (double)f[q] * (1.0 - (double)level / (double)phi);
                            }
                        }
                    }
                    wk = make_float4(wv[0], wv[1], wv[2], wv[3]);
                    if (!(fabs(den) < (double)1.0e-6f)) {
                        update = true;
                        inv = (float)(1.0 / den);
                    }
                }
            }
            if (counted) m |= MODE_COUNTED;
            if (!ring) m |= update ? MODE_UPDATE : MODE_ZERO;  // the outer ring never updates here
            if (!ring && update && wk.x == 1.0f && wk.y == 1.0f && wk.z == 1.0f && wk.w == 1.0f) m |= MODE_STD;
        }
        T.mode[c][k] = m;
        T.den[c][k] = den;
        T.inv[c][k] = inv;
        T.b[c][k] = bb;
        T.w[c][k] = wk;
        T.p[c][k] = pv;
    }
    __syncthreads();
    const double cdiv = P.cdiv, factor = P.factor;
    const float w = (float)P.weight, omw = 1.0f - (float)P.weight;
    unsigned iters = 0;
    double2 part = mix_check(T, base, H, tx, ty, cdiv, factor);
    if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
    bool ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
    double r = ok ? ps_total_relative(P.partials, nblocks) : 0.0;
    const double r0 = r;
    // pending: the partials of the current p are written but their total is not read yet.  A check
    // whose next block has more than KMAX iterations skips its own grid barrier: the total is read
    // at the next block's first halo exchange, and if the solve had converged, the iterations run
    // meanwhile only changed the correction d, which is dropped -- p, the iteration count and r
    // are those of the check.
    bool pending = false;
    while (ok && (pending || (!(r <= P.tol) && iters < P.max_iters))) {
        unsigned todo = min(P.check_interval, P.max_iters - iters);
        unsigned done = 0;
        bool converged = false;
        while (ok && todo > 0) {
            const unsigned kk = min((unsigned)KMAX, todo);
            for (unsigned it = 0; it < kk; ++it) {
                mix_half_sweep(T, base, 1, 2 * it, w, omw);  // red: (x+y) odd
                __syncthreads();
                mix_half_sweep(T, base, 0, 2 * it + 1, w, omw);  // black
                __syncthreads();
            }
            todo -= kk;
            done += kk;
            if (todo > 0) {  // exchange the correction's halo
                for (int i = threadIdx.x; i < tx * ty; i += PS_THREADS) {
                    const int ly = H + i / tx, lx = H + i % tx, gx = gx0 + lx, gy = gy0 + ly;
                    if ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
                        __stcg(&dbuf.p[(size_t)gy * dbuf.P + gx], T.d[(base + lx + ly) & 1][ly * W2 + (lx >> 1)]);
                }
                ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
                if (!ok) break;
                if (pending) {
                    pending = false;
                    r = ps_total_relative(P.partials, nblocks);
                    if (r <= P.tol) {
                        converged = true;
                        break;
                    }
                }
                halo_reload<EX, EY, H>(T.d, dbuf.p, (size_t)dbuf.P, gx0, gy0, base, L.nx, L.ny);
                __syncthreads();
            }
        }
        if (!ok || converged) break;
        iters += done;
        // p += d on the owned cells (0 where the reference zeroes p), then exchange p.
        for (int i = threadIdx.x; i < tx * ty; i += PS_THREADS) {
            const int ly = H + i / tx, lx = H + i % tx, gx = gx0 + lx, gy = gy0 + ly;
            const int c = (base + lx + ly) & 1, k = ly * W2 + (lx >> 1);
            if ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
                const double pv = (T.mode[c][k] & MODE_UPDATE) ? T.p[c][k] + (double)T.d[c][k] : 0.0;
                T.p[c][k] = pv;
                __stcg(&L.x.p[(size_t)gy * L.x.P + gx], pv);
            }
        }
        ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
        if (!ok) break;
        halo_reload<EX, EY, H>(T.p, L.x.p, (size_t)L.x.P, gx0, gy0, base, L.nx, L.ny);
        __syncthreads();
        part = mix_check(T, base, H, tx, ty, cdiv, factor);
        if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
        if (min(P.check_interval, P.max_iters - iters) > (unsigned)KMAX) {
            pending = true;  // read at the next block's first halo exchange
        } else {
            ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
            if (!ok) break;
            r = ps_total_relative(P.partials, nblocks);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.result->iterations = iters;
        P.result->converged = (ok && r <= P.tol) ? 1 : 0;
        P.result->error = ok ? 0 : 1;
        P.result->r0 = r0;
        P.result->r1 = r;
    }
}

// ---------------------------------------------------------------------------
// Register-resident form of the persistent mixed solve.
//
// The same iterates as k_gsmix_persistent on every owned cell (the same f32
// update in the same operation order, the same checks), with the sweep made
// branch-free and short:
//  * Thread (bx, by) owns the 2 x 2 block of cells (2bx + i, 2by + j) of the
//    extended tile for the whole solve.  The tile origin is even, so the
//    block's colours are fixed: cells 0 = (0, 0) and 3 = (1, 1) have the
//    tile's base colour, cells 1 = (1, 0) and 2 = (0, 1) the other.  A
//    half-sweep updates two of a thread's cells; of each cell's four
//    neighbours, two are the thread's own cells (registers) and two belong to
//    the blocks beside it (shared memory).
//  * The correction d, right-hand side rc and 1/den live in registers; the
//    face weights in shared memory in thread order (one 16-byte load per
//    update, conflict-free); the shared image of d is stored per colour,
//    compressed along x, so a warp's neighbour loads are consecutive words.
//  * Every cell of rings >= 1 updates in every half-sweep (no shrinking
//    ranges, no per-cell tests): a wrong value from the stale outer ring
//    moves inwards one ring per half-sweep, so after the K iterations between
//    two halo exchanges (2K half-sweeps, halo 2K) the owned cells are exact.
//    Cells that are not update cells keep d = 0 (rc = 0, 1/den = 0); the
//    outermost ring, which only the halo exchange writes, is skipped.
// The FP64 iterate, right-hand side and diagonal stay in shared memory; only
// the residual checks read them.
template <int EX, int EY>
struct QuadTile {
    static constexpr int W2 = EX / 2, NB = (EX / 2) * (EY / 2);
    static constexpr int WP = W2 % 16 == 4 ? W2 : W2 + ((4 - W2 % 16) + 16) % 16;  // row stride of d
    double p[EY][EX];
    double b[EY][EX];
    double den[EY][EX];
    float4 w[4][NB];     // face weights of cell q of block t at [q][t]
    float d[2][EY][WP];  // [k][y][x / 2] with k = (x + y) & 1 in the image (k = 0: the tile's base colour)
};

// FP64 residual of the block's cells of rings >= 1 (rc = f32(cdiv r) on update
// cells, d = 0) and the block's norms over its owned counted cells, summed in
// a fixed order (returned by thread 0).
template <int EX, int EY, int NT>
EFL_DEV double2 quad_check(QuadTile<EX, EY>& T, int bx, int by, bool active, unsigned fl, float (&rc)[4],
                           float (&dv)[4], double cdiv, double factor) {
    constexpr int NB = QuadTile<EX, EY>::NB;
    double ar = 0.0, ab = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int lx = 2 * bx + (q & 1), ly = 2 * by + (q >> 1);
        float rcv = 0.0f;
        if ((fl >> (8 + q)) & 1u) {  // counted and not on the outermost ring
            const float4 wq = T.w[q][threadIdx.x < NB ? threadIdx.x : 0];
            double sum = (double)wq.x * T.p[ly][lx - 1];
            sum = sum + (double)wq.y * T.p[ly][lx + 1];
            sum = sum + (double)wq.z * T.p[ly - 1][lx];
            sum = sum + (double)wq.w * T.p[ly + 1][lx];
            const double bb = T.b[ly][lx];
            const double r = bb - factor * (T.den[ly][lx] * T.p[ly][lx] - sum);
            if ((fl >> q) & 1u) rcv = (float)(cdiv * r);
            if ((fl >> (16 + q)) & 1u) {
                ar += r * r;
                ab += bb * bb;
            }
        }
        rc[q] = rcv;
        dv[q] = 0.0f;
    }
    if (active) {
#pragma unroll
        for (int q = 0; q < 4; ++q) T.d[q == 0 || q == 3 ? 0 : 1][2 * by + (q >> 1)][bx] = 0.0f;
    }
    ar = warp_sum(ar);
    ab = warp_sum(ab);
    __shared__ double red_r[NT / 32], red_b[NT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red_r[wid] = ar;
        red_b[wid] = ab;
    }
    __syncthreads();
    double2 out = make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        for (int k = 0; k < NT / 32; ++k) {
            out.x += red_r[k];
            out.y += red_b[k];
        }
    }
    __syncthreads();
    return out;
}

// One cell update (gauss_seidel.wgsl:45-88 on the correction, in the
// reference's operation order: left, right, up, down).
EFL_DEV float quad_update(float rc, float4 w, float inv, float d, float dl, float dr, float du, float dd, float wgt,
                          float omw) {
    float nume = rc;
    nume = nume + w.x * dl;
    nume = nume + w.y * dr;
    nume = nume + w.z * du;
    nume = nume + w.w * dd;
    return wgt * (nume * inv) + omw * d;
}

template <int EX, int EY, int KMAX, int NT>
__global__ void __launch_bounds__(NT, 1) k_gsmix_quad(PersistentParams P, PF dbuf) {
    static_assert(KMAX >= 1 && EX % 2 == 0 && EY % 2 == 0, "even tile image");
    static_assert((EX / 2) * (EY / 2) <= NT && NT % 32 == 0, "one thread per 2 x 2 block");
    extern __shared__ __align__(16) unsigned char ps_raw[];
    QuadTile<EX, EY>& T = *reinterpret_cast<QuadTile<EX, EY>*>(ps_raw);
    constexpr int H = 2 * KMAX, W2 = EX / 2, NB = QuadTile<EX, EY>::NB;
    constexpr int TXo = EX - 2 * H, TYo = EY - 2 * H;
    static_assert(H % 2 == 0, "even halo: blocks are wholly owned or wholly halo");
    const Level64& L = P.L;
    const int tile = blockIdx.x;
    const int gx0 = (tile % P.tiles_x) * TXo - H, gy0 = (tile / P.tiles_x) * TYo - H;
    const unsigned nblocks = gridDim.x;
    const bool active = threadIdx.x < NB;
    const int bx = active ? (int)threadIdx.x % W2 : 0, by = active ? (int)threadIdx.x / W2 : 0;
    const int base = (gx0 + gy0) & 1;  // colour of cells 0 and 3 (1 = red, (x + y) odd)
    const bool owned = bx >= H / 2 && bx < (H + TXo) / 2 && by >= H / 2 && by < (H + TYo) / 2;
    const bool ring0x = bx == 0 || bx == W2 - 1, ring0y = by == 0 || by == EY / 2 - 1;
    float inv[4], rc[4], dv[4];
    // bit q: update cell; bit 4 + q: live (not on the outermost ring); bit 8 + q: counted and live;
    // bit 16 + q: owned and in the domain
    unsigned fl = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int lx = 2 * bx + (q & 1), ly = 2 * by + (q >> 1);
        const int gx = gx0 + lx, gy = gy0 + ly;
        const bool edge = (ring0x && ((q & 1) == (bx == 0 ? 0 : 1))) || (ring0y && ((q >> 1) == (by == 0 ? 0 : 1)));
        if (active && !edge) fl |= 1u << (4 + q);
        float4 wq = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        inv[q] = 0.0f;
        rc[q] = 0.0f;
        dv[q] = 0.0f;
        double den = 0.0, bb = 0.0, pv = 0.0;
        if (active && (unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
            const float phi = L.ls.at(gx, gy);
            bb = L.b.at(gx, gy);
            pv = __ldcg(&L.x.p[(size_t)gy * L.x.P + gx]);
            if (owned) fl |= 1u << (16 + q);
            if (phi < 0.0f) {
                const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
                if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                    if (!edge) fl |= 1u << (8 + q);
                    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
                    float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int jx = gx + ox[k], jy = gy + oy[k];
                        if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                            const float level = L.ls.at(jx, jy);
                            if (level < 0.0f) {
                                den += (double)f[k];
                                wv[k] = f[k];
                            } else {
                                den += (double)f[k] * (1.0 - (double)level / (double)phi);
                            }
                        }
                    }
                    wq = make_float4(wv[0], wv[1], wv[2], wv[3]);
                    if (!(fabs(den) < (double)1.0e-6f) && !edge) {
                        fl |= 1u << q;
                        inv[q] = (float)(1.0 / den);
                    }
                }
            }
        }
        if (active) {
            T.p[ly][lx] = pv;
            T.b[ly][lx] = bb;
            T.den[ly][lx] = den;
            T.w[q][threadIdx.x] = wq;
        }
    }
    __syncthreads();
    const double cdiv = P.cdiv, factor = P.factor;
    const float wgt = (float)P.weight, omw = 1.0f - (float)P.weight;
    const int t = active ? (int)threadIdx.x : 0;
    const int r0 = 2 * by, r1 = 2 * by + 1;
    // Shared-memory rows of the neighbours that belong to other blocks (clamped inside the image for the
    // outermost blocks, whose loads are skipped).
    const int bxl = bx > 0 ? bx - 1 : 0, bxr = bx < W2 - 1 ? bx + 1 : bx;
    const int rup = r0 > 0 ? r0 - 1 : 0, rdn = r1 < EY - 1 ? r1 + 1 : r1;
    // ring of the block (its outermost cell's distance to the image edge, + 1 for its inner cells)
    const int bring = min(min(2 * bx + 1, EX - 2 * bx), min(2 * by + 1, EY - 2 * by)) - 1;
    auto sweep_base = [&]() {  // cells 0 and 3 (the base colour c0 = base); neighbours of the other colour
        float(*Do)[QuadTile<EX, EY>::WP] = T.d[1];
        const float dl0 = (fl & 0x10u) ? Do[r0][bxl] : 0.0f, du0 = (fl & 0x10u) ? Do[rup][bx] : 0.0f;
        const float dr3 = (fl & 0x80u) ? Do[r1][bxr] : 0.0f, dd3 = (fl & 0x80u) ? Do[rdn][bx] : 0.0f;
        if (fl & 0x10u) {
            dv[0] = quad_update(rc[0], T.w[0][t], inv[0], dv[0], dl0, dv[1], du0, dv[2], wgt, omw);
            T.d[0][r0][bx] = dv[0];
        }
        if (fl & 0x80u) {
            dv[3] = quad_update(rc[3], T.w[3][t], inv[3], dv[3], dv[2], dr3, dv[1], dd3, wgt, omw);
            T.d[0][r1][bx] = dv[3];
        }
    };
    auto sweep_other = [&]() {  // cells 1 and 2; neighbours of the base colour
        float(*Do)[QuadTile<EX, EY>::WP] = T.d[0];
        const float dr1 = (fl & 0x20u) ? Do[r0][bxr] : 0.0f, du1 = (fl & 0x20u) ? Do[rup][bx] : 0.0f;
        const float dl2 = (fl & 0x40u) ? Do[r1][bxl] : 0.0f, dd2 = (fl & 0x40u) ? Do[rdn][bx] : 0.0f;
        if (fl & 0x20u) {
            dv[1] = quad_update(rc[1], T.w[1][t], inv[1], dv[1], dv[0], dr1, du1, dv[3], wgt, omw);
            T.d[1][r0][bx] = dv[1];
        }
        if (fl & 0x40u) {
            dv[2] = quad_update(rc[2], T.w[2][t], inv[2], dv[2], dl2, dv[3], dv[0], dd2, wgt, omw);
            T.d[1][r1][bx] = dv[2];
        }
    };
    auto store_d = [&]() {  // all four cells into the shared image
        if (active) {
            T.d[0][r0][bx] = dv[0];
            T.d[1][r0][bx] = dv[1];
            T.d[1][r1][bx] = dv[2];
            T.d[0][r1][bx] = dv[3];
        }
    };

    unsigned iters = 0, xch = 0;  // xch: correction exchanges so far
    double2 part = quad_check<EX, EY, NT>(T, bx, by, active, fl, rc, dv, cdiv, factor);
    if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
    bool ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
    double r = ok ? ps_total_relative(P.partials, nblocks) : 0.0;
    const double r0v = r;
    bool pending = false;  // as in k_gsmix_persistent: a check's total read at the next block's first exchange
    while (ok && (pending || (!(r <= P.tol) && iters < P.max_iters))) {
        unsigned todo = min(P.check_interval, P.max_iters - iters);
        unsigned done = 0;
        bool converged = false;
        while (ok && todo > 0) {
            const unsigned kk = min((unsigned)KMAX, todo);
            for (unsigned it = 0; it < kk; ++it) {
                if (bring + 1 >= 1 + 2 * (int)it) {  // a cell of the block lies in the region still needed
                    if (base) sweep_base();  // red ((x + y) odd) first
                    else sweep_other();
                }
                __syncthreads();
                if (bring + 1 >= 2 + 2 * (int)it) {
                    if (base) sweep_other();
                    else sweep_base();
                }
                __syncthreads();
            }
            todo -= kk;
            done += kk;
            if (todo > 0) {  // exchange the correction's halo through L2
                // Alternate planes: a CTA that runs on to the next exchange writes the other plane, so it
                // cannot overwrite values a slower neighbour is still reloading (two exchanges apart there
                // is always a grid barrier).
                const PF& db = (xch++ & 1) ? P.dbuf2 : dbuf;
                if (owned) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if ((fl >> (16 + q)) & 1u)
                            __stcg(&db.p[(size_t)(gy0 + 2 * by + (q >> 1)) * db.P + gx0 + 2 * bx + (q & 1)], dv[q]);
                }
                ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
                if (!ok) break;
                if (pending) {
                    pending = false;
                    r = ps_total_relative(P.partials, nblocks);
                    if (r <= P.tol) {
                        converged = true;
                        break;
                    }
                }
                if (active && !owned) {
                    float hv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int gx = gx0 + 2 * bx + (q & 1), gy = gy0 + 2 * by + (q >> 1);
                        hv[q] = ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
                                    ? __ldcg(&db.p[(size_t)gy * db.P + gx])
                                    : 0.0f;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) dv[q] = hv[q];
                    store_d();
                }
                __syncthreads();
            }
        }
        if (!ok || converged) break;
        iters += done;
        // p += d on the owned cells (0 where the reference zeroes p), then exchange p.
        if (owned) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if ((fl >> (16 + q)) & 1u) {
                    const int lx = 2 * bx + (q & 1), ly = 2 * by + (q >> 1);
                    const double pv = ((fl >> q) & 1u) ? T.p[ly][lx] + (double)dv[q] : 0.0;
                    T.p[ly][lx] = pv;
                    __stcg(&L.x.p[(size_t)(gy0 + ly) * L.x.P + gx0 + lx], pv);
                }
            }
        }
        ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
        if (!ok) break;
        if (active && !owned) {
            double hp[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int gx = gx0 + 2 * bx + (q & 1), gy = gy0 + 2 * by + (q >> 1);
                hp[q] = ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
                            ? __ldcg(&L.x.p[(size_t)gy * L.x.P + gx])
                            : 0.0;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) T.p[2 * by + (q >> 1)][2 * bx + (q & 1)] = hp[q];
        }
        __syncthreads();
        part = quad_check<EX, EY, NT>(T, bx, by, active, fl, rc, dv, cdiv, factor);
        if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
        if (min(P.check_interval, P.max_iters - iters) > (unsigned)KMAX) {
            pending = true;
        } else {
            ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
            if (!ok) break;
            r = ps_total_relative(P.partials, nblocks);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.result->iterations = iters;
        P.result->converged = (ok && r <= P.tol) ? 1 : 0;
        P.result->error = ok ? 0 : 1;
        P.result->r0 = r0v;
        P.result->r1 = r;
    }
}

// ---------------------------------------------------------------------------
// Paired-lane form of the persistent mixed solve (4 x 2 cells per thread).
//
// The same iterates as k_gsmix_quad (the same f32 update in the same
// operation order on every cell, the same FP64 checks), with each thread
// owning a 4 x 2 block of the extended tile: cells c0..c3 in its upper row,
// c4..c7 in its lower one.  A half-sweep updates four of them, in two pairs
// of one colour (c0, c2) and (c5, c7), or (c1, c3) and (c4, c6), and the two
// cells of a pair are the two lanes of Blackwell's paired f32 instructions
// (mul.rn.f32x2 for the products, fma.rn.f32x2 by a run-time 1.0 for the
// sums: per lane the IEEE-rounded f32 product and sum, so each lane is the
// scalar update exactly).  The layout makes the operand pairs fall out of it:
//  * in the colour-compressed shared image of the correction
//    (d[k][y][x / 2]) a pair's two cells are adjacent words, so one 8-byte
//    load brings both neighbours above (or below) a pair and one 8-byte store
//    publishes the pair;
//  * of the eight neighbour values a pair needs, four come from the thread's
//    own registers as ready-made pairs, two from one 8-byte load and two
//    (left of c0 / c4, right of c3 / c7) from a 4-byte load packed with a
//    register lane;
//  * the face weights, 1/den and the right-hand side stay in registers as
//    lane pairs for the whole solve.
// Cells on the tile image's outermost ring update too, from clamped
// neighbour values: their results are as wrong as the stale values a frozen
// ring would hold, and like those they move inwards one ring per half-sweep,
// so the owned cells are exact after the 2K half-sweeps between exchanges
// (every value stays finite, and the exchange reloads the ring).
typedef unsigned long long f32x2;  // lane 0 = low word
EFL_DEV f32x2 x2_pack(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
EFL_DEV float x2_lane(f32x2 v, int lane) {
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    return lane ? b : a;
}
EFL_DEV f32x2 x2_mul(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
// round(a + c) per lane, written as fma(a, one, c) with one = 1.0 known only at
// run time.  ptxas contracts a paired product feeding a paired add (mul.rn /
// add.rn f32x2) into one fused multiply-add, -fmad=false notwithstanding,
// which drops the product's rounding; a product feeding the multiplicand of
// an FMA by an unknown factor cannot be contracted, and a * 1 + c rounds once,
// exactly like the add (signed zeros included).
EFL_DEV f32x2 x2_add1(f32x2 a, f32x2 one, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(one), "l"(c));
    return r;
}
// The update of two cells: nume = rc + wl L + wr R + wu U + wd D (in that
// order, each product rounded), d' = wgt (nume inv) + omw d.
EFL_DEV f32x2 oct_update(f32x2 rc, f32x2 wl, f32x2 wr, f32x2 wu, f32x2 wd, f32x2 inv, f32x2 omw, f32x2 d, f32x2 L,
                         f32x2 R, f32x2 U, f32x2 D, f32x2 wgt, f32x2 one) {
    f32x2 n = x2_add1(x2_mul(wl, L), one, rc);
    n = x2_add1(x2_mul(wr, R), one, n);
    n = x2_add1(x2_mul(wu, U), one, n);
    n = x2_add1(x2_mul(wd, D), one, n);
    return x2_add1(x2_mul(wgt, x2_mul(n, inv)), one, x2_mul(omw, d));
}

template <int EX, int EY, int ROWS>
struct OctTile {
    static constexpr int W2 = EX / 2, W4 = EX / 4, NB = (EX / 4) * (EY / ROWS);
    static constexpr int WP = W2 % 16 == 4 ? W2 : W2 + ((4 - W2 % 16) + 16) % 16;  // row stride of d (words)
    // The FP64 planes hold cell (x, y) at y * RS + (x & 3) * W4 + (x >> 2): the threads of a warp (consecutive
    // blocks) reading the same cell of their blocks read consecutive words, and RS puts the next row of
    // blocks (ROWS rows down) 16 banks over, so a half-warp that spans two block rows does not conflict.
    static constexpr int rs_pad() {
        int pad = 0;
        while ((ROWS * (4 * W4 + pad)) % 16 != 8 && pad < 16) ++pad;
        return pad;
    }
    static constexpr int RS = 4 * W4 + rs_pad();
    EFL_DEV static int ix(int y, int x) { return y * RS + (x & 3) * W4 + (x >> 2); }
    double p[EY * RS];
    double b[EY * RS];
    double den[EY * RS];
    float d[2][EY][WP];  // [k][y][x / 2], k = (x + y) & 1 in the image (k = 0: the tile's base colour)
};

// Cell q of a thread's 4 x ROWS block sits at (i, j) = (q & 3, q >> 2); its colour in the image is
// k = (i + j) & 1, and it is lane i >> 1 of pair 2 j + k: the pair of the two cells of colour k in row j,
// which are adjacent words (2 bx, 2 bx + 1) of the colour-compressed image.
EFL_DEV constexpr int oct_pair(int q) { return 2 * (q >> 2) + (((q & 3) + (q >> 2)) & 1); }
EFL_DEV constexpr int oct_lane(int q) { return (q & 3) >> 1; }

template <int EX, int EY, int KMAX, int NT, int ROWS>
__global__ void __launch_bounds__(NT, 1) k_gsmix_oct(PersistentParams P, PF dbuf) {
    using Tile = OctTile<EX, EY, ROWS>;
    constexpr int NC = 4 * ROWS, NPAIR = 2 * ROWS;
    static_assert(KMAX >= 1 && EX % 4 == 0 && EY % ROWS == 0 && ROWS % 2 == 0, "4 x ROWS blocks");
    static_assert(Tile::NB <= NT && NT % 32 == 0, "one thread per block");
    static_assert((2 * KMAX) % 4 == 0 && (2 * KMAX) % ROWS == 0, "halo of whole blocks");
    static_assert(NC <= 16, "cell flags in 64 bits");
    extern __shared__ __align__(16) unsigned char ps_raw[];
    Tile& T = *reinterpret_cast<Tile*>(ps_raw);
    constexpr int H = 2 * KMAX, W2 = Tile::W2, W4 = Tile::W4, NB = Tile::NB, WP = Tile::WP;
    constexpr int TXo = EX - 2 * H, TYo = EY - 2 * H;
    const Level64& L = P.L;
    const int tile = blockIdx.x;
    const int gx0 = (tile % P.tiles_x) * TXo - H, gy0 = (tile / P.tiles_x) * TYo - H;
    const unsigned nblocks = gridDim.x;
    const bool active = threadIdx.x < NB;
    const int bx = active ? (int)threadIdx.x % W4 : 0, by = active ? (int)threadIdx.x / W4 : 0;
    const int base = (gx0 + gy0) & 1;  // colour of the k = 0 cells (1 = red, (x + y) odd)
    const bool owned = active && bx >= H / 4 && bx < (H + TXo) / 4 && by >= H / ROWS && by < (H + TYo) / ROWS;
    const int x0 = 4 * bx, y0 = ROWS * by;
    // FP64 plane index of the cell (x0 + i, y0 + j), i in -1 .. 4 and j in -1 .. ROWS (constants once unrolled)
    const int pbase = y0 * Tile::RS + bx;
    auto pix = [&](int i, int j) { return pbase + j * Tile::RS + (i & 3) * W4 + (i >> 2); };
    const float wgt = (float)P.weight, omw1 = 1.0f - (float)P.weight;
    // bit q: update cell; 16 + q: live (not on the outermost ring); 32 + q: counted and live; 48 + q: owned and
    // in the domain
    unsigned long long fl = 0;
    f32x2 wl[NPAIR], wr[NPAIR], wu[NPAIR], wd[NPAIR], inv[NPAIR], rc[NPAIR], dv[NPAIR];
    {
        float fw[4][NC], finv[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const int lx = x0 + (q & 3), ly = y0 + (q >> 2);
            const int gx = gx0 + lx, gy = gy0 + ly;
            const bool live = active && lx > 0 && lx < EX - 1 && ly > 0 && ly < EY - 1;
            if (live) fl |= 1ull << (16 + q);
            float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            finv[q] = 0.0f;
            double den = 0.0, bb = 0.0, pv = 0.0;
            if (active && (unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
                const float phi = L.ls.at(gx, gy);
                bb = L.b.at(gx, gy);
                pv = __ldcg(&L.x.p[(size_t)gy * L.x.P + gx]);
                if (owned) fl |= 1ull << (48 + q);
                if (phi < 0.0f) {
                    const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
                    if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                        if (live) fl |= 1ull << (32 + q);
                        const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int jx = gx + ox[k], jy = gy + oy[k];
                            if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                                const float level = L.ls.at(jx, jy);
                                if (level < 0.0f) {
                                    den += (double)f[k];
                                    wv[k] = f[k];
                                } else {
                                    den += (double)f[k] * (1.0 - (double)level / (double)phi);
                                }
                            }
                        }
                        if (!(fabs(den) < (double)1.0e-6f)) {
                            if (live) fl |= 1ull << q;
                            finv[q] = (float)(1.0 / den);
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) fw[k][q] = wv[k];
            if (active) {
                T.p[pix(q & 3, q >> 2)] = pv;
                T.b[pix(q & 3, q >> 2)] = bb;
                T.den[pix(q & 3, q >> 2)] = den;
            }
        }
        // pair 2 j + k = the cells (i0, j), (i0 + 2, j) with i0 = (k + j) & 1
#pragma unroll
        for (int j = 0; j < ROWS; ++j)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int i0 = (k + j) & 1, qa = 4 * j + i0, qb = qa + 2, pi = 2 * j + k;
                wl[pi] = x2_pack(fw[0][qa], fw[0][qb]);
                wr[pi] = x2_pack(fw[1][qa], fw[1][qb]);
                wu[pi] = x2_pack(fw[2][qa], fw[2][qb]);
                wd[pi] = x2_pack(fw[3][qa], fw[3][qb]);
                inv[pi] = x2_pack(finv[qa], finv[qb]);
                rc[pi] = 0;
                dv[pi] = 0;
            }
    }
    // every word of the correction image starts at 0 (rows' padding included)
    for (int i = threadIdx.x; i < 2 * EY * WP; i += NT) (&T.d[0][0][0])[i] = 0.0f;
    __syncthreads();
    const double cdiv = P.cdiv, factor = P.factor;
    const f32x2 wgt2 = x2_pack(wgt, wgt), omw2 = x2_pack(omw1, omw1), one2 = x2_pack(P.one, P.one);
    // Shared-memory words of the neighbours in other blocks, clamped inside the image for the outermost blocks.
    // The one-word neighbours left and right of the block come from 8-byte loads of the aligned word pair that
    // holds them (the left one is the pair's high word, the right one its low word): a warp's side loads are
    // then consecutive 8-byte words, free of bank conflicts like the pair loads.
    const int cl = max(2 * bx - 2, 0), cr = min(2 * bx + 2, W2 - 2);
    const int ru = max(y0 - 1, 0), rd = min(y0 + ROWS, EY - 1);
    // most central ring among the block's cells
    const int bmax = min(min(x0 + 3, EX - 1 - x0), min(y0 + ROWS - 1, EY - 1 - y0));
    // Half-sweep of colour K01: the pairs 2 j + K01 of every row j, neighbours of the other colour: above and
    // below from the pairs of the rows beside it (shared memory past the block's edge rows), left and right
    // from the other pair of the same row and one word of shared memory past the block's edge columns.
    auto sweep = [&](auto kc) {
        constexpr int K01 = decltype(kc)::value;
        float(*Do)[WP] = T.d[1 - K01];
        const f32x2 upw = *reinterpret_cast<const f32x2*>(&Do[ru][2 * bx]);
        const f32x2 dnw = *reinterpret_cast<const f32x2*>(&Do[rd][2 * bx]);
        float side[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            const f32x2 w2 = *reinterpret_cast<const f32x2*>(&Do[y0 + j][((K01 + j) & 1) ? cr : cl]);
            side[j] = x2_lane(w2, ((K01 + j) & 1) ? 0 : 1);
        }
#pragma unroll
        for (int j = 0; j < ROWS; ++j) {
            const int pi = 2 * j + K01, po = 2 * j + (1 - K01);
            const f32x2 U = j > 0 ? dv[2 * (j - 1) + (1 - K01)] : upw;
            const f32x2 D = j < ROWS - 1 ? dv[2 * (j + 1) + (1 - K01)] : dnw;
            f32x2 Lf, Rt;
            if ((K01 + j) & 1) {  // cells 1 and 3: left (0, 2) in registers, right (2, 4)
                Lf = dv[po];
                Rt = x2_pack(x2_lane(dv[po], 1), side[j]);
            } else {  // cells 0 and 2: left (-1, 1), right (1, 3) in registers
                Lf = x2_pack(side[j], x2_lane(dv[po], 0));
                Rt = dv[po];
            }
            dv[pi] = oct_update(rc[pi], wl[pi], wr[pi], wu[pi], wd[pi], inv[pi], omw2, dv[pi], Lf, Rt, U, D, wgt2,
                                one2);
        }
        if (active) {
#pragma unroll
            for (int j = 0; j < ROWS; ++j) *reinterpret_cast<f32x2*>(&T.d[K01][y0 + j][2 * bx]) = dv[2 * j + K01];
        }
    };
    // FP64 residual of the live counted cells, rc = f32(cdiv r) on update cells, d = 0, and the CTA's norms over
    // its owned counted cells (fixed order; returned by thread 0).
    auto check = [&]() -> double2 {
        double ar = 0.0, ab = 0.0;
        float frc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const int i = oct_pair(q), ln = oct_lane(q);
            float rcv = 0.0f;
            if ((fl >> (32 + q)) & 1ull) {
                const int ci = q & 3, cj = q >> 2;
                double sum = (double)x2_lane(wl[i], ln) * T.p[pix(ci - 1, cj)];
                sum = sum + (double)x2_lane(wr[i], ln) * T.p[pix(ci + 1, cj)];
                sum = sum + (double)x2_lane(wu[i], ln) * T.p[pix(ci, cj - 1)];
                sum = sum + (double)x2_lane(wd[i], ln) * T.p[pix(ci, cj + 1)];
                const double bb = T.b[pix(ci, cj)];
                const double r = bb - factor * (T.den[pix(ci, cj)] * T.p[pix(ci, cj)] - sum);
                if ((fl >> q) & 1ull) rcv = (float)(cdiv * r);
                if ((fl >> (48 + q)) & 1ull) {
                    ar += r * r;
                    ab += bb * bb;
                }
            }
            frc[q] = rcv;
        }
#pragma unroll
        for (int j = 0; j < ROWS; ++j)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int qa = 4 * j + ((k + j) & 1);
                rc[2 * j + k] = x2_pack(frc[qa], frc[qa + 2]);
                dv[2 * j + k] = 0;
            }
        if (active) {
#pragma unroll
            for (int j = 0; j < ROWS; ++j) {
                *reinterpret_cast<f32x2*>(&T.d[0][y0 + j][2 * bx]) = 0;
                *reinterpret_cast<f32x2*>(&T.d[1][y0 + j][2 * bx]) = 0;
            }
        }
        ar = warp_sum(ar);
        ab = warp_sum(ab);
        __shared__ double red_r[NT / 32], red_b[NT / 32];
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) {
            red_r[wid] = ar;
            red_b[wid] = ab;
        }
        __syncthreads();
        double2 out = make_double2(0.0, 0.0);
        if (threadIdx.x == 0) {
            for (int k = 0; k < NT / 32; ++k) {
                out.x += red_r[k];
                out.y += red_b[k];
            }
        }
        __syncthreads();
        return out;
    };
    const std::integral_constant<int, 0> c0{};
    const std::integral_constant<int, 1> c1{};

    unsigned iters = 0, xch = 0;
    double2 part = check();
    if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
    bool ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
    double r = ok ? ps_total_relative(P.partials, nblocks) : 0.0;
    const double r0v = r;
    bool pending = false;  // a check's total, read at the next block's first exchange
    while (ok && (pending || (!(r <= P.tol) && iters < P.max_iters))) {
        unsigned todo = min(P.check_interval, P.max_iters - iters);
        unsigned done = 0;
        bool converged = false;
        while (ok && todo > 0) {
            const unsigned kk = min((unsigned)KMAX, todo);
            for (unsigned it = 0; it < kk; ++it) {
                if (bmax >= 1 + 2 * (int)it) {  // a cell of the block lies in the region still needed
                    if (base) sweep(c0);  // red ((x + y) odd) first
                    else sweep(c1);
                }
                __syncthreads();
                if (bmax >= 2 + 2 * (int)it) {
                    if (base) sweep(c1);
                    else sweep(c0);
                }
                __syncthreads();
            }
            todo -= kk;
            done += kk;
            if (todo > 0) {  // exchange the correction's halo through L2, alternating planes
                const PF& db = (xch++ & 1) ? P.dbuf2 : dbuf;
                if (owned) {
#pragma unroll
                    for (int q = 0; q < NC; ++q)
                        if ((fl >> (48 + q)) & 1ull)
                            __stcg(&db.p[(size_t)(gy0 + y0 + (q >> 2)) * db.P + gx0 + x0 + (q & 3)],
                                   x2_lane(dv[oct_pair(q)], oct_lane(q)));
                }
                ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
                if (!ok) break;
                if (pending) {
                    pending = false;
                    r = ps_total_relative(P.partials, nblocks);
                    if (r <= P.tol) {
                        converged = true;
                        break;
                    }
                }
                if (active && !owned) {
                    float hv[NC];
#pragma unroll
                    for (int q = 0; q < NC; ++q) {
                        const int gx = gx0 + x0 + (q & 3), gy = gy0 + y0 + (q >> 2);
                        hv[q] = ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
                                    ? __ldcg(&db.p[(size_t)gy * db.P + gx])
                                    : 0.0f;
                    }
#pragma unroll
                    for (int j = 0; j < ROWS; ++j)
#pragma unroll
                        for (int k = 0; k < 2; ++k) {
                            const int qa = 4 * j + ((k + j) & 1);
                            dv[2 * j + k] = x2_pack(hv[qa], hv[qa + 2]);
                            *reinterpret_cast<f32x2*>(&T.d[k][y0 + j][2 * bx]) = dv[2 * j + k];
                        }
                }
                __syncthreads();
            }
        }
        if (!ok || converged) break;
        iters += done;
        // p += d on the owned cells (0 where the reference zeroes p), then exchange p.
        if (owned) {
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                if ((fl >> (48 + q)) & 1ull) {
                    const int lx = x0 + (q & 3), ly = y0 + (q >> 2);
                    const double pv =
                        ((fl >> q) & 1ull) ? T.p[pix(q & 3, q >> 2)] + (double)x2_lane(dv[oct_pair(q)], oct_lane(q)) : 0.0;
                    T.p[pix(q & 3, q >> 2)] = pv;
                    __stcg(&L.x.p[(size_t)(gy0 + ly) * L.x.P + gx0 + lx], pv);
                }
            }
        }
        ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
        if (!ok) break;
        if (active && !owned) {
            double hp[NC];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const int gx = gx0 + x0 + (q & 3), gy = gy0 + y0 + (q >> 2);
                hp[q] = ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
                            ? __ldcg(&L.x.p[(size_t)gy * L.x.P + gx])
                            : 0.0;
            }
#pragma unroll
            for (int q = 0; q < NC; ++q) T.p[pix(q & 3, q >> 2)] = hp[q];
        }
        __syncthreads();
        part = check();
        if (threadIdx.x == 0) P.partials[blockIdx.x] = part;
        if (min(P.check_interval, P.max_iters - iters) > (unsigned)KMAX) {
            pending = true;
        } else {
            ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
            if (!ok) break;
            r = ps_total_relative(P.partials, nblocks);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.result->iterations = iters;
        P.result->converged = (ok && r <= P.tol) ? 1 : 0;
        P.result->error = ok ? 0 : 1;
        P.result->r0 = r0v;
        P.result->r1 = r;
    }
}

// The reference's fixed-count f32 sweeps (gauss_seidel.wgsl:12-88, `iters`
// red-black iterations, red first) as ONE cooperative launch for grids of at
// most one 64 x 32 tile per SM (C1's 256^2, 512^2): the 2 x 2-block layout
// of k_gsmix_quad on the pressure itself.  Per cell, with the reference's f32
// coefficients: update cells p = w (nume / den) + (1 - w) p, zero cells
// (air, fully solid, |den| < 1e-6) p = 0, the outermost ring untouched.  The
// owned cells are exchanged through L2 every 4 iterations (alternating
// planes) and stored to `out` after a last grid barrier (no CTA may still be
// loading its first image from `out`).
template <int EX, int EY>
struct Quad32Tile {
    static constexpr int W2 = EX / 2, NB = (EX / 2) * (EY / 2);
    static constexpr int WP = W2 % 16 == 4 ? W2 : W2 + ((4 - W2 % 16) + 16) % 16;
    float4 w[4][NB];
    float p[2][EY][WP];  // [k][y][x / 2], k = (x + y) & 1 in the image (k = 0: the tile's base colour)
};
struct Gs32Params {
    Level L;  // x = the pressure (read at the start, written at the end), b, ls, fu, fv
    PF xb[2];  // exchange planes
    int tiles_x, iters;
    float cdiv, weight;
    GridBarrier* barrier;
    long long spin_limit;
    int* err;  // set to 2 if a grid barrier timed out (reported with the TMA sweep's flag)
};
EFL_DEV float gs32_update(float cb, float4 w, float den, float p, float pl, float pr, float pu, float pd, float wgt,
                          float omw, unsigned upd, unsigned zero) {
    float nume = cb;
    nume = nume + w.x * pl;
    nume = nume + w.y * pr;
    nume = nume + w.z * pu;
    nume = nume + w.w * pd;
    const float pn = nume / den;
    const float v = wgt * pn + omw * p;
    return upd ? v : (zero ? 0.0f : p);
}
template <int EX, int EY, int KMAX, int NT>
__global__ void __launch_bounds__(NT, 1) k_gs32_quad(Gs32Params P) {
    static_assert((EX / 2) * (EY / 2) <= NT && NT % 32 == 0 && EX % 2 == 0 && EY % 2 == 0, "2 x 2 blocks");
    extern __shared__ __align__(16) unsigned char q32_raw[];
    Quad32Tile<EX, EY>& T = *reinterpret_cast<Quad32Tile<EX, EY>*>(q32_raw);
    constexpr int H = 2 * KMAX, W2 = EX / 2, NB = Quad32Tile<EX, EY>::NB, WP = Quad32Tile<EX, EY>::WP;
    constexpr int TXo = EX - 2 * H, TYo = EY - 2 * H;
    const Level& L = P.L;
    const int gx0 = (blockIdx.x % P.tiles_x) * TXo - H, gy0 = (blockIdx.x / P.tiles_x) * TYo - H;
    const unsigned nblocks = gridDim.x;
    const bool active = threadIdx.x < NB;
    const int bx = active ? (int)threadIdx.x % W2 : 0, by = active ? (int)threadIdx.x / W2 : 0;
    const int base = (gx0 + gy0) & 1;
    const bool owned = bx >= H / 2 && bx < (H + TXo) / 2 && by >= H / 2 && by < (H + TYo) / 2;
    const bool ring0x = bx == 0 || bx == W2 - 1, ring0y = by == 0 || by == EY / 2 - 1;
    float pv[4], cb[4], den[4];
    unsigned fl = 0;  // bit q: update; bit 4 + q: zero; bit 8 + q: live (in the domain, not the outer ring);
                      // bit 16 + q: owned and in the domain
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int lx = 2 * bx + (q & 1), ly = 2 * by + (q >> 1);
        const int gx = gx0 + lx, gy = gy0 + ly;
        const bool edge = (ring0x && ((q & 1) == (bx == 0 ? 0 : 1))) || (ring0y && ((q >> 1) == (by == 0 ? 0 : 1)));
        float4 wk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        pv[q] = 0.0f;
        cb[q] = 0.0f;
        den[q] = 0.0f;
        if (active && (unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
            pv[q] = L.x.at(gx, gy);
            if (owned) fl |= 1u << (16 + q);
            const float lij = L.ls.at(gx, gy);
            bool update = false;
            float dn = 0.0f;
            if (lij < 0.0f) {
                const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
                if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                    cb[q] = P.cdiv * L.b.at(gx, gy);
                    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
                    float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int jx = gx + ox[k], jy = gy + oy[k];
                        if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                            const float level = L.ls.at(jx, jy);
                            if (level < 0.0f) {
                                dn += f[k];
                                wv[k] = f[k];
                            } else {
                                dn += f[k] * (1.0f - level / lij);
                            }
                        }
                    }
                    wk = make_float4(wv[0], wv[1], wv[2], wv[3]);
                    update = !(fabsf(dn) < 1.0e-6f);
                }
            }
            den[q] = update ? dn : 1.0f;
            if (!edge) fl |= (update ? 1u << q : 1u << (4 + q)) | (1u << (8 + q));
        }
        if (active) {
            T.w[q][threadIdx.x] = wk;
            T.p[(q == 0 || q == 3) ? 0 : 1][ly][bx] = pv[q];
        }
    }
    __syncthreads();
    const float wgt = P.weight, omw = 1.0f - P.weight;
    const int t = active ? (int)threadIdx.x : 0;
    const int r0 = 2 * by, r1 = 2 * by + 1;
    const int bxl = bx > 0 ? bx - 1 : 0, bxr = bx < W2 - 1 ? bx + 1 : bx;
    const int rup = r0 > 0 ? r0 - 1 : 0, rdn = r1 < EY - 1 ? r1 + 1 : r1;
    const int bring = min(min(2 * bx + 1, EX - 2 * bx), min(2 * by + 1, EY - 2 * by)) - 1;
    auto sweep_base = [&]() {  // cells 0 and 3; neighbours of the other colour
        float(*Po)[WP] = T.p[1];
        const float pl0 = Po[r0][bxl], pu0 = Po[rup][bx], pr3 = Po[r1][bxr], pd3 = Po[rdn][bx];
        if (fl & 0x100u) {
            pv[0] = gs32_update(cb[0], T.w[0][t], den[0], pv[0], pl0, pv[1], pu0, pv[2], wgt, omw, fl & 1u, fl & 0x10u);
            T.p[0][r0][bx] = pv[0];
        }
        if (fl & 0x800u) {
            pv[3] = gs32_update(cb[3], T.w[3][t], den[3], pv[3], pv[2], pr3, pv[1], pd3, wgt, omw, fl & 8u, fl & 0x80u);
            T.p[0][r1][bx] = pv[3];
        }
    };
    auto sweep_other = [&]() {  // cells 1 and 2; neighbours of the base colour
        float(*Po)[WP] = T.p[0];
        const float pr1 = Po[r0][bxr], pu1 = Po[rup][bx], pl2 = Po[r1][bxl], pd2 = Po[rdn][bx];
        if (fl & 0x200u) {
            pv[1] = gs32_update(cb[1], T.w[1][t], den[1], pv[1], pv[0], pr1, pu1, pv[3], wgt, omw, fl & 2u, fl & 0x20u);
            T.p[1][r0][bx] = pv[1];
        }
        if (fl & 0x400u) {
            pv[2] = gs32_update(cb[2], T.w[2][t], den[2], pv[2], pl2, pv[3], pv[0], pd2, wgt, omw, fl & 4u, fl & 0x40u);
            T.p[1][r1][bx] = pv[2];
        }
    };
    bool ok = true;
    int xch = 0;
    for (int done = 0; done < P.iters && ok;) {
        const int kk = min(KMAX, P.iters - done);
        for (int it = 0; it < kk; ++it) {
            if (bring + 1 >= 1 + 2 * it) {  // a cell of the block lies in the region still needed
                if (base) sweep_base();       // red ((x + y) odd) first
                else sweep_other();
            }
            __syncthreads();
            if (bring + 1 >= 2 + 2 * it) {
                if (base) sweep_other();
                else sweep_base();
            }
            __syncthreads();
        }
        done += kk;
        if (done < P.iters) {  // exchange the halo through L2 (alternating planes)
            const PF& xb = P.xb[xch++ & 1];
            if (owned) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if ((fl >> (16 + q)) & 1u)
                        __stcg(&xb.p[(size_t)(gy0 + 2 * by + (q >> 1)) * xb.P + gx0 + 2 * bx + (q & 1)], pv[q]);
            }
            ok = grid_barrier(P.barrier, nblocks, P.spin_limit);
            if (!ok) break;
            if (active && !owned) {
                float hv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int gx = gx0 + 2 * bx + (q & 1), gy = gy0 + 2 * by + (q >> 1);
                    hv[q] = ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
                                ? __ldcg(&xb.p[(size_t)gy * xb.P + gx])
                                : 0.0f;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) pv[q] = hv[q];
                T.p[0][r0][bx] = pv[0];
                T.p[1][r0][bx] = pv[1];
                T.p[1][r1][bx] = pv[2];
                T.p[0][r1][bx] = pv[3];
            }
            __syncthreads();
        }
    }
    if (ok) ok = grid_barrier(P.barrier, nblocks, P.spin_limit);  // every CTA has read its first image of x
    if (!ok && threadIdx.x == 0) atomicExch(P.err, 2);
    if (ok && owned) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if ((fl >> (16 + q)) & 1u) L.x.at(gx0 + 2 * bx + (q & 1), gy0 + 2 * by + (q >> 1)) = pv[q];
    }
}

// n fixed f32 red-black iterations at level 0 as one cooperative launch, when
// the grid fits one 64 x 32 tile per SM.  EFL_ERR_STATE: it does not (use the
// TMA-streamed sweeps).
inline efl_status solve_gs32_persistent(SolverWorkspace& ws, const Level& L, const PF& xa, const PF& xb,
                                        float dx_scaled, float rho, float dt, float weight, uint32_t n,
                                        int* dev_err, cudaStream_t stream, std::string* err) {
    constexpr int EX = 80, EY = 48, KMAX = 4, NT = 960;
    constexpr int TXo = EX - 4 * KMAX, TYo = EY - 4 * KMAX;
    const int tiles_x = (L.nx + TXo - 1) / TXo, tiles_y = (L.ny + TYo - 1) / TYo;
    if (n == 0) return EFL_OK;
    if (tiles_x * tiles_y > ws.num_sms) return EFL_ERR_STATE;
    const void* kern = (const void*)k_gs32_quad<EX, EY, KMAX, NT>;
    const size_t smem = sizeof(Quad32Tile<EX, EY>);
    static bool attr_done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return EFL_ERR_STATE;
    if (!attr_done[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            cudaGetLastError();
            return EFL_ERR_STATE;
        }
        attr_done[dev] = true;
    }
    Gs32Params P;
    P.L = L;
    P.xb[0] = xa;
    P.xb[1] = xb;
    P.tiles_x = tiles_x;
    P.iters = (int)n;
    P.cdiv = dx_scaled * dx_scaled * rho / dt;  // gauss_seidel.wgsl:58
    P.weight = weight;
    P.barrier = ws.barrier;
    P.spin_limit = ws.spin_limit > 0 ? ws.spin_limit : kBarrierSpinLimit;
    P.err = dev_err;
    if (!dev_err) return EFL_ERR_STATE;
    if (cudaMemsetAsync(ws.barrier, 0, sizeof(GridBarrier), stream) != cudaSuccess) {
        *err = "barrier reset failed";
        return EFL_ERR_CUDA;
    }
    void* args[] = {&P};
    count_launch();
    const cudaError_t e = cudaLaunchCooperativeKernel(kern, dim3(tiles_x * tiles_y), dim3(NT), args, smem, stream);
    if (e != cudaSuccess) {
        *err = std::string("cooperative launch of the fixed-count sweep failed: ") + cudaGetErrorString(e);
        return EFL_ERR_CUDA;
    }
    return EFL_OK;
}

// Global-memory form of the same solve for grids the persistent scheme
// cannot hold (one launch per step of the algorithm).
struct MixPlanes {
    Plane<float4> w;
    PF inv, rc, d;
    Plane<double> den;
    Plane<unsigned char> mode;
};
__global__ void k_mix_coefficients(Level64 L, MixPlanes M) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= L.nx || gy >= L.ny) return;
    unsigned char m = MODE_ZERO;
    double den = 0.0;
    float inv = 0.0f;
    float4 wk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float phi = L.ls.at(gx, gy);
    if (phi < 0.0f) {
        const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
        if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
            m |= MODE_COUNTED;
            const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
            float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int jx = gx + ox[q], jy = gy + oy[q];
                if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                    const float level = L.ls.at(jx, jy);
                    if (level < 0.0f) {
                        den += (double)f[q];
                        wv[q] = f[q];
                    } else {
                        den += (double)f[q] * (1.0 - (double)level / (double)phi);
                    }
                }
            }
            wk = make_float4(wv[0], wv[1], wv[2], wv[3]);
            if (!(fabs(den) < (double)1.0e-6f)) {
                m = (unsigned char)((m & MODE_COUNTED) | MODE_UPDATE);
                inv = (float)(1.0 / den);
            }
        }
    }
    M.mode.at(gx, gy) = m;
    M.den.at(gx, gy) = den;
    M.inv.at(gx, gy) = inv;
    M.w.at(gx, gy) = wk;
}
__global__ void __launch_bounds__(NORM_THREADS) k_mix_residual(Level64 L, MixPlanes M, double cdiv, double factor,
                                                               double2* partials) {
    __shared__ double sr[NORM_THREADS / 32], sb[NORM_THREADS / 32];
    double ar = 0.0, ab = 0.0;
    const int n = L.nx * L.ny;
    for (int i = blockIdx.x * NORM_THREADS + threadIdx.x; i < n; i += gridDim.x * NORM_THREADS) {
        const int y = i / L.nx, x = i - y * L.nx;
        const unsigned char m = M.mode.at(x, y);
        float rcv = 0.0f;
        if (m & MODE_COUNTED) {
            const float4 wk = M.w.at(x, y);
            double sum = (double)wk.x * L.x.ld(x - 1, y);
            sum = sum + (double)wk.y * L.x.ld(x + 1, y);
            sum = sum + (double)wk.z * L.x.ld(x, y - 1);
            sum = sum + (double)wk.w * L.x.ld(x, y + 1);
            const double bb = L.b.at(x, y);
            const double r = bb - factor * (M.den.at(x, y) * L.x.at(x, y) - sum);
            if (m & MODE_UPDATE) rcv = (float)(cdiv * r);
            ar += r * r;
            ab += bb * bb;
        }
        M.rc.at(x, y) = rcv;
        M.d.at(x, y) = 0.0f;
    }
    ar = warp_sum(ar);
    ab = warp_sum(ab);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sr[wid] = ar;
        sb[wid] = ab;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, tb = 0.0;
        for (int k = 0; k < NORM_THREADS / 32; ++k) {
            tr += sr[k];
            tb += sb[k];
        }
        partials[blockIdx.x] = make_double2(tr, tb);
    }
}
__global__ void k_mix_sweep(MixPlanes M, int nx, int ny, float w, int color) {
    const int tx = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = 2 * tx + ((y + color) & 1);
    if (x >= nx || y >= ny) return;
    if (!(M.mode.at(x, y) & MODE_UPDATE)) return;
    const float4 wk = M.w.at(x, y);
    float nume = M.rc.at(x, y);
    nume = nume + wk.x * M.d.ld(x - 1, y);
    nume = nume + wk.y * M.d.ld(x + 1, y);
    nume = nume + wk.z * M.d.ld(x, y - 1);
    nume = nume + wk.w * M.d.ld(x, y + 1);
    M.d.at(x, y) = w * (nume * M.inv.at(x, y)) + (1.0f - w) * M.d.at(x, y);
}
__global__ void k_mix_apply(Level64 L, MixPlanes M) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= L.nx || y >= L.ny) return;
    double& pv = L.x.at(x, y);
    pv = (M.mode.at(x, y) & MODE_UPDATE) ? pv + (double)M.d.at(x, y) : 0.0;
}

// ---------------------------------------------------------------------------
// Fixed-count f32 sweeps (the reference's mode) as tiled, temporally blocked
// launches: each CTA loads its tile plus a halo of 2K cells, builds the
// per-cell coefficients of gauss_seidel.wgsl:44-80 in the reference's f32
// operation order (c*div, denom, neighbour weights), runs K red-black
// iterations from shared memory and writes its owned cells to the other
// buffer of a ping-pong pair.  Bit-identical to K global red/black sweeps.
template <int EX, int EY>
struct GsTile32 {
    static constexpr int W2 = EX / 2;
    static constexpr int N2 = W2 * EY;
    float p[2][N2];
    float cb[2][N2];
    float den[2][N2];
    float4 w[2][N2];
    unsigned char mode[2][N2];
};
constexpr int GT_THREADS = 256;

template <int EX, int EY, int K>
__global__ void __launch_bounds__(GT_THREADS) k_gs32_tile(Level L, PF out, float dx_scaled, float rho, float dt,
                                                          float weight, int tiles_x, int iters) {
    extern __shared__ __align__(16) unsigned char gt_raw[];
    GsTile32<EX, EY>& T = *reinterpret_cast<GsTile32<EX, EY>*>(gt_raw);
    constexpr int H = 2 * K, W2 = EX / 2, TX = EX - 2 * H, TY = EY - 2 * H;
    const int gx0 = (blockIdx.x % tiles_x) * TX - H, gy0 = (blockIdx.x / tiles_x) * TY - H;
    const int base = (gx0 + gy0) & 1;
    const float cdiv = dx_scaled * dx_scaled * rho / dt;  // gauss_seidel.wgsl:58
    for (int i = threadIdx.x; i < EX * EY; i += GT_THREADS) {
        const int ly = i / EX, lx = i - ly * EX;
        const int gx = gx0 + lx, gy = gy0 + ly;
        const int c = (base + lx + ly) & 1, k = ly * W2 + (lx >> 1);
        unsigned char m = MODE_SKIP;
        float den = 0.0f, cb = 0.0f, pv = 0.0f;
        float4 wk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny) {
            pv = L.x.at(gx, gy);
            const float lij = L.ls.at(gx, gy);
            bool update = false;
            if (lij < 0.0f) {
                const float f[4] = {L.fu.at(gx, gy), L.fu.at(gx + 1, gy), L.fv.at(gx, gy), L.fv.at(gx, gy + 1)};
                if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                    cb = cdiv * L.b.at(gx, gy);
                    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
                    float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int jx = gx + ox[q], jy = gy + oy[q];
                        if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                            const float level = L.ls.at(jx, jy);
                            if (level < 0.0f) {
                                den += f[q];
                                wv[q] = f[q];
                            } else {
                                den += f[q] * (1.0f - level / lij);
                            }
                        }
                    }
                    wk = make_float4(wv[0], wv[1], wv[2], wv[3]);
                    update = !(fabsf(den) < 1.0e-6f);
                }
            }
            const bool ring = lx == 0 || ly == 0 || lx == EX - 1 || ly == EY - 1;
            if (!ring) m = update ? MODE_UPDATE : MODE_ZERO;
        }
        T.p[c][k] = pv;
        T.cb[c][k] = cb;
        T.den[c][k] = den;
        T.w[c][k] = wk;
        T.mode[c][k] = m;
    }
    __syncthreads();
    const float omw = 1.0f - weight;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int c = half == 0 ? 1 : 0, o = 1 - c;  // red ((x+y) odd) first
            constexpr int TOTAL = (EY - 2) * W2;
            for (int i = threadIdx.x; i < TOTAL; i += GT_THREADS) {
                const int ly = 1 + i / W2;
                const int k = ly * W2 + (i - (ly - 1) * W2);
                const unsigned char m = T.mode[c][k];
                if (m & MODE_UPDATE) {
                    const int odd = (base + ly + c) & 1;
                    const float4 wk = T.w[c][k];
                    float nume = T.cb[c][k];
                    nume = nume + wk.x * T.p[o][k - 1 + odd];
                    nume = nume + wk.y * T.p[o][k + odd];
                    nume = nume + wk.z * T.p[o][k - W2];
                    nume = nume + wk.w * T.p[o][k + W2];
                    const float pn = nume / T.den[c][k];
                    T.p[c][k] = weight * pn + omw * T.p[c][k];
                } else if (m & MODE_ZERO) {
                    T.p[c][k] = 0.0f;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < TX * TY; i += GT_THREADS) {
        const int ly = H + i / TX, lx = H + i % TX;
        const int gx = gx0 + lx, gy = gy0 + ly;
        if ((unsigned)gx < (unsigned)L.nx && (unsigned)gy < (unsigned)L.ny)
            out.at(gx, gy) = T.p[(base + lx + ly) & 1][ly * W2 + (lx >> 1)];
    }
}

// n fixed f32 red-black iterations on level L, ping-ponging between L.x and
// `alt` (same extent and pitch); the result ends in L.x.
inline efl_status solve_gs32_tiled(const Level& L, const PF& alt, float dx_scaled, float rho, float dt, float weight,
                                   uint32_t n, cudaStream_t stream) {
    constexpr int K = 2, EX = 64 + 4 * K, EY = 32 + 4 * K;  // 64 x 32 owned, two CTAs per SM
    constexpr int TX = EX - 4 * K, TY = EY - 4 * K;
    const size_t smem = sizeof(GsTile32<EX, EY>);
    int dev = 0;
    cudaGetDevice(&dev);
    static bool attr_done[64] = {};
    if (dev < 0 || dev >= 64) return EFL_ERR_CUDA;
    if (!attr_done[dev]) {
        if (cudaFuncSetAttribute(k_gs32_tile<EX, EY, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return EFL_ERR_CUDA;
        attr_done[dev] = true;
    }
    const int tiles_x = (L.nx + TX - 1) / TX, tiles_y = (L.ny + TY - 1) / TY;
    Level cur = L;
    PF dst = alt;
    uint32_t launches = 0;
    for (uint32_t done = 0; done < n;) {
        const int k = (int)std::min<uint32_t>(K, n - done);
        k_gs32_tile<EX, EY, K><<<tiles_x * tiles_y, GT_THREADS, smem + count_launch(), stream>>>(
            cur, dst, dx_scaled, rho, dt, weight, tiles_x, k);
        PF prev = cur.x;
        cur.x = dst;
        dst = prev;
        done += (uint32_t)k;
        ++launches;
    }
    if (launches & 1) {  // result is in alt: copy back
        if (cudaMemcpy2DAsync(L.x.p, (size_t)L.x.P * 4, alt.p, (size_t)alt.P * 4, (size_t)L.nx * 4, L.ny,
                              cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
            return EFL_ERR_CUDA;
    }
    return EFL_OK;
}

struct PersistentPlan {
    int tx = 0, ty = 0, kmax = 0, tiles_x = 0, tiles_y = 0;
    int threads = PS_THREADS;
    size_t smem = 0;
    const void* kernel = nullptr;
    bool ok = false;
};

// One CTA of `threads` threads with `smem` bytes of dynamic shared memory resident per SM (registers and shared
// memory both; sets the kernel's shared-memory limit), checked once per kernel and device.
template <const void* (*KernelOf)()>
inline bool plan_resident(int threads, size_t smem) {
    int dev = 0;
    cudaGetDevice(&dev);
    static signed char state[64] = {};  // 0 unknown, 1 resident, -1 not
    if (dev < 0 || dev >= 64) return false;
    if (!state[dev]) {
        const void* k = KernelOf();
        int per_sm = 0;
        const bool ok = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
                        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) == cudaSuccess &&
                        per_sm >= 1;
        cudaGetLastError();
        state[dev] = ok ? 1 : -1;
    }
    return state[dev] == 1;
}
template <int EX, int EY, int KMAX, int NT, int ROWS>
inline const void* oct_kernel() { return (const void*)k_gsmix_oct<EX, EY, KMAX, NT, ROWS>; }
template <int EX, int EY, int KMAX, int NT>
inline const void* quad_kernel() { return (const void*)k_gsmix_quad<EX, EY, KMAX, NT>; }

// Plans for the mixed persistent solve (MixTile: 53 bytes per cell).
template <int EX, int EY, int KMAX>
inline bool try_plan_mix(const SolverWorkspace& ws, int nx, int ny, PersistentPlan* p) {
    const int tx = EX - 4 * KMAX, ty = EY - 4 * KMAX;
    p->kmax = KMAX;
    p->tx = tx;
    p->ty = ty;
    p->tiles_x = (nx + tx - 1) / tx;
    p->tiles_y = (ny + ty - 1) / ty;
    p->smem = sizeof(MixTile<EX, EY>);
    p->kernel = (const void*)k_gsmix_persistent<EX, EY, KMAX>;
    if (p->smem + 1024 > ws.max_smem) return false;
    if (p->tiles_x * p->tiles_y > ws.num_sms || p->tiles_x * p->tiles_y > ws.max_blocks) return false;
    return true;
}
// Plans for the register-resident form (QuadTile: 44 bytes of shared memory per cell).
template <int EX, int EY, int KMAX, int NT>
inline bool try_plan_quad(const SolverWorkspace& ws, int nx, int ny, PersistentPlan* p) {
    const int tx = EX - 4 * KMAX, ty = EY - 4 * KMAX;
    p->kmax = KMAX;
    p->tx = tx;
    p->ty = ty;
    p->tiles_x = (nx + tx - 1) / tx;
    p->tiles_y = (ny + ty - 1) / ty;
    p->smem = sizeof(QuadTile<EX, EY>);
    p->kernel = (const void*)k_gsmix_quad<EX, EY, KMAX, NT>;
    p->threads = NT;
    if (p->smem + 2048 > ws.max_smem) return false;
    if (p->tiles_x * p->tiles_y > ws.num_sms || p->tiles_x * p->tiles_y > ws.max_blocks) return false;
    return plan_resident<quad_kernel<EX, EY, KMAX, NT>>(NT, p->smem);
}
// Plans for the paired-lane form (OctTile: 26 bytes of shared memory per cell).
template <int EX, int EY, int KMAX, int NT, int ROWS>
inline bool try_plan_oct(const SolverWorkspace& ws, int nx, int ny, PersistentPlan* p) {
    const int tx = EX - 4 * KMAX, ty = EY - 4 * KMAX;
    p->kmax = KMAX;
    p->tx = tx;
    p->ty = ty;
    p->tiles_x = (nx + tx - 1) / tx;
    p->tiles_y = (ny + ty - 1) / ty;
    p->smem = sizeof(OctTile<EX, EY, ROWS>);
    p->kernel = (const void*)k_gsmix_oct<EX, EY, KMAX, NT, ROWS>;
    p->threads = NT;
    if (p->smem + 2048 > ws.max_smem) return false;
    if (p->tiles_x * p->tiles_y > ws.num_sms || p->tiles_x * p->tiles_y > ws.max_blocks) return false;
    return plan_resident<oct_kernel<EX, EY, KMAX, NT, ROWS>>(NT, p->smem);
}
inline PersistentPlan plan_mix(const SolverWorkspace& ws, int nx, int ny) {
    PersistentPlan p;
    if (ws.use_reg && (try_plan_oct<96, 64, 8, 384, 4>(ws, nx, ny, &p) ||   // 64 x 32 owned, 8 iterations
                       try_plan_oct<80, 48, 4, 480, 2>(ws, nx, ny, &p) ||   // 64 x 32
                       try_plan_oct<48, 48, 4, 288, 2>(ws, nx, ny, &p) ||   // 32 x 32
                       try_plan_oct<72, 56, 2, 512, 2>(ws, nx, ny, &p) ||   // 64 x 48
                       try_plan_oct<40, 40, 4, 224, 2>(ws, nx, ny, &p))) {  // 24 x 24
        p.ok = true;
        return p;
    }
    if (ws.use_reg && (try_plan_quad<80, 48, 4, 960>(ws, nx, ny, &p) ||  // 64 x 32 owned
                       try_plan_quad<48, 48, 4, 576>(ws, nx, ny, &p) ||  // 32 x 32
                       try_plan_quad<72, 56, 2, 1024>(ws, nx, ny, &p) ||  // 64 x 48
                       try_plan_quad<40, 40, 4, 416>(ws, nx, ny, &p))) {  // 24 x 24
        p.ok = true;
        return p;
    }
    if (try_plan_mix<80, 48, 4>(ws, nx, ny, &p) ||  // 64 x 32 owned
        try_plan_mix<48, 48, 4>(ws, nx, ny, &p) ||  // 32 x 32
        try_plan_mix<72, 56, 2>(ws, nx, ny, &p) ||  // 64 x 48
        try_plan_mix<40, 40, 4>(ws, nx, ny, &p)) {  // 24 x 24
        p.ok = true;
        return p;
    }
    return PersistentPlan{};
}

// Tolerance-driven solve, one cooperative launch.  dbuf: an f32 plane of the
// level's extent for the correction's halo exchange.  EFL_ERR_STATE: the grid
// does not fit the persistent scheme.
inline efl_status solve_gsmix_persistent(SolverWorkspace& ws, const Level64& L, const PF& dbuf, const PF& dbuf2,
                                         const Uniform& U,
                                         float weight, double tol, uint32_t max_iters, uint32_t check_interval,
                                         cudaStream_t stream, SolveResult* out, std::string* err) {
    PersistentPlan plan = plan_mix(ws, L.nx, L.ny);
    if (!plan.ok) return EFL_ERR_STATE;
    if (cudaFuncSetAttribute(plan.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan.smem) !=
        cudaSuccess) {
        cudaGetLastError();
        return EFL_ERR_STATE;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plan.kernel, plan.threads, plan.smem) != cudaSuccess ||
        per_sm < 1 || plan.tiles_x * plan.tiles_y > per_sm * ws.num_sms) {
        cudaGetLastError();
        return EFL_ERR_STATE;
    }
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
    P.spin_limit = ws.spin_limit > 0 ? ws.spin_limit : kBarrierSpinLimit;
    P.dbuf2 = dbuf2;
    P.one = 1.0f;
    if (cudaMemsetAsync(ws.barrier, 0, sizeof(GridBarrier), stream) != cudaSuccess) {
        *err = "barrier reset failed";
        return EFL_ERR_CUDA;
    }
    PF db = dbuf;
    void* args[] = {&P, &db};
    count_launch();
    cudaError_t e = cudaLaunchCooperativeKernel(plan.kernel, dim3(plan.tiles_x * plan.tiles_y), dim3(plan.threads),
                                                args, plan.smem, stream);
    if (e != cudaSuccess) {
        *err = std::string("cooperative launch of the mixed solver failed: ") + cudaGetErrorString(e);
        return EFL_ERR_CUDA;
    }
    if (cudaMemcpyAsync(ws.h_result, ws.result, sizeof(SolveResult), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
        *err = std::string("mixed solver failed: ") + cudaGetErrorString(cudaGetLastError());
        return EFL_ERR_CUDA;
    }
    *out = *ws.h_result;
    if (out->error) {
        *err = "mixed solver: a grid barrier timed out";
        return EFL_ERR_CUDA;
    }
    return EFL_OK;
}

// The same solve with global-memory kernels and a host loop (grids beyond the
// persistent scheme).  M must hold planes of the level's extent.
inline efl_status solve_gsmix_global(SolverWorkspace& ws, const Level64& L, const MixPlanes& M, const Uniform& U,
                                     float weight, double tol, uint32_t max_iters, uint32_t check_interval,
                                     cudaStream_t stream, SolveResult* out, std::string* err) {
    const dim3 b(32, 8);
    const dim3 g((L.nx + 31) / 32, (L.ny + 7) / 8);
    const dim3 gh(((L.nx + 1) / 2 + 31) / 32, (L.ny + 7) / 8);
    const double dx = (double)U.dx;
    const double cdiv = dx * dx * (double)U.rho / (double)U.dt;
    const double factor = (double)U.dt / (double)U.rho / dx / dx;
    const int nblocks = std::min(ws.max_blocks, std::max(1, (L.nx * L.ny + NORM_THREADS - 1) / NORM_THREADS));
    k_mix_coefficients<<<g, b, count_launch(), stream>>>(L, M);
    auto residual = [&](double* rel) -> efl_status {
        k_mix_residual<<<nblocks, NORM_THREADS, count_launch(), stream>>>(L, M, cdiv, factor, ws.partials);
        std::vector<double2> h(nblocks);
        if (cudaMemcpyAsync(h.data(), ws.partials, nblocks * sizeof(double2), cudaMemcpyDeviceToHost, stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            *err = std::string("mixed solver (global): ") + cudaGetErrorString(cudaGetLastError());
            return EFL_ERR_CUDA;
        }
        double r = 0.0, bb = 0.0;
        for (int i = 0; i < nblocks; ++i) {
            r += h[i].x;
            bb += h[i].y;
        }
        *rel = bb > 0.0 ? std::sqrt(r) / std::sqrt(bb) : (r > 0.0 ? INFINITY : 0.0);
        return EFL_OK;
    };
    double rel;
    efl_status st = residual(&rel);
    if (st != EFL_OK) return st;
    out->r0 = rel;
    uint32_t iters = 0;
    const uint32_t chk = std::max<uint32_t>(1, check_interval);
    while (!(rel <= tol) && iters < max_iters) {
        const uint32_t n = std::min(chk, max_iters - iters);
        for (uint32_t it = 0; it < n; ++it) {
            k_mix_sweep<<<gh, b, count_launch(), stream>>>(M, L.nx, L.ny, weight, 1);
            k_mix_sweep<<<gh, b, count_launch(), stream>>>(M, L.nx, L.ny, weight, 0);
        }
        k_mix_apply<<<g, b, count_launch(), stream>>>(L, M);
        iters += n;
        st = residual(&rel);
        if (st != EFL_OK) return st;
    }
    out->iterations = iters;
    out->r1 = rel;
    out->converged = rel <= tol ? 1 : 0;
    out->error = 0;
    return EFL_OK;
}

}  // namespace efl
