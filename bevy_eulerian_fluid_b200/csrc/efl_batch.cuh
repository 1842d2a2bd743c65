// efl_batch.cuh — the tolerance-driven pressure solves of many independent
// simulations (uneven grid sizes) in ONE cooperative launch.
//
// Work is a packed list of (simulation, 64 x 32 tile) items.  Every
// simulation runs the same mixed-precision iterative refinement as its
// single-simulation solve (FP64 residual and iterate, f32 red-black sweeps on
// the correction), so each one's iterates, iteration count and result are
// exactly those it would have alone.  The simulations advance in lockstep by
// rounds of K red-black iterations: a round streams each active tile plus a
// 2K-cell halo of the correction and its f32 coefficients from global
// memory into shared memory, runs K iterations there and writes the owned
// cells to the other buffer of a ping-pong pair.  Every check_interval
// iterations the kernel applies p += d, forms each tile's FP64 residual
// partials, reduces them per simulation in tile order, and retires the
// simulations that converged or reached max_iterations; their tiles are
// skipped from then on.  Grid barriers are bounded (see grid_barrier).
#pragma once

#include "efl_kernels.cuh"
#include "efl_solver.cuh"

namespace efl {

struct BatchSim {
    Level64 L;    // level 0: x = FP64 iterate, b = widened divergence, ls / fu / fv
    MixPlanes M;  // per-cell f32 coefficients, rc, FP64 denom, mode
    PF d[2];      // correction ping-pong
    double cdiv, factor;
    float weight;
    int tiles_x, tile_start, tile_count;
};
struct BatchState {
    unsigned iterations;
    int active;
    int converged;
    int pad;
    double r0, r1;
};
struct BatchParams {
    const BatchSim* sims;
    int nsims;
    int ntiles;
    const int2* tiles;  // (simulation, tile index within the simulation)
    double tol;
    unsigned max_iters, check_interval;
    double2* partials;  // one per tile
    BatchState* state;  // one per simulation
    GridBarrier* barrier;
};

template <int EX, int EY>
struct BatchTile {
    static constexpr int W2 = EX / 2;
    static constexpr int N2 = W2 * EY;
    float4 w[2][N2];
    float d[2][N2];
    float rc[2][N2];
    float inv[2][N2];
    unsigned char mode[2][N2];
};
constexpr int BT_THREADS = 512;

EFL_DEV void bt_tile_origin(const BatchSim& S, int lt, int tx, int ty, int* x0, int* y0) {
    *x0 = (lt % S.tiles_x) * tx;
    *y0 = (lt / S.tiles_x) * ty;
}

template <int TX, int TY, int K>
__global__ void __launch_bounds__(BT_THREADS, 2) k_batch_mix(BatchParams P) {
    constexpr int H = 2 * K, EX = TX + 2 * H, EY = TY + 2 * H, W2 = EX / 2;
    extern __shared__ __align__(16) unsigned char bt_raw[];
    BatchTile<EX, EY>& T = *reinterpret_cast<BatchTile<EX, EY>*>(bt_raw);
    const unsigned nb = gridDim.x;
    __shared__ int s_any;

    // Per-cell coefficients of every simulation (owned cells of each tile).
    for (int t = blockIdx.x; t < P.ntiles; t += nb) {
        const int2 it = P.tiles[t];
        const BatchSim& S = P.sims[it.x];
        int x0, y0;
        bt_tile_origin(S, it.y, TX, TY, &x0, &y0);
        const Level64& L = S.L;
        for (int i = threadIdx.x; i < TX * TY; i += BT_THREADS) {
            const int gx = x0 + i % TX, gy = y0 + i / TX;
            if (gx >= L.nx || gy >= L.ny) continue;
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
            S.M.mode.at(gx, gy) = m;
            S.M.den.at(gx, gy) = den;
            S.M.inv.at(gx, gy) = inv;
            S.M.w.at(gx, gy) = wk;
        }
    }
    bool ok = grid_barrier(P.barrier, nb);
    int cur = 0;
    unsigned iters = 0;
    bool first = true;
    while (ok) {
        // ---- check: p += d (not before the first), residual partials, per-simulation reduction
        if (!first) {
            for (int t = blockIdx.x; t < P.ntiles; t += nb) {
                const int2 it = P.tiles[t];
                if (!__ldcg(&P.state[it.x].active)) continue;
                const BatchSim& S = P.sims[it.x];
                int x0, y0;
                bt_tile_origin(S, it.y, TX, TY, &x0, &y0);
                for (int i = threadIdx.x; i < TX * TY; i += BT_THREADS) {
                    const int gx = x0 + i % TX, gy = y0 + i / TX;
                    if (gx >= S.L.nx || gy >= S.L.ny) continue;
                    double& pv = S.L.x.at(gx, gy);
                    pv = (S.M.mode.at(gx, gy) & MODE_UPDATE) ? pv + (double)__ldcg(&S.d[cur].at(gx, gy)) : 0.0;
                }
            }
            ok = grid_barrier(P.barrier, nb);
            if (!ok) break;
        }
        for (int t = blockIdx.x; t < P.ntiles; t += nb) {
            const int2 it = P.tiles[t];
            if (!__ldcg(&P.state[it.x].active)) continue;
            const BatchSim& S = P.sims[it.x];
            const Level64& L = S.L;
            int x0, y0;
            bt_tile_origin(S, it.y, TX, TY, &x0, &y0);
            double ar = 0.0, ab = 0.0;
            for (int i = threadIdx.x; i < TX * TY; i += BT_THREADS) {
                const int gx = x0 + i % TX, gy = y0 + i / TX;
                if (gx >= L.nx || gy >= L.ny) continue;
                const unsigned char m = S.M.mode.at(gx, gy);
                float rcv = 0.0f;
                if (m & MODE_COUNTED) {
                    const float4 wk = S.M.w.at(gx, gy);
                    double sum = (double)wk.x * (gx > 0 ? __ldcg(&L.x.p[(size_t)gy * L.x.P + gx - 1]) : 0.0);
                    sum = sum + (double)wk.y * (gx + 1 < L.nx ? __ldcg(&L.x.p[(size_t)gy * L.x.P + gx + 1]) : 0.0);
                    sum = sum + (double)wk.z * (gy > 0 ? __ldcg(&L.x.p[(size_t)(gy - 1) * L.x.P + gx]) : 0.0);
                    sum = sum + (double)wk.w * (gy + 1 < L.ny ? __ldcg(&L.x.p[(size_t)(gy + 1) * L.x.P + gx]) : 0.0);
                    const double bb = L.b.at(gx, gy);
                    const double r =
                        bb - S.factor * (S.M.den.at(gx, gy) * __ldcg(&L.x.p[(size_t)gy * L.x.P + gx]) - sum);
                    if (m & MODE_UPDATE) rcv = (float)(S.cdiv * r);
                    ar += r * r;
                    ab += bb * bb;
                }
                S.M.rc.at(gx, gy) = rcv;
                S.d[cur].at(gx, gy) = 0.0f;
            }
            ar = warp_sum(ar);
            ab = warp_sum(ab);
            __shared__ double red_r[BT_THREADS / 32], red_b[BT_THREADS / 32];
            if ((threadIdx.x & 31) == 0) {
                red_r[threadIdx.x >> 5] = ar;
                red_b[threadIdx.x >> 5] = ab;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                double tr = 0.0, tb = 0.0;
                for (int q = 0; q < BT_THREADS / 32; ++q) {
                    tr += red_r[q];
                    tb += red_b[q];
                }
                P.partials[t] = make_double2(tr, tb);
            }
            __syncthreads();
        }
        ok = grid_barrier(P.barrier, nb);
        if (!ok) break;
        if (blockIdx.x == 0) {
            for (int s = threadIdx.x; s < P.nsims; s += BT_THREADS) {
                BatchState& st = P.state[s];
                if (!st.active) continue;
                const BatchSim& S = P.sims[s];
                double r = 0.0, b = 0.0;
                for (int t = S.tile_start; t < S.tile_start + S.tile_count; ++t) {
                    const double2 v = __ldcg(&P.partials[t]);
                    r += v.x;
                    b += v.y;
                }
                const double rel = b > 0.0 ? sqrt(r) / sqrt(b) : (r > 0.0 ? __longlong_as_double(0x7ff0000000000000ll) : 0.0);
                if (first) st.r0 = rel;
                st.r1 = rel;
                st.iterations = iters;
                st.converged = rel <= P.tol ? 1 : 0;
                if (st.converged || iters >= P.max_iters) st.active = 0;
            }
        }
        ok = grid_barrier(P.barrier, nb);
        if (!ok) break;
        if (threadIdx.x == 0) {
            int any = 0;
            for (int s = 0; s < P.nsims && !any; ++s) any = __ldcg(&P.state[s].active);
            s_any = any;
        }
        __syncthreads();
        if (!s_any) break;
        first = false;
        // ---- rounds of up to K red-black iterations until the next check
        unsigned todo = min(P.check_interval, P.max_iters - iters);
        while (ok && todo > 0) {
            const int kk = (int)min((unsigned)K, todo);
            for (int t = blockIdx.x; t < P.ntiles; t += nb) {
                const int2 it = P.tiles[t];
                if (!__ldcg(&P.state[it.x].active)) continue;
                const BatchSim& S = P.sims[it.x];
                const int nx = S.L.nx, ny = S.L.ny;
                int x0, y0;
                bt_tile_origin(S, it.y, TX, TY, &x0, &y0);
                const int gx0 = x0 - H, gy0 = y0 - H, base = (gx0 + gy0) & 1;
                for (int i = threadIdx.x; i < EX * EY; i += BT_THREADS) {
                    const int ly = i / EX, lx = i - ly * EX;
                    const int gx = gx0 + lx, gy = gy0 + ly;
                    const int c = (base + lx + ly) & 1, k = ly * W2 + (lx >> 1);
                    unsigned char m = MODE_SKIP;
                    float dv = 0.0f, rcv = 0.0f, iv = 0.0f;
                    float4 wk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if ((unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny) {
                        const bool ring = lx == 0 || ly == 0 || lx == EX - 1 || ly == EY - 1;
                        m = ring ? MODE_SKIP : (unsigned char)(S.M.mode.at(gx, gy) & MODE_UPDATE);
                        dv = __ldcg(&S.d[cur].at(gx, gy));
                        if (m) {
                            rcv = __ldcg(&S.M.rc.at(gx, gy));
                            iv = S.M.inv.at(gx, gy);
                            wk = S.M.w.at(gx, gy);
                        }
                    }
                    T.mode[c][k] = m;
                    T.d[c][k] = dv;
                    T.rc[c][k] = rcv;
                    T.inv[c][k] = iv;
                    T.w[c][k] = wk;
                }
                __syncthreads();
                const float w = S.weight, omw = 1.0f - S.weight;
                for (int q = 0; q < kk; ++q) {
#pragma unroll
                    for (int half = 0; half < 2; ++half) {
                        const int c = half == 0 ? 1 : 0, o = 1 - c, h = 2 * q + half;  // red ((x+y) odd) first
                        const int total = (EY - 2 - 2 * h) * W2;
                        for (int i = threadIdx.x; i < total; i += BT_THREADS) {
                            const int ly = 1 + h + i / W2;
                            const int j = i - (ly - 1 - h) * W2;
                            const int odd = (base + ly + c) & 1;
                            const int lx = 2 * j + odd;
                            if (lx < 1 + h || lx > EX - 2 - h) continue;
                            const int k = ly * W2 + j;
                            if (T.mode[c][k] & MODE_UPDATE) {
                                const float4 wk = T.w[c][k];
                                float nume = T.rc[c][k];
                                nume = nume + wk.x * T.d[o][k - 1 + odd];
                                nume = nume + wk.y * T.d[o][k + odd];
                                nume = nume + wk.z * T.d[o][k - W2];
                                nume = nume + wk.w * T.d[o][k + W2];
                                T.d[c][k] = w * (nume * T.inv[c][k]) + omw * T.d[c][k];
                            }
                        }
                        __syncthreads();
                    }
                }
                for (int i = threadIdx.x; i < TX * TY; i += BT_THREADS) {
                    const int ly = H + i / TX, lx = H + i % TX;
                    const int gx = gx0 + lx, gy = gy0 + ly;
                    if (gx < nx && gy < ny) __stcg(&S.d[cur ^ 1].at(gx, gy), T.d[(base + lx + ly) & 1][ly * W2 + (lx >> 1)]);
                }
                __syncthreads();
            }
            ok = grid_barrier(P.barrier, nb);
            cur ^= 1;
            todo -= (unsigned)kk;
        }
        iters += min(P.check_interval, P.max_iters - iters);
    }
}

}  // namespace efl
