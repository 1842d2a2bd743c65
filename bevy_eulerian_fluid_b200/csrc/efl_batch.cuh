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
    int* n_active;      // simulations still iterating after the last check
    int2* work;         // (simulation, tile) of the rounds until the next check; ntiles entries
    int* work_count;
    BatchState* state;  // one per simulation
    GridBarrier* barrier;
    long long spin_limit;  // grid-barrier polls before giving up
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

// A cell whose four neighbours are fluid with full faces (MODE_STD): w = (1, 1,
// 1, 1), den = 4, inv = 0.25f, so none of its coefficients is read from memory.
// Per-tile flags of the owned region.
constexpr int TILE_UPDATE = 1, TILE_COUNTED = 2;

// Tiles one CTA owns (tile t belongs to CTA t % gridDim.x); the host checks
// ntiles <= BT_MAX_OWN * gridDim.x.
constexpr int BT_MAX_OWN = 128;

// Compacts the CTA's own tiles that satisfy `pred(j)` into list[0..*n).
template <class Pred>
EFL_DEV void bt_compact(int nown, int* list, int* n, int* warp_cnt, Pred pred) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int NW = BT_MAX_OWN / 32;
    bool pj = false;
    unsigned bal = 0;
    if (wid < NW) {
        pj = tid < nown && pred(tid);
        bal = __ballot_sync(0xffffffffu, pj);
        if (lane == 0) warp_cnt[wid] = __popc(bal);
    }
    __syncthreads();
    if (wid < NW) {
        int off = 0;
        for (int q = 0; q < wid; ++q) off += warp_cnt[q];
        if (pj) list[off + __popc(bal & ((1u << lane) - 1u))] = tid;
        if (tid == 0) {
            int tot = 0;
            for (int q = 0; q < NW; ++q) tot += warp_cnt[q];
            *n = tot;
        }
    }
    __syncthreads();
}

template <int TX, int TY, int K>
__global__ void __launch_bounds__(BT_THREADS, 2) k_batch_mix(BatchParams P) {
    constexpr int H = 2 * K, EX = TX + 2 * H, EY = TY + 2 * H, W2 = EX / 2;
    constexpr int NO = (TX * TY + BT_THREADS - 1) / BT_THREADS;  // owned cells per thread
    constexpr unsigned char MODE_OUT = 0xFF;                     // outside the grid or the tile
    extern __shared__ __align__(16) unsigned char bt_raw[];
    BatchTile<EX, EY>& T = *reinterpret_cast<BatchTile<EX, EY>*>(bt_raw);
    const int nb = (int)gridDim.x;
    __shared__ int s_sim[BT_MAX_OWN];             // simulation of own tile j (tile blockIdx.x + j * nb)
    __shared__ unsigned char s_flags[BT_MAX_OWN];  // TILE_UPDATE | TILE_COUNTED
    __shared__ unsigned char s_act[BT_MAX_OWN];    // its simulation is still iterating
    __shared__ int s_list[BT_MAX_OWN];
    __shared__ int s_nlist, s_cnt, s_any;
    __shared__ int s_wcnt[BT_MAX_OWN / 32];
    __shared__ double red_r[BT_THREADS / 32], red_b[BT_THREADS / 32];
    const int nown = (int)blockIdx.x < P.ntiles ? (P.ntiles - (int)blockIdx.x + nb - 1) / nb : 0;

    // Per-cell coefficients of every simulation (owned cells of each tile)
    // and the tile's flags.
    for (int j = 0; j < nown; ++j) {
        const int t = (int)blockIdx.x + j * nb;
        const int2 it = P.tiles[t];
        const BatchSim& S = P.sims[it.x];
        int x0, y0;
        bt_tile_origin(S, it.y, TX, TY, &x0, &y0);
        const Level64& L = S.L;
        int flags = 0;
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
                        if (wv[0] == 1.0f && wv[1] == 1.0f && wv[2] == 1.0f && wv[3] == 1.0f) m |= MODE_STD;
                    }
                }
            }
            flags |= (m & MODE_UPDATE) ? TILE_UPDATE : 0;
            flags |= (m & MODE_COUNTED) ? TILE_COUNTED : 0;
            S.M.mode.at(gx, gy) = m;
            if (m & MODE_COUNTED) {
                S.M.den.at(gx, gy) = den;
                S.M.inv.at(gx, gy) = inv;
                S.M.w.at(gx, gy) = wk;
            }
        }
        flags = __syncthreads_or(flags & TILE_UPDATE) * TILE_UPDATE | __syncthreads_or(flags & TILE_COUNTED) * TILE_COUNTED;
        if (threadIdx.x == 0) {
            s_sim[j] = it.x;
            s_flags[j] = (unsigned char)flags;
            s_act[j] = 1;  // every simulation starts active
        }
    }
    __syncthreads();
    bool ok = grid_barrier(P.barrier, nb, P.spin_limit);
    int cur = 0;
    unsigned iters = 0;
    bool first = true, first_apply = true;
    while (ok) {
        // ---- check: p += d (not before the first), residual partials, per-simulation reduction
        if (!first) {
            // The first apply zeroes p on every non-update cell; after it only
            // tiles with update cells change.
            const bool fa = first_apply;
            bt_compact(nown, s_list, &s_nlist, s_wcnt,
                       [&](int j) { return s_act[j] && (fa || (s_flags[j] & TILE_UPDATE)); });
            for (int q = 0; q < s_nlist; ++q) {
                const int j = s_list[q];
                const BatchSim& S = P.sims[s_sim[j]];
                const int t = (int)blockIdx.x + j * nb;
                int x0, y0;
                bt_tile_origin(S, t - S.tile_start, TX, TY, &x0, &y0);
                unsigned char mo[NO];
#pragma unroll
                for (int jj = 0; jj < NO; ++jj) {
                    const int i = threadIdx.x + jj * BT_THREADS;
                    const int gx = x0 + i % TX, gy = y0 + i / TX;
                    mo[jj] = (i < TX * TY && gx < S.L.nx && gy < S.L.ny) ? S.M.mode.at(gx, gy) : MODE_OUT;
                }
#pragma unroll
                for (int jj = 0; jj < NO; ++jj) {
                    const int i = threadIdx.x + jj * BT_THREADS;
                    const int gx = x0 + i % TX, gy = y0 + i / TX;
                    if (mo[jj] == MODE_OUT) continue;
                    double& pv = S.L.x.at(gx, gy);
                    if (mo[jj] & MODE_UPDATE) pv = pv + (double)__ldcg(&S.d[cur].at(gx, gy));
                    else if (fa) pv = 0.0;  // non-update cells stay 0 afterwards
                }
            }
            first_apply = false;
            ok = grid_barrier(P.barrier, nb, P.spin_limit);
            if (!ok) break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) *P.work_count = 0;  // nobody reads it in this phase
        bt_compact(nown, s_list, &s_nlist, s_wcnt, [&](int j) { return s_act[j] != 0; });
        for (int q = 0; q < s_nlist; ++q) {
            const int j = s_list[q];
            const int t = (int)blockIdx.x + j * nb;
            if (!(s_flags[j] & TILE_COUNTED)) {
                if (threadIdx.x == 0) P.partials[t] = make_double2(0.0, 0.0);
                continue;
            }
            const BatchSim& S = P.sims[s_sim[j]];
            const Level64& L = S.L;
            int x0, y0;
            bt_tile_origin(S, t - S.tile_start, TX, TY, &x0, &y0);
            double ar = 0.0, ab = 0.0;
            unsigned char mo[NO];
#pragma unroll
            for (int jj = 0; jj < NO; ++jj) {
                const int i = threadIdx.x + jj * BT_THREADS;
                const int gx = x0 + i % TX, gy = y0 + i / TX;
                mo[jj] = (i < TX * TY && gx < L.nx && gy < L.ny) ? S.M.mode.at(gx, gy) : MODE_OUT;
            }
#pragma unroll
            for (int jj = 0; jj < NO; ++jj) {
                const int i = threadIdx.x + jj * BT_THREADS;
                const int gx = x0 + i % TX, gy = y0 + i / TX;
                const unsigned char m = mo[jj];
                if (m == MODE_OUT || !(m & MODE_COUNTED)) continue;
                const double* row = L.x.p + (size_t)gy * L.x.P + gx;
                const double pl = gx > 0 ? __ldcg(row - 1) : 0.0;
                const double pr = gx + 1 < L.nx ? __ldcg(row + 1) : 0.0;
                const double pu = gy > 0 ? __ldcg(row - L.x.P) : 0.0;
                const double pd = gy + 1 < L.ny ? __ldcg(row + L.x.P) : 0.0;
                const double pc = __ldcg(row);
                const double bb = L.b.at(gx, gy);
                double sum, den;
                if (m & MODE_STD) {
                    sum = pl;  // 1.0 * pl, exactly
                    sum = sum + pr;
                    sum = sum + pu;
                    sum = sum + pd;
                    den = 4.0;
                } else {
                    const float4 wk = S.M.w.at(gx, gy);
                    sum = (double)wk.x * pl;
                    sum = sum + (double)wk.y * pr;
                    sum = sum + (double)wk.z * pu;
                    sum = sum + (double)wk.w * pd;
                    den = S.M.den.at(gx, gy);
                }
                const double r = bb - S.factor * (den * pc - sum);
                if (m & MODE_UPDATE) {
                    S.M.rc.at(gx, gy) = (float)(S.cdiv * r);
                    S.d[cur].at(gx, gy) = 0.0f;
                }
                ar += r * r;
                ab += bb * bb;
            }
            ar = warp_sum(ar);
            ab = warp_sum(ab);
            if ((threadIdx.x & 31) == 0) {
                red_r[threadIdx.x >> 5] = ar;
                red_b[threadIdx.x >> 5] = ab;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                double tr = 0.0, tb = 0.0;
                for (int w = 0; w < BT_THREADS / 32; ++w) {
                    tr += red_r[w];
                    tb += red_b[w];
                }
                P.partials[t] = make_double2(tr, tb);
            }
            __syncthreads();
        }
        ok = grid_barrier(P.barrier, nb, P.spin_limit);
        if (!ok) break;
        // Per-simulation reduction (CTA 0, one warp per simulation, a fixed order).
        if (blockIdx.x == 0) {
            if (threadIdx.x == 0) s_cnt = 0;
            __syncthreads();
            const int lane = threadIdx.x & 31;
            for (int si = threadIdx.x >> 5; si < P.nsims; si += BT_THREADS / 32) {
                BatchState& st = P.state[si];
                if (!__ldcg(&st.active)) continue;
                const BatchSim& S = P.sims[si];
                double r = 0.0, b = 0.0;
                for (int t = S.tile_start + lane; t < S.tile_start + S.tile_count; t += 32) {
                    const double2 v = __ldcg(&P.partials[t]);
                    r += v.x;
                    b += v.y;
                }
                r = warp_sum(r);
                b = warp_sum(b);
                if (lane == 0) {
                    const double rel =
                        b > 0.0 ? sqrt(r) / sqrt(b) : (r > 0.0 ? __longlong_as_double(0x7ff0000000000000ll) : 0.0);
                    if (first) st.r0 = rel;
                    st.r1 = rel;
                    st.iterations = iters;
                    st.converged = rel <= P.tol ? 1 : 0;
                    if (st.converged || iters >= P.max_iters) st.active = 0;
                    else atomicAdd(&s_cnt, 1);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) *P.n_active = s_cnt;
        }
        ok = grid_barrier(P.barrier, nb, P.spin_limit);
        if (!ok) break;
        if (threadIdx.x == 0) s_any = __ldcg(P.n_active);
        for (int j = threadIdx.x; j < nown; j += BT_THREADS) s_act[j] = s_act[j] && __ldcg(&P.state[s_sim[j]].active);
        __syncthreads();
        if (!s_any) break;
        first = false;
        // ---- rounds of up to K red-black iterations until the next check.
        // Only update cells are loaded: every other cell's correction is 0 and
        // its coefficients are never used.
        // Work list of the rounds: every CTA appends its own active tiles that
        // hold update cells; the rounds deal the list out round-robin, so the
        // CTAs' loads differ by one tile at most.  (The order of the list does
        // not matter: within a round the tiles are independent.)
        bt_compact(nown, s_list, &s_nlist, s_wcnt, [&](int j) { return s_act[j] && (s_flags[j] & TILE_UPDATE); });
        if (threadIdx.x == 0) s_cnt = s_nlist ? atomicAdd(P.work_count, s_nlist) : 0;
        __syncthreads();
        for (int q = threadIdx.x; q < s_nlist; q += BT_THREADS) {
            const int j = s_list[q];
            P.work[s_cnt + q] = make_int2(s_sim[j], (int)blockIdx.x + j * nb);
        }
        ok = grid_barrier(P.barrier, nb, P.spin_limit);
        const int nwork = __ldcg(P.work_count);
        unsigned todo = min(P.check_interval, P.max_iters - iters);
        while (ok && todo > 0) {
            const int kk = (int)min((unsigned)K, todo);
            for (int qi = (int)blockIdx.x; qi < nwork; qi += nb) {
                const int2 wk2 = __ldcg(&P.work[qi]);
                const BatchSim& S = P.sims[wk2.x];
                const int t = wk2.y;
                const int nx = S.L.nx, ny = S.L.ny;
                int x0, y0;
                bt_tile_origin(S, t - S.tile_start, TX, TY, &x0, &y0);
                const int gx0 = x0 - H, gy0 = y0 - H, base = (gx0 + gy0) & 1;
                // Two passes so that every load of a thread is in flight at once:
                // the modes, then the corrections, right-hand sides and (for the
                // few non-standard cells) coefficients of the update cells.
                constexpr int NL = (EX * EY + BT_THREADS - 1) / BT_THREADS;
                unsigned char mm[NL];
#pragma unroll
                for (int j = 0; j < NL; ++j) {
                    const int i = threadIdx.x + j * BT_THREADS;
                    const int ly = i / EX, lx = i - ly * EX;
                    const int gx = gx0 + lx, gy = gy0 + ly;
                    mm[j] = (i < EX * EY && (unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny)
                                ? S.M.mode.at(gx, gy)
                                : (unsigned char)0;
                }
#pragma unroll
                for (int j = 0; j < NL; ++j) {
                    const int i = threadIdx.x + j * BT_THREADS;
                    if (i >= EX * EY) continue;
                    const int ly = i / EX, lx = i - ly * EX;
                    const int gx = gx0 + lx, gy = gy0 + ly;
                    const int c = (base + lx + ly) & 1, k = ly * W2 + (lx >> 1);
                    const bool ring = lx == 0 || ly == 0 || lx == EX - 1 || ly == EY - 1;
                    const bool upd = (mm[j] & MODE_UPDATE) != 0;
                    T.d[c][k] = upd ? __ldcg(&S.d[cur].at(gx, gy)) : 0.0f;
                    T.mode[c][k] = (upd && !ring) ? MODE_UPDATE : MODE_SKIP;
                    if (upd && !ring) {
                        T.rc[c][k] = __ldcg(&S.M.rc.at(gx, gy));
                        if (mm[j] & MODE_STD) {
                            T.inv[c][k] = 0.25f;
                            T.w[c][k] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
                        } else {
                            T.inv[c][k] = S.M.inv.at(gx, gy);
                            T.w[c][k] = S.M.w.at(gx, gy);
                        }
                    }
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
                    const int c = (base + lx + ly) & 1, k = ly * W2 + (lx >> 1);
                    if (gx < nx && gy < ny && (T.mode[c][k] & MODE_UPDATE)) __stcg(&S.d[cur ^ 1].at(gx, gy), T.d[c][k]);
                }
                __syncthreads();
            }
            ok = grid_barrier(P.barrier, nb, P.spin_limit);
            cur ^= 1;
            todo -= (unsigned)kk;
        }
        iters += min(P.check_interval, P.max_iters - iters);
    }
}

}  // namespace efl
