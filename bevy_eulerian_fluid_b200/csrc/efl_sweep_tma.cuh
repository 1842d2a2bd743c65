// efl_sweep_tma.cuh — fixed-count f32 red-black sweeps (the reference's
// mode, gauss_seidel.wgsl:12-88) as a persistent TMA-streaming kernel.
//
// One CTA per SM walks a list of 64 x 32 tiles.  For each tile, the Tensor
// Memory Accelerator copies five boxes -- air level set (with a one-cell
// ring), x- and y-face fractions, divergence and pressure, each covering
// the tile plus a halo of 2K = 4 cells -- from HBM into shared memory
// (cp.async.bulk.tensor, completion on an mbarrier) two tiles ahead: a
// staging buffer is refilled as soon as its tile's coefficients are built.  TMA fills
// boxes outside the field with zeros, which is the out-of-bounds
// convention of the reference's robust texture loads.  The CTA builds the
// per-cell coefficients of gauss_seidel.wgsl:44-80 in the reference's f32
// operation order, runs K = 2 red-black iterations from a
// checkerboard-compressed shared-memory image (each half-sweep over the
// cells within the distance the remaining half-sweeps still need), and
// writes its 64 x 32 owned cells to the other buffer of a ping-pong pair: one
// pass over HBM per two iterations, bit-identical to four global
// half-sweeps.
//
// Every mbarrier wait is bounded; a wait that gives up sets the error flag,
// waits (bounded again) for the CTA's own copies still in flight, and
// leaves the kernel.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "efl_kernels.cuh"
#include "efl_solver.cuh"

namespace efl {

constexpr int TS_K = 2;
constexpr int TS_H = 2 * TS_K;
constexpr int TS_TX = 64, TS_TY = 32;
constexpr int TS_EX = TS_TX + 2 * TS_H;  // 72
constexpr int TS_EY = TS_TY + 2 * TS_H;  // 40
constexpr int TS_W2 = TS_EX / 2;
constexpr int TS_THREADS = 1024;
// TMA boxes (columns x rows); x origins are multiples of 4 floats.
constexpr int BOX_PHI_W = TS_EX + 8, BOX_PHI_H = TS_EY + 2;  // from (gx0 - 4, gy0 - 1)
constexpr int BOX_FU_W = TS_EX + 4, BOX_FU_H = TS_EY;        // from (gx0, gy0)
constexpr int BOX_FV_W = TS_EX, BOX_FV_H = TS_EY + 1;
constexpr int BOX_C_W = TS_EX, BOX_C_H = TS_EY;              // divergence, pressure
constexpr int al128(int b) { return (b + 127) / 128 * 128; }
constexpr int ST_PHI = 0;
constexpr int ST_FU = ST_PHI + al128(BOX_PHI_W * BOX_PHI_H * 4);
constexpr int ST_FV = ST_FU + al128(BOX_FU_W * BOX_FU_H * 4);
constexpr int ST_DIV = ST_FV + al128(BOX_FV_W * BOX_FV_H * 4);
constexpr int ST_P = ST_DIV + al128(BOX_C_W * BOX_C_H * 4);
constexpr int ST_BYTES = ST_P + al128(BOX_C_W * BOX_C_H * 4);
constexpr unsigned TS_TX_BYTES =
    (BOX_PHI_W * BOX_PHI_H + BOX_FU_W * BOX_FU_H + BOX_FV_W * BOX_FV_H + 2 * BOX_C_W * BOX_C_H) * 4;
constexpr int TS_TILE_OFF = 2 * ST_BYTES;
constexpr int TS_BAR_OFF = TS_TILE_OFF + al128((int)sizeof(GsTile32<TS_EX, TS_EY>));
constexpr size_t TS_SMEM = (size_t)TS_BAR_OFF + 2 * sizeof(uint64_t);
constexpr long long kMbarSpinLimit = 1ll << 24;

struct SweepMaps {
    CUtensorMap phi, fu, fv, div, p[2];
};

EFL_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
EFL_DEV void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
EFL_DEV void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
EFL_DEV void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
EFL_DEV void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
EFL_DEV void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
// Waits for phase `parity` of an mbarrier, at most `limit` polls.  The
// default limit polls with try_wait, which may suspend the warp for a while
// per poll; a shorter limit (set by the caller to bound the wait tightly)
// polls with the non-blocking test_wait, so it runs out after that many
// polls whatever the hardware's suspend time.
EFL_DEV bool mbar_wait(uint64_t* bar, unsigned parity, long long limit = kMbarSpinLimit) {
    if (limit < kMbarSpinLimit) {
        for (long long i = 0; i < limit; ++i) {
            uint32_t done;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(done)
                : "r"(smem_u32(bar)), "r"(parity)
                : "memory");
            if (done) return true;
        }
        return false;
    }
    for (long long i = 0; i < kMbarSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One half-sweep of color c over the cells within D of the owned tile
// (gauss_seidel.wgsl:12-88).  A pass of K iterations needs, after half-sweep
// h (0-based), correct values only within 2K - 1 - h cells of the owned
// tile (each half-sweep reads distance-1 neighbours), so the sweeps shrink
// from the halo inwards and the owned cells come out the same.
template <int D>
EFL_DEV void ts_sweep_half(GsTile32<TS_EX, TS_EY>& T, int c, int base, float weight, float omw) {
    constexpr int NJ = TS_TX / 2 + D, ROWS = TS_TY + 2 * D, TOTAL = NJ * ROWS;
    constexpr int Y0 = TS_H - D, X0 = TS_H - D;
    const int o = 1 - c;
    for (int i = threadIdx.x; i < TOTAL; i += TS_THREADS) {
        const int r = i / NJ;
        const int ly = Y0 + r;
        const int odd = (base + ly + c) & 1;  // color-c cells of row ly sit at x = 2j + odd
        const int k = ly * TS_W2 + ((X0 - odd + 1) >> 1) + (i - r * NJ);
        const unsigned char m = T.mode[c][k];
        if (m & MODE_STD) {  // w = 1 (1 * p is p) and den = 4 (nume / 4 is nume * 0.25 exactly)
            float nume = T.cb[c][k];
            nume = nume + T.p[o][k - 1 + odd];
            nume = nume + T.p[o][k + odd];
            nume = nume + T.p[o][k - TS_W2];
            nume = nume + T.p[o][k + TS_W2];
            T.p[c][k] = weight * (nume * 0.25f) + omw * T.p[c][k];
        } else if (m & MODE_UPDATE) {
            const float4 wk = T.w[c][k];
            float nume = T.cb[c][k];
            nume = nume + wk.x * T.p[o][k - 1 + odd];
            nume = nume + wk.y * T.p[o][k + odd];
            nume = nume + wk.z * T.p[o][k - TS_W2];
            nume = nume + wk.w * T.p[o][k + TS_W2];
            const float pn = nume / T.den[c][k];
            T.p[c][k] = weight * pn + omw * T.p[c][k];
        } else if (m & MODE_ZERO) {
            T.p[c][k] = 0.0f;
        }
    }
}

__global__ void __launch_bounds__(TS_THREADS, 1)
    k_gs32_tma(const __grid_constant__ SweepMaps maps, int nx, int ny, PF out, int pin, float dx_scaled, float rho,
               float dt, float weight, int tiles_x, int ntiles, int iters, int* err, int first,
               long long wait_limit) {
    extern __shared__ __align__(128) unsigned char sm[];
    GsTile32<TS_EX, TS_EY>& T = *reinterpret_cast<GsTile32<TS_EX, TS_EY>*>(sm + TS_TILE_OFF);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + TS_BAR_OFF);
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int b) {
        const int gx0 = (t % tiles_x) * TS_TX - TS_H, gy0 = (t / tiles_x) * TS_TY - TS_H;
        unsigned char* st = sm + b * ST_BYTES;
        mbar_expect_tx(&bars[b], TS_TX_BYTES);
        tma_load_2d(st + ST_PHI, &maps.phi, gx0 - 4, gy0 - 1, &bars[b]);
        tma_load_2d(st + ST_FU, &maps.fu, gx0, gy0, &bars[b]);
        tma_load_2d(st + ST_FV, &maps.fv, gx0, gy0, &bars[b]);
        tma_load_2d(st + ST_DIV, &maps.div, gx0, gy0, &bars[b]);
        tma_load_2d(st + ST_P, pin ? &maps.p[1] : &maps.p[0], gx0, gy0, &bars[b]);
    };
    const float cdiv = dx_scaled * dx_scaled * rho / dt;  // gauss_seidel.wgsl:58
    const float omw = 1.0f - weight;
    // Tile n is staged in buffer n & 1.  Tiles 0 and 1 are issued up front; tile n + 2 goes into
    // buffer n & 1 as soon as tile n's coefficients are built (the stage is not read after that),
    // so every load has about two tiles of work to complete behind.
    int t = blockIdx.x;
    if (threadIdx.x == 0) {
        if (t < ntiles) issue(t, 0);
        if (t + (int)gridDim.x < ntiles) issue(t + gridDim.x, 1);
    }
    for (int n = 0; t < ntiles; t += gridDim.x, ++n) {
        const int b = n & 1;
        const bool next = t + (int)gridDim.x < ntiles;
        const bool after = t + 2 * (int)gridDim.x < ntiles;
        // Warp 0 waits for the copies; the barrier then orders the other warps' reads after its
        // acquire (the other 31 warps sleep in the barrier instead of spinning on the mbarrier).
        const bool got = threadIdx.x < 32 ? mbar_wait(&bars[b], (n >> 1) & 1, wait_limit) : true;
        if (__syncthreads_or(!got)) {
            if (threadIdx.x == 0) {
                atomicExch(err, 1);
                mbar_wait(&bars[b], (n >> 1) & 1);  // copies of this CTA still in flight (default limit)
                if (next) mbar_wait(&bars[b ^ 1], ((n + 1) >> 1) & 1);
            }
            return;
        }
        const unsigned char* stb = sm + b * ST_BYTES;
        const float* phi_s = reinterpret_cast<const float*>(stb + ST_PHI);
        const float* fu_s = reinterpret_cast<const float*>(stb + ST_FU);
        const float* fv_s = reinterpret_cast<const float*>(stb + ST_FV);
        const float* div_s = reinterpret_cast<const float*>(stb + ST_DIV);
        const float* p_s = reinterpret_cast<const float*>(stb + ST_P);
        const int gx0 = (t % tiles_x) * TS_TX - TS_H, gy0 = (t / tiles_x) * TS_TY - TS_H;
        const int base = (gx0 + gy0) & 1;
        // Coefficients of every cell of the extended tile (gauss_seidel.wgsl:44-80).
        for (int i = threadIdx.x; i < TS_EX * TS_EY; i += TS_THREADS) {
            const int ly = i / TS_EX, lx = i - ly * TS_EX;
            const int gx = gx0 + lx, gy = gy0 + ly;
            const int c = (base + lx + ly) & 1, k = ly * TS_W2 + (lx >> 1);
            T.p[c][k] = p_s[ly * BOX_C_W + lx];
            // the outermost ring is only read as neighbour pressure
            if (lx == 0 || ly == 0 || lx == TS_EX - 1 || ly == TS_EY - 1) continue;
            unsigned char m = MODE_SKIP;
            float den = 0.0f, cb = 0.0f;
            float4 wk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if ((unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny) {
                const int pc = (ly + 1) * BOX_PHI_W + lx + 4;
                const float lij = phi_s[pc];
                bool update = false;
                if (lij < 0.0f) {
                    const float f[4] = {fu_s[ly * BOX_FU_W + lx], fu_s[ly * BOX_FU_W + lx + 1],
                                        fv_s[ly * BOX_FV_W + lx], fv_s[(ly + 1) * BOX_FV_W + lx]};
                    if (!(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) {
                        cb = cdiv * div_s[ly * BOX_C_W + lx];
                        const bool inb[4] = {gx - 1 >= 0, gx + 1 < nx, gy - 1 >= 0, gy + 1 < ny};
                        const float lv[4] = {phi_s[pc - 1], phi_s[pc + 1], phi_s[pc - BOX_PHI_W],
                                             phi_s[pc + BOX_PHI_W]};
                        float wv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            if (inb[q]) {
                                if (lv[q] < 0.0f) {
                                    den += f[q];
                                    wv[q] = f[q];
                                } else {
                                    den += f[q] * (1.0f - lv[q] / lij);
                                }
                            }
                        }
                        wk = make_float4(wv[0], wv[1], wv[2], wv[3]);
                        update = !(fabsf(den) < 1.0e-6f);
                    }
                }
                m = update ? MODE_UPDATE : MODE_ZERO;
                if (update && wk.x == 1.0f && wk.y == 1.0f && wk.z == 1.0f && wk.w == 1.0f) m |= MODE_STD;
            }
            T.cb[c][k] = cb;
            T.den[c][k] = den;
            T.w[c][k] = wk;
            T.mode[c][k] = m;
        }
        __syncthreads();
        if (threadIdx.x == 0 && after) {
            fence_proxy_async();  // the generic reads of stage[b] above before the async writes
            issue(t + 2 * gridDim.x, b);
        }
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int c = half == 0 ? first : 1 - first;  // red ((x+y) odd) first unless first = 0
                switch (2 * (iters - it) - 1 - half) {  // distance still needed after this half-sweep
                    case 3: ts_sweep_half<3>(T, c, base, weight, omw); break;
                    case 2: ts_sweep_half<2>(T, c, base, weight, omw); break;
                    case 1: ts_sweep_half<1>(T, c, base, weight, omw); break;
                    default: ts_sweep_half<0>(T, c, base, weight, omw); break;
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < TS_TX * TS_TY; i += TS_THREADS) {
            const int ly = TS_H + i / TS_TX, lx = TS_H + i % TS_TX;
            const int gx = gx0 + lx, gy = gy0 + ly;
            if ((unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny)
                out.at(gx, gy) = T.p[(base + lx + ly) & 1][ly * TS_W2 + (lx >> 1)];
        }
        __syncthreads();  // the tile image and stage[b] are free again
    }
}

// Host side: tensor maps of the five planes, created once per simulation.
struct SweepTma {
    SweepMaps maps;
    bool ok = false;
    int* d_err = nullptr;
    long long wait_limit = kMbarSpinLimit;  // polls of a tile's mbarrier wait before giving up
};

inline PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled)p;
    }
    return fn;
}

inline bool make_map_2d(CUtensorMap* m, const void* base, uint64_t w, uint64_t h, int pitch_floats, uint32_t box_w,
                        uint32_t box_h) {
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {w, h};
    cuuint64_t strides[1] = {(cuuint64_t)pitch_floats * 4};
    cuuint32_t box[2] = {box_w, box_h};
    cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline bool sweep_tma_init(SweepTma& st, const Level& L, const PF& alt) {
    const int nx = L.nx, ny = L.ny;
    st.ok = make_map_2d(&st.maps.phi, L.ls.p, nx, ny, L.ls.P, BOX_PHI_W, BOX_PHI_H) &&
            make_map_2d(&st.maps.fu, L.fu.p, nx + 1, ny, L.fu.P, BOX_FU_W, BOX_FU_H) &&
            make_map_2d(&st.maps.fv, L.fv.p, nx, ny + 1, L.fv.P, BOX_FV_W, BOX_FV_H) &&
            make_map_2d(&st.maps.div, L.b.p, nx, ny, L.b.P, BOX_C_W, BOX_C_H) &&
            make_map_2d(&st.maps.p[0], L.x.p, nx, ny, L.x.P, BOX_C_W, BOX_C_H) &&
            make_map_2d(&st.maps.p[1], alt.p, nx, ny, alt.P, BOX_C_W, BOX_C_H);
    // The flag starts clear: cudaMalloc returns memory with whatever an earlier allocation left in it, and
    // only the fixed-count solve clears the flag before its sweeps (the MGPCG preconditioner's do not).
    if (st.ok && !st.d_err)
        st.ok = cudaMalloc(&st.d_err, sizeof(int)) == cudaSuccess && cudaMemset(st.d_err, 0, sizeof(int)) == cudaSuccess;
    return st.ok;
}
inline void sweep_tma_free(SweepTma& st) {
    if (st.d_err) cudaFree(st.d_err);
    st = SweepTma{};
}

// The kernel's dynamic shared-memory size, set once per device.
inline bool tma_kernel_ready() {
    int dev = 0;
    cudaGetDevice(&dev);
    static bool attr_done[64] = {};
    if (dev < 0 || dev >= 64) return false;
    if (!attr_done[dev]) {
        if (cudaFuncSetAttribute(k_gs32_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS_SMEM) !=
            cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        attr_done[dev] = true;
    }
    return true;
}

// One pass of `iters` (<= 2) red-black iterations, first colour `first`
// (1 = red, the reference's order), reading the pressure of map p[pin] and
// writing `out`.
inline efl_status tma_sweep_pass(const SweepTma& st, int nx, int ny, const PF& out, int pin, int num_sms,
                                 float dx_scaled, float rho, float dt, float weight, int iters, int first, int* err,
                                 cudaStream_t stream) {
    if (!st.ok || iters < 1 || iters > TS_K || !tma_kernel_ready()) return EFL_ERR_STATE;
    const int tiles_x = (nx + TS_TX - 1) / TS_TX, ntiles = tiles_x * ((ny + TS_TY - 1) / TS_TY);
    k_gs32_tma<<<std::min(ntiles, num_sms), TS_THREADS, TS_SMEM + count_launch(), stream>>>(
        st.maps, nx, ny, out, pin, dx_scaled, rho, dt, weight, tiles_x, ntiles, iters, err, first, st.wait_limit);
    return cudaGetLastError() == cudaSuccess ? EFL_OK : EFL_ERR_CUDA;
}

// n fixed f32 red-black iterations at level 0 with the TMA kernel,
// ping-ponging between L.x (map p[0]) and alt (map p[1]); the result ends in
// L.x.  Returns EFL_ERR_STATE when the TMA path is unavailable.
inline efl_status solve_gs32_tma(SweepTma& st, const Level& L, const PF& alt, int num_sms, float dx_scaled,
                                 float rho, float dt, float weight, uint32_t n, cudaStream_t stream,
                                 std::string* err) {
    if (!st.ok || !tma_kernel_ready()) return EFL_ERR_STATE;
    const int tiles_x = (L.nx + TS_TX - 1) / TS_TX, tiles_y = (L.ny + TS_TY - 1) / TS_TY;
    const int ntiles = tiles_x * tiles_y;
    const int grid = std::min(ntiles, num_sms);
    if (cudaMemsetAsync(st.d_err, 0, sizeof(int), stream) != cudaSuccess) return EFL_ERR_CUDA;
    int pin = 0;
    uint32_t launches = 0;
    for (uint32_t done = 0; done < n;) {
        const int k = (int)std::min<uint32_t>(TS_K, n - done);
        PF out = pin == 0 ? alt : L.x;
        k_gs32_tma<<<grid, TS_THREADS, TS_SMEM + count_launch(), stream>>>(st.maps, L.nx, L.ny, out, pin, dx_scaled,
                                                                           rho, dt, weight, tiles_x, ntiles, k,
                                                                           st.d_err, 1, st.wait_limit);
        pin ^= 1;
        done += (uint32_t)k;
        ++launches;
    }
    if (launches & 1) {
        if (cudaMemcpy2DAsync(L.x.p, (size_t)L.x.P * 4, alt.p, (size_t)alt.P * 4, (size_t)L.nx * 4, L.ny,
                              cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
            return EFL_ERR_CUDA;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        *err = std::string("TMA sweep launch failed: ") + cudaGetErrorString(e);
        return EFL_ERR_CUDA;
    }
    return EFL_OK;
}

}  // namespace efl
