// efl_unet.cuh — the learned warm start (an extension with no reference
// counterpart): a small U-Net in BF16 with FP32 accumulation whose 3x3
// convolutions run on the 5th-generation tensor cores (tcgen05.mma,
// kind::f16, operands in shared memory, accumulator in tensor memory).
//
// Activations are NHWC bf16 with the channel count a multiple of 16; a tensor
// may be a channel slice (stride, offset) of a wider one, which is how the
// skip connections are concatenated without copies.  Master weights are fp32
// [tap = 9][cout][cin] (tap = (dy + 1) * 3 + (dx + 1)), biases fp32; the
// convolutions read BF16 copies laid out as one K-major tile per tap.
//
// One convolution = one implicit GEMM per CTA: 128 consecutive output pixels
// (M = 128) x cout (N), accumulated over 9 taps x cin / 16 MMAs of K = 16.
// Operand tiles use the canonical K-major, non-swizzled core-matrix layout
// (8 rows x 16 bytes per core matrix, core matrices along K 128 bytes apart
// (LBO), along M/N (K/8) * 128 bytes apart (SBO)).  The backward pass over
// the data is the same kernel with the weights flipped in space and
// transposed; the weight gradient is a second tcgen05 GEMM whose reduction
// dimension is the pixels.  Every wait on an mbarrier is bounded.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "efl_sweep_tma.cuh"

namespace efl {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// tcgen05 helpers

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (M/N) byte offsets in 16-byte units, version 1, no swizzle.
EFL_DEV uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
EFL_DEV void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
EFL_DEV void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
EFL_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
EFL_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
EFL_DEV void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {  // whole warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
EFL_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // whole warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 16 consecutive fp32 columns of this thread's TMEM lane.
EFL_DEV void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__host__ __device__ constexpr uint32_t tmem_cols(int n) { return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : 256u; }

EFL_DEV float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Byte offset of element (row, k) in a K-major non-swizzled tile with K columns.
EFL_DEV uint32_t kmajor_off(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// ---------------------------------------------------------------------------
// 3x3 convolution, stride 1, zero padding: the multistage form, for any width
// (the network runs it where the width is not a multiple of 128; the row-tile
// form below covers the others).

constexpr int CV_THREADS = 128, CV_MAX_CIN = 128, CV_MAX_COUT = 128;
constexpr int CV_STAGES = 4;              // A stages: taps t + 1 and t + 2 load while tap t multiplies
constexpr int CV_SMEM = 226 * 1024;       // dynamic shared memory ceiling (227 KB per CTA less static)
constexpr int CV_BULK_CHUNK = 32768;      // bytes per bulk weight copy

// Shared memory of one convolution CTA, in this order:
//  - CV_STAGES A stages (128 x cin, K-major core matrices), tap t in stage
//    t % CV_STAGES, filled by 16-byte asynchronous copies two taps ahead;
//  - the weight tiles (cout x cin per tap, K-major, bulk-copied): all nine
//    taps when that costs no occupancy, else a ring of three filled one tap
//    ahead;
//  - mbarriers: one per A stage (its MMAs done), three for the weight copies.
__host__ __device__ constexpr int conv_a_bytes(int cin) { return 128 * cin * 2; }
__host__ __device__ constexpr int conv_b_bytes(int cin, int cout) { return cout * cin * 2; }
__host__ __device__ constexpr int conv_smem_with(int cin, int cout, int btiles) {
    return CV_STAGES * conv_a_bytes(cin) + btiles * conv_b_bytes(cin, cout) + 64;
}
// CTAs per SM: shared memory (228 KB per SM, 1 KB reserved per CTA), tensor
// memory columns (512 per SM) and threads (2048 per SM).
__host__ __device__ constexpr int conv_ctas_per_sm(int smem, int cout) {
    return (228 * 1024) / (smem + 1024) < 512 / (int)tmem_cols(cout)
               ? ((228 * 1024) / (smem + 1024) < 2048 / CV_THREADS ? (228 * 1024) / (smem + 1024) : 2048 / CV_THREADS)
               : (512 / (int)tmem_cols(cout) < 2048 / CV_THREADS ? 512 / (int)tmem_cols(cout) : 2048 / CV_THREADS);
}
__host__ __device__ constexpr bool conv_weights_resident(int cin, int cout) {
    return conv_smem_with(cin, cout, 9) <= CV_SMEM &&
           conv_ctas_per_sm(conv_smem_with(cin, cout, 9), cout) >= conv_ctas_per_sm(conv_smem_with(cin, cout, 3), cout);
}
__host__ __device__ constexpr int conv_smem_bytes(int cin, int cout) {
    return conv_smem_with(cin, cout, conv_weights_resident(cin, cout) ? 9 : 3);
}

// Element index of (row, k) in a K-major non-swizzled tile with K columns
// (the element form of kmajor_off).
__host__ __device__ constexpr int kmajor_index(int row, int k, int K) {
    return ((row >> 3) * (K >> 3) + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7);
}

struct ConvArgs {
    const bf16* x;  // input [H*W][xs], channels [xo, xo + cin)
    int xs, xo;
    const bf16* w;       // 9 tap tiles of cout x cin, each K-major (kmajor_index(co, ci, cin))
    const float* bias;   // [cout] or null
    bf16* y;             // bf16 output [H*W][ys] at [yo, yo + cout), or null
    int ys, yo;
    float* yf;           // fp32 output [H*W][ys] at [yo, yo + cout) (used when y is null; ys, yo multiples of 4)
    int relu;
    int H, W, cin, cout;
    int* err;
    const unsigned char* gap = nullptr;  // [H*W]: 0 = a canvas gap pixel, whose outputs are written as zeros
    int resident = -1;  // k_conv3x3_tc: all nine weight tiles resident (1), the ring of three (0), by the rule (-1)
};
// k_conv3x3_tc's weights: resident for a grid of one round (its latency, not the occupancy, counts), else by the
// occupancy rule.
inline bool conv_tc_resident(const ConvArgs& a) { return a.resident >= 0 ? a.resident != 0 : conv_weights_resident(a.cin, a.cout); }

// 16-byte asynchronous copy global -> shared through L1 (the nine taps of a
// pixel tile re-read overlapping rows); zero-fills when !full.
EFL_DEV void cp_async16(void* dst, const void* src, bool full) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(full ? 16 : 0)
                 : "memory");
}
EFL_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
EFL_DEV void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// Bulk copy global -> shared of `bytes` (a multiple of 16, both addresses
// 16-byte aligned), completing on bar's transaction count.
EFL_DEV void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// One thread: arms bar for `bytes` and copies them in chunks.
EFL_DEV void bulk_load_all(unsigned char* dst, const unsigned char* src, uint32_t bytes, uint64_t* bar) {
    mbar_expect_tx(bar, bytes);
    for (uint32_t o = 0; o < bytes; o += CV_BULK_CHUNK)
        bulk_load(dst + o, src + o, bytes - o < (uint32_t)CV_BULK_CHUNK ? bytes - o : (uint32_t)CV_BULK_CHUNK, bar);
}
// This thread's input row of one tap (zero outside the image) into an A stage.
EFL_DEV void conv_load_tap(const ConvArgs& a, int tap, int m, int py, int px, bool inside, unsigned char* As) {
    const int sy = py + tap / 3 - 1, sx = px + tap % 3 - 1;
    const bool valid = inside && (unsigned)sy < (unsigned)a.H && (unsigned)sx < (unsigned)a.W;
    const bf16* src = valid ? a.x + (size_t)(sy * a.W + sx) * a.xs + a.xo : a.x;
    for (int j = 0; j < (a.cin >> 3); ++j) cp_async16(As + kmajor_off(m, 8 * j, a.cin), src + (valid ? 8 * j : 0), valid);
}

__global__ void __launch_bounds__(CV_THREADS) k_conv3x3_tc(ConvArgs a) {
    extern __shared__ __align__(128) unsigned char cv_smem[];
    const int abytes = conv_a_bytes(a.cin), bbytes = conv_b_bytes(a.cin, a.cout);
    const bool resident = a.resident >= 0 ? a.resident != 0 : conv_weights_resident(a.cin, a.cout);
    unsigned char* Ab = cv_smem;
    unsigned char* Bb = Ab + CV_STAGES * abytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bb + (resident ? 9 : 3) * bbytes);  // [CV_STAGES]: MMAs done
    uint64_t* wbar = bar + CV_STAGES;                                                // [3]: weight copies done
    const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int npix = a.H * a.W, p0 = blockIdx.x * 128;
    const uint32_t ncols = tmem_cols(a.cout);
    const int m = tid, p = p0 + m;
    const int py = p / a.W, px = p - py * a.W;
    // The first taps' rows start loading before anything else (one copy group per tap).
    for (int t = 0; t < CV_STAGES - 2; ++t) {
        conv_load_tap(a, t, m, py, px, p < npix, Ab + t * abytes);
        cp_async_commit();
    }
    if (warp == 0) tmem_alloc(&s_tmem, ncols);
    if (tid == 0) {
        for (int i = 0; i < CV_STAGES + 3; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Weight copies, issued and awaited by thread 0 in order: unit u is the
    // whole resident block (u = 0) or ring tap u, on wbar[u % 3] with phase
    // parity (u / 3) & 1.
    int wissued = 0, wdone = 0;
    if (tid == 0) {
        if (resident) {
            bulk_load_all(Bb, wsrc, 9 * bbytes, &wbar[0]);
            wissued = 1;
        } else {
            bulk_load_all(Bb, wsrc, bbytes, &wbar[0]);
            bulk_load_all(Bb + bbytes, wsrc + bbytes, bbytes, &wbar[1]);
            wissued = 2;
        }
    }
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = umma_idesc_bf16(128, a.cout);
    const uint32_t sbo = (uint32_t)(a.cin >> 3) * 128;
    // Tap t is the (t / CV_STAGES)-th completion of bar[t % CV_STAGES], so its
    // phase parity is (t / CV_STAGES) & 1; each completion is awaited (two taps
    // after its issue) before the next one on the same barrier can happen.
    bool ok = true;
    int last = -1;  // last tap whose MMAs were committed
    for (int tap = 0; tap < 9; ++tap) {
        const int s = tap % CV_STAGES;
        unsigned char* As = Ab + s * abytes;
        unsigned char* Bs = Bb + (resident ? tap : tap % 3) * bbytes;
        cp_async_wait<CV_STAGES - 3>();  // this thread's rows of this tap have landed
        fence_proxy_async();
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        if (tid == 0) {
            if (ok && (!resident || tap == 0)) {
                const int u = resident ? 0 : tap;
                if (mbar_wait(&wbar[u % 3], (u / 3) & 1)) wdone = u + 1;
                else ok = false;
            }
            tc_fence_after();
            if (ok) {
                const uint32_t sa = smem_u32(As), sb = smem_u32(Bs);
                for (int kc = 0; kc < (a.cin >> 4); ++kc)
                    umma_bf16(tmem, umma_desc(sa + kc * 256, 128, sbo), umma_desc(sb + kc * 256, 128, sbo), idesc,
                              (tap | kc) != 0);
            }
            umma_commit(&bar[s]);  // also when skipped, so that the waits on it end
        }
        last = tap;
        if (tap >= 2) {  // the MMAs of tap - 2 are done with their A stage and weight tile
            const int d = tap - 2;
            ok = mbar_wait(&bar[d % CV_STAGES], (d / CV_STAGES) & 1) && ok;
        }
        if (ok && tap + CV_STAGES - 2 < 9) {
            const int u = tap + CV_STAGES - 2;  // into the A stage the MMAs of tap - 2 read
            conv_load_tap(a, u, m, py, px, p < npix, Ab + (u % CV_STAGES) * abytes);
        }
        cp_async_commit();
        if (!resident && tid == 0 && ok && tap >= 1 && tap + 1 < 9) {
            const int u = tap + 1;  // into ring tile u % 3, last read by the MMAs of tap - 2
            bulk_load_all(Bb + (u % 3) * bbytes, wsrc + (size_t)u * bbytes, bbytes, &wbar[u % 3]);
            wissued = u + 1;
        }
    }
    if (ok) ok = mbar_wait(&bar[8 % CV_STAGES], (8 / CV_STAGES) & 1);  // tap 8's commit tracks every earlier MMA
    cp_async_wait<0>();
    ok = !__syncthreads_or(!ok);
    if (!ok) {
        if (tid == 0) {
            atomicExch(a.err, 1);
            for (int u = wdone; u < wissued; ++u) mbar_wait(&wbar[u % 3], (u / 3) & 1);  // copies in flight
        }
        // give the MMAs in flight a last bounded chance before releasing TMEM
        if (last >= 0) mbar_wait(&bar[last % CV_STAGES], (last / CV_STAGES) & 1);
    }
    tc_fence_after();
    if (ok) {
        const int row = 32 * warp + lane, pp = p0 + row;
        const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);
        for (int c0 = 0; c0 < a.cout; c0 += 16) {
            float v[16];
            tmem_ld16(taddr + (uint32_t)c0, v);
            if (pp >= npix) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float t = v[i] + (a.bias ? a.bias[c0 + i] : 0.0f);
                if (a.relu) t = fmaxf(t, 0.0f);
                if (a.gap && !a.gap[pp]) t = 0.0f;
                v[i] = t;
            }
            if (a.y) {
                __align__(16) bf16 o[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) o[i] = __float2bfloat16_rn(v[i]);
                uint4* dst = reinterpret_cast<uint4*>(a.y + (size_t)pp * a.ys + a.yo + c0);
                dst[0] = reinterpret_cast<const uint4*>(o)[0];
                dst[1] = reinterpret_cast<const uint4*>(o)[1];
            } else {
                float4* dst = reinterpret_cast<float4*>(a.yf + (size_t)pp * a.ys + a.yo + c0);  // 16-byte aligned
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// 3x3 convolution for image widths that are a multiple of 128: a CTA's
// output pixels are 128-pixel stretches of one image row, so the input it
// needs is three rows of those pixels and one pixel either side (130 for one
// stretch; zero outside the image), staged once.  In shared memory the three
// rows form one plane per 8-channel group (16 bytes per pixel), and tap
// (dy, dx)'s A operand for a stretch is its 128 rows shifted by dx within
// segment row dy: a K-major non-swizzled operand with core matrices 128 bytes
// apart along M (SBO) and one plane apart along K (LBO), starting on a
// 16-byte boundary.  The nine taps' MMAs then go out back to back with no
// copies or block barriers between them.

constexpr int CR_RING = 4;  // weight tiles in flight when not all nine are resident
// Two stretches per CTA only while the CTA stays this small (three or more per
// SM): at 48 -> 16 and 96 -> 32 channels the larger CTAs lost more residency
// than the halved CTA count gained (40 vs 33 us and 30 vs 25 us at 512^2 and
// 256^2), at cin <= 32 they gained (19 vs 25 us at 16 -> 16, 512^2).
constexpr int CR_PAIR_SMEM = 64 * 1024;

// A CTA of the row-tile kernel covers TILES adjacent 128-pixel stretches of
// one row (threads 128 * TILES); its input segment per tap row is those
// pixels and one either side.
__host__ __device__ constexpr int crow_seg_rows(int tiles) { return 128 * tiles + 2; }
__host__ __device__ constexpr int crow_plane(int tiles) { return 3 * crow_seg_rows(tiles) * 16; }
__host__ __device__ constexpr int crow_seg_bytes(int cin, int tiles) { return ((cin >> 3) * crow_plane(tiles) + 127) & ~127; }
__host__ __device__ constexpr int crow_smem_with(int cin, int cout, int btiles, int tiles) {
    return crow_seg_bytes(cin, tiles) + btiles * conv_b_bytes(cin, cout) + 128;
}
__host__ __device__ constexpr int crow_smem_bytes(int cin, int cout, bool resident, int tiles) {
    return crow_smem_with(cin, cout, resident ? 9 : CR_RING, tiles);
}

// RESIDENT: all nine weight tiles in one bulk copy, else the ring.  TILES
// (1 or 2): 128-pixel stretches per CTA, each with its own accumulator; two
// halve the CTAs (and tensor-memory allocations) of the large grids and share
// one segment and one weight stream.
template <bool RESIDENT, int TILES>
__global__ void __launch_bounds__(CV_THREADS * TILES) k_conv3x3_rows(ConvArgs a) {
    extern __shared__ __align__(128) unsigned char cv_smem[];
    constexpr int SEG = crow_seg_rows(TILES), PLANE = crow_plane(TILES), NT = CV_THREADS * TILES;
    const int kg = a.cin >> 3, bbytes = conv_b_bytes(a.cin, a.cout);
    constexpr bool resident = RESIDENT;
    unsigned char* seg = cv_smem;
    unsigned char* Bb = cv_smem + crow_seg_bytes(a.cin, TILES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bb + (resident ? 9 : CR_RING) * bbytes);  // [CR_RING]: slot's MMAs done
    uint64_t* wbar = bar + CR_RING;                                                         // [CR_RING]: slot's copy done
    uint64_t* done = bar + 2 * CR_RING;                                                     // every MMA done
    const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ctas_per_row = a.W / (128 * TILES);
    const int y = blockIdx.x / ctas_per_row, x0 = (blockIdx.x - y * ctas_per_row) * 128 * TILES;
    const uint32_t acols = tmem_cols(a.cout), ncols = TILES * acols;
    {  // segment row r * SEG + o holds pixel (y + r - 1, x0 - 1 + o); channel group fastest across threads
        const int total = 3 * SEG * kg;
        const int drow = NT / kg, dg = NT - drow * kg;
        int row = tid / kg, g = tid - row * kg;  // of element c = row * kg + g
        for (int c = tid; c < total; c += NT) {
            const int r = row >= 2 * SEG ? 2 : row >= SEG ? 1 : 0;
            const int sy = y + r - 1, sx = x0 - 1 + (row - r * SEG);
            const bool in = (unsigned)sy < (unsigned)a.H && (unsigned)sx < (unsigned)a.W;
            cp_async16(seg + g * PLANE + row * 16, in ? a.x + (size_t)(sy * a.W + sx) * a.xs + a.xo + 8 * g : a.x, in);
            row += drow;
            g += dg;
            if (g >= kg) {
                g -= kg;
                ++row;
            }
        }
        cp_async_commit();
    }
    if (warp == 0) tmem_alloc(&s_tmem, ncols);
    if (tid == 0) {
        for (int i = 0; i < 2 * CR_RING + 1; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    cp_async_wait<0>();
    fence_proxy_async();  // the segment writes before the tensor cores read them
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    bool ok = true;
    if (tid == 0) {
        // Weight copies, issued and awaited in order: unit u is the whole
        // resident block (u = 0) or ring tap u, on wbar[u % CR_RING] with
        // phase parity (u / CR_RING) & 1; ring slot u % CR_RING is refilled
        // with tap u + CR_RING once the MMAs of tap u are done, two taps later.
        int wissued, wdone = 0;
        if (resident) {
            bulk_load_all(Bb, wsrc, 9 * bbytes, &wbar[0]);
            wissued = 1;
        } else {
            for (int u = 0; u < CR_RING; ++u)
                bulk_load_all(Bb + u * bbytes, wsrc + (size_t)u * bbytes, bbytes, &wbar[u]);
            wissued = CR_RING;
        }
        const uint32_t idesc = umma_idesc_bf16(128, a.cout);
        const uint32_t sseg = smem_u32(seg), sbo_b = (uint32_t)kg * 128;
        for (int tap = 0; tap < 9 && ok; ++tap) {
            if (!resident || tap == 0) {
                const int u = resident ? 0 : tap;
                if (!mbar_wait(&wbar[u % CR_RING], (u / CR_RING) & 1)) {
                    ok = false;
                    break;
                }
                wdone = u + 1;
            }
            tc_fence_after();
            const uint32_t sb = smem_u32(Bb + (resident ? tap : tap % CR_RING) * bbytes);
            for (int t = 0; t < TILES; ++t) {
                // tile t's rows start 128 * t further along the segment
                const uint32_t sa = sseg + (uint32_t)(((tap / 3) * SEG + tap % 3 + 128 * t) * 16);
                for (int kc = 0; kc < (a.cin >> 4); ++kc)
                    umma_bf16(tmem + t * acols, umma_desc(sa + (uint32_t)(2 * kc * PLANE), PLANE, 128),
                              umma_desc(sb + kc * 256, 128, sbo_b), idesc, (tap | kc) != 0);
            }
            if (!resident) {
                umma_commit(&bar[tap % CR_RING]);
                const int d = tap + 2 - CR_RING, u = tap + 2;
                if (d >= 0 && u < 9) {  // ring slot of tap d takes tap u once d's MMAs are done
                    if (!mbar_wait(&bar[d % CR_RING], (d / CR_RING) & 1)) {
                        ok = false;
                        break;
                    }
                    bulk_load_all(Bb + (u % CR_RING) * bbytes, wsrc + (size_t)u * bbytes, bbytes, &wbar[u % CR_RING]);
                    wissued = u + 1;
                }
            }
        }
        umma_commit(done);  // also after a failure, so that the waits on it end
        if (!ok) {
            atomicExch(a.err, 1);
            for (int u = wdone; u < wissued; ++u) mbar_wait(&wbar[u % CR_RING], (u / CR_RING) & 1);  // in flight
        }
    }
    ok = mbar_wait(done, 0) && ok;
    ok = !__syncthreads_or(!ok);
    if (!ok && tid == 0) atomicExch(a.err, 1);
    tc_fence_after();
    if (ok) {  // warp w drains tile w / 4 from TMEM lanes 32 * (w % 4) ..
        const int t = warp >> 2, row = 32 * (warp & 3) + lane;
        const size_t pp = (size_t)y * a.W + x0 + 128 * t + row;
        const uint32_t taddr = tmem + t * acols + ((uint32_t)(32 * (warp & 3)) << 16);
        for (int c0 = 0; c0 < a.cout; c0 += 16) {
            float v[16];
            tmem_ld16(taddr + (uint32_t)c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float tv = v[i] + (a.bias ? a.bias[c0 + i] : 0.0f);
                if (a.relu) tv = fmaxf(tv, 0.0f);
                if (a.gap && !a.gap[pp]) tv = 0.0f;
                v[i] = tv;
            }
            if (a.y) {
                __align__(16) bf16 o[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) o[i] = __float2bfloat16_rn(v[i]);
                uint4* dst = reinterpret_cast<uint4*>(a.y + pp * a.ys + a.yo + c0);
                dst[0] = reinterpret_cast<const uint4*>(o)[0];
                dst[1] = reinterpret_cast<const uint4*>(o)[1];
            } else {
                float4* dst = reinterpret_cast<float4*>(a.yf + pp * a.ys + a.yo + c0);  // 16-byte aligned
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// Weight gradient: dW[tap][co][ci] = sum_p dy[p][co] * x[p + tap][ci].
// GEMM D[(tap, ci)][co] over K = pixels: A rows r = tap * cin + ci (M tiles of
// 128 rows; rows beyond 9 * cin are zero), B rows co.  Each CTA reduces one
// chunk of pixels for one M tile and writes its partial D; k_wgrad_reduce
// sums the chunks in order.

constexpr int WG_THREADS = 128, WG_K = 64;  // pixels per staged block
constexpr int WG_SMEM = 128 * WG_K * 2 + CV_MAX_COUT * WG_K * 2 + 64;

struct WgradArgs {
    const bf16* x;  // forward input [H*W][xs] at xo
    int xs, xo;
    const bf16* dy;  // [H*W][cout] dense
    int H, W, cin, cout;
    int pix_per_cta;  // multiple of WG_K
    float* part;      // [chunks][mtiles][128][cout]
    int* err;
};

__global__ void __launch_bounds__(WG_THREADS) k_wgrad_tc(WgradArgs a) {
    extern __shared__ __align__(128) unsigned char wg_smem[];
    unsigned char* As = wg_smem;                  // 128 x WG_K
    unsigned char* Bs = wg_smem + 128 * WG_K * 2;  // cout x WG_K
    uint64_t* bar = reinterpret_cast<uint64_t*>(wg_smem + 128 * WG_K * 2 + CV_MAX_COUT * WG_K * 2);
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int npix = a.H * a.W;
    const int chunk = blockIdx.x, tile = blockIdx.y, mtiles = gridDim.y;
    const uint32_t ncols = tmem_cols(a.cout);
    if (warp == 0) tmem_alloc(&s_tmem, ncols);
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = umma_idesc_bf16(128, a.cout);
    const uint32_t sbo = (WG_K / 8) * 128;
    const int og = a.cout >> 3;
    const int pbeg = chunk * a.pix_per_cta, pend = min(npix, pbeg + a.pix_per_cta);
    bool ok = true;
    int stage = 0;
    for (int pb = pbeg; pb < pend && ok; pb += WG_K, ++stage) {
        // A: 16 row groups of 8 (tap, ci) rows x WG_K pixels; one 16-byte load = 8 channels of one pixel.
        for (int i = tid; i < 16 * WG_K; i += WG_THREADS) {
            const int g = i / WG_K, k = i - g * WG_K;
            const int r0 = tile * 128 + 8 * g;  // first row of the group
            const int tap = r0 / a.cin, ci0 = r0 - tap * a.cin;
            const int pp = pb + k;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (tap < 9 && pp < pend) {
                const int py = pp / a.W, px = pp - py * a.W;
                const int sy = py + tap / 3 - 1, sx = px + tap % 3 - 1;
                if ((unsigned)sy < (unsigned)a.H && (unsigned)sx < (unsigned)a.W)
                    v = __ldg(reinterpret_cast<const uint4*>(a.x + (size_t)(sy * a.W + sx) * a.xs + a.xo + ci0));
            }
            const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
            for (int q = 0; q < 8; ++q) *reinterpret_cast<bf16*>(As + kmajor_off(8 * g + q, k, WG_K)) = e[q];
        }
        // B: cout rows x WG_K pixels.
        for (int i = tid; i < og * WG_K; i += WG_THREADS) {
            const int g = i / WG_K, k = i - g * WG_K;
            const int pp = pb + k;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (pp < pend) v = __ldg(reinterpret_cast<const uint4*>(a.dy + (size_t)pp * a.cout + 8 * g));
            const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
            for (int q = 0; q < 8; ++q) *reinterpret_cast<bf16*>(Bs + kmajor_off(8 * g + q, k, WG_K)) = e[q];
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sa = smem_u32(As), sb = smem_u32(Bs);
            for (int kc = 0; kc < WG_K / 16; ++kc)
                umma_bf16(tmem, umma_desc(sa + kc * 256, 128, sbo), umma_desc(sb + kc * 256, 128, sbo), idesc,
                          (stage | kc) != 0);
            umma_commit(bar);
        }
        ok = mbar_wait(bar, stage & 1);
        if (__syncthreads_or(!ok)) ok = false;
    }
    if (!ok) {
        if (tid == 0) atomicExch(a.err, 1);
        mbar_wait(bar, 0);
    }
    tc_fence_after();
    const int row = 32 * warp + lane;
    float* dst = a.part + (((size_t)chunk * mtiles + tile) * 128 + row) * a.cout;
    const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);
    for (int c0 = 0; c0 < a.cout; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + (uint32_t)c0, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) dst[c0 + i] = (ok && stage > 0) ? v[i] : 0.0f;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// dw[tap][co][ci] = sum over chunks in order of part[chunk][tile][r][co], r = tap * cin + ci - 128 * tile.
__global__ void k_wgrad_reduce(const float* part, int chunks, int mtiles, int cin, int cout, float* dw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over 9 * cout * cin
    if (i >= 9 * cout * cin) return;
    const int tap = i / (cout * cin), rem = i - tap * cout * cin, co = rem / cin, ci = rem - co * cin;
    const int r = tap * cin + ci, tile = r >> 7, row = r & 127;
    float s = 0.0f;
    for (int c = 0; c < chunks; ++c) s += part[(((size_t)c * mtiles + tile) * 128 + row) * cout + co];
    dw[i] = s;
}

// db[co] = sum over pixels of dy[p][co]: per block of pix_per_block pixels,
// thread t sums channel t % cout over pixels t / cout, t / cout + 256 / cout,
// ... in order; the groups are then added in order (deterministic).
__global__ void __launch_bounds__(256) k_bgrad_partial(const bf16* dy, int npix, int cout, int pix_per_block,
                                                       float* part) {
    __shared__ float red[256];
    const int t = threadIdx.x, groups = 256 / cout, c = t % cout, g = t / cout;
    const int p0 = blockIdx.x * pix_per_block, p1 = min(npix, p0 + pix_per_block);
    float s = 0.0f;
    if (g < groups)
        for (int p = p0 + g; p < p1; p += groups) s += __bfloat162float(dy[(size_t)p * cout + c]);
    red[t] = s;
    __syncthreads();
    if (t < cout) {
        float tot = 0.0f;
        for (int q = 0; q < groups; ++q) tot += red[q * cout + t];
        part[(size_t)blockIdx.x * cout + t] = tot;
    }
}
__global__ void k_bgrad_reduce(const float* part, int blocks, int cout, float* db) {
    const int co = threadIdx.x;
    if (co >= cout) return;
    float s = 0.0f;
    for (int b = 0; b < blocks; ++b) s += part[(size_t)b * cout + co];
    db[co] = s;
}

// ---------------------------------------------------------------------------
// Elementwise parts of the network.

// The resampling kernels move 8 bf16 (or 4 fp32) channels per thread; every
// channel count, tensor stride and slice offset is a multiple of 8, so the
// 16-byte accesses are aligned.  Per-element arithmetic is the scalar form's.

// out[Y, X] = the mean of in's 2x2 block (in is a channel slice), summed as
// ((a + b) + c) + d in fp32.
__global__ void k_pool2(const bf16* in, int is, int io, int H, int W, int C, bf16* out) {
    const int h = H / 2, w = W / 2, g8 = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over h * w * C / 8
    if (i >= h * w * g8) return;
    const int g = i % g8, q = i / g8, Y = q / w, X = q - Y * w;
    auto at = [&](int y, int x) { return *reinterpret_cast<const uint4*>(in + (size_t)(y * W + x) * is + io + 8 * g); };
    const uint4 va = at(2 * Y, 2 * X), vb = at(2 * Y, 2 * X + 1), vc = at(2 * Y + 1, 2 * X), vd = at(2 * Y + 1, 2 * X + 1);
    const bf16 *a = reinterpret_cast<const bf16*>(&va), *b = reinterpret_cast<const bf16*>(&vb),
               *c = reinterpret_cast<const bf16*>(&vc), *d = reinterpret_cast<const bf16*>(&vd);
    __align__(16) bf16 o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float s = ((__bfloat162float(a[k]) + __bfloat162float(b[k])) + __bfloat162float(c[k])) + __bfloat162float(d[k]);
        o[k] = __float2bfloat16_rn(0.25f * s);
    }
    *reinterpret_cast<uint4*>(out + (size_t)q * C + 8 * g) = *reinterpret_cast<const uint4*>(o);
}
// g_in[2Y+i, 2X+j] += g_out[Y, X] / 4 (fp32 gradients; g_in is a channel slice).
__global__ void k_pool2_bwd(const float* gout, int H, int W, int C, float* gin, int gs, int go) {
    const int g4 = C / 4;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over H * W * C / 4
    if (i >= H * W * g4) return;
    const int g = i % g4, q = i / g4, y = q / W, x = q - y * W;
    const float4 v = *reinterpret_cast<const float4*>(gout + (size_t)((y >> 1) * (W / 2) + (x >> 1)) * C + 4 * g);
    float4* dst = reinterpret_cast<float4*>(gin + (size_t)q * gs + go + 4 * g);
    float4 t = *dst;
    t.x += 0.25f * v.x;
    t.y += 0.25f * v.y;
    t.z += 0.25f * v.z;
    t.w += 0.25f * v.w;
    *dst = t;
}
// out slice [y, x] = in[y / 2, x / 2] (nearest upsampling into a channel slice).
__global__ void k_up2(const bf16* in, int H, int W, int C, bf16* out, int os, int oo) {
    const int g8 = C / 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over H * W * C / 8
    if (i >= H * W * g8) return;
    const int g = i % g8, q = i / g8, y = q / W, x = q - y * W;
    *reinterpret_cast<uint4*>(out + (size_t)q * os + oo + 8 * g) =
        *reinterpret_cast<const uint4*>(in + (size_t)((y >> 1) * (W / 2) + (x >> 1)) * C + 8 * g);
}
// g_in[Y, X] = sum of the 2x2 block of g_out's channel slice, ((a + b) + c) + d.
__global__ void k_up2_bwd(const float* gout, int gs, int go, int H, int W, int C, float* gin) {
    const int h = H / 2, w = W / 2, g4 = C / 4;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over h * w * C / 4
    if (i >= h * w * g4) return;
    const int g = i % g4, q = i / g4, Y = q / w, X = q - Y * w;
    auto at = [&](int y, int x) { return *reinterpret_cast<const float4*>(gout + (size_t)(y * W + x) * gs + go + 4 * g); };
    const float4 a = at(2 * Y, 2 * X), b = at(2 * Y, 2 * X + 1), c = at(2 * Y + 1, 2 * X), d = at(2 * Y + 1, 2 * X + 1);
    *reinterpret_cast<float4*>(gin + (size_t)q * C + 4 * g) =
        make_float4(((a.x + b.x) + c.x) + d.x, ((a.y + b.y) + c.y) + d.y, ((a.z + b.z) + c.z) + d.z,
                    ((a.w + b.w) + c.w) + d.w);
}
// dy = bf16(g) where the forward output y > 0 (relu) or everywhere (relu = 0).
__global__ void k_relu_bwd(const float* g, int gs, int go, const bf16* y, int ys, int yo, int npix, int C, int relu,
                           bf16* dy) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)npix * C) return;
    const int c = (int)(i % C);
    const size_t p = i / C;
    float v = g[p * gs + go + c];
    if (relu && !(__bfloat162float(y[p * ys + yo + c]) > 0.0f)) v = 0.0f;
    dy[i] = __float2bfloat16_rn(v);
}
// BF16 weight tiles of the convolutions, each tap's cout x cin tile in the
// K-major order the tensor cores read (so a CTA fetches it with one bulk
// copy), and those of the backward pass over the data:
// wt[tap'][ci][co] = w[8 - tap'][co][ci].
__global__ void k_flip_transpose(const float* w32, int cin, int cout, bf16* w16, bf16* wt16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * cin * cout) return;
    const int tap = i / (cout * cin), rem = i - tap * cout * cin, co = rem / cin, ci = rem - co * cin;
    const bf16 v = __float2bfloat16_rn(w32[i]);
    w16[(size_t)tap * cout * cin + kmajor_index(co, ci, cin)] = v;
    wt16[(size_t)(8 - tap) * cin * cout + kmajor_index(ci, co, cout)] = v;
}
// Per-block sums of g^2 (1024 elements per block), for the global-norm clip.
__global__ void __launch_bounds__(256) k_sumsq(const float* g, int n, float* part) {
    float s = 0.0f;
    const int i0 = blockIdx.x * 1024;
    for (int i = i0 + threadIdx.x; i < min(n, i0 + 1024); i += 256) s += g[i] * g[i];
    s = warp_sum_f(s);
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < 8; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}
// Adam on fp32 master parameters; the gradient is scaled by gscale first
// (global-norm clipping).
__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2, float gscale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace efl

namespace efl {

// ---------------------------------------------------------------------------
// Features of one pressure system and the warm start.
//
// The start iterate p_prev (the previous step's pressure) leaves the residual
// r = b - A p_prev on the new system; the exact correction e = A^-1 r is what
// the network approximates.  Both are scaled by sigma, the RMS of cdiv * r
// over the counted cells (cdiv * r is in pressure units), so the map is
// scale-free.  Channels (16, zero beyond 5): 0 = cdiv * r / sigma, 1 / 2 =
// the u / v face fractions averaged to the cell centre, 3 = phi / ny clamped
// to [-1, 1], 4 = 1 on the counted cells; output channel 0 = e / sigma.

struct UnetFeatureArgs {
    PF ls, fu, fv;
    Plane<double> prev, b;  // the solve's start iterate and right-hand side
    double cdiv, factor;    // dx^2 rho / dt, dt / (rho dx^2)
    int nx, ny;
};
// res[p] = cdiv * (b - A prev) on the counted cells (the operator of
// residual.wgsl:33-54 in factored form, as the mixed solve builds it), the
// mask, prev32 = prev, and per-block partial sums (res^2, count).
// (Block (bx, by) of a grid bgx blocks wide; a batch's launch covers several simulations' grids.)
// The in-order sums of a block's reductions: thread t adds partials t, t + 256, ... in turn, then a fixed tree
// over the 256 threads (blocks of 256 threads; the same order for a simulation alone and in a batch).
constexpr int UNET_RED_THREADS = 256;
EFL_DEV double2 block_sum2(double a, double b, int t) {
    __shared__ double2 red[UNET_RED_THREADS];
    red[t] = make_double2(a, b);
    __syncthreads();
#pragma unroll
    for (int o = UNET_RED_THREADS / 2; o > 0; o >>= 1) {
        if (t < o) red[t] = make_double2(red[t].x + red[t + o].x, red[t].y + red[t + o].y);
        __syncthreads();
    }
    return red[0];
}
// sigma = RMS of the residual over the counted cells (1 if there are none); t = the linear thread index of a
// block of UNET_RED_THREADS threads.  The partials are read through L2 (other blocks of the same launch may
// have written them).
EFL_DEV void unet_sigma_blk(const float2* part, int n, float* sigma, int t) {
    double r2 = 0.0, c = 0.0;
    for (int i = t; i < n; i += UNET_RED_THREADS) {
        const float2 q = __ldcg(part + i);
        r2 += q.x;
        c += q.y;
    }
    const double2 s2 = block_sum2(r2, c, t);
    if (t == 0) {
        const double v = s2.y > 0.0 ? sqrt(s2.x / s2.y) : 0.0;
        *sigma = v > 0.0 ? (float)v : 1.0f;
    }
}
// The sum of the squares of the four 8 x 8 guard-block sums of v over a block of 32 x 8 threads (the 8 cells of a
// row by shuffles, then the 8 rows in order), returned by thread 0; every thread of the block calls it.
EFL_DEV double guard_block_squares(double v) {
    __shared__ double rsum[8][4];
    for (int o = 1; o < 8; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 7) == 0) rsum[threadIdx.y][threadIdx.x >> 3] = v;
    __syncthreads();
    double acc = 0.0;
    if (threadIdx.x == 0 && threadIdx.y == 0)
        for (int k = 0; k < 4; ++k) {
            double sp = 0.0;
            for (int r = 0; r < 8; ++r) sp += rsum[r][k];
            acc += sp * sp;
        }
    return acc;
}
// With epart (the coarse warm start; blocks of 32 x 8 threads), also the guard's "before" half: the squared
// 8 x 8 block sums of the start iterate's unscaled residual, into epart[block].x.  With p32 / d32 (the f32
// pressure and divergence), the cells are widened here into a.prev and a.b, the solve's FP64 start iterate and
// right-hand side (neighbours read from the f32 planes: the same values).  With count (zero between launches),
// the block that finishes last sums the partials into sigma (in the fixed order of unet_sigma_blk).
__global__ void __launch_bounds__(256) k_unet_residual(UnetFeatureArgs a, float* res, float* prev32, unsigned char* mask,
                                                        float2* part, double2* epart, PF p32, PF d32, unsigned* count,
                                                        float* sigma) {
    const int bx = blockIdx.x, by = blockIdx.y, bgx = gridDim.x;
    const bool wide = p32.p != nullptr;
    auto X = [&](int x, int y) -> double { return wide ? (double)p32.at(x, y) : a.prev.at(x, y); };
    const int gx = bx * blockDim.x + threadIdx.x, gy = by * blockDim.y + threadIdx.y;
    float r2 = 0.0f, c = 0.0f;
    double rd = 0.0;
    if (gx < a.nx && gy < a.ny) {
        const size_t p = (size_t)gy * a.nx + gx;
        const double xc = X(gx, gy), bc = wide ? (double)d32.at(gx, gy) : a.b.at(gx, gy);
        if (wide) {
            a.prev.at(gx, gy) = xc;
            a.b.at(gx, gy) = bc;
        }
        const float phi = a.ls.at(gx, gy);
        const float f[4] = {a.fu.at(gx, gy), a.fu.at(gx + 1, gy), a.fv.at(gx, gy), a.fv.at(gx, gy + 1)};
        const bool counted = phi < 0.0f && !(f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f);
        float rv = 0.0f;
        if (counted) {
            const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
            double den = 0.0, sum = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int jx = gx + ox[q], jy = gy + oy[q];
                if ((unsigned)jx < (unsigned)a.nx && (unsigned)jy < (unsigned)a.ny) {
                    const float level = a.ls.at(jx, jy);
                    if (level < 0.0f) {
                        den += (double)f[q];
                        sum += (double)f[q] * X(jx, jy);
                    } else {
                        den += (double)f[q] * (1.0 - (double)level / (double)phi);
                    }
                }
            }
            rd = bc - a.factor * (den * xc - sum);
            rv = (float)(a.cdiv * rd);
            r2 = rv * rv;
            c = 1.0f;
        }
        res[p] = rv;
        prev32[p] = (float)xc;
        mask[p] = counted ? 1 : 0;
    }
    r2 = warp_sum_f(r2);
    c = warp_sum_f(c);
    __shared__ float2 red[8];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if ((t & 31) == 0) red[t >> 5] = make_float2(r2, c);
    __syncthreads();
    if (t == 0) {
        float2 s2 = make_float2(0.0f, 0.0f);
        for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) {
            s2.x += red[w].x;
            s2.y += red[w].y;
        }
        part[by * bgx + bx] = s2;
    }
    if (epart) {
        const double sq = guard_block_squares(rd);
        if (t == 0) epart[by * bgx + bx].x = sq;
    }
    if (count) {
        __shared__ unsigned s_last;
        const unsigned nblk = gridDim.x * gridDim.y;
        if (t == 0) {
            __threadfence();  // this block's partial before its arrival
            s_last = atomicAdd(count, 1u) == nblk - 1 ? 1u : 0u;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            unet_sigma_blk(part, (int)nblk, sigma, t);
            if (t == 0) *count = 0u;  // for the next launch
        }
    }
}

__global__ void k_unet_features(const float* res, const UnetFeatureArgs a, const unsigned char* mask,
                                const float* sigma, bf16* x0) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= a.nx || gy >= a.ny) return;
    const size_t p = (size_t)gy * a.nx + gx;
    const float inv = 1.0f / *sigma;
    __align__(16) bf16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16_rn(0.0f);
    v[0] = __float2bfloat16_rn(res[p] * inv);
    v[1] = __float2bfloat16_rn(0.5f * (a.fu.at(gx, gy) + a.fu.at(gx + 1, gy)));
    v[2] = __float2bfloat16_rn(0.5f * (a.fv.at(gx, gy) + a.fv.at(gx, gy + 1)));
    v[3] = __float2bfloat16_rn(fminf(1.0f, fmaxf(-1.0f, a.ls.at(gx, gy) / (float)a.ny)));
    v[4] = __float2bfloat16_rn(mask[p] ? 1.0f : 0.0f);
    uint4* dst = reinterpret_cast<uint4*>(x0 + p * 16);
    dst[0] = reinterpret_cast<const uint4*>(v)[0];
    dst[1] = reinterpret_cast<const uint4*>(v)[1];
}
// x += sigma * prediction on the masked cells (the solve's start iterate).
__global__ void k_unet_warm(Plane<double> x, const float* out16, const unsigned char* mask, const float* sigma, int nx,
                            int ny) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny) return;
    const size_t p = (size_t)gy * nx + gx;
    if (mask[p]) x.at(gx, gy) = x.at(gx, gy) + (double)*sigma * (double)out16[p * 16];
}
// Training target after the solve: (p - p_prev) / sigma.
__global__ void k_unet_target(Plane<double> x, const float* prev32, const float* sigma, int nx, int ny,
                              float* target) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny) return;
    const size_t p = (size_t)gy * nx + gx;
    target[p] = (float)((x.at(gx, gy) - (double)prev32[p]) / (double)*sigma);
}
// The warm start's guard.  The sweeps remove smooth error slowest, and a
// residual norm hardly sees it (A damps smooth modes), so a prediction can
// lower ||r|| and still add the error that costs the iterations.  Summed
// over g x g blocks, the residual of smooth error adds up while the
// fine-scale part cancels, so the guard compares the norms of the block sums
// of r before and after the warm start and keeps the warm start only if it
// made them smaller.  One thread per block; .x = (sum of r over the block)^2
// for the start iterate p (= prev32) and .y for the warm-started x, per
// 32 x 8 group of blocks.
// xv(x, y) is the warm-started iterate at a cell (read from the plane, or formed on the fly).
template <class XV>
EFL_DEV void unet_block_residual_blk(const UnetFeatureArgs& a, const float* prev32, int g, double2* part, int bx, int by,
                                     int bgx, XV xv) {
    const int cx = bx * blockDim.x + threadIdx.x, cy = by * blockDim.y + threadIdx.y;
    const int Wc = (a.nx + g - 1) / g, Hc = (a.ny + g - 1) / g;
    double sp = 0.0, sx = 0.0;
    if (cx < Wc && cy < Hc) {
        for (int j = 0; j < g; ++j)
            for (int i = 0; i < g; ++i) {
                const int gx = cx * g + i, gy = cy * g + j;
                if (gx >= a.nx || gy >= a.ny) continue;
                const float phi = a.ls.at(gx, gy);
                const float f[4] = {a.fu.at(gx, gy), a.fu.at(gx + 1, gy), a.fv.at(gx, gy), a.fv.at(gx, gy + 1)};
                if (!(phi < 0.0f) || (f[0] == 0.0f && f[1] == 0.0f && f[2] == 0.0f && f[3] == 0.0f)) continue;
                const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
                double den = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int jx = gx + ox[q], jy = gy + oy[q];
                    if ((unsigned)jx < (unsigned)a.nx && (unsigned)jy < (unsigned)a.ny) {
                        const float level = a.ls.at(jx, jy);
                        if (level < 0.0f) {
                            den += (double)f[q];
                            s1 += (double)f[q] * (double)prev32[(size_t)jy * a.nx + jx];
                            s2 += (double)f[q] * xv(jx, jy);
                        } else {
                            den += (double)f[q] * (1.0 - (double)level / (double)phi);
                        }
                    }
                }
                const double bb = a.b.at(gx, gy);
                sp += bb - a.factor * (den * (double)prev32[(size_t)gy * a.nx + gx] - s1);
                sx += bb - a.factor * (den * xv(gx, gy) - s2);
            }
    }
    double vp = sp * sp, vx = sx * sx;
    vp = warp_sum(vp);
    vx = warp_sum(vx);
    __shared__ double red_p[8], red_x[8];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    if ((t & 31) == 0) {
        red_p[t >> 5] = vp;
        red_x[t >> 5] = vx;
    }
    __syncthreads();
    if (t == 0) {
        double a1 = 0.0, a2 = 0.0;
        for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) {
            a1 += red_p[w];
            a2 += red_x[w];
        }
        part[by * bgx + bx] = make_double2(a1, a2);
    }
}
__global__ void __launch_bounds__(256) k_unet_block_residual(UnetFeatureArgs a, const float* prev32, int g,
                                                             double2* part) {
    unet_block_residual_blk(a, prev32, g, part, blockIdx.x, blockIdx.y, gridDim.x,
                            [&](int x, int y) { return a.prev.at(x, y); });
}
// keep (*alpha = 1) or drop (*alpha = 0) the warm start, from the block-residual partials.
EFL_DEV void unet_guard_blk(const double2* part, int n, double* alpha) {
    double before = 0.0, after = 0.0;
    for (int i = threadIdx.x; i < n; i += UNET_RED_THREADS) {
        before += part[i].x;
        after += part[i].y;
    }
    const double2 s2 = block_sum2(before, after, threadIdx.x);
    if (threadIdx.x == 0) *alpha = s2.y < s2.x ? 1.0 : 0.0;
}
__global__ void __launch_bounds__(UNET_RED_THREADS) k_unet_guard(const double2* part, int n, double* alpha) {
    unet_guard_blk(part, n, alpha);
}
// Where the guard dropped it, the start iterate p (= prev32, exactly: it is the f32 pressure widened) back on
// the counted cells.
__global__ void k_unet_guard_restore(Plane<double> x, const float* prev32, const unsigned char* mask,
                                     const double* alpha, int nx, int ny) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny || *alpha != 0.0) return;
    const size_t p = (size_t)gy * nx + gx;
    if (mask[p]) x.at(gx, gy) = (double)prev32[p];
}

// Coarse form of the warm start.  The red-black sweeps remove the
// basin-scale part of the error slowest (hundreds of iterations per e-fold at
// 512^2), and that part is smooth: the network therefore runs on the grid
// coarsened by f (one coarse cell per f x f cells), where four levels of
// pooling span the whole domain, and its output is interpolated back
// bilinearly; the sweeps then remove the fine-scale remainder quickly.
// Coarse features: the mean over the block of each fine channel; maskc = 1
// where the block holds a counted cell.
// x0 holds row cy of the coarse features at x0 + cy * cs * 16 (cs = the coarse width, or the row pitch of
// the canvas that packs a batch's simulations side by side).
// One thread per fine cell, blocks of 32 x 8 threads: a block's cells hold (32 / f) x (8 / f) coarse cells
// (f = 2, 4 or 8; the grid a multiple of 8 f).  A coarse cell's sums run over the f cells of each row by
// shuffles, then over its f rows in order.
EFL_DEV void unet_features_coarse_blk(const float* res, const UnetFeatureArgs& a, const unsigned char* mask,
                                      const float* sigma, int f, bf16* x0, int cs, unsigned char* maskc, int bx, int by) {
    __shared__ float rows[8][32][5];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int gx = bx * 32 + tx, gy = by * 8 + ty;
    const float inv = 1.0f / *sigma;
    float v[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (gx < a.nx && gy < a.ny) {
        const size_t p = (size_t)gy * a.nx + gx;
        v[0] = res[p] * inv;
        v[1] = 0.5f * (a.fu.at(gx, gy) + a.fu.at(gx + 1, gy));
        v[2] = 0.5f * (a.fv.at(gx, gy) + a.fv.at(gx, gy + 1));
        v[3] = fminf(1.0f, fmaxf(-1.0f, a.ls.at(gx, gy) / (float)a.ny));
        v[4] = mask[p] ? 1.0f : 0.0f;
    }
    for (int o = 1; o < f; o <<= 1)
#pragma unroll
        for (int c = 0; c < 5; ++c) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
    if (tx % f == 0)
#pragma unroll
        for (int c = 0; c < 5; ++c) rows[ty][tx][c] = v[c];
    __syncthreads();
    const int Wc = a.nx / f, Hc = a.ny / f, cx = gx / f, cy = gy / f;
    if (tx % f != 0 || ty % f != 0 || cx >= Wc || cy >= Hc) return;
    float acc[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        acc[c] = rows[ty][tx][c];
        for (int r = 1; r < f; ++r) acc[c] += rows[ty + r][tx][c];
    }
    const float nrm = 1.0f / (float)(f * f);
    __align__(16) bf16 o16[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) o16[c] = __float2bfloat16_rn(c < 5 ? acc[c] * nrm : 0.0f);
    uint4* dst = reinterpret_cast<uint4*>(x0 + ((size_t)cy * cs + cx) * 16);
    dst[0] = reinterpret_cast<const uint4*>(o16)[0];
    dst[1] = reinterpret_cast<const uint4*>(o16)[1];
    maskc[(size_t)cy * Wc + cx] = acc[4] > 0.0f ? 1 : 0;
}
__global__ void k_unet_features_coarse(const float* res, const UnetFeatureArgs a, const unsigned char* mask,
                                       const float* sigma, int f, bf16* x0, int cs, unsigned char* maskc) {
    unet_features_coarse_blk(res, a, mask, sigma, f, x0, cs, maskc, blockIdx.x, blockIdx.y);
}
// The coarse prediction at fine cell (gx, gy), interpolated bilinearly: coarse cell (i, j) is centred on fine
// coordinate ((i + 1/2) f - 1/2, ...), clamped at the edges; row j of the prediction at outc + j * cs * 16.
EFL_DEV float unet_coarse_pred(const float* outc, int cs, int nx, int ny, int f, int gx, int gy) {
    const int Wc = nx / f, Hc = ny / f;
    const float u = ((float)gx + 0.5f) / (float)f - 0.5f, v = ((float)gy + 0.5f) / (float)f - 0.5f;
    int i0 = (int)floorf(u), j0 = (int)floorf(v);
    float tu = u - (float)i0, tv = v - (float)j0;
    if (i0 < 0) i0 = 0, tu = 0.0f;
    if (i0 >= Wc - 1) i0 = Wc - 1, tu = 0.0f;
    if (j0 < 0) j0 = 0, tv = 0.0f;
    if (j0 >= Hc - 1) j0 = Hc - 1, tv = 0.0f;
    const int i1 = min(i0 + 1, Wc - 1), j1 = min(j0 + 1, Hc - 1);
    const float o00 = outc[((size_t)j0 * cs + i0) * 16], o10 = outc[((size_t)j0 * cs + i1) * 16];
    const float o01 = outc[((size_t)j1 * cs + i0) * 16], o11 = outc[((size_t)j1 * cs + i1) * 16];
    // explicit roundings: the guard's on-the-fly value and the applied one agree in every kernel they inline into
    const float su = __fsub_rn(1.0f, tu), sv = __fsub_rn(1.0f, tv);
    const float top = __fadd_rn(__fmul_rn(o00, su), __fmul_rn(o10, tu));
    const float bot = __fadd_rn(__fmul_rn(o01, su), __fmul_rn(o11, tu));
    return __fadd_rn(__fmul_rn(top, sv), __fmul_rn(bot, tv));
}
// The warm-started iterate at (gx, gy): x + sigma * prediction on the counted cells, x elsewhere.
EFL_DEV double unet_warm_value(const Plane<double>& x, const float* outc, int cs, const unsigned char* mask,
                               float sigma, int nx, int ny, int f, int gx, int gy) {
    const double v = x.at(gx, gy);
    return mask[(size_t)gy * nx + gx]
               ? __dadd_rn(v, __dmul_rn((double)sigma, (double)unet_coarse_pred(outc, cs, nx, ny, f, gx, gy)))
               : v;
}
// The guard's "after" half for the coarse warm start, one thread per fine cell (blocks of 32 x 8 threads): the
// residual of the warm-started iterate, formed on the fly from the coarse prediction (x is still the start
// iterate) with a one-cell halo in shared memory, summed over the 8 x 8 guard blocks and squared, into
// part[block].y (the residual kernel wrote the start iterate's half into .x, in the same order).
EFL_DEV void unet_guard_residual_blk(const UnetFeatureArgs& a, const unsigned char* mask, const float* outc, int cs,
                                     const float* sigma, int f, double2* part, int bx, int by, int bgx) {
    __shared__ double wv[10][34];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int X0 = bx * 32 - 1, Y0 = by * 8 - 1;
    const float sg = *sigma;
    for (int i = tid; i < 340; i += 256) {
        const int ly = i / 34, lx = i - ly * 34, hx = X0 + lx, hy = Y0 + ly;
        const bool in = (unsigned)hx < (unsigned)a.nx && (unsigned)hy < (unsigned)a.ny;
        wv[ly][lx] = in ? unet_warm_value(a.prev, outc, cs, mask, sg, a.nx, a.ny, f, hx, hy) : 0.0;
    }
    __syncthreads();
    const int gx = bx * 32 + tx, gy = by * 8 + ty;
    double rx = 0.0;
    if (gx < a.nx && gy < a.ny) {
        const float phi = a.ls.at(gx, gy);
        const float fq[4] = {a.fu.at(gx, gy), a.fu.at(gx + 1, gy), a.fv.at(gx, gy), a.fv.at(gx, gy + 1)};
        if (phi < 0.0f && !(fq[0] == 0.0f && fq[1] == 0.0f && fq[2] == 0.0f && fq[3] == 0.0f)) {
            const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
            double den = 0.0, s2 = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int jx = gx + ox[q], jy = gy + oy[q];
                if ((unsigned)jx < (unsigned)a.nx && (unsigned)jy < (unsigned)a.ny) {
                    const float level = a.ls.at(jx, jy);
                    if (level < 0.0f) {
                        den += (double)fq[q];
                        s2 += (double)fq[q] * wv[ty + 1 + oy[q]][tx + 1 + ox[q]];
                    } else {
                        den += (double)fq[q] * (1.0 - (double)level / (double)phi);
                    }
                }
            }
            rx = a.b.at(gx, gy) - a.factor * (den * wv[ty + 1][tx + 1] - s2);
        }
    }
    const double sq = guard_block_squares(rx);
    if (tid == 0) part[by * bgx + bx].y = sq;
}
__global__ void __launch_bounds__(256) k_unet_guard_residual(UnetFeatureArgs a, const unsigned char* mask,
                                                             const float* outc, int cs, const float* sigma, int f,
                                                             double2* part) {
    unet_guard_residual_blk(a, mask, outc, cs, sigma, f, part, blockIdx.x, blockIdx.y, gridDim.x);
}
// Where the guard kept it (*alpha != 0), the coarse warm start written into the iterate.
EFL_DEV void unet_apply_warm_blk(const Plane<double>& x, const float* outc, int cs, const unsigned char* mask,
                                 const float* sigma, const double* alpha, int nx, int ny, int f, int bx, int by) {
    const int gx = bx * blockDim.x + threadIdx.x, gy = by * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny || *alpha == 0.0) return;
    x.at(gx, gy) = unet_warm_value(x, outc, cs, mask, *sigma, nx, ny, f, gx, gy);
}
__global__ void k_unet_apply_warm(Plane<double> x, const float* outc, int cs, const unsigned char* mask,
                                  const float* sigma, const double* alpha, int nx, int ny, int f) {
    unet_apply_warm_blk(x, outc, cs, mask, sigma, alpha, nx, ny, f, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// A batch's coarse warm start after the canvas forward pass: the guard and the prediction's application, one
// launch per phase for all the simulations on the canvas.  Simulation i's blocks in a launch are start[i] ..
// start[i + 1] - 1, numbered row-major over its own grid of 32 x 8 blocks as its own launches number them, so
// that every per-block partial, and its place in the in-order sums, is the same as in its own warm start.
struct WarmSim {
    UnetFeatureArgs a;
    float* sigma;
    unsigned char* mask;
    double2* epart;     // the guard's partials, one per thread block, its decision after them
    const float* outc;  // the simulation's prediction on the canvas (row pitch cs coarse pixels)
    int cs, f;          // canvas pitch, coarsening
    int fgx, fgy;       // the simulation's grid of 32 x 8 thread blocks
};
// The simulation whose block range holds block b (start[0] = 0 <= b < start[n]).
EFL_DEV int warm_sim_of(const int* start, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}
// The phases after the forward pass, one thread per fine cell: simulation i owns blocks start[i] .. start[i + 1] - 1.
__global__ void __launch_bounds__(256) k_warm_batch_guard_residual(const WarmSim* S, const int* start, int n) {
    const int i = warm_sim_of(start, n, blockIdx.x), t = blockIdx.x - start[i];
    const WarmSim w = S[i];
    unet_guard_residual_blk(w.a, w.mask, w.outc, w.cs, w.sigma, w.f, w.epart, t % w.fgx, t / w.fgx, w.fgx);
}
__global__ void __launch_bounds__(UNET_RED_THREADS) k_warm_batch_guard(const WarmSim* S) {
    const WarmSim w = S[blockIdx.x];
    const int nb = w.fgx * w.fgy;
    unet_guard_blk(w.epart, nb, (double*)(w.epart + nb));
}
__global__ void __launch_bounds__(256) k_warm_batch_apply(const WarmSim* S, const int* start, int n) {
    const int i = warm_sim_of(start, n, blockIdx.x), t = blockIdx.x - start[i];
    const WarmSim w = S[i];
    const int nb = w.fgx * w.fgy;
    unet_apply_warm_blk(w.a.prev, w.outc, w.cs, w.mask, w.sigma, (const double*)(w.epart + nb), w.a.nx, w.a.ny, w.f,
                        t % w.fgx, t / w.fgx);
}

// Coarse training target: the mean of (p - p_prev) / sigma over the block's counted cells (0 if none).
__global__ void k_unet_target_coarse(Plane<double> x, const float* prev32, const unsigned char* mask,
                                     const float* sigma, int nx, int ny, int f, float* targetc) {
    const int Wc = nx / f, Hc = ny / f;
    const int cx = blockIdx.x * blockDim.x + threadIdx.x, cy = blockIdx.y * blockDim.y + threadIdx.y;
    if (cx >= Wc || cy >= Hc) return;
    double acc = 0.0;
    int cnt = 0;
    for (int j = 0; j < f; ++j)
        for (int i = 0; i < f; ++i) {
            const int gx = cx * f + i, gy = cy * f + j;
            const size_t p = (size_t)gy * nx + gx;
            if (mask[p]) {
                acc += x.at(gx, gy) - (double)prev32[p];
                ++cnt;
            }
        }
    targetc[(size_t)cy * Wc + cx] = cnt ? (float)(acc / cnt / (double)*sigma) : 0.0f;
}
// Relative squared error of one sample, sum_mask (pred - t)^2 / sum_mask t^2:
// g_out[p][0] = 2 (pred - t) * inv_norm (inv_norm = 1 / sum_mask t^2), and
// per-block partial sums of (pred - t)^2.
__global__ void k_unet_loss(const float* out16, const float* target, const unsigned char* mask, int npix,
                            int pix_per_block, float inv_norm, float* g_out16, float2* part) {
    float se = 0.0f;
    const int p0 = blockIdx.x * pix_per_block;
    for (int i = threadIdx.x; i < pix_per_block; i += blockDim.x) {
        const int p = p0 + i;
        if (p >= npix) break;
        float g = 0.0f;
        if (mask[p]) {
            const float d = out16[(size_t)p * 16] - target[p];
            se += d * d;
            g = 2.0f * d * inv_norm;
        }
        float* gp = g_out16 + (size_t)p * 16;
        gp[0] = g;
#pragma unroll
        for (int c = 1; c < 16; ++c) gp[c] = 0.0f;
    }
    se = warp_sum_f(se);
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = se;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        part[blockIdx.x] = make_float2(t, 0.0f);
    }
}
// Per-block partial sums of (count, t^2) over the masked cells.
__global__ void k_target_stats(const float* target, const unsigned char* mask, int npix, int pix_per_block,
                               float2* part) {
    float c = 0.0f, t2 = 0.0f;
    const int p0 = blockIdx.x * pix_per_block;
    for (int i = threadIdx.x; i < pix_per_block; i += blockDim.x) {
        const int p = p0 + i;
        if (p >= npix) break;
        if (mask[p]) {
            c += 1.0f;
            t2 += target[p] * target[p];
        }
    }
    c = warp_sum_f(c);
    t2 = warp_sum_f(t2);
    __shared__ float2 red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_float2(c, t2);
    __syncthreads();
    if (threadIdx.x == 0) {
        float2 t = make_float2(0.0f, 0.0f);
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t.x += red[w].x;
            t.y += red[w].y;
        }
        part[blockIdx.x] = t;
    }
}

// ---------------------------------------------------------------------------
// The network: 4 levels, channels 16/32/64/64, two 3x3 convolutions + ReLU
// per level, 2x2 average pooling down, nearest upsampling and concatenation
// up, a linear 3x3 head (16 outputs, channel 0 used).

struct UConvSpec {
    int cin, cout, relu;
};
constexpr int UNET_NCONV = 15;
constexpr UConvSpec kUnetSpec[UNET_NCONV] = {
    {16, 16, 1}, {16, 16, 1},   // level 0
    {16, 32, 1}, {32, 32, 1},   // level 1
    {32, 64, 1}, {64, 64, 1},   // level 2
    {64, 64, 1}, {64, 64, 1},   // level 3 (bottleneck)
    {128, 64, 1}, {64, 64, 1},  // up to level 2 (64 up + 64 skip)
    {96, 32, 1}, {32, 32, 1},   // up to level 1 (64 up + 32 skip)
    {48, 16, 1}, {16, 16, 1},   // up to level 0 (32 up + 16 skip)
    {16, 16, 0},                // head
};
// Every convolution (forward, and backward over the data with cin and cout
// swapped) fits one CTA's shared memory.
constexpr bool unet_convs_fit() {
    for (int i = 0; i < UNET_NCONV; ++i)
        if (conv_smem_bytes(kUnetSpec[i].cin, kUnetSpec[i].cout) > CV_SMEM ||
            conv_smem_bytes(kUnetSpec[i].cout, kUnetSpec[i].cin) > CV_SMEM ||
            crow_smem_bytes(kUnetSpec[i].cin, kUnetSpec[i].cout, false, 1) > CV_SMEM ||
            crow_smem_bytes(kUnetSpec[i].cout, kUnetSpec[i].cin, false, 1) > CV_SMEM)
            return false;
    return true;
}
static_assert(unet_convs_fit(), "a U-Net convolution exceeds the shared-memory budget");

struct UNet {
    int device = 0, maxH = 0, maxW = 0;
    size_t woff[UNET_NCONV], boff[UNET_NCONV], nparams = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    bf16 *w16[UNET_NCONV], *wt16[UNET_NCONV];
    int adam_t = 0;
    // activations (bf16), sized for maxH x maxW
    bf16 *X0, *t0, *cat0, *p1, *t1, *cat1, *p2, *t2, *cat2, *p3, *t3, *u3, *t4, *u4, *t5, *u5, *t6, *u6;
    float* out;  // [H*W][16] fp32 head output
    // gradients (fp32)
    float *g_out, *g_u6, *g_t6, *g_cat0, *g_u5, *g_t5, *g_cat1, *g_u4, *g_t4, *g_cat2, *g_u3, *g_t3, *g_p3, *g_t2,
        *g_p2, *g_t1, *g_p1, *g_t0;
    bf16* dym;
    float *wpart, *bpart;
    size_t wpart_elems = 0;
    float2* lpart;
    float *target, *prev32, *res32, *sigma;
    double2* epart;  // the warm start guard's partials (one per 32 x 8 group of blocks) and its decision after them
    unsigned char* mask;
    int coarse = 1;          // the grid coarsening factor f of the warm start (1, 2, 4 or 8)
    float* targetc;          // coarse training target and mask (coarse form)
    unsigned char* maskc;
    int* err;
    unsigned* red_count;  // arrivals of k_unet_residual's blocks (its last block computes sigma); zero between launches
    void* arena = nullptr;
    std::vector<void*> extra;
    std::string last_error;
};

inline size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// One allocation for everything: parameters, Adam moments, bf16 weights,
// activations and gradients for maxH x maxW.
inline cudaError_t unet_alloc(UNet& n, int maxH, int maxW) {
    n.maxH = maxH;
    n.maxW = maxW;
    size_t off = 0;
    for (int i = 0; i < UNET_NCONV; ++i) {
        n.woff[i] = off;
        off += (size_t)9 * kUnetSpec[i].cin * kUnetSpec[i].cout;
        n.boff[i] = off;
        off += kUnetSpec[i].cout;
    }
    n.nparams = off;
    const size_t P0 = (size_t)maxH * maxW, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
    struct Item {
        void** ptr;
        size_t bytes;
    };
    std::vector<Item> items;
    auto F = [&](float** p, size_t n_) { items.push_back({(void**)p, up256(n_ * 4)}); };
    auto B = [&](bf16** p, size_t n_) { items.push_back({(void**)p, up256(n_ * 2)}); };
    F(&n.params, n.nparams);
    F(&n.grads, n.nparams);
    F(&n.adam_m, n.nparams);
    F(&n.adam_v, n.nparams);
    for (int i = 0; i < UNET_NCONV; ++i) {
        B(&n.w16[i], (size_t)9 * kUnetSpec[i].cin * kUnetSpec[i].cout);
        B(&n.wt16[i], (size_t)9 * kUnetSpec[i].cin * kUnetSpec[i].cout);
    }
    B(&n.X0, P0 * 16); B(&n.t0, P0 * 16); B(&n.cat0, P0 * 48);
    B(&n.p1, P1 * 16); B(&n.t1, P1 * 32); B(&n.cat1, P1 * 96);
    B(&n.p2, P2 * 32); B(&n.t2, P2 * 64); B(&n.cat2, P2 * 128);
    B(&n.p3, P3 * 64); B(&n.t3, P3 * 64); B(&n.u3, P3 * 64);
    B(&n.t4, P2 * 64); B(&n.u4, P2 * 64); B(&n.t5, P1 * 32); B(&n.u5, P1 * 32);
    B(&n.t6, P0 * 16); B(&n.u6, P0 * 16);
    F(&n.out, P0 * 16);
    F(&n.g_out, P0 * 16); F(&n.g_u6, P0 * 16); F(&n.g_t6, P0 * 16); F(&n.g_cat0, P0 * 48);
    F(&n.g_u5, P1 * 32); F(&n.g_t5, P1 * 32); F(&n.g_cat1, P1 * 96);
    F(&n.g_u4, P2 * 64); F(&n.g_t4, P2 * 64); F(&n.g_cat2, P2 * 128);
    F(&n.g_u3, P3 * 64); F(&n.g_t3, P3 * 64); F(&n.g_p3, P3 * 64);
    F(&n.g_t2, P2 * 64); F(&n.g_p2, P2 * 32); F(&n.g_t1, P1 * 32); F(&n.g_p1, P1 * 16); F(&n.g_t0, P0 * 16);
    B(&n.dym, P0 * 16);
    // weight-gradient partials: chunks of 1024 pixels x up to 9 row tiles x 128 x 64
    n.wpart_elems = ((P0 + 1023) / 1024) * 9 * 128 * 64;
    F(&n.wpart, n.wpart_elems);
    F(&n.bpart, ((P0 + 1023) / 1024) * 64);
    // per-block partials: loss blocks of 1024 pixels, residual blocks of 32 x 8 cells
    items.push_back({(void**)&n.lpart, up256((P0 / 256 + (size_t)maxW / 32 + (size_t)maxH / 8 + 8) * sizeof(float2))});
    items.push_back({(void**)&n.epart, up256((P0 / 256 + (size_t)maxW / 32 + (size_t)maxH / 8 + 9) * sizeof(double2))});
    F(&n.target, P0);
    F(&n.prev32, P0);
    F(&n.res32, P0);
    F(&n.sigma, 64);
    items.push_back({(void**)&n.mask, up256(P0)});
    F(&n.targetc, P0);
    items.push_back({(void**)&n.maskc, up256(P0)});
    items.push_back({(void**)&n.err, 256});
    size_t total = 0;
    for (auto& it : items) total += it.bytes;
    cudaError_t e = cudaMalloc(&n.arena, total);
    if (e != cudaSuccess) return e;
    e = cudaMemset(n.arena, 0, total);
    if (e != cudaSuccess) return e;
    char* base = (char*)n.arena;
    for (auto& it : items) {
        *it.ptr = base;
        base += it.bytes;
    }
    n.red_count = reinterpret_cast<unsigned*>(n.err + 32);  // the second half of the zeroed 256-byte flag block
    return cudaSuccess;
}

// A forward-only workspace of a network for one simulation of a batch: a
// copy of `net` (weights, biases and their device copies shared) whose
// activations and feature buffers are its own, sized for that simulation's
// fine grid fh x fw and its network grid (fh / f) x (fw / f).  Forwards of
// different simulations can then run at the same time on their own streams.
// The forward-only workspace of a network for fh x fw fine cells: its activations, and with `fine` the
// fine-grid buffers of the warm start (features' residual, guard partials, masks).  A batch's canvas takes
// the activations alone.
inline cudaError_t unet_alloc_forward(UNet& v, const UNet& net, int fh, int fw, bool fine = true) {
    v = net;
    v.arena = nullptr;
    v.extra.clear();
    v.last_error.clear();
    const int f = net.coarse;
    v.maxH = fh;
    v.maxW = fw;
    const size_t P0 = (size_t)(fh / f) * (fw / f), P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64, PF_ = (size_t)fh * fw;
    struct Item {
        void** ptr;
        size_t bytes;
    };
    std::vector<Item> items;
    auto F = [&](float** p, size_t n_) { items.push_back({(void**)p, up256(n_ * 4)}); };
    auto B = [&](bf16** p, size_t n_) { items.push_back({(void**)p, up256(n_ * 2)}); };
    B(&v.X0, P0 * 16); B(&v.t0, P0 * 16); B(&v.cat0, P0 * 48);
    B(&v.p1, P1 * 16); B(&v.t1, P1 * 32); B(&v.cat1, P1 * 96);
    B(&v.p2, P2 * 32); B(&v.t2, P2 * 64); B(&v.cat2, P2 * 128);
    B(&v.p3, P3 * 64); B(&v.t3, P3 * 64); B(&v.u3, P3 * 64);
    B(&v.t4, P2 * 64); B(&v.u4, P2 * 64); B(&v.t5, P1 * 32); B(&v.u5, P1 * 32);
    B(&v.t6, P0 * 16); B(&v.u6, P0 * 16);
    F(&v.out, P0 * 16);
    v.lpart = nullptr;
    v.epart = nullptr;
    v.prev32 = v.res32 = v.sigma = nullptr;
    v.mask = v.maskc = nullptr;
    if (fine) {
        items.push_back({(void**)&v.lpart, up256((PF_ / 256 + (size_t)fw / 32 + (size_t)fh / 8 + 8) * sizeof(float2))});
        items.push_back({(void**)&v.epart, up256((PF_ / 256 + (size_t)fw / 32 + (size_t)fh / 8 + 9) * sizeof(double2))});
        F(&v.prev32, PF_);
        F(&v.res32, PF_);
        F(&v.sigma, 64);
        items.push_back({(void**)&v.mask, up256(PF_)});
        items.push_back({(void**)&v.maskc, up256(P0)});
    }
    items.push_back({(void**)&v.err, 256});
    size_t total = 0;
    for (auto& it : items) total += it.bytes;
    cudaError_t e = cudaMalloc(&v.arena, total);
    if (e != cudaSuccess) return e;
    e = cudaMemset(v.arena, 0, total);
    if (e != cudaSuccess) return e;
    char* base = (char*)v.arena;
    for (auto& it : items) {
        *it.ptr = base;
        base += it.bytes;
    }
    v.red_count = reinterpret_cast<unsigned*>(v.err + 32);  // the second half of the zeroed 256-byte flag block
    // nothing of the training state belongs to a forward-only workspace
    v.grads = v.adam_m = v.adam_v = nullptr;
    v.target = v.targetc = nullptr;
    v.wpart = v.bpart = nullptr;
    v.dym = nullptr;
    return cudaSuccess;
}

inline dim3 lin_grid(size_t n, int block = 256) { return dim3((unsigned)((n + block - 1) / block)); }

// Refreshes the bf16 weights (and their flipped transposes) from the fp32 master copy.
inline void unet_sync_weights(UNet& n, cudaStream_t st) {
    for (int i = 0; i < UNET_NCONV; ++i) {
        const int c = 9 * kUnetSpec[i].cin * kUnetSpec[i].cout;
        k_flip_transpose<<<lin_grid(c), 256, count_launch(), st>>>(n.params + n.woff[i], kUnetSpec[i].cin,
                                                                   kUnetSpec[i].cout, n.w16[i], n.wt16[i]);
    }
}

// SMs of the device, read when the network's kernels are set up (outside any
// stream capture; the devices of a node are alike).
inline int& conv_sm_count() {
    static int n = 0;
    return n;
}
inline bool conv_sm_count_init() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return false;
    conv_sm_count() = n;
    return true;
}

// Widths that are a multiple of 128 take the row-tile kernel (input rows
// staged once, no per-tap copies), the others the multistage one.  The row
// kernel keeps all nine weight tiles resident when the grid is one CTA per SM
// at most; larger grids take the ring, whose smaller footprint lets more CTAs
// share an SM, and two 128-pixel stretches per CTA where the width allows
// (each CTA allocates tensor memory, which throttles how fast CTAs start on an
// SM, so the grids that need several rounds per SM want few, fat CTAs and as
// many of them resident at once as possible).
#ifndef EFL_CONV_RESIDENT_BYTES
#define EFL_CONV_RESIDENT_BYTES 20000
#endif
// Nine weight tiles resident on the multi-round grids too while they take at most this many bytes (0: never):
// the ring makes thread 0 wait for five refills in turn, each behind an MMA commit, and small layers' tiles cost
// little shared memory (512^2 forward: 0.255 ms with the ring everywhere, 0.244 ms with up to 20 KB resident,
// 0.254 ms with up to 60 KB).
inline bool crow_resident_small(int cin, int cout) { return 9 * conv_b_bytes(cin, cout) <= EFL_CONV_RESIDENT_BYTES; }
inline void conv3x3_launch(const ConvArgs& a, cudaStream_t st) {
    const int ntiles = a.H * a.W / 128;
    if (a.W % 128 == 0) {
        const bool pair = a.W % 256 == 0;
        if (ntiles <= conv_sm_count() && crow_smem_bytes(a.cin, a.cout, true, 1) <= CV_SMEM)
            k_conv3x3_rows<true, 1>
                <<<ntiles, CV_THREADS, crow_smem_bytes(a.cin, a.cout, true, 1) + count_launch(), st>>>(a);
        else if (pair && crow_resident_small(a.cin, a.cout) && crow_smem_bytes(a.cin, a.cout, false, 2) <= CR_PAIR_SMEM)
            k_conv3x3_rows<true, 2>
                <<<ntiles / 2, 2 * CV_THREADS, crow_smem_bytes(a.cin, a.cout, true, 2) + count_launch(), st>>>(a);
        else if (pair && crow_smem_bytes(a.cin, a.cout, false, 2) <= CR_PAIR_SMEM)
            k_conv3x3_rows<false, 2>
                <<<ntiles / 2, 2 * CV_THREADS, crow_smem_bytes(a.cin, a.cout, false, 2) + count_launch(), st>>>(a);
        else if (crow_resident_small(a.cin, a.cout))
            k_conv3x3_rows<true, 1>
                <<<ntiles, CV_THREADS, crow_smem_bytes(a.cin, a.cout, true, 1) + count_launch(), st>>>(a);
        else
            k_conv3x3_rows<false, 1>
                <<<ntiles, CV_THREADS, crow_smem_bytes(a.cin, a.cout, false, 1) + count_launch(), st>>>(a);
    } else {
        ConvArgs b = a;
        const int ctas = (a.H * a.W + 127) / 128;
        if (b.resident < 0 && ctas <= conv_sm_count() && conv_smem_with(a.cin, a.cout, 9) <= CV_SMEM) b.resident = 1;
        const int smem = conv_smem_with(b.cin, b.cout, conv_tc_resident(b) ? 9 : 3);
        k_conv3x3_tc<<<ctas, CV_THREADS, smem + count_launch(), st>>>(b);
    }
}

inline void unet_conv(UNet& n, int i, const bf16* x, int xs, int xo, int H, int W, bf16* y, int ys, int yo,
                      float* yf, cudaStream_t st, const unsigned char* gap = nullptr) {
    ConvArgs a;
    a.gap = gap;
    a.x = x;
    a.xs = xs;
    a.xo = xo;
    a.w = n.w16[i];
    a.bias = n.params + n.boff[i];
    a.y = y;
    a.yf = yf;
    a.ys = ys;
    a.yo = yo;
    a.relu = kUnetSpec[i].relu;
    a.H = H;
    a.W = W;
    a.cin = kUnetSpec[i].cin;
    a.cout = kUnetSpec[i].cout;
    a.err = n.err;
    conv3x3_launch(a, st);
}

// The forward pass over an H x W image (H and W multiples of 8).  With `gaps` (four masks, one per level, of a
// canvas whose rectangles start and end on multiples of 8) every convolution that feeds another writes zeros
// at the gap pixels, so that each rectangle sees zeros around it, as the zero padding of its simulation's own
// forward; average pooling and nearest upsampling keep the gaps zero by themselves.
inline void unet_forward(UNet& n, int H, int W, cudaStream_t st, const unsigned char* const* gaps = nullptr) {
    const int Hs[4] = {H, H / 2, H / 4, H / 8}, Ws[4] = {W, W / 2, W / 4, W / 8};
    auto conv = [&](int i, const bf16* x, int xs, int lvl, bf16* y, int ys, int yo) {
        unet_conv(n, i, x, xs, 0, Hs[lvl], Ws[lvl], y, ys, yo, nullptr, st, gaps ? gaps[lvl] : nullptr);
    };
    auto pool = [&](const bf16* in, int is, int io, int lvl, int C, bf16* out) {  // level lvl -> lvl + 1
        k_pool2<<<lin_grid((size_t)Hs[lvl + 1] * Ws[lvl + 1] * C / 8), 256, count_launch(), st>>>(in, is, io, Hs[lvl],
                                                                                                   Ws[lvl], C, out);
    };
    auto up = [&](const bf16* in, int lvl, int C, bf16* out, int os) {  // level lvl + 1 -> lvl, channels [0, C)
        k_up2<<<lin_grid((size_t)Hs[lvl] * Ws[lvl] * C / 8), 256, count_launch(), st>>>(in, Hs[lvl], Ws[lvl], C, out,
                                                                                         os, 0);
    };
    conv(0, n.X0, 16, 0, n.t0, 16, 0);
    conv(1, n.t0, 16, 0, n.cat0, 48, 32);
    pool(n.cat0, 48, 32, 0, 16, n.p1);
    conv(2, n.p1, 16, 1, n.t1, 32, 0);
    conv(3, n.t1, 32, 1, n.cat1, 96, 64);
    pool(n.cat1, 96, 64, 1, 32, n.p2);
    conv(4, n.p2, 32, 2, n.t2, 64, 0);
    conv(5, n.t2, 64, 2, n.cat2, 128, 64);
    pool(n.cat2, 128, 64, 2, 64, n.p3);
    conv(6, n.p3, 64, 3, n.t3, 64, 0);
    conv(7, n.t3, 64, 3, n.u3, 64, 0);
    up(n.u3, 2, 64, n.cat2, 128);
    conv(8, n.cat2, 128, 2, n.t4, 64, 0);
    conv(9, n.t4, 64, 2, n.u4, 64, 0);
    up(n.u4, 1, 64, n.cat1, 96);
    conv(10, n.cat1, 96, 1, n.t5, 32, 0);
    conv(11, n.t5, 32, 1, n.u5, 32, 0);
    up(n.u5, 0, 32, n.cat0, 48);
    conv(12, n.cat0, 48, 0, n.t6, 16, 0);
    conv(13, n.t6, 16, 0, n.u6, 16, 0);
    unet_conv(n, 14, n.u6, 16, 0, H, W, nullptr, 16, 0, n.out, st);  // the head: fp32, read inside the rectangles
}

// Backward of conv i: dy = relu'(y) * g (bf16), weight and bias gradients,
// and (if gx) the gradient of its input, written over gx's slice.
inline void unet_conv_bwd(UNet& n, int i, const bf16* x, int xs, int xo, const bf16* y, int ys, int yo,
                          const float* g, int gs, int go, int H, int W, float* gx, int gxs, int gxo,
                          cudaStream_t st) {
    const int cin = kUnetSpec[i].cin, cout = kUnetSpec[i].cout, npix = H * W;
    k_relu_bwd<<<lin_grid((size_t)npix * cout), 256, count_launch(), st>>>(g, gs, go, y, ys, yo, npix, cout,
                                                                           kUnetSpec[i].relu, n.dym);
    // weight gradient
    WgradArgs w;
    w.x = x;
    w.xs = xs;
    w.xo = xo;
    w.dy = n.dym;
    w.H = H;
    w.W = W;
    w.cin = cin;
    w.cout = cout;
    w.pix_per_cta = 1024;
    w.part = n.wpart;
    w.err = n.err;
    const int chunks = (npix + 1023) / 1024, mtiles = (9 * cin + 127) / 128;
    k_wgrad_tc<<<dim3(chunks, mtiles), WG_THREADS, WG_SMEM + count_launch(), st>>>(w);
    k_wgrad_reduce<<<lin_grid((size_t)9 * cin * cout), 256, count_launch(), st>>>(n.wpart, chunks, mtiles, cin, cout,
                                                                                  n.grads + n.woff[i]);
    const int bblocks = (npix + 1023) / 1024;
    k_bgrad_partial<<<bblocks, 256, count_launch(), st>>>(n.dym, npix, cout, 1024, n.bpart);
    k_bgrad_reduce<<<1, 64, count_launch(), st>>>(n.bpart, bblocks, cout, n.grads + n.boff[i]);
    if (gx) {
        ConvArgs a;
        a.x = n.dym;
        a.xs = cout;
        a.xo = 0;
        a.w = n.wt16[i];
        a.bias = nullptr;
        a.y = nullptr;
        a.yf = gx;
        a.ys = gxs;
        a.yo = gxo;
        a.relu = 0;
        a.H = H;
        a.W = W;
        a.cin = cout;
        a.cout = cin;
        a.err = n.err;
        conv3x3_launch(a, st);
    }
}

// Backward pass from n.g_out; fills n.grads.
inline void unet_backward(UNet& n, int H, int W, cudaStream_t st) {
    const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
    unet_conv_bwd(n, 14, n.u6, 16, 0, nullptr, 16, 0, n.g_out, 16, 0, H, W, n.g_u6, 16, 0, st);
    unet_conv_bwd(n, 13, n.t6, 16, 0, n.u6, 16, 0, n.g_u6, 16, 0, H, W, n.g_t6, 16, 0, st);
    unet_conv_bwd(n, 12, n.cat0, 48, 0, n.t6, 16, 0, n.g_t6, 16, 0, H, W, n.g_cat0, 48, 0, st);
    k_up2_bwd<<<lin_grid((size_t)H1 * W1 * 32 / 4), 256, count_launch(), st>>>(n.g_cat0, 48, 0, H, W, 32, n.g_u5);
    unet_conv_bwd(n, 11, n.t5, 32, 0, n.u5, 32, 0, n.g_u5, 32, 0, H1, W1, n.g_t5, 32, 0, st);
    unet_conv_bwd(n, 10, n.cat1, 96, 0, n.t5, 32, 0, n.g_t5, 32, 0, H1, W1, n.g_cat1, 96, 0, st);
    k_up2_bwd<<<lin_grid((size_t)H2 * W2 * 64 / 4), 256, count_launch(), st>>>(n.g_cat1, 96, 0, H1, W1, 64, n.g_u4);
    unet_conv_bwd(n, 9, n.t4, 64, 0, n.u4, 64, 0, n.g_u4, 64, 0, H2, W2, n.g_t4, 64, 0, st);
    unet_conv_bwd(n, 8, n.cat2, 128, 0, n.t4, 64, 0, n.g_t4, 64, 0, H2, W2, n.g_cat2, 128, 0, st);
    k_up2_bwd<<<lin_grid((size_t)H3 * W3 * 64 / 4), 256, count_launch(), st>>>(n.g_cat2, 128, 0, H2, W2, 64, n.g_u3);
    unet_conv_bwd(n, 7, n.t3, 64, 0, n.u3, 64, 0, n.g_u3, 64, 0, H3, W3, n.g_t3, 64, 0, st);
    unet_conv_bwd(n, 6, n.p3, 64, 0, n.t3, 64, 0, n.g_t3, 64, 0, H3, W3, n.g_p3, 64, 0, st);
    k_pool2_bwd<<<lin_grid((size_t)H2 * W2 * 64 / 4), 256, count_launch(), st>>>(n.g_p3, H2, W2, 64, n.g_cat2, 128, 64);
    unet_conv_bwd(n, 5, n.t2, 64, 0, n.cat2, 128, 64, n.g_cat2, 128, 64, H2, W2, n.g_t2, 64, 0, st);
    unet_conv_bwd(n, 4, n.p2, 32, 0, n.t2, 64, 0, n.g_t2, 64, 0, H2, W2, n.g_p2, 32, 0, st);
    k_pool2_bwd<<<lin_grid((size_t)H1 * W1 * 32 / 4), 256, count_launch(), st>>>(n.g_p2, H1, W1, 32, n.g_cat1, 96, 64);
    unet_conv_bwd(n, 3, n.t1, 32, 0, n.cat1, 96, 64, n.g_cat1, 96, 64, H1, W1, n.g_t1, 32, 0, st);
    unet_conv_bwd(n, 2, n.p1, 16, 0, n.t1, 32, 0, n.g_t1, 32, 0, H1, W1, n.g_p1, 16, 0, st);
    k_pool2_bwd<<<lin_grid((size_t)H * W * 16 / 4), 256, count_launch(), st>>>(n.g_p1, H, W, 16, n.g_cat0, 48, 32);
    unet_conv_bwd(n, 1, n.t0, 16, 0, n.cat0, 48, 32, n.g_cat0, 48, 32, H, W, n.g_t0, 16, 0, st);
    unet_conv_bwd(n, 0, n.X0, 16, 0, n.t0, 16, 0, n.g_t0, 16, 0, H, W, nullptr, 0, 0, st);
}

}  // namespace efl
