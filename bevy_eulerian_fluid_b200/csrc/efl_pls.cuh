// efl_pls.cuh — two-layer particle level set (Enright et al. 2002) as the
// reference's particle_levelset_two_layers plugin computes it
// (src/euler_fluid/particle_levelset_two_layers/**).
//
// Layout: one struct-of-arrays set per layer (0 = positive particles,
// 1 = negative), x, y, radius as f32 planes and the escaped flag as a byte;
// the sign is implied by the layer.  Capacity per layer is nx*ny*16 like the
// reference's particle buffers (plugin.rs:221-225).  The live count stays on
// the device; per-particle kernels are grid-stride loops that read it, so a
// step never waits for the host and the whole pass can be graph-captured.
//
// Order.  The reference appends particles with atomicAdd and sorts them into
// cells with an atomic cursor, so the order of particles (and which
// particles the per-cell heap keeps on ties) varies from run to run.  This
// implementation fixes one of those orders: seeding and reseeding append in
// cell order (x fastest), attempt order inside a cell; the counting sort is
// stable (a cell's bucket is ordered by particle index before the heap runs).
// The CPU oracle uses the same order, so the two agree bit for bit.
#pragma once

#include "efl_kernels.cuh"

namespace efl {

constexpr int PLS_MAX_PER_CELL = 16;   // constants.wgsl:3 (MAX_PARTICLES_PER_CELL)
constexpr float PLS_BAND = 3.0f;       // constants.wgsl:5 (BAND_WIDTH)
constexpr float PLS_SCALE = 10000.0f;  // fixed_point.wgsl:3
constexpr int PLS_THREADS = 256;       // constants.wgsl:4 (PARTICLE_WORKWGROUP_SIZE)

// Everything the particle kernels touch.  [l] = layer, [b] = buffer.
// Each layer has two particle buffers; sel[l] names the live one and the
// reseed compacts into the other, then flips sel (no copy back, and the
// launch arguments stay the same from step to step for graph replay).
struct PlsArgs {
    float* px[2][2];
    float* py[2][2];
    float* rad[2][2];
    uint8_t* esc[2][2];
    int* sel;                 // [2] live buffer per layer
    uint32_t* count;          // [2] live particles
    uint32_t* cnt;            // [2][L] particles per cell
    uint32_t* cur;            // [2][L] scatter cursors
    uint32_t* off;            // [2][L] exclusive scan of cnt
    uint32_t* sidx;           // [2][cap] particle index per slot (scatter order)
    uint32_t* scell;          // [2][cap] cell of the slot
    uint32_t* sorted;         // [2][cap] particle index per slot, buckets in index order
    float* prio;              // [2][cap] heap priority per sorted slot (buckets of > 16)
    uint8_t* sesc;            // [2][cap] escaped per sorted slot (buckets of > 16)
    uint8_t* alive;           // [2][cap] reseed decision per sorted slot
    uint32_t* prank;          // [2][cap] rank of a kept slot among its bucket's kept slots
    unsigned long long* val;  // [2][L] kept | new << 32, then its exclusive scan
    unsigned long long* tot;  // [2] totals of val
    uint32_t* ctot;           // [2] totals of cnt
    uint8_t* addn;            // [2][L] refill attempts per cell
    uint16_t* vmask;          // [2][L] accepted refill attempts per cell (bit i = attempt i)
    float* stx;               // [2][L*16] accepted attempt i of cell c at c*16 + i (staged)
    float* sty;
    float* str;
    uint32_t* work;           // [2][L] cells with attempts to make (any order)
    uint32_t* nwork;          // [2] length of work
    uint32_t* slow;           // [2][L] band cells of more than 16 particles (any order)
    uint32_t* nslow;          // [2] length of slow
    int32_t* phip;            // [L] phi_plus  (fixed point)
    int32_t* phim;            // [L] phi_minus (fixed point)
    uint32_t* dropped;        // particles not stored for lack of capacity
    uint32_t* ticket;         // blocks of k_pls_emit done (0 between launches)
    uint32_t cap;             // per layer
    uint32_t L;               // nx * ny
    int nx, ny;
};

struct PView {
    float* x;
    float* y;
    float* r;
    uint8_t* e;
};
EFL_DEV PView pls_buf(const PlsArgs& a, int l, int b) { return PView{a.px[l][b], a.py[l][b], a.rad[l][b], a.esc[l][b]}; }
EFL_DEV PView pls_live(const PlsArgs& a, int l) { return pls_buf(a, l, a.sel[l]); }
EFL_DEV PView pls_spare(const PlsArgs& a, int l) { return pls_buf(a, l, 1 - a.sel[l]); }

// ---------------------------------------------------------------------------
// WGSL helpers used by the plugin

// u32(f32): toward zero, saturating; NaN -> 0.
EFL_DEV uint32_t f2u(float v) { return __float2uint_rz(v); }

// utils/coordinate.wgsl:19-49 (interp2d_center, interp2d_center_rg32float);
// loads outside the texture read 0.
EFL_DEV float interp_center(const PF& t, float x, float y) {
    int i = f2i(floorf(x)), j = f2i(floorf(y));
    float fi = x - (float)i, fj = y - (float)j;
    float a = t.ld(i, j), b = t.ld(i + 1, j), c = t.ld(i, j + 1), d = t.ld(i + 1, j + 1);
    return wmix(wmix(a, b, fi), wmix(c, d, fi), fj);
}
EFL_DEV float2 interp_center2(const P2& t, float x, float y) {
    int i = f2i(floorf(x)), j = f2i(floorf(y));
    float fi = x - (float)i, fj = y - (float)j;
    float2 a = t.ld(i, j), b = t.ld(i + 1, j), c = t.ld(i, j + 1), d = t.ld(i + 1, j + 1);
    return make_float2(wmix(wmix(a.x, b.x, fi), wmix(c.x, d.x, fi), fj),
                       wmix(wmix(a.y, b.y, fi), wmix(c.y, d.y, fi), fj));
}

// utils/hash.wgsl: one 4-byte block of MurmurHash3 (x86_32) with the
// reference's seeds; both rotations are by 15 bits (the h rotation of the
// published hash is 13; the reference's rotl32 is used for both).
EFL_DEV uint32_t pls_rotl(uint32_t x) { return (x << 15) | (x >> 17); }
EFL_DEV uint32_t pls_murmur(uint32_t k, uint32_t h) {
    k *= 0xcc9e2d51u;
    k = pls_rotl(k);
    k *= 0x1b873593u;
    h ^= k;
    h = pls_rotl(h);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
EFL_DEV float pls_unit(uint32_t h) { return __uint_as_float((h & 0x007fffffu) | 0x3f800000u) - 1.0f; }
EFL_DEV float pls_hash11(float v) { return pls_unit(pls_murmur(__float_as_uint(v), 11111u)); }
EFL_DEV float2 pls_hash22(float x, float y) {
    return make_float2(pls_unit(pls_murmur(__float_as_uint(x), 12345u)),
                       pls_unit(pls_murmur(__float_as_uint(y), 98765u)));
}

// particle.wgsl:50-54
EFL_DEV float pls_radius(float phi) { return fminf(fmaxf(fabsf(phi), 0.1f), 0.5f); }

// particle.wgsl:36-82 (attract once with lambda 1, then accept inside the
// domain and within [bmin, bmax]).  normalize(g) is g / sqrt(dot(g, g)).
EFL_DEV bool pls_spawn(float x, float y, float goal, float bmin, float bmax, const PF& ls, const P2& grad, int nx,
                       int ny, float& ox, float& oy, float& orad) {
    float phi = interp_center(ls, x, y);
    float2 g = interp_center2(grad, x, y);
    float len = sqrtf(g.x * g.x + g.y * g.y);
    float gx = g.x / len, gy = g.y / len;
    float k = 1.0f * (goal - phi);
    float xn = x + k * gx, yn = y + k * gy;
    if (!(0.0f < xn && 0.0f < yn && xn < (float)nx - 1.0f && yn < (float)ny - 1.0f)) return false;
    float pn = interp_center(ls, xn, yn);
    if (!(bmin <= pn && pn <= bmax)) return false;
    ox = xn;
    oy = yn;
    orad = pls_radius(pn);
    return true;
}

// Attempt i of cell (x, y) for layer l.
// init = true: initialize_particles.wgsl:31-57 -- the negative particle
// starts from the POSITIVE attempt's position x (x_neg is computed there but
// never used) with its own goal drawn from seed + 1000.
// init = false: add_particles.wgsl:17-45.
EFL_DEV bool pls_attempt(bool init, int l, int x, int y, uint32_t i, const PF& ls, const P2& grad, int nx, int ny,
                         float& ox, float& oy, float& orad) {
    const float bmin = 0.1f, bmax = PLS_BAND;
    uint32_t cell = (uint32_t)x + (uint32_t)nx * (uint32_t)y;
    uint32_t seed = cell + i;
    float xb = (float)x, yb = (float)y;
    float sf = (float)seed;
    float2 h = pls_hash22(xb + sf, yb + sf);
    float sx = xb + h.x, sy = yb + h.y;
    if (l == 0) {
        float goal = pls_hash11(sf) * (bmax - bmin) + bmin;
        return pls_spawn(sx, sy, goal, bmin, bmax, ls, grad, nx, ny, ox, oy, orad);
    }
    const float nmin = -bmax, nmax = -bmin;
    float gs = init ? (float)(seed + 1000u) : sf;
    float goal = pls_hash11(gs) * (nmax - nmin) + nmin;
    return pls_spawn(sx, sy, goal, nmin, nmax, ls, grad, nx, ny, ox, oy, orad);
}

// count_particles_in_cell.wgsl:14-20: the cell of a particle, u32 arithmetic;
// an index past the buffer is clamped to its last element (bounds-checked
// storage access).
EFL_DEV uint32_t pls_bin(float x, float y, uint32_t nx, uint32_t L) {
    uint32_t c = f2u(x) + nx * f2u(y);
    return c < L ? c : L - 1;
}

// ---------------------------------------------------------------------------
// Exclusive scans per layer (blockIdx.y = layer): block-local scan, one block
// per layer scanning the block totals, then the add.  Integer sums, so the
// result does not depend on the order.
constexpr int SC_T = 512, SC_I = 8, SC_N = SC_T * SC_I;

template <class T>
EFL_DEV T block_excl_scan(T v, T* s_warp, T& total) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        T t = lane < SC_T / 32 ? s_warp[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < SC_T / 32) s_warp[lane] = t;
    }
    __syncthreads();
    total = s_warp[SC_T / 32 - 1];
    T base = w > 0 ? s_warp[w - 1] : T(0);
    return base + x - v;
}

template <class Tin, class T>
__global__ void __launch_bounds__(SC_T) k_scan_local(const Tin* in, T* out, T* part, uint32_t n, uint32_t stride,
                                                      uint32_t nb) {
    __shared__ T s[SC_N];
    __shared__ T s_warp[SC_T / 32];
    const int l = blockIdx.y;
    const Tin* src = in + (size_t)l * stride;
    T* dst = out + (size_t)l * stride;
    size_t b0 = (size_t)blockIdx.x * SC_N;
#pragma unroll
    for (int k = 0; k < SC_I; ++k) {
        size_t i = b0 + k * SC_T + threadIdx.x;
        s[k * SC_T + threadIdx.x] = i < n ? (T)src[i] : T(0);
    }
    __syncthreads();
    T loc[SC_I];
    T sum = 0;
#pragma unroll
    for (int k = 0; k < SC_I; ++k) {
        loc[k] = sum;
        sum += s[threadIdx.x * SC_I + k];
    }
    T total;
    T base = block_excl_scan<T>(sum, s_warp, total);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SC_I; ++k) s[threadIdx.x * SC_I + k] = base + loc[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SC_I; ++k) {
        size_t i = b0 + k * SC_T + threadIdx.x;
        if (i < n) dst[i] = s[k * SC_T + threadIdx.x];
    }
    if (threadIdx.x == 0) part[(size_t)l * nb + blockIdx.x] = total;
}

template <class T>
__global__ void __launch_bounds__(SC_T) k_scan_parts(T* part, T* tot, uint32_t nb) {
    __shared__ T s_warp[SC_T / 32];
    T* p = part + (size_t)blockIdx.y * nb;
    T carry = 0;
    for (uint32_t b = 0; b < nb; b += SC_T) {
        uint32_t i = b + threadIdx.x;
        T v = i < nb ? p[i] : T(0);
        T total;
        T e = block_excl_scan<T>(v, s_warp, total);
        if (i < nb) p[i] = carry + e;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) tot[blockIdx.y] = carry;
}

template <class T>
__global__ void k_scan_add(T* out, const T* part, uint32_t n, uint32_t stride, uint32_t nb) {
    const int l = blockIdx.y;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[(size_t)l * stride + i] += part[(size_t)l * nb + i / SC_N];
}

// ---------------------------------------------------------------------------
// Per-particle kernels: grid-stride over the live count, blockIdx.y = layer.

// advect_particles.wgsl:15-33 with utils/coordinate.wgsl:96-109 (tvd_rk3).
__global__ void k_pls_advect(PlsArgs a, PF u, PF v, float dt) {
    const int l = blockIdx.y;
    const uint32_t n = a.count[l];
    const PView P = pls_live(a, l);
    const float third = 1.0f / 3.0f, two_thirds = 2.0f / 3.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float x = P.x[i], y = P.y[i];
        float u0 = interp_edge_x(u, x, y), v0 = interp_edge_y(v, x, y);
        float x1 = x + dt * u0, y1 = y + dt * v0;
        float u1 = interp_edge_x(u, x1, y1), v1 = interp_edge_y(v, x1, y1);
        float x2 = 0.75f * x + 0.25f * (x1 + dt * u1), y2 = 0.75f * y + 0.25f * (y1 + dt * v1);
        float u2 = interp_edge_x(u, x2, y2), v2 = interp_edge_y(v, x2, y2);
        P.x[i] = third * x + two_thirds * (x2 + dt * u2);
        P.y[i] = third * y + two_thirds * (y2 + dt * v2);
    }
}

// reset_levelset_correction.wgsl:7-16: both correction buffers start from
// the level set in fixed point.
__global__ void k_pls_reset(PlsArgs a, PF ls) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.L) return;
    int x = (int)(c % (uint32_t)a.nx), y = (int)(c / (uint32_t)a.nx);
    int32_t q = f2i(ls.ld(x, y) * PLS_SCALE);
    a.phip[c] = q;
    a.phim[c] = q;
}

// mark_escaped_particles.wgsl:12-22 (particle.wgsl:19-30) fused with
// accumulate_levelset_correction.wgsl:11-40: an escaped particle pushes
// sign * (r - |x - cell|) into the 4 cells at and above-right of floor(x),
// atomicMax for the positive layer, atomicMin for the negative.
__global__ void k_pls_mark_accumulate(PlsArgs a, PF ls) {
    const int l = blockIdx.y;
    const float sgn = l == 0 ? 1.0f : -1.0f;
    const uint32_t n = a.count[l];
    const PView P = pls_live(a, l);
    int32_t* phi = l == 0 ? a.phip : a.phim;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float x = P.x[i], y = P.y[i], r = P.r[i];
        bool e = sgn * interp_center(ls, x, y) + r < 0.0f;
        P.e[i] = e ? 1 : 0;
        if (!e) continue;
        uint32_t bx = f2u(x), by = f2u(y);
        for (uint32_t di = 0; di < 2; ++di)
            for (uint32_t dj = 0; dj < 2; ++dj) {
                uint32_t cx = bx + di, cy = by + dj;
                if (cx >= (uint32_t)a.nx || cy >= (uint32_t)a.ny) continue;
                float dx = x - (float)cx, dy = y - (float)cy;
                float p = sgn * (r - sqrtf(dx * dx + dy * dy));
                int32_t q = f2i(p * PLS_SCALE);
                uint32_t c = cx + (uint32_t)a.nx * cy;
                if (l == 0) atomicMax(&phi[c], q);
                else atomicMin(&phi[c], q);
            }
    }
}

// correct_levelset.wgsl:8-24: the corrected level set takes whichever of
// phi+ and phi- is smaller in magnitude (phi+ on ties), back in f32.  Every
// cell passes through the fixed point.
__global__ void k_pls_correct(PlsArgs a, PF ls) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.L) return;
    int x = (int)(c % (uint32_t)a.nx), y = (int)(c / (uint32_t)a.nx);
    float pp = (float)a.phip[c] / PLS_SCALE;
    float pm = (float)a.phim[c] / PLS_SCALE;
    ls.st(x, y, fabsf(pp) <= fabsf(pm) ? pp : pm);
}

// update_particle_radii.wgsl:8-19: radius from the level set at the
// particle's cell (no interpolation; 0 outside the grid -> radius 0.1).
__global__ void k_pls_radii(PlsArgs a, PF ls) {
    const int l = blockIdx.y;
    const uint32_t n = a.count[l];
    const PView P = pls_live(a, l);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        P.r[i] = pls_radius(ls.ld(f2i(P.x[i]), f2i(P.y[i])));
}

// Warp-aggregated bucket append: lanes of a warp that share a cell make one
// atomicAdd; returns this lane's position among the appends to its cell.
EFL_DEV uint32_t pls_aggregated_add(uint32_t* counter, uint32_t cell, bool active) {
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (!active) return 0;
    const unsigned peers = __match_any_sync(act, cell);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

// count_particles_in_cell.wgsl:10-21; with radii != 0 also the preceding
// update_particle_radii.wgsl on ls (one pass over the positions for both).
__global__ void k_pls_bin(PlsArgs a, PF ls, int radii) {
    const int l = blockIdx.y;
    const uint32_t n = a.count[l];
    const PView P = pls_live(a, l);
    uint32_t* cnt = a.cnt + (size_t)l * a.L;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += stride) {  // warp-uniform trip count
        const uint32_t i = i0 + threadIdx.x;
        const bool on = i < n;
        const float x = on ? P.x[i] : 0.0f, y = on ? P.y[i] : 0.0f;
        if (on && radii) P.r[i] = pls_radius(ls.ld(f2i(x), f2i(y)));
        const uint32_t c = on ? pls_bin(x, y, (uint32_t)a.nx, a.L) : 0u;
        const unsigned act = __ballot_sync(0xffffffffu, on);
        if (on) {
            const unsigned peers = __match_any_sync(act, c);
            if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&cnt[c], (uint32_t)__popc(peers));
        }
    }
}

// sort_particles.wgsl:12-26: each particle's slot in its cell's bucket (the
// order inside a bucket depends on atomic arrival; k_pls_rank orders it).
__global__ void k_pls_scatter(PlsArgs a) {
    const int l = blockIdx.y;
    const uint32_t n = a.count[l];
    const PView P = pls_live(a, l);
    const uint32_t* off = a.off + (size_t)l * a.L;
    uint32_t* cur = a.cur + (size_t)l * a.L;
    uint32_t* sidx = a.sidx + (size_t)l * a.cap;
    uint32_t* scell = a.scell + (size_t)l * a.cap;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint32_t i = i0 + threadIdx.x;
        const bool on = i < n;
        const uint32_t c = on ? pls_bin(P.x[i], P.y[i], (uint32_t)a.nx, a.L) : 0u;
        const uint32_t k = pls_aggregated_add(&cur[c], c, on);
        if (on) {
            const uint32_t slot = off[c] + k;
            sidx[slot] = i;
            scell[slot] = c;
        }
    }
}

// The stable order: each slot's rank among its bucket's particle indices
// (distinct), so bucket order = particle-index order.  For buckets of more
// than 16 particles the heap inputs of reseed_particles.wgsl are staged here
// in sorted order: priority sign * phi(x) - r (eval_priority, :101-103;
// +inf for escaped particles, whose priority the heap never reads) and the
// escaped test (particle.wgsl:19-30), on levelset_air0.
__global__ void k_pls_rank(PlsArgs a, PF ls) {
    const int l = blockIdx.y;
    const uint32_t n = a.count[l];
    const float sgn = l == 0 ? 1.0f : -1.0f;
    const PView P = pls_live(a, l);
    const size_t lc = (size_t)l * a.cap, ll = (size_t)l * a.L;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint32_t c = a.scell[lc + s];
        const uint32_t o = a.off[ll + c], m = a.cnt[ll + c];
        const uint32_t v = a.sidx[lc + s];
        const uint32_t* b = a.sidx + lc + o;
        uint32_t r = 0;
        for (uint32_t t = 0; t < m; ++t) r += b[t] < v ? 1u : 0u;
        const size_t d = lc + o + r;
        a.sorted[d] = v;
        if (m > PLS_MAX_PER_CELL) {
            const float rad = P.r[v];
            const float phi = interp_center(ls, P.x[v], P.y[v]);
            const bool e = sgn * phi + rad < 0.0f;
            // escaped: +inf, so that k_pls_select ranks the others without a branch
            a.prio[d] = e ? __int_as_float(0x7f800000) : sgn * phi - rad;
            a.sesc[d] = e ? 1 : 0;
        }
    }
}

// ---------------------------------------------------------------------------
// reseed_particles.wgsl:14-148 per cell and layer.
//
// A bucket of at most 16 particles in a band cell keeps every particle and
// asks for 16 - n new ones whatever their escape state: the heap never
// overflows (inserted + escaped <= n <= 16 = capacity), so no eviction
// happens.  Larger buckets get the heap's outcome from k_pls_select, or run
// the reference's heap itself (pls_heap_serial), including its index
// arithmetic: sift_up from slot 0 computes the parent (0 - 1) / 2 in u32,
// and an index past the 16-entry array is clamped to 15 (bounds-checked
// local array access); the heap starts zero-initialised.  An eviction of a
// zero node (capacity used up by escaped particles before any insertion)
// names slot 0 of the whole buffer; inside this cell's bucket it applies,
// for another cell's bucket it is the racy write the reference orders
// arbitrarily -- taken as landing before that cell's own writes, i.e.
// without effect.
struct PlsNode {
    uint32_t index;
    float value;
};

EFL_DEV void pls_correct_heap(PlsNode* h, uint32_t cap) {  // correct_heap, start 0
    uint32_t i = 0;
    for (;;) {
        uint32_t lft = 2 * i + 1, rgt = 2 * i + 2, big = i;
        if (lft < cap && h[lft].value > h[big].value) big = lft;
        if (rgt < cap && h[rgt].value > h[big].value) big = rgt;
        if (big == i) return;
        PlsNode t = h[big];
        h[big] = h[i];
        h[i] = t;
        i = big;
    }
}
EFL_DEV uint32_t pls_clamp16(uint32_t i) { return i < 15u ? i : 15u; }
EFL_DEV void pls_sift_up(PlsNode* h, uint32_t size) {
    uint32_t i = size - 1;
    for (;;) {
        uint32_t p = (i - 1) / 2;
        uint32_t pc = pls_clamp16(p), ic = pls_clamp16(i);
        if (h[pc].value > h[ic].value) return;
        PlsNode t = h[pc];
        h[pc] = h[ic];
        h[ic] = t;
        i = p;
        if (i == 0) return;
    }
}

// Band cells of at most 16 particles and cells outside the band, one thread
// per cell; band cells of more than 16 particles are listed for
// k_pls_select.  Cells that will make refill attempts are listed in work.
__global__ void k_pls_heap(PlsArgs a, PF ls) {
    const int l = blockIdx.y;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = c < a.L;
    const uint32_t cc = valid ? c : 0u;
    const int x = (int)(cc % (uint32_t)a.nx), y = (int)(cc / (uint32_t)a.nx);
    const size_t ll = (size_t)l * a.L, lc = (size_t)l * a.cap;
    const uint32_t n = valid ? a.cnt[ll + cc] : 0u;
    const uint32_t off = a.off[ll + cc];
    const bool near = valid && fabsf(interp_center(ls, (float)x, (float)y)) < PLS_BAND;
    const bool slow = near && n > PLS_MAX_PER_CELL;
    uint32_t to_add = 0;
    if (valid && !slow) {
        uint8_t* alive = a.alive + lc + off;
        uint32_t* prank = a.prank + lc + off;
        for (uint32_t i = 0; i < n; ++i) {
            alive[i] = near ? 1 : 0;
            prank[i] = i;
        }
        to_add = near ? PLS_MAX_PER_CELL - n : 0u;
        a.val[ll + c] = near ? n : 0u;
        a.addn[ll + c] = (uint8_t)to_add;
    }
    const uint32_t ks = pls_aggregated_add(a.nslow + l, 0u, slow);  // every lane of the warp
    if (slow) a.slow[ll + ks] = c;
    const uint32_t kw = pls_aggregated_add(a.nwork + l, 0u, to_add != 0);
    if (to_add) a.work[ll + kw] = c;
}

// The reference's heap, serially, for one listed cell (the exact fallback of
// k_pls_select).  Returns the number of refill attempts.
EFL_DEV uint32_t pls_heap_serial(const PlsArgs& a, int l, uint32_t c) {
    const size_t ll = (size_t)l * a.L, lc = (size_t)l * a.cap;
    const uint32_t n = a.cnt[ll + c];
    const uint32_t off = a.off[ll + c];
    uint8_t* alive = a.alive + lc + off;
    uint32_t* prank = a.prank + lc + off;
    const float* prio = a.prio + lc + off;
    const uint8_t* esc = a.sesc + lc + off;
    PlsNode heap[PLS_MAX_PER_CELL];
    for (int k = 0; k < PLS_MAX_PER_CELL; ++k) heap[k] = PlsNode{0u, 0.0f};
    uint32_t hcap = PLS_MAX_PER_CELL, hidx = 0;
    auto kill = [&](uint32_t slot) {  // heap nodes hold global slots
        if (slot >= off && slot - off < n) alive[slot - off] = 0;
    };
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t slot = off + i;
        const float pr = prio[i];
        if (esc[i]) {
            if (hcap != 0) {
                alive[i] = 1;
                hcap -= 1;
                if (hidx > hcap) {
                    kill(heap[0].index);
                    heap[0] = heap[hidx - 1];
                    hidx -= 1;
                    pls_correct_heap(heap, hcap);
                }
            } else {
                alive[i] = 0;
            }
            continue;
        }
        if (hidx < hcap) {
            alive[i] = 1;
            heap[hidx] = PlsNode{slot, pr};
            hidx += 1;
            pls_sift_up(heap, hidx);
        } else if (pr < heap[0].value) {
            alive[i] = 1;
            kill(heap[0].index);
            heap[0] = PlsNode{slot, pr};
            pls_correct_heap(heap, hcap);
        } else {
            alive[i] = 0;
        }
    }
    uint32_t kept = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (alive[i]) prank[i] = kept++;
    a.val[ll + c] = kept;
    a.addn[ll + c] = (uint8_t)(hcap - hidx);
    return hcap - hidx;
}

// The heap's outcome for the listed band cells of more than 16 particles,
// one warp per cell.  Let E be the number of escaped particles.
//
// E < 16: the heap of reseed_particles.wgsl keeps every escaped particle
// and, of the others, those whose priority is among the keep = 16 - E
// lowest, and asks for keep - min(others, keep) new ones.  Why: every step
// keeps the MULTISET of heap values equal to the lowest min(seen, capacity)
// values of the non-escaped seen so far (insert while not full; replace the
// maximum by a strictly lower newcomer; an escaped arrival lowers the
// capacity and evicts the maximum of a full heap) -- decisions depend on
// values only -- and the capacity never reaches 0, so no zero node is ever
// evicted.  A full heap stays full and its maximum never rises, so a value
// below the final maximum is never evicted or rejected, and a value above it
// never survives.  The particles are therefore determined unless equal
// priorities straddle the cut (r_lt lower and r_eq equal others with
// r_lt < keep <= r_lt + r_eq); then which of them the heap keeps depends on
// its internal order.
//
// E >= 16: the first 16 escaped particles are kept and the capacity reaches
// 0 at the 16th (position q); the heap is emptied then, so every other
// particle before q is dropped, and heap[0] keeps the last node evicted --
// the lowest of them, value v0 -- or, with none, the zero node (value 0,
// slot 0 of the buffer).  After q, escaped particles are dropped and each
// other particle replaces heap[0] when strictly lower (evicting the
// previous holder), so the one kept is the first occurrence of the lowest
// value after q, if that value is below v0; no refill.  The zero node's
// eviction drops slot 0 of this bucket when the bucket starts the buffer.
//
// A NaN or infinite priority, or a straddling tie with E < 16, runs the heap
// itself (pls_heap_serial).
__global__ void k_pls_select(PlsArgs a) {
    const int l = blockIdx.y;
    const uint32_t ns = a.nslow[l];
    const size_t ll = (size_t)l * a.L, lc = (size_t)l * a.cap;
    const uint32_t lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t wpb = blockDim.x / 32;
    const float inf = __int_as_float(0x7f800000);
    for (uint32_t w = blockIdx.x * wpb + threadIdx.x / 32; w < ns; w += gridDim.x * wpb) {  // warp-uniform
        const uint32_t c = a.slow[ll + w];
        const uint32_t n = a.cnt[ll + c];
        const uint32_t off = a.off[ll + c];
        const float* prio = a.prio + lc + off;
        const uint8_t* esc = a.sesc + lc + off;
        uint8_t* alive = a.alive + lc + off;
        uint32_t* prank = a.prank + lc + off;
        // escaped count, the position q of the 16th escaped, NaN priorities
        uint32_t nesc = 0, q = n;
        bool nan = false;
        for (uint32_t b = 0; b < n; b += 32) {
            const uint32_t i = b + lane;
            const bool e = i < n && esc[i] != 0;
            nan |= i < n && !e && !(prio[i] < inf);  // NaN or +inf (+inf marks escaped ones)
            const unsigned me = __ballot_sync(0xffffffffu, e);
            if (nesc < PLS_MAX_PER_CELL && nesc + __popc(me) >= PLS_MAX_PER_CELL) {
                unsigned m = me;  // the (16 - nesc)-th set bit: drop the lowest 15 - nesc
                for (uint32_t k = nesc + 1; k < PLS_MAX_PER_CELL; ++k) m &= m - 1;
                q = b + (uint32_t)(__ffs(m) - 1);
            }
            nesc += (uint32_t)__popc(me);
        }
        bool bad = __any_sync(0xffffffffu, nan);
        const bool full = nesc >= PLS_MAX_PER_CELL;
        const uint32_t keep = full ? 0u : PLS_MAX_PER_CELL - nesc;
        // E >= 16: v0, then the first occurrence of the lowest value after q
        float v0 = 0.0f;
        uint32_t holder = n;
        bool zero_kill = false;
        if (!bad && full) {
            float lo = inf, lo_after = inf;
            bool before = false;
            for (uint32_t b = 0; b < n; b += 32) {
                const uint32_t i = b + lane;
                if (i < n && !esc[i]) {
                    const float p = prio[i];
                    if (i < q) {
                        before = true;
                        lo = fminf(lo, p);
                    } else {
                        lo_after = fminf(lo_after, p);
                    }
                }
            }
            for (int o = 16; o; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                lo_after = fminf(lo_after, __shfl_xor_sync(0xffffffffu, lo_after, o));
            }
            before = __any_sync(0xffffffffu, before);
            v0 = before ? lo : 0.0f;
            if (lo_after < v0) {
                uint32_t first = n;
                for (uint32_t b = 0; b < n; b += 32) {
                    const uint32_t i = b + lane;
                    if (i < n && i > q && !esc[i] && prio[i] == lo_after) first = min(first, i);
                }
                for (int o = 16; o; o >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
                holder = first;
                zero_kill = !before && off == 0;
            }
        }
        if (!bad && !full) {
            // rank of each non-escaped particle among the non-escaped, kept in prank for now
            bool tie = false;
            for (uint32_t b = 0; b < n; b += 32) {
                const uint32_t i = b + lane;
                if (i < n && !esc[i]) {
                    // escaped particles are staged as +inf: never lower, never
                    // equal (a finite p; a NaN p has already sent the bucket
                    // to the serial heap)
                    const float p = prio[i];
                    uint32_t r = 0, eq = 0;
#pragma unroll 8
                    for (uint32_t j = 0; j < n; ++j) {
                        const float qv = prio[j];
                        r += qv < p ? 1u : 0u;
                        eq += qv == p ? 1u : 0u;  // includes i itself
                    }
                    tie |= r < keep && keep <= r + eq - 1;
                    prank[i] = r;
                }
            }
            bad = __any_sync(0xffffffffu, tie);
        }
        uint32_t to_add;
        if (bad) {
            uint32_t t = 0;
            if (lane == 0) t = pls_heap_serial(a, l, c);
            to_add = __shfl_sync(0xffffffffu, t, 0);
        } else {
            const uint32_t others = n - nesc;
            uint32_t kept = 0;
            for (uint32_t b = 0; b < n; b += 32) {
                const uint32_t i = b + lane;
                bool v = false;
                if (i < n) {
                    if (full) v = esc[i] ? (i <= q && !(zero_kill && i == 0)) : i == holder;
                    else v = esc[i] != 0 || prank[i] < keep;
                }
                const unsigned m = __ballot_sync(0xffffffffu, v);
                if (i < n) {
                    alive[i] = v ? 1 : 0;
                    if (v) prank[i] = kept + (uint32_t)__popc(m & lt);
                }
                kept += (uint32_t)__popc(m);
            }
            to_add = keep - (others < keep ? others : keep);
            if (lane == 0) {
                a.val[ll + c] = kept;
                a.addn[ll + c] = (uint8_t)to_add;
            }
        }
        if (lane == 0 && to_add) a.work[ll + atomicAdd(a.nwork + l, 1u)] = c;
    }
}

// ---------------------------------------------------------------------------
// Seeding and refill, 16 lanes per listed cell (one lane per attempt), over
// the work list of cells that make attempts.  Which list entry a cell has
// does not matter: positions come from the cell-order scan of val.
// init = 1: initialize_particles.wgsl:17-58 with update_interface_band_mask
// (16 attempts in every cell with |levelset_air0| < 3); init = 0: the
// reseed's add_particles.wgsl (addn[c] attempts).
constexpr int PLS_GROUP = 16;

// update_interface_band_mask.wgsl:7-17: the band cells, listed.
__global__ void k_pls_band(PlsArgs a, PF ls) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = c < a.L && fabsf(ls.ld((int)(c % (uint32_t)a.nx), (int)(c / (uint32_t)a.nx))) < PLS_BAND;
    if (c < a.L) a.val[c] = a.val[(size_t)a.L + c] = 0;  // cells without attempts add nothing
    const uint32_t k = pls_aggregated_add(a.nwork, 0u, on);
    if (on) a.work[k] = a.work[(size_t)a.L + k] = c;
}

EFL_DEV bool pls_group_attempt(const PlsArgs& a, const PF& ls, const P2& grad, int init, int l, uint32_t c,
                               uint32_t i, float& ox, float& oy, float& orad) {
    const int x = (int)(c % (uint32_t)a.nx), y = (int)(c / (uint32_t)a.nx);
    const uint32_t attempts = init ? PLS_MAX_PER_CELL : (uint32_t)a.addn[(size_t)l * a.L + c];
    if (i >= attempts) return false;
    return pls_attempt(init != 0, l, x, y, i, ls, grad, a.nx, a.ny, ox, oy, orad);
}

// Accepted attempts per listed cell: vmask (bit i = attempt i), val's high
// half (val's low half = kept particles, from k_pls_heap; 0 at init), and
// the particles themselves, staged for k_pls_emit.
__global__ void k_pls_spawn_count(PlsArgs a, PF ls, P2 grad, int init) {
    const int l = blockIdx.y;
    const uint32_t nw = init ? a.nwork[0] : a.nwork[l];
    const uint32_t* work = a.work + (size_t)l * a.L;
    const uint32_t i = threadIdx.x % PLS_GROUP;
    const uint32_t per = blockDim.x / PLS_GROUP;
    for (uint32_t w0 = blockIdx.x * per; w0 < nw; w0 += gridDim.x * per) {  // block-uniform
        const uint32_t w = w0 + threadIdx.x / PLS_GROUP;
        const bool on = w < nw;
        const uint32_t c = on ? work[w] : 0u;
        float ox, oy, orad;
        const bool ok = on && pls_group_attempt(a, ls, grad, init, l, c, i, ox, oy, orad);
        if (ok) {
            const size_t t = ((size_t)l * a.L + c) * PLS_GROUP + i;
            a.stx[t] = ox;
            a.sty[t] = oy;
            a.str[t] = orad;
        }
        const uint32_t m = (__ballot_sync(0xffffffffu, ok) >> (threadIdx.x & 16)) & 0xffffu;
        if (on && i == 0) {
            const size_t k = (size_t)l * a.L + c;
            a.vmask[k] = (uint16_t)m;
            a.val[k] = (a.val[k] & 0xffffffffull) | ((unsigned long long)__popc(m) << 32);
        }
    }
}

// The writes of a seeding or a reseed, one launch: blocks [0, kb) move the
// kept particles (reseed only; delete_particles.wgsl:12-17) to the spare
// buffer at (kept before this cell) + (rank in the cell's bucket); the
// other blocks write the accepted attempts of the listed cells (staged by
// k_pls_spawn_count), 16 lanes per cell -- init appends them to the live buffer after count[l]
// (initialize_particles.wgsl:44-56 appends to the existing count), a reseed
// writes them after all kept particles (update_particles_count.wgsl,
// add_particles.wgsl:36-45).  The last block to finish sets the new counts
// (capped at the capacity; the overflow is in a.dropped) and, after a
// reseed, makes the compacted buffer live.
__global__ void k_pls_emit(PlsArgs a, PF ls, P2 grad, int init, uint32_t kb) {
    const int l = blockIdx.y;
    if (!init && blockIdx.x < kb) {
        const uint32_t n = a.count[l];
        const PView S = pls_live(a, l), D = pls_spare(a, l);
        const size_t lc = (size_t)l * a.cap, ll = (size_t)l * a.L;
        for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += kb * blockDim.x) {
            // independent loads first, one dependent round for val and the particle
            const bool keep = a.alive[lc + s] != 0;
            const uint32_t c = a.scell[lc + s], r = a.prank[lc + s], j = a.sorted[lc + s];
            if (!keep) continue;
            const uint32_t dst = (uint32_t)(a.val[ll + c] & 0xffffffffull) + r;
            const float x = S.x[j], y = S.y[j], rad = S.r[j];
            const uint8_t e = S.e[j];
            D.x[dst] = x;
            D.y[dst] = y;
            D.r[dst] = rad;
            D.e[dst] = e;
        }
    } else {
        const uint32_t nb = gridDim.x - (init ? 0u : kb), b0 = blockIdx.x - (init ? 0u : kb);
        const uint32_t nw = init ? a.nwork[0] : a.nwork[l];
        const uint32_t* work = a.work + (size_t)l * a.L;
        const uint32_t i = threadIdx.x % PLS_GROUP;
        const uint32_t per = blockDim.x / PLS_GROUP;
        const uint64_t base = init ? (uint64_t)a.count[l] : (a.tot[l] & 0xffffffffull);
        const PView D = init ? pls_live(a, l) : pls_spare(a, l);
        for (uint32_t w = b0 * per + threadIdx.x / PLS_GROUP; w < nw; w += nb * per) {
            const uint32_t c = work[w];
            const size_t k = (size_t)l * a.L + c;
            const uint32_t m = a.vmask[k];
            if (!((m >> i) & 1u)) continue;
            const size_t t = k * PLS_GROUP + i;
            const float ox = a.stx[t], oy = a.sty[t], orad = a.str[t];
            const uint64_t dst = base + (a.val[k] >> 32) + (uint64_t)__popc(m & ((1u << i) - 1u));
            if (dst >= a.cap) {
                atomicAdd(a.dropped, 1u);
                continue;
            }
            D.x[dst] = ox;
            D.y[dst] = oy;
            D.r[dst] = orad;
            D.e[dst] = 0;
        }
    }
    // last block of the launch: counts and the live buffer
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t ticket = atomicAdd(a.ticket, 1u);
        s_last = ticket == gridDim.x * gridDim.y - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x < 2) {
        __threadfence();
        const int m = threadIdx.x;
        const unsigned long long t = a.tot[m];
        const uint64_t nn = init ? (uint64_t)a.count[m] + (t >> 32) : (t & 0xffffffffull) + (t >> 32);
        a.count[m] = (uint32_t)(nn < a.cap ? nn : a.cap);
        if (!init) a.sel[m] = 1 - a.sel[m];
        if (m == 0) *a.ticket = 0;
    }
}

}  // namespace efl
