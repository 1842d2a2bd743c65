// efl_pls.cuh — two-layer particle level set (Enright et al. 2002) as the
// reference's particle_levelset_two_layers plugin computes it
// (src/euler_fluid/particle_levelset_two_layers/**).
//
// Layout: one struct-of-arrays set per layer (0 = positive particles,
// 1 = negative), x, y, radius as f32 planes and the escaped flag as a byte;
// the sign is implied by the layer.  Capacity per layer is nx*ny*16 like the
// reference's particle buffers (plugin.rs:212-215).  The live count stays on
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

// Everything the particle kernels touch.  [l] = layer.
struct PlsArgs {
    float* px[2];
    float* py[2];
    float* rad[2];
    uint8_t* esc[2];
    float* qx[2];  // compaction target (reseed), copied back afterwards
    float* qy[2];
    float* qrad[2];
    uint8_t* qesc[2];
    uint32_t* count;          // [2] live particles
    uint32_t* cnt;            // [2][L] particles per cell
    uint32_t* cur;            // [2][L] scatter cursors
    uint32_t* off;            // [2][L] exclusive scan of cnt
    uint32_t* sidx;           // [2][cap] particle index per sorted slot
    uint8_t* alive;           // [2][cap] reseed decision per sorted slot
    unsigned long long* val;  // [2][L] kept | new << 32, then its exclusive scan
    unsigned long long* tot;  // [2] totals of val
    uint32_t* ctot;           // [2] totals of cnt
    uint8_t* addn;            // [2][L] particles to add per cell
    int32_t* phip;            // [L] phi_plus  (fixed point)
    int32_t* phim;            // [L] phi_minus (fixed point)
    uint32_t* dropped;        // particles not stored for lack of capacity
    uint32_t cap;             // per layer
    uint32_t L;               // nx * ny
    int nx, ny;
};

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
    uint32_t n = a.count[l];
    float* px = a.px[l];
    float* py = a.py[l];
    const float third = 1.0f / 3.0f, two_thirds = 2.0f / 3.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float x = px[i], y = py[i];
        float u0 = interp_edge_x(u, x, y), v0 = interp_edge_y(v, x, y);
        float x1 = x + dt * u0, y1 = y + dt * v0;
        float u1 = interp_edge_x(u, x1, y1), v1 = interp_edge_y(v, x1, y1);
        float x2 = 0.75f * x + 0.25f * (x1 + dt * u1), y2 = 0.75f * y + 0.25f * (y1 + dt * v1);
        float u2 = interp_edge_x(u, x2, y2), v2 = interp_edge_y(v, x2, y2);
        px[i] = third * x + two_thirds * (x2 + dt * u2);
        py[i] = third * y + two_thirds * (y2 + dt * v2);
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
    uint32_t n = a.count[l];
    int32_t* phi = l == 0 ? a.phip : a.phim;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float x = a.px[l][i], y = a.py[l][i], r = a.rad[l][i];
        bool e = sgn * interp_center(ls, x, y) + r < 0.0f;
        a.esc[l][i] = e ? 1 : 0;
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
    uint32_t n = a.count[l];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a.rad[l][i] = pls_radius(ls.ld(f2i(a.px[l][i]), f2i(a.py[l][i])));
}

// count_particles_in_cell.wgsl:10-21
__global__ void k_pls_bin(PlsArgs a) {
    const int l = blockIdx.y;
    uint32_t n = a.count[l];
    uint32_t* cnt = a.cnt + (size_t)l * a.L;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&cnt[pls_bin(a.px[l][i], a.py[l][i], (uint32_t)a.nx, a.L)], 1u);
}

// sort_particles.wgsl:12-26: the slot of each particle in its cell's bucket
// (arbitrary order inside the bucket; k_pls_reseed orders it).
__global__ void k_pls_scatter(PlsArgs a) {
    const int l = blockIdx.y;
    uint32_t n = a.count[l];
    const uint32_t* off = a.off + (size_t)l * a.L;
    uint32_t* cur = a.cur + (size_t)l * a.L;
    uint32_t* sidx = a.sidx + (size_t)l * a.cap;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t c = pls_bin(a.px[l][i], a.py[l][i], (uint32_t)a.nx, a.L);
        sidx[off[c] + atomicAdd(&cur[c], 1u)] = i;
    }
}

// ---------------------------------------------------------------------------
// reseed_particles.wgsl:14-148, one thread per cell and layer.
//
// The heap is the reference's, including its index arithmetic: sift_up from
// slot 0 computes the parent (0 - 1) / 2 in u32, and an index past the
// 16-entry array is clamped to 15 (bounds-checked local array access); the
// heap starts zero-initialised.  An eviction of a zero node (capacity used
// up by escaped particles before any insertion) names slot 0 of the whole
// buffer; inside this cell's bucket it applies, for another cell's bucket it
// is the racy write the reference orders arbitrarily -- taken as landing
// before that cell's own writes, i.e. without effect.
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

__global__ void k_pls_reseed(PlsArgs a, PF ls, P2 grad) {
    const int l = blockIdx.y;
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.L) return;
    const float sgn = l == 0 ? 1.0f : -1.0f;
    const int x = (int)(c % (uint32_t)a.nx), y = (int)(c / (uint32_t)a.nx);
    const uint32_t n = a.cnt[(size_t)l * a.L + c];
    const uint32_t off = a.off[(size_t)l * a.L + c];
    uint32_t* b = a.sidx + (size_t)l * a.cap + off;
    uint8_t* alive = a.alive + (size_t)l * a.cap;
    const bool near = fabsf(interp_center(ls, (float)x, (float)y)) < PLS_BAND;

    // stable order: the bucket by particle index
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t v = b[i];
        uint32_t j = i;
        while (j > 0 && b[j - 1] > v) {
            b[j] = b[j - 1];
            --j;
        }
        b[j] = v;
    }

    PlsNode heap[PLS_MAX_PER_CELL];
#pragma unroll
    for (int k = 0; k < PLS_MAX_PER_CELL; ++k) heap[k] = PlsNode{0u, 0.0f};
    uint32_t hcap = PLS_MAX_PER_CELL, hidx = 0;
    auto kill = [&](uint32_t slot) {
        if (slot >= off && slot - off < n) alive[slot] = 0;
    };
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t slot = off + i;
        if (!near) {
            alive[slot] = 0;
            continue;
        }
        uint32_t j = b[i];
        float r = a.rad[l][j];
        float phi = interp_center(ls, a.px[l][j], a.py[l][j]);
        if (sgn * phi + r < 0.0f) {  // escaped
            if (hcap != 0) {
                alive[slot] = 1;
                hcap -= 1;
                if (hidx > hcap) {
                    kill(heap[0].index);
                    heap[0] = heap[hidx - 1];
                    hidx -= 1;
                    pls_correct_heap(heap, hcap);
                }
            } else {
                alive[slot] = 0;
            }
            continue;
        }
        float prio = sgn * phi - r;
        if (hidx < hcap) {
            alive[slot] = 1;
            heap[hidx] = PlsNode{slot, prio};
            hidx += 1;
            pls_sift_up(heap, hidx);
        } else if (prio < heap[0].value) {
            alive[slot] = 1;
            kill(heap[0].index);
            heap[0] = PlsNode{slot, prio};
            pls_correct_heap(heap, hcap);
        } else {
            alive[slot] = 0;
        }
    }
    uint32_t to_add = near ? hcap - hidx : 0u;
    uint32_t kept = 0;
    for (uint32_t i = 0; i < n; ++i) kept += alive[off + i];
    uint32_t fresh = 0;
    for (uint32_t i = 0; i < to_add; ++i) {
        float ox, oy, orad;
        fresh += pls_attempt(false, l, x, y, i, ls, grad, a.nx, a.ny, ox, oy, orad) ? 1u : 0u;
    }
    a.val[(size_t)l * a.L + c] = (unsigned long long)kept | ((unsigned long long)fresh << 32);
    a.addn[(size_t)l * a.L + c] = (uint8_t)to_add;
}

// initialize_particles.wgsl:17-58 with update_interface_band_mask.wgsl:7-17:
// the number of accepted attempts per cell and layer.
__global__ void k_pls_seed_count(PlsArgs a, PF ls, P2 grad) {
    const int l = blockIdx.y;
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.L) return;
    const int x = (int)(c % (uint32_t)a.nx), y = (int)(c / (uint32_t)a.nx);
    uint32_t fresh = 0;
    if (fabsf(ls.ld(x, y)) < PLS_BAND) {
        for (uint32_t i = 0; i < PLS_MAX_PER_CELL; ++i) {
            float ox, oy, orad;
            fresh += pls_attempt(true, l, x, y, i, ls, grad, a.nx, a.ny, ox, oy, orad) ? 1u : 0u;
        }
    }
    a.val[(size_t)l * a.L + c] = (unsigned long long)fresh << 32;
}

// The writes: kept particles of the cell's bucket (reseed), then its new
// ones.  init: new particles are appended to the live set after count[l]
// (initialize_particles.wgsl:44-56 appends to the existing count); reseed:
// kept ones go to the compaction target at their rank, new ones after all
// kept ones (delete_particles.wgsl, update_particles_count.wgsl,
// add_particles.wgsl).
__global__ void k_pls_emit(PlsArgs a, PF ls, P2 grad, int init) {
    const int l = blockIdx.y;
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.L) return;
    const int x = (int)(c % (uint32_t)a.nx), y = (int)(c / (uint32_t)a.nx);
    unsigned long long e = a.val[(size_t)l * a.L + c];
    unsigned long long t = a.tot[l];
    float* dx = init ? a.px[l] : a.qx[l];
    float* dy = init ? a.py[l] : a.qy[l];
    float* dr = init ? a.rad[l] : a.qrad[l];
    uint8_t* de = init ? a.esc[l] : a.qesc[l];
    uint64_t dst;
    uint32_t attempts;
    if (init) {
        dst = (uint64_t)a.count[l] + (e >> 32);
        attempts = fabsf(ls.ld(x, y)) < PLS_BAND ? PLS_MAX_PER_CELL : 0u;
    } else {
        const uint32_t n = a.cnt[(size_t)l * a.L + c];
        const uint32_t off = a.off[(size_t)l * a.L + c];
        const uint32_t* b = a.sidx + (size_t)l * a.cap + off;
        const uint8_t* alive = a.alive + (size_t)l * a.cap + off;
        uint64_t k = e & 0xffffffffull;
        for (uint32_t i = 0; i < n; ++i) {
            if (!alive[i]) continue;
            uint32_t j = b[i];
            if (k < a.cap) {
                dx[k] = a.px[l][j];
                dy[k] = a.py[l][j];
                dr[k] = a.rad[l][j];
                de[k] = a.esc[l][j];
            } else {
                atomicAdd(a.dropped, 1u);
            }
            ++k;
        }
        dst = (t & 0xffffffffull) + (e >> 32);
        attempts = a.addn[(size_t)l * a.L + c];
    }
    for (uint32_t i = 0; i < attempts; ++i) {
        float ox, oy, orad;
        if (!pls_attempt(init != 0, l, x, y, i, ls, grad, a.nx, a.ny, ox, oy, orad)) continue;
        if (dst < a.cap) {
            dx[dst] = ox;
            dy[dst] = oy;
            dr[dst] = orad;
            de[dst] = 0;
        } else {
            atomicAdd(a.dropped, 1u);
        }
        ++dst;
    }
}

// New live counts (capped at the capacity; the overflow is in a.dropped).
__global__ void k_pls_set_count(PlsArgs a, int init) {
    int l = threadIdx.x;
    if (l >= 2) return;
    unsigned long long t = a.tot[l];
    uint64_t n = init ? (uint64_t)a.count[l] + (t >> 32) : (t & 0xffffffffull) + (t >> 32);
    a.count[l] = (uint32_t)(n < a.cap ? n : a.cap);
}

// The compacted set back into the live arrays.
__global__ void k_pls_copyback(PlsArgs a) {
    const int l = blockIdx.y;
    uint32_t n = a.count[l];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a.px[l][i] = a.qx[l][i];
        a.py[l][i] = a.qy[l][i];
        a.rad[l][i] = a.qrad[l][i];
        a.esc[l][i] = a.qesc[l][i];
    }
}

}  // namespace efl
