// efl_kernels.cuh — sm_100a kernels of the per-step Eulerian fluid path.
//
// Each kernel computes what one WGSL entry point of the reference computes
// (file:line cited per kernel), over the same invocation domain, with the
// same floating-point operation order.  The library is built with
// -fmad=false and IEEE division/sqrt so that results are bit-identical to
// the CPU restatement wherever the reference's math is not
// implementation-defined (exp is the only such function on this path).
//
// Device layout: every field is one pitched f32 plane (pitch P floats,
// P = round_up(nx + 1, 32), 128-byte aligned rows).  Cell (x, y), x-face
// (x, y) and y-face (x, y) all live at y * P + x.  Area fractions are kept
// as two face planes fu ((nx+1) x ny) and fv (nx x (ny+1)) instead of the
// reference's per-cell RGBA: the reference computes the fraction of a face
// shared by two cells from the same four level-set samples in the same
// order on both sides, so one value per face is exact and halves the bytes
// the projection reads.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/efl.h"

namespace efl {

#define EFL_DEV __device__ __forceinline__

// Number of kernels this library has launched (all simulations, all
// devices).  Evaluated in every launch configuration as the dynamic
// shared-memory size argument, which it leaves at 0.
uint64_t launches_total();
size_t count_launch();

constexpr float LARGE_FLOAT = 1.0e6f;      // update_solid.wgsl:4, update_fluid_source.wgsl:22
constexpr float FIM_LARGE = 1e30f;         // fast_iterative_method/initialize.wgsl:5
constexpr float FIM_EPS = 1e-6f;           // fast_iterative_method/update.wgsl:9
constexpr float SQRT2_F = 1.41421356237309504880f;
constexpr uint32_t LABEL_NONE = 0, LABEL_SOURCE = 1, LABEL_ACTIVE = 2, LABEL_CONVERGED = 3;

struct Uniform {  // fluid_uniform.wgsl:3-10
    float dx, dt, rho;
    float g[2];
    float m[16];
    float size[2];
};

// A pitched plane with its logical extent.
template <class T>
struct Plane {
    T* p;
    int w, h, P;
    EFL_DEV bool in(int x, int y) const { return (unsigned)x < (unsigned)w && (unsigned)y < (unsigned)h; }
    EFL_DEV T ld(int x, int y) const { return in(x, y) ? p[(size_t)y * P + x] : T{}; }
    EFL_DEV void st(int x, int y, T v) const { if (in(x, y)) p[(size_t)y * P + x] = v; }
    EFL_DEV T& at(int x, int y) const { return p[(size_t)y * P + x]; }
};
using PF = Plane<float>;
using PI = Plane<int32_t>;
using PU = Plane<uint32_t>;
using P2 = Plane<float2>;

// WGSL helpers ---------------------------------------------------------------
EFL_DEV float fclamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
EFL_DEV float fclampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
EFL_DEV float wsign(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
EFL_DEV float wlength(float x, float y) { return sqrtf(x * x + y * y); }
EFL_DEV float wmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
EFL_DEV int f2i(float v) { return __float2int_rz(v); }  // truncate, saturate, NaN -> 0
EFL_DEV float2 mat_xy(const float* m, float x, float y) {
    float2 r;
    r.x = ((m[0] * x + m[4] * y) + m[8] * 0.0f) + m[12] * 1.0f;
    r.y = ((m[1] * x + m[5] * y) + m[9] * 0.0f) + m[13] * 1.0f;
    return r;
}
EFL_DEV float det4(const float* m) {
#define A_(r, c) m[(c)*4 + (r)]
    float s0 = A_(0, 0) * A_(1, 1) - A_(1, 0) * A_(0, 1);
    float s1 = A_(0, 0) * A_(1, 2) - A_(1, 0) * A_(0, 2);
    float s2 = A_(0, 0) * A_(1, 3) - A_(1, 0) * A_(0, 3);
    float s3 = A_(0, 1) * A_(1, 2) - A_(1, 1) * A_(0, 2);
    float s4 = A_(0, 1) * A_(1, 3) - A_(1, 1) * A_(0, 3);
    float s5 = A_(0, 2) * A_(1, 3) - A_(1, 2) * A_(0, 3);
    float c5 = A_(2, 2) * A_(3, 3) - A_(3, 2) * A_(2, 3);
    float c4 = A_(2, 1) * A_(3, 3) - A_(3, 1) * A_(2, 3);
    float c3 = A_(2, 1) * A_(3, 2) - A_(3, 1) * A_(2, 2);
    float c2 = A_(2, 0) * A_(3, 3) - A_(3, 0) * A_(2, 3);
    float c1 = A_(2, 0) * A_(3, 2) - A_(3, 0) * A_(2, 2);
    float c0 = A_(2, 0) * A_(3, 1) - A_(3, 0) * A_(2, 1);
#undef A_
    return s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
}

// utils/area_fraction.wgsl:10-12
EFL_DEV float area_fraction(float l0, float l1) { return fclamp01(fmaxf(l0, l1) / fabsf(l0 - l1)); }
// utils/area_fraction.wgsl:14-56 -> (i-1/2, i+1/2, j-1/2, j+1/2)
EFL_DEV float4 area_fractions(const PF& ls, int x, int y) {
    float c0 = ls.ld(x - 1, y - 1), c1 = ls.ld(x, y - 1), c2 = ls.ld(x + 1, y - 1);
    float c3 = ls.ld(x - 1, y), c4 = ls.ld(x, y), c5 = ls.ld(x + 1, y);
    float c6 = ls.ld(x - 1, y + 1), c7 = ls.ld(x, y + 1), c8 = ls.ld(x + 1, y + 1);
    float mm = 0.25f * (c0 + c1 + c3 + c4);
    float pm = 0.25f * (c1 + c2 + c4 + c5);
    float mp = 0.25f * (c3 + c4 + c6 + c7);
    float pp = 0.25f * (c4 + c5 + c7 + c8);
    return make_float4(area_fraction(mm, mp), area_fraction(pm, pp), area_fraction(mm, pm), area_fraction(mp, pp));
}

// Dispatch-domain helpers (pipeline.rs:175-186).
struct Dom {
    int nx, ny;
    EFL_DEV int cx() const { return (nx / 8) * 8; }
    EFL_DEV int cy() const { return (ny / 8) * 8; }
    EFL_DEV int xrows() const { return (ny / 64) * 64; }
    EFL_DEV int ycols() const { return (nx / 64) * 64; }
};

EFL_DEV int gx() { return blockIdx.x * blockDim.x + threadIdx.x; }
EFL_DEV int gy() { return blockIdx.y * blockDim.y + threadIdx.y; }

// ---------------------------------------------------------------------------
// initialize_grid_center.wgsl:5-15
__global__ void k_init_center(PF ls0, PF ls1, P2 grad, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float level = (float)(uint32_t)(d.ny - y);
    ls0.st(x, y, level);
    ls1.st(x, y, level);
    grad.st(x, y, make_float2(0.0f, -1.0f));
}
// initialize_grid_edge.wgsl:6-17, (nx+1, ny/64) x (1, 64); v index transposed
__global__ void k_init_edge(PF u0, PF u1, PF v0, PF v1, Dom d) {
    int x = gx(), y = gy();
    if (x > d.nx || y >= d.xrows()) return;
    u0.st(x, y, 0.0f);
    v0.st(y, x, 0.0f);
    u1.st(x, y, 0.0f);
    v1.st(y, x, 0.0f);
}

// update_solid.wgsl:80-85
EFL_DEV float2 to_world(const Uniform& U, float px, float py, int nx, int ny) {
    float uvx = px / (float)nx, uvy = py / (float)ny;
    float xx = (uvx - 0.5f) * U.size[0];
    float yy = (-uvy + 0.5f) * U.size[1];
    return mat_xy(U.m, xx, yy);
}
// update_solid.wgsl:164-175
EFL_DEV float dist_segment(float2 x, float2 a, float2 b) {
    float abx = b.x - a.x, aby = b.y - a.y;
    float t = fclampf(((x.x - a.x) * abx + (x.y - a.y) * aby) / (abx * abx + aby * aby), 0.0f, 1.0f);
    float px = a.x + t * abx, py = a.y + t * aby;
    return wlength(x.x - px, x.y - py);
}
EFL_DEV float dist_sign(float2 x, float2 a, float2 b) {
    float x1x = x.x - a.x, x1y = x.y - a.y;
    float abx = b.x - a.x, aby = b.y - a.y;
    return wsign(x1y * abx - x1x * aby);
}
// update_solid.wgsl:87-109
EFL_DEV float level_rectangle(const efl_solid_obstacle& o, float2 x) {
    float level = LARGE_FLOAT;
    if (det4(o.transform) == 0.0f) return level;
    float2 x0 = mat_xy(o.inverse_transform, x.x, x.y);
    float hx = o.values[0], hy = o.values[1];
    bool ix = fabsf(x0.x) < hx, iy = fabsf(x0.y) < hy;
    if (ix) level = iy ? fmaxf(fabsf(x0.x) - hx, fabsf(x0.y) - hy) : fabsf(x0.y) - hy;
    else level = iy ? fabsf(x0.x) - hx : wlength(fabsf(x0.x) - hx, fabsf(x0.y) - hy);
    return level;
}
// update_solid.wgsl:121-162
EFL_DEV float level_obstacle(const efl_solid_obstacle& o, float2 x) {
    switch (o.shape) {
        case EFL_SHAPE_CIRCLE:
            return wlength(x.x - o.transform[12], x.y - o.transform[13]) - o.values[0];
        case EFL_SHAPE_RECTANGLE:
            return level_rectangle(o, x);
        case EFL_SHAPE_CAPSULE: {
            float2 a = mat_xy(o.transform, o.values[0], o.values[1]);
            float2 b = mat_xy(o.transform, o.values[2], o.values[3]);
            return dist_segment(x, a, b) - o.values[4];
        }
        case EFL_SHAPE_TRIANGLE: {
            float2 p0 = mat_xy(o.transform, o.values[0], o.values[1]);
            float2 p1 = mat_xy(o.transform, o.values[2], o.values[3]);
            float2 p2 = mat_xy(o.transform, o.values[4], o.values[5]);
            float d0 = dist_segment(x, p0, p1), d1 = dist_segment(x, p1, p2), d2 = dist_segment(x, p2, p0);
            float s0 = dist_sign(x, p0, p1), s1 = dist_sign(x, p1, p2), s2 = dist_sign(x, p2, p0);
            float m = fminf(fminf(d0, d1), d2);
            return (s0 > 0.0f && s1 > 0.0f && s2 > 0.0f) ? -m : m;
        }
        default:
            return LARGE_FLOAT;
    }
}
EFL_DEV float2 velocity_at(const efl_solid_obstacle& o, float2 x) {  // update_solid.wgsl:111-119
    float rx = x.x - o.transform[12], ry = x.y - o.transform[13];
    float w = o.angular_velocity;
    return make_float2(o.linear_velocity[0] + -w * ry, o.linear_velocity[1] + w * rx);
}

// update_solid.wgsl:15-78.  Obstacles are staged through shared memory in
// chunks; every invocation walks them in index order as the reference does.
constexpr int OBS_CHUNK = 32;
__global__ void k_update_solid(PF us, PF vs, PF ls_s, PI sid, const efl_solid_obstacle* __restrict__ obs, int n_obs,
                               Uniform U, Dom d) {
    __shared__ efl_solid_obstacle so[OBS_CHUNK];
    int x = gx(), y = gy();
    const int nx = d.nx, ny = d.ny;
    bool active = x < d.cx() && y < d.cy();
    bool border = x == 0 || y == 0 || x == nx - 1 || y == ny - 1;
    float2 xc = to_world(U, (float)x, (float)y, nx, ny);
    float2 xex = to_world(U, (float)x - 0.5f, (float)y - 0.0f, nx, ny);
    float2 xey = to_world(U, (float)x - 0.0f, (float)y - 0.5f, nx, ny);
    int tx = min(x, abs(nx - 1 - x)), ty = min(y, abs(ny - 1 - y));
    float level = (float)min(tx, ty);
    float u = 0.0f, v = 0.0f;
    int32_t id = -1;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nthreads = blockDim.x * blockDim.y;
    for (int base = 0; base < n_obs; base += OBS_CHUNK) {
        int cnt = min(OBS_CHUNK, n_obs - base);
        __syncthreads();
        const int words = cnt * (int)(sizeof(efl_solid_obstacle) / 4);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(obs + base);
        uint32_t* dst = reinterpret_cast<uint32_t*>(so);
        for (int i = tid; i < words; i += nthreads) dst[i] = src[i];
        __syncthreads();
        if (active && !border) {
            for (int k = 0; k < cnt; ++k) {
                const efl_solid_obstacle& o = so[k];
                float lo = level_obstacle(o, xc);
                if (lo < level) level = lo;
                if (lo < 0.5f) id = (int32_t)o.entity_id;
                float lex = level_obstacle(o, xex);
                if (lex < 0.5f) u = velocity_at(o, xex).x;
                float ley = level_obstacle(o, xey);
                if (ley < 0.5f) v = -velocity_at(o, xey).y;
            }
        }
    }
    if (!active) return;
    if (border) {
        ls_s.st(x, y, 0.0f);
        us.st(x, y, 0.0f);
        vs.st(x, y, 0.0f);
        sid.st(x, y, -1);
        return;
    }
    us.st(x, y, u);
    vs.st(x, y, v);
    ls_s.st(x, y, level);
    sid.st(x, y, id);
}

// update_area_fraction.wgsl:6-14, written as face planes.
__global__ void k_area_fraction(PF ls_s, PF fu, PF fv, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float4 f = area_fractions(ls_s, x, y);
    fu.st(x, y, f.x);
    fv.st(x, y, f.z);
    if (x == d.nx - 1) fu.st(x + 1, y, f.y);
    if (y == d.ny - 1) fv.st(x, y + 1, f.w);
}

// utils/coordinate.wgsl:51-94
EFL_DEV float interp_edge_x(const PF& u, float px, float py) {
    int i = f2i(rintf(px));
    int j = f2i(floorf(py));
    float fi = px + 0.5f - (float)i;
    float fj = py - (float)j;
    float u00 = u.ld(i, j), u10 = u.ld(i + 1, j), u01 = u.ld(i, j + 1), u11 = u.ld(i + 1, j + 1);
    return wmix(wmix(u00, u10, fi), wmix(u01, u11, fi), fj);
}
EFL_DEV float interp_edge_y(const PF& v, float px, float py) {
    int i = f2i(floorf(px));
    int j = f2i(rintf(py));
    float fi = px - (float)i;
    float fj = py + 0.5f - (float)j;
    float v00 = v.ld(i, j), v10 = v.ld(i + 1, j), v01 = v.ld(i, j + 1), v11 = v.ld(i + 1, j + 1);
    return wmix(wmix(v00, v10, fi), wmix(v01, v11, fi), fj);
}
EFL_DEV float2 runge_kutta(const PF& u, const PF& v, float px, float py, float dt) {
    float vx = interp_edge_x(u, px, py), vy = interp_edge_y(v, px, py);
    float h = 0.5f * dt;
    float mx = px - h * vx, my = py - h * vy;
    float wx = interp_edge_x(u, mx, my), wy = interp_edge_y(v, mx, my);
    return make_float2(px - dt * wx, py - dt * wy);
}
// advect_velocity.wgsl:11-27 (x-major) and :29-45 (y-major)
EFL_DEV void advect_u_at(const PF& u0, const PF& v0, const PF& u1, float dt, const Dom& d) {
    int x = gx(), y = gy();
    if (x > d.nx || y >= d.xrows()) return;
    float px = (float)x + -0.5f, py = (float)y + 0.0f;
    float2 b = runge_kutta(u0, v0, px, py, dt);
    float dimx = (float)u0.w, dimy = (float)u0.h;
    bool inside = b.x >= 0.0f && b.y >= 0.0f && b.x <= dimx - 1.0f && b.y <= dimy - 1.0f;
    u1.st(x, y, inside ? interp_edge_x(u0, b.x, b.y) : u0.ld(x, y));
}
EFL_DEV void advect_v_at(const PF& u0, const PF& v0, const PF& v1, float dt, const Dom& d) {
    int x = gx(), y = gy();
    if (x >= d.ycols() || y > d.ny) return;
    float px = (float)x + 0.0f, py = (float)y + -0.5f;
    float2 b = runge_kutta(u0, v0, px, py, dt);
    float dimx = (float)v0.w, dimy = (float)v0.h;
    bool inside = b.x >= 0.0f && b.y >= 0.0f && b.x <= dimx - 1.0f && b.y <= dimy - 1.0f;
    v1.st(x, y, inside ? interp_edge_y(v0, b.x, b.y) : v0.ld(x, y));
}
// Both passes in one launch over the larger of their grids: blockIdx.z 0 the x-major faces, 1 the y-major ones.
__global__ void k_advect_uv(PF u0, PF v0, PF u1, PF v1, float dt, Dom d) {
    if (blockIdx.z == 0)
        advect_u_at(u0, v0, u1, dt, d);
    else
        advect_v_at(u0, v0, v1, dt, d);
}

// exp for the Gaussian force splat.  WGSL's exp is implementation-defined
// (any few-ulp result is conforming), so the library and the CPU oracle both
// evaluate this restatement of the Cody-Waite method: x = k ln2 + r with ln2
// split into an exactly-multipliable high part and a low part, |r| <= ln2/2,
// exp(r) by its degree-7 Taylor polynomial in Horner form (truncation error
// < 1e-8 relative), exact scaling by 2^k.  Within 2 ulp of exp.
EFL_DEV float efl_exp(float x) {
    if (x < -104.0f) return 0.0f;
    if (x > 88.5f) return __int_as_float(0x7f800000);
    float kf = rintf(x * 1.44269504088896341f);
    float r = (x - kf * 0.693145751953125f) - kf * 1.42860682030941723e-6f;
    float p = 1.98412698412698413e-4f;  // 1/7!
    p = p * r + 1.38888888888888889e-3f;
    p = p * r + 8.33333333333333333e-3f;
    p = p * r + 4.16666666666666667e-2f;
    p = p * r + 1.66666666666666667e-1f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    return ldexpf(p, (int)kf);
}
// apply_forces.wgsl:73-76
EFL_DEV float gaussian_2d(float x, float y, float x0, float y0, float sigma) {
    float b = -1.0f / (2.0f * sigma * sigma);
    float dx = x - x0, dy = y - y0;
    return efl_exp(b * (dx * dx + dy * dy));
}
// apply_forces.wgsl:17-43 / 45-71 (comp 0 = u, x-major; comp 1 = v, y-major)
template <int COMP>
EFL_DEV void apply_forces_at(const PF& vel, const PF& ls0, const PF& face_frac, const efl_force* __restrict__ forces,
                             int n_forces, const Uniform& U, const Dom& d) {
    int x = gx(), y = gy();
    if (COMP == 0 ? (x > d.nx || y >= d.xrows()) : (x >= d.ycols() || y > d.ny)) return;
    float4 f = area_fractions(ls0, x, y);
    float fair = COMP == 0 ? f.x : f.z;
    // af(idx).x / af(idx).z; outside the cell texture the reference reads 0,
    // and the face planes hold 0 there too (border faces of the solid ring).
    float fs = (x < d.nx && y < d.ny) ? face_frac.ld(x, y) : 0.0f;
    if (fair == 1.0f || fs == 0.0f) {
        vel.st(x, y, 0.0f);
        return;
    }
    float net = U.g[COMP];
    for (int n = n_forces; n > 0; --n) {
        const efl_force F = forces[n - 1];
        net = net + F.force[COMP] * gaussian_2d((float)x, (float)y, F.position[0], F.position[1], 10.0f);
    }
    float val = vel.ld(x, y);
    vel.st(x, y, val + net * U.dt / U.dx);
}
// Both components in one launch over the larger of their grids (blockIdx.z: 0 = u, 1 = v).
__global__ void k_apply_forces_uv(PF u, PF v, PF ls0, PF fu, PF fv, const efl_force* __restrict__ forces, int n_forces,
                                  Uniform U, Dom d) {
    if (blockIdx.z == 0)
        apply_forces_at<0>(u, ls0, fu, forces, n_forces, U, d);
    else
        apply_forces_at<1>(v, ls0, fv, forces, n_forces, U, d);
}

// divergence.wgsl:16-42 (fractions of levelset_solid = the face planes)
__global__ void k_divergence(PF u1, PF v1, PF us, PF vs, PF fu, PF fv, PF div, float dx, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float fx0 = fu.ld(x, y), fx1 = fu.ld(x + 1, y), fy0 = fv.ld(x, y), fy1 = fv.ld(x, y + 1);
    float u_ij = u1.ld(x, y), u_ip = u1.ld(x + 1, y);
    float v_ij = v1.ld(x, y), v_jp = v1.ld(x, y + 1);
    float du_f = fx1 * u_ip - fx0 * u_ij;
    float dv_f = fy1 * v_jp - fy0 * v_ij;
    float us_m = us.ld(x, y), us_p = us.ld(x + 1, y);
    float vs_m = vs.ld(x, y), vs_p = vs.ld(x, y + 1);
    float du_s = (1.0f - fx1) * us_p - (1.0f - fx0) * us_m;
    float dv_s = (1.0f - fy1) * vs_p - (1.0f - fy0) * vs_m;
    div.st(x, y, -(du_f + dv_f + du_s + dv_s) / dx);
}

// One level of the pressure system: iterate x, right-hand side b and
// residual r of type T (f32: the reference's fixed-count solve; f64: the
// tolerance-driven solve), with the level's f32 air level set and face
// fractions.
template <class T>
struct LevelT {
    Plane<T> x, b, r;
    PF ls, fu, fv;
    int nx, ny;
};
using Level = LevelT<float>;
using Level64 = LevelT<double>;

// projection/shaders/gauss_seidel.wgsl:44-88.  T = float is the reference's
// arithmetic; T = double evaluates the same expression tree in f64 from the
// f32 inputs.
template <class T>
EFL_DEV T gs_update(const LevelT<T>& L, T c_div, T weight, int x, int y) {
    float lij = L.ls.at(x, y);
    if (lij >= 0.0f) return T(0);
    float f0 = L.fu.at(x, y), f1 = L.fu.at(x + 1, y), f2 = L.fv.at(x, y), f3 = L.fv.at(x, y + 1);
    T p_old = L.x.at(x, y);
    if (f0 == 0.0f && f1 == 0.0f && f2 == 0.0f && f3 == 0.0f) return T(0);
    T denom = T(0);
    T nume = c_div * L.b.at(x, y);
    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    const T fvv[4] = {(T)f0, (T)f1, (T)f2, (T)f3};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int jx = x + ox[i], jy = y + oy[i];
        if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
            float level = L.ls.at(jx, jy);
            if (level < 0.0f) {
                denom += fvv[i];
                nume += fvv[i] * L.x.at(jx, jy);
            } else {
                denom += fvv[i] * (T(1) - (T)level / (T)lij);
            }
        }
    }
    if (fabs(denom) < (T)1.0e-6f) return T(0);
    // f32: the reference's division; f64 (tolerance-driven, an extension):
    // nume * (1/denom), the form the persistent solver evaluates.
    T p_new;
    if constexpr (sizeof(T) == 8) p_new = nume * (T(1) / denom);
    else p_new = nume / denom;
    return weight * p_new + (T(1) - weight) * p_old;
}
// ((dx*dx)*rho)/dt as gauss_seidel.wgsl:58 evaluates it, dx = resolution_scale*dx.
template <class T>
EFL_DEV T gs_cdiv(float dx_scaled, float rho, float dt) {
    T d = (T)dx_scaled;
    return d * d * (T)rho / (T)dt;
}
// gauss_seidel.wgsl:12-42: colour 1 = red ((x+y) odd), 0 = black.  One
// thread per cell of the colour.
template <class T>
__global__ void k_gs_color(LevelT<T> L, float dx_scaled, float rho, float dt, float weight, int color) {
    int tx = gx(), y = gy();
    int x = 2 * tx + ((y + color) & 1);
    if (x >= L.nx || y >= L.ny) return;
    L.x.at(x, y) = gs_update(L, gs_cdiv<T>(dx_scaled, rho, dt), (T)weight, x, y);
}

// projection/shaders/residual.wgsl:12-57
template <class T>
EFL_DEV T residual_factor(float dt, float rho, float dx_scaled) {
    T d = (T)dx_scaled;
    return (T)dt / (T)rho / d / d;
}
// f32: the reference's operation order.  f64: the same operator in
// factored form r = b - factor * (denom * x - sum_fluid f * x_nb), denom
// accumulated in the reference's neighbour order.
template <class T>
EFL_DEV T residual_at(const LevelT<T>& L, T factor, int x, int y, bool* counted) {
    *counted = false;
    float phi = L.ls.at(x, y);
    if (phi >= 0.0f) return T(0);
    float f0 = L.fu.at(x, y), f1 = L.fu.at(x + 1, y), f2 = L.fv.at(x, y), f3 = L.fv.at(x, y + 1);
    if (f0 == 0.0f && f1 == 0.0f && f2 == 0.0f && f3 == 0.0f) return T(0);
    *counted = true;
    T xc = L.x.at(x, y);
    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    const T fvv[4] = {(T)f0, (T)f1, (T)f2, (T)f3};
    if constexpr (sizeof(T) == 8) {
        T denom = T(0), sum = T(0);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int jx = x + ox[i], jy = y + oy[i];
            if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                float pn = L.ls.at(jx, jy);
                if (pn < 0.0f) {
                    denom += fvv[i];
                    sum += fvv[i] * L.x.at(jx, jy);
                } else {
                    denom += fvv[i] * (T(1) - (T)pn / (T)phi);
                }
            }
        }
        return L.b.at(x, y) - factor * (denom * xc - sum);
    } else {
        T r = L.b.at(x, y);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int jx = x + ox[i], jy = y + oy[i];
            if ((unsigned)jx < (unsigned)L.nx && (unsigned)jy < (unsigned)L.ny) {
                float pn = L.ls.at(jx, jy);
                if (pn < 0.0f) r -= fvv[i] * (xc - L.x.at(jx, jy)) * factor;
                else r -= fvv[i] * (T(1) - (T)pn / (T)phi) * xc * factor;
            }
        }
        return r;
    }
}
template <class T>
__global__ void k_residual(LevelT<T> L, float dt, float rho, float dx_scaled) {
    int x = gx(), y = gy();
    if (x >= L.nx || y >= L.ny) return;
    bool c;
    L.r.at(x, y) = residual_at(L, residual_factor<T>(dt, rho, dx_scaled), x, y, &c);
}
// restriction.wgsl:10-60 (the fractions on face planes)
// The coarse cell (x, y) from its four children's residuals r(2x + i, 2y + j) = rij (0 outside the level).
template <class T>
EFL_DEV void restrict_from(const LevelT<T>& F, const LevelT<T>& C, int x, int y, T r00, T r01, T r10, T r11) {
    int fx = 2 * x, fy = 2 * y;
    T br = T(0.25) * (r00 + r01 + r10 + r11);
    float ph0 = F.ls.ld(fx, fy), ph1 = F.ls.ld(fx, fy + 1), ph2 = F.ls.ld(fx + 1, fy), ph3 = F.ls.ld(fx + 1, fy + 1);
    float pr = ph0;
    if (fabsf(ph1) < fabsf(pr)) pr = ph1;
    if (fabsf(ph2) < fabsf(pr)) pr = ph2;
    if (fabsf(ph3) < fabsf(pr)) pr = ph3;
    C.b.at(x, y) = br;
    C.ls.at(x, y) = pr;
    C.fu.at(x, y) = 0.5f * (F.fu.ld(fx, fy) + F.fu.ld(fx, fy + 1));
    C.fv.at(x, y) = 0.5f * (F.fv.ld(fx, fy) + F.fv.ld(fx + 1, fy));
    if (x == C.nx - 1) C.fu.at(x + 1, y) = 0.5f * (F.fu.ld(fx + 2, fy) + F.fu.ld(fx + 2, fy + 1));
    if (y == C.ny - 1) C.fv.at(x, y + 1) = 0.5f * (F.fv.ld(fx, fy + 2) + F.fv.ld(fx + 1, fy + 2));
    C.x.at(x, y) = T(0);
}
template <class T>
EFL_DEV void restrict_cell(const LevelT<T>& F, const LevelT<T>& C, int x, int y) {
    int fx = 2 * x, fy = 2 * y;
    restrict_from(F, C, x, y, F.r.ld(fx, fy), F.r.ld(fx, fy + 1), F.r.ld(fx + 1, fy), F.r.ld(fx + 1, fy + 1));
}
// The residual (k_residual) and the restriction in one pass: each coarse cell computes its four children's
// residuals (residual_at, 0 outside the level, as the residual plane reads there) and restricts them, so the
// fine residual plane is neither written nor read back.  The same values, in the same order.
template <class T>
__global__ void k_residual_restrict(LevelT<T> F, LevelT<T> C, float dt, float rho, float dx_scaled) {
    int x = gx(), y = gy();
    if (x >= C.nx || y >= C.ny) return;
    const T fac = residual_factor<T>(dt, rho, dx_scaled);
    auto rr = [&](int ax, int ay) -> T {
        bool c;
        return (ax < F.nx && ay < F.ny) ? residual_at(F, fac, ax, ay, &c) : T(0);
    };
    const int fx = 2 * x, fy = 2 * y;
    const T r00 = rr(fx, fy), r01 = rr(fx, fy + 1), r10 = rr(fx + 1, fy), r11 = rr(fx + 1, fy + 1);
    restrict_from(F, C, x, y, r00, r01, r10, r11);
}
// prolongation.wgsl:5-34
template <class T>
EFL_DEV void prolong_cell(const LevelT<T>& F, const LevelT<T>& C, int x, int y) {
    T corr = C.x.at(x, y);
    const int ox[4] = {0, 1, 0, 1}, oy[4] = {0, 0, 1, 1};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int fx = 2 * x + ox[i], fy = 2 * y + oy[i];
        if (F.ls.ld(fx, fy) < 0.0f && F.x.in(fx, fy)) F.x.at(fx, fy) = corr + F.x.at(fx, fy);
    }
}
template <class T>
__global__ void k_prolongation(LevelT<T> F, LevelT<T> C) {
    int x = gx(), y = gy();
    if (x >= C.nx || y >= C.ny) return;
    prolong_cell(F, C, x, y);
}

// The coarse tail of a V-cycle (multi_grid.rs:390-475) in ONE launch of one
// CTA: every level from `first` down (each at most VT_MAX_CELLS cells, held
// in L2) with block barriers between the steps instead of a launch per
// half-sweep, residual, restriction and prolongation.  Same per-cell
// functions and the same step order as the launch-per-step form (smoother
// weight 1, resolution scale 2^level; `symmetric`: post-smoothing black then
// red), so the result is identical.
constexpr int VT_THREADS = 1024, VT_MAX_LEVELS = 14;
constexpr int VT_MAX_CELLS = 128 * 128;
template <class T>
struct VTailArgs {
    LevelT<T> lv[VT_MAX_LEVELS];
    int first, count;  // levels first .. count - 1
    float dx, rho, dt;
    int pre, post, coarsest, symmetric;
};
template <class T>
EFL_DEV void vt_sweeps(const LevelT<T>& L, float dxs, float rho, float dt, int n, int c0) {
    const T cd = gs_cdiv<T>(dxs, rho, dt);
    const int hw = (L.nx + 1) / 2;
    for (int k = 0; k < n; ++k) {
        for (int h = 0; h < 2; ++h) {
            const int color = h == 0 ? c0 : 1 - c0;
            for (int i = threadIdx.x; i < hw * L.ny; i += VT_THREADS) {
                const int y = i / hw, x = 2 * (i - y * hw) + ((y + color) & 1);
                if (x < L.nx) L.x.at(x, y) = gs_update(L, cd, T(1), x, y);
            }
            __syncthreads();
        }
    }
}
template <class T>
__global__ void __launch_bounds__(VT_THREADS, 1) k_vcycle_tail(VTailArgs<T> a) {
    const int last = a.count - 1;
    // down: pre-smoothing, residual, restriction
    for (int i = a.first; i < last; ++i) {
        const LevelT<T>& L = a.lv[i];
        const LevelT<T>& C = a.lv[i + 1];
        const float dxs = (float)(1u << i) * a.dx;
        vt_sweeps(L, dxs, a.rho, a.dt, a.pre, 1);
        const T fac = residual_factor<T>(a.dt, a.rho, dxs);
        for (int j = threadIdx.x; j < L.nx * L.ny; j += VT_THREADS) {
            const int y = j / L.nx, x = j - y * L.nx;
            bool c;
            L.r.at(x, y) = residual_at(L, fac, x, y, &c);
        }
        __syncthreads();
        for (int j = threadIdx.x; j < C.nx * C.ny; j += VT_THREADS) {
            const int y = j / C.nx;
            restrict_cell(L, C, j - y * C.nx, y);
        }
        __syncthreads();
    }
    vt_sweeps(a.lv[last], (float)(1u << last) * a.dx, a.rho, a.dt, a.coarsest, 1);
    // up: prolongation, post-smoothing
    for (int i = last - 1; i >= a.first; --i) {
        const LevelT<T>& L = a.lv[i];
        const LevelT<T>& C = a.lv[i + 1];
        for (int j = threadIdx.x; j < C.nx * C.ny; j += VT_THREADS) {
            const int y = j / C.nx;
            prolong_cell(L, C, j - y * C.nx, y);
        }
        __syncthreads();
        vt_sweeps(L, (float)(1u << i) * a.dx, a.rho, a.dt, a.post, a.symmetric ? 0 : 1);
    }
}

// Residual norms ||r||^2, ||b||^2 over cells with phi < 0 that are not
// fully solid; FP64, warp-shuffle + block reduction, per-block partials
// summed in block order by k_norm_finalize (deterministic).
constexpr int NORM_THREADS = 256;
EFL_DEV double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
__global__ void __launch_bounds__(NORM_THREADS)
    k_residual_norm(LevelT<T> L, float dt, float rho, float dx, double2* partials) {
    __shared__ double sr[NORM_THREADS / 32], sb[NORM_THREADS / 32];
    const T factor = residual_factor<T>(dt, rho, dx);
    const int n = L.nx * L.ny;
    double ar = 0.0, ab = 0.0;
    for (int i = blockIdx.x * NORM_THREADS + threadIdx.x; i < n; i += gridDim.x * NORM_THREADS) {
        int y = i / L.nx, x = i - y * L.nx;
        bool c;
        T r = residual_at(L, factor, x, y, &c);
        if (c) {
            double b = (double)L.b.at(x, y);
            ar += (double)r * (double)r;
            ab += b * b;
        }
    }
    ar = warp_sum(ar);
    ab = warp_sum(ab);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sr[w] = ar;
        sb[w] = ab;
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
// Post-projection divergence diagnostic: the operator of divergence.wgsl:16-42
// applied to the projected velocity (u0, v0) at the cells the residual
// counts (phi < 0, not fully solid).  Per block: x = FP64 sum of squares,
// y = the largest magnitude; k_div_norm_finalize sums x in block order and
// takes the maximum of y (deterministic).
__global__ void __launch_bounds__(NORM_THREADS)
    k_divergence_norm(PF u0, PF v0, PF us, PF vs, PF fu, PF fv, PF ls0, float dx, Dom d, double2* partials) {
    __shared__ double ss[NORM_THREADS / 32], sm[NORM_THREADS / 32];
    const int n = d.nx * d.ny;
    double a2 = 0.0, amax = 0.0;
    for (int i = blockIdx.x * NORM_THREADS + threadIdx.x; i < n; i += gridDim.x * NORM_THREADS) {
        const int y = i / d.nx, x = i - y * d.nx;
        if (!(ls0.at(x, y) < 0.0f)) continue;
        const float fx0 = fu.ld(x, y), fx1 = fu.ld(x + 1, y), fy0 = fv.ld(x, y), fy1 = fv.ld(x, y + 1);
        if (fx0 == 0.0f && fx1 == 0.0f && fy0 == 0.0f && fy1 == 0.0f) continue;
        const float du_f = fx1 * u0.ld(x + 1, y) - fx0 * u0.ld(x, y);
        const float dv_f = fy1 * v0.ld(x, y + 1) - fy0 * v0.ld(x, y);
        const float du_s = (1.0f - fx1) * us.ld(x + 1, y) - (1.0f - fx0) * us.ld(x, y);
        const float dv_s = (1.0f - fy1) * vs.ld(x, y + 1) - (1.0f - fy0) * vs.ld(x, y);
        const double dv = (double)(-(du_f + dv_f + du_s + dv_s) / dx);
        a2 += dv * dv;
        amax = fmax(amax, fabs(dv));
    }
    a2 = warp_sum(a2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        ss[w] = a2;
        sm[w] = amax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t2 = 0.0, tm = 0.0;
        for (int k = 0; k < NORM_THREADS / 32; ++k) {
            t2 += ss[k];
            tm = fmax(tm, sm[k]);
        }
        partials[blockIdx.x] = make_double2(t2, tm);
    }
}
__global__ void k_div_norm_finalize(const double2* partials, int n, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a2 = 0.0, m = 0.0;
    for (int i = 0; i < n; ++i) {
        a2 += partials[i].x;
        m = fmax(m, partials[i].y);
    }
    out[0] = a2;
    out[1] = m;
}
__global__ void k_norm_finalize(const double2* partials, int n, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double r = 0.0, b = 0.0;
    for (int i = 0; i < n; ++i) {
        r += partials[i].x;
        b += partials[i].y;
    }
    out[0] = r;
    out[1] = b;
}
// f32 <-> f64 transfers of the tolerance-driven solve.
__global__ void k_widen(PF p0, PF div, Plane<double> x, Plane<double> b) {
    int i = gx(), y = gy();
    if (i >= p0.w || y >= p0.h) return;
    x.at(i, y) = (double)p0.at(i, y);
    b.at(i, y) = (double)div.at(i, y);
}
__global__ void k_narrow(Plane<double> x, PF p0) {
    int i = gx(), y = gy();
    if (i >= p0.w || y >= p0.h) return;
    p0.at(i, y) = (float)x.at(i, y);
}

// shaders/jacobi_iteration.wgsl:39-91 (levelset_solid fractions = face planes)
__global__ void k_jacobi(PF p_in, PF p_out, PF ls0, PF fu, PF fv, PF div, Uniform U, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float lij = ls0.ld(x, y);
    float out;
    if (lij >= 0.0f) {
        out = 0.0f;
    } else {
        float f0 = fu.ld(x, y), f1 = fu.ld(x + 1, y), f2 = fv.ld(x, y), f3 = fv.ld(x, y + 1);
        if (f0 == 0.0f && f1 == 0.0f && f2 == 0.0f && f3 == 0.0f) {
            out = p_in.ld(x, y);
        } else {
            float p_m = p_in.ld(x - 1, y), p_p = p_in.ld(x + 1, y), p_jm = p_in.ld(x, y - 1), p_jp = p_in.ld(x, y + 1);
            float l_m = ls0.ld(x - 1, y), l_p = ls0.ld(x + 1, y), l_jm = ls0.ld(x, y - 1), l_jp = ls0.ld(x, y + 1);
            float ff_m = fminf(0.0f, l_m / lij), ff_p = fminf(0.0f, l_p / lij);
            float ff_jm = fminf(0.0f, l_jm / lij), ff_jp = fminf(0.0f, l_jp / lij);
            float coef = f0 * (1.0f - ff_m) + f1 * (1.0f - ff_p) + f2 * (1.0f - ff_jm) + f3 * (1.0f - ff_jp);
            if (fabsf(coef) < 1.0e-6f) {
                out = 0.0f;
            } else {
                float div_ij = div.ld(x, y);
                float factor = U.dx * U.rho / U.dt;
                float d00 = f0 * (ff_m >= 0.0f ? 1.0f : 0.0f) * p_m;
                float d10 = f1 * (ff_p >= 0.0f ? 1.0f : 0.0f) * p_p;
                float d01 = f2 * (ff_jm >= 0.0f ? 1.0f : 0.0f) * p_jm;
                float d11 = f3 * (ff_jp >= 0.0f ? 1.0f : 0.0f) * p_jp;
                out = (d00 + d10 + d01 + d11 - factor * div_ij) / coef;
            }
        }
    }
    p_out.st(x, y, out);
}

// solve_velocity_u.wgsl:15-47 / solve_velocity_v.wgsl:15-45
template <int COMP>
EFL_DEV void solve_velocity_at(const PF& out0, const PF& in1, const PF& solid, const PF& p0, const PF& ls0,
                               const PF& face_frac, const Uniform& U, const Dom& d) {
    int x = gx(), y = gy();
    if (COMP == 0 ? (x > d.nx || y >= d.xrows()) : (x >= d.ycols() || y > d.ny)) return;
    const float factor = U.dt / (U.dx * U.rho);
    float fr = (x < d.nx && y < d.ny) ? face_frac.ld(x, y) : 0.0f;
    if (fr == 0.0f) {
        out0.st(x, y, solid.ld(x, y));
        return;
    }
    const int ox = COMP == 0 ? 1 : 0, oy = COMP == 0 ? 0 : 1;
    float pij = p0.ld(x, y), pm = p0.ld(x - ox, y - oy);
    float lp = ls0.ld(x, y), lm = ls0.ld(x - ox, y - oy);
    if (lm >= 0.0f && lp < 0.0f) {
        pm = lm / lp * pij;
    } else if (lm < 0.0f && lp >= 0.0f) {
        pij = lp / lm * pm;
    } else if (COMP == 0 && lm >= 0.0f && lp >= 0.0f) {
        out0.st(x, y, 0.0f);
        return;
    }
    float val = in1.ld(x, y);
    out0.st(x, y, val - factor * (pij - pm));
}
// Both components in one launch over the larger of their grids (blockIdx.z: 0 = u, 1 = v).
__global__ void k_solve_velocity_uv(PF u0, PF u1, PF us, PF v0, PF v1, PF vs, PF p0, PF ls0, PF fu, PF fv, Uniform U,
                                    Dom d) {
    if (blockIdx.z == 0)
        solve_velocity_at<0>(u0, u1, us, p0, ls0, fu, U, d);
    else
        solve_velocity_at<1>(v0, v1, vs, p0, ls0, fv, U, d);
}

// extrapolate/initialize_u_valid.wgsl:6-30 / initialize_v_valid.wgsl:6-30
template <int COMP>
__global__ void k_init_valid(PI valid, PF ls0, Dom d) {
    int x = gx(), y = gy();
    if (COMP == 0 ? (x > d.nx || y >= d.xrows()) : (x >= d.ycols() || y > d.ny)) return;
    float c0, c1, c2, c3, c4, c5;
    if (COMP == 0) {
        c0 = ls0.ld(x - 1, y - 1); c1 = ls0.ld(x, y - 1); c2 = ls0.ld(x - 1, y);
        c3 = ls0.ld(x, y); c4 = ls0.ld(x - 1, y + 1); c5 = ls0.ld(x, y + 1);
    } else {
        c0 = ls0.ld(x - 1, y - 1); c1 = ls0.ld(x - 1, y); c2 = ls0.ld(x, y - 1);
        c3 = ls0.ld(x, y); c4 = ls0.ld(x + 1, y - 1); c5 = ls0.ld(x + 1, y);
    }
    float vm = 0.25f * (c0 + c1 + c2 + c3);
    float vp = 0.25f * (c2 + c3 + c4 + c5);
    valid.st(x, y, area_fraction(vm, vp) > 0.0f ? 0 : 1);
}
// extrapolate/extrapolate_{u,v}.wgsl:5-63 over [0,x1) x [0,y1)
__global__ void k_extrapolate(PF f, PI vin, PI vout, int x1, int y1) {
    int x = gx(), y = gy();
    if (x >= x1 || y >= y1) return;
    const int W = vin.w, H = vin.h;
    if (vin.ld(x, y) == 1) {
        vout.st(x, y, 1);
        return;
    }
    int count = 0;
    float nu = 0.0f;
    if (x + 1 < W && y < H && vin.ld(x + 1, y) == 1) { nu += f.ld(x + 1, y); count += 1; }
    if (x - 1 > 0 && y > 0 && vin.ld(x - 1, y) == 1) { nu += f.ld(x - 1, y); count += 1; }
    if (x < W && y + 1 < H && vin.ld(x, y + 1) == 1) { nu += f.ld(x, y + 1); count += 1; }
    if (x > 0 && y - 1 > 0 && vin.ld(x, y - 1) == 1) { nu += f.ld(x, y - 1); count += 1; }
    if (count > 0) {
        nu /= (float)count;
        f.st(x, y, nu);
        vout.st(x, y, 1);
    } else {
        vout.st(x, y, 0);
    }
}

// initialize_{u,v}_valid + the 10 extrapolation sweeps of render_node.rs:540-608
// in ONE launch, for grids whose dispatches cover every face (nx and ny
// multiples of 64): blockIdx.z = component; each CTA owns a 32 x 32 tile of
// faces, holds it with a 10-face halo in shared memory and runs the sweeps
// there (each sweep reads the valid flags of the previous one and only
// valid neighbours' velocities, so the result equals 10 global sweeps).
// Writes the velocity, the final flags (the "in" plane) and the flags after
// the ninth sweep (the "out" plane), as the per-sweep kernels leave them.
constexpr int EX_T = 32, EX_H = 10, EX_E = EX_T + 2 * EX_H;
struct ExtrapArgs {
    PF f[2];
    PI vin[2], vout[2];
    PF ls;
    const float2* range;  // per 32 x 32 cell tile of ls: (min, max)
    int rtx, rty;         // cell tiles per row / column
};
// (min, max) of the level set over each 32 x 32 tile of cells (one CTA per tile).
__global__ void __launch_bounds__(256) k_ls_tile_range(PF ls, float2* range, int rtx) {
    const int x0 = blockIdx.x * EX_T, y0 = blockIdx.y * EX_T;
    float lo = INFINITY, hi = -INFINITY;
    for (int i = threadIdx.x; i < EX_T * EX_T; i += 256) {
        const int x = x0 + (i & (EX_T - 1)), y = y0 + i / EX_T;
        if (x < ls.w && y < ls.h) {
            const float v = ls.at(x, y);
            lo = fminf(lo, v);
            hi = fmaxf(hi, v);
            if (v != v) lo = hi = NAN;  // a NaN makes the tile non-uniform below
        }
    }
    __shared__ float slo[256], shi[256];
    slo[threadIdx.x] = lo;
    shi[threadIdx.x] = hi;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) {
            const float a = slo[threadIdx.x + k], b = shi[threadIdx.x + k];
            slo[threadIdx.x] = (a != a || slo[threadIdx.x] != slo[threadIdx.x]) ? NAN : fminf(slo[threadIdx.x], a);
            shi[threadIdx.x] = (b != b || shi[threadIdx.x] != shi[threadIdx.x]) ? NAN : fmaxf(shi[threadIdx.x], b);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) range[blockIdx.y * rtx + blockIdx.x] = make_float2(slo[0], shi[0]);
}
__global__ void __launch_bounds__(256) k_extrapolate_fused(ExtrapArgs a) {
    __shared__ float sf[EX_E][EX_E];
    __shared__ unsigned char sv[2][EX_E][EX_E];
    const int comp = blockIdx.z;
    const PF f = a.f[comp];
    const int W = f.w, H = f.h;
    const int x0 = blockIdx.x * EX_T - EX_H, y0 = blockIdx.y * EX_T - EX_H;
    const int tid = threadIdx.x;
    // Every face the tile's image and flags read lies over the 3 x 3 cell tiles around it (the 10-face halo
    // and the one-cell level-set stencil stay within one tile).  All of their level set < 0: every face is
    // valid (area_fraction <= 0); all of it > 1e-30: none is (area_fraction > 0; the bound keeps the corner
    // averages normal).  Either way the ten sweeps change nothing: write the flags only.
    {
        int neg = 1, pos = 1;
        if (tid < 9) {
            const int tx = min(max((int)blockIdx.x - 1 + tid % 3, 0), a.rtx - 1);
            const int ty = min(max((int)blockIdx.y - 1 + tid / 3, 0), a.rty - 1);
            const float2 r = a.range[ty * a.rtx + tx];
            neg = r.y < 0.0f;    // false for NaN
            pos = r.x > 1e-30f;  // false for NaN
        }
        const int all_neg = __syncthreads_and(neg), all_pos = __syncthreads_and(pos);
        if (all_neg || all_pos) {
            const int v = all_neg ? 1 : 0;
            for (int i = tid; i < EX_T * EX_T; i += 256) {
                const int x = x0 + EX_H + (i & (EX_T - 1)), y = y0 + EX_H + i / EX_T;
                if ((unsigned)x >= (unsigned)W || (unsigned)y >= (unsigned)H) continue;
                a.vin[comp].at(x, y) = v;
                a.vout[comp].at(x, y) = v;
            }
            return;
        }
    }
    for (int i = tid; i < EX_E * EX_E; i += 256) {
        const int ly = i / EX_E, lx = i - ly * EX_E, x = x0 + lx, y = y0 + ly;
        float fv = 0.0f;
        unsigned char v = 0;
        if ((unsigned)x < (unsigned)W && (unsigned)y < (unsigned)H) {
            fv = f.at(x, y);
            float c0, c1, c2, c3, c4, c5;  // extrapolate/initialize_{u,v}_valid.wgsl
            if (comp == 0) {
                c0 = a.ls.ld(x - 1, y - 1); c1 = a.ls.ld(x, y - 1); c2 = a.ls.ld(x - 1, y);
                c3 = a.ls.ld(x, y); c4 = a.ls.ld(x - 1, y + 1); c5 = a.ls.ld(x, y + 1);
            } else {
                c0 = a.ls.ld(x - 1, y - 1); c1 = a.ls.ld(x - 1, y); c2 = a.ls.ld(x, y - 1);
                c3 = a.ls.ld(x, y); c4 = a.ls.ld(x + 1, y - 1); c5 = a.ls.ld(x + 1, y);
            }
            const float vm = 0.25f * (c0 + c1 + c2 + c3);
            const float vp = 0.25f * (c2 + c3 + c4 + c5);
            v = area_fraction(vm, vp) > 0.0f ? 0 : 1;
        }
        sf[ly][lx] = fv;
        sv[0][ly][lx] = v;
    }
    // A tile whose image is all valid or all invalid (away from the fluid's boundary: most of a large grid)
    // comes out of the ten sweeps unchanged, with both flag planes equal to the start flag: write the flags
    // and skip the sweeps and the face values (only faces inside the domain count).
    int any_valid = 0, any_invalid = 0;
    for (int i = tid; i < EX_E * EX_E; i += 256) {
        const int ly = i / EX_E, lx = i - ly * EX_E, x = x0 + lx, y = y0 + ly;
        if ((unsigned)x < (unsigned)W && (unsigned)y < (unsigned)H) {
            if (sv[0][ly][lx]) any_valid = 1;
            else any_invalid = 1;
        }
    }
    const bool mixed = __syncthreads_or(any_valid) && __syncthreads_or(any_invalid);
    if (!mixed) {
        for (int i = tid; i < EX_T * EX_T; i += 256) {
            const int ly = EX_H + i / EX_T, lx = EX_H + i % EX_T, x = x0 + lx, y = y0 + ly;
            if ((unsigned)x >= (unsigned)W || (unsigned)y >= (unsigned)H) continue;
            const int v = sv[0][ly][lx];
            a.vin[comp].at(x, y) = v;
            a.vout[comp].at(x, y) = v;
        }
        return;
    }
    for (int s = 0; s < 10; ++s) {
        const int in = s & 1, out = in ^ 1, lo = 1 + s, n = EX_E - 2 * lo;
        for (int i = tid; i < n * n; i += 256) {
            const int ly = lo + i / n, lx = lo + i % n, x = x0 + lx, y = y0 + ly;
            if ((unsigned)x >= (unsigned)W || (unsigned)y >= (unsigned)H) continue;
            if (sv[in][ly][lx] == 1) {
                sv[out][ly][lx] = 1;
                continue;
            }
            int count = 0;
            float nu = 0.0f;  // extrapolate_{u,v}.wgsl:5-63, neighbour order and bounds as the reference
            if (x + 1 < W && sv[in][ly][lx + 1] == 1) { nu += sf[ly][lx + 1]; count += 1; }
            if (x - 1 > 0 && y > 0 && sv[in][ly][lx - 1] == 1) { nu += sf[ly][lx - 1]; count += 1; }
            if (y + 1 < H && sv[in][ly + 1][lx] == 1) { nu += sf[ly + 1][lx]; count += 1; }
            if (x > 0 && y - 1 > 0 && sv[in][ly - 1][lx] == 1) { nu += sf[ly - 1][lx]; count += 1; }
            if (count > 0) {
                sf[ly][lx] = nu / (float)count;
                sv[out][ly][lx] = 1;
            } else {
                sv[out][ly][lx] = 0;
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < EX_T * EX_T; i += 256) {
        const int ly = EX_H + i / EX_T, lx = EX_H + i % EX_T, x = x0 + lx, y = y0 + ly;
        if ((unsigned)x >= (unsigned)W || (unsigned)y >= (unsigned)H) continue;
        f.at(x, y) = sf[ly][lx];
        a.vin[comp].at(x, y) = sv[0][ly][lx];   // after the tenth sweep
        a.vout[comp].at(x, y) = sv[1][ly][lx];  // after the ninth
    }
}

// advect_levelset.wgsl:49-74
EFL_DEV float cubic1d(float y0, float y1, float y2, float y3, float t) {
    float d1 = 0.5f * (y2 - y0);
    float d2 = 0.5f * (y3 - y1);
    float a0 = y1, a1 = d1;
    float a2 = -2.0f * d1 - d2 + 3.0f * (y2 - y1);
    float a3 = d1 + d2 - 2.0f * (y2 - y1);
    return a3 * t * t * t + a2 * t * t + a1 * t + a0;
}
EFL_DEV float cubic1d_x(const PF& t, int bx, int by, float tx) {
    return cubic1d(t.ld(bx - 1, by), t.ld(bx, by), t.ld(bx + 1, by), t.ld(bx + 2, by), tx);
}
// advect_levelset.wgsl:11-34 (CUBIC defined, advect_levelset.rs:62)
__global__ void k_advect_levelset(PF u0, PF v0, PF ls0, PF ls1, float dt, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float2 xn = runge_kutta(u0, v0, (float)x, (float)y, dt);
    xn.x = fclampf(xn.x, 0.0f, (float)d.nx - 1.0f);
    xn.y = fclampf(xn.y, 0.0f, (float)d.ny - 1.0f);
    int bx = f2i(xn.x), by = f2i(xn.y);
    float tx = xn.x - (float)bx, ty = xn.y - (float)by;
    float y0 = cubic1d_x(ls0, bx, by - 1, tx), y1 = cubic1d_x(ls0, bx, by, tx);
    float y2 = cubic1d_x(ls0, bx, by + 1, tx), y3 = cubic1d_x(ls0, bx, by + 2, tx);
    float nl = cubic1d(y0, y1, y2, y3, ty);
    if (fabsf(nl) < 1000.0f) ls1.st(x, y, nl);
}

// update_fluid_source.wgsl:72-107
struct Sources {
    efl_source s[EFL_MAX_FLUID_SOURCE];
    int n;
};
EFL_DEV float level_aabb(float hx, float hy, float cx, float cy, float px, float py) {
    float dx = fabsf(cx - px) - hx, dy = fabsf(cy - py) - hy;
    bool ix = dx < 0.0f, iy = dy < 0.0f;
    if (ix) return iy ? fmaxf(dx, dy) : dy;
    return iy ? dx : wlength(dx, dy);
}
EFL_DEV float level_source(const efl_source& s, float px, float py) {
    switch (s.shape) {
        case EFL_SOURCE_CIRCLE: return wlength(s.center[0] - px, s.center[1] - py) - s.data[0];
        case EFL_SOURCE_AABB: return level_aabb(s.data[0], s.data[1], s.center[0], s.center[1], px, py);
        default: return 0.0f;
    }
}
// update_fluid_source.wgsl:30-62: level set and per-cell source velocity.
__global__ void k_fluid_source_cells(PF ls1, PU upd, P2 vel, Sources S, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    const float dimx = (float)d.nx, dimy = (float)d.ny;
    float uvx = (float)(uint32_t)x / dimx, uvy = (float)(uint32_t)y / dimy;
    float ndcx = uvx * 2.0f + -1.0f, ndcy = uvy * -2.0f + 1.0f;  // bevy uv_to_ndc
    float px = 0.5f * dimx * ndcx, py = 0.5f * dimy * ndcy;
    float nl = ls1.ld(x, y);
    float vx = 0.0f, vy = 0.0f;
    bool has_source = false, vu = false;
    for (int i = 0; i < S.n; ++i) {
        const efl_source& src = S.s[i];
        float sdf = level_source(src, px, py);
        if (src.mode == EFL_SOURCE_MODE_SOURCE) {
            nl = fminf(nl, sdf);
            has_source = true;
            if (sdf < 0.0f) {
                vx = vx + src.velocity[0];
                vy = vy + src.velocity[1];
                vu = true;
            }
        } else if (!has_source) {
            nl = fmaxf(nl, -sdf);
        }
    }
    ls1.st(x, y, nl);
    upd.st(x, y, vu ? 1u : 0u);
    vel.st(x, y, make_float2(vx, vy));
}
// update_fluid_source.wgsl:64-69: a face written by two invocations takes
// the raster-last writer's value (the cell on its high side).
__global__ void k_fluid_source_faces(PF u0, PF v0, PU upd, P2 vel, Dom d) {
    int x = gx(), y = gy();
    const int W = d.cx(), H = d.cy();
    if (x <= W && y < H) {  // u face (x, y): writers (x, y) then (x-1, y)
        if (x < W && upd.ld(x, y)) u0.st(x, y, vel.ld(x, y).x);
        else if (x >= 1 && upd.ld(x - 1, y)) u0.st(x, y, vel.ld(x - 1, y).x);
    }
    if (x < W && y <= H) {  // v face (x, y): writers (x, y) then (x, y-1)
        if (y < H && upd.ld(x, y)) v0.st(x, y, vel.ld(x, y).y);
        else if (y >= 1 && upd.ld(x, y - 1)) v0.st(x, y, vel.ld(x, y - 1).y);
    }
}

// jump_flooding/initialize.wgsl:8-41
__global__ void k_jfa_init(PF ls1, P2 seeds, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float md = 10.0f;
    float2 seed = make_float2(-1.0f, -1.0f);
    float level = ls1.ld(x, y);
    for (int i = -1; i <= 1; ++i)
        for (int j = -1; j <= 1; ++j) {
            if (i == 0 && j == 0) continue;
            int ax = x + i, ay = y + j;
            if (ax < 0 || ay < 0 || ax >= d.nx || ay >= d.ny) continue;
            float nl = ls1.ld(ax, ay);
            if (nl >= 0.0f && !(level >= 0.0f)) {
                float t = level / (level - nl);
                if (fabsf(t) < md) {
                    md = fabsf(t);
                    seed = make_float2((float)x + t * (float)i, (float)y + t * (float)j);
                }
            }
        }
    seeds.st(x, y, seed);
}
EFL_DEV bool valid_seed(float2 s) { return s.x != -1.0f && s.y != -1.0f; }
// jump_flooding/iterate.wgsl:18-56
__global__ void k_jfa_iterate(P2 in, P2 out, int step, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float2 cur = in.ld(x, y), best = cur;
    float bd = 1e10f;
    if (valid_seed(cur)) bd = wlength(cur.x - (float)x, cur.y - (float)y);
    for (int i = -1; i <= 1; ++i)
        for (int j = -1; j <= 1; ++j) {
            if (i == 0 && j == 0) continue;
            int ax = x + i * step, ay = y + j * step;
            if (ax < 0 || ay < 0 || ax >= in.w || ay >= in.h) continue;
            float2 ns = in.at(ax, ay);
            if (!valid_seed(ns)) continue;
            float cd = wlength(ns.x - (float)x, ns.y - (float)y);
            if (cd < bd) {
                best = ns;
                bd = cd;
            }
        }
    out.st(x, y, best);
}
// jump_flooding/calculate_sdf.wgsl:9-23
__global__ void k_jfa_sdf(P2 seeds, PF ls1, PF ls0, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float2 s = seeds.ld(x, y);
    float sdf = wlength(s.x - (float)x, s.y - (float)y);
    float level = ls1.ld(x, y);
    ls0.st(x, y, sdf * (level < 0.0f ? -1.0f : 1.0f));
}

// fast_iterative_method/initialize.wgsl:10-40
__global__ void k_fim_init(PF ls1, PF ls0, PU lab0, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    float level = ls1.ld(x, y);
    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    bool src = false;
    for (int i = 0; i < 4 && !src; ++i) {
        int ax = x + ox[i], ay = y + oy[i];
        if (ax >= 0 && ay >= 0 && ax < d.nx && ay < d.ny && level * ls1.ld(ax, ay) <= 0.0f) src = true;
    }
    if (src) {
        ls0.st(x, y, level);
        lab0.st(x, y, LABEL_SOURCE);
    } else {
        ls0.st(x, y, wsign(level) * FIM_LARGE);
        lab0.st(x, y, LABEL_NONE);
    }
}
// fast_iterative_method/initialize_active_label.wgsl:8-40.  tile_active (optional): set to 1 for every
// 32 x 32 tile (FIM_TILE) that holds an active cell.
__global__ void k_fim_active(PU lab0, PU lab, Dom d, unsigned* tile_active, int tiles_x) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    if (lab0.ld(x, y) == LABEL_SOURCE) {
        lab.st(x, y, LABEL_SOURCE);
        return;
    }
    const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
    uint32_t out = LABEL_NONE;
    for (int i = 0; i < 4; ++i) {
        int ax = x + ox[i], ay = y + oy[i];
        if (ax >= 0 && ay >= 0 && ax < d.nx && ay < d.ny && lab0.ld(ax, ay) == LABEL_SOURCE) {
            out = LABEL_ACTIVE;
            break;
        }
    }
    lab.st(x, y, out);
    if (tile_active && out == LABEL_ACTIVE) {
        unsigned* f = &tile_active[(y / 32) * tiles_x + x / 32];
        if (*f == 0u) atomicOr(f, 1u);
    }
}
// fast_iterative_method/update.wgsl:56-83
EFL_DEV float abs_get_phi(const PF& p, int x, int y) {
    if (x < 0 || y < 0 || x >= p.w || y >= p.h) return FIM_LARGE;
    return fabsf(p.at(x, y));
}
EFL_DEV float solve_quadratic_2d(const PF& p, int x, int y) {
    float xm = fminf(abs_get_phi(p, x - 1, y), abs_get_phi(p, x + 1, y));
    float ym = fminf(abs_get_phi(p, x, y - 1), abs_get_phi(p, x, y + 1));
    float d = xm - ym;
    if (d > SQRT2_F) return ym + 1.0f;
    if (d < -SQRT2_F) return xm + 1.0f;
    return 0.5f * (xm + ym + sqrtf(2.0f - d * d));
}
// Deterministic two-phase form of fast_iterative_method/update.wgsl:13-54
// (the reference writes neighbours from inside one dispatch, a data race).
// Phase A: active cells update from the iteration-start phi and flag
// convergence.  Phase B: an inactive cell next to a cell that converged in
// A is re-solved from the post-A phi and activated, with the sign of the
// raster-last converged neighbour (down, right, left, up).
__global__ void k_fim_phase_a(PF S, PU L, PF T, PU LT, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    uint32_t l = L.at(x, y);
    float p = S.at(x, y);
    if (l != LABEL_ACTIVE) {
        T.at(x, y) = p;
        LT.at(x, y) = l;
        return;
    }
    float q = solve_quadratic_2d(S, x, y) * wsign(p);
    T.at(x, y) = q;
    LT.at(x, y) = (fabsf(p - q) > FIM_EPS) ? LABEL_ACTIVE : LABEL_CONVERGED;
}
__global__ void k_fim_phase_b(PF T, PU LT, PF S, PU L, Dom d) {
    int x = gx(), y = gy();
    const int W = d.cx(), H = d.cy();
    if (x >= W || y >= H) return;
    uint32_t l = LT.at(x, y);
    float t = T.at(x, y);
    if (l == LABEL_NONE) {
        const int wo[4][2] = {{0, 1}, {1, 0}, {-1, 0}, {0, -1}};
        int wx = -1, wy = -1;
        for (int k = 0; k < 4; ++k) {
            int ax = x + wo[k][0], ay = y + wo[k][1];
            if (ax >= 0 && ay >= 0 && ax < W && ay < H && LT.at(ax, ay) == LABEL_CONVERGED) {
                wx = ax;
                wy = ay;
                break;
            }
        }
        if (wx >= 0) {
            float pn = fabsf(t);
            float qn = solve_quadratic_2d(T, x, y);
            if (pn > qn) {
                S.at(x, y) = qn * wsign(T.at(wx, wy));
                L.at(x, y) = LABEL_ACTIVE;
                return;
            }
        }
        S.at(x, y) = t;
        L.at(x, y) = LABEL_NONE;
    } else {
        S.at(x, y) = t;
        L.at(x, y) = l == LABEL_CONVERGED ? LABEL_NONE : l;
    }
}

// Iterations of the two-phase FIM update (k_fim_phase_a then k_fim_phase_b,
// `iters` times) in one launch, temporally blocked: a CTA holds its 32 x 32
// tile plus a halo of HALO cells in shared memory and runs the iterations
// there.  One iteration's result at a cell depends on cells at most 2 away
// (phase A reads radius 1, phase B reads phase A's result at radius 1), so
// values go wrong only near the image edge, 2 cells deeper per iteration:
// with iters <= HALO / 2 the owned tile is exact.  A cell changes only while
// it is active, and activity spreads one cell per iteration, so a tile whose
// image holds no active cell is left untouched (most of a large grid, away
// from the interface): such CTAs read the labels and leave.  Two halos: 20
// (the 10 iterations in one launch; large grids, where most tiles leave at
// once) and 4 (2 iterations per launch, 1.56x the owned cells in the image;
// small grids, where a 72 x 72 image per 32 x 32 tile would be 5x the work).
constexpr int FIM_TILE = 32, FIM_HALO = 20, FIM_THREADS = 512, FIM_HALO_NARROW = 4, FIM_THREADS_NARROW = 256;
__host__ __device__ constexpr size_t fim_smem(int halo) {
    return (size_t)4 * (FIM_TILE + 2 * halo) * (FIM_TILE + 2 * halo) * 4;
}
constexpr size_t FIM_SMEM = fim_smem(FIM_HALO);
// Each launch reads (S, L) and writes its tiles into (SD, LD), another pair of planes: a CTA that started late
// must still see its neighbours' values of the launch's start in its halo.  A tile that leaves early copies its
// cells across.  tile_active: the flags k_fim_active left (a tile whose 3 x 3 neighbourhood holds no active
// cell has none in its image, HALO < FIM_TILE, and leaves at once); valid for the first launch only.
template <int HALO, int THREADS>
__global__ void __launch_bounds__(THREADS) k_fim_tiled(PF S, PU L, PF SD, PU LD, Dom d, int iters, int tiles_x,
                                                       const unsigned* tile_active) {
    extern __shared__ __align__(16) unsigned char fim_raw[];
    constexpr int FIM_IMG = FIM_TILE + 2 * HALO, N = FIM_IMG * FIM_IMG;
    static_assert(HALO < FIM_TILE, "the image lies within the 3 x 3 tiles around the owned one");
    auto copy_across = [&]() {  // the owned tile unchanged
        const int tx0 = (int)(blockIdx.x % tiles_x) * FIM_TILE, ty0 = (int)(blockIdx.x / tiles_x) * FIM_TILE;
        for (int i = threadIdx.x; i < FIM_TILE * FIM_TILE; i += THREADS) {
            const int gx = tx0 + i % FIM_TILE, gy = ty0 + i / FIM_TILE;
            if (gx < d.nx && gy < d.ny) {
                SD.at(gx, gy) = S.at(gx, gy);
                LD.at(gx, gy) = L.at(gx, gy);
            }
        }
    };
    if (tile_active) {
        const int tiles_y = (d.ny + FIM_TILE - 1) / FIM_TILE;
        int any = 0;
        if (threadIdx.x < 9) {
            const int tx = (int)(blockIdx.x % tiles_x) - 1 + (int)threadIdx.x % 3;
            const int ty = (int)(blockIdx.x / tiles_x) - 1 + (int)threadIdx.x / 3;
            if (tx >= 0 && ty >= 0 && tx < tiles_x && ty < tiles_y) any = tile_active[ty * tiles_x + tx] != 0u;
        }
        if (!__syncthreads_or(any)) {
            copy_across();
            return;
        }
    }
    float* s = reinterpret_cast<float*>(fim_raw);
    float* t = s + N;
    uint32_t* l = reinterpret_cast<uint32_t*>(t + N);
    uint32_t* lt = l + N;
    const int x0 = (int)(blockIdx.x % tiles_x) * FIM_TILE - HALO, y0 = (int)(blockIdx.x / tiles_x) * FIM_TILE - HALO;
    const int W = d.nx, H = d.ny;  // the dispatch domain (sizes are multiples of 8) and the planes' extent
    int act = 0;
    for (int i = threadIdx.x; i < N; i += THREADS) {
        const int gx = x0 + i % FIM_IMG, gy = y0 + i / FIM_IMG;
        const bool in = gx >= 0 && gy >= 0 && gx < W && gy < H;
        const uint32_t lv = in ? L.at(gx, gy) : LABEL_NONE;
        l[i] = lv;
        act |= lv == LABEL_ACTIVE;
    }
    if (!__syncthreads_or(act)) {
        copy_across();
        return;
    }
    for (int i = threadIdx.x; i < N; i += THREADS) {
        const int gx = x0 + i % FIM_IMG, gy = y0 + i / FIM_IMG;
        s[i] = (gx >= 0 && gy >= 0 && gx < W && gy < H) ? S.at(gx, gy) : 0.0f;
    }
    __syncthreads();
    // |phi| of a neighbour: FIM_LARGE outside the domain (update.wgsl:56-60) and, where the image ends,
    // a stand-in whose error stays in the halo.
    auto absphi = [&](const float* a, int ix, int iy) -> float {
        const int gx = x0 + ix, gy = y0 + iy;
        if (gx < 0 || gy < 0 || gx >= W || gy >= H) return FIM_LARGE;
        if (ix < 0 || iy < 0 || ix >= FIM_IMG || iy >= FIM_IMG) return FIM_LARGE;
        return fabsf(a[iy * FIM_IMG + ix]);
    };
    auto quad = [&](const float* a, int ix, int iy) -> float {  // solve_quadratic_2d (update.wgsl:62-83)
        const float xm = fminf(absphi(a, ix - 1, iy), absphi(a, ix + 1, iy));
        const float ym = fminf(absphi(a, ix, iy - 1), absphi(a, ix, iy + 1));
        const float dd = xm - ym;
        if (dd > SQRT2_F) return ym + 1.0f;
        if (dd < -SQRT2_F) return xm + 1.0f;
        return 0.5f * (xm + ym + sqrtf(2.0f - dd * dd));
    };
    for (int it = 0; it < iters; ++it) {
        for (int i = threadIdx.x; i < N; i += THREADS) {  // phase A
            const int ix = i % FIM_IMG, iy = i / FIM_IMG;
            const uint32_t lv = l[i];
            const float p = s[i];
            if (lv != LABEL_ACTIVE) {
                t[i] = p;
                lt[i] = lv;
            } else {
                const float q = quad(s, ix, iy) * wsign(p);
                t[i] = q;
                lt[i] = (fabsf(p - q) > FIM_EPS) ? LABEL_ACTIVE : LABEL_CONVERGED;
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < N; i += THREADS) {  // phase B
            const int ix = i % FIM_IMG, iy = i / FIM_IMG;
            const int gx = x0 + ix, gy = y0 + iy;
            const uint32_t lv = lt[i];
            const float tv = t[i];
            if (lv == LABEL_NONE) {
                const int wo[4][2] = {{0, 1}, {1, 0}, {-1, 0}, {0, -1}};
                int wi = -1;
                for (int k = 0; k < 4; ++k) {
                    const int ax = ix + wo[k][0], ay = iy + wo[k][1];
                    const int bx = gx + wo[k][0], by = gy + wo[k][1];
                    if (bx >= 0 && by >= 0 && bx < W && by < H && ax >= 0 && ay >= 0 && ax < FIM_IMG &&
                        ay < FIM_IMG && lt[ay * FIM_IMG + ax] == LABEL_CONVERGED) {
                        wi = ay * FIM_IMG + ax;
                        break;
                    }
                }
                if (wi >= 0) {
                    const float pn = fabsf(tv);
                    const float qn = quad(t, ix, iy);
                    if (pn > qn) {
                        s[i] = qn * wsign(t[wi]);
                        l[i] = LABEL_ACTIVE;
                        continue;
                    }
                }
                s[i] = tv;
                l[i] = LABEL_NONE;
            } else {
                s[i] = tv;
                l[i] = lv == LABEL_CONVERGED ? LABEL_NONE : lv;
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < FIM_TILE * FIM_TILE; i += THREADS) {
        const int ix = HALO + i % FIM_TILE, iy = HALO + i / FIM_TILE;
        const int gx = x0 + ix, gy = y0 + iy;
        if (gx < W && gy < H) {
            SD.at(gx, gy) = s[iy * FIM_IMG + ix];
            LD.at(gx, gy) = l[iy * FIM_IMG + ix];
        }
    }
}

// levelset_gradient.wgsl:4-21
__global__ void k_gradient(PF ls0, P2 grad, Dom d) {
    int x = gx(), y = gy();
    if (x >= d.cx() || y >= d.cy()) return;
    if (x == 0 || y == 0 || x >= d.nx || y >= d.ny) return;
    grad.st(x, y, make_float2(0.5f * (ls0.ld(x + 1, y) - ls0.ld(x - 1, y)), 0.5f * (ls0.ld(x, y + 1) - ls0.ld(x, y - 1))));
}

// solid_obstacle.wgsl:67-89
EFL_DEV float2 center_of_mass(const efl_solid_obstacle& o) {
    switch (o.shape) {
        case EFL_SHAPE_CIRCLE:
        case EFL_SHAPE_RECTANGLE:
        case EFL_SHAPE_CAPSULE:
            return make_float2(o.transform[12], o.transform[13]);
        case EFL_SHAPE_TRIANGLE: {
            float lx = (o.values[0] + o.values[2] + o.values[4]) / 3.0f;
            float ly = (o.values[1] + o.values[3] + o.values[5]) / 3.0f;
            return mat_xy(o.transform, lx, ly);
        }
        default:
            return make_float2(0.0f, 0.0f);
    }
}
// sample_forces.wgsl:20-53.  Per-cell force/torque in fixed point
// (fixed_point_conversion.wgsl:2-13, scale 0.1 -> x10), accumulated in a
// block-private shared-memory copy of the 3 x 256 bins and flushed with
// one global atomic per touched bin.  Integer sums are order-independent,
// so the bins are bit-identical to the reference's per-cell atomics.
__global__ void k_solid_forces(PF fu, PF fv, PI sid, PF p0, const efl_solid_obstacle* __restrict__ obs, int n_obs,
                               Uniform U, Dom d, int* __restrict__ bins) {
    __shared__ int sb[3 * EFL_MAX_SOLIDS];
    __shared__ int touched;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nth = blockDim.x * blockDim.y;
    for (int i = tid; i < 3 * EFL_MAX_SOLIDS; i += nth) sb[i] = 0;
    if (tid == 0) touched = 0;
    __syncthreads();
    int x = gx(), y = gy();
    if (x < d.cx() && y < d.cy()) {
        float f0 = fu.at(x, y), f1 = fu.at(x + 1, y), f2 = fv.at(x, y), f3 = fv.at(x, y + 1);
        int32_t id = sid.at(x, y);
        if (!(f0 == 0.0f && f1 == 0.0f && f2 == 0.0f && f3 == 0.0f) && id != -1) {
            float p = p0.at(x, y);
            float fx = -(f1 - f0) * p * U.dx;
            float fy = -(f3 - f2) * p * U.dx;
            float2 c = make_float2(0.0f, 0.0f);
            if (id >= 0 && id < n_obs) c = center_of_mass(obs[id]);
            float uvx = (float)x / U.size[0], uvy = (float)y / U.size[1];
            float xx = (uvx - 0.5f) * U.size[0], yy = (-uvy + 0.5f) * U.size[1];
            float2 w = mat_xy(U.m, xx, yy);
            float rx = w.x - c.x, ry = w.y - c.y;
            float torque = rx * fy - ry * fx;
            if (id >= 0 && id < EFL_MAX_SOLIDS) {
                atomicAdd(&sb[id], f2i(fx * 10.0f));
                atomicAdd(&sb[EFL_MAX_SOLIDS + id], f2i(fy * 10.0f));
                atomicAdd(&sb[2 * EFL_MAX_SOLIDS + id], f2i(torque * 10.0f));
                touched = 1;
            }
        }
    }
    __syncthreads();
    if (!touched) return;
    for (int i = tid; i < 3 * EFL_MAX_SOLIDS; i += nth)
        if (sb[i] != 0) atomicAdd(&bins[i], sb[i]);
}
// accumulate_forces.wgsl:16-32
__global__ void k_accumulate_forces(const int* bins, efl_solid_force* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= EFL_MAX_SOLIDS) return;
    efl_solid_force f;
    f.force[0] = (float)bins[i] * 0.1f;
    f.force[1] = (float)bins[EFL_MAX_SOLIDS + i] * 0.1f;
    f.torque = (float)bins[2 * EFL_MAX_SOLIDS + i] * 0.1f;
    f._pad = 0.0f;
    out[i] = f;
}

// calculate_volume.wgsl:11-75 as an exact integer count of phi < 0.
__global__ void k_volume(PF ls0, unsigned long long* out) {
    int x = gx(), y = gy();
    unsigned long long c = (x < ls0.w && y < ls0.h && ls0.at(x, y) < 0.0f) ? 1ull : 0ull;
    unsigned mask = __ballot_sync(0xffffffffu, c != 0);
    if ((threadIdx.x & 31) == 0 && mask) atomicAdd(out, (unsigned long long)__popc(mask));
}

// diagnostics/{min,max}_velocity.wgsl partial_reduction: one 16 x 16 block
// per workgroup; min over fluid cells (1e30 elsewhere), max over all cells.
__global__ void __launch_bounds__(256) k_velocity_partial(PF u, PF v, PF ls, float* pmin, float* pmax) {
    __shared__ float smin[256], smax[256];
    const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
    const int lid = threadIdx.y * 16 + threadIdx.x;
    const float u0 = 0.5f * (u.ld(x, y) + u.ld(x + 1, y));
    const float v0 = 0.5f * (v.ld(x, y) + v.ld(x, y + 1));
    const float mag = sqrtf(u0 * u0 + v0 * v0);
    smin[lid] = ls.ld(x, y) < 0.0f ? mag : 1e30f;
    smax[lid] = mag;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (lid < st) {
            smin[lid] = fminf(smin[lid], smin[lid + st]);
            smax[lid] = fmaxf(smax[lid], smax[lid + st]);
        }
        __syncthreads();
    }
    if (lid == 0) {
        const int w = blockIdx.x + blockIdx.y * gridDim.x;
        pmin[w] = smin[0];
        pmax[w] = smax[0];
    }
}
// diagnostics/{min,max}_velocity.wgsl reduction: 512 lanes each ADD their
// partials i = lane, lane + 512, ... from 0.0 (as the reference does), then min / max.
__global__ void __launch_bounds__(512) k_velocity_final(const float* pmin, const float* pmax, int n, float* out) {
    __shared__ float smin[512], smax[512];
    const int lid = threadIdx.x;
    float a = 0.0f, b = 0.0f;
    for (int i = lid; i < n; i += 512) {
        a += pmin[i];
        b += pmax[i];
    }
    smin[lid] = a;
    smax[lid] = b;
    __syncthreads();
    for (int st = 256; st > 0; st >>= 1) {
        if (lid < st) {
            smin[lid] = fminf(smin[lid], smin[lid + st]);
            smax[lid] = fmaxf(smax[lid], smax[lid + st]);
        }
        __syncthreads();
    }
    if (lid == 0) {
        out[0] = smin[0];
        out[1] = smax[0];
    }
}

}  // namespace efl
