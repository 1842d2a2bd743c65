// efl_oracle.cpp — TEST INFRASTRUCTURE, not product code.
//
// CPU restatement of the reference's per-step Eulerian fluid pipeline
// (narasan49/bevy_eulerian_fluid v0.4.0).  Every kernel below follows one
// WGSL entry point, statement by statement and in the same floating-point
// operation order, with these fixed semantics:
//   * texture loads out of bounds return 0, out-of-bounds stores are
//     dropped (robust buffer access, the DX12 behaviour the examples use);
//   * no FMA contraction (built with -ffp-contract=off), IEEE division and
//     sqrt, WGSL round() = round-half-to-even, clamp(NaN,0,1) = 0 (the
//     maxNum/minNum behaviour of GPUs), f32->i32 truncates and saturates,
//     NaN -> 0;
//   * every kernel covers exactly the invocation domain of its reference
//     dispatch (pipeline.rs:175-186, render_node.rs:226-230);
//   * racy reference kernels get a fixed resolution that the CUDA library
//     shares: update_fluid_source's shared faces take the value of the
//     raster-last writer; the FIM update is the deterministic two-phase
//     form documented at fim_update_two_phase().
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU leg use this file.
// Parity is unpinned (the reference has no golden vectors); the oracle's
// known-answer tests pin it.

#include "efl_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr float LARGE_FLOAT_SOLID = 1.0e6f;   // update_solid.wgsl:4
constexpr float LARGE_FLOAT_SOURCE = 1.0e6f;  // update_fluid_source.wgsl:22
constexpr float FIM_LARGE = 1e30f;            // fast_iterative_method/initialize.wgsl:5
constexpr float FIM_EPS = 1e-6f;              // fast_iterative_method/update.wgsl:9
constexpr float SQRT2_F = 1.41421356237309504880f;  // update.wgsl:11 (f32)
constexpr uint32_t LABEL_NONE = 0, LABEL_SOURCE = 1, LABEL_ACTIVE = 2, LABEL_CONVERGED = 3;

int g_threads = 0;

struct F2 { float x, y; };
struct F4 { float x, y, z, w; };

template <class T>
struct Tex {
    int w = 0, h = 0;
    std::vector<T> a;
    void init(int w_, int h_) { w = w_; h = h_; a.assign((size_t)w * h, T{}); }
    inline bool in(int x, int y) const { return x >= 0 && y >= 0 && x < w && y < h; }
    inline T ld(int x, int y) const { return in(x, y) ? a[(size_t)y * w + x] : T{}; }
    inline void st(int x, int y, T v) { if (in(x, y)) a[(size_t)y * w + x] = v; }
    inline T& at(int x, int y) { return a[(size_t)y * w + x]; }
};

// WGSL helpers ---------------------------------------------------------------
inline float fclamp01(float v) { return std::fmin(std::fmax(v, 0.0f), 1.0f); }
inline float fclamp(float v, float lo, float hi) { return std::fmin(std::fmax(v, lo), hi); }
inline float wsign(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
inline float wlength(float x, float y) { return std::sqrt(x * x + y * y); }
inline float wmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline int32_t f2i(float v) {  // WGSL i32(f32): truncate, saturate, NaN -> 0
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0f) return std::numeric_limits<int32_t>::max();
    if (v <= -2147483648.0f) return std::numeric_limits<int32_t>::min();
    return (int32_t)v;
}
// mat4 (column-major) * vec4(x, y, 0, 1), .xy
inline F2 mat_xy(const float* m, float x, float y) {
    F2 r;
    r.x = ((m[0] * x + m[4] * y) + m[8] * 0.0f) + m[12] * 1.0f;
    r.y = ((m[1] * x + m[5] * y) + m[9] * 0.0f) + m[13] * 1.0f;
    return r;
}
// determinant of a column-major 4x4 (only compared against 0)
inline float det4(const float* m) {
    auto a = [&](int r, int c) { return m[c * 4 + r]; };
    float s0 = a(0, 0) * a(1, 1) - a(1, 0) * a(0, 1);
    float s1 = a(0, 0) * a(1, 2) - a(1, 0) * a(0, 2);
    float s2 = a(0, 0) * a(1, 3) - a(1, 0) * a(0, 3);
    float s3 = a(0, 1) * a(1, 2) - a(1, 1) * a(0, 2);
    float s4 = a(0, 1) * a(1, 3) - a(1, 1) * a(0, 3);
    float s5 = a(0, 2) * a(1, 3) - a(1, 2) * a(0, 3);
    float c5 = a(2, 2) * a(3, 3) - a(3, 2) * a(2, 3);
    float c4 = a(2, 1) * a(3, 3) - a(3, 1) * a(2, 3);
    float c3 = a(2, 1) * a(3, 2) - a(3, 1) * a(2, 2);
    float c2 = a(2, 0) * a(3, 3) - a(3, 0) * a(2, 3);
    float c1 = a(2, 0) * a(3, 2) - a(3, 0) * a(2, 2);
    float c0 = a(2, 0) * a(3, 1) - a(3, 0) * a(2, 1);
    return s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
}

// utils/area_fraction.wgsl:10-12
inline float area_fraction(float l0, float l1) {
    return fclamp01(std::fmax(l0, l1) / std::fabs(l0 - l1));
}
// utils/area_fraction.wgsl:14-56
inline F4 area_fractions(const Tex<float>& ls, int x, int y) {
    float c0 = ls.ld(x - 1, y - 1), c1 = ls.ld(x, y - 1), c2 = ls.ld(x + 1, y - 1);
    float c3 = ls.ld(x - 1, y), c4 = ls.ld(x, y), c5 = ls.ld(x + 1, y);
    float c6 = ls.ld(x - 1, y + 1), c7 = ls.ld(x, y + 1), c8 = ls.ld(x + 1, y + 1);
    float mm = 0.25f * (c0 + c1 + c3 + c4);
    float pm = 0.25f * (c1 + c2 + c4 + c5);
    float mp = 0.25f * (c3 + c4 + c6 + c7);
    float pp = 0.25f * (c4 + c5 + c7 + c8);
    return F4{area_fraction(mm, mp), area_fraction(pm, pp), area_fraction(mm, pm), area_fraction(mp, pp)};
}

struct Uniform {  // fluid_uniform.wgsl:3-10
    float dx, dt, rho;
    float g[2];
    float m[16];
    float size[2];
};

// One multigrid level (multi_grid.rs:77-83).  The iterate x, right-hand
// side b and residual r are of type T: f32 in the reference's fixed-count
// mode, f64 in the tolerance-driven mode; the level set and the area
// fractions are always the reference's f32 data.
template <class T>
struct LevelT {
    int nx, ny;
    Tex<T> x, b, r;
    Tex<float> ls;
    Tex<F4> af;
};
using Level = LevelT<float>;
using Level64 = LevelT<double>;

// particle.wgsl:5-11
struct OParticle {
    float x, y, radius, sign;
    uint32_t escaped;
};

}  // namespace

struct eflo_sim {
    efl_config cfg;
    int nx, ny;
    Uniform U;
    std::string err;
    int status = 0;  // 0 = Reset/Uninitialized, 1 = Initialized
    bool fim_serial = false;

    Tex<float> u0, u1, v0, v1, us, vs, ls_solid, div, p0, p1, ls0, ls1;
    Tex<int32_t> solid_id, u_valid_in, u_valid_out, v_valid_in, v_valid_out;
    Tex<F4> af;
    Tex<F2> grad, seeds[2];
    int seeds_final = 0;
    Tex<uint32_t> labels0, labels, labelsT;
    Tex<float> phiT;
    std::vector<Level> mg;
    std::vector<Level64> mg64;

    std::vector<efl_solid_obstacle> obstacles;
    std::vector<efl_force> forces;
    std::vector<efl_source> src_once, src_cont;
    int32_t bins[3][EFL_MAX_SOLIDS];
    efl_solid_force out_forces[EFL_MAX_SOLIDS];

    // two-layer particle level set (particle_levelset_two_layers/plugin.rs)
    bool pls_on = false;
    std::vector<OParticle> parts[2];      // [0] positive, [1] negative
    std::vector<int32_t> phi_plus, phi_minus;
    uint32_t pls_dropped = 0;

    // dispatch domains (pipeline.rs:175-186)
    int cx() const { return (nx / 8) * 8; }
    int cy() const { return (ny / 8) * 8; }
    int xrows() const { return (ny / 64) * 64; }
    int ycols() const { return (nx / 64) * 64; }
};

namespace {

efl_status fail(eflo_sim* s, efl_status st, const std::string& m) {
    if (s) s->err = m;
    return st;
}

template <class F>
inline void par_rows(int y0, int y1, F f) {
#pragma omp parallel for schedule(static) if (g_threads != 1)
    for (int y = y0; y < y1; ++y) f(y);
}

// ---------------------------------------------------------------------------
// initialize_grid_center.wgsl:5-15 (dispatch_center)
void k_init_center(eflo_sim& s) {
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            float level = (float)(uint32_t)(s.ny - y);
            s.ls0.st(x, y, level);
            s.ls1.st(x, y, level);
            s.grad.st(x, y, F2{0.0f, -1.0f});
        }
    });
}
// initialize_grid_edge.wgsl:6-17, dispatched (nx+1, ny/64) x (1,64), v transposed
void k_init_edge(eflo_sim& s) {
    for (int gy = 0; gy < s.xrows(); ++gy)
        for (int gx = 0; gx <= s.nx; ++gx) {
            s.u0.st(gx, gy, 0.0f);
            s.v0.st(gy, gx, 0.0f);
            s.u1.st(gx, gy, 0.0f);
            s.v1.st(gy, gx, 0.0f);
        }
}

// update_solid.wgsl:80-85
inline F2 to_world(const Uniform& U, float px, float py, int nx, int ny) {
    float uvx = px / (float)nx, uvy = py / (float)ny;
    float xx = (uvx - 0.5f) * U.size[0];
    float yy = (-uvy + 0.5f) * U.size[1];
    return mat_xy(U.m, xx, yy);
}
// update_solid.wgsl:164-169
inline float dist_segment(F2 x, F2 a, F2 b) {
    float abx = b.x - a.x, aby = b.y - a.y;
    float t = fclamp(((x.x - a.x) * abx + (x.y - a.y) * aby) / (abx * abx + aby * aby), 0.0f, 1.0f);
    float px = a.x + t * abx, py = a.y + t * aby;
    return wlength(x.x - px, x.y - py);
}
// update_solid.wgsl:171-175
inline float dist_sign(F2 x, F2 a, F2 b) {
    float x1x = x.x - a.x, x1y = x.y - a.y;
    float abx = b.x - a.x, aby = b.y - a.y;
    return wsign(x1y * abx - x1x * aby);
}
// update_solid.wgsl:87-109
inline float level_rectangle(const efl_solid_obstacle& o, F2 x) {
    float level = LARGE_FLOAT_SOLID;
    if (det4(o.transform) == 0.0f) return level;
    F2 x0 = mat_xy(o.inverse_transform, x.x, x.y);
    float hx = o.values[0], hy = o.values[1];
    bool ix = std::fabs(x0.x) < hx, iy = std::fabs(x0.y) < hy;
    if (ix) {
        if (iy) level = std::fmax(std::fabs(x0.x) - hx, std::fabs(x0.y) - hy);
        else level = std::fabs(x0.y) - hy;
    } else {
        if (iy) level = std::fabs(x0.x) - hx;
        else level = wlength(std::fabs(x0.x) - hx, std::fabs(x0.y) - hy);
    }
    return level;
}
// update_solid.wgsl:121-162
inline float level_obstacle(const efl_solid_obstacle& o, F2 x) {
    switch (o.shape) {
        case EFL_SHAPE_CIRCLE:
            return wlength(x.x - o.transform[12], x.y - o.transform[13]) - o.values[0];
        case EFL_SHAPE_RECTANGLE:
            return level_rectangle(o, x);
        case EFL_SHAPE_CAPSULE: {
            F2 a = mat_xy(o.transform, o.values[0], o.values[1]);
            F2 b = mat_xy(o.transform, o.values[2], o.values[3]);
            return dist_segment(x, a, b) - o.values[4];
        }
        case EFL_SHAPE_TRIANGLE: {
            F2 p0 = mat_xy(o.transform, o.values[0], o.values[1]);
            F2 p1 = mat_xy(o.transform, o.values[2], o.values[3]);
            F2 p2 = mat_xy(o.transform, o.values[4], o.values[5]);
            float d0 = dist_segment(x, p0, p1), d1 = dist_segment(x, p1, p2), d2 = dist_segment(x, p2, p0);
            float s0 = dist_sign(x, p0, p1), s1 = dist_sign(x, p1, p2), s2 = dist_sign(x, p2, p0);
            float m = std::fmin(std::fmin(d0, d1), d2);
            if (s0 > 0.0f && s1 > 0.0f && s2 > 0.0f) return -m;
            return m;
        }
        default:
            return LARGE_FLOAT_SOLID;
    }
}
// update_solid.wgsl:111-119
inline F2 velocity_at(const efl_solid_obstacle& o, F2 x) {
    float rx = x.x - o.transform[12], ry = x.y - o.transform[13];
    float w = o.angular_velocity;
    return F2{o.linear_velocity[0] + -w * ry, o.linear_velocity[1] + w * rx};
}
// update_solid.wgsl:15-78 (dispatch_center)
void k_update_solid(eflo_sim& s) {
    const int nx = s.nx, ny = s.ny;
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            F2 xc = to_world(s.U, (float)x, (float)y, nx, ny);
            F2 xex = to_world(s.U, (float)x - 0.5f, (float)y - 0.0f, nx, ny);
            F2 xey = to_world(s.U, (float)x - 0.0f, (float)y - 0.5f, nx, ny);
            if (x == 0 || y == 0 || x == nx - 1 || y == ny - 1) {
                s.ls_solid.st(x, y, 0.0f);
                s.us.st(x, y, 0.0f);
                s.vs.st(x, y, 0.0f);
                s.solid_id.st(x, y, -1);
                continue;
            }
            int tx = std::min(x, std::abs(nx - 1 - x)), ty = std::min(y, std::abs(ny - 1 - y));
            float level = (float)std::min(tx, ty);
            float u = 0.0f, v = 0.0f;
            int32_t sid = -1;
            for (const auto& o : s.obstacles) {
                float lo = level_obstacle(o, xc);
                if (lo < level) level = lo;
                if (lo < 0.5f) sid = (int32_t)o.entity_id;
                float lex = level_obstacle(o, xex);
                if (lex < 0.5f) u = velocity_at(o, xex).x;
                float ley = level_obstacle(o, xey);
                if (ley < 0.5f) v = -velocity_at(o, xey).y;
            }
            s.us.st(x, y, u);
            s.vs.st(x, y, v);
            s.ls_solid.st(x, y, level);
            s.solid_id.st(x, y, sid);
        }
    });
}
// update_area_fraction.wgsl:6-14
void k_area_fraction(eflo_sim& s) {
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) s.af.st(x, y, area_fractions(s.ls_solid, x, y));
    });
}

// utils/coordinate.wgsl:51-81
inline float interp_edge_x(const Tex<float>& u, float px, float py) {
    int i = f2i(std::rint(px));
    int j = f2i(std::floor(py));
    float fi = px + 0.5f - (float)i;
    float fj = py - (float)j;
    float u00 = u.ld(i, j), u10 = u.ld(i + 1, j), u01 = u.ld(i, j + 1), u11 = u.ld(i + 1, j + 1);
    return wmix(wmix(u00, u10, fi), wmix(u01, u11, fi), fj);
}
inline float interp_edge_y(const Tex<float>& v, float px, float py) {
    int i = f2i(std::floor(px));
    int j = f2i(std::rint(py));
    float fi = px - (float)i;
    float fj = py + 0.5f - (float)j;
    float v00 = v.ld(i, j), v10 = v.ld(i + 1, j), v01 = v.ld(i, j + 1), v11 = v.ld(i + 1, j + 1);
    return wmix(wmix(v00, v10, fi), wmix(v01, v11, fi), fj);
}
// utils/coordinate.wgsl:83-94
inline F2 runge_kutta(const Tex<float>& u, const Tex<float>& v, float px, float py, float dt) {
    float vx = interp_edge_x(u, px, py), vy = interp_edge_y(v, px, py);
    float h = 0.5f * dt;
    float mx = px - h * vx, my = py - h * vy;
    float wx = interp_edge_x(u, mx, my), wy = interp_edge_y(v, mx, my);
    return F2{px - dt * wx, py - dt * wy};
}
// advect_velocity.wgsl:11-52
void k_advect(eflo_sim& s) {
    const float dt = s.U.dt;
    // advect_u: dispatch_x_major
    par_rows(0, s.xrows(), [&](int y) {
        for (int x = 0; x <= s.nx; ++x) {
            float px = (float)x + -0.5f, py = (float)y + 0.0f;
            F2 b = runge_kutta(s.u0, s.v0, px, py, dt);
            float dimx = (float)s.u0.w, dimy = (float)s.u0.h;
            bool inside = b.x >= 0.0f && b.y >= 0.0f && b.x <= dimx - 1.0f && b.y <= dimy - 1.0f;
            s.u1.st(x, y, inside ? interp_edge_x(s.u0, b.x, b.y) : s.u0.ld(x, y));
        }
    });
    // advect_v: dispatch_y_major
    par_rows(0, s.ny + 1, [&](int y) {
        for (int x = 0; x < s.ycols(); ++x) {
            float px = (float)x + 0.0f, py = (float)y + -0.5f;
            F2 b = runge_kutta(s.u0, s.v0, px, py, dt);
            float dimx = (float)s.v0.w, dimy = (float)s.v0.h;
            bool inside = b.x >= 0.0f && b.y >= 0.0f && b.x <= dimx - 1.0f && b.y <= dimy - 1.0f;
            s.v1.st(x, y, inside ? interp_edge_y(s.v0, b.x, b.y) : s.v0.ld(x, y));
        }
    });
}

// exp of the Gaussian force splat: WGSL's exp is implementation-defined, so
// the oracle and the CUDA library share one restated method -- Cody-Waite
// reduction x = k ln2 + r (ln2 split hi/lo, |r| <= ln2/2), degree-7 Taylor
// polynomial for exp(r) in Horner form, exact scaling by 2^k.
inline float efl_exp(float x) {
    if (x < -104.0f) return 0.0f;
    if (x > 88.5f) return std::numeric_limits<float>::infinity();
    float kf = std::rint(x * 1.44269504088896341f);
    float r = (x - kf * 0.693145751953125f) - kf * 1.42860682030941723e-6f;
    float p = 1.98412698412698413e-4f;
    p = p * r + 1.38888888888888889e-3f;
    p = p * r + 8.33333333333333333e-3f;
    p = p * r + 4.16666666666666667e-2f;
    p = p * r + 1.66666666666666667e-1f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    return std::ldexp(p, (int)kf);
}
// apply_forces.wgsl:73-76
inline float gaussian_2d(float x, float y, float x0, float y0, float sigma) {
    float b = -1.0f / (2.0f * sigma * sigma);
    float dx = x - x0, dy = y - y0;
    return efl_exp(b * (dx * dx + dy * dy));
}
float exp_for_test(float x) { return efl_exp(x); }
// apply_forces.wgsl:17-71
void k_apply_forces(eflo_sim& s) {
    const Uniform& U = s.U;
    par_rows(0, s.xrows(), [&](int y) {
        for (int x = 0; x <= s.nx; ++x) {
            F4 f = area_fractions(s.ls0, x, y);
            float fs = s.af.ld(x, y).x;
            if (f.x == 1.0f || fs == 0.0f) { s.u1.st(x, y, 0.0f); continue; }
            float net = U.g[0];
            for (size_t n = s.forces.size(); n > 0; --n) {
                const efl_force& F = s.forces[n - 1];
                net = net + F.force[0] * gaussian_2d((float)x, (float)y, F.position[0], F.position[1], 10.0f);
            }
            float uv = s.u1.ld(x, y);
            s.u1.st(x, y, uv + net * U.dt / U.dx);
        }
    });
    par_rows(0, s.ny + 1, [&](int y) {
        for (int x = 0; x < s.ycols(); ++x) {
            F4 f = area_fractions(s.ls0, x, y);
            float fs = s.af.ld(x, y).z;
            if (f.z == 1.0f || fs == 0.0f) { s.v1.st(x, y, 0.0f); continue; }
            float net = U.g[1];
            for (size_t n = s.forces.size(); n > 0; --n) {
                const efl_force& F = s.forces[n - 1];
                net = net + F.force[1] * gaussian_2d((float)x, (float)y, F.position[0], F.position[1], 10.0f);
            }
            float vv = s.v1.ld(x, y);
            s.v1.st(x, y, vv + net * U.dt / U.dx);
        }
    });
}

// divergence.wgsl:16-42 (dispatch_center)
void k_divergence(eflo_sim& s) {
    const float dx = s.U.dx;
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            F4 f = area_fractions(s.ls_solid, x, y);
            float u_ij = s.u1.ld(x, y), u_ip = s.u1.ld(x + 1, y);
            float v_ij = s.v1.ld(x, y), v_jp = s.v1.ld(x, y + 1);
            float du_f = f.y * u_ip - f.x * u_ij;
            float dv_f = f.w * v_jp - f.z * v_ij;
            float us_m = s.us.ld(x, y), us_p = s.us.ld(x + 1, y);
            float vs_m = s.vs.ld(x, y), vs_p = s.vs.ld(x, y + 1);
            float du_s = (1.0f - f.y) * us_p - (1.0f - f.x) * us_m;
            float dv_s = (1.0f - f.w) * vs_p - (1.0f - f.z) * vs_m;
            float rhs = -(du_f + dv_f + du_s + dv_s) / dx;
            s.div.st(x, y, rhs);
        }
    });
}

// projection/shaders/gauss_seidel.wgsl:44-88 (update_pressure).  With
// T = float this is the reference's f32 arithmetic.  With T = double (the
// tolerance-driven solve, an extension) the same loop runs in f64 from the
// f32 inputs and the final division is nume * (1/denom): the CUDA solver
// keeps 1/denom per cell for the whole solve.
template <class T>
inline T gs_update(const Tex<T>& p, const Tex<T>& b, const Tex<float>& ls, const Tex<F4>& af, const Uniform& U,
                   float weight, float res_scale, int x, int y) {
    float lij = ls.ld(x, y);
    if (lij >= 0.0f) return T(0);
    F4 f = af.ld(x, y);
    bool fully_solid = f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f;
    T p_old = p.ld(x, y);
    if (fully_solid) return T(0);
    T denom = T(0);
    T dx = (T)(res_scale * U.dx);
    T nume = dx * dx * (T)U.rho / (T)U.dt * b.ld(x, y);
    static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    const T fv[4] = {(T)f.x, (T)f.y, (T)f.z, (T)f.w};
    for (int i = 0; i < 4; ++i) {
        int jx = x + off[i][0], jy = y + off[i][1];
        if (jx >= 0 && jy >= 0 && jx < ls.w && jy < ls.h) {
            float level = ls.ld(jx, jy);
            if (level < 0.0f) {
                denom += fv[i];
                nume += fv[i] * p.ld(jx, jy);
            } else {
                denom += fv[i] * (T(1) - (T)level / (T)lij);
            }
        }
    }
    if (std::fabs(denom) < (T)1.0e-6f) return T(0);
    T p_new;
    if (std::is_same<T, double>::value) p_new = nume * (T(1) / denom);
    else p_new = nume / denom;
    T w = (T)weight;
    return w * p_new + (T(1) - w) * p_old;
}
// gauss_seidel.wgsl:12-42: red = (x+y) odd, black = (x+y) even; dispatched
// over ceil(dim/8)*8 with a dim guard, so every cell of the level.
template <class T>
void gs_half(Tex<T>& p, const Tex<T>& b, const Tex<float>& ls, const Tex<F4>& af, const Uniform& U, float weight,
             float res_scale, int parity) {
    par_rows(0, p.h, [&](int y) {
        for (int x = (y + parity) & 1; x < p.w; x += 2) p.at(x, y) = gs_update(p, b, ls, af, U, weight, res_scale, x, y);
    });
}
template <class T>
void gs_iterations(Tex<T>& p, const Tex<T>& b, const Tex<float>& ls, const Tex<F4>& af, const Uniform& U,
                   float weight, float res_scale, uint32_t n, bool black_first = false) {
    for (uint32_t k = 0; k < n; ++k) {
        gs_half(p, b, ls, af, U, weight, res_scale, black_first ? 0 : 1);  // red first in the reference
        gs_half(p, b, ls, af, U, weight, res_scale, black_first ? 1 : 0);
    }
}

// projection/shaders/residual.wgsl:12-57.  T = float: the reference's
// operation order.  T = double: the same operator in factored form,
// r = b - factor * (denom * x - sum_fluid f * x_nb), with denom accumulated
// in the reference's neighbour order (the CUDA solver keeps denom per cell).
template <class T>
inline T residual_at(const Tex<T>& xt, const Tex<T>& b, const Tex<float>& ls, const Tex<F4>& af, const Uniform& U,
                     float res_scale, int x, int y, bool* counted) {
    *counted = false;
    float phi = ls.ld(x, y);
    if (phi >= 0.0f) return T(0);
    F4 f = af.ld(x, y);
    if (f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f) return T(0);
    *counted = true;
    T xc = xt.ld(x, y);
    T dx = (T)(U.dx * res_scale);
    T factor = (T)U.dt / (T)U.rho / dx / dx;
    static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    const T fv[4] = {(T)f.x, (T)f.y, (T)f.z, (T)f.w};
    if (std::is_same<T, double>::value) {
        T denom = T(0), sum = T(0);
        for (int i = 0; i < 4; ++i) {
            int jx = x + off[i][0], jy = y + off[i][1];
            if (jx >= 0 && jy >= 0 && jx < ls.w && jy < ls.h) {
                float pn = ls.ld(jx, jy);
                if (pn < 0.0f) {
                    denom += fv[i];
                    sum += fv[i] * xt.ld(jx, jy);
                } else {
                    denom += fv[i] * (T(1) - (T)pn / (T)phi);
                }
            }
        }
        return b.ld(x, y) - factor * (denom * xc - sum);
    }
    T r = b.ld(x, y);
    for (int i = 0; i < 4; ++i) {
        int jx = x + off[i][0], jy = y + off[i][1];
        if (jx >= 0 && jy >= 0 && jx < ls.w && jy < ls.h) {
            float pn = ls.ld(jx, jy);
            if (pn < 0.0f) r -= fv[i] * (xc - xt.ld(jx, jy)) * factor;
            else r -= fv[i] * (T(1) - (T)pn / (T)phi) * xc * factor;
        }
    }
    return r;
}
template <class T>
void k_residual(LevelT<T>& L, const Uniform& U, float res_scale) {
    par_rows(0, L.ny, [&](int y) {
        bool c;
        for (int x = 0; x < L.nx; ++x) L.r.at(x, y) = residual_at(L.x, L.b, L.ls, L.af, U, res_scale, x, y, &c);
    });
}
// restriction.wgsl:10-60
template <class T>
void k_restriction(const LevelT<T>& F, LevelT<T>& C) {
    par_rows(0, C.ny, [&](int y) {
        for (int x = 0; x < C.nx; ++x) {
            int fx = 2 * x, fy = 2 * y;
            T br = T(0.25) * (F.r.ld(fx, fy) + F.r.ld(fx, fy + 1) + F.r.ld(fx + 1, fy) + F.r.ld(fx + 1, fy + 1));
            float ph0 = F.ls.ld(fx, fy), ph1 = F.ls.ld(fx, fy + 1), ph2 = F.ls.ld(fx + 1, fy),
                  ph3 = F.ls.ld(fx + 1, fy + 1);
            float pr = ph0;
            if (std::fabs(ph1) < std::fabs(pr)) pr = ph1;
            if (std::fabs(ph2) < std::fabs(pr)) pr = ph2;
            if (std::fabs(ph3) < std::fabs(pr)) pr = ph3;
            F4 a0 = F.af.ld(fx, fy), a1 = F.af.ld(fx + 1, fy), a2 = F.af.ld(fx, fy + 1), a3 = F.af.ld(fx + 1, fy + 1);
            F4 fr{0.5f * (a0.x + a2.x), 0.5f * (a1.y + a3.y), 0.5f * (a0.z + a1.z), 0.5f * (a2.w + a3.w)};
            C.b.st(x, y, br);
            C.ls.st(x, y, pr);
            C.af.st(x, y, fr);
            C.x.st(x, y, T(0));
        }
    });
}
// prolongation.wgsl:5-34
template <class T>
void k_prolongation(LevelT<T>& F, const LevelT<T>& C) {
    par_rows(0, C.ny, [&](int y) {
        for (int x = 0; x < C.nx; ++x) {
            T corr = C.x.ld(x, y);
            static const int off[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
            for (int i = 0; i < 4; ++i) {
                int fx = 2 * x + off[i][0], fy = 2 * y + off[i][1];
                if (F.ls.ld(fx, fy) < 0.0f && F.x.in(fx, fy)) F.x.at(fx, fy) = corr + F.x.at(fx, fy);
            }
        }
    });
}
// multi_grid.rs:390-475; smoother weight 1.0 and resolution_scale 2^i (multi_grid.rs:268-270)
// symmetric = true (the MGPCG preconditioner, an extension): post-smoothing
// runs black then red, the reverse of pre-smoothing.
template <class T>
void v_cycle(std::vector<LevelT<T>>& mg, const Uniform& U, size_t i, const efl_projection& P, bool symmetric = false) {
    LevelT<T>& L = mg[i];
    float scale = (float)(1u << i);
    if (i == mg.size() - 1) {
        gs_iterations(L.x, L.b, L.ls, L.af, U, 1.0f, scale, P.mg_coarsest);
        return;
    }
    gs_iterations(L.x, L.b, L.ls, L.af, U, 1.0f, scale, P.mg_pre);
    k_residual(L, U, scale);
    k_restriction(L, mg[i + 1]);
    v_cycle(mg, U, i + 1, P, symmetric);
    k_prolongation(L, mg[i + 1]);
    gs_iterations(L.x, L.b, L.ls, L.af, U, 1.0f, scale, P.mg_post, symmetric);
}

// shaders/jacobi_iteration.wgsl:39-91 (levelset_solid fractions = af)
inline float jacobi_update(const Tex<float>& p, const eflo_sim& s, int x, int y) {
    float lij = s.ls0.ld(x, y);
    if (lij >= 0.0f) return 0.0f;
    F4 f = area_fractions(s.ls_solid, x, y);
    bool fully_solid = f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f;
    if (fully_solid) return p.ld(x, y);
    float p_m = p.ld(x - 1, y), p_p = p.ld(x + 1, y), p_jm = p.ld(x, y - 1), p_jp = p.ld(x, y + 1);
    float l_m = s.ls0.ld(x - 1, y), l_p = s.ls0.ld(x + 1, y), l_jm = s.ls0.ld(x, y - 1), l_jp = s.ls0.ld(x, y + 1);
    float ff_m = std::fmin(0.0f, l_m / lij), ff_p = std::fmin(0.0f, l_p / lij);
    float ff_jm = std::fmin(0.0f, l_jm / lij), ff_jp = std::fmin(0.0f, l_jp / lij);
    float coef = f.x * (1.0f - ff_m) + f.y * (1.0f - ff_p) + f.z * (1.0f - ff_jm) + f.w * (1.0f - ff_jp);
    if (std::fabs(coef) < 1.0e-6f) return 0.0f;
    float div_ij = s.div.ld(x, y);
    float factor = s.U.dx * s.U.rho / s.U.dt;
    auto step0 = [](float v) { return v >= 0.0f ? 1.0f : 0.0f; };
    float d00 = f.x * step0(ff_m) * p_m;
    float d10 = f.y * step0(ff_p) * p_p;
    float d01 = f.z * step0(ff_jm) * p_jm;
    float d11 = f.w * step0(ff_jp) * p_jp;
    return (d00 + d10 + d01 + d11 - factor * div_ij) / coef;
}
void k_jacobi(eflo_sim& s) {  // projection.rs:135-143, dispatch_center
    for (int it = 0; it < 50; ++it) {
        par_rows(0, s.cy(), [&](int y) {
            for (int x = 0; x < s.cx(); ++x) s.p1.st(x, y, jacobi_update(s.p0, s, x, y));
        });
        par_rows(0, s.cy(), [&](int y) {
            for (int x = 0; x < s.cx(); ++x) s.p0.st(x, y, jacobi_update(s.p1, s, x, y));
        });
    }
}

// ||b - A x||^2 and ||b||^2 at level 0 over cells with phi < 0 that are
// not fully solid (FP64 accumulation, per-row partials summed in order).
template <class T>
void residual_norms(const Tex<T>& xt, const Tex<T>& b, const Tex<float>& ls, const Tex<F4>& af, const Uniform& U,
                    double* rr, double* bb) {
    const int W = ls.w, H = ls.h;
    std::vector<double> pr(H, 0.0), pb(H, 0.0);
    par_rows(0, H, [&](int y) {
        double sr = 0.0, sb = 0.0;
        for (int x = 0; x < W; ++x) {
            bool c;
            T r = residual_at(xt, b, ls, af, U, 1.0f, x, y, &c);
            if (c) {
                double bv = (double)b.ld(x, y);
                sr += (double)r * (double)r;
                sb += bv * bv;
            }
        }
        pr[y] = sr;
        pb[y] = sb;
    });
    double R = 0.0, B = 0.0;
    for (int y = 0; y < H; ++y) { R += pr[y]; B += pb[y]; }
    *rr = R;
    *bb = B;
}
double rel_from(double R, double B) {
    if (B > 0.0) return std::sqrt(R) / std::sqrt(B);
    return R > 0.0 ? std::numeric_limits<double>::infinity() : 0.0;
}
void residual_norms_f32(const eflo_sim& s, double* R, double* B) {
    residual_norms(s.p0, s.div, s.ls0, s.af, s.U, R, B);
}

void mg_copy_level0(eflo_sim& s) {
    Level& L = s.mg[0];
    L.x = s.p0;
    L.b = s.div;
    L.ls = s.ls0;
    L.af = s.af;
}
// FP64 iterate of the tolerance-driven solve: x = p0, b = div (widened).
void mg64_load_level0(eflo_sim& s) {
    Level64& L = s.mg64[0];
    for (size_t i = 0; i < L.x.a.size(); ++i) {
        L.x.a[i] = (double)s.p0.a[i];
        L.b.a[i] = (double)s.div.a[i];
    }
    L.ls = s.ls0;
    L.af = s.af;
}
void mg64_store_p0(eflo_sim& s) {
    const Level64& L = s.mg64[0];
    for (size_t i = 0; i < L.x.a.size(); ++i) s.p0.a[i] = (float)L.x.a[i];
}

// Tolerance-driven red-black Gauss-Seidel (an extension of projection.rs,
// gauss_seidel.wgsl:44-88) in mixed-precision iterative-refinement form.
// Every check block of n iterations: the FP64 residual r of the FP64 iterate
// p (factored operator, see residual_at<double>) gives the convergence test
// and the f32 right-hand side rc = f32(cdiv * r); n SOR red-black iterations
// then run in f32 on the correction d (start 0) with the per-cell f32
// coefficients w_k (face fraction of fluid in-bounds neighbours, else 0) and
// inv = f32(1 / denom); finally p += d (f64), and cells the reference sets to
// zero (air, fully solid, |denom| < 1e-6) get p = 0.  In exact arithmetic
// this is the SOR iteration itself (it is affine), so iteration counts are
// those of RBGS; the f32 sweeps only carry the correction.
struct MixCell {
    unsigned char mode;  // 0 skip, 1 zero, 2 update; +4 counted
    float w[4];
    float inv;
    double den;
};
void mix_coefficients(const eflo_sim& s, std::vector<MixCell>& cells) {
    const int W = s.nx, Hh = s.ny;
    cells.assign((size_t)W * Hh, MixCell{});
    par_rows(0, Hh, [&](int y) {
        static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
        for (int x = 0; x < W; ++x) {
            MixCell& c = cells[(size_t)y * W + x];
            c.mode = 1;
            float lij = s.ls0.ld(x, y);
            if (!(lij < 0.0f)) continue;
            F4 f = s.af.ld(x, y);
            if (f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f) continue;
            c.mode |= 4;
            const float fv[4] = {f.x, f.y, f.z, f.w};
            double den = 0.0;
            for (int i = 0; i < 4; ++i) {
                int jx = x + off[i][0], jy = y + off[i][1];
                if (jx >= 0 && jy >= 0 && jx < W && jy < Hh) {
                    float level = s.ls0.ld(jx, jy);
                    if (level < 0.0f) {
                        den += (double)fv[i];
                        c.w[i] = fv[i];
                    } else {
                        den += (double)fv[i] * (1.0 - (double)level / (double)lij);
                    }
                }
            }
            c.den = den;
            if (!(std::fabs(den) < (double)1.0e-6f)) {
                c.mode = (unsigned char)((c.mode & 4) | 2);
                c.inv = (float)(1.0 / den);
            }
        }
    });
}
efl_status gs_mixed_solve(eflo_sim& s, uint32_t* iters_out, double* r0_out, double* r1_out) {
    const efl_projection& P = s.cfg.projection;
    const int W = s.nx, Hh = s.ny;
    Level64& L = s.mg64[0];
    std::vector<MixCell> cells;
    mix_coefficients(s, cells);
    const double dx = (double)s.U.dx;
    const double cdiv = dx * dx * (double)s.U.rho / (double)s.U.dt;
    const double factor = (double)s.U.dt / (double)s.U.rho / dx / dx;
    const float w = P.sor_weight, omw = 1.0f - P.sor_weight;
    std::vector<double> r((size_t)W * Hh);
    std::vector<float> rc((size_t)W * Hh), d((size_t)W * Hh);
    auto residual = [&]() {  // fills r, returns the relative residual
        std::vector<double> pr(Hh), pb(Hh);
        par_rows(0, Hh, [&](int y) {
            double sr = 0.0, sb = 0.0;
            static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
            for (int x = 0; x < W; ++x) {
                const MixCell& c = cells[(size_t)y * W + x];
                double rv = 0.0;
                if (c.mode & 4) {
                    double sum = 0.0;
                    for (int i = 0; i < 4; ++i) {
                        int jx = x + off[i][0], jy = y + off[i][1];
                        double pn = (jx >= 0 && jy >= 0 && jx < W && jy < Hh) ? L.x.at(jx, jy) : 0.0;
                        if (i == 0) sum = (double)c.w[0] * pn;
                        else sum = sum + (double)c.w[i] * pn;
                    }
                    const double bv = L.b.at(x, y);
                    rv = bv - factor * (c.den * L.x.at(x, y) - sum);
                    sr += rv * rv;
                    sb += bv * bv;
                }
                r[(size_t)y * W + x] = rv;
            }
            pr[y] = sr;
            pb[y] = sb;
        });
        double R = 0.0, B = 0.0;
        for (int y = 0; y < Hh; ++y) {
            R += pr[y];
            B += pb[y];
        }
        return rel_from(R, B);
    };
    uint32_t iters = 0;
    double rel = residual();
    *r0_out = rel;
    const uint32_t chk = std::max<uint32_t>(1, P.check_interval);
    while (!(rel <= (double)P.tolerance) && iters < P.max_iterations) {
        const uint32_t n = std::min(chk, P.max_iterations - iters);
        par_rows(0, Hh, [&](int y) {
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * W + x;
                rc[i] = (cells[i].mode & 2) ? (float)(cdiv * r[i]) : 0.0f;
                d[i] = 0.0f;
            }
        });
        for (uint32_t it = 0; it < n; ++it) {
            for (int color = 1; color >= 0; --color) {  // red ((x+y) odd) then black
                par_rows(0, Hh, [&](int y) {
                    for (int x = (y + color) & 1; x < W; x += 2) {
                        size_t i = (size_t)y * W + x;
                        const MixCell& c = cells[i];
                        if (!(c.mode & 2)) continue;
                        const float dl = x > 0 ? d[i - 1] : 0.0f, dr = x + 1 < W ? d[i + 1] : 0.0f;
                        const float du = y > 0 ? d[i - W] : 0.0f, dd = y + 1 < Hh ? d[i + W] : 0.0f;
                        float nume = rc[i];
                        nume = nume + c.w[0] * dl;
                        nume = nume + c.w[1] * dr;
                        nume = nume + c.w[2] * du;
                        nume = nume + c.w[3] * dd;
                        d[i] = w * (nume * c.inv) + omw * d[i];
                    }
                });
            }
        }
        par_rows(0, Hh, [&](int y) {
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * W + x;
                double& pv = L.x.at(x, y);
                pv = (cells[i].mode & 2) ? pv + (double)d[i] : 0.0;
            }
        });
        iters += n;
        rel = residual();
    }
    *iters_out = iters;
    *r1_out = rel;
    return EFL_OK;
}

// Reductions of the MGPCG solve, in a fixed order that the CUDA kernels
// reproduce: per row, chunks of 32 columns are each summed in x order from
// 0.0, the chunk sums are added in chunk order from 0.0; the row sums are
// added in row order within groups of 32 rows and the group sums in group
// order, each from 0.0.
struct D2 {
    double x, y;
};
template <class F>
D2 row_ordered_sum(int W, int H, F term) {
    std::vector<D2> rows(H);
    par_rows(0, H, [&](int y) {
        D2 row{0.0, 0.0};
        for (int c = 0; c < W; c += 32) {
            D2 ch{0.0, 0.0};
            for (int x = c; x < std::min(W, c + 32); ++x) {
                D2 t = term(x, y);
                ch.x = ch.x + t.x;
                ch.y = ch.y + t.y;
            }
            row.x = row.x + ch.x;
            row.y = row.y + ch.y;
        }
        rows[y] = row;
    });
    D2 tot{0.0, 0.0};
    for (int g = 0; g < H; g += 32) {  // rows in order within groups of 32, groups in order
        D2 grp{0.0, 0.0};
        for (int y = g; y < std::min(H, g + 32); ++y) {
            grp.x = grp.x + rows[y].x;
            grp.y = grp.y + rows[y].y;
        }
        tot.x = tot.x + grp.x;
        tot.y = tot.y + grp.y;
    }
    return tot;
}

// Multigrid-preconditioned conjugate gradients (EFL_PROJECTION_MGPCG, an
// extension: the reference iterates neither solver to a tolerance).  The
// unknowns are the update cells of the mixed solve (fluid, not fully solid,
// |denom| >= 1e-6); A is the factored FP64 operator of residual_at<double>
// restricted to them (every other cell is held at p = 0).  The
// preconditioner is one f32 V-cycle of the reference's structure
// (multi_grid.rs:390-475: smoother weight 1, mg_pre / mg_post / mg_coarsest
// sweeps, the reference's restriction and prolongation, the f32 arithmetic of
// the reference's shaders) applied to f32(r) from a zero start and made
// symmetric by running post-smoothing black-then-red; its result is widened
// to FP64.  The convergence test is the true relative residual over the
// counted cells after every iteration.
efl_status mgpcg_solve(eflo_sim& s, uint32_t* iters_out, double* r0_out, double* r1_out) {
    const efl_projection& P = s.cfg.projection;
    const int W = s.nx, Hh = s.ny;
    Level64& L = s.mg64[0];
    std::vector<MixCell> cells;
    mix_coefficients(s, cells);
    const double dx = (double)s.U.dx;
    const double factor = (double)s.U.dt / (double)s.U.rho / dx / dx;
    static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    const int PW = L.x.w;  // row stride of the level's textures
    std::vector<double>& X = L.x.a;
    const std::vector<double>& B = L.b.a;
    auto upd = [&](int x, int y) { return (cells[(size_t)y * W + x].mode & 2) != 0; };
    // (A v)(x, y), the factored operator, v = 0 off the unknowns.
    auto apply_at = [&](const std::vector<double>& v, int x, int y) {
        const MixCell& c = cells[(size_t)y * W + x];
        double sum = 0.0;
        for (int i = 0; i < 4; ++i) {
            int jx = x + off[i][0], jy = y + off[i][1];
            double pn = (jx >= 0 && jy >= 0 && jx < W && jy < Hh) ? v[(size_t)jy * PW + jx] : 0.0;
            if (i == 0) sum = (double)c.w[0] * pn;
            else sum = sum + (double)c.w[i] * pn;
        }
        return factor * (c.den * v[(size_t)y * PW + x] - sum);
    };
    auto true_rel = [&]() {
        D2 t = row_ordered_sum(W, Hh, [&](int x, int y) {
            if (!(cells[(size_t)y * W + x].mode & 4)) return D2{0.0, 0.0};
            const double bv = B[(size_t)y * PW + x];
            const double rv = bv - apply_at(X, x, y);
            return D2{rv * rv, bv * bv};
        });
        return rel_from(t.x, t.y);
    };
    // z = M r: the f32 V-cycle on the f32 levels with level 0 set to
    // (x = 0, b = f32(r), the current phi and fractions); z is widened and
    // zero off the unknowns.
    Level& F = s.mg[0];
    auto precondition = [&](const std::vector<double>& r, std::vector<double>& z) {
        for (size_t i = 0; i < F.x.a.size(); ++i) {
            F.x.a[i] = 0.0f;
            F.b.a[i] = (float)r[i];
        }
        F.ls = s.ls0;
        F.af = s.af;
        v_cycle(s.mg, s.U, 0, P, true);
        par_rows(0, Hh, [&](int y) {
            for (int x = 0; x < W; ++x) z[(size_t)y * PW + x] = upd(x, y) ? (double)F.x.at(x, y) : 0.0;
        });
    };
    double rel = true_rel();
    *r0_out = rel;
    uint32_t iters = 0;
    if (!(rel <= (double)P.tolerance) && P.max_iterations > 0) {
        const size_t M = X.size();
        par_rows(0, Hh, [&](int y) {
            for (int x = 0; x < W; ++x)
                if (!upd(x, y)) X[(size_t)y * PW + x] = 0.0;
        });
        std::vector<double> r(M, 0.0), z(M, 0.0), p(M, 0.0), ap(M, 0.0);
        par_rows(0, Hh, [&](int y) {
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * PW + x;
                r[i] = upd(x, y) ? B[i] - apply_at(X, x, y) : 0.0;
            }
        });
        precondition(r, z);
        p = z;
        double rz = row_ordered_sum(W, Hh, [&](int x, int y) {
                        size_t i = (size_t)y * PW + x;
                        return D2{upd(x, y) ? r[i] * z[i] : 0.0, 0.0};
                    }).x;
        while (iters < P.max_iterations) {
            // ap = A p and p . ap in one pass
            const double pap = row_ordered_sum(W, Hh, [&](int x, int y) {
                                   size_t i = (size_t)y * PW + x;
                                   if (!upd(x, y)) {
                                       ap[i] = 0.0;
                                       return D2{0.0, 0.0};
                                   }
                                   ap[i] = apply_at(p, x, y);
                                   return D2{p[i] * ap[i], 0.0};
                               }).x;
            if (!(pap > 0.0)) break;  // breakdown: not positive definite here
            const double alpha = rz / pap;
            par_rows(0, Hh, [&](int y) {
                for (int x = 0; x < W; ++x) {
                    if (!upd(x, y)) continue;
                    size_t i = (size_t)y * PW + x;
                    X[i] = X[i] + alpha * p[i];
                    r[i] = r[i] - alpha * ap[i];
                }
            });
            ++iters;
            rel = true_rel();
            if (rel <= (double)P.tolerance) break;
            precondition(r, z);
            const double rz1 = row_ordered_sum(W, Hh, [&](int x, int y) {
                                   size_t i = (size_t)y * PW + x;
                                   return D2{upd(x, y) ? r[i] * z[i] : 0.0, 0.0};
                               }).x;
            const double beta = rz1 / rz;
            rz = rz1;
            par_rows(0, Hh, [&](int y) {
                for (int x = 0; x < W; ++x) {
                    size_t i = (size_t)y * PW + x;
                    p[i] = upd(x, y) ? z[i] + beta * p[i] : 0.0;
                }
            });
        }
    }
    *iters_out = iters;
    *r1_out = rel;
    return EFL_OK;
}

// projection.rs:89-164.  tolerance > 0 (an extension) solves to
// ||b - A p|| / ||b|| <= tolerance with an FP64 iterate: the f32 pressure
// cannot represent a solution that accurate when the hydrostatic pressure
// dominates.  p0 receives the f32 rounding of the converged iterate.
efl_status k_projection(eflo_sim& s, efl_step_stats* st) {
    const efl_projection& P = s.cfg.projection;
    efl_status ret = EFL_OK;
    uint32_t iters = 0;
    int conv = 1;
    double r0 = -1.0, r1 = -1.0;
    if (P.method == EFL_PROJECTION_JACOBI) {
        k_jacobi(s);
        iters = 50;
    } else if (P.tolerance <= 0.0f) {
        if (P.method == EFL_PROJECTION_GAUSS_SEIDEL) {
            gs_iterations(s.p0, s.div, s.ls0, s.af, s.U, P.sor_weight, 1.0f, P.gs_iterations);
            iters = P.gs_iterations;
        } else {
            mg_copy_level0(s);  // level 0 aliases p0/div/phi0/af (multi_grid.rs:104-107)
            v_cycle(s.mg, s.U, 0, P);
            iters = 1;
            s.p0 = s.mg[0].x;
        }
    } else {
        mg64_load_level0(s);
        Level64& L = s.mg64[0];
        auto rel = [&]() {
            double R, B;
            residual_norms(L.x, L.b, L.ls, L.af, s.U, &R, &B);
            return rel_from(R, B);
        };
        double r = rel();
        r0 = r;
        if (P.method == EFL_PROJECTION_GAUSS_SEIDEL || P.method == EFL_PROJECTION_MGPCG) {
            double a, b;
            if (P.method == EFL_PROJECTION_GAUSS_SEIDEL) gs_mixed_solve(s, &iters, &a, &b);
            else mgpcg_solve(s, &iters, &a, &b);
            r0 = a;
            r = b;
        } else {
            while (!(r <= (double)P.tolerance) && iters < P.max_iterations) {
                v_cycle(s.mg64, s.U, 0, P);
                ++iters;
                r = rel();
            }
        }
        r1 = r;
        conv = r <= (double)P.tolerance;
        mg64_store_p0(s);
    }
    if (!conv) ret = EFL_NOT_CONVERGED;
    if (st) {
        st->pressure_iterations = iters;
        st->converged = conv;
        st->residual = r1;
        st->residual_initial = r0;
    }
    return ret;
}

// solve_velocity_u.wgsl:15-47 / solve_velocity_v.wgsl:15-45
void k_solve_velocity(eflo_sim& s) {
    const float factor = s.U.dt / (s.U.dx * s.U.rho);
    par_rows(0, s.xrows(), [&](int y) {
        for (int x = 0; x <= s.nx; ++x) {
            float fr = s.af.ld(x, y).x;
            if (fr == 0.0f) { s.u0.st(x, y, s.us.ld(x, y)); continue; }
            float pij = s.p0.ld(x, y), pim = s.p0.ld(x - 1, y);
            float lp = s.ls0.ld(x, y), lm = s.ls0.ld(x - 1, y);
            if (lm >= 0.0f && lp < 0.0f) pim = lm / lp * pij;
            else if (lm < 0.0f && lp >= 0.0f) pij = lp / lm * pim;
            else if (lm >= 0.0f && lp >= 0.0f) { s.u0.st(x, y, 0.0f); continue; }
            float u = s.u1.ld(x, y);
            s.u0.st(x, y, u - factor * (pij - pim));
        }
    });
    par_rows(0, s.ny + 1, [&](int y) {
        for (int x = 0; x < s.ycols(); ++x) {
            float fr = s.af.ld(x, y).z;
            if (fr == 0.0f) { s.v0.st(x, y, s.vs.ld(x, y)); continue; }
            float pij = s.p0.ld(x, y), pjm = s.p0.ld(x, y - 1);
            float lp = s.ls0.ld(x, y), lm = s.ls0.ld(x, y - 1);
            if (lm >= 0.0f && lp < 0.0f) pjm = lm / lp * pij;
            else if (lm < 0.0f && lp >= 0.0f) pij = lp / lm * pjm;
            float v = s.v1.ld(x, y);
            s.v0.st(x, y, v - factor * (pij - pjm));
        }
    });
}

// extrapolate/initialize_{u,v}_valid.wgsl:6-30
void k_init_valid(eflo_sim& s) {
    par_rows(0, s.xrows(), [&](int y) {
        for (int x = 0; x <= s.nx; ++x) {
            float c0 = s.ls0.ld(x - 1, y - 1), c1 = s.ls0.ld(x, y - 1), c2 = s.ls0.ld(x - 1, y),
                  c3 = s.ls0.ld(x, y), c4 = s.ls0.ld(x - 1, y + 1), c5 = s.ls0.ld(x, y + 1);
            float vm = 0.25f * (c0 + c1 + c2 + c3);
            float vp = 0.25f * (c2 + c3 + c4 + c5);
            s.u_valid_in.st(x, y, area_fraction(vm, vp) > 0.0f ? 0 : 1);
        }
    });
    par_rows(0, s.ny + 1, [&](int y) {
        for (int x = 0; x < s.ycols(); ++x) {
            float c0 = s.ls0.ld(x - 1, y - 1), c1 = s.ls0.ld(x - 1, y), c2 = s.ls0.ld(x, y - 1),
                  c3 = s.ls0.ld(x, y), c4 = s.ls0.ld(x + 1, y - 1), c5 = s.ls0.ld(x + 1, y);
            float vm = 0.25f * (c0 + c1 + c2 + c3);
            float vp = 0.25f * (c2 + c3 + c4 + c5);
            s.v_valid_in.st(x, y, area_fraction(vm, vp) > 0.0f ? 0 : 1);
        }
    });
}
// extrapolate/extrapolate_{u,v}.wgsl:5-63 (one dispatch over [x0,x1) x [y0,y1))
void extrap_pass(Tex<float>& f, const Tex<int32_t>& vin, Tex<int32_t>& vout, int x1, int y1) {
    const int dx_ = vin.w, dy_ = vin.h;
    par_rows(0, y1, [&](int y) {
        for (int x = 0; x < x1; ++x) {
            if (vin.ld(x, y) == 1) { vout.st(x, y, 1); continue; }
            int count = 0;
            float nu = 0.0f;
            if (x + 1 < dx_ && y < dy_ && vin.ld(x + 1, y) == 1) { nu += f.ld(x + 1, y); count += 1; }
            if (x - 1 > 0 && y > 0 && vin.ld(x - 1, y) == 1) { nu += f.ld(x - 1, y); count += 1; }
            if (x < dx_ && y + 1 < dy_ && vin.ld(x, y + 1) == 1) { nu += f.ld(x, y + 1); count += 1; }
            if (x > 0 && y - 1 > 0 && vin.ld(x, y - 1) == 1) { nu += f.ld(x, y - 1); count += 1; }
            if (count > 0) {
                nu /= (float)count;
                f.st(x, y, nu);
                vout.st(x, y, 1);
            } else {
                vout.st(x, y, 0);
            }
        }
    });
}
// render_node.rs:540-608
void k_extrapolate(eflo_sim& s) {
    k_init_valid(s);
    for (int k = 0; k < 10 / 2; ++k) {
        extrap_pass(s.u0, s.u_valid_in, s.u_valid_out, s.nx + 1, s.xrows());
        extrap_pass(s.u0, s.u_valid_out, s.u_valid_in, s.nx + 1, s.xrows());
        extrap_pass(s.v0, s.v_valid_in, s.v_valid_out, s.ycols(), s.ny + 1);
        extrap_pass(s.v0, s.v_valid_out, s.v_valid_in, s.ycols(), s.ny + 1);
    }
}

// advect_levelset.wgsl:49-61
inline float cubic1d(float y0, float y1, float y2, float y3, float t) {
    float d1 = 0.5f * (y2 - y0);
    float d2 = 0.5f * (y3 - y1);
    float a0 = y1, a1 = d1;
    float a2 = -2.0f * d1 - d2 + 3.0f * (y2 - y1);
    float a3 = d1 + d2 - 2.0f * (y2 - y1);
    return a3 * t * t * t + a2 * t * t + a1 * t + a0;
}
inline float cubic1d_x(const Tex<float>& t, int bx, int by, float tx) {
    return cubic1d(t.ld(bx - 1, by), t.ld(bx, by), t.ld(bx + 1, by), t.ld(bx + 2, by), tx);
}
// advect_levelset.wgsl:11-34 with CUBIC (advect_levelset.rs:62)
void k_advect_levelset(eflo_sim& s) {
    const float dt = s.U.dt;
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            F2 xn = runge_kutta(s.u0, s.v0, (float)x, (float)y, dt);
            xn.x = fclamp(xn.x, 0.0f, (float)s.nx - 1.0f);
            xn.y = fclamp(xn.y, 0.0f, (float)s.ny - 1.0f);
            int bx = f2i(xn.x), by = f2i(xn.y);
            float tx = xn.x - (float)bx, ty = xn.y - (float)by;
            float y0 = cubic1d_x(s.ls0, bx, by - 1, tx), y1 = cubic1d_x(s.ls0, bx, by, tx);
            float y2 = cubic1d_x(s.ls0, bx, by + 1, tx), y3 = cubic1d_x(s.ls0, bx, by + 2, tx);
            float nl = cubic1d(y0, y1, y2, y3, ty);
            if (std::fabs(nl) < 1000.0f) s.ls1.st(x, y, nl);
        }
    });
}

// update_fluid_source.wgsl:89-107
inline float level_aabb(float hx, float hy, float cx, float cy, float px, float py) {
    float level = LARGE_FLOAT_SOURCE;
    float dx = std::fabs(cx - px) - hx, dy = std::fabs(cy - py) - hy;
    bool ix = dx < 0.0f, iy = dy < 0.0f;
    if (ix) level = iy ? std::fmax(dx, dy) : dy;
    else level = iy ? dx : wlength(dx, dy);
    return level;
}
// update_fluid_source.wgsl:72-87
inline float level_source(const efl_source& d, float px, float py) {
    switch (d.shape) {
        case EFL_SOURCE_CIRCLE: return wlength(d.center[0] - px, d.center[1] - py) - d.data[0];
        case EFL_SOURCE_AABB: return level_aabb(d.data[0], d.data[1], d.center[0], d.center[1], px, py);
        default: return 0.0f;
    }
}
// update_fluid_source.wgsl:30-70 (dispatch_center).  Faces written by two
// invocations take the raster-last writer's value.
void k_fluid_source(eflo_sim& s, const std::vector<efl_source>& src) {
    const int W = s.cx(), H = s.cy();
    std::vector<uint8_t> upd((size_t)W * H, 0);
    std::vector<F2> vel((size_t)W * H, F2{0, 0});
    const float dimx = (float)s.nx, dimy = (float)s.ny;
    par_rows(0, H, [&](int y) {
        for (int x = 0; x < W; ++x) {
            float uvx = (float)(uint32_t)x / dimx, uvy = (float)(uint32_t)y / dimy;
            float ndcx = uvx * 2.0f + -1.0f, ndcy = uvy * -2.0f + 1.0f;  // bevy uv_to_ndc
            float px = 0.5f * dimx * ndcx, py = 0.5f * dimy * ndcy;
            float nl = s.ls1.ld(x, y);
            float vx = 0.0f, vy = 0.0f;
            bool has_source = false, vu = false;
            for (const auto& d : src) {
                float sdf = level_source(d, px, py);
                if (d.mode == EFL_SOURCE_MODE_SOURCE) {
                    nl = std::fmin(nl, sdf);
                    has_source = true;
                    if (sdf < 0.0f) { vx = vx + d.velocity[0]; vy = vy + d.velocity[1]; vu = true; }
                } else {
                    if (!has_source) nl = std::fmax(nl, -sdf);
                }
            }
            s.ls1.st(x, y, nl);
            upd[(size_t)y * W + x] = vu;
            vel[(size_t)y * W + x] = F2{vx, vy};
        }
    });
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            if (!upd[i]) continue;
            s.u0.st(x, y, vel[i].x);
            s.u0.st(x + 1, y, vel[i].x);
            s.v0.st(x, y, vel[i].y);
            s.v0.st(x, y + 1, vel[i].y);
        }
}

// jump_flooding/initialize.wgsl:8-41
void k_jfa_init(eflo_sim& s) {
    Tex<F2>& sd = s.seeds[0];
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            float md = 10.0f;
            F2 seed{-1.0f, -1.0f};
            float level = s.ls1.ld(x, y);
            for (int i = -1; i <= 1; ++i)
                for (int j = -1; j <= 1; ++j) {
                    if (i == 0 && j == 0) continue;
                    int nx_ = x + i, ny_ = y + j;
                    if (nx_ < 0 || ny_ < 0 || nx_ >= s.nx || ny_ >= s.ny) continue;
                    float nl = s.ls1.ld(nx_, ny_);
                    if (nl >= 0.0f && !(level >= 0.0f)) {
                        float t = level / (level - nl);
                        if (std::fabs(t) < md) {
                            md = std::fabs(t);
                            seed = F2{(float)x + t * (float)i, (float)y + t * (float)j};
                        }
                    }
                }
            sd.st(x, y, seed);
        }
    });
}
inline bool valid_seed(F2 s) { return s.x != -1.0f && s.y != -1.0f; }
// jump_flooding/iterate.wgsl:18-56
void k_jfa_iterate(const Tex<F2>& in, Tex<F2>& out, int step, int cx, int cy) {
    par_rows(0, cy, [&](int y) {
        for (int x = 0; x < cx; ++x) {
            F2 cur = in.ld(x, y), best = cur;
            float bd = 1e10f;
            if (valid_seed(cur)) bd = wlength(cur.x - (float)x, cur.y - (float)y);
            for (int i = -1; i <= 1; ++i)
                for (int j = -1; j <= 1; ++j) {
                    if (i == 0 && j == 0) continue;
                    int nx_ = x + i * step, ny_ = y + j * step;
                    if (nx_ < 0 || ny_ < 0 || nx_ >= in.w || ny_ >= in.h) continue;
                    F2 ns = in.ld(nx_, ny_);
                    if (!valid_seed(ns)) continue;
                    float cd = wlength(ns.x - (float)x, ns.y - (float)y);
                    if (cd < bd) { best = ns; bd = cd; }
                }
            out.st(x, y, best);
        }
    });
}
// jump_flooding/calculate_sdf.wgsl:9-23
void k_jfa_sdf(eflo_sim& s, const Tex<F2>& sd) {
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            F2 seed = sd.ld(x, y);
            float sdf = wlength(seed.x - (float)x, seed.y - (float)y);
            float level = s.ls1.ld(x, y);
            float sg = level < 0.0f ? -1.0f : 1.0f;
            s.ls0.st(x, y, sdf * sg);
        }
    });
}
// jump_flooding.rs:201-209: steps 2^max_power .. 1, max_power = floor(log2(max(nx,ny)) - 1)
std::vector<int> jfa_steps(int nx, int ny) {
    int mp = (int)std::floor(std::log2((float)std::max(nx, ny)) - 1.0f);
    std::vector<int> st;
    uint32_t step = 1u << (mp + 1);
    for (int k = 0; k < mp + 1; ++k) { step /= 2; st.push_back((int)step); }
    return st;
}
void k_jfa(eflo_sim& s) {  // reinitialize_levelset.rs:170-206
    k_jfa_init(s);
    int src = 0, dst = 1;
    for (int step : jfa_steps(s.nx, s.ny)) {
        k_jfa_iterate(s.seeds[src], s.seeds[dst], step, s.cx(), s.cy());
        std::swap(src, dst);
    }
    s.seeds_final = src;
    k_jfa_sdf(s, s.seeds[src]);
}

// fast_iterative_method/initialize.wgsl:10-40
void k_fim_init(eflo_sim& s) {
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            float level = s.ls1.ld(x, y);
            static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
            bool src = false;
            for (int i = 0; i < 4 && !src; ++i) {
                int jx = x + off[i][0], jy = y + off[i][1];
                if (jx >= 0 && jy >= 0 && jx < s.nx && jy < s.ny) {
                    if (level * s.ls1.ld(jx, jy) <= 0.0f) src = true;
                }
            }
            if (src) { s.ls0.st(x, y, level); s.labels0.st(x, y, LABEL_SOURCE); }
            else { s.ls0.st(x, y, wsign(level) * FIM_LARGE); s.labels0.st(x, y, LABEL_NONE); }
        }
    });
}
// fast_iterative_method/initialize_active_label.wgsl:8-40
void k_fim_active(eflo_sim& s) {
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            uint32_t l = s.labels0.ld(x, y);
            if (l == LABEL_SOURCE) { s.labels.st(x, y, LABEL_SOURCE); continue; }
            static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
            uint32_t out = LABEL_NONE;
            for (int i = 0; i < 4; ++i) {
                int jx = x + off[i][0], jy = y + off[i][1];
                if (jx >= 0 && jy >= 0 && jx < s.nx && jy < s.ny && s.labels0.ld(jx, jy) == LABEL_SOURCE) {
                    out = LABEL_ACTIVE;
                    break;
                }
            }
            s.labels.st(x, y, out);
        }
    });
}
// fast_iterative_method/update.wgsl:73-83
inline float abs_get_phi(const Tex<float>& p, int x, int y) {
    if (x < 0 || y < 0 || x >= p.w || y >= p.h) return FIM_LARGE;
    return std::fabs(p.ld(x, y));
}
// fast_iterative_method/update.wgsl:56-71
inline float solve_quadratic_2d(const Tex<float>& p, int x, int y) {
    float xm = std::fmin(abs_get_phi(p, x - 1, y), abs_get_phi(p, x + 1, y));
    float ym = std::fmin(abs_get_phi(p, x, y - 1), abs_get_phi(p, x, y + 1));
    float d = xm - ym;
    if (d > SQRT2_F) return ym + 1.0f;
    if (d < -SQRT2_F) return xm + 1.0f;
    return 0.5f * (xm + ym + std::sqrt(2.0f - d * d));
}
// Deterministic resolution of fast_iterative_method/update.wgsl:13-54.
// The reference writes neighbours' phi and labels from inside one dispatch
// (a data race).  Both the oracle and the CUDA library run it as two
// phases per iteration:
//   A (every ACTIVE cell, reading the iteration-start phi S): q = solve(S)*sign(p);
//     the cell keeps q; it is marked converged if !(|p-q| > eps).
//   B (every cell whose label was NONE): if any 4-neighbour converged in A,
//     the writer is the raster-last such neighbour (down, right, left, up);
//     q_c = solve(phi after A); if |phi_c| > q_c the cell takes q_c*sign(writer)
//     and becomes ACTIVE.  Converged cells become NONE.
void fim_update_two_phase(eflo_sim& s) {
    Tex<float>& S = s.ls0;
    Tex<float>& T = s.phiT;
    Tex<uint32_t>& L = s.labels;
    Tex<uint32_t>& LT = s.labelsT;
    const int W = s.cx(), H = s.cy();
    par_rows(0, H, [&](int y) {  // phase A
        for (int x = 0; x < W; ++x) {
            uint32_t l = L.ld(x, y);
            float p = S.ld(x, y);
            if (l != LABEL_ACTIVE) { T.st(x, y, p); LT.st(x, y, l); continue; }
            float q = solve_quadratic_2d(S, x, y) * wsign(p);
            T.st(x, y, q);
            LT.st(x, y, (std::fabs(p - q) > FIM_EPS) ? LABEL_ACTIVE : LABEL_CONVERGED);
        }
    });
    par_rows(0, H, [&](int y) {  // phase B
        for (int x = 0; x < W; ++x) {
            uint32_t l = LT.ld(x, y);
            float t = T.ld(x, y);
            if (l == LABEL_NONE) {
                // writers in raster-last order: (x,y+1), (x+1,y), (x-1,y), (x,y-1)
                static const int wo[4][2] = {{0, 1}, {1, 0}, {-1, 0}, {0, -1}};
                int wx = -1, wy = -1;
                for (int k = 0; k < 4; ++k) {
                    int ax = x + wo[k][0], ay = y + wo[k][1];
                    if (ax >= 0 && ay >= 0 && ax < W && ay < H && LT.ld(ax, ay) == LABEL_CONVERGED) {
                        wx = ax; wy = ay;
                        break;
                    }
                }
                if (wx >= 0) {
                    float pn = std::fabs(t);
                    float qn = solve_quadratic_2d(T, x, y);
                    if (pn > qn) {
                        S.st(x, y, qn * wsign(T.ld(wx, wy)));
                        L.st(x, y, LABEL_ACTIVE);
                        continue;
                    }
                }
                S.st(x, y, t);
                L.st(x, y, LABEL_NONE);
            } else {
                S.st(x, y, t);
                L.st(x, y, l == LABEL_CONVERGED ? LABEL_NONE : l);
            }
        }
    });
}
// Literal single-invocation-at-a-time raster execution of update.wgsl:13-54.
void fim_update_serial(eflo_sim& s) {
    Tex<float>& phi = s.ls0;
    Tex<uint32_t>& lab = s.labels;
    for (int y = 0; y < s.cy(); ++y)
        for (int x = 0; x < s.cx(); ++x) {
            if (lab.ld(x, y) != LABEL_ACTIVE) continue;
            float p = phi.ld(x, y);
            float q = solve_quadratic_2d(phi, x, y) * wsign(p);
            phi.st(x, y, q);
            if (std::fabs(p - q) > FIM_EPS) continue;
            lab.st(x, y, LABEL_NONE);
            static const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
            for (int i = 0; i < 4; ++i) {
                int jx = x + off[i][0], jy = y + off[i][1];
                if (jx >= 0 && jy >= 0 && jx < s.nx && jy < s.ny) {
                    uint32_t ln = lab.ld(jx, jy);
                    if (ln != LABEL_ACTIVE && ln != LABEL_SOURCE) {
                        float pn = std::fabs(phi.ld(jx, jy));
                        float qn = solve_quadratic_2d(phi, jx, jy);
                        if (pn > qn) {
                            phi.st(jx, jy, qn * wsign(p));
                            lab.st(jx, jy, LABEL_ACTIVE);
                        }
                    }
                }
            }
        }
}
void k_fim(eflo_sim& s) {  // reinitialize_levelset.rs:207-241
    k_fim_init(s);
    k_fim_active(s);
    for (uint32_t k = 0; k < s.cfg.reinit.fim_iterations; ++k) {
        if (s.fim_serial) fim_update_serial(s);
        else fim_update_two_phase(s);
    }
}
void k_reinit(eflo_sim& s) {
    if (s.cfg.reinit.method == EFL_REINIT_JUMP_FLOODING) k_jfa(s);
    else k_fim(s);
}

// levelset_gradient.wgsl:4-21
void k_gradient(eflo_sim& s) {
    par_rows(0, s.cy(), [&](int y) {
        for (int x = 0; x < s.cx(); ++x) {
            if (x == 0 || y == 0 || x >= s.nx || y >= s.ny) continue;
            F2 g{0.5f * (s.ls0.ld(x + 1, y) - s.ls0.ld(x - 1, y)), 0.5f * (s.ls0.ld(x, y + 1) - s.ls0.ld(x, y - 1))};
            s.grad.st(x, y, g);
        }
    });
}

// solid_obstacle.wgsl:67-89
inline F2 center_of_mass(const efl_solid_obstacle& o) {
    switch (o.shape) {
        case EFL_SHAPE_CIRCLE:
        case EFL_SHAPE_RECTANGLE:
        case EFL_SHAPE_CAPSULE:
            return F2{o.transform[12], o.transform[13]};
        case EFL_SHAPE_TRIANGLE: {
            float lx = (o.values[0] + o.values[2] + o.values[4]) / 3.0f;
            float ly = (o.values[1] + o.values[3] + o.values[5]) / 3.0f;
            return mat_xy(o.transform, lx, ly);
        }
        default:
            return F2{0.0f, 0.0f};
    }
}
// fixed_point_conversion.wgsl:2-13
inline int32_t f32_to_i32(float v) { return f2i(v * 10.0f); }
inline float i32_to_f32(int32_t v) { return (float)v * 0.1f; }
// sample_forces.wgsl:20-53 + accumulate_forces.wgsl:16-32; bins zeroed
// every frame (fluid_to_solid.rs:211-229).
void k_solid_forces(eflo_sim& s) {
    std::memset(s.bins, 0, sizeof(s.bins));
    const Uniform& U = s.U;
    efl_solid_obstacle zero_ob;
    std::memset(&zero_ob, 0, sizeof(zero_ob));
    // integer atomics are order-independent: accumulate row partials
    for (int y = 0; y < s.cy(); ++y)
        for (int x = 0; x < s.cx(); ++x) {
            F4 f = area_fractions(s.ls_solid, x, y);
            if (f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f) continue;
            int32_t id = s.solid_id.ld(x, y);
            if (id == -1) continue;
            float p = s.p0.ld(x, y);
            float fx = -(f.y - f.x) * p * U.dx;
            float fy = -(f.w - f.z) * p * U.dx;
            const efl_solid_obstacle& o =
                (id >= 0 && (uint32_t)id < s.obstacles.size()) ? s.obstacles[id] : zero_ob;
            F2 c = center_of_mass(o);
            float uvx = (float)x / U.size[0], uvy = (float)y / U.size[1];
            float xx = (uvx - 0.5f) * U.size[0], yy = (-uvy + 0.5f) * U.size[1];
            F2 w = mat_xy(U.m, xx, yy);
            float rx = w.x - c.x, ry = w.y - c.y;
            float torque = rx * fy - ry * fx;
            if (id >= 0 && id < EFL_MAX_SOLIDS) {
                s.bins[0][id] += f32_to_i32(fx);
                s.bins[1][id] += f32_to_i32(fy);
                s.bins[2][id] += f32_to_i32(torque);
            }
        }
    for (int i = 0; i < EFL_MAX_SOLIDS; ++i) {
        s.out_forces[i].force[0] = i32_to_f32(s.bins[0][i]);
        s.out_forces[i].force[1] = i32_to_f32(s.bins[1][i]);
        s.out_forces[i].torque = i32_to_f32(s.bins[2][i]);
        s.out_forces[i]._pad = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Two-layer particle level set (particle_levelset_two_layers/**).
//
// The reference appends with atomicAdd and sorts into cells with an atomic
// cursor; here every append runs in cell order (x fastest) and attempt order,
// and the sort is a stable counting sort, the order the CUDA library fixes.

constexpr uint32_t PLS_PER_CELL = 16;  // constants.wgsl:3
constexpr float PLS_BAND = 3.0f;       // constants.wgsl:5
constexpr float PLS_SCALE = 10000.0f;  // fixed_point.wgsl:3

inline uint32_t f2u(float v) {  // WGSL u32(f32): truncate, saturate, NaN -> 0
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
}
inline int32_t pls_fixed(float v) { return f2i(v * PLS_SCALE); }           // fixed_point.wgsl:8-10
inline float pls_float(int32_t v) { return (float)v / PLS_SCALE; }          // fixed_point.wgsl:4-6

// utils/coordinate.wgsl:19-33
inline float interp_center(const Tex<float>& t, float x, float y) {
    int i = f2i(std::floor(x));
    int j = f2i(std::floor(y));
    float fi = x - (float)i;
    float fj = y - (float)j;
    float l00 = t.ld(i, j), l10 = t.ld(i + 1, j), l01 = t.ld(i, j + 1), l11 = t.ld(i + 1, j + 1);
    return wmix(wmix(l00, l10, fi), wmix(l01, l11, fi), fj);
}
// utils/coordinate.wgsl:35-49
inline F2 interp_center_rg(const Tex<F2>& t, float x, float y) {
    int i = f2i(std::floor(x));
    int j = f2i(std::floor(y));
    float fi = x - (float)i;
    float fj = y - (float)j;
    F2 l00 = t.ld(i, j), l10 = t.ld(i + 1, j), l01 = t.ld(i, j + 1), l11 = t.ld(i + 1, j + 1);
    return F2{wmix(wmix(l00.x, l10.x, fi), wmix(l01.x, l11.x, fi), fj),
              wmix(wmix(l00.y, l10.y, fi), wmix(l01.y, l11.y, fi), fj)};
}

// utils/hash.wgsl:3-74 (both rotations by 15 bits, as written there)
inline uint32_t rotl32(uint32_t x) { return (x << 15u) | (x >> 17u); }
inline uint32_t murmur3_block(uint32_t src, uint32_t seed) {
    uint32_t k = src, h = seed;
    k *= 0xcc9e2d51u;
    k = rotl32(k);
    k *= 0x1b873593u;
    h ^= k;
    h = rotl32(h);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
inline float bits_to_unit(uint32_t h) {
    uint32_t b = (h & 0x007fffffu) | 0x3f800000u;
    float f;
    std::memcpy(&f, &b, 4);
    return f - 1.0f;
}
inline uint32_t fbits(float v) {
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return b;
}
inline F2 hash22(F2 v) {
    return F2{bits_to_unit(murmur3_block(fbits(v.x), 12345u)), bits_to_unit(murmur3_block(fbits(v.y), 98765u))};
}
inline float hash11(float v) { return bits_to_unit(murmur3_block(fbits(v), 11111u)); }

// particle.wgsl:50-54
inline float particle_radius(float phi) { return fclamp(std::fabs(phi), 0.1f, 0.5f); }

// particle.wgsl:19-30
inline bool is_escaped(const OParticle& p, const Tex<float>& ls) {
    float phi = interp_center(ls, p.x, p.y);
    return p.sign * phi + p.radius < 0.0f;
}

// particle.wgsl:36-82; normalize(g) = g / length(g)
bool spawn_and_attract(const eflo_sim& s, F2 x, float phi_goal, float bmin, float bmax, float sign, OParticle* out) {
    const Tex<float>& ls = s.ls0;
    float lambda = 1.0f;
    float phi = interp_center(ls, x.x, x.y);
    F2 g = interp_center_rg(s.grad, x.x, x.y);
    float len = wlength(g.x, g.y);
    F2 gn{g.x / len, g.y / len};
    float step = lambda * (phi_goal - phi);
    F2 xn{x.x + step * gn.x, x.y + step * gn.y};
    float fx = (float)s.nx, fy = (float)s.ny;
    if (!(0.0f < xn.x && 0.0f < xn.y && xn.x < fx - 1.0f && xn.y < fy - 1.0f)) return false;
    float phi_new = interp_center(ls, xn.x, xn.y);
    if (!(bmin <= phi_new && phi_new <= bmax)) return false;
    *out = OParticle{xn.x, xn.y, particle_radius(phi_new), sign, 0u};
    return true;
}

void pls_append(eflo_sim& s, int layer, const OParticle& p) {
    if (s.parts[layer].size() >= (size_t)s.nx * s.ny * PLS_PER_CELL) {
        ++s.pls_dropped;
        return;
    }
    s.parts[layer].push_back(p);
}

// update_interface_band_mask.wgsl:7-17 + initialize_particles.wgsl:17-58
void pls_initialize(eflo_sim& s) {
    const float bmin = 0.1f, bmax = PLS_BAND;
    const float bmin_neg = -bmax, bmax_neg = -bmin;
    for (int y = 0; y < s.cy(); ++y)
        for (int x = 0; x < s.cx(); ++x) {
            if (!(std::fabs(s.ls0.ld(x, y)) < PLS_BAND)) continue;
            const F2 xb{(float)x, (float)y};
            const uint32_t cell_id = (uint32_t)x + (uint32_t)s.nx * (uint32_t)y;
            for (uint32_t i = 0; i < PLS_PER_CELL; ++i) {
                uint32_t seed = cell_id + i;
                F2 h = hash22(F2{xb.x + (float)seed, xb.y + (float)seed});
                F2 xp{xb.x + h.x, xb.y + h.y};
                float goal = hash11((float)seed) * (bmax - bmin) + bmin;
                OParticle p;
                if (spawn_and_attract(s, xp, goal, bmin, bmax, 1.0f, &p)) pls_append(s, 0, p);
                uint32_t seed_neg = cell_id + i + 1000u;
                float goal_neg = hash11((float)seed_neg) * (bmax_neg - bmin_neg) + bmin_neg;
                // initialize_particles.wgsl:50 spawns from x, not x_neg
                if (spawn_and_attract(s, xp, goal_neg, bmin_neg, bmax_neg, -1.0f, &p)) pls_append(s, 1, p);
            }
        }
}

// advect_particles.wgsl:15-33, utils/coordinate.wgsl:96-109
void pls_advect(eflo_sim& s) {
    const float dt = s.U.dt;
    for (auto& layer : s.parts) {
        const int64_t n = (int64_t)layer.size();
#pragma omp parallel for schedule(static) if (g_threads != 1)
        for (int64_t i = 0; i < n; ++i) {
            OParticle& p = layer[i];
            float x = p.x, y = p.y;
            float u0x = interp_edge_x(s.u0, x, y), u0y = interp_edge_y(s.v0, x, y);
            float x1 = x + dt * u0x, y1 = y + dt * u0y;
            float u1x = interp_edge_x(s.u0, x1, y1), u1y = interp_edge_y(s.v0, x1, y1);
            float x2 = 0.75f * x + 0.25f * (x1 + dt * u1x);
            float y2 = 0.75f * y + 0.25f * (y1 + dt * u1y);
            float u2x = interp_edge_x(s.u0, x2, y2), u2y = interp_edge_y(s.v0, x2, y2);
            p.x = (float)(1.0 / 3.0) * x + (float)(2.0 / 3.0) * (x2 + dt * u2x);
            p.y = (float)(1.0 / 3.0) * y + (float)(2.0 / 3.0) * (y2 + dt * u2y);
        }
    }
}

// levelset_correction.rs:96-155 / :157-236 in dispatch order:
// mark_escaped_particles, reset_levelset_correction,
// accumulate_levelset_correction (+, then -), correct_levelset
// [, update_particle_radii for both layers].
void pls_correct(eflo_sim& s, Tex<float>& ls, bool second) {
    for (auto& layer : s.parts)
        for (auto& p : layer) p.escaped = is_escaped(p, ls) ? 1u : 0u;
    const uint32_t nx = (uint32_t)s.nx, ny = (uint32_t)s.ny;
    s.phi_plus.assign((size_t)nx * ny, 0);
    s.phi_minus.assign((size_t)nx * ny, 0);
    for (int y = 0; y < s.cy(); ++y)
        for (int x = 0; x < s.cx(); ++x) {
            int32_t q = pls_fixed(ls.ld(x, y));
            s.phi_plus[(size_t)y * nx + x] = q;
            s.phi_minus[(size_t)y * nx + x] = q;
        }
    for (int layer = 0; layer < 2; ++layer) {
        std::vector<int32_t>& phi = layer == 0 ? s.phi_plus : s.phi_minus;
        for (const OParticle& p : s.parts[layer]) {
            if (p.escaped != 1u) continue;
            const uint32_t bx = f2u(p.x), by = f2u(p.y);
            for (uint32_t i = 0; i < 2; ++i)
                for (uint32_t j = 0; j < 2; ++j) {
                    const uint32_t cx = bx + i, cy = by + j;
                    if (nx <= cx || ny <= cy) continue;
                    const float dx = p.x - (float)cx, dy = p.y - (float)cy;
                    const float phi_p = p.sign * (p.radius - wlength(dx, dy));
                    int32_t& dst = phi[(size_t)cx + nx * cy];
                    const int32_t q = pls_fixed(phi_p);
                    dst = p.sign > 0.0f ? std::max(dst, q) : std::min(dst, q);
                }
        }
    }
    for (int y = 0; y < s.cy(); ++y)
        for (int x = 0; x < s.cx(); ++x) {
            float pp = pls_float(s.phi_plus[(size_t)y * nx + x]);
            float pm = pls_float(s.phi_minus[(size_t)y * nx + x]);
            ls.st(x, y, std::fabs(pp) <= std::fabs(pm) ? pp : pm);
        }
    if (!second) return;
    for (auto& layer : s.parts)
        for (auto& p : layer) p.radius = particle_radius(ls.ld(f2i(p.x), f2i(p.y)));
}

// reseed_particles.wgsl:97-148: the heap with WGSL's bounds-checked local
// array (an index past the end reads and writes element 15) and its
// zero-initialised contents.
struct HeapNode {
    uint32_t index;
    float value;
};
struct CellHeap {
    HeapNode h[PLS_PER_CELL] = {};
    HeapNode& at(uint32_t i) { return h[std::min(i, PLS_PER_CELL - 1)]; }
    void correct(uint32_t capacity, uint32_t start) {  // correct_heap
        uint32_t i = start;
        for (;;) {
            uint32_t l = 2 * i + 1, r = 2 * i + 2, largest = i;
            if (l < capacity && at(l).value > at(largest).value) largest = l;
            if (r < capacity && at(r).value > at(largest).value) largest = r;
            if (largest == i) return;
            std::swap(at(largest), at(i));
            i = largest;
        }
    }
    void sift_up(uint32_t capacity) {
        uint32_t i = capacity - 1;
        for (;;) {
            uint32_t p = (i - 1) / 2;
            if (at(p).value > at(i).value) return;
            std::swap(at(p), at(i));
            i = p;
            if (i == 0) return;
        }
    }
};

// reseed.rs:130-296 for one layer: count_particles_in_cell, prefix sum,
// sort_particles, reseed_particles, prefix sum of the alive mask,
// delete_particles, update_particles_count, add_particles.
void pls_reseed_layer(eflo_sim& s, int layer) {
    const float sign = layer == 0 ? 1.0f : -1.0f;
    const uint32_t nx = (uint32_t)s.nx, L = (uint32_t)s.nx * (uint32_t)s.ny;
    std::vector<OParticle>& parts = s.parts[layer];
    const uint32_t count = (uint32_t)parts.size();
    auto cell_of = [&](const OParticle& p) {
        uint32_t c = f2u(p.x) + nx * f2u(p.y);
        return std::min(c, L - 1);  // bounds-checked storage index
    };
    std::vector<uint32_t> num(L, 0), offsets(L, 0), cursor(L, 0);
    for (const OParticle& p : parts) ++num[cell_of(p)];
    for (uint32_t c = 1; c < L; ++c) offsets[c] = offsets[c - 1] + num[c - 1];
    std::vector<OParticle> sorted(count);
    for (const OParticle& p : parts) {
        uint32_t c = cell_of(p);
        sorted[offsets[c] + cursor[c]++] = p;
    }
    std::vector<uint32_t> alive(count, 0), to_add(L, 0);
    for (uint32_t cy = 0; cy < (uint32_t)s.cy(); ++cy)
        for (uint32_t cx = 0; cx < (uint32_t)s.cx(); ++cx) {
            const uint32_t c = cx + nx * cy;
            const uint32_t n = num[c], base = offsets[c];
            const bool near = std::fabs(interp_center(s.ls0, (float)cx, (float)cy)) < PLS_BAND;
            CellHeap heap;
            uint32_t capacity = PLS_PER_CELL, idx = 0;
            auto mark_dead = [&](uint32_t slot) {
                // slot 0 of another cell's bucket (a zero node): the racy
                // write is ordered before that cell's own writes
                if (slot >= base && slot < base + n) alive[slot] = 0;
            };
            for (uint32_t i = 0; i < n; ++i) {
                const uint32_t slot = base + i;
                const OParticle& p = sorted[slot];
                if (!near) {
                    alive[slot] = 0;
                    continue;
                }
                if (is_escaped(p, s.ls0)) {
                    if (capacity != 0) {
                        alive[slot] = 1;
                        capacity -= 1;
                        if (idx > capacity) {
                            mark_dead(heap.at(0).index);
                            heap.at(0) = heap.at(idx - 1);
                            idx -= 1;
                            heap.correct(capacity, 0);
                        }
                    } else {
                        alive[slot] = 0;
                    }
                    continue;
                }
                const float prio = p.sign * interp_center(s.ls0, p.x, p.y) - p.radius;
                if (idx < capacity) {
                    alive[slot] = 1;
                    heap.at(idx) = HeapNode{slot, prio};
                    idx += 1;
                    heap.sift_up(idx);
                } else if (prio < heap.at(0).value) {
                    alive[slot] = 1;
                    mark_dead(heap.at(0).index);
                    heap.at(0) = HeapNode{slot, prio};
                    heap.correct(capacity, 0);
                } else {
                    alive[slot] = 0;
                }
            }
            to_add[c] = near ? capacity - idx : 0u;
        }
    std::vector<uint32_t> scan(count, 0);
    for (uint32_t i = 1; i < count; ++i) scan[i] = scan[i - 1] + alive[i - 1];
    const uint32_t kept = count ? scan[count - 1] + alive[count - 1] : 0u;
    parts.assign(kept, OParticle{});
    for (uint32_t i = 0; i < count; ++i)
        if (alive[i]) parts[scan[i]] = sorted[i];
    // add_particles.wgsl:12-46
    const float bmin = sign > 0.0f ? 0.1f : -PLS_BAND;
    const float bmax = sign > 0.0f ? PLS_BAND : -0.1f;
    for (uint32_t cy = 0; cy < (uint32_t)s.cy(); ++cy)
        for (uint32_t cx = 0; cx < (uint32_t)s.cx(); ++cx) {
            const uint32_t c = cx + nx * cy;
            const F2 xb{(float)cx, (float)cy};
            for (uint32_t i = 0; i < to_add[c]; ++i) {
                const uint32_t seed = c + i;
                F2 h = hash22(F2{xb.x + (float)seed, xb.y + (float)seed});
                F2 x{xb.x + h.x, xb.y + h.y};
                float goal = hash11((float)seed) * (bmax - bmin) + bmin;
                OParticle p;
                if (spawn_and_attract(s, x, goal, bmin, bmax, sign, &p)) pls_append(s, layer, p);
            }
        }
}

void pls_reseed(eflo_sim& s) {
    pls_reseed_layer(s, 0);
    pls_reseed_layer(s, 1);
}

// render_node.rs:219-277
void run_init(eflo_sim& s) {
    k_init_center(s);
    k_init_edge(s);
    if (s.pls_on) pls_initialize(s);  // render_node.rs:250-258
    k_fluid_source(s, s.src_once);
    k_reinit(s);
}

efl_status run_stage(eflo_sim& s, int stage, efl_step_stats* st) {
    switch (stage) {
        case EFL_STAGE_INIT: run_init(s); s.status = 1; return EFL_OK;
        case EFL_STAGE_UPDATE_SOLID: k_update_solid(s); return EFL_OK;
        case EFL_STAGE_AREA_FRACTION: k_area_fraction(s); return EFL_OK;
        case EFL_STAGE_ADVECT_VELOCITY: k_advect(s); return EFL_OK;
        case EFL_STAGE_APPLY_FORCES: k_apply_forces(s); return EFL_OK;
        case EFL_STAGE_DIVERGENCE: k_divergence(s); return EFL_OK;
        case EFL_STAGE_PROJECTION: return k_projection(s, st);
        case EFL_STAGE_SOLVE_VELOCITY: k_solve_velocity(s); return EFL_OK;
        case EFL_STAGE_EXTRAPOLATE: k_extrapolate(s); return EFL_OK;
        case EFL_STAGE_ADVECT_LEVELSET: k_advect_levelset(s); return EFL_OK;
        case EFL_STAGE_FLUID_SOURCE:  // + render_node.rs:389-419
            k_fluid_source(s, s.src_cont);
            if (s.pls_on) {
                pls_advect(s);
                pls_correct(s, s.ls1, false);
            }
            return EFL_OK;
        case EFL_STAGE_REINITIALIZE:  // + render_node.rs:421-441
            k_reinit(s);
            if (s.pls_on) {
                pls_correct(s, s.ls0, true);
                pls_reseed(s);
            }
            return EFL_OK;
        case EFL_STAGE_LEVELSET_GRADIENT: k_gradient(s); return EFL_OK;
        case EFL_STAGE_SOLID_FORCES: k_solid_forces(s); return EFL_OK;
        default: return fail(&s, EFL_ERR_INVALID_ARGUMENT, "unknown stage");
    }
}

int mg_num_levels(const efl_config& c) {
    if (c.projection.mg_levels > 0) return (int)c.projection.mg_levels;
    int n = (int)std::log2((float)std::min(c.nx, c.ny)) - 2;  // multi_grid.rs:95-97
    return std::max(1, n);
}

template <class T>
void alloc_levels(std::vector<LevelT<T>>& mg, int L, int w, int h) {
    mg.clear();
    mg.resize(L);
    for (int i = 0; i < L; ++i) {
        LevelT<T>& l = mg[i];
        l.nx = w; l.ny = h;
        l.x.init(w, h); l.b.init(w, h); l.ls.init(w, h); l.r.init(w, h); l.af.init(w, h);
        w /= 2; h /= 2;
    }
}
void alloc_mg(eflo_sim& s) {
    int L = mg_num_levels(s.cfg);
    alloc_levels(s.mg, L, s.nx, s.ny);
    alloc_levels(s.mg64, L, s.nx, s.ny);
}

efl_status validate_cfg(const efl_config* c, std::string* why) {
    if (!c) { *why = "null config"; return EFL_ERR_INVALID_ARGUMENT; }
    if (!(c->length_unit > 0.0f)) { *why = "length_unit must be positive value."; return EFL_ERR_INVALID_ARGUMENT; }
    if (c->nx < 16 || c->ny < 16 || c->nx % 8 || c->ny % 8) {
        *why = "grid size must be a multiple of 8 and at least 16";
        return EFL_ERR_INVALID_ARGUMENT;
    }
    if (c->nx > 32768 || c->ny > 32768) { *why = "grid size too large"; return EFL_ERR_INVALID_ARGUMENT; }
    const efl_projection& p = c->projection;
    if (p.method < 0 || p.method > 3) { *why = "unknown projection method"; return EFL_ERR_INVALID_ARGUMENT; }
    if (p.method == EFL_PROJECTION_MGPCG && !(p.tolerance > 0.0f)) { *why = "MGPCG needs a tolerance > 0"; return EFL_ERR_INVALID_ARGUMENT; }
    if (c->reinit.method < 0 || c->reinit.method > 1) { *why = "unknown reinitialize method"; return EFL_ERR_INVALID_ARGUMENT; }
    return EFL_OK;
}

std::string g_err;

}  // namespace

extern "C" {

efl_status eflo_create(const efl_config* cfg, eflo_sim** out) {
    if (!out) { g_err = "null output pointer"; return EFL_ERR_INVALID_ARGUMENT; }
    *out = nullptr;
    std::string why;
    efl_status st = validate_cfg(cfg, &why);
    if (st != EFL_OK) { g_err = why; return st; }
    eflo_sim* s = new eflo_sim();
    s->cfg = *cfg;
    s->nx = (int)cfg->nx;
    s->ny = (int)cfg->ny;
    int nx = s->nx, ny = s->ny;
    s->U.dx = 1.0f / cfg->length_unit;  // euler_fluid.rs:89
    s->U.dt = 0.0f;
    s->U.rho = cfg->rho;
    s->U.g[0] = cfg->gravity[0];
    s->U.g[1] = cfg->gravity[1];
    std::memcpy(s->U.m, cfg->transform, sizeof(s->U.m));
    s->U.size[0] = (float)nx;
    s->U.size[1] = (float)ny;
    s->u0.init(nx + 1, ny); s->u1.init(nx + 1, ny); s->us.init(nx + 1, ny);
    s->v0.init(nx, ny + 1); s->v1.init(nx, ny + 1); s->vs.init(nx, ny + 1);
    s->u_valid_in.init(nx + 1, ny); s->u_valid_out.init(nx + 1, ny);
    s->v_valid_in.init(nx, ny + 1); s->v_valid_out.init(nx, ny + 1);
    s->solid_id.init(nx, ny); s->ls_solid.init(nx, ny); s->div.init(nx, ny);
    s->p0.init(nx, ny); s->p1.init(nx, ny); s->ls0.init(nx, ny); s->ls1.init(nx, ny);
    s->af.init(nx, ny); s->grad.init(nx, ny); s->seeds[0].init(nx, ny); s->seeds[1].init(nx, ny);
    s->labels0.init(nx, ny); s->labels.init(nx, ny); s->labelsT.init(nx, ny); s->phiT.init(nx, ny);
    alloc_mg(*s);
    std::memset(s->bins, 0, sizeof(s->bins));
    std::memset(s->out_forces, 0, sizeof(s->out_forces));
    *out = s;
    return EFL_OK;
}

efl_status eflo_destroy(eflo_sim* s) {
    delete s;
    return EFL_OK;
}

const char* eflo_last_error(const eflo_sim* s) { return s ? s->err.c_str() : g_err.c_str(); }

efl_status eflo_reset(eflo_sim* s) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    s->status = 0;
    return EFL_OK;
}

efl_status eflo_set_projection(eflo_sim* s, const efl_projection* p) {
    if (!s || !p) return EFL_ERR_INVALID_ARGUMENT;
    if (p->method < 0 || p->method > 3) return fail(s, EFL_ERR_INVALID_ARGUMENT, "unknown projection method");
    if (p->method == EFL_PROJECTION_MGPCG && !(p->tolerance > 0.0f))
        return fail(s, EFL_ERR_INVALID_ARGUMENT, "MGPCG needs a tolerance > 0");
    s->cfg.projection = *p;
    alloc_mg(*s);
    return EFL_OK;
}
efl_status eflo_set_reinit(eflo_sim* s, const efl_reinit* r) {
    if (!s || !r) return EFL_ERR_INVALID_ARGUMENT;
    if (r->method < 0 || r->method > 1) return fail(s, EFL_ERR_INVALID_ARGUMENT, "unknown reinitialize method");
    s->cfg.reinit = *r;
    return EFL_OK;
}
efl_status eflo_set_transform(eflo_sim* s, const float t[16]) {
    if (!s || !t) return EFL_ERR_INVALID_ARGUMENT;
    std::memcpy(s->U.m, t, sizeof(s->U.m));
    std::memcpy(s->cfg.transform, t, sizeof(s->U.m));
    return EFL_OK;
}
efl_status eflo_set_obstacles(eflo_sim* s, const efl_solid_obstacle* o, uint32_t n) {
    if (!s || (n && !o)) return EFL_ERR_INVALID_ARGUMENT;
    if (n > EFL_MAX_SOLIDS) return fail(s, EFL_ERR_TOO_MANY, "too many obstacles (max 256)");
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t sh = o[i].shape;
        if (sh != 0 && sh != 1 && sh != 2 && sh != 4) return fail(s, EFL_ERR_UNSUPPORTED_SHAPE, "Unsupported shape type for solid");
    }
    s->obstacles.assign(o, o + n);
    return EFL_OK;
}
efl_status eflo_set_local_forces(eflo_sim* s, const efl_force* f, uint32_t n) {
    if (!s || (n && !f)) return EFL_ERR_INVALID_ARGUMENT;
    s->forces.assign(f, f + n);
    return EFL_OK;
}
efl_status eflo_set_sources(eflo_sim* s, const efl_source* src, uint32_t n, int32_t oneshot) {
    if (!s || (n && !src)) return EFL_ERR_INVALID_ARGUMENT;
    if (n > EFL_MAX_FLUID_SOURCE)
        return fail(s, EFL_ERR_TOO_MANY, "The maximum number of fluid source per fluid component is 16.");
    (oneshot ? s->src_once : s->src_cont).assign(src, src + n);
    return EFL_OK;
}

efl_status eflo_step(eflo_sim* s, float dt, efl_step_stats* st) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->residual = -1.0;
        st->residual_initial = -1.0;
        st->converged = 1;
    }
    if (s->status == 0) {  // FluidStatus::Uninitialized -> init sequence only
        run_init(*s);
        s->status = 1;
        if (st) st->initialized_only = 1;
        return EFL_OK;
    }
    s->U.dt = dt;
    efl_status ret = EFL_OK;
    for (int stage = EFL_STAGE_UPDATE_SOLID; stage <= EFL_STAGE_SOLID_FORCES; ++stage) {
        efl_status r = run_stage(*s, stage, st);
        if (r == EFL_NOT_CONVERGED) ret = r;
        else if (r != EFL_OK) return r;
    }
    s->forces.clear();  // apply_forces.rs:166
    return ret;
}

efl_status eflo_run_stage(eflo_sim* s, int32_t stage, float dt, efl_step_stats* st) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->residual = -1.0;
        st->residual_initial = -1.0;
        st->converged = 1;
    }
    s->U.dt = dt;
    return run_stage(*s, stage, st);
}

efl_status eflo_read_solid_forces(eflo_sim* s, efl_solid_force out[EFL_MAX_SOLIDS]) {
    if (!s || !out) return EFL_ERR_INVALID_ARGUMENT;
    std::memcpy(out, s->out_forces, sizeof(s->out_forces));
    return EFL_OK;
}
efl_status eflo_read_force_bins(eflo_sim* s, int32_t out[3 * EFL_MAX_SOLIDS]) {
    if (!s || !out) return EFL_ERR_INVALID_ARGUMENT;
    std::memcpy(out, s->bins, sizeof(s->bins));
    return EFL_OK;
}

efl_status eflo_field_shape(const eflo_sim* s, int32_t field, uint32_t* w, uint32_t* h, uint32_t* ch,
                            uint32_t* eb) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    uint32_t nx = s->nx, ny = s->ny, W = nx, H = ny, C = 1;
    switch (field) {
        case EFL_FIELD_U: case EFL_FIELD_U1: case EFL_FIELD_U_SOLID: case EFL_FIELD_U_VALID:
        case EFL_FIELD_AREA_FRACTION_U: W = nx + 1; break;
        case EFL_FIELD_V: case EFL_FIELD_V1: case EFL_FIELD_V_SOLID: case EFL_FIELD_V_VALID:
        case EFL_FIELD_AREA_FRACTION_V: H = ny + 1; break;
        case EFL_FIELD_AREA_FRACTION: C = 4; break;
        case EFL_FIELD_GRAD_LEVELSET: case EFL_FIELD_JFA_SEEDS: C = 2; break;
        case EFL_FIELD_LEVELSET_AIR: case EFL_FIELD_LEVELSET_AIR1: case EFL_FIELD_LEVELSET_SOLID:
        case EFL_FIELD_SOLID_ID: case EFL_FIELD_DIVERGENCE: case EFL_FIELD_PRESSURE: case EFL_FIELD_FIM_LABELS:
            break;
        default: return EFL_ERR_INVALID_ARGUMENT;
    }
    if (w) *w = W;
    if (h) *h = H;
    if (ch) *ch = C;
    if (eb) *eb = 4;
    return EFL_OK;
}

}  // extern "C"

namespace {
template <class T>
efl_status copy_out(const Tex<T>& t, void* dst, size_t bytes) {
    if (bytes != t.a.size() * sizeof(T)) return EFL_ERR_INVALID_ARGUMENT;
    std::memcpy(dst, t.a.data(), bytes);
    return EFL_OK;
}
template <class T>
efl_status copy_in(Tex<T>& t, const void* src, size_t bytes) {
    if (bytes != t.a.size() * sizeof(T)) return EFL_ERR_INVALID_ARGUMENT;
    std::memcpy(t.a.data(), src, bytes);
    return EFL_OK;
}
// x-face / y-face fraction views of the RGBA texture
void af_faces(const eflo_sim& s, std::vector<float>& fu, std::vector<float>& fv) {
    int nx = s.nx, ny = s.ny;
    fu.assign((size_t)(nx + 1) * ny, 0.0f);
    fv.assign((size_t)nx * (ny + 1), 0.0f);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            F4 f = s.af.a[(size_t)y * nx + x];
            fu[(size_t)y * (nx + 1) + x] = f.x;
            if (x == nx - 1) fu[(size_t)y * (nx + 1) + x + 1] = f.y;
            fv[(size_t)y * nx + x] = f.z;
            if (y == ny - 1) fv[(size_t)(y + 1) * nx + x] = f.w;
        }
}
}  // namespace

extern "C" {

efl_status eflo_get_field(eflo_sim* s, int32_t field, void* dst, size_t bytes) {
    if (!s || !dst) return EFL_ERR_INVALID_ARGUMENT;
    switch (field) {
        case EFL_FIELD_U: return copy_out(s->u0, dst, bytes);
        case EFL_FIELD_V: return copy_out(s->v0, dst, bytes);
        case EFL_FIELD_U1: return copy_out(s->u1, dst, bytes);
        case EFL_FIELD_V1: return copy_out(s->v1, dst, bytes);
        case EFL_FIELD_U_SOLID: return copy_out(s->us, dst, bytes);
        case EFL_FIELD_V_SOLID: return copy_out(s->vs, dst, bytes);
        case EFL_FIELD_LEVELSET_AIR: return copy_out(s->ls0, dst, bytes);
        case EFL_FIELD_LEVELSET_AIR1: return copy_out(s->ls1, dst, bytes);
        case EFL_FIELD_LEVELSET_SOLID: return copy_out(s->ls_solid, dst, bytes);
        case EFL_FIELD_SOLID_ID: return copy_out(s->solid_id, dst, bytes);
        case EFL_FIELD_AREA_FRACTION: return copy_out(s->af, dst, bytes);
        case EFL_FIELD_DIVERGENCE: return copy_out(s->div, dst, bytes);
        case EFL_FIELD_PRESSURE: return copy_out(s->p0, dst, bytes);
        case EFL_FIELD_GRAD_LEVELSET: return copy_out(s->grad, dst, bytes);
        case EFL_FIELD_JFA_SEEDS: return copy_out(s->seeds[s->seeds_final], dst, bytes);
        case EFL_FIELD_FIM_LABELS: return copy_out(s->labels, dst, bytes);
        case EFL_FIELD_U_VALID: return copy_out(s->u_valid_in, dst, bytes);
        case EFL_FIELD_V_VALID: return copy_out(s->v_valid_in, dst, bytes);
        case EFL_FIELD_AREA_FRACTION_U:
        case EFL_FIELD_AREA_FRACTION_V: {
            std::vector<float> fu, fv;
            af_faces(*s, fu, fv);
            const std::vector<float>& v = field == EFL_FIELD_AREA_FRACTION_U ? fu : fv;
            if (bytes != v.size() * 4) return EFL_ERR_INVALID_ARGUMENT;
            std::memcpy(dst, v.data(), bytes);
            return EFL_OK;
        }
        default: return EFL_ERR_INVALID_ARGUMENT;
    }
}

efl_status eflo_set_field(eflo_sim* s, int32_t field, const void* src, size_t bytes) {
    if (!s || !src) return EFL_ERR_INVALID_ARGUMENT;
    switch (field) {
        case EFL_FIELD_U: return copy_in(s->u0, src, bytes);
        case EFL_FIELD_V: return copy_in(s->v0, src, bytes);
        case EFL_FIELD_U1: return copy_in(s->u1, src, bytes);
        case EFL_FIELD_V1: return copy_in(s->v1, src, bytes);
        case EFL_FIELD_U_SOLID: return copy_in(s->us, src, bytes);
        case EFL_FIELD_V_SOLID: return copy_in(s->vs, src, bytes);
        case EFL_FIELD_LEVELSET_AIR: return copy_in(s->ls0, src, bytes);
        case EFL_FIELD_LEVELSET_AIR1: return copy_in(s->ls1, src, bytes);
        case EFL_FIELD_LEVELSET_SOLID: return copy_in(s->ls_solid, src, bytes);
        case EFL_FIELD_SOLID_ID: return copy_in(s->solid_id, src, bytes);
        case EFL_FIELD_AREA_FRACTION: return copy_in(s->af, src, bytes);
        case EFL_FIELD_DIVERGENCE: return copy_in(s->div, src, bytes);
        case EFL_FIELD_PRESSURE: return copy_in(s->p0, src, bytes);
        case EFL_FIELD_GRAD_LEVELSET: return copy_in(s->grad, src, bytes);
        case EFL_FIELD_JFA_SEEDS: return copy_in(s->seeds[s->seeds_final], src, bytes);
        case EFL_FIELD_FIM_LABELS: return copy_in(s->labels, src, bytes);
        case EFL_FIELD_U_VALID: return copy_in(s->u_valid_in, src, bytes);
        case EFL_FIELD_V_VALID: return copy_in(s->v_valid_in, src, bytes);
        default: return EFL_ERR_INVALID_ARGUMENT;
    }
}

efl_status eflo_residual(eflo_sim* s, double* rel, double* nr, double* nb) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    double R, B;
    residual_norms_f32(*s, &R, &B);
    if (nr) *nr = std::sqrt(R);
    if (nb) *nb = std::sqrt(B);
    if (rel) *rel = B > 0.0 ? std::sqrt(R) / std::sqrt(B) : (R > 0.0 ? std::numeric_limits<double>::infinity() : 0.0);
    return EFL_OK;
}

// diagnostics/{min,max}_velocity.wgsl: partial_reduction over 16 x 16
// workgroups of the cells x < nx, y < ny, then `reduction` with 512 lanes,
// each adding its partials in order from 0.0 before the min / max.
efl_status eflo_velocity_magnitude(eflo_sim* s, float* min_mag, float* max_mag) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    const int gx = s->nx / 16, gy = s->ny / 16, n = gx * gy;
    std::vector<float> pmin(n), pmax(n);
    for (int wy = 0; wy < gy; ++wy)
        for (int wx = 0; wx < gx; ++wx) {
            float mn = 0.0f, mx = 0.0f;
            bool first = true;
            for (int y = 16 * wy; y < 16 * wy + 16; ++y)
                for (int x = 16 * wx; x < 16 * wx + 16; ++x) {
                    const float u0 = 0.5f * (s->u0.ld(x, y) + s->u0.ld(x + 1, y));
                    const float v0 = 0.5f * (s->v0.ld(x, y) + s->v0.ld(x, y + 1));
                    const float mag = std::sqrt(u0 * u0 + v0 * v0);
                    const float lo = s->ls0.ld(x, y) < 0.0f ? mag : 1e30f;
                    mn = first ? lo : std::fmin(mn, lo);
                    mx = first ? mag : std::fmax(mx, mag);
                    first = false;
                }
            pmin[wy * gx + wx] = mn;
            pmax[wy * gx + wx] = mx;
        }
    float rmin = 0.0f, rmax = 0.0f;
    for (int lane = 0; lane < 512; ++lane) {
        float a = 0.0f, b = 0.0f;
        for (int i = lane; i < n; i += 512) {
            a += pmin[i];
            b += pmax[i];
        }
        rmin = lane == 0 ? a : std::fmin(rmin, a);
        rmax = lane == 0 ? b : std::fmax(rmax, b);
    }
    if (min_mag) *min_mag = rmin;
    if (max_mag) *max_mag = rmax;
    return EFL_OK;
}

// divergence.wgsl:16-42 applied to the projected velocity (u0, v0) at the
// cells the residual counts (phi < 0, not fully solid): sqrt of the FP64 sum
// of squares in row order and the largest magnitude.
efl_status eflo_divergence_norms(eflo_sim* s, double* l2, double* linf) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    const float dx = s->U.dx;
    double a2 = 0.0, m = 0.0;
    for (int y = 0; y < s->ny; ++y)
        for (int x = 0; x < s->nx; ++x) {
            if (!(s->ls0.ld(x, y) < 0.0f)) continue;
            const F4 f = s->af.ld(x, y);
            if (f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f) continue;
            const float du_f = f.y * s->u0.ld(x + 1, y) - f.x * s->u0.ld(x, y);
            const float dv_f = f.w * s->v0.ld(x, y + 1) - f.z * s->v0.ld(x, y);
            const float du_s = (1.0f - f.y) * s->us.ld(x + 1, y) - (1.0f - f.x) * s->us.ld(x, y);
            const float dv_s = (1.0f - f.w) * s->vs.ld(x, y + 1) - (1.0f - f.z) * s->vs.ld(x, y);
            const double d = (double)(-(du_f + dv_f + du_s + dv_s) / dx);
            a2 += d * d;
            m = std::fmax(m, std::fabs(d));
        }
    if (l2) *l2 = std::sqrt(a2);
    if (linf) *linf = m;
    return EFL_OK;
}

efl_status eflo_fluid_volume(eflo_sim* s, uint64_t* cells) {
    if (!s || !cells) return EFL_ERR_INVALID_ARGUMENT;
    uint64_t c = 0;
    for (float v : s->ls0.a) c += v < 0.0f;
    *cells = c;
    return EFL_OK;
}

void eflo_set_threads(int32_t n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}
int32_t eflo_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}
float eflo_exp(float x) { return exp_for_test(x); }

void eflo_set_fim_serial(eflo_sim* s, int32_t on) {
    if (s) s->fim_serial = on != 0;
}

efl_status eflo_set_particle_levelset(eflo_sim* s, int32_t enable) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    s->pls_on = enable != 0;
    return EFL_OK;
}

efl_status eflo_particle_counts(eflo_sim* s, uint32_t counts[2], uint32_t* dropped) {
    if (!s || !counts) return EFL_ERR_INVALID_ARGUMENT;
    counts[0] = (uint32_t)s->parts[0].size();
    counts[1] = (uint32_t)s->parts[1].size();
    if (dropped) *dropped = s->pls_dropped;
    return EFL_OK;
}

efl_status eflo_read_particles(eflo_sim* s, int32_t layer, efl_particle* dst, uint32_t capacity, uint32_t* n) {
    if (!s || !n || (capacity && !dst)) return EFL_ERR_INVALID_ARGUMENT;
    if (layer != EFL_PLS_POSITIVE && layer != EFL_PLS_NEGATIVE) return fail(s, EFL_ERR_INVALID_ARGUMENT, "layer");
    const std::vector<OParticle>& v = s->parts[layer];
    *n = (uint32_t)v.size();
    const uint32_t m = std::min(*n, capacity);
    for (uint32_t i = 0; i < m; ++i) {
        dst[i].position[0] = v[i].x;
        dst[i].position[1] = v[i].y;
        dst[i].radius = v[i].radius;
        dst[i].sign = v[i].sign;
        dst[i].escaped = v[i].escaped;
        dst[i]._pad = 0;
    }
    return EFL_OK;
}

efl_status eflo_write_particles(eflo_sim* s, int32_t layer, const efl_particle* src, uint32_t n) {
    if (!s || (n && !src)) return EFL_ERR_INVALID_ARGUMENT;
    if (layer != EFL_PLS_POSITIVE && layer != EFL_PLS_NEGATIVE) return fail(s, EFL_ERR_INVALID_ARGUMENT, "layer");
    if ((uint64_t)n > (uint64_t)s->nx * s->ny * PLS_PER_CELL) return fail(s, EFL_ERR_TOO_MANY, "capacity");
    const float sign = layer == EFL_PLS_POSITIVE ? 1.0f : -1.0f;
    std::vector<OParticle> v(n);
    for (uint32_t i = 0; i < n; ++i) {
        if (src[i].sign != sign) return fail(s, EFL_ERR_INVALID_ARGUMENT, "sign does not match the layer");
        v[i] = OParticle{src[i].position[0], src[i].position[1], src[i].radius, sign, src[i].escaped ? 1u : 0u};
    }
    s->parts[layer] = std::move(v);
    return EFL_OK;
}

efl_status eflo_pls_run_phase(eflo_sim* s, int32_t phase, float dt) {
    if (!s) return EFL_ERR_INVALID_ARGUMENT;
    switch (phase) {
        case EFL_PLS_INITIALIZE: pls_initialize(*s); return EFL_OK;
        case EFL_PLS_ADVECT: {
            const float keep = s->U.dt;
            s->U.dt = dt;
            pls_advect(*s);
            s->U.dt = keep;
            return EFL_OK;
        }
        case EFL_PLS_CORRECT: pls_correct(*s, s->ls1, false); return EFL_OK;
        case EFL_PLS_CORRECT_SECOND: pls_correct(*s, s->ls0, true); return EFL_OK;
        case EFL_PLS_RESEED: pls_reseed(*s); return EFL_OK;
        default: return fail(s, EFL_ERR_INVALID_ARGUMENT, "unknown phase");
    }
}

}  // extern "C"
