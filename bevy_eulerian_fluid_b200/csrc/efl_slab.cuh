// efl_slab.cuh — one row slab of the tolerance-driven pressure solve, for a
// domain split into horizontal slabs across devices (one process per GPU).
//
// The slab owns rows [row0, row0 + rows) of the nx x ny grid and keeps one
// halo row above and below for the fields its stencil reads across the cut:
// the FP64 iterate x, the f32 correction d and the level set (for the
// ghost-fluid coefficient of the rows next to the cut).  The arithmetic is
// that of the single-device mixed-precision solve (the red-black update of
// gauss_seidel.wgsl:44-88 on the correction, the residual of
// residual.wgsl:33-54 in FP64): every cell reads the same neighbour values it
// would read unsplit, so with the halos exchanged before each half-sweep and
// before each residual the slabs together reproduce the unsplit solve bit for
// bit.  The host driver (bevy_eulerian_fluid_b200/slab.py) does the exchange
// and combines the per-row residual partials of all slabs in row order.
#pragma once

#include <cuda_runtime.h>

namespace efl {

constexpr int kSlabRowThreads = 256;

struct SlabPlanes {
    int nx = 0, ny = 0, row0 = 0, rows = 0;
    // (rows + 2) x nx, row 0 = global row row0 - 1 (zero where the domain ends)
    double* x = nullptr;
    float* d = nullptr;
    float* ls = nullptr;
    // rows x nx
    float4* af = nullptr;  // face fractions (i-1/2, i+1/2, j-1/2, j+1/2)
    double* b = nullptr;
    float* rc = nullptr;
    float4* w = nullptr;
    float* inv = nullptr;
    double* den = nullptr;
    unsigned char* mode = nullptr;  // 0 skip, 1 zero, 2 update; +4 counted by the residual
    double2* rowpart = nullptr;     // per own row: (sum r^2, sum b^2) over counted cells
};

// Coefficients of the own rows: mode, the neighbour weights w (the face
// fraction of an in-domain fluid neighbour, else 0), den (fluid faces plus
// the ghost-fluid part f * (1 - phi_n / phi) of air faces, FP64) and
// inv = f32(1 / den), as the single-device solve builds them.
__global__ void k_slab_coeffs(SlabPlanes S) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, ly = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= S.nx || ly >= S.rows) return;
    const int gy = S.row0 + ly;
    const size_t o = (size_t)ly * S.nx + gx;
    unsigned char mode = 1;
    float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
    double den = 0.0;
    float inv = 0.0f;
    const float lij = S.ls[(size_t)(ly + 1) * S.nx + gx];
    const float4 f = S.af[o];
    if (lij < 0.0f && !(f.x == 0.0f && f.y == 0.0f && f.z == 0.0f && f.w == 0.0f)) {
        mode |= 4;
        const float fv[4] = {f.x, f.y, f.z, f.w};
        const int ox[4] = {-1, 1, 0, 0}, oy[4] = {0, 0, -1, 1};
        float wv[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int jx = gx + ox[q], jy = gy + oy[q];
            if (jx >= 0 && jy >= 0 && jx < S.nx && jy < S.ny) {
                const float level = S.ls[(size_t)(jy - S.row0 + 1) * S.nx + jx];
                if (level < 0.0f) {
                    den += (double)fv[q];
                    wv[q] = fv[q];
                } else {
                    den += (double)fv[q] * (1.0 - (double)level / (double)lij);
                }
            }
        }
        w = make_float4(wv[0], wv[1], wv[2], wv[3]);
        if (!(fabs(den) < (double)1.0e-6f)) {
            mode = (unsigned char)((mode & 4) | 2);
            inv = (float)(1.0 / den);
        }
    }
    S.mode[o] = mode;
    S.w[o] = w;
    S.den[o] = den;
    S.inv[o] = inv;
}

// FP64 residual r = b - factor * (den * x - sum_k w_k x_k) of the own rows
// (neighbours in the sum in the order left, right, up, down), the f32
// right-hand side of the next correction rc = f32(cdiv * r) on updated
// cells, d = 0, and per row the sums of r^2 and b^2 over counted cells.  One
// CTA per row; the row sum is a fixed-order tree, so it is deterministic but
// not the sequential order of a CPU loop.
__global__ void __launch_bounds__(kSlabRowThreads) k_slab_residual(SlabPlanes S, double factor, double cdiv) {
    const int ly = blockIdx.x;
    const int nx = S.nx;
    const double* xr = S.x + (size_t)(ly + 1) * nx;
    double sr = 0.0, sb = 0.0;
    for (int gx = threadIdx.x; gx < nx; gx += kSlabRowThreads) {
        const size_t o = (size_t)ly * nx + gx;
        const unsigned char m = S.mode[o];
        double rv = 0.0;
        if (m & 4) {
            const float4 w = S.w[o];
            const double pl = gx > 0 ? xr[gx - 1] : 0.0, pr = gx + 1 < nx ? xr[gx + 1] : 0.0;
            double sum = (double)w.x * pl;
            sum = sum + (double)w.y * pr;
            sum = sum + (double)w.z * xr[gx - nx];
            sum = sum + (double)w.w * xr[gx + nx];
            const double bv = S.b[o];
            rv = bv - factor * (S.den[o] * xr[gx] - sum);
            sr += rv * rv;
            sb += bv * bv;
        }
        S.rc[o] = (m & 2) ? (float)(cdiv * rv) : 0.0f;
        S.d[(size_t)(ly + 1) * nx + gx] = 0.0f;
    }
    sr = warp_sum(sr);
    sb = warp_sum(sb);
    __shared__ double red[2][kSlabRowThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wid] = sr;
        red[1][wid] = sb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int k = 0; k < kSlabRowThreads / 32; ++k) {
            a += red[0][k];
            c += red[1][k];
        }
        S.rowpart[ly] = make_double2(a, c);
    }
}

// One half-sweep of the f32 correction on the cells of one colour
// ((x + y) % 2 == color, global coordinates): over-relaxed Gauss-Seidel,
// nume = rc + w_l d_l + w_r d_r + w_u d_u + w_d d_d in that order.
__global__ void k_slab_sweep(SlabPlanes S, int color, float weight) {
    const int hx = blockIdx.x * blockDim.x + threadIdx.x, ly = blockIdx.y * blockDim.y + threadIdx.y;
    if (ly >= S.rows) return;
    const int gy = S.row0 + ly;
    const int gx = 2 * hx + ((gy + color) & 1);
    if (gx >= S.nx) return;
    const int nx = S.nx;
    const size_t o = (size_t)ly * nx + gx;
    if (!(S.mode[o] & 2)) return;
    float* dr = S.d + (size_t)(ly + 1) * nx;
    const float4 w = S.w[o];
    const float dl = gx > 0 ? dr[gx - 1] : 0.0f, drr = gx + 1 < nx ? dr[gx + 1] : 0.0f;
    const float du = dr[gx - nx], dd = dr[gx + nx];
    float nume = S.rc[o];
    nume = nume + w.x * dl;
    nume = nume + w.y * drr;
    nume = nume + w.z * du;
    nume = nume + w.w * dd;
    dr[gx] = weight * (nume * S.inv[o]) + (1.0f - weight) * dr[gx];
}

// x += d on updated cells, x = 0 on the cells the reference zeroes.
__global__ void k_slab_apply(SlabPlanes S) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, ly = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= S.nx || ly >= S.rows) return;
    const size_t o = (size_t)ly * S.nx + gx, h = (size_t)(ly + 1) * S.nx + gx;
    S.x[h] = (S.mode[o] & 2) ? S.x[h] + (double)S.d[h] : 0.0;
}

// Widening loads of the caller's f32 pressure and divergence rows.
__global__ void k_slab_widen(SlabPlanes S, const float* p, const float* div) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, ly = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= S.nx || ly >= S.rows) return;
    const size_t o = (size_t)ly * S.nx + gx;
    S.x[(size_t)(ly + 1) * S.nx + gx] = (double)p[o];
    S.b[o] = (double)div[o];
}

}  // namespace efl
