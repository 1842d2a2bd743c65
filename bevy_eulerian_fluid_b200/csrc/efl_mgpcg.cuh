// efl_mgpcg.cuh — multigrid-preconditioned conjugate gradients on the FP64
// pressure system (EFL_PROJECTION_MGPCG, an extension: the reference never
// iterates a solver to a tolerance; its V-cycle, multi_grid.rs:390-475, is
// the preconditioner here).
//
// Unknowns are the update cells of the mixed solve (fluid, not fully solid,
// |denom| >= 1e-6); every other cell is held at p = 0.  A is the factored
// operator of residual.wgsl:33-54, factor * (denom * p - sum w_k p_k), with
// the per-cell coefficients of k_mix_coefficients.  The preconditioner is one
// f32 V-cycle of the reference's structure (the reference's f32 shader
// arithmetic) applied to f32(r) from a zero start, made symmetric by running
// post-smoothing black then red, and widened back to FP64.
//
// Reductions are in a FIXED ORDER so that they are bitwise reproducible and
// restated exactly by the CPU oracle: per row, every chunk of 32 columns is
// summed in x order from 0.0 (one thread per chunk row, the 32 x 32 tile
// staged through shared memory so that loads stay coalesced), the chunk sums
// are added in chunk order; the row sums are added in row order within groups
// of 32 rows, and the group sums in group order.  Cells outside the sum
// contribute +0.0, which leaves a running sum unchanged.
#pragma once

#include "efl_solver.cuh"

namespace efl {

struct CgScalars {
    double rz, alpha, beta;
    int breakdown, pad;
};
struct CgRead {  // what the host reads after each iteration
    double2 norm;   // (||r||^2, ||b||^2) over the counted cells
    int breakdown;  // p . ap <= 0 in this iteration
    int pad;
};
struct CgPlanes {
    Plane<double> r, p, ap;  // residual, direction, A * direction (the iterate is level 0's x)
    PF r32, z32;             // the preconditioner's level 0: b = f32(r), x = z
    double2* part = nullptr;    // chunk sums, ny x ceil(nx / 32)
    double2* rowsum = nullptr;  // one per row
    double2* totals = nullptr;  // [0] p . ap, [1] norms, [2] r . z
    CgScalars* sc = nullptr;
    CgRead* h_read = nullptr;   // pinned
};

// A v on update cells (0 elsewhere), v = 0 off the unknowns.
EFL_DEV double cg_apply(const Plane<double>& v, const MixPlanes& M, double factor, int x, int y, int nx, int ny) {
    const float4 wk = M.w.at(x, y);
    const double* row = v.p + (size_t)y * v.P + x;
    double sum = (double)wk.x * (x > 0 ? row[-1] : 0.0);
    sum = sum + (double)wk.y * (x + 1 < nx ? row[1] : 0.0);
    sum = sum + (double)wk.z * (y > 0 ? row[-(ptrdiff_t)v.P] : 0.0);
    sum = sum + (double)wk.w * (y + 1 < ny ? row[v.P] : 0.0);
    return factor * (M.den.at(x, y) * row[0] - sum);
}

// Per-cell terms of the reductions.
struct TermDotRZ {  // (r . z over update cells, 0)
    Plane<double> r;
    PF z;
    MixPlanes M;
    EFL_DEV double2 operator()(int x, int y) const {
        return make_double2((M.mode.at(x, y) & MODE_UPDATE) ? r.at(x, y) * (double)z.at(x, y) : 0.0, 0.0);
    }
};
struct TermMatvecDot {  // ap = A p (stored), (p . ap over update cells, 0)
    Plane<double> p, ap;
    MixPlanes M;
    double factor;
    int nx, ny;
    EFL_DEV double2 operator()(int x, int y) const {
        if (!(M.mode.at(x, y) & MODE_UPDATE)) {
            ap.at(x, y) = 0.0;
            return make_double2(0.0, 0.0);
        }
        const double v = cg_apply(p, M, factor, x, y, nx, ny);
        ap.at(x, y) = v;
        return make_double2(p.at(x, y) * v, 0.0);
    }
};
struct TermNorm {  // (r^2, b^2) over counted cells, r = b - A x (true residual)
    Plane<double> x, b;
    MixPlanes M;
    double factor;
    int nx, ny;
    EFL_DEV double2 operator()(int gx, int gy) const {
        if (!(M.mode.at(gx, gy) & MODE_COUNTED)) return make_double2(0.0, 0.0);
        const double bv = b.at(gx, gy);
        const double rv = bv - cg_apply(x, M, factor, gx, gy, nx, ny);
        return make_double2(rv * rv, bv * bv);
    }
};

constexpr int RS_CHUNK = 32, RS_THREADS = 256;

// part[y * nch + cx] = sum over the 32 columns of chunk cx, in x order, of term(x, y).
template <class Term>
__global__ void __launch_bounds__(RS_THREADS) k_chunk_sums(Term term, int nx, int ny, int nch, double2* part) {
    __shared__ double2 tile[RS_CHUNK][RS_CHUNK + 1];
    const int x0 = blockIdx.x * RS_CHUNK, y0 = blockIdx.y * RS_CHUNK;
    for (int i = threadIdx.x; i < RS_CHUNK * RS_CHUNK; i += RS_THREADS) {
        const int ly = i / RS_CHUNK, lx = i % RS_CHUNK;
        const int gx = x0 + lx, gy = y0 + ly;
        tile[ly][lx] = (gx < nx && gy < ny) ? term(gx, gy) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (threadIdx.x < RS_CHUNK && y0 + (int)threadIdx.x < ny) {
        double2 acc = make_double2(0.0, 0.0);
        for (int lx = 0; lx < RS_CHUNK; ++lx) {
            acc.x = acc.x + tile[threadIdx.x][lx].x;
            acc.y = acc.y + tile[threadIdx.x][lx].y;
        }
        part[(size_t)(y0 + threadIdx.x) * nch + blockIdx.x] = acc;
    }
}
// rowsum[y] = sum over chunks in order of part[y][.]
__global__ void k_chunk_rows(const double2* part, int nch, int ny, double2* rowsum) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= ny) return;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 8
    for (int c = 0; c < nch; ++c) {
        const double2 v = part[(size_t)y * nch + c];
        acc.x = acc.x + v.x;
        acc.y = acc.y + v.y;
    }
    rowsum[y] = acc;
}

// total = sum over groups of 32 rows, in group order, of each group's rows
// summed in row order (one block: thread g adds group g, thread 0 the groups).
__global__ void __launch_bounds__(1024) k_rows_total(const double2* rowsum, int ny, double2* total) {
    __shared__ double2 grp[1024];
    const int ngroups = (ny + 31) / 32;  // ny <= 32768
    for (int g = threadIdx.x; g < ngroups; g += blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int y = 32 * g; y < min(ny, 32 * g + 32); ++y) {
            const double2 v = rowsum[y];
            acc.x = acc.x + v.x;
            acc.y = acc.y + v.y;
        }
        grp[g] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 acc = make_double2(0.0, 0.0);
        for (int g = 0; g < ngroups; ++g) {
            acc.x = acc.x + grp[g].x;
            acc.y = acc.y + grp[g].y;
        }
        *total = acc;
    }
}

// x = 0 off the unknowns.
__global__ void k_cg_mask(Plane<double> x, MixPlanes M, int nx, int ny) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny) return;
    if (!(M.mode.at(gx, gy) & MODE_UPDATE)) x.at(gx, gy) = 0.0;
}
// r = b - A x on the unknowns, 0 elsewhere; r32 = f32(r).
__global__ void k_cg_residual(Plane<double> x, Plane<double> b, Plane<double> r, PF r32, MixPlanes M, double factor,
                              int nx, int ny) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny) return;
    const double v =
        (M.mode.at(gx, gy) & MODE_UPDATE) ? b.at(gx, gy) - cg_apply(x, M, factor, gx, gy, nx, ny) : 0.0;
    r.at(gx, gy) = v;
    r32.at(gx, gy) = (float)v;
}
enum { CG_RESET = 0, CG_RZ = 1, CG_ALPHA = 2, CG_BETA = 3 };
// The CG scalar recurrences (one thread): the same IEEE double operations as
// the host-side restatement.
__global__ void k_cg_scalar(int op, const double2* totals, CgScalars* sc) {
    if (op == CG_RESET) {
        sc->breakdown = 0;
    } else if (op == CG_RZ) {
        sc->rz = totals[2].x;
    } else if (op == CG_ALPHA) {
        const double pap = totals[0].x;
        if (pap > 0.0) {
            sc->alpha = sc->rz / pap;
        } else {
            sc->alpha = 0.0;
            sc->breakdown = 1;
        }
    } else {
        const double rz1 = totals[2].x;
        sc->beta = rz1 / sc->rz;
        sc->rz = rz1;
    }
}
// x += alpha p, r -= alpha ap on the unknowns; r32 = f32(r).  Nothing moves
// after a breakdown.
__global__ void k_cg_axpy(Plane<double> x, Plane<double> r, PF r32, Plane<double> p, Plane<double> ap, MixPlanes M,
                          const CgScalars* sc, int nx, int ny) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny || !(M.mode.at(gx, gy) & MODE_UPDATE) || sc->breakdown) return;
    const double alpha = sc->alpha;
    x.at(gx, gy) = x.at(gx, gy) + alpha * p.at(gx, gy);
    const double rv = r.at(gx, gy) - alpha * ap.at(gx, gy);
    r.at(gx, gy) = rv;
    r32.at(gx, gy) = (float)rv;
}
// p = z (first) or z + beta p on the unknowns, 0 elsewhere (z widened from f32).
__global__ void k_cg_direction(Plane<double> p, PF z, MixPlanes M, const CgScalars* sc, int first, int nx, int ny) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= nx || gy >= ny) return;
    double v = 0.0;
    if (M.mode.at(gx, gy) & MODE_UPDATE) {
        const double zv = (double)z.at(gx, gy);
        v = first ? zv : zv + sc->beta * p.at(gx, gy);
    }
    p.at(gx, gy) = v;
}

}  // namespace efl
