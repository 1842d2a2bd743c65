// efl_sim.cu — host orchestration and C ABI of libefl_b200.so.
//
// One efl_sim is one fluid entity of the reference plugin: its textures
// (setup_components.rs:38-328), its per-frame compute pass
// (EulerFluidNode::run, render_node.rs:193-476) and its force read-back
// (fluid_to_solid.rs:180-209).  All device work of a simulation is issued on
// the simulation's own CUDA stream; nothing here falls back to the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <random>

#include "../../include/efl.h"
#include "efl_kernels.cuh"
#include "efl_solver.cuh"
#include "efl_sweep_tma.cuh"
#include "efl_batch.cuh"
#include "efl_mgpcg.cuh"
#include "efl_unet.cuh"
#include "efl_pls.cuh"
#include "efl_slab.cuh"

using namespace efl;

namespace efl {
static std::atomic<uint64_t> g_launches{0};
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }
void add_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
size_t count_launch() {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return 0;
}
}  // namespace efl

namespace {

std::string g_last_error;

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }
inline dim3 grid2d(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }
const dim3 kBlock(32, 8);

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct efl_unet {
    UNet net;
    int rec_nx = 0, rec_ny = 0;  // size of the recorded training sample (0: none)
    bool rec_coarse = false;     // the recorded sample is on the coarse grid (targetc / maskc)
};

// Captured CUDA graphs of step segments, keyed by a signature of the
// host-side values their kernels were launched with.
struct GraphCache {
    struct Graph {
        uint64_t sig = 0;
        cudaGraphExec_t exec = nullptr;
        uint64_t kernels = 0;
    };
    Graph graphs[8];
    int next = 0;
    uint64_t last_sig[4] = {0, 0, 0, 0};  // per segment: signature of the last eager run
    bool on = true;
    void clear() {
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g = Graph{};
        }
        for (auto& l : last_sig) l = 0;
    }
};

// Two-layer particle level set state (particle_levelset_two_layers/plugin.rs,
// PLSResources).  Allocated when first enabled.
struct PlsState {
    bool on = false;
    bool ready = false;
    PlsArgs a{};
    uint32_t* part32 = nullptr;            // scan block totals, [2][nb]
    unsigned long long* part64 = nullptr;  // scan block totals, [2][nb]
    uint32_t nb = 0;                       // scan blocks per layer
    uint32_t* h_read = nullptr;            // pinned: count[2], dropped
};

struct efl_sim {
    efl_config cfg{};
    int nx = 0, ny = 0, P = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int status = 0;  // 0: Reset/Uninitialized, 1: Initialized (fluid_status.rs:15-21)
    Uniform U{};

    std::vector<DevBuf> bufs;
    // fields (see efl_kernels.cuh for the layout)
    PF u0, u1, v0, v1, us, vs, ls_s, div, p0, p1, ls0, ls1, fu, fv, phiT, r0;
    PI sid, uvi, uvo, vvi, vvo;
    PU lab0, lab, labT, upd;
    P2 grad, seeds[2], srcvel;
    int seeds_final = 0;
    std::vector<Level> mg;      // reference fixed-count solve (f32 iterate)
    std::vector<Level64> mg64;  // tolerance-driven solve (f64 iterate), same geometry planes

    efl_solid_obstacle* d_obs = nullptr;
    int n_obs = 0;
    efl_force* d_forces = nullptr;
    int n_forces = 0, cap_forces = 0;
    std::vector<efl_source> src_once, src_cont;
    int* d_bins = nullptr;
    efl_solid_force* d_forces_out = nullptr;
    double2* d_partials = nullptr;
    int n_partials = 0;
    float2* d_lsrange = nullptr;     // level-set (min, max) per 32 x 32 cell tile (fused extrapolation)
    unsigned* d_fimtiles = nullptr;  // per 32 x 32 tile: holds an active cell at the start of the FIM iterations
    double* d_norms = nullptr;
    double* h_norms = nullptr;  // pinned
    unsigned long long* d_count = nullptr;
    SolverWorkspace solver;
    SweepTma tma;
    MixPlanes mixp{};  // global-memory planes of the mixed solve, allocated on first use
    bool mixp_ready = false;
    CgPlanes cg{};  // MGPCG vectors, allocated on first use
    bool cg_ready = false;
    PF alt32{};          // the MGPCG preconditioner's level-0 ping-pong plane
    PF alt32_1{};        // its level-1 ping-pong plane (allocated with alt32 when level 1 exists)
    SweepTma tma_pre1;   // TMA maps of the preconditioner's level 1 (error flag shared with tma)
    const float* tma_pre1_x = nullptr;  // level 1's iterate plane the maps were built over
    SweepTma tma_pre;    // TMA maps of the preconditioner's level 0 (error flag shared with tma)
    GraphCache gc;                // captured step segments
    uint64_t graph_epoch = 1;     // counts the setters that change kernel arguments
    PF mix_d2{};       // second correction buffer (batched solve)
    PF xbuf{};         // second halo-exchange plane of the persistent solves, allocated on first use
    bool owns_stream = true;
    bool batch_member = false;  // its stages run beside the other simulations' (a batch's fan-out)
    float* d_vel = nullptr;  // velocity-magnitude partials (efl_velocity_magnitude)
    int cap_vel = 0;
    efl_rigid_body* d_rigid = nullptr;  // device-integrated bodies (efl_set_rigid_bodies)
    int n_rigid = 0;
    double rigid_gravity = 0.0, rigid_grid_length = 1.0;
    int rigid_substeps = 1;
    struct efl_unet* unet = nullptr;  // learned warm start / training recorder
    uint32_t unet_flags = 0;
    UNet* unet_view = nullptr;  // forward-only workspace of the network (batch members), owned
    int* h_err = nullptr;  // pinned copy of the TMA sweep's error flag
    cudaEvent_t ev_proj[2] = {nullptr, nullptr};  // around the last projection stage
    bool proj_timed = false;
    PlsState pls;

    Dom dom() const { return Dom{nx, ny}; }
};

namespace {

efl_status set_err(efl_sim* s, efl_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    else g_last_error = buf;
    return st;
}

#define CU(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return set_err(s, e_ == cudaErrorMemoryAllocation ? EFL_ERR_OUT_OF_MEMORY : EFL_ERR_CUDA,      \
                           "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);   \
    } while (0)

#define LAUNCH_CHECK()                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                                              \
        if (e_ != cudaSuccess)                                                                            \
            return set_err(s, EFL_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_),   \
                           __FILE__, __LINE__);                                                           \
    } while (0)

template <class T>
efl_status alloc_plane(efl_sim* s, Plane<T>& pl, int w, int h, int pitch, int rows) {
    DevBuf b;
    b.bytes = (size_t)pitch * rows * sizeof(T);
    CU(cudaMalloc(&b.p, b.bytes));
    CU(cudaMemsetAsync(b.p, 0, b.bytes, s->stream));
    s->bufs.push_back(b);
    pl.p = (T*)b.p;
    pl.w = w;
    pl.h = h;
    pl.P = pitch;
    return EFL_OK;
}
template <class T>
efl_status alloc_raw(efl_sim* s, T*& p, size_t count) {
    DevBuf b;
    b.bytes = count * sizeof(T);
    CU(cudaMalloc(&b.p, b.bytes));
    CU(cudaMemsetAsync(b.p, 0, b.bytes, s->stream));
    s->bufs.push_back(b);
    p = (T*)b.p;
    return EFL_OK;
}

#define TRY_U(x)                       \
    do {                               \
        efl_status _s = (x);           \
        if (_s != EFL_OK) return _s;   \
    } while (0)
#define TRY(x)                                  \
    do {                                        \
        efl_status st_ = (x);                   \
        if (st_ != EFL_OK) return st_;          \
    } while (0)

int mg_num_levels(const efl_config& c) {
    if (c.projection.mg_levels > 0) return (int)c.projection.mg_levels;
    int n = (int)std::log2((float)std::min(c.nx, c.ny)) - 2;  // multi_grid.rs:95-97
    return std::max(1, n);
}

efl_status alloc_mg(efl_sim* s) {
    int L = mg_num_levels(s->cfg);
    // Coarse levels live in s->bufs like every other buffer; they are only
    // rebuilt when the level count changes (efl_set_projection), and the
    // replaced ones are released with the simulation.
    s->mg.assign(L, Level{});
    s->mg64.assign(L, Level64{});
    int w = s->nx, h = s->ny;
    for (int i = 0; i < L; ++i) {
        Level& l = s->mg[i];
        Level64& d = s->mg64[i];
        l.nx = d.nx = w;
        l.ny = d.ny = h;
        int pitch = round_up(w + 1, 32);
        if (i == 0) {
            l.x = s->p0;
            l.b = s->div;
            l.ls = s->ls0;
            l.fu = s->fu;
            l.fv = s->fv;
            l.r = s->r0;
        } else {
            TRY(alloc_plane(s, l.x, w, h, pitch, h + 1));
            TRY(alloc_plane(s, l.b, w, h, pitch, h + 1));
            TRY(alloc_plane(s, l.ls, w, h, pitch, h + 1));
            TRY(alloc_plane(s, l.fu, w + 1, h, pitch, h + 1));
            TRY(alloc_plane(s, l.fv, w, h + 1, pitch, h + 1));
            TRY(alloc_plane(s, l.r, w, h, pitch, h + 1));
        }
        d.ls = l.ls;
        d.fu = l.fu;
        d.fv = l.fv;
        TRY(alloc_plane(s, d.x, w, h, pitch, h + 1));
        TRY(alloc_plane(s, d.b, w, h, pitch, h + 1));
        TRY(alloc_plane(s, d.r, w, h, pitch, h + 1));
        w /= 2;
        h /= 2;
    }
    return EFL_OK;
}

efl_status validate_cfg(const efl_config* c) {
    if (!c) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null config");
    if (!(c->length_unit > 0.0f))
        return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "length_unit must be positive value.");
    if (c->nx < 16 || c->ny < 16 || c->nx % 8 || c->ny % 8)
        return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "grid size must be a multiple of 8 and at least 16 (got %ux%u)",
                       c->nx, c->ny);
    if (c->nx > 32768 || c->ny > 32768) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "grid size too large");
    if (c->projection.method < 0 || c->projection.method > 3)
        return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "unknown projection method %d", c->projection.method);
    if (c->projection.method == EFL_PROJECTION_MGPCG && !(c->projection.tolerance > 0.0f))
        return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "MGPCG needs a tolerance > 0");
    if (c->reinit.method < 0 || c->reinit.method > 1)
        return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "unknown reinitialize method %d", c->reinit.method);
    return EFL_OK;
}

// ---------------------------------------------------------------------------
// Stages (render_node.rs:219-466)

efl_status st_init(efl_sim* s) {  // render_node.rs:219-277
    Dom d = s->dom();
    k_init_center<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->ls0, s->ls1, s->grad, d);
    k_init_edge<<<grid2d(d.nx + 1, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->u0, s->u1, s->v0, s->v1, d);
    LAUNCH_CHECK();
    return EFL_OK;
}

efl_status st_fluid_source(efl_sim* s, const std::vector<efl_source>& src) {  // update_fluid_source.wgsl
    Dom d = s->dom();
    Sources S;
    std::memset(&S, 0, sizeof(S));
    S.n = (int)src.size();
    for (int i = 0; i < S.n; ++i) S.s[i] = src[i];
    k_fluid_source_cells<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->ls1, s->upd, s->srcvel, S, d);
    k_fluid_source_faces<<<grid2d(d.nx + 1, d.ny + 1, kBlock), kBlock, count_launch(), s->stream>>>(s->u0, s->v0, s->upd,
                                                                                       s->srcvel, d);
    LAUNCH_CHECK();
    return EFL_OK;
}

std::vector<int> jfa_steps(int nx, int ny) {  // jump_flooding.rs:201-209
    int mp = (int)std::floor(std::log2((float)std::max(nx, ny)) - 1.0f);
    std::vector<int> st;
    uint32_t step = 1u << (mp + 1);
    for (int k = 0; k < mp + 1; ++k) {
        step /= 2;
        st.push_back((int)step);
    }
    return st;
}

// The tiled FIM kernel's dynamic shared memory (above the 48 KB default), set once per device.
bool fim_tiled_ready() {
    int dev = 0;
    cudaGetDevice(&dev);
    static int state[64] = {};  // 0 unknown, 1 ready, 2 refused
    if (dev < 0 || dev >= 64) return false;
    if (!state[dev]) {
        state[dev] = cudaFuncSetAttribute(k_fim_tiled<FIM_HALO, FIM_THREADS>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FIM_SMEM) ==
                             cudaSuccess
                         ? 1
                         : 2;
        cudaGetLastError();
    }
    return state[dev] == 1;
}

// Which FIM form runs: EFL_FIM_TILED=0 the per-phase launches, =1 the temporally blocked kernel with the
// 20-cell halo (10 iterations per launch), =2 the one with the 4-cell halo (2 per launch), at every size; unset
// (or anything else) the size rule in st_reinit.  All forms give bit-identical level sets.
int fim_form_override() {
    static const int v = [] {
        const char* e = std::getenv("EFL_FIM_TILED");
        return e && e[0] >= '0' && e[0] <= '2' && !e[1] ? e[0] - '0' : -1;
    }();
    return v;
}

efl_status st_reinit(efl_sim* s) {  // reinitialize_levelset.rs:162-243
    Dom d = s->dom();
    dim3 g = grid2d(d.nx, d.ny, kBlock);
    if (s->cfg.reinit.method == EFL_REINIT_JUMP_FLOODING) {
        k_jfa_init<<<g, kBlock, count_launch(), s->stream>>>(s->ls1, s->seeds[0], d);
        int src = 0, dst = 1;
        for (int step : jfa_steps(d.nx, d.ny)) {
            k_jfa_iterate<<<g, kBlock, count_launch(), s->stream>>>(s->seeds[src], s->seeds[dst], step, d);
            std::swap(src, dst);
        }
        s->seeds_final = src;
        k_jfa_sdf<<<g, kBlock, count_launch(), s->stream>>>(s->seeds[src], s->ls1, s->ls0, d);
    } else {
        const int tx = (d.nx + FIM_TILE - 1) / FIM_TILE, ty = (d.ny + FIM_TILE - 1) / FIM_TILE;
        // The wide halo pays where the grid is large and the interface a small part of it (C3: 4096^2: one
        // launch, most tiles leave at once).  On small grids a simulation stepped alone is latency-bound and
        // takes the per-phase launches (each shorter than a tiled launch); a batch member, whose launches run
        // beside the other simulations', takes the narrow halo (a quarter of the launches, a fifth of the
        // traffic).
        const int force = fim_form_override();
        int form = force >= 0 ? force : tx * ty >= 4 * s->solver.num_sms ? 1 : s->batch_member ? 2 : 0;
        if (form == 1 && !fim_tiled_ready()) form = 2;
        const uint32_t iters = s->cfg.reinit.fim_iterations;
        const int per = form == 1 ? FIM_HALO / 2 : FIM_HALO_NARROW / 2;
        const int launches = form ? (int)((iters + per - 1) / per) : 0;
        // The tiled launches alternate between (ls0, lab) and (phiT, labT) and must end in (ls0, lab): the
        // start state goes into the pair that makes the last launch land there.
        PF S[2] = {s->ls0, s->phiT};
        PU L[2] = {s->lab, s->labT};
        const int first = launches & 1;
        k_fim_init<<<g, kBlock, count_launch(), s->stream>>>(s->ls1, S[first], s->lab0, d);
        if (form) CU(cudaMemsetAsync(s->d_fimtiles, 0, (size_t)tx * ty * sizeof(unsigned), s->stream));
        k_fim_active<<<g, kBlock, count_launch(), s->stream>>>(s->lab0, L[first], d, form ? s->d_fimtiles : nullptr,
                                                                tx);
        if (form) {  // the iterations, halo / 2 per launch
            int cur = first;
            for (uint32_t k = 0; k < iters; k += per, cur ^= 1) {
                const int n = (int)std::min<uint32_t>(per, iters - k);
                const unsigned* act = k == 0 ? s->d_fimtiles : nullptr;
                if (form == 1)
                    k_fim_tiled<FIM_HALO, FIM_THREADS><<<tx * ty, FIM_THREADS, FIM_SMEM + count_launch(), s->stream>>>(
                        S[cur], L[cur], S[cur ^ 1], L[cur ^ 1], d, n, tx, act);
                else
                    k_fim_tiled<FIM_HALO_NARROW, FIM_THREADS_NARROW>
                        <<<tx * ty, FIM_THREADS_NARROW, fim_smem(FIM_HALO_NARROW) + count_launch(), s->stream>>>(
                            S[cur], L[cur], S[cur ^ 1], L[cur ^ 1], d, n, tx, act);
            }
        } else {
            for (uint32_t k = 0; k < s->cfg.reinit.fim_iterations; ++k) {
                k_fim_phase_a<<<g, kBlock, count_launch(), s->stream>>>(s->ls0, s->lab, s->phiT, s->labT, d);
                k_fim_phase_b<<<g, kBlock, count_launch(), s->stream>>>(s->phiT, s->labT, s->ls0, s->lab, d);
            }
        }
    }
    LAUNCH_CHECK();
    return EFL_OK;
}

// ---------------------------------------------------------------------------
// Two-layer particle level set (particle_levelset_two_layers/**)

efl_status pls_alloc(efl_sim* s) {
    PlsState& P = s->pls;
    PlsArgs& a = P.a;
    a.nx = s->nx;
    a.ny = s->ny;
    a.L = (uint32_t)s->nx * (uint32_t)s->ny;
    a.cap = a.L * PLS_MAX_PER_CELL;  // plugin.rs:221-225
    for (int l = 0; l < 2; ++l)
        for (int b = 0; b < 2; ++b) {
            TRY(alloc_raw(s, a.px[l][b], a.cap));
            TRY(alloc_raw(s, a.py[l][b], a.cap));
            TRY(alloc_raw(s, a.rad[l][b], a.cap));
            TRY(alloc_raw(s, a.esc[l][b], a.cap));
        }
    const size_t L2 = 2 * (size_t)a.L, C2 = 2 * (size_t)a.cap;
    TRY(alloc_raw(s, a.sel, 2));
    TRY(alloc_raw(s, a.count, 2));
    TRY(alloc_raw(s, a.cnt, L2));
    TRY(alloc_raw(s, a.cur, L2));
    TRY(alloc_raw(s, a.off, L2));
    TRY(alloc_raw(s, a.sidx, C2));
    TRY(alloc_raw(s, a.scell, C2));
    TRY(alloc_raw(s, a.sorted, C2));
    TRY(alloc_raw(s, a.prio, C2));
    TRY(alloc_raw(s, a.sesc, C2));
    TRY(alloc_raw(s, a.alive, C2));
    TRY(alloc_raw(s, a.prank, C2));
    TRY(alloc_raw(s, a.val, L2));
    TRY(alloc_raw(s, a.tot, 2));
    TRY(alloc_raw(s, a.ctot, 2));
    TRY(alloc_raw(s, a.addn, L2));
    TRY(alloc_raw(s, a.vmask, L2));
    TRY(alloc_raw(s, a.stx, L2 * PLS_GROUP));
    TRY(alloc_raw(s, a.sty, L2 * PLS_GROUP));
    TRY(alloc_raw(s, a.str, L2 * PLS_GROUP));
    TRY(alloc_raw(s, a.work, L2));
    TRY(alloc_raw(s, a.nwork, 2));
    TRY(alloc_raw(s, a.slow, L2));
    TRY(alloc_raw(s, a.nslow, 2));
    TRY(alloc_raw(s, a.phip, (size_t)a.L));
    TRY(alloc_raw(s, a.phim, (size_t)a.L));
    TRY(alloc_raw(s, a.dropped, 1));
    TRY(alloc_raw(s, a.ticket, 1));
    P.nb = (a.L + SC_N - 1) / SC_N;
    TRY(alloc_raw(s, P.part32, 2 * (size_t)P.nb));
    TRY(alloc_raw(s, P.part64, 2 * (size_t)P.nb));
    CU(cudaMallocHost(&P.h_read, 4 * sizeof(uint32_t)));
    P.ready = true;
    return EFL_OK;
}

// Grid-stride launches over the particles of both layers, and one thread per
// cell (and layer).
dim3 pls_pgrid(const PlsArgs& a) {
    return dim3((unsigned)std::min<uint32_t>((a.cap + PLS_THREADS - 1) / PLS_THREADS, 148u * 8u), 2);
}
dim3 pls_cgrid(const PlsArgs& a, int layers) { return dim3((a.L + PLS_THREADS - 1) / PLS_THREADS, layers); }
// Grid-stride launches over the work list, 16 lanes per listed cell.
dim3 pls_ggrid(const PlsArgs& a) {
    return dim3((unsigned)std::min<size_t>(((size_t)a.L * PLS_GROUP + PLS_THREADS - 1) / PLS_THREADS, 148u * 8u), 2);
}

// Exclusive scan of each layer's L values (common_pass/prefix_sum.rs).
template <class Tin, class T>
efl_status pls_scan(efl_sim* s, const Tin* in, T* out, T* part, T* tot) {
    const PlsArgs& a = s->pls.a;
    const uint32_t nb = s->pls.nb;
    k_scan_local<Tin, T><<<dim3(nb, 2), SC_T, count_launch(), s->stream>>>(in, out, part, a.L, a.L, nb);
    k_scan_parts<T><<<dim3(1, 2), SC_T, count_launch(), s->stream>>>(part, tot, nb);
    k_scan_add<T><<<pls_cgrid(a, 2), PLS_THREADS, count_launch(), s->stream>>>(out, part, a.L, a.L, nb);
    LAUNCH_CHECK();
    return EFL_OK;
}

// plugin.rs:131-158 (dispatch_initialize): band mask and seeding from
// levelset_air0 and its gradient.
efl_status pls_initialize(efl_sim* s) {
    PlsArgs& a = s->pls.a;
    CU(cudaMemsetAsync(a.nwork, 0, 2 * sizeof(uint32_t), s->stream));
    k_pls_band<<<pls_cgrid(a, 1), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0);
    k_pls_spawn_count<<<pls_ggrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0, s->grad, 1);
    LAUNCH_CHECK();
    TRY(pls_scan(s, a.val, a.val, s->pls.part64, a.tot));
    k_pls_emit<<<pls_ggrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0, s->grad, 1, 0u);
    LAUNCH_CHECK();
    return EFL_OK;
}

// plugin.rs:160-182 (dispatch_update)
efl_status pls_advect(efl_sim* s, float dt) {
    PlsArgs& a = s->pls.a;
    k_pls_advect<<<pls_pgrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, s->u0, s->v0, dt);
    LAUNCH_CHECK();
    return EFL_OK;
}

// levelset_correction.rs:96-155 (dispatch, on levelset_air1) and :157-236
// (dispatch_second, on levelset_air0, then the particle radii unless the
// reseed that follows does them with its binning pass).
efl_status pls_correct(efl_sim* s, PF ls, bool second, bool radii = true) {
    PlsArgs& a = s->pls.a;
    k_pls_reset<<<pls_cgrid(a, 1), PLS_THREADS, count_launch(), s->stream>>>(a, ls);
    k_pls_mark_accumulate<<<pls_pgrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, ls);
    k_pls_correct<<<pls_cgrid(a, 1), PLS_THREADS, count_launch(), s->stream>>>(a, ls);
    if (second && radii) k_pls_radii<<<pls_pgrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, ls);
    LAUNCH_CHECK();
    return EFL_OK;
}

// reseed.rs:130-296: bin, counting sort, per-cell heap, compaction, refill.
// radii: the binning pass first does update_particle_radii on levelset_air0.
efl_status pls_reseed(efl_sim* s, bool radii = false) {
    PlsArgs& a = s->pls.a;
    CU(cudaMemsetAsync(a.cnt, 0, 2 * (size_t)a.L * sizeof(uint32_t), s->stream));
    CU(cudaMemsetAsync(a.cur, 0, 2 * (size_t)a.L * sizeof(uint32_t), s->stream));
    CU(cudaMemsetAsync(a.nwork, 0, 2 * sizeof(uint32_t), s->stream));
    CU(cudaMemsetAsync(a.nslow, 0, 2 * sizeof(uint32_t), s->stream));
    k_pls_bin<<<pls_pgrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0, radii ? 1 : 0);
    LAUNCH_CHECK();
    TRY(pls_scan(s, a.cnt, a.off, s->pls.part32, a.ctot));
    k_pls_scatter<<<pls_pgrid(a), PLS_THREADS, count_launch(), s->stream>>>(a);
    k_pls_rank<<<pls_pgrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0);
    k_pls_heap<<<pls_cgrid(a, 2), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0);
    k_pls_select<<<dim3(std::min<uint32_t>((a.L + 7) / 8, 148u * 16u), 2), PLS_THREADS, count_launch(), s->stream>>>(a);
    k_pls_spawn_count<<<pls_ggrid(a), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0, s->grad, 0);
    LAUNCH_CHECK();
    TRY(pls_scan(s, a.val, a.val, s->pls.part64, a.tot));
    const uint32_t kb = pls_pgrid(a).x;
    k_pls_emit<<<dim3(kb + pls_ggrid(a).x, 2), PLS_THREADS, count_launch(), s->stream>>>(a, s->ls0, s->grad, 0, kb);
    LAUNCH_CHECK();
    return EFL_OK;
}

efl_status run_init(efl_sim* s) {
    TRY(st_init(s));
    if (s->pls.on) TRY(pls_initialize(s));  // render_node.rs:250-258
    TRY(st_fluid_source(s, s->src_once));
    TRY(st_reinit(s));
    return EFL_OK;
}

efl_status st_update_solid(efl_sim* s) {
    Dom d = s->dom();
    k_update_solid<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->us, s->vs, s->ls_s, s->sid, s->d_obs,
                                                                       s->n_obs, s->U, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_area_fraction(efl_sim* s) {
    Dom d = s->dom();
    k_area_fraction<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->ls_s, s->fu, s->fv, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_advect(efl_sim* s) {
    Dom d = s->dom();
    dim3 g = grid2d(d.nx + 1, d.ny + 1, kBlock);
    g.z = 2;  // u and v faces
    k_advect_uv<<<g, kBlock, count_launch(), s->stream>>>(s->u0, s->v0, s->u1, s->v1, s->U.dt, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_apply_forces(efl_sim* s) {
    Dom d = s->dom();
    dim3 g = grid2d(d.nx + 1, d.ny + 1, kBlock);
    g.z = 2;  // u and v faces
    k_apply_forces_uv<<<g, kBlock, count_launch(), s->stream>>>(s->u1, s->v1, s->ls0, s->fu, s->fv, s->d_forces,
                                                                 s->n_forces, s->U, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_divergence(efl_sim* s) {
    Dom d = s->dom();
    k_divergence<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->u1, s->v1, s->us, s->vs, s->fu, s->fv,
                                                                     s->div, s->U.dx, d);
    LAUNCH_CHECK();
    return EFL_OK;
}

// ||b - A x||^2 and ||b||^2 at level 0 into d_norms (async).
template <class T>
efl_status launch_norms(efl_sim* s, const LevelT<T>& L0) {
    k_residual_norm<T><<<s->n_partials, NORM_THREADS, count_launch(), s->stream>>>(L0, s->U.dt, s->U.rho, s->U.dx,
                                                                      s->d_partials);
    k_norm_finalize<<<1, 32, count_launch(), s->stream>>>(s->d_partials, s->n_partials, s->d_norms);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status read_norms(efl_sim* s, double* R, double* B) {
    CU(cudaMemcpyAsync(s->h_norms, s->d_norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    *R = s->h_norms[0];
    *B = s->h_norms[1];
    return EFL_OK;
}
double rel_from(double R, double B) {
    if (B > 0.0) return std::sqrt(R) / std::sqrt(B);
    return R > 0.0 ? INFINITY : 0.0;
}
template <class T>
efl_status relative_residual(efl_sim* s, const LevelT<T>& L0, double* rel) {
    TRY(launch_norms(s, L0));
    double R, B;
    TRY(read_norms(s, &R, &B));
    *rel = rel_from(R, B);
    return EFL_OK;
}

template <class T>
efl_status gs_iterations(efl_sim* s, const LevelT<T>& L, float weight, float res_scale, uint32_t n,
                         bool black_first = false) {
    float dxs = res_scale * s->U.dx;  // gauss_seidel.wgsl:57
    dim3 g = grid2d((L.nx + 1) / 2, L.ny, kBlock);
    const int c0 = black_first ? 0 : 1;  // the reference sweeps red ((x+y) odd) first
    for (uint32_t k = 0; k < n; ++k) {
        k_gs_color<T><<<g, kBlock, count_launch(), s->stream>>>(L, dxs, s->U.rho, s->U.dt, weight, c0);
        k_gs_color<T><<<g, kBlock, count_launch(), s->stream>>>(L, dxs, s->U.rho, s->U.dt, weight, 1 - c0);
    }
    LAUNCH_CHECK();
    return EFL_OK;
}

// multi_grid.rs:390-475 (smoother weight 1.0, resolution_scale 2^i: multi_grid.rs:268-270).
// symmetric (the MGPCG preconditioner): post-smoothing black then red.
template <class T>
efl_status v_cycle(efl_sim* s, std::vector<LevelT<T>>& mg, size_t i, bool symmetric = false) {
    const efl_projection& P = s->cfg.projection;
    const LevelT<T>& L = mg[i];
    if ((int64_t)L.nx * L.ny <= VT_MAX_CELLS && mg.size() <= VT_MAX_LEVELS) {  // the rest in one launch
        VTailArgs<T> a{};
        for (size_t k = 0; k < mg.size(); ++k) a.lv[k] = mg[k];
        a.first = (int)i;
        a.count = (int)mg.size();
        a.dx = s->U.dx;
        a.rho = s->U.rho;
        a.dt = s->U.dt;
        a.pre = (int)P.mg_pre;
        a.post = (int)P.mg_post;
        a.coarsest = (int)P.mg_coarsest;
        a.symmetric = symmetric ? 1 : 0;
        k_vcycle_tail<T><<<1, VT_THREADS, count_launch(), s->stream>>>(a);
        LAUNCH_CHECK();
        return EFL_OK;
    }
    float scale = (float)(1u << i);
    if (i == mg.size() - 1) return gs_iterations(s, L, 1.0f, scale, P.mg_coarsest);
    TRY(gs_iterations(s, L, 1.0f, scale, P.mg_pre));
    const LevelT<T>& C = mg[i + 1];
    k_residual_restrict<T><<<grid2d(C.nx, C.ny, kBlock), kBlock, count_launch(), s->stream>>>(L, C, s->U.dt, s->U.rho,
                                                                                          scale * s->U.dx);
    LAUNCH_CHECK();
    TRY(v_cycle(s, mg, i + 1, symmetric));
    k_prolongation<T><<<grid2d(C.nx, C.ny, kBlock), kBlock, count_launch(), s->stream>>>(L, C);
    LAUNCH_CHECK();
    return gs_iterations(s, L, 1.0f, scale, P.mg_post, symmetric);
}

// n reference (f32) red-black iterations on the pressure field: the TMA
// streaming kernel, or the shared-memory tiled kernel where TMA is
// unavailable.
efl_status sweeps_f32(efl_sim* s, float weight, uint32_t n) {
    std::string e;
    // Grids of at most one 64 x 32 tile per SM: all n iterations in one cooperative launch.
    if (!s->xbuf.p) TRY(alloc_plane(s, s->xbuf, s->nx, s->ny, s->P, s->ny + 1));
    efl_status st = solve_gs32_persistent(s->solver, s->mg[0], s->p1, s->xbuf, s->U.dx, s->U.rho, s->U.dt, weight, n,
                                          s->tma.d_err, s->stream, &e);
    if (st == EFL_OK) {
        LAUNCH_CHECK();
        return EFL_OK;
    }
    if (st != EFL_ERR_STATE) return set_err(s, st, "%s", e.c_str());
    st = solve_gs32_tma(s->tma, s->mg[0], s->p1, s->solver.num_sms, s->U.dx, s->U.rho, s->U.dt, weight, n,
                        s->stream, &e);
    if (st == EFL_ERR_STATE) {
        if (solve_gs32_tiled(s->mg[0], s->p1, s->U.dx, s->U.rho, s->U.dt, weight, n, s->stream) != EFL_OK)
            return set_err(s, EFL_ERR_CUDA, "tiled Gauss-Seidel launch failed: %s",
                           cudaGetErrorString(cudaGetLastError()));
    } else if (st != EFL_OK) {
        return set_err(s, st, "%s", e.c_str());
    }
    LAUNCH_CHECK();
    return EFL_OK;
}

efl_status ensure_mix_planes(efl_sim* s) {
    if (s->mixp_ready) return EFL_OK;
    const int nx = s->nx, ny = s->ny, P = s->P, R = ny + 1;
    TRY(alloc_plane(s, s->mixp.w, nx, ny, P, R));
    TRY(alloc_plane(s, s->mixp.inv, nx, ny, P, R));
    TRY(alloc_plane(s, s->mixp.rc, nx, ny, P, R));
    TRY(alloc_plane(s, s->mixp.d, nx, ny, P, R));
    TRY(alloc_plane(s, s->mixp.den, nx, ny, P, R));
    TRY(alloc_plane(s, s->mixp.mode, nx, ny, P, R));
    TRY(alloc_plane(s, s->mix_d2, nx, ny, P, R));
    s->mixp_ready = true;
    return EFL_OK;
}

// The tolerance-driven red-black solve (mixed-precision refinement) on the
// FP64 iterate of level 0: one cooperative launch when the grid fits the
// persistent scheme, else global-memory kernels.
efl_status gs_mixed(efl_sim* s, float weight, double tol, uint32_t max_iters, uint32_t check, SolveResult* res) {
    const Level64& L = s->mg64[0];
    std::string perr;
    if (!s->xbuf.p) TRY(alloc_plane(s, s->xbuf, s->nx, s->ny, s->P, s->ny + 1));
    efl_status ps = solve_gsmix_persistent(s->solver, L, s->r0, s->xbuf, s->U, weight, tol, max_iters, check,
                                           s->stream, res, &perr);
    if (ps == EFL_OK) return EFL_OK;
    if (ps != EFL_ERR_STATE) return set_err(s, ps, "%s", perr.c_str());
    TRY(ensure_mix_planes(s));
    ps = solve_gsmix_global(s->solver, L, s->mixp, s->U, weight, tol, max_iters, check, s->stream, res, &perr);
    if (ps != EFL_OK)
        return set_err(s, ps == EFL_ERR_STATE ? EFL_ERR_CUDA : ps, "mixed solve (global form) failed: %s",
                       perr.empty() ? "no workspace for this grid" : perr.c_str());
    LAUNCH_CHECK();
    return EFL_OK;
}

// Step segments that are replayed as CUDA graphs.
enum { SEG_FULL = 0, SEG_PRE = 1, SEG_POST = 2, SEG_CG = 3 };

uint64_t fnv(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xffu;
        h *= 1099511628211ull;
    }
    return h;
}
// The host-side values a segment's kernels are launched with.
uint64_t segment_sig(const efl_sim* s, int seg) {
    uint64_t h = 1469598103934665603ull;
    uint32_t dtb;
    std::memcpy(&dtb, &s->U.dt, 4);
    h = fnv(h, (uint64_t)seg);
    h = fnv(h, s->graph_epoch);
    h = fnv(h, dtb);
    h = fnv(h, (uint64_t)s->n_obs);
    h = fnv(h, (uint64_t)s->n_forces);
    h = fnv(h, (uint64_t)(uintptr_t)s->d_forces);
    return h | 1;  // never 0
}

// Runs body() on `stream`.  A segment whose signature repeats is captured
// into a CUDA graph on its second run and replayed from then on (the first
// run of a signature stays eager, so lazily created resources are made
// outside any capture).  If capture fails, graphs are switched off for this
// cache and the body runs eagerly.
template <class F>
efl_status run_segment(GraphCache& gc, cudaStream_t stream, uint64_t sig, int seg, F body) {
    if (!gc.on) return body();
    for (auto& g : gc.graphs)
        if (g.exec && g.sig == sig) {
            if (cudaGraphLaunch(g.exec, stream) != cudaSuccess) return EFL_ERR_CUDA;
            add_launches(g.kernels);
            return EFL_OK;
        }
    if (gc.last_sig[seg] != sig) {
        gc.last_sig[seg] = sig;
        return body();
    }
    const uint64_t n0 = launches_total();
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        gc.on = false;
        return body();
    }
    const efl_status st = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (st != EFL_OK || e != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        gc.on = false;
        if (st != EFL_OK) return st;
        return body();  // nothing ran during the failed capture
    }
    cudaGraphDestroy(graph);
    auto& slot = gc.graphs[gc.next];
    gc.next = (gc.next + 1) % (int)(sizeof(gc.graphs) / sizeof(gc.graphs[0]));
    if (slot.exec) cudaGraphExecDestroy(slot.exec);
    slot.sig = sig;
    slot.exec = exec;
    slot.kernels = launches_total() - n0;  // counted once at capture: this first launch
    if (cudaGraphLaunch(exec, stream) != cudaSuccess) return EFL_ERR_CUDA;
    return EFL_OK;
}
template <class F>
efl_status run_segment(efl_sim* s, int seg, F body) {
    const efl_status st = run_segment(s->gc, s->stream, segment_sig(s, seg), seg, body);
    if (st == EFL_ERR_CUDA && s->err.empty()) set_err(s, st, "graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return st;
}

// A fixed-order reduction (k_chunk_sums, k_chunk_rows, k_rows_total) into
// C.totals[slot], enqueued on the simulation's stream.
template <class Term>
void cg_sum_enqueue(efl_sim* s, const Term& term, int slot) {
    const int nch = (s->nx + RS_CHUNK - 1) / RS_CHUNK;
    k_chunk_sums<Term><<<dim3(nch, (s->ny + RS_CHUNK - 1) / RS_CHUNK), RS_THREADS, count_launch(), s->stream>>>(
        term, s->nx, s->ny, nch, s->cg.part);
    k_chunk_rows<<<(s->ny + 127) / 128, 128, count_launch(), s->stream>>>(s->cg.part, nch, s->ny, s->cg.rowsum);
    k_rows_total<<<1, 1024, count_launch(), s->stream>>>(s->cg.rowsum, s->ny, s->cg.totals + slot);
}

// EFL_PROJECTION_MGPCG on the FP64 level 0 (x = iterate, b = widened div):
// conjugate gradients preconditioned by one symmetric f32 V-cycle of the
// reference's structure.  Same steps and arithmetic as the oracle's
// mgpcg_solve, reductions included (fixed order), so results are bit-exact.
// The CG scalars stay on the device; one CG iteration is one segment (a CUDA
// graph from the third iteration of a signature on) followed by one read of
// the residual norms.
efl_status mgpcg(efl_sim* s, SolveResult* res) {
    const efl_projection& P = s->cfg.projection;
    const int nx = s->nx, ny = s->ny;
    TRY(ensure_mix_planes(s));
    if (!s->cg_ready) {
        const int R = ny + 1;
        TRY(alloc_plane(s, s->cg.r, nx, ny, s->P, R));
        TRY(alloc_plane(s, s->cg.p, nx, ny, s->P, R));
        TRY(alloc_plane(s, s->cg.ap, nx, ny, s->P, R));
        TRY(alloc_plane(s, s->cg.r32, nx, ny, s->P, R));
        TRY(alloc_plane(s, s->cg.z32, nx, ny, s->P, R));
        TRY(alloc_raw(s, s->cg.part, (size_t)ny * ((nx + RS_CHUNK - 1) / RS_CHUNK)));
        TRY(alloc_raw(s, s->cg.rowsum, (size_t)ny));
        TRY(alloc_raw(s, s->cg.totals, 3));
        TRY(alloc_raw(s, s->cg.sc, 1));
        CU(cudaMallocHost(&s->cg.h_read, sizeof(CgRead)));
        TRY(alloc_plane(s, s->alt32, nx, ny, s->P, R));
        if (s->mg.size() > 1)
            TRY(alloc_plane(s, s->alt32_1, s->mg[1].nx, s->mg[1].ny, s->mg[1].x.P, s->mg[1].ny + 1));
        if (s->tma.ok) {  // maps of (phi, fractions, b = r32, p = z32 / alt32)
            Level pre0 = s->mg[0];
            pre0.x = s->cg.z32;
            pre0.b = s->cg.r32;
            s->tma_pre.d_err = s->tma.d_err;
            sweep_tma_init(s->tma_pre, pre0, s->alt32);
        }
        s->cg_ready = true;
    }
    // Level 1 of the preconditioner streams through TMA too where it is too large for the single-CTA tail
    // (C3: 2048^2); its maps follow the level's planes, which efl_set_projection may reallocate.
    if (s->tma.ok && s->mg.size() > 2 && s->alt32_1.p && (int64_t)s->mg[1].nx * s->mg[1].ny > VT_MAX_CELLS &&
        s->tma_pre1_x != s->mg[1].x.p) {
        s->tma_pre1.d_err = s->tma.d_err;
        sweep_tma_init(s->tma_pre1, s->mg[1], s->alt32_1);
        s->tma_pre1_x = s->mg[1].x.p;
    }
    Level64& L = s->mg64[0];
    const MixPlanes& M = s->mixp;
    CgPlanes& C = s->cg;
    const dim3 g = grid2d(nx, ny, kBlock);
    const double dx = (double)s->U.dx;
    const double factor = (double)s->U.dt / (double)s->U.rho / dx / dx;
    k_mix_coefficients<<<g, kBlock, count_launch(), s->stream>>>(L, M);
    LAUNCH_CHECK();
    auto read_back = [&]() -> efl_status {  // C.h_read <- (norm totals, breakdown flag)
        CU(cudaMemcpyAsync(&C.h_read->norm, C.totals + 1, sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
        CU(cudaMemcpyAsync(&C.h_read->breakdown, &C.sc->breakdown, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        return EFL_OK;
    };
    // The preconditioner's f32 levels: level 0 is (x = z32, b = r32, the
    // current phi and fractions, r0 as scratch); coarse levels as usual.
    std::vector<Level> pre = s->mg;
    pre[0].x = C.z32;
    pre[0].b = C.r32;
    // Level 0's smoothing (2 + 2 red-black iterations) as two passes of the
    // TMA-streamed sweep: z32 (zero) -> alt32 red first, the coarse
    // correction on alt32, alt32 -> z32 black first; the same iterates as
    // four k_gs_color launches each.
    const bool tma0 = s->tma_pre.ok && P.mg_pre == 2 && P.mg_post == 2 && pre.size() > 1;
    const bool tma1 = tma0 && s->tma_pre1.ok && s->tma_pre1_x == pre[1].x.p && pre.size() > 2;
    auto precondition = [&]() -> efl_status {  // z = M r, then r . z into totals[2]
        CU(cudaMemset2DAsync(C.z32.p, (size_t)C.z32.P * sizeof(float), 0, (size_t)nx * sizeof(float), ny, s->stream));
        if (tma0) {
            const float dxs = s->U.dx;  // resolution scale 1 at level 0
            TRY(tma_sweep_pass(s->tma_pre, nx, ny, s->alt32, 0, s->solver.num_sms, dxs, s->U.rho, s->U.dt, 1.0f, 2,
                               1, s->tma.d_err, s->stream));
            Level L0 = pre[0];
            L0.x = s->alt32;
            const Level& C1 = pre[1];
            k_residual_restrict<float><<<grid2d(C1.nx, C1.ny, kBlock), kBlock, count_launch(), s->stream>>>(
                L0, C1, s->U.dt, s->U.rho, dxs);
            LAUNCH_CHECK();
            if (tma1) {  // level 1 as at level 0: x (zero) -> alt32_1 red first, coarse correction, back black first
                const float dxs1 = 2.0f * s->U.dx;  // resolution scale 2 (multi_grid.rs:268-270)
                TRY(tma_sweep_pass(s->tma_pre1, C1.nx, C1.ny, s->alt32_1, 0, s->solver.num_sms, dxs1, s->U.rho,
                                   s->U.dt, 1.0f, 2, 1, s->tma.d_err, s->stream));
                Level L1 = C1;
                L1.x = s->alt32_1;
                const Level& C2 = pre[2];
                k_residual_restrict<float><<<grid2d(C2.nx, C2.ny, kBlock), kBlock, count_launch(), s->stream>>>(
                    L1, C2, s->U.dt, s->U.rho, dxs1);
                LAUNCH_CHECK();
                TRY(v_cycle(s, pre, 2, true));
                k_prolongation<float><<<grid2d(C2.nx, C2.ny, kBlock), kBlock, count_launch(), s->stream>>>(L1, C2);
                LAUNCH_CHECK();
                TRY(tma_sweep_pass(s->tma_pre1, C1.nx, C1.ny, C1.x, 1, s->solver.num_sms, dxs1, s->U.rho, s->U.dt,
                                   1.0f, 2, 0, s->tma.d_err, s->stream));
            } else {
                TRY(v_cycle(s, pre, 1, true));
            }
            k_prolongation<float><<<grid2d(C1.nx, C1.ny, kBlock), kBlock, count_launch(), s->stream>>>(L0, C1);
            LAUNCH_CHECK();
            TRY(tma_sweep_pass(s->tma_pre, nx, ny, C.z32, 1, s->solver.num_sms, dxs, s->U.rho, s->U.dt, 1.0f, 2,
                               0, s->tma.d_err, s->stream));
        } else {
            TRY(v_cycle(s, pre, 0, true));
        }
        cg_sum_enqueue(s, TermDotRZ{C.r, C.z32, M}, 2);
        return EFL_OK;
    };
    cg_sum_enqueue(s, TermNorm{L.x, L.b, M, factor, nx, ny}, 1);
    k_cg_scalar<<<1, 1, count_launch(), s->stream>>>(CG_RESET, C.totals, C.sc);
    TRY(read_back());
    CU(cudaStreamSynchronize(s->stream));
    double rel = rel_from(C.h_read->norm.x, C.h_read->norm.y);
    res->r0 = rel;
    uint32_t iters = 0;
    if (!(rel <= (double)P.tolerance) && P.max_iterations > 0) {
        k_cg_mask<<<g, kBlock, count_launch(), s->stream>>>(L.x, M, nx, ny);
        k_cg_residual<<<g, kBlock, count_launch(), s->stream>>>(L.x, L.b, C.r, C.r32, M, factor, nx, ny);
        TRY(precondition());
        k_cg_scalar<<<1, 1, count_launch(), s->stream>>>(CG_RZ, C.totals, C.sc);
        k_cg_direction<<<g, kBlock, count_launch(), s->stream>>>(C.p, C.z32, M, C.sc, 1, nx, ny);
        LAUNCH_CHECK();
        // One iteration: ap = A p and p . ap; alpha = rz / p.ap (0 and a
        // breakdown flag unless p.ap > 0); x += alpha p, r -= alpha ap; the
        // true residual norms; z = M r and r . z; beta = rz' / rz; p = z + beta p.
        // The last three only matter when the host continues.
        auto iteration = [&]() -> efl_status {
            cg_sum_enqueue(s, TermMatvecDot{C.p, C.ap, M, factor, nx, ny}, 0);
            k_cg_scalar<<<1, 1, count_launch(), s->stream>>>(CG_ALPHA, C.totals, C.sc);
            k_cg_axpy<<<g, kBlock, count_launch(), s->stream>>>(L.x, C.r, C.r32, C.p, C.ap, M, C.sc, nx, ny);
            cg_sum_enqueue(s, TermNorm{L.x, L.b, M, factor, nx, ny}, 1);
            TRY(precondition());
            k_cg_scalar<<<1, 1, count_launch(), s->stream>>>(CG_BETA, C.totals, C.sc);
            k_cg_direction<<<g, kBlock, count_launch(), s->stream>>>(C.p, C.z32, M, C.sc, 0, nx, ny);
            LAUNCH_CHECK();
            return read_back();
        };
        while (iters < P.max_iterations) {
            TRY(run_segment(s, SEG_CG, iteration));
            CU(cudaStreamSynchronize(s->stream));
            if (C.h_read->breakdown) break;  // p . ap <= 0: not positive definite here (x unchanged)
            ++iters;
            rel = rel_from(C.h_read->norm.x, C.h_read->norm.y);
            if (rel <= (double)P.tolerance) break;
        }
    }
    res->iterations = iters;
    res->r1 = rel;
    res->converged = rel <= (double)P.tolerance ? 1 : 0;
    return EFL_OK;
}

// Errors that kernels report through device flags (a bounded wait that gave
// up); called after the stream has been synchronised.
efl_status check_device_errors(efl_sim* s) {
    if (!s->tma.d_err) return EFL_OK;
    CU(cudaMemcpy(s->h_err, s->tma.d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (*s->h_err) {
        const int code = *s->h_err;
        *s->h_err = 0;
        cudaMemset(s->tma.d_err, 0, sizeof(int));
        if (code == 2) return set_err(s, EFL_ERR_CUDA, "fixed-count sweep: a grid barrier timed out");
        return set_err(s, EFL_ERR_CUDA, "TMA sweep: an mbarrier wait timed out");
    }
    return EFL_OK;
}

// Learned warm start: the features of the system about to be solved, and
// (when warm-starting) x += sigma * prediction on the counted cells.
UnetFeatureArgs unet_feature_args(const efl_sim* s) {
    const Level64& L = s->mg64[0];
    const double dx = (double)s->U.dx;
    return UnetFeatureArgs{s->ls0, s->fu, s->fv, L.x, L.b, dx * dx * (double)s->U.rho / (double)s->U.dt,
                           (double)s->U.dt / (double)s->U.rho / dx / dx, s->nx, s->ny};
}

// The warm start in two halves around the network's forward pass: the features (into x0, row pitch cs coarse
// pixels: a batch's canvas; the workspace's own input when x0 is null; with widen, the f32 pressure and
// divergence widened into the solve's FP64 planes by the same kernel, in place of k_widen), then the guard that
// keeps the prediction only where it lowers the block-summed residual, and the prediction added to the iterate.
efl_status unet_features(efl_sim* s, bf16* x0 = nullptr, int cs = 0, bool widen = false) {
    UNet& n = s->unet_view ? *s->unet_view : s->unet->net;
    const int f = s->unet->net.coarse;
    if (n.coarse != f)
        return set_err(s, EFL_ERR_STATE, "the network's coarsening changed after efl_batch_attach_unet: attach again");
    const dim3 g = grid2d(s->nx, s->ny, kBlock);
    const UnetFeatureArgs a = unet_feature_args(s);
    k_unet_residual<<<g, kBlock, count_launch(), s->stream>>>(a, n.res32, n.prev32, n.mask, n.lpart,
                                                              f > 1 ? n.epart : nullptr, widen ? s->p0 : PF{},
                                                              widen ? s->div : PF{}, n.red_count, n.sigma);
    if (f > 1) {
        k_unet_features_coarse<<<g, kBlock, count_launch(), s->stream>>>(n.res32, a, n.mask, n.sigma, f,
                                                                         x0 ? x0 : n.X0, x0 ? cs : s->nx / f, n.maskc);
    } else {
        k_unet_features<<<g, kBlock, count_launch(), s->stream>>>(n.res32, a, n.mask, n.sigma, n.X0);
    }
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status unet_apply(efl_sim* s) {
    UNet& n = s->unet_view ? *s->unet_view : s->unet->net;
    const int f = n.coarse;
    const Level64& L = s->mg64[0];
    const dim3 g = grid2d(s->nx, s->ny, kBlock);
    const UnetFeatureArgs a = unet_feature_args(s);
    // The guard: kept only if it lowers the summed squares of the residual's sums over 8 x 8 blocks.
    if (f > 1) {  // the warm-started iterate formed on the fly for the guard, written only where it is kept
        const int nb = (int)(g.x * g.y);
        double* alpha = (double*)(n.epart + nb);
        k_unet_guard_residual<<<g, kBlock, count_launch(), s->stream>>>(a, n.mask, n.out, s->nx / f, n.sigma, f,
                                                                        n.epart);
        k_unet_guard<<<1, UNET_RED_THREADS, count_launch(), s->stream>>>(n.epart, nb, alpha);
        k_unet_apply_warm<<<g, kBlock, count_launch(), s->stream>>>(L.x, n.out, s->nx / f, n.mask, n.sigma, alpha,
                                                                    s->nx, s->ny, f);
    } else {
        const int gb = 8;
        const dim3 gg = grid2d((s->nx + gb - 1) / gb, (s->ny + gb - 1) / gb, kBlock);
        const int nb = (int)(gg.x * gg.y);
        double* alpha = (double*)(n.epart + nb);
        k_unet_warm<<<g, kBlock, count_launch(), s->stream>>>(L.x, n.out, n.mask, n.sigma, s->nx, s->ny);
        k_unet_block_residual<<<gg, kBlock, count_launch(), s->stream>>>(a, n.prev32, gb, n.epart);
        k_unet_guard<<<1, UNET_RED_THREADS, count_launch(), s->stream>>>(n.epart, nb, alpha);
        k_unet_guard_restore<<<g, kBlock, count_launch(), s->stream>>>(L.x, n.prev32, n.mask, alpha, s->nx, s->ny);
    }
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status unet_before_solve(efl_sim* s, bool widen = false) {
    TRY(unet_features(s, nullptr, 0, widen));
    if (s->unet_flags & EFL_UNET_WARM_START) {
        UNet& n = s->unet_view ? *s->unet_view : s->unet->net;
        unet_forward(n, s->ny / n.coarse, s->nx / n.coarse, s->stream);
        TRY(unet_apply(s));
    }
    return EFL_OK;
}
efl_status unet_after_solve(efl_sim* s) {
    UNet& n = s->unet->net;
    const int f = n.coarse;
    if (f > 1) {
        k_unet_target_coarse<<<grid2d(s->nx / f, s->ny / f, kBlock), kBlock, count_launch(), s->stream>>>(
            s->mg64[0].x, n.prev32, n.mask, n.sigma, s->nx, s->ny, f, n.targetc);
    } else {
        k_unet_target<<<grid2d(s->nx, s->ny, kBlock), kBlock, count_launch(), s->stream>>>(s->mg64[0].x, n.prev32,
                                                                                          n.sigma, s->nx, s->ny,
                                                                                          n.target);
    }
    LAUNCH_CHECK();
    s->unet->rec_nx = s->nx / f;
    s->unet->rec_ny = s->ny / f;
    s->unet->rec_coarse = f > 1;
    return EFL_OK;
}

// projection.rs:89-164.  tolerance > 0 (an extension) solves to
// ||b - A p|| / ||b|| <= tolerance with an FP64 iterate: an f32 pressure
// cannot represent a solution that accurate when hydrostatic pressure
// dominates.  p0 receives the f32 rounding of the converged iterate.
efl_status st_projection(efl_sim* s, efl_step_stats* st) {
    const efl_projection& P = s->cfg.projection;
    Dom d = s->dom();
    uint32_t iters = 0;
    int conv = 1;
    double r0 = -1.0, r1 = -1.0;
    if (P.method == EFL_PROJECTION_JACOBI) {
        dim3 g = grid2d(d.nx, d.ny, kBlock);
        for (int it = 0; it < 50; ++it) {  // projection.rs:135-143
            k_jacobi<<<g, kBlock, count_launch(), s->stream>>>(s->p0, s->p1, s->ls0, s->fu, s->fv, s->div, s->U, d);
            k_jacobi<<<g, kBlock, count_launch(), s->stream>>>(s->p1, s->p0, s->ls0, s->fu, s->fv, s->div, s->U, d);
        }
        LAUNCH_CHECK();
        iters = 50;
    } else if (P.tolerance <= 0.0f) {
        if (P.method == EFL_PROJECTION_GAUSS_SEIDEL) {
            TRY(sweeps_f32(s, P.sor_weight, P.gs_iterations));
            iters = P.gs_iterations;
        } else {
            TRY(v_cycle(s, s->mg, 0));
            iters = 1;
        }
    } else {
        const Level64& L = s->mg64[0];
        dim3 g = grid2d(d.nx, d.ny, kBlock);
        if (s->unet && s->unet_flags) {
            if ((s->unet_flags & EFL_UNET_RECORD) && s->unet_view)
                return set_err(s, EFL_ERR_STATE, "a batch member's network workspace is forward-only: record "
                                                 "training samples on a simulation of its own");
            TRY(unet_before_solve(s, true));  // its residual kernel widens p and b
        } else {
            k_widen<<<g, kBlock, count_launch(), s->stream>>>(s->p0, s->div, L.x, L.b);
            LAUNCH_CHECK();
        }
        double r = -1.0;
        bool done = false;
        if (P.method == EFL_PROJECTION_GAUSS_SEIDEL || P.method == EFL_PROJECTION_MGPCG) {
            SolveResult res{};
            if (P.method == EFL_PROJECTION_GAUSS_SEIDEL)
                TRY(gs_mixed(s, P.sor_weight, (double)P.tolerance, P.max_iterations, P.check_interval, &res));
            else
                TRY(mgpcg(s, &res));
            iters = res.iterations;
            r0 = res.r0;
            r = res.r1;
            done = true;
        }
        if (!done) {  // multigrid: FP64 V-cycles with a host-side residual test
            TRY(relative_residual(s, L, &r));
            r0 = r;
            while (!(r <= (double)P.tolerance) && iters < P.max_iterations) {
                TRY(v_cycle(s, s->mg64, 0));
                ++iters;
                TRY(relative_residual(s, L, &r));
            }
        }
        r1 = r;
        conv = r <= (double)P.tolerance;
        if (s->unet && (s->unet_flags & EFL_UNET_RECORD)) TRY(unet_after_solve(s));
        k_narrow<<<g, kBlock, count_launch(), s->stream>>>(L.x, s->p0);
        LAUNCH_CHECK();
    }
    if (st) {
        st->pressure_iterations = iters;
        st->converged = conv;
        st->residual = r1;
        st->residual_initial = r0;
    }
    return conv ? EFL_OK : EFL_NOT_CONVERGED;
}

efl_status st_solve_velocity(efl_sim* s) {
    Dom d = s->dom();
    dim3 g = grid2d(d.nx + 1, d.ny + 1, kBlock);
    g.z = 2;  // u and v faces
    k_solve_velocity_uv<<<g, kBlock, count_launch(), s->stream>>>(s->u0, s->u1, s->us, s->v0, s->v1, s->vs, s->p0,
                                                                   s->ls0, s->fu, s->fv, s->U, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_extrapolate(efl_sim* s) {  // render_node.rs:540-608
    Dom d = s->dom();
    if (d.nx % 64 == 0 && d.ny % 64 == 0) {  // every face covered: one fused launch
        const int rtx = (d.nx + EX_T - 1) / EX_T, rty = (d.ny + EX_T - 1) / EX_T;
        k_ls_tile_range<<<dim3(rtx, rty), 256, count_launch(), s->stream>>>(s->ls0, s->d_lsrange, rtx);
        ExtrapArgs a{{s->u0, s->v0}, {s->uvi, s->vvi}, {s->uvo, s->vvo}, s->ls0, s->d_lsrange, rtx, rty};
        const dim3 g((d.nx + 1 + EX_T - 1) / EX_T, (d.ny + 1 + EX_T - 1) / EX_T, 2);
        k_extrapolate_fused<<<g, 256, count_launch(), s->stream>>>(a);
        LAUNCH_CHECK();
        return EFL_OK;
    }
    dim3 gu = grid2d(d.nx + 1, d.ny, kBlock), gv = grid2d(d.nx, d.ny + 1, kBlock);
    int xrows = (d.ny / 64) * 64, ycols = (d.nx / 64) * 64;
    k_init_valid<0><<<gu, kBlock, count_launch(), s->stream>>>(s->uvi, s->ls0, d);
    k_init_valid<1><<<gv, kBlock, count_launch(), s->stream>>>(s->vvi, s->ls0, d);
    for (int k = 0; k < 10 / 2; ++k) {
        k_extrapolate<<<gu, kBlock, count_launch(), s->stream>>>(s->u0, s->uvi, s->uvo, d.nx + 1, xrows);
        k_extrapolate<<<gu, kBlock, count_launch(), s->stream>>>(s->u0, s->uvo, s->uvi, d.nx + 1, xrows);
        k_extrapolate<<<gv, kBlock, count_launch(), s->stream>>>(s->v0, s->vvi, s->vvo, ycols, d.ny + 1);
        k_extrapolate<<<gv, kBlock, count_launch(), s->stream>>>(s->v0, s->vvo, s->vvi, ycols, d.ny + 1);
    }
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_advect_levelset(efl_sim* s) {
    Dom d = s->dom();
    k_advect_levelset<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->u0, s->v0, s->ls0, s->ls1, s->U.dt, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_gradient(efl_sim* s) {
    Dom d = s->dom();
    k_gradient<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->ls0, s->grad, d);
    LAUNCH_CHECK();
    return EFL_OK;
}
efl_status st_solid_forces(efl_sim* s) {  // render_node.rs:610-641; bins zeroed per frame (fluid_to_solid.rs:211-229)
    Dom d = s->dom();
    CU(cudaMemsetAsync(s->d_bins, 0, 3 * EFL_MAX_SOLIDS * sizeof(int), s->stream));
    k_solid_forces<<<grid2d(d.nx, d.ny, kBlock), kBlock, count_launch(), s->stream>>>(s->fu, s->fv, s->sid, s->p0, s->d_obs,
                                                                       s->n_obs, s->U, d, s->d_bins);
    k_accumulate_forces<<<1, EFL_MAX_SOLIDS, count_launch(), s->stream>>>(s->d_bins, s->d_forces_out);
    LAUNCH_CHECK();
    return EFL_OK;
}

// Semi-implicit Euler of the device-coupled bodies (one thread per body),
// then their obstacles' column-major transforms, inverses and velocities.
__global__ void k_rigid_step(efl_rigid_body* bodies, int n, const efl_solid_force* forces, efl_solid_obstacle* obs,
                             double gravity, double grid_length, double dt, int substeps, double half_w,
                             double half_h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    efl_rigid_body b = bodies[i];
    if (b.dynamic) {
        const efl_solid_force f = forces[b.obstacle];
        const double sc = dt / grid_length;
        const double fx = (double)f.force[0] * sc, fy = -(double)f.force[1] * sc, tq = -(double)f.torque * sc;
        const double h = dt / substeps;
        for (int k = 0; k < substeps; ++k) {
            double vx = b.linear_velocity[0], vy = b.linear_velocity[1];
            vx += (fx / b.mass) * h;
            vy += (fy / b.mass - gravity) * h;
            const double w = b.inertia > 0.0 ? b.angular_velocity + (tq / b.inertia) * h : b.angular_velocity;
            double px = b.position[0] + vx * h, py = b.position[1] + vy * h;
            const double lox = -half_w + 1.0 + b.extent, hix = half_w - 1.0 - b.extent;
            const double loy = -half_h + 1.0 + b.extent, hiy = half_h - 1.0 - b.extent;
            if (px < lox) {
                px = lox;
                vx = fmax(vx, 0.0);
            } else if (px > hix) {
                px = hix;
                vx = fmin(vx, 0.0);
            }
            if (py < loy) {
                py = loy;
                vy = fmax(vy, 0.0);
            } else if (py > hiy) {
                py = hiy;
                vy = fmin(vy, 0.0);
            }
            b.position[0] = px;
            b.position[1] = py;
            b.linear_velocity[0] = vx;
            b.linear_velocity[1] = vy;
            b.angular_velocity = w;
            b.rotation = fmod(b.rotation + w * h, 6.283185307179586);
        }
        bodies[i] = b;
    }
    efl_solid_obstacle& o = obs[b.obstacle];
    const double c = cos(b.rotation), sn = sin(b.rotation), px = b.position[0], py = b.position[1];
    float* m = o.transform;
    float* v = o.inverse_transform;
    for (int q = 0; q < 16; ++q) m[q] = v[q] = 0.0f;
    m[0] = (float)c, m[1] = (float)sn, m[4] = (float)-sn, m[5] = (float)c, m[10] = 1.0f, m[12] = (float)px,
    m[13] = (float)py, m[15] = 1.0f;
    v[0] = (float)c, v[1] = (float)-sn, v[4] = (float)sn, v[5] = (float)c, v[10] = 1.0f,
    v[12] = (float)(-(c * px + sn * py)), v[13] = (float)(sn * px - c * py), v[15] = 1.0f;
    o.linear_velocity[0] = (float)b.linear_velocity[0];
    o.linear_velocity[1] = (float)b.linear_velocity[1];
    o.angular_velocity = (float)b.angular_velocity;
}

efl_status st_rigid(efl_sim* s) {
    if (!s->n_rigid) return EFL_OK;
    k_rigid_step<<<(s->n_rigid + 63) / 64, 64, count_launch(), s->stream>>>(
        s->d_rigid, s->n_rigid, s->d_forces_out, s->d_obs, s->rigid_gravity, s->rigid_grid_length, (double)s->U.dt,
        s->rigid_substeps, 0.5 * s->nx, 0.5 * s->ny);
    LAUNCH_CHECK();
    return EFL_OK;
}

efl_status run_stage(efl_sim* s, int stage, efl_step_stats* st) {
    switch (stage) {
        case EFL_STAGE_INIT: TRY(run_init(s)); s->status = 1; return EFL_OK;
        case EFL_STAGE_UPDATE_SOLID: return st_update_solid(s);
        case EFL_STAGE_AREA_FRACTION: return st_area_fraction(s);
        case EFL_STAGE_ADVECT_VELOCITY: return st_advect(s);
        case EFL_STAGE_APPLY_FORCES: return st_apply_forces(s);
        case EFL_STAGE_DIVERGENCE: return st_divergence(s);
        case EFL_STAGE_PROJECTION: {
            if (!s->ev_proj[0]) {
                CU(cudaEventCreate(&s->ev_proj[0]));
                CU(cudaEventCreate(&s->ev_proj[1]));
            }
            CU(cudaEventRecord(s->ev_proj[0], s->stream));
            const efl_status r = st_projection(s, st);
            CU(cudaEventRecord(s->ev_proj[1], s->stream));
            s->proj_timed = true;
            return r;
        }
        case EFL_STAGE_SOLVE_VELOCITY: return st_solve_velocity(s);
        case EFL_STAGE_EXTRAPOLATE: return st_extrapolate(s);
        case EFL_STAGE_ADVECT_LEVELSET: return st_advect_levelset(s);
        case EFL_STAGE_FLUID_SOURCE:  // + render_node.rs:389-419 (particles advected, first correction)
            TRY(st_fluid_source(s, s->src_cont));
            if (s->pls.on) {
                TRY(pls_advect(s, s->U.dt));
                TRY(pls_correct(s, s->ls1, false));
            }
            return EFL_OK;
        case EFL_STAGE_REINITIALIZE:  // + render_node.rs:421-441 (second correction, reseed)
            TRY(st_reinit(s));
            if (s->pls.on) {
                TRY(pls_correct(s, s->ls0, true, false));
                TRY(pls_reseed(s, true));
            }
            return EFL_OK;
        case EFL_STAGE_LEVELSET_GRADIENT: return st_gradient(s);
        case EFL_STAGE_SOLID_FORCES: TRY(st_solid_forces(s)); return st_rigid(s);
        default: return set_err(s, EFL_ERR_INVALID_ARGUMENT, "unknown stage %d", stage);
    }
}

void init_stats(efl_step_stats* st) {
    if (!st) return;
    std::memset(st, 0, sizeof(*st));
    st->residual = -1.0;
    st->residual_initial = -1.0;
    st->converged = 1;
}

struct FieldDesc {
    void* base;
    int w, h, ch, P;  // P in elements of ch*4 bytes
};
bool field_desc(const efl_sim* s, int f, FieldDesc* o) {
    auto pf = [&](const PF& p) { *o = FieldDesc{p.p, p.w, p.h, 1, p.P}; };
    auto pi = [&](const PI& p) { *o = FieldDesc{p.p, p.w, p.h, 1, p.P}; };
    auto pu = [&](const PU& p) { *o = FieldDesc{p.p, p.w, p.h, 1, p.P}; };
    auto p2 = [&](const P2& p) { *o = FieldDesc{p.p, p.w, p.h, 2, p.P}; };
    switch (f) {
        case EFL_FIELD_U: pf(s->u0); return true;
        case EFL_FIELD_V: pf(s->v0); return true;
        case EFL_FIELD_U1: pf(s->u1); return true;
        case EFL_FIELD_V1: pf(s->v1); return true;
        case EFL_FIELD_U_SOLID: pf(s->us); return true;
        case EFL_FIELD_V_SOLID: pf(s->vs); return true;
        case EFL_FIELD_LEVELSET_AIR: pf(s->ls0); return true;
        case EFL_FIELD_LEVELSET_AIR1: pf(s->ls1); return true;
        case EFL_FIELD_LEVELSET_SOLID: pf(s->ls_s); return true;
        case EFL_FIELD_SOLID_ID: pi(s->sid); return true;
        case EFL_FIELD_DIVERGENCE: pf(s->div); return true;
        case EFL_FIELD_PRESSURE: pf(s->p0); return true;
        case EFL_FIELD_GRAD_LEVELSET: p2(s->grad); return true;
        case EFL_FIELD_JFA_SEEDS: p2(s->seeds[s->seeds_final]); return true;
        case EFL_FIELD_FIM_LABELS: pu(s->lab); return true;
        case EFL_FIELD_U_VALID: pi(s->uvi); return true;
        case EFL_FIELD_V_VALID: pi(s->vvi); return true;
        case EFL_FIELD_AREA_FRACTION_U: pf(s->fu); return true;
        case EFL_FIELD_AREA_FRACTION_V: pf(s->fv); return true;
        default: return false;
    }
}

efl_status copy_field_out(efl_sim* s, const FieldDesc& fd, void* dst) {
    size_t row = (size_t)fd.w * fd.ch * 4;
    CU(cudaMemcpy2DAsync(dst, row, fd.base, (size_t)fd.P * fd.ch * 4, row, fd.h, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return EFL_OK;
}
efl_status copy_field_in(efl_sim* s, const FieldDesc& fd, const void* src) {
    size_t row = (size_t)fd.w * fd.ch * 4;
    CU(cudaMemcpy2DAsync(fd.base, (size_t)fd.P * fd.ch * 4, src, row, row, fd.h, cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return EFL_OK;
}

}  // namespace

extern "C" {

int32_t efl_abi_version(void) { return EFL_ABI_VERSION; }

efl_status efl_default_config(uint32_t nx, uint32_t ny, efl_config* c) {
    if (!c) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null config");
    std::memset(c, 0, sizeof(*c));
    c->nx = nx;
    c->ny = ny;
    c->length_unit = 1.0f;
    c->rho = 1.0f;
    c->gravity[0] = 0.0f;
    c->gravity[1] = 9.8f;
    for (int i = 0; i < 4; ++i) c->transform[i * 5] = 1.0f;
    c->projection.method = EFL_PROJECTION_GAUSS_SEIDEL;
    c->projection.gs_iterations = 20;
    c->projection.sor_weight = 1.9f;
    c->projection.mg_pre = 2;
    c->projection.mg_post = 2;
    c->projection.mg_coarsest = 3;
    c->projection.mg_levels = 0;
    c->projection.tolerance = 0.0f;
    c->projection.max_iterations = 20000;
    c->projection.check_interval = 16;
    c->reinit.method = EFL_REINIT_FAST_ITERATIVE;
    c->reinit.fim_iterations = 10;
    c->device = 0;
    return EFL_OK;
}

efl_status efl_create(const efl_config* cfg, efl_sim** out) {
    efl_sim* s = nullptr;
    if (!out) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    efl_status vs = validate_cfg(cfg);
    if (vs != EFL_OK) return vs;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_err(nullptr, EFL_ERR_NO_DEVICE, "no CUDA device available: %s", cudaGetErrorString(e));
    if (cfg->device < 0 || cfg->device >= ndev)
        return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "device %d out of range (%d devices)", cfg->device, ndev);
    s = new efl_sim();
    s->cfg = *cfg;
    s->nx = (int)cfg->nx;
    s->ny = (int)cfg->ny;
    s->P = round_up(s->nx + 1, 32);
    s->device = cfg->device;
    auto fail = [&](efl_status st) {
        g_last_error = s->err;
        efl_destroy(s);
        return st;
    };
#define CTRY(x)                          \
    do {                                 \
        efl_status st_ = (x);            \
        if (st_ != EFL_OK) return fail(st_); \
    } while (0)
    if (cudaSetDevice(s->device) != cudaSuccess) return fail(set_err(s, EFL_ERR_CUDA, "cudaSetDevice failed"));
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_err(s, EFL_ERR_CUDA, "cudaStreamCreate failed"));
    s->U.dx = 1.0f / cfg->length_unit;  // euler_fluid.rs:89
    s->U.dt = 0.0f;
    s->U.rho = cfg->rho;
    s->U.g[0] = cfg->gravity[0];
    s->U.g[1] = cfg->gravity[1];
    std::memcpy(s->U.m, cfg->transform, sizeof(s->U.m));
    s->U.size[0] = (float)s->nx;
    s->U.size[1] = (float)s->ny;
    const int nx = s->nx, ny = s->ny, P = s->P, R = ny + 1;
    CTRY(alloc_plane(s, s->u0, nx + 1, ny, P, R));
    CTRY(alloc_plane(s, s->u1, nx + 1, ny, P, R));
    CTRY(alloc_plane(s, s->us, nx + 1, ny, P, R));
    CTRY(alloc_plane(s, s->v0, nx, ny + 1, P, R));
    CTRY(alloc_plane(s, s->v1, nx, ny + 1, P, R));
    CTRY(alloc_plane(s, s->vs, nx, ny + 1, P, R));
    CTRY(alloc_plane(s, s->ls_s, nx, ny, P, R));
    CTRY(alloc_plane(s, s->div, nx, ny, P, R));
    CTRY(alloc_plane(s, s->p0, nx, ny, P, R));
    CTRY(alloc_plane(s, s->p1, nx, ny, P, R));
    CTRY(alloc_plane(s, s->ls0, nx, ny, P, R));
    CTRY(alloc_plane(s, s->ls1, nx, ny, P, R));
    CTRY(alloc_plane(s, s->fu, nx + 1, ny, P, R));
    CTRY(alloc_plane(s, s->fv, nx, ny + 1, P, R));
    CTRY(alloc_plane(s, s->phiT, nx, ny, P, R));
    CTRY(alloc_plane(s, s->r0, nx, ny, P, R));
    CTRY(alloc_plane(s, s->sid, nx, ny, P, R));
    CTRY(alloc_plane(s, s->uvi, nx + 1, ny, P, R));
    CTRY(alloc_plane(s, s->uvo, nx + 1, ny, P, R));
    CTRY(alloc_plane(s, s->vvi, nx, ny + 1, P, R));
    CTRY(alloc_plane(s, s->vvo, nx, ny + 1, P, R));
    CTRY(alloc_plane(s, s->lab0, nx, ny, P, R));
    CTRY(alloc_plane(s, s->lab, nx, ny, P, R));
    CTRY(alloc_plane(s, s->labT, nx, ny, P, R));
    CTRY(alloc_plane(s, s->upd, nx, ny, P, R));
    CTRY(alloc_plane(s, s->grad, nx, ny, P, R));
    CTRY(alloc_plane(s, s->seeds[0], nx, ny, P, R));
    CTRY(alloc_plane(s, s->seeds[1], nx, ny, P, R));
    CTRY(alloc_plane(s, s->srcvel, nx, ny, P, R));
    CTRY(alloc_raw(s, s->d_obs, EFL_MAX_SOLIDS));
    CTRY(alloc_raw(s, s->d_bins, 3 * EFL_MAX_SOLIDS));
    CTRY(alloc_raw(s, s->d_forces_out, EFL_MAX_SOLIDS));
    s->n_partials = std::min(1024, std::max(1, (nx * ny + NORM_THREADS - 1) / NORM_THREADS));
    CTRY(alloc_raw(s, s->d_partials, s->n_partials));
    CTRY(alloc_raw(s, s->d_lsrange, (size_t)((nx + EX_T - 1) / EX_T) * ((ny + EX_T - 1) / EX_T)));
    CTRY(alloc_raw(s, s->d_fimtiles, (size_t)((nx + FIM_TILE - 1) / FIM_TILE) * ((ny + FIM_TILE - 1) / FIM_TILE)));
    CTRY(alloc_raw(s, s->d_norms, 2));
    CTRY(alloc_raw(s, s->d_count, 1));
    if (cudaMallocHost(&s->h_norms, 4 * sizeof(double)) != cudaSuccess)
        return fail(set_err(s, EFL_ERR_OUT_OF_MEMORY, "cudaMallocHost failed"));
    CTRY(alloc_mg(s));
    CTRY(solver_init(s->solver, nx, ny, s->device, &s->err));
    if (cudaMallocHost(&s->h_err, sizeof(int)) != cudaSuccess)
        return fail(set_err(s, EFL_ERR_OUT_OF_MEMORY, "cudaMallocHost failed"));
    *s->h_err = 0;
    sweep_tma_init(s->tma, s->mg[0], s->p1);  // falls back to the tiled kernel if unavailable
    cudaGetLastError();
    if (cudaStreamSynchronize(s->stream) != cudaSuccess)
        return fail(set_err(s, EFL_ERR_CUDA, "initial clear failed: %s", cudaGetErrorString(cudaGetLastError())));
#undef CTRY
    *out = s;
    return EFL_OK;
}

efl_status efl_destroy(efl_sim* s) {
    if (!s) return EFL_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    solver_free(s->solver);
    sweep_tma_free(s->tma);
    if (s->h_err) cudaFreeHost(s->h_err);
    for (auto& b : s->bufs) cudaFree(b.p);
    if (s->d_forces) cudaFree(s->d_forces);
    if (s->h_norms) cudaFreeHost(s->h_norms);
    if (s->cg.h_read) cudaFreeHost(s->cg.h_read);
    if (s->d_vel) cudaFree(s->d_vel);
    if (s->pls.h_read) cudaFreeHost(s->pls.h_read);
    if (s->unet_view) {
        cudaFree(s->unet_view->arena);
        delete s->unet_view;
    }
    for (cudaEvent_t e : s->ev_proj)
        if (e) cudaEventDestroy(e);
    s->gc.clear();
    if (s->stream && s->owns_stream) cudaStreamDestroy(s->stream);
    delete s;
    return EFL_OK;
}

const char* efl_last_error(const efl_sim* s) { return s ? s->err.c_str() : g_last_error.c_str(); }

efl_status efl_reset(efl_sim* s) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    s->status = 0;
    ++s->graph_epoch;
    return EFL_OK;
}

efl_status efl_set_projection(efl_sim* s, const efl_projection* p) {
    if (!s || !p) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (p->method < 0 || p->method > 3) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "unknown projection method");
    if (p->method == EFL_PROJECTION_MGPCG && !(p->tolerance > 0.0f))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "MGPCG needs a tolerance > 0");
    cudaSetDevice(s->device);
    int old = mg_num_levels(s->cfg);
    s->cfg.projection = *p;
    ++s->graph_epoch;
    if (mg_num_levels(s->cfg) != old) TRY(alloc_mg(s));
    return EFL_OK;
}
efl_status efl_set_reinit(efl_sim* s, const efl_reinit* r) {
    if (!s || !r) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (r->method < 0 || r->method > 1) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "unknown reinitialize method");
    s->cfg.reinit = *r;
    ++s->graph_epoch;
    return EFL_OK;
}
efl_status efl_set_transform(efl_sim* s, const float t[16]) {
    if (!s || !t) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    std::memcpy(s->U.m, t, sizeof(s->U.m));
    std::memcpy(s->cfg.transform, t, sizeof(s->U.m));
    ++s->graph_epoch;
    return EFL_OK;
}

efl_status efl_set_obstacles(efl_sim* s, const efl_solid_obstacle* o, uint32_t n) {
    if (!s || (n && !o)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (n > EFL_MAX_SOLIDS) return set_err(s, EFL_ERR_TOO_MANY, "too many obstacles: %u (max %d)", n, EFL_MAX_SOLIDS);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t sh = o[i].shape;
        if (sh != EFL_SHAPE_CIRCLE && sh != EFL_SHAPE_RECTANGLE && sh != EFL_SHAPE_CAPSULE && sh != EFL_SHAPE_TRIANGLE)
            return set_err(s, EFL_ERR_UNSUPPORTED_SHAPE, "Unsupported shape type for solid: %u (obstacle %u)", sh, i);
    }
    cudaSetDevice(s->device);
    if (n) CU(cudaMemcpyAsync(s->d_obs, o, n * sizeof(efl_solid_obstacle), cudaMemcpyHostToDevice, s->stream));
    s->n_obs = (int)n;
    return EFL_OK;
}

efl_status efl_set_rigid_bodies(efl_sim* s, const efl_rigid_body* b, uint32_t n, double gravity, double grid_length,
                                uint32_t substeps) {
    if (!s || (n && !b)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (n > EFL_MAX_SOLIDS) return set_err(s, EFL_ERR_TOO_MANY, "too many rigid bodies: %u (max %d)", n, EFL_MAX_SOLIDS);
    if (n && !(grid_length > 0.0)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "grid_length must be positive");
    for (uint32_t i = 0; i < n; ++i)
        if (b[i].obstacle < 0 || b[i].obstacle >= s->n_obs || (b[i].dynamic && !(b[i].mass > 0.0)))
            return set_err(s, EFL_ERR_INVALID_ARGUMENT, "rigid body %u: obstacle index or mass out of range", i);
    cudaSetDevice(s->device);
    if (n && !s->d_rigid) TRY(alloc_raw(s, s->d_rigid, EFL_MAX_SOLIDS));
    if (n) CU(cudaMemcpyAsync(s->d_rigid, b, n * sizeof(efl_rigid_body), cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->n_rigid = (int)n;
    s->rigid_gravity = gravity;
    s->rigid_grid_length = grid_length;
    s->rigid_substeps = std::max<uint32_t>(1, substeps);
    ++s->graph_epoch;
    return EFL_OK;
}

efl_status efl_get_rigid_bodies(efl_sim* s, efl_rigid_body* b, uint32_t n) {
    if (!s || (n && !b)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if ((int)n > s->n_rigid) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "only %d rigid bodies", s->n_rigid);
    cudaSetDevice(s->device);
    if (n) CU(cudaMemcpyAsync(b, s->d_rigid, n * sizeof(efl_rigid_body), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return check_device_errors(s);
}

efl_status efl_set_local_forces(efl_sim* s, const efl_force* f, uint32_t n) {
    if (!s || (n && !f)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    if ((int)n > s->cap_forces) {
        CU(cudaStreamSynchronize(s->stream));
        if (s->d_forces) cudaFree(s->d_forces);
        s->d_forces = nullptr;
        s->cap_forces = 0;
        int cap = std::max<int>(64, (int)n);
        CU(cudaMalloc(&s->d_forces, (size_t)cap * sizeof(efl_force)));
        s->cap_forces = cap;
        ++s->graph_epoch;
    }
    if (n) CU(cudaMemcpyAsync(s->d_forces, f, n * sizeof(efl_force), cudaMemcpyHostToDevice, s->stream));
    s->n_forces = (int)n;
    return EFL_OK;
}

efl_status efl_set_sources(efl_sim* s, const efl_source* src, uint32_t n, int32_t oneshot) {
    if (!s || (n && !src)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (n > EFL_MAX_FLUID_SOURCE)
        return set_err(s, EFL_ERR_TOO_MANY, "The maximum number of fluid source per fluid component is %d.",
                       EFL_MAX_FLUID_SOURCE);
    (oneshot ? s->src_once : s->src_cont).assign(src, src + n);
    if (!oneshot) ++s->graph_epoch;
    return EFL_OK;
}

}  // extern "C"

namespace {
efl_status run_stages(efl_sim* s, int first, int last, efl_step_stats* st) {
    efl_status ret = EFL_OK;
    for (int stage = first; stage <= last; ++stage) {
        efl_status r = run_stage(s, stage, st);
        if (r == EFL_NOT_CONVERGED) ret = r;
        else if (r != EFL_OK) return r;
    }
    return ret;
}

// Iteration count of a fixed-count projection (projection.rs:89-164).
uint32_t fixed_iterations(const efl_projection& P) {
    if (P.method == EFL_PROJECTION_JACOBI) return 50;
    return P.method == EFL_PROJECTION_GAUSS_SEIDEL ? P.gs_iterations : 1;
}
}  // namespace

extern "C" {

efl_status efl_step(efl_sim* s, float dt, efl_step_stats* st) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    init_stats(st);
    cudaSetDevice(s->device);
    if (s->status == 0) {  // FluidStatus::Uninitialized: the init sequence only
        TRY(run_init(s));
        s->status = 1;
        if (st) st->initialized_only = 1;
        return EFL_OK;
    }
    s->U.dt = dt;
    efl_status ret = EFL_OK;
    const efl_projection& P = s->cfg.projection;
    if (P.method == EFL_PROJECTION_JACOBI || P.tolerance <= 0.0f) {
        // No host round trip anywhere: the whole step is one segment.
        TRY(run_segment(s, SEG_FULL, [&] { return run_stages(s, EFL_STAGE_UPDATE_SOLID, EFL_STAGE_SOLID_FORCES, nullptr); }));
        if (st) st->pressure_iterations = fixed_iterations(P);
    } else {
        TRY(run_segment(s, SEG_PRE, [&] { return run_stages(s, EFL_STAGE_UPDATE_SOLID, EFL_STAGE_DIVERGENCE, nullptr); }));
        ret = run_stage(s, EFL_STAGE_PROJECTION, st);
        if (ret != EFL_OK && ret != EFL_NOT_CONVERGED) return ret;
        TRY(run_segment(s, SEG_POST, [&] { return run_stages(s, EFL_STAGE_SOLVE_VELOCITY, EFL_STAGE_SOLID_FORCES, nullptr); }));
    }
    s->n_forces = 0;  // apply_forces.rs:166 clears the forces after upload
    return ret;
}

efl_status efl_set_wait_limits(efl_sim* s, uint64_t barrier_polls, uint64_t mbarrier_polls) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    const uint64_t cap = (uint64_t)1 << 40;
    if (barrier_polls > cap || mbarrier_polls > cap)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "wait limits above 2^40 polls");
    cudaSetDevice(s->device);
    CU(cudaStreamSynchronize(s->stream));
    s->solver.spin_limit = (long long)barrier_polls;  // 0: kBarrierSpinLimit
    const long long mb = mbarrier_polls ? (long long)mbarrier_polls : kMbarSpinLimit;
    s->tma.wait_limit = mb;
    s->tma_pre.wait_limit = mb;
    ++s->graph_epoch;  // captured sweeps hold the old limit as a kernel argument
    return EFL_OK;
}

efl_status efl_set_graph_capture(efl_sim* s, int32_t enable) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    cudaSetDevice(s->device);
    CU(cudaStreamSynchronize(s->stream));
    s->gc.clear();
    s->gc.on = enable != 0;
    return EFL_OK;
}

efl_status efl_projection_ms(efl_sim* s, float* ms) {
    if (!s || !ms) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (!s->proj_timed) return set_err(s, EFL_ERR_STATE, "no projection has run yet");
    CU(cudaEventSynchronize(s->ev_proj[1]));
    CU(cudaEventElapsedTime(ms, s->ev_proj[0], s->ev_proj[1]));
    return EFL_OK;
}

efl_status efl_run_stage(efl_sim* s, int32_t stage, float dt, efl_step_stats* st) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    init_stats(st);
    cudaSetDevice(s->device);
    s->U.dt = dt;
    return run_stage(s, stage, st);
}

efl_status efl_read_solid_forces(efl_sim* s, efl_solid_force out[EFL_MAX_SOLIDS]) {
    if (!s || !out) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    CU(cudaMemcpyAsync(out, s->d_forces_out, EFL_MAX_SOLIDS * sizeof(efl_solid_force), cudaMemcpyDeviceToHost,
                       s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return check_device_errors(s);
}
efl_status efl_read_force_bins(efl_sim* s, int32_t out[3 * EFL_MAX_SOLIDS]) {
    if (!s || !out) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    CU(cudaMemcpyAsync(out, s->d_bins, 3 * EFL_MAX_SOLIDS * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return EFL_OK;
}

efl_status efl_field_shape(const efl_sim* s, int32_t field, uint32_t* w, uint32_t* h, uint32_t* ch, uint32_t* eb) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    uint32_t W, H, C = 1;
    if (field == EFL_FIELD_AREA_FRACTION) {
        W = s->nx;
        H = s->ny;
        C = 4;
    } else {
        FieldDesc fd;
        if (!field_desc(s, field, &fd)) return set_err(const_cast<efl_sim*>(s), EFL_ERR_INVALID_ARGUMENT, "bad field %d", field);
        W = fd.w;
        H = fd.h;
        C = fd.ch;
    }
    if (w) *w = W;
    if (h) *h = H;
    if (ch) *ch = C;
    if (eb) *eb = 4;
    return EFL_OK;
}

efl_status efl_get_field(efl_sim* s, int32_t field, void* dst, size_t bytes) {
    if (!s || !dst) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    const int nx = s->nx, ny = s->ny;
    if (field == EFL_FIELD_AREA_FRACTION) {  // RGBA view of the face planes
        if (bytes != (size_t)nx * ny * 16) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "size mismatch");
        std::vector<float> fu((size_t)(nx + 1) * ny), fv((size_t)nx * (ny + 1));
        FieldDesc a, b;
        field_desc(s, EFL_FIELD_AREA_FRACTION_U, &a);
        field_desc(s, EFL_FIELD_AREA_FRACTION_V, &b);
        TRY(copy_field_out(s, a, fu.data()));
        TRY(copy_field_out(s, b, fv.data()));
        float* o = (float*)dst;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                float* c = o + ((size_t)y * nx + x) * 4;
                c[0] = fu[(size_t)y * (nx + 1) + x];
                c[1] = fu[(size_t)y * (nx + 1) + x + 1];
                c[2] = fv[(size_t)y * nx + x];
                c[3] = fv[(size_t)(y + 1) * nx + x];
            }
        return EFL_OK;
    }
    FieldDesc fd;
    if (!field_desc(s, field, &fd)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "bad field %d", field);
    if (bytes != (size_t)fd.w * fd.h * fd.ch * 4) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "size mismatch");
    return copy_field_out(s, fd, dst);
}

efl_status efl_set_field(efl_sim* s, int32_t field, const void* src, size_t bytes) {
    if (!s || !src) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    const int nx = s->nx, ny = s->ny;
    if (field == EFL_FIELD_AREA_FRACTION) {
        // (i-1/2) and (j-1/2) components of every cell; (i+1/2) of the last
        // column and (j+1/2) of the last row.
        if (bytes != (size_t)nx * ny * 16) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "size mismatch");
        const float* a = (const float*)src;
        std::vector<float> fu((size_t)(nx + 1) * ny), fv((size_t)nx * (ny + 1));
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const float* c = a + ((size_t)y * nx + x) * 4;
                fu[(size_t)y * (nx + 1) + x] = c[0];
                if (x == nx - 1) fu[(size_t)y * (nx + 1) + x + 1] = c[1];
                fv[(size_t)y * nx + x] = c[2];
                if (y == ny - 1) fv[(size_t)(y + 1) * nx + x] = c[3];
            }
        FieldDesc A, B;
        field_desc(s, EFL_FIELD_AREA_FRACTION_U, &A);
        field_desc(s, EFL_FIELD_AREA_FRACTION_V, &B);
        TRY(copy_field_in(s, A, fu.data()));
        return copy_field_in(s, B, fv.data());
    }
    FieldDesc fd;
    if (!field_desc(s, field, &fd)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "bad field %d", field);
    if (bytes != (size_t)fd.w * fd.h * fd.ch * 4) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "size mismatch");
    return copy_field_in(s, fd, src);
}

efl_status efl_field_device_ptr(efl_sim* s, int32_t field, void** dptr, size_t* pitch) {
    if (!s || !dptr) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    FieldDesc fd;
    if (!field_desc(s, field, &fd)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "field %d has no device plane", field);
    *dptr = fd.base;
    if (pitch) *pitch = (size_t)fd.P * fd.ch * 4;
    return EFL_OK;
}

efl_status efl_stream(efl_sim* s, void** stream) {
    if (!s || !stream) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    *stream = (void*)s->stream;
    return EFL_OK;
}

efl_status efl_synchronize(efl_sim* s) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    cudaSetDevice(s->device);
    CU(cudaStreamSynchronize(s->stream));
    return check_device_errors(s);
}

efl_status efl_residual(efl_sim* s, double* rel, double* nr, double* nb) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    cudaSetDevice(s->device);
    TRY(launch_norms(s, s->mg[0]));
    double R, B;
    TRY(read_norms(s, &R, &B));
    if (nr) *nr = std::sqrt(R);
    if (nb) *nb = std::sqrt(B);
    if (rel) *rel = rel_from(R, B);
    return EFL_OK;
}

efl_status efl_divergence_norms(efl_sim* s, double* l2, double* linf) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    cudaSetDevice(s->device);
    k_divergence_norm<<<s->n_partials, NORM_THREADS, count_launch(), s->stream>>>(s->u0, s->v0, s->us, s->vs, s->fu,
                                                                                 s->fv, s->ls0, s->U.dx, s->dom(),
                                                                                 s->d_partials);
    k_div_norm_finalize<<<1, 32, count_launch(), s->stream>>>(s->d_partials, s->n_partials, s->d_norms);
    LAUNCH_CHECK();
    double a2, m;
    TRY(read_norms(s, &a2, &m));
    if (l2) *l2 = std::sqrt(a2);
    if (linf) *linf = m;
    return EFL_OK;
}

efl_status efl_fluid_volume(efl_sim* s, uint64_t* cells) {
    if (!s || !cells) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    CU(cudaMemsetAsync(s->d_count, 0, sizeof(unsigned long long), s->stream));
    k_volume<<<grid2d(s->nx, s->ny, kBlock), kBlock, count_launch(), s->stream>>>(s->ls0, s->d_count);
    LAUNCH_CHECK();
    unsigned long long c = 0;
    CU(cudaMemcpyAsync(&c, s->d_count, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    *cells = c;
    return EFL_OK;
}

efl_status efl_velocity_magnitude(efl_sim* s, float* min_mag, float* max_mag) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    cudaSetDevice(s->device);
    const int gx = s->nx / 16, gy = s->ny / 16, n = gx * gy;
    if (s->cap_vel < n) {
        if (s->d_vel) cudaFree(s->d_vel);
        s->d_vel = nullptr;
        CU(cudaMalloc(&s->d_vel, (size_t)(2 * n + 2) * sizeof(float)));
        s->cap_vel = n;
    }
    k_velocity_partial<<<dim3(gx, gy), dim3(16, 16), count_launch(), s->stream>>>(s->u0, s->v0, s->ls0, s->d_vel,
                                                                                  s->d_vel + n);
    k_velocity_final<<<1, 512, count_launch(), s->stream>>>(s->d_vel, s->d_vel + n, n, s->d_vel + 2 * n);
    LAUNCH_CHECK();
    float r[2];
    CU(cudaMemcpyAsync(r, s->d_vel + 2 * n, sizeof(r), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    if (min_mag) *min_mag = r[0];
    if (max_mag) *max_mag = r[1];
    return EFL_OK;
}

// ---------------------------------------------------------------------------
// Two-layer particle level set (ParticleLevelsetTwoLayersPlugin, plugin.rs)

efl_status efl_set_particle_levelset(efl_sim* s, int32_t enable) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    cudaSetDevice(s->device);
    if (enable && !s->pls.ready) TRY(pls_alloc(s));
    s->pls.on = enable != 0;
    ++s->graph_epoch;
    return EFL_OK;
}

efl_status efl_particle_counts(efl_sim* s, uint32_t counts[2], uint32_t* dropped) {
    if (!s || !counts) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    counts[0] = counts[1] = 0;
    if (dropped) *dropped = 0;
    if (!s->pls.ready) return EFL_OK;
    cudaSetDevice(s->device);
    uint32_t* h = s->pls.h_read;
    CU(cudaMemcpyAsync(h, s->pls.a.count, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(h + 2, s->pls.a.dropped, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    counts[0] = h[0];
    counts[1] = h[1];
    if (dropped) *dropped = h[2];
    return EFL_OK;
}

efl_status efl_read_particles(efl_sim* s, int32_t layer, efl_particle* dst, uint32_t capacity, uint32_t* n) {
    if (!s || !n || (capacity && !dst)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (layer != EFL_PLS_POSITIVE && layer != EFL_PLS_NEGATIVE)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "unknown particle layer %d", layer);
    uint32_t counts[2];
    TRY(efl_particle_counts(s, counts, nullptr));
    *n = counts[layer];
    const uint32_t m = std::min(counts[layer], capacity);
    if (!m) return EFL_OK;
    const PlsArgs& a = s->pls.a;
    int b = 0;
    CU(cudaMemcpyAsync(&b, a.sel + layer, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    std::vector<float> x(m), y(m), r(m);
    std::vector<uint8_t> e(m);
    CU(cudaMemcpyAsync(x.data(), a.px[layer][b], m * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(y.data(), a.py[layer][b], m * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(r.data(), a.rad[layer][b], m * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CU(cudaMemcpyAsync(e.data(), a.esc[layer][b], m, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    const float sgn = layer == EFL_PLS_POSITIVE ? 1.0f : -1.0f;
    for (uint32_t i = 0; i < m; ++i) {
        dst[i].position[0] = x[i];
        dst[i].position[1] = y[i];
        dst[i].radius = r[i];
        dst[i].sign = sgn;
        dst[i].escaped = e[i];
        dst[i]._pad = 0;
    }
    return EFL_OK;
}

efl_status efl_write_particles(efl_sim* s, int32_t layer, const efl_particle* src, uint32_t n) {
    if (!s || (n && !src)) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (layer != EFL_PLS_POSITIVE && layer != EFL_PLS_NEGATIVE)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "unknown particle layer %d", layer);
    if (!s->pls.ready) return set_err(s, EFL_ERR_STATE, "the particle level set is not enabled");
    const PlsArgs& a = s->pls.a;
    if (n > a.cap) return set_err(s, EFL_ERR_TOO_MANY, "%u particles exceed the capacity %u", n, a.cap);
    const float sgn = layer == EFL_PLS_POSITIVE ? 1.0f : -1.0f;
    std::vector<float> x(n), y(n), r(n);
    std::vector<uint8_t> e(n);
    for (uint32_t i = 0; i < n; ++i) {
        if (src[i].sign != sgn)
            return set_err(s, EFL_ERR_INVALID_ARGUMENT, "particle %u has sign %g in layer %d", i, src[i].sign, layer);
        x[i] = src[i].position[0];
        y[i] = src[i].position[1];
        r[i] = src[i].radius;
        e[i] = src[i].escaped ? 1 : 0;
    }
    cudaSetDevice(s->device);
    if (n) {  // into buffer 0, which becomes the live one
        CU(cudaMemcpyAsync(a.px[layer][0], x.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        CU(cudaMemcpyAsync(a.py[layer][0], y.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        CU(cudaMemcpyAsync(a.rad[layer][0], r.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        CU(cudaMemcpyAsync(a.esc[layer][0], e.data(), n, cudaMemcpyHostToDevice, s->stream));
    }
    const int zero = 0;
    CU(cudaMemcpyAsync(a.sel + layer, &zero, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    CU(cudaMemcpyAsync(a.count + layer, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return EFL_OK;
}

efl_status efl_pls_run_phase(efl_sim* s, int32_t phase, float dt) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    if (!s->pls.ready) return set_err(s, EFL_ERR_STATE, "the particle level set is not enabled");
    cudaSetDevice(s->device);
    switch (phase) {
        case EFL_PLS_INITIALIZE: return pls_initialize(s);
        case EFL_PLS_ADVECT: return pls_advect(s, dt);
        case EFL_PLS_CORRECT: return pls_correct(s, s->ls1, false);
        case EFL_PLS_CORRECT_SECOND: return pls_correct(s, s->ls0, true);
        case EFL_PLS_RESEED: return pls_reseed(s);
        default: return set_err(s, EFL_ERR_INVALID_ARGUMENT, "unknown particle level set phase %d", phase);
    }
}

uint64_t efl_kernel_launches(void) { return efl::launches_total(); }

efl_status efl_pressure_sweeps(efl_sim* s, int32_t precision, uint32_t iterations) {
    if (!s) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null sim");
    if (precision != 32 && precision != 64) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "precision must be 32 or 64");
    cudaSetDevice(s->device);
    const float w = s->cfg.projection.sor_weight;
    if (precision == 32) {
        TRY(sweeps_f32(s, w, iterations));
    } else {
        // The tolerance-driven solver with an unreachable tolerance: exactly
        // `iterations` iterations, residual evaluated before and after only.
        SolveResult res{};
        TRY(gs_mixed(s, w, 0.0, iterations, std::max<uint32_t>(1, iterations), &res));
    }
    LAUNCH_CHECK();
    return EFL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free residual norms.
//
// Some callers cannot let a library allocate device memory: an engine that
// owns every GPU buffer through its own arena (for example fields exported
// from its renderer), or a real-time frame loop that forbids allocation once
// it is running.  efl_residual_norms_noalloc serves them: it reads the
// caller's buffers, writes the caller's output, and keeps its per-block
// partial sums in the fixed file-scope array below instead of in memory from
// cudaMalloc.  Every GPU that loads this library holds the array (256 KiB)
// until the process exits.
namespace {

constexpr int kNoAllocCellsPerBlock = 1024;  // NORM_THREADS threads x 4 cells
constexpr int kNoAllocMaxBlocks = 16384;
constexpr uint64_t kNoAllocMaxCells = (uint64_t)kNoAllocMaxBlocks * kNoAllocCellsPerBlock;  // 4096 x 4096
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double2 g_noalloc_partials[kNoAllocMaxBlocks];

// Device address of g_noalloc_partials per device ordinal.  Host code must
// not pass the symbol itself to a kernel: on the host it only names a
// stand-in object.
std::mutex g_noalloc_mu;
double2* g_noalloc_addr[kNoAllocMaxDevices] = {};

// One block sums the per-block partials: thread t adds partials t, t + 256,
// ... in order, then a shared-memory tree halves the 256 sums in a fixed
// pattern, so the result does not depend on scheduling.
constexpr int kNoAllocFinalizeThreads = 256;
__global__ void __launch_bounds__(kNoAllocFinalizeThreads)
    k_norm_finalize_rel(const double2* partials, int n, double* out) {
    __shared__ double sr[kNoAllocFinalizeThreads], sb[kNoAllocFinalizeThreads];
    const int t = threadIdx.x;
    double r = 0.0, b = 0.0;
    for (int i = t; i < n; i += kNoAllocFinalizeThreads) {
        const double2 q = partials[i];
        r += q.x;
        b += q.y;
    }
    sr[t] = r;
    sb[t] = b;
    __syncthreads();
    for (int h = kNoAllocFinalizeThreads / 2; h > 0; h >>= 1) {
        if (t < h) {
            sr[t] += sr[t + h];
            sb[t] += sb[t + h];
        }
        __syncthreads();
    }
    if (t != 0) return;
    const double nr = sqrt(sr[0]), nb = sqrt(sb[0]);
    out[0] = sb[0] > 0.0 ? nr / nb : (sr[0] > 0.0 ? INFINITY : 0.0);
    out[1] = nr;
    out[2] = nb;
}

}  // namespace

extern "C" efl_status efl_residual_norms_noalloc(const float* pressure, const float* divergence,
                                                 const float* levelset_air, const float* area_fraction_u,
                                                 const float* area_fraction_v, uint32_t nx, uint32_t ny,
                                                 size_t pitch_bytes, float dx, float dt, float rho,
                                                 double* out_device, void* stream) {
    efl_sim* s = nullptr;  // errors go to efl_last_error(NULL)
    if (!pressure || !divergence || !levelset_air || !area_fraction_u || !area_fraction_v || !out_device)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_residual_norms_noalloc: null pointer argument");
    if (nx == 0 || ny == 0)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_residual_norms_noalloc: empty grid %ux%u", nx, ny);
    if ((uint64_t)nx * ny > kNoAllocMaxCells)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT,
                       "efl_residual_norms_noalloc: %ux%u = %llu cells exceeds the fixed scratch limit of %llu cells "
                       "(4096 x 4096); use efl_residual on an efl_sim for larger grids",
                       nx, ny, (unsigned long long)nx * ny, (unsigned long long)kNoAllocMaxCells);
    if (pitch_bytes % sizeof(float) != 0 || pitch_bytes < (size_t)(nx + 1) * sizeof(float))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT,
                       "efl_residual_norms_noalloc: pitch %zu bytes must be a multiple of 4 and hold nx+1 floats",
                       pitch_bytes);
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_residual_norms_noalloc: device ordinal %d unsupported", dev);
    double2* partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {  // once per device, with that device current
            void* p = nullptr;
            CU(cudaGetSymbolAddress(&p, g_noalloc_partials));
            g_noalloc_addr[dev] = (double2*)p;
        }
        partials = g_noalloc_addr[dev];
    }
    const int P = (int)(pitch_bytes / sizeof(float));
    Level L{};
    L.nx = (int)nx;
    L.ny = (int)ny;
    L.x = PF{const_cast<float*>(pressure), (int)nx, (int)ny, P};
    L.b = PF{const_cast<float*>(divergence), (int)nx, (int)ny, P};
    L.r = L.x;  // not read by the norm kernel
    L.ls = PF{const_cast<float*>(levelset_air), (int)nx, (int)ny, P};
    L.fu = PF{const_cast<float*>(area_fraction_u), (int)nx + 1, (int)ny, P};
    L.fv = PF{const_cast<float*>(area_fraction_v), (int)nx, (int)ny + 1, P};
    const int blocks = (int)(((uint64_t)nx * ny + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock);
    cudaStream_t st = (cudaStream_t)stream;
    k_residual_norm<float><<<blocks, NORM_THREADS, count_launch(), st>>>(L, dt, rho, dx, partials);
    k_norm_finalize_rel<<<1, kNoAllocFinalizeThreads, count_launch(), st>>>(partials, blocks, out_device);
    LAUNCH_CHECK();
    return EFL_OK;
}

// ---------------------------------------------------------------------------
// Batches of simulations.

struct efl_batch {
    std::vector<efl_sim*> sims;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    BatchSim* d_sims = nullptr;
    int2* d_tiles = nullptr;
    double2* d_partials = nullptr;
    int* d_n_active = nullptr;
    int2* d_work = nullptr;
    int* d_work_count = nullptr;
    BatchState* d_state = nullptr;
    BatchState* h_state = nullptr;  // pinned
    GridBarrier* d_barrier = nullptr;
    int ntiles = 0;
    std::vector<int> tile_start;
    cudaEvent_t ev[2] = {nullptr, nullptr};  // around the last batched solve
    bool timed = false;
    GraphCache gc;  // the stages before and after the batched solve, all simulations
    // Autotuner of the batched solve's tile shape and iterations per round:
    // the first solves try each configuration once, timing ns per
    // cell-iteration; the fastest is kept.
    int tile_cfg = -1;           // chosen configuration, -1 while tuning
    int tile_fixed = -1;         // set by efl_batch_set_tiles, -1 = autotune
    int tune_next = 0;
    std::vector<double> tune_cost;  // ns per cell-iteration, per configuration (0 = not tried)
    long long spin_limit = 0;       // grid-barrier polls of the batched solve (0: the default)
    // The simulations' stages run on one work stream each, forked from and joined back into the batch
    // stream, so that the small kernels of different simulations overlap on the GPU (and, captured into
    // a CUDA graph, form independent branches).  The simulations' public stream stays the batch stream.
    std::vector<cudaStream_t> work;
    std::vector<cudaEvent_t> ev_join;
    cudaEvent_t ev_fork = nullptr;
    // The network's forward pass for all simulations at once (efl_batch_attach_unet with a coarsening f > 1):
    // each simulation's coarse features sit in a rectangle of one canvas, 8-pixel gaps around them, and one
    // launch per layer covers the canvas.
    UNet* canvas = nullptr;
    const efl_unet* canvas_net = nullptr;  // the network the canvas was set up for
    unsigned char* d_gaps = nullptr;       // the four levels' masks (1 inside a rectangle), one allocation
    const unsigned char* gaps[4] = {};
    int cw = 0, ch = 0;                    // canvas width and height, coarse pixels
    std::vector<int2> corigin;             // per simulation: its rectangle's origin
    // The warm start's phases around the canvas forward, one launch each for the simulations on the canvas:
    // their descriptors and block starts on the device, and the host copies last uploaded.
    WarmSim* d_warm = nullptr;
    int* d_warm_start = nullptr;
    std::vector<WarmSim> h_warm;
    std::vector<int> h_warm_start;
};

namespace {
// Tile shapes (owned cells) and red-black iterations per streamed round of
// the batched solve.  32 x 32 is the smallest tile: buffers are sized for it.
struct BatchTileConfig {
    int tx, ty, k;
    const void* kern;
    size_t smem;
};
template <int TX, int TY, int K>
BatchTileConfig batch_config() {
    constexpr int EX = TX + 4 * K, EY = TY + 4 * K;
    return {TX, TY, K, (const void*)k_batch_mix<TX, TY, K>, sizeof(BatchTile<EX, EY>)};
}
const BatchTileConfig& batch_configs(int i) {
    static const BatchTileConfig c[] = {batch_config<64, 32, 2>(), batch_config<64, 32, 4>(), batch_config<32, 32, 2>(),
                                        batch_config<64, 32, 8>()};
    return c[i];
}
constexpr int kBatchConfigs = 4, kMinTile = 32;
std::string g_batch_error;

efl_status batch_err(efl_batch* b, efl_status st, const std::string& m) {
    if (b) b->err = m;
    else g_batch_error = m;
    return st;
}

void canvas_free(efl_batch* b) {
    if (b->canvas) {
        cudaFree(b->canvas->arena);
        delete b->canvas;
    }
    cudaFree(b->d_gaps);
    cudaFree(b->d_warm);
    cudaFree(b->d_warm_start);
    b->d_warm = nullptr;
    b->d_warm_start = nullptr;
    b->h_warm.clear();
    b->h_warm_start.clear();
    b->canvas = nullptr;
    b->canvas_net = nullptr;
    b->d_gaps = nullptr;
    b->cw = b->ch = 0;
    b->corigin.clear();
}

void batch_free(efl_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    canvas_free(b);
    for (efl_sim* s : b->sims) efl_destroy(s);
    cudaFree(b->d_sims);
    cudaFree(b->d_tiles);
    cudaFree(b->d_partials);
    cudaFree(b->d_n_active);
    cudaFree(b->d_work);
    cudaFree(b->d_work_count);
    cudaFree(b->d_state);
    cudaFree(b->d_barrier);
    if (b->h_state) cudaFreeHost(b->h_state);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    b->gc.clear();
    for (cudaStream_t w : b->work)
        if (w) cudaStreamDestroy(w);
    for (cudaEvent_t e : b->ev_join)
        if (e) cudaEventDestroy(e);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

// Runs per_sim(i, s) for every simulation on its own work stream: the work
// streams wait for the batch stream, each simulation's launches go to its
// work stream (s->stream is switched for the call), and the batch stream then
// waits for every work stream.  Inside a stream capture this makes one graph
// branch per simulation.
template <class F>
efl_status batch_fanout(efl_batch* b, F per_sim) {
    if (cudaEventRecord(b->ev_fork, b->stream) != cudaSuccess) return EFL_ERR_CUDA;
    for (cudaStream_t w : b->work)
        if (cudaStreamWaitEvent(w, b->ev_fork, 0) != cudaSuccess) return EFL_ERR_CUDA;
    efl_status st = EFL_OK;
    for (size_t i = 0; i < b->sims.size() && st == EFL_OK; ++i) {
        efl_sim* s = b->sims[i];
        s->stream = b->work[i];
        st = per_sim(i, s);
        s->stream = b->stream;
    }
    for (size_t i = 0; i < b->sims.size(); ++i) {  // always rejoin, so that a capture stays well formed
        if (cudaEventRecord(b->ev_join[i], b->work[i]) != cudaSuccess ||
            cudaStreamWaitEvent(b->stream, b->ev_join[i], 0) != cudaSuccess)
            return EFL_ERR_CUDA;
    }
    return st;
}

// One cooperative launch for the tolerance-driven solves of the batch's
// simulations listed in `which` (equal check_interval, max_iterations and
// tolerance), results into stats.
efl_status batch_solve(efl_batch* b, const std::vector<int>& which, efl_step_stats* stats) {
    if (which.empty()) return EFL_OK;
    if ((int)b->tune_cost.size() != kBatchConfigs) b->tune_cost.assign(kBatchConfigs, 0.0);
    const int ci = b->tile_fixed >= 0 ? b->tile_fixed : (b->tile_cfg >= 0 ? b->tile_cfg : b->tune_next);
    const BatchTileConfig& cfg = batch_configs(ci);
    std::vector<BatchSim> hs;
    std::vector<int2> tiles;
    for (int idx : which) {
        efl_sim* s = b->sims[idx];
        BatchSim S{};
        S.L = s->mg64[0];
        S.M = s->mixp;
        S.d[0] = s->mixp.d;
        S.d[1] = s->mix_d2;
        const double dx = (double)s->U.dx;
        S.cdiv = dx * dx * (double)s->U.rho / (double)s->U.dt;
        S.factor = (double)s->U.dt / (double)s->U.rho / dx / dx;
        S.weight = s->cfg.projection.sor_weight;
        S.tiles_x = (s->nx + cfg.tx - 1) / cfg.tx;
        const int ty = (s->ny + cfg.ty - 1) / cfg.ty;
        S.tile_start = (int)tiles.size();
        S.tile_count = S.tiles_x * ty;
        for (int t = 0; t < S.tile_count; ++t) tiles.push_back(make_int2((int)hs.size(), t));
        hs.push_back(S);
    }
    const int ns = (int)hs.size(), nt = (int)tiles.size();
    if (nt > b->ntiles || ns > (int)b->sims.size()) return batch_err(b, EFL_ERR_STATE, "batch tile list overflow");
    cudaStream_t st = b->stream;
    if (cudaMemcpyAsync(b->d_sims, hs.data(), ns * sizeof(BatchSim), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(b->d_tiles, tiles.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return batch_err(b, EFL_ERR_CUDA, "batch upload failed");
    for (int i = 0; i < ns; ++i) {
        b->h_state[i] = BatchState{};
        b->h_state[i].active = 1;
    }
    if (cudaMemcpyAsync(b->d_state, b->h_state, ns * sizeof(BatchState), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(b->d_barrier, 0, sizeof(GridBarrier), st) != cudaSuccess)
        return batch_err(b, EFL_ERR_CUDA, "batch state upload failed");
    const efl_projection& P0 = b->sims[which[0]]->cfg.projection;
    BatchParams Pm;
    Pm.sims = b->d_sims;
    Pm.nsims = ns;
    Pm.ntiles = nt;
    Pm.tiles = b->d_tiles;
    Pm.tol = (double)P0.tolerance;
    Pm.max_iters = P0.max_iterations;
    Pm.check_interval = std::max<uint32_t>(1, P0.check_interval);
    Pm.partials = b->d_partials;
    Pm.n_active = b->d_n_active;
    Pm.work = b->d_work;
    Pm.work_count = b->d_work_count;
    Pm.state = b->d_state;
    Pm.barrier = b->d_barrier;
    Pm.spin_limit = b->spin_limit > 0 ? b->spin_limit : kBarrierSpinLimit;
    const size_t smem = cfg.smem;
    const void* kern = cfg.kern;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return batch_err(b, EFL_ERR_CUDA, "batched solver: shared-memory attribute refused");
    int per_sm = 0, sms = b->sims[which[0]]->solver.num_sms;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT_THREADS, smem) != cudaSuccess || per_sm < 1)
        return batch_err(b, EFL_ERR_CUDA, "batched solver: no co-resident CTA fits");
    const int grid = std::min(per_sm * sms, std::max(1, nt));
    if (nt > BT_MAX_OWN * grid)
        return batch_err(b, EFL_ERR_INVALID_ARGUMENT,
                         "batch too large: " + std::to_string(nt) + " tiles, at most " +
                             std::to_string(BT_MAX_OWN * grid) + " per cooperative launch");
    void* args[] = {&Pm};
    count_launch();
    if (!b->ev[0] && (cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess))
        return batch_err(b, EFL_ERR_CUDA, "event creation failed");
    cudaEventRecord(b->ev[0], st);
    cudaError_t e = cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(BT_THREADS), args, smem, st);
    cudaEventRecord(b->ev[1], st);
    b->timed = true;
    if (e != cudaSuccess)
        return batch_err(b, EFL_ERR_CUDA, std::string("batched solver launch failed: ") + cudaGetErrorString(e));
    GridBarrier hb{};
    if (cudaMemcpyAsync(b->h_state, b->d_state, ns * sizeof(BatchState), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&hb, b->d_barrier, sizeof(hb), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return batch_err(b, EFL_ERR_CUDA, std::string("batched solver failed: ") + cudaGetErrorString(cudaGetLastError()));
    if (hb.error) return batch_err(b, EFL_ERR_CUDA, "batched solver: a grid barrier timed out");
    // Autotuner bookkeeping: device time per cell-iteration of this configuration.
    double work = 0.0;
    for (int i = 0; i < ns; ++i) {
        const efl_sim* s = b->sims[which[i]];
        work += (double)s->nx * s->ny * b->h_state[i].iterations;
    }
    float ms = 0.0f;
    if (work > 0.0 && cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]) == cudaSuccess) {
        const double cost = ms * 1e6 / work;
        if (b->tune_cost[ci] == 0.0 || cost < b->tune_cost[ci]) b->tune_cost[ci] = cost;
        if (b->tile_fixed < 0 && b->tile_cfg < 0) {
            if (++b->tune_next == kBatchConfigs) {
                int best = 0;
                for (int c = 1; c < kBatchConfigs; ++c)
                    if (b->tune_cost[c] < b->tune_cost[best]) best = c;
                b->tile_cfg = best;
            }
        }
    }
    for (int i = 0; i < ns; ++i) {
        efl_step_stats* o = stats ? &stats[which[i]] : nullptr;
        if (!o) continue;
        o->pressure_iterations = b->h_state[i].iterations;
        o->converged = b->h_state[i].converged;
        o->residual = b->h_state[i].r1;
        o->residual_initial = b->h_state[i].r0;
    }
    return EFL_OK;
}
}  // namespace

extern "C" {

efl_status efl_batch_create(const efl_config* cfgs, uint32_t n, efl_batch** out) {
    if (!out || !cfgs || n == 0) return batch_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null argument or empty batch");
    *out = nullptr;
    efl_batch* b = new efl_batch();
    b->device = cfgs[0].device;
    for (uint32_t i = 0; i < n; ++i)
        if (cfgs[i].device != b->device) {
            delete b;
            return batch_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "all simulations of a batch must be on one device");
        }
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return batch_err(nullptr, EFL_ERR_CUDA, "batch stream creation failed");
    }
    int total_tiles = 0;
    for (uint32_t i = 0; i < n; ++i) {
        efl_sim* s = nullptr;
        efl_status st = efl_create(&cfgs[i], &s);
        if (st != EFL_OK) {
            std::string m = std::string("simulation ") + std::to_string(i) + ": " + efl_last_error(nullptr);
            batch_free(b);
            return batch_err(nullptr, st, m);
        }
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
        s->stream = b->stream;
        s->owns_stream = false;
        s->batch_member = true;
        b->sims.push_back(s);
        if (ensure_mix_planes(s) != EFL_OK) {
            std::string m = s->err;
            batch_free(b);
            return batch_err(nullptr, EFL_ERR_OUT_OF_MEMORY, m);
        }
        total_tiles += ((s->nx + kMinTile - 1) / kMinTile) * ((s->ny + kMinTile - 1) / kMinTile);
    }
    b->ntiles = total_tiles;
    b->work.assign(n, nullptr);
    b->ev_join.assign(n, nullptr);
    bool ok = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (uint32_t i = 0; i < n && ok; ++i)
        ok = cudaStreamCreateWithFlags(&b->work[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        batch_free(b);
        return batch_err(nullptr, EFL_ERR_CUDA, "batch work stream creation failed");
    }
    if (cudaMalloc(&b->d_sims, n * sizeof(BatchSim)) != cudaSuccess ||
        cudaMalloc(&b->d_tiles, total_tiles * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&b->d_partials, total_tiles * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&b->d_n_active, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_work, total_tiles * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&b->d_work_count, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_state, n * sizeof(BatchState)) != cudaSuccess ||
        cudaMalloc(&b->d_barrier, sizeof(GridBarrier)) != cudaSuccess ||
        cudaMallocHost(&b->h_state, n * sizeof(BatchState)) != cudaSuccess) {
        batch_free(b);
        return batch_err(nullptr, EFL_ERR_OUT_OF_MEMORY, "batch workspace allocation failed");
    }
    *out = b;
    return EFL_OK;
}

efl_status efl_batch_destroy(efl_batch* b) {
    batch_free(b);
    return EFL_OK;
}

const char* efl_batch_last_error(const efl_batch* b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

efl_status efl_batch_sim(efl_batch* b, uint32_t i, efl_sim** sim) {
    if (!b || !sim || i >= b->sims.size()) return batch_err(b, EFL_ERR_INVALID_ARGUMENT, "bad batch index");
    *sim = b->sims[i];
    return EFL_OK;
}

efl_status efl_batch_set_tiles(efl_batch* b, int32_t config) {
    if (!b || config < -1 || config >= kBatchConfigs) return batch_err(b, EFL_ERR_INVALID_ARGUMENT, "bad tile configuration");
    b->tile_fixed = config;
    return EFL_OK;
}

efl_status efl_batch_tiles(const efl_batch* b, int32_t* tx, int32_t* ty, int32_t* k, double* ns_per_cell_iteration) {
    if (!b) return batch_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null batch");
    const int ci = b->tile_fixed >= 0 ? b->tile_fixed : (b->tile_cfg >= 0 ? b->tile_cfg : -1);
    const BatchTileConfig* c = ci >= 0 ? &batch_configs(ci) : nullptr;
    if (tx) *tx = c ? c->tx : 0;
    if (ty) *ty = c ? c->ty : 0;
    if (k) *k = c ? c->k : 0;
    if (ns_per_cell_iteration)
        for (int i = 0; i < kBatchConfigs; ++i)
            ns_per_cell_iteration[i] = i < (int)b->tune_cost.size() ? b->tune_cost[i] : 0.0;
    return EFL_OK;
}

// Shelf packing of n images (wh[2 i] x wh[2 i + 1] pixels, multiples of 8) into one canvas: the width is the
// smallest multiple of 512 that holds the widest image (so that the three finer levels are multiples of 128
// wide); tallest images first, left to right with 8-pixel gaps, a new shelf 8 pixels below the tallest image
// of the last one.  Every rectangle starts on a multiple of 8, and none touches another.
efl_status efl_canvas_pack(const int32_t* wh, uint32_t n, int32_t* origins, int32_t* width, int32_t* height) {
    if (!wh || !origins || !width || !height) return EFL_ERR_INVALID_ARGUMENT;
    int maxw = 8;
    for (uint32_t i = 0; i < n; ++i) {
        if (wh[2 * i] <= 0 || wh[2 * i + 1] <= 0 || wh[2 * i] % 8 || wh[2 * i + 1] % 8 || wh[2 * i] > (1 << 16) ||
            wh[2 * i + 1] > (1 << 16))
            return EFL_ERR_INVALID_ARGUMENT;
        maxw = std::max(maxw, (int)wh[2 * i]);
    }
    const int W = (maxw + 511) / 512 * 512;
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) {
        return wh[2 * a + 1] != wh[2 * c + 1] ? wh[2 * a + 1] > wh[2 * c + 1] : wh[2 * a] > wh[2 * c];
    });
    long long x = 0, y = 0, shelf = 0;
    for (uint32_t i : order) {
        const int w = wh[2 * i], h = wh[2 * i + 1];
        if (x > 0 && x + w > W) {
            y += shelf + 8;
            x = 0;
            shelf = 0;
        }
        if (y + h > (1 << 20)) return EFL_ERR_INVALID_ARGUMENT;
        origins[2 * i] = (int32_t)x;
        origins[2 * i + 1] = (int32_t)y;
        x += w + 8;
        shelf = std::max<long long>(shelf, h);
    }
    *width = W;
    *height = (int32_t)(y + shelf);
    return EFL_OK;
}

// Lays the batch's simulations out on a canvas for the network's forward pass (see efl_canvas_pack) and
// allocates its activations and gap masks.  Leaves the batch without a canvas (each simulation's forward
// then runs on its own) where the coarsening is 1 or a simulation's coarse grid is not a multiple of 8 in
// both directions.
efl_status canvas_setup(efl_batch* b, const efl_unet* u) {
    canvas_free(b);
    b->gc.clear();  // captured stages before the solve may hold the previous canvas
    const int f = u->net.coarse;
    const size_t n = b->sims.size();
    if (f <= 1 || n == 0) return EFL_OK;
    std::vector<int32_t> wh(2 * n), org(2 * n);
    for (size_t i = 0; i < n; ++i) {
        const efl_sim* s = b->sims[i];
        if (s->nx % (8 * f) || s->ny % (8 * f)) return EFL_OK;
        wh[2 * i] = s->nx / f;
        wh[2 * i + 1] = s->ny / f;
    }
    int32_t W = 0, H = 0;
    if (efl_canvas_pack(wh.data(), (uint32_t)n, org.data(), &W, &H) != EFL_OK) return EFL_OK;
    UNet* v = new UNet();
    if (unet_alloc_forward(*v, u->net, H * f, W * f, false) != cudaSuccess) {
        if (v->arena) cudaFree(v->arena);
        delete v;
        return EFL_ERR_OUT_OF_MEMORY;
    }
    b->canvas = v;
    size_t off[4], total = 0;
    for (int l = 0; l < 4; ++l) {
        off[l] = total;
        total += up256((size_t)(W >> l) * (H >> l));
    }
    std::vector<unsigned char> m(total, 0);
    for (size_t i = 0; i < n; ++i)
        for (int l = 0; l < 4; ++l) {
            const int x0 = org[2 * i] >> l, y0 = org[2 * i + 1] >> l, w = wh[2 * i] >> l, h = wh[2 * i + 1] >> l;
            for (int y = y0; y < y0 + h; ++y) std::memset(&m[off[l] + (size_t)y * (W >> l) + x0], 1, (size_t)w);
        }
    if (cudaMalloc(&b->d_gaps, total) != cudaSuccess ||
        cudaMemcpy(b->d_gaps, m.data(), total, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&b->d_warm, n * sizeof(WarmSim)) != cudaSuccess ||
        cudaMalloc(&b->d_warm_start, (n + 1) * sizeof(int)) != cudaSuccess) {
        canvas_free(b);
        return EFL_ERR_OUT_OF_MEMORY;
    }
    for (int l = 0; l < 4; ++l) b->gaps[l] = b->d_gaps + off[l];
    b->cw = W;
    b->ch = H;
    b->corigin.resize(n);
    for (size_t i = 0; i < n; ++i) b->corigin[i] = make_int2(org[2 * i], org[2 * i + 1]);
    b->canvas_net = u;
    return EFL_OK;
}

// The warm-start descriptors of the simulations `on` (on the canvas), uploaded when the simulations or their
// time step differ from the last upload's (the batch stream drained first: a replayed graph may still read the
// old descriptors).  Everything else they hold is fixed from efl_batch_attach_unet on.
efl_status warm_upload(efl_batch* b, const std::vector<int>& on) {
    const int n = (int)on.size();
    std::vector<int> key(on);
    for (int i : on) {
        uint32_t dtb;
        std::memcpy(&dtb, &b->sims[i]->U.dt, 4);
        key.push_back((int)dtb);
    }
    if ((int)b->h_warm.size() == n && b->h_warm_start.size() == key.size() + (size_t)(n + 1) &&
        std::equal(key.begin(), key.end(), b->h_warm_start.begin() + (n + 1)))
        return EFL_OK;
    std::vector<WarmSim> hw(n);
    std::vector<int> st(n + 1, 0);
    for (int k = 0; k < n; ++k) {
        efl_sim* s = b->sims[on[k]];
        const UNet& v = *s->unet_view;
        WarmSim& w = hw[k];
        w.a = unet_feature_args(s);
        w.sigma = v.sigma;
        w.mask = v.mask;
        w.epart = v.epart;
        const size_t off = ((size_t)b->corigin[on[k]].y * b->cw + b->corigin[on[k]].x) * 16;
        w.outc = b->canvas->out + off;
        w.cs = b->cw;
        w.f = v.coarse;
        const dim3 fg = grid2d(s->nx, s->ny, kBlock);
        w.fgx = (int)fg.x;
        w.fgy = (int)fg.y;
        st[k + 1] = st[k] + w.fgx * w.fgy;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess ||
        cudaMemcpy(b->d_warm, hw.data(), n * sizeof(WarmSim), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_warm_start, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return EFL_ERR_CUDA;
    b->h_warm = hw;
    st.insert(st.end(), key.begin(), key.end());
    b->h_warm_start = st;
    return EFL_OK;
}

efl_status efl_batch_attach_unet(efl_batch* b, efl_unet* u, uint32_t flags) {
    if (!b) return batch_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null batch");
    if (flags & ~(uint32_t)EFL_UNET_WARM_START)
        return batch_err(b, EFL_ERR_INVALID_ARGUMENT, "a batch takes EFL_UNET_WARM_START only (record on a single "
                                                      "simulation)");
    cudaSetDevice(b->device);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return batch_err(b, EFL_ERR_CUDA, "batch stream failed");
    for (efl_sim* s : b->sims) {
        if (efl_unet_attach(s, flags ? u : nullptr, flags) != EFL_OK)
            return batch_err(b, EFL_ERR_INVALID_ARGUMENT, std::string("attach: ") + efl_unet_last_error(u));
        if (!flags || !u) continue;
        if (s->unet_view && s->unet_view->coarse != u->net.coarse) {  // sized for another coarsening
            cudaFree(s->unet_view->arena);
            delete s->unet_view;
            s->unet_view = nullptr;
        }
        if (!s->unet_view) {
            UNet* v = new UNet();
            if (unet_alloc_forward(*v, u->net, s->ny, s->nx) != cudaSuccess) {
                if (v->arena) cudaFree(v->arena);
                delete v;
                return batch_err(b, EFL_ERR_OUT_OF_MEMORY, "network workspace allocation failed");
            }
            s->unet_view = v;
        }
    }
    if (!flags || !u) {
        canvas_free(b);
        b->gc.clear();
        return EFL_OK;
    }
    const efl_status cs = canvas_setup(b, u);
    return cs == EFL_OK ? EFL_OK : batch_err(b, cs, "network canvas allocation failed");
}

efl_status efl_batch_unet_canvas(const efl_batch* b, int32_t* width, int32_t* height) {
    if (!b || !width || !height) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null argument");
    *width = b->canvas ? b->cw : 0;
    *height = b->canvas ? b->ch : 0;
    return EFL_OK;
}

efl_status efl_batch_set_wait_limits(efl_batch* b, uint64_t barrier_polls) {
    if (!b) return set_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null batch");
    if (barrier_polls > ((uint64_t)1 << 40)) return batch_err(b, EFL_ERR_INVALID_ARGUMENT, "wait limit above 2^40 polls");
    b->spin_limit = (long long)barrier_polls;
    return EFL_OK;
}

efl_status efl_batch_projection_ms(efl_batch* b, float* ms) {
    if (!b || !ms) return batch_err(b, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (!b->timed) return batch_err(b, EFL_ERR_STATE, "no batched solve has run yet");
    if (cudaEventSynchronize(b->ev[1]) != cudaSuccess || cudaEventElapsedTime(ms, b->ev[0], b->ev[1]) != cudaSuccess)
        return batch_err(b, EFL_ERR_CUDA, "event timing failed");
    return EFL_OK;
}

efl_status efl_batch_step(efl_batch* b, float dt, efl_step_stats* stats) {
    if (!b) return batch_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null batch");
    cudaSetDevice(b->device);
    const size_t n = b->sims.size();
    for (size_t i = 0; i < n; ++i) init_stats(stats ? &stats[i] : nullptr);
    std::vector<int> solve_batched;
    std::vector<char> init_only(n, 0);
    efl_status ret = EFL_OK;
    auto fail = [&](efl_sim* s, efl_status st) { return batch_err(b, st, s->err); };
    // Common case: every simulation initialised and solved by the batched
    // solve.  The stages before and after it then run as two segments over
    // all simulations (CUDA graphs once their arguments repeat).
    bool fast = true;
    for (size_t i = 0; i < n && fast; ++i) {
        const efl_sim* s = b->sims[i];
        const efl_projection& P = s->cfg.projection;
        const efl_projection& Q = b->sims[0]->cfg.projection;
        fast = s->status != 0 && P.method == EFL_PROJECTION_GAUSS_SEIDEL && P.tolerance > 0.0f &&
               P.tolerance == Q.tolerance && P.max_iterations == Q.max_iterations &&
               P.check_interval == Q.check_interval;
    }
    if (fast) {
        uint64_t sig_pre = 1469598103934665603ull, sig_post = sig_pre;
        for (efl_sim* s : b->sims) {
            s->U.dt = dt;
            sig_pre = fnv(sig_pre, segment_sig(s, SEG_PRE));
            sig_post = fnv(sig_post, segment_sig(s, SEG_POST));
        }
        // With a canvas, each simulation on it writes its features into its rectangle on its own stream (where
        // those small kernels overlap the other simulations' stages), one forward pass over the canvas follows
        // on the batch stream, and the guard and the application run as one launch each for all of them; the
        // others run their own warm start.
        auto on_canvas = [&](const efl_sim* s) {
            return b->canvas && s->unet == b->canvas_net && (s->unet_flags & EFL_UNET_WARM_START);
        };
        std::vector<int> on;
        for (size_t i = 0; i < n; ++i)
            if (on_canvas(b->sims[i])) on.push_back((int)i);
        if (!on.empty() && warm_upload(b, on) != EFL_OK)
            return batch_err(b, EFL_ERR_CUDA, "warm-start descriptor upload failed");
        sig_pre = fnv(sig_pre, (uint64_t)(uintptr_t)b->canvas);
        for (int i : on) sig_pre = fnv(sig_pre, (uint64_t)i);
        efl_status st = run_segment(b->gc, b->stream, sig_pre | 1, SEG_PRE, [&]() -> efl_status {
            TRY(batch_fanout(b, [&](size_t i, efl_sim* s) -> efl_status {
                TRY(run_stages(s, EFL_STAGE_UPDATE_SOLID, EFL_STAGE_DIVERGENCE, nullptr));
                if (on_canvas(s))  // its residual kernel widens p and b
                    return unet_features(s, b->canvas->X0 + ((size_t)b->corigin[i].y * b->cw + b->corigin[i].x) * 16,
                                         b->cw, true);
                if (s->unet && (s->unet_flags & EFL_UNET_WARM_START)) return unet_before_solve(s, true);
                const Level64& L = s->mg64[0];
                k_widen<<<grid2d(s->nx, s->ny, kBlock), kBlock, count_launch(), s->stream>>>(s->p0, s->div, L.x, L.b);
                return EFL_OK;
            }));
            if (on.empty()) return EFL_OK;
            for (int i : on)
                if (b->sims[i]->unet_view->coarse != b->canvas_net->net.coarse)
                    return set_err(b->sims[i], EFL_ERR_STATE,
                                   "the network's coarsening changed after efl_batch_attach_unet: attach again");
            const int m = (int)on.size(), nblk = b->h_warm_start[m];  // thread blocks over all their cells
            const WarmSim* W = b->d_warm;
            const int* S = b->d_warm_start;
            unet_forward(*b->canvas, b->ch, b->cw, b->stream, b->gaps);
            k_warm_batch_guard_residual<<<nblk, kBlock, count_launch(), b->stream>>>(W, S, m);
            k_warm_batch_guard<<<m, UNET_RED_THREADS, count_launch(), b->stream>>>(W);
            k_warm_batch_apply<<<nblk, kBlock, count_launch(), b->stream>>>(W, S, m);
            return cudaGetLastError() == cudaSuccess ? EFL_OK : EFL_ERR_CUDA;
        });
        if (st != EFL_OK) return batch_err(b, st, "batched stages before the solve failed");
        std::vector<int> all(n);
        for (size_t i = 0; i < n; ++i) all[i] = (int)i;
        std::vector<efl_step_stats> local;
        if (!stats) {
            local.resize(n);
            for (auto& x : local) init_stats(&x);
        }
        efl_step_stats* sp = stats ? stats : local.data();
        st = batch_solve(b, all, sp);
        if (st != EFL_OK) return st;
        for (size_t i = 0; i < n; ++i)
            if (!sp[i].converged) ret = EFL_NOT_CONVERGED;
        st = run_segment(b->gc, b->stream, sig_post | 1, SEG_POST, [&]() -> efl_status {
            return batch_fanout(b, [&](size_t, efl_sim* s) -> efl_status {
                k_narrow<<<grid2d(s->nx, s->ny, kBlock), kBlock, count_launch(), s->stream>>>(s->mg64[0].x, s->p0);
                return run_stages(s, EFL_STAGE_SOLVE_VELOCITY, EFL_STAGE_SOLID_FORCES, nullptr);
            });
        });
        if (st != EFL_OK) return batch_err(b, st, "batched stages after the solve failed");
        for (efl_sim* s : b->sims) s->n_forces = 0;
        if (cudaGetLastError() != cudaSuccess) return batch_err(b, EFL_ERR_CUDA, "batch step launch failed");
        return ret;
    }
    for (size_t i = 0; i < n; ++i) {
        efl_sim* s = b->sims[i];
        if (s->status == 0) {
            efl_status st = run_init(s);
            if (st != EFL_OK) return fail(s, st);
            s->status = 1;
            init_only[i] = 1;
            if (stats) stats[i].initialized_only = 1;
            continue;
        }
        s->U.dt = dt;
        for (int stage = EFL_STAGE_UPDATE_SOLID; stage <= EFL_STAGE_DIVERGENCE; ++stage) {
            efl_status st = run_stage(s, stage, stats ? &stats[i] : nullptr);
            if (st != EFL_OK) return fail(s, st);
        }
        const efl_projection& P = s->cfg.projection;
        const efl_projection& Q = b->sims[solve_batched.empty() ? i : solve_batched[0]]->cfg.projection;
        const bool batchable = P.method == EFL_PROJECTION_GAUSS_SEIDEL && P.tolerance > 0.0f &&
                               P.tolerance == Q.tolerance && P.max_iterations == Q.max_iterations &&
                               P.check_interval == Q.check_interval;
        if (batchable) {
            const Level64& L = s->mg64[0];
            if (s->unet && (s->unet_flags & EFL_UNET_WARM_START)) {
                efl_status st = unet_before_solve(s, true);  // its residual kernel widens p and b
                if (st != EFL_OK) return fail(s, st);
            } else {
                k_widen<<<grid2d(s->nx, s->ny, kBlock), kBlock, count_launch(), s->stream>>>(s->p0, s->div, L.x, L.b);
            }
            solve_batched.push_back((int)i);
        } else {
            efl_status st = run_stage(s, EFL_STAGE_PROJECTION, stats ? &stats[i] : nullptr);
            if (st == EFL_NOT_CONVERGED) ret = st;
            else if (st != EFL_OK) return fail(s, st);
        }
    }
    std::vector<efl_step_stats> local;
    if (!stats) {
        local.resize(n);
        for (auto& x : local) init_stats(&x);
    }
    efl_step_stats* sp = stats ? stats : local.data();
    efl_status st = batch_solve(b, solve_batched, sp);
    if (st != EFL_OK) return st;
    for (int idx : solve_batched) {
        efl_sim* s = b->sims[idx];
        k_narrow<<<grid2d(s->nx, s->ny, kBlock), kBlock, count_launch(), s->stream>>>(s->mg64[0].x, s->p0);
        if (!sp[idx].converged) ret = EFL_NOT_CONVERGED;
    }
    for (size_t i = 0; i < n; ++i) {
        efl_sim* s = b->sims[i];
        if (init_only[i]) continue;
        for (int stage = EFL_STAGE_SOLVE_VELOCITY; stage <= EFL_STAGE_SOLID_FORCES; ++stage) {
            efl_status st2 = run_stage(s, stage, nullptr);
            if (st2 != EFL_OK) return fail(s, st2);
        }
        s->n_forces = 0;
    }
    if (cudaGetLastError() != cudaSuccess) return batch_err(b, EFL_ERR_CUDA, "batch step launch failed");
    return ret;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The learned warm start's network.

namespace {
std::string g_unet_error;
efl_status unet_err(efl_unet* u, efl_status st, const std::string& m) {
    if (u) u->net.last_error = m;
    else g_unet_error = m;
    return st;
}
// Sets up the kernels' shared-memory limits once per device.
bool unet_kernel_attrs() {
    return cudaFuncSetAttribute(k_conv3x3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM) == cudaSuccess &&
           cudaFuncSetAttribute(k_conv3x3_rows<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_conv3x3_rows<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_conv3x3_rows<true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_conv3x3_rows<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, CV_SMEM) ==
               cudaSuccess &&
           conv_sm_count_init() &&
           cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, WG_SMEM) == cudaSuccess;
}
efl_status unet_finish(efl_unet* u, cudaStream_t st) {
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, std::string("network kernels failed: ") + cudaGetErrorString(cudaGetLastError()));
    int e = 0;
    cudaMemcpy(&e, u->net.err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e) {
        cudaMemset(u->net.err, 0, sizeof(int));
        return unet_err(u, EFL_ERR_CUDA, "a tensor-core MMA did not complete (bounded wait gave up)");
    }
    return EFL_OK;
}
__global__ void k_f32_to_bf16(const float* a, size_t n, bf16* b) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}
__global__ void k_copy_f32(const float* a, size_t n, size_t stride, float* b) {  // channel 0 of [n][stride]
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i * stride];
}
// Loss on the sample in X0/target/mask (relative squared error, see
// k_unet_loss); fills g_out and the parameter gradients.
efl_status unet_loss_and_grads(efl_unet* u, int H, int W, cudaStream_t st, float* loss) {
    UNet& n = u->net;
    const int npix = H * W, blocks = (npix + 1023) / 1024;
    std::vector<float2> part(blocks);
    const float* target = u->rec_coarse ? n.targetc : n.target;
    const unsigned char* mask = u->rec_coarse ? n.maskc : n.mask;
    k_target_stats<<<blocks, 256, count_launch(), st>>>(target, mask, npix, 1024, n.lpart);
    cudaMemcpyAsync(part.data(), n.lpart, blocks * sizeof(float2), cudaMemcpyDeviceToHost, st);
    unet_forward(n, H, W, st);
    TRY_U(unet_finish(u, st));
    double t2 = 0.0;
    for (auto& q : part) t2 += q.y;
    const float inv = t2 > 0.0 ? (float)(1.0 / t2) : 0.0f;
    k_unet_loss<<<blocks, 256, count_launch(), st>>>(n.out, target, mask, npix, 1024, inv, n.g_out, n.lpart);
    unet_backward(n, H, W, st);
    cudaMemcpyAsync(part.data(), n.lpart, blocks * sizeof(float2), cudaMemcpyDeviceToHost, st);
    TRY_U(unet_finish(u, st));
    double se = 0.0;
    for (auto& q : part) se += q.x;
    *loss = (float)(se * (double)inv);
    return EFL_OK;
}
}  // namespace

extern "C" {

efl_status efl_unet_create(int32_t device, uint32_t max_nx, uint32_t max_ny, uint64_t seed, efl_unet** out) {
    if (!out) return unet_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (max_nx < 16 || max_ny < 16 || max_nx % 8 || max_ny % 8 || max_nx > 4096 || max_ny > 4096)
        return unet_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "network grid must be a multiple of 8 in [16, 4096]");
    if (cudaSetDevice(device) != cudaSuccess) return unet_err(nullptr, EFL_ERR_NO_DEVICE, "no such CUDA device");
    if (!unet_kernel_attrs()) return unet_err(nullptr, EFL_ERR_CUDA, "tensor-core kernels unavailable on this device");
    efl_unet* u = new efl_unet();
    u->net.device = device;
    if (unet_alloc(u->net, (int)max_ny, (int)max_nx) != cudaSuccess) {
        if (u->net.arena) cudaFree(u->net.arena);
        delete u;
        return unet_err(nullptr, EFL_ERR_OUT_OF_MEMORY, "network allocation failed");
    }
    // He-normal weights for the ReLU layers, a zero head (the warm start
    // begins as the previous pressure), zero biases.
    std::vector<float> h(u->net.nparams, 0.0f);
    std::mt19937_64 rng(seed);
    for (int i = 0; i < UNET_NCONV; ++i) {
        if (!kUnetSpec[i].relu) continue;
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * kUnetSpec[i].cin)));
        for (size_t k = 0; k < (size_t)9 * kUnetSpec[i].cin * kUnetSpec[i].cout; ++k) h[u->net.woff[i] + k] = nd(rng);
    }
    cudaMemcpy(u->net.params, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
    unet_sync_weights(u->net, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cudaFree(u->net.arena);
        delete u;
        return unet_err(nullptr, EFL_ERR_CUDA, "network initialisation failed");
    }
    *out = u;
    return EFL_OK;
}

efl_status efl_unet_destroy(efl_unet* u) {
    if (!u) return EFL_OK;
    cudaSetDevice(u->net.device);
    cudaDeviceSynchronize();
    cudaFree(u->net.arena);
    delete u;
    return EFL_OK;
}

const char* efl_unet_last_error(const efl_unet* u) { return u ? u->net.last_error.c_str() : g_unet_error.c_str(); }

efl_status efl_unet_num_params(const efl_unet* u, uint64_t* n) {
    if (!u || !n) return unet_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null argument");
    *n = u->net.nparams;
    return EFL_OK;
}

efl_status efl_unet_get_params(efl_unet* u, float* host, uint64_t n) {
    if (!u || !host || n != u->net.nparams) return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "bad parameter buffer");
    cudaSetDevice(u->net.device);
    if (cudaMemcpy(host, u->net.params, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, "copy failed");
    return EFL_OK;
}

efl_status efl_unet_set_params(efl_unet* u, const float* host, uint64_t n) {
    if (!u || !host || n != u->net.nparams) return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "bad parameter buffer");
    cudaSetDevice(u->net.device);
    if (cudaMemcpy(u->net.params, host, n * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, "copy failed");
    unet_sync_weights(u->net, 0);
    cudaMemset(u->net.adam_m, 0, n * 4);
    cudaMemset(u->net.adam_v, 0, n * 4);
    u->net.adam_t = 0;
    return unet_finish(u, 0);
}

// Host features [ny][nx][16] into X0 (the network's input).
static efl_status unet_upload_features(efl_unet* u, uint32_t nx, uint32_t ny, const float* features) {
    UNet& n = u->net;
    if (nx < 16 || ny < 16 || nx % 8 || ny % 8 || (int)nx > n.maxW || (int)ny > n.maxH)
        return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "grid larger than the network was created for, or not a multiple of 8");
    const size_t cnt = (size_t)nx * ny * 16;
    if (cudaMemcpy(n.g_out, features, cnt * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, "copy failed");
    k_f32_to_bf16<<<lin_grid(cnt), 256, count_launch(), 0>>>(n.g_out, cnt, n.X0);
    return EFL_OK;
}

efl_status efl_unet_forward(efl_unet* u, uint32_t nx, uint32_t ny, const float* features, float* pred) {
    if (!u || !features || !pred) return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(u->net.device);
    TRY_U(unet_upload_features(u, nx, ny, features));
    unet_forward(u->net, (int)ny, (int)nx, 0);
    const size_t np = (size_t)nx * ny;
    k_copy_f32<<<lin_grid(np), 256, count_launch(), 0>>>(u->net.out, np, 16, u->net.target);
    TRY_U(unet_finish(u, 0));
    if (cudaMemcpy(pred, u->net.target, np * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, "copy failed");
    return EFL_OK;
}

efl_status efl_unet_gradients(efl_unet* u, uint32_t nx, uint32_t ny, const float* features, const float* target,
                              const uint8_t* mask, float* loss, float* grads) {
    if (!u || !features || !target || !mask || !loss || !grads)
        return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(u->net.device);
    TRY_U(unet_upload_features(u, nx, ny, features));
    const size_t np = (size_t)nx * ny;
    cudaMemcpy(u->net.target, target, np * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(u->net.mask, mask, np, cudaMemcpyHostToDevice);
    TRY_U(unet_loss_and_grads(u, (int)ny, (int)nx, 0, loss));
    if (cudaMemcpy(grads, u->net.grads, u->net.nparams * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, "copy failed");
    return EFL_OK;
}

efl_status efl_unet_time_forward(efl_unet* u, uint32_t nx, uint32_t ny, uint32_t reps, float* ms) {
    if (!u || !ms || !reps) return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (nx < 16 || ny < 16 || nx % 8 || ny % 8 || (int)nx > u->net.maxW || (int)ny > u->net.maxH)
        return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "bad grid");
    cudaSetDevice(u->net.device);
    cudaStream_t sm = nullptr;
    if (cudaStreamCreateWithFlags(&sm, cudaStreamNonBlocking) != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, "stream creation failed");
    unet_forward(u->net, (int)ny, (int)nx, sm);  // warm-up
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool captured = cudaStreamBeginCapture(sm, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (captured) {
        unet_forward(u->net, (int)ny, (int)nx, sm);
        captured = cudaStreamEndCapture(sm, &graph) == cudaSuccess && graph &&
                   cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    }
    efl_status st = EFL_OK;
    float t = 0.0f;
    if (captured) {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaGraphLaunch(exec, sm);  // warm-up replay
        cudaEventRecord(e0, sm);
        for (uint32_t i = 0; i < reps; ++i) cudaGraphLaunch(exec, sm);
        cudaEventRecord(e1, sm);
        st = unet_finish(u, sm);
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    } else {
        st = unet_err(u, EFL_ERR_CUDA, "graph capture of the forward pass failed");
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamSynchronize(sm);
    cudaStreamDestroy(sm);
    *ms = t / (float)reps;
    return st;
}

efl_status efl_unet_attach(efl_sim* s, efl_unet* u, uint32_t flags) {
    if (!s) return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "null sim");
    if (u && (s->nx > u->net.maxW || s->ny > u->net.maxH || s->cfg.device != u->net.device))
        return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "simulation larger than the network, or on another device");
    if (u && flags && (s->nx % (8 * u->net.coarse) || s->ny % (8 * u->net.coarse)))
        return unet_err(u, EFL_ERR_INVALID_ARGUMENT,
                        "grid size must be a multiple of 8 x the network's coarsening factor");
    if (s->unet_view && (!u || flags == 0 || s->unet != u)) {  // the workspace belonged to the previous network
        cudaStreamSynchronize(s->stream);
        cudaFree(s->unet_view->arena);
        delete s->unet_view;
        s->unet_view = nullptr;
    }
    s->unet = flags ? u : nullptr;
    s->unet_flags = u ? flags : 0;
    ++s->graph_epoch;  // captured segments hold the previous network's launches
    return EFL_OK;
}

efl_status efl_unet_set_coarsening(efl_unet* u, uint32_t factor) {
    if (!u) return unet_err(nullptr, EFL_ERR_INVALID_ARGUMENT, "null network");
    if (factor != 1 && factor != 2 && factor != 4 && factor != 8)
        return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "coarsening factor must be 1, 2, 4 or 8");
    u->net.coarse = (int)factor;
    u->rec_nx = u->rec_ny = 0;  // a recorded sample of the other form is void
    return EFL_OK;
}

efl_status efl_unet_train_step(efl_unet* u, float lr, float* loss) {
    if (!u || !loss) return unet_err(u, EFL_ERR_INVALID_ARGUMENT, "null argument");
    if (!u->rec_nx) return unet_err(u, EFL_ERR_STATE, "no training sample recorded (attach with EFL_UNET_RECORD and step)");
    cudaSetDevice(u->net.device);
    UNet& n = u->net;
    // The sample was written on the simulation's stream: wait for it.
    if (cudaDeviceSynchronize() != cudaSuccess)
        return unet_err(u, EFL_ERR_CUDA, std::string("device error: ") + cudaGetErrorString(cudaGetLastError()));
    TRY_U(unet_loss_and_grads(u, u->rec_ny, u->rec_nx, 0, loss));
    // Global-norm clip at 1 (a sample far from the network's range would
    // otherwise inflate Adam's second moments for thousands of steps).
    const int nb = (int)((n.nparams + 1023) / 1024);
    k_sumsq<<<nb, 256, count_launch(), 0>>>(n.grads, (int)n.nparams, n.wpart);
    std::vector<float> part(nb);
    cudaMemcpy(part.data(), n.wpart, nb * sizeof(float), cudaMemcpyDeviceToHost);
    double g2 = 0.0;
    for (float q : part) g2 += q;
    const double gn = std::sqrt(g2);
    const float gscale = (gn > 1.0 && std::isfinite(gn)) ? (float)(1.0 / gn) : (std::isfinite(gn) ? 1.0f : 0.0f);
    ++n.adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)n.adam_t), c2 = 1.0f - std::pow(b2, (float)n.adam_t);
    k_adam<<<lin_grid(n.nparams), 256, count_launch(), 0>>>(n.params, n.grads, n.adam_m, n.adam_v, (int)n.nparams,
                                                             lr, b1, b2, 1e-8f, c1, c2, gscale);
    unet_sync_weights(n, 0);
    return unet_finish(u, 0);
}

}  // extern "C"

// ---- Row slabs of one domain ----------------------------------------------

struct efl_slab {
    efl_slab_desc desc{};
    SlabPlanes S{};
    cudaStream_t stream = nullptr;
    void* block = nullptr;  // every plane, one allocation
    double* h_part = nullptr;
};

namespace {

efl_status slab_free(efl_slab* sl) {
    if (!sl) return EFL_OK;
    cudaSetDevice(sl->desc.device);
    if (sl->stream) cudaStreamSynchronize(sl->stream);
    if (sl->block) cudaFree(sl->block);
    if (sl->h_part) cudaFreeHost(sl->h_part);
    if (sl->stream) cudaStreamDestroy(sl->stream);
    delete sl;
    return EFL_OK;
}

efl_status slab_finish(efl_slab* sl) {
    efl_sim* s = nullptr;
    LAUNCH_CHECK();
    CU(cudaStreamSynchronize(sl->stream));
    return EFL_OK;
}

}  // namespace

extern "C" {

efl_status efl_slab_create(const efl_slab_desc* d, efl_slab** out) {
    efl_sim* s = nullptr;  // errors go to efl_last_error(NULL)
    if (!d || !out) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_create: null argument");
    *out = nullptr;
    if (d->nx == 0 || d->ny == 0 || d->rows == 0 || (uint64_t)d->row0 + d->rows > d->ny)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_create: rows [%u, %u) outside a grid of %u rows",
                       d->row0, d->row0 + d->rows, d->ny);
    if ((uint64_t)d->nx * (d->rows + 2) > (1ull << 31))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_create: slab of %u x %u cells too large", d->nx,
                       d->rows);
    if (!(d->dx > 0.0f) || !(d->dt > 0.0f) || !(d->rho > 0.0f) || !(d->sor_weight > 0.0f && d->sor_weight < 2.0f))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_create: dx, dt, rho must be > 0 and sor_weight in (0, 2)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err(s, EFL_ERR_NO_DEVICE, "efl_slab_create: no CUDA device");
    if (d->device < 0 || d->device >= ndev)
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_create: device %d of %d", d->device, ndev);
    CU(cudaSetDevice(d->device));
    efl_slab* sl = new efl_slab();
    sl->desc = *d;
    SlabPlanes& S = sl->S;
    S.nx = (int)d->nx;
    S.ny = (int)d->ny;
    S.row0 = (int)d->row0;
    S.rows = (int)d->rows;
    const size_t hal = (size_t)S.nx * (S.rows + 2), own = (size_t)S.nx * S.rows;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t sizes[] = {al(hal * 8), al(hal * 4), al(hal * 4), al(own * 16), al(own * 8), al(own * 4),
                            al(own * 16), al(own * 4), al(own * 8), al(own), al((size_t)S.rows * 16)};
    size_t total = 0;
    for (size_t z : sizes) total += z;
    cudaError_t e = cudaMalloc(&sl->block, total);
    if (e == cudaSuccess) e = cudaMemset(sl->block, 0, total);  // halo rows beyond the domain stay zero
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&sl->h_part, (size_t)S.rows * 16);
    if (e != cudaSuccess) {
        slab_free(sl);
        return set_err(s, e == cudaErrorMemoryAllocation ? EFL_ERR_OUT_OF_MEMORY : EFL_ERR_CUDA,
                       "efl_slab_create: %s", cudaGetErrorString(e));
    }
    char* p = (char*)sl->block;
    auto take = [&](int i) {
        char* q = p;
        p += sizes[i];
        return q;
    };
    S.x = (double*)take(0);
    S.d = (float*)take(1);
    S.ls = (float*)take(2);
    S.af = (float4*)take(3);
    S.b = (double*)take(4);
    S.rc = (float*)take(5);
    S.w = (float4*)take(6);
    S.inv = (float*)take(7);
    S.den = (double*)take(8);
    S.mode = (unsigned char*)take(9);
    S.rowpart = (double2*)take(10);
    *out = sl;
    return EFL_OK;
}

efl_status efl_slab_destroy(efl_slab* sl) { return slab_free(sl); }

efl_status efl_slab_load(efl_slab* sl, const float* ls, const float* af, const float* div, const float* p) {
    efl_sim* s = nullptr;
    if (!sl || !ls || !af || !div || !p) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_load: null argument");
    CU(cudaSetDevice(sl->desc.device));
    SlabPlanes& S = sl->S;
    const size_t own = (size_t)S.nx * S.rows;
    // The f32 pressure and divergence rows go through the (not yet built) coefficient planes as staging.
    CU(cudaMemcpyAsync(S.ls + S.nx, ls, own * 4, cudaMemcpyDefault, sl->stream));
    CU(cudaMemcpyAsync(S.af, af, own * 16, cudaMemcpyDefault, sl->stream));
    CU(cudaMemcpyAsync(S.rc, p, own * 4, cudaMemcpyDefault, sl->stream));
    CU(cudaMemcpyAsync(S.inv, div, own * 4, cudaMemcpyDefault, sl->stream));
    k_slab_widen<<<grid2d(S.nx, S.rows, kBlock), kBlock, count_launch(), sl->stream>>>(S, S.rc, S.inv);
    return slab_finish(sl);
}

efl_status efl_slab_halo(efl_slab* sl, int32_t field, int32_t side, int32_t write, void* buf) {
    efl_sim* s = nullptr;
    if (!sl || !buf) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_halo: null argument");
    if (field < EFL_SLAB_X || field > EFL_SLAB_LEVELSET || (side != 0 && side != 1) || (write != 0 && write != 1))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_halo: field %d, side %d, write %d", field, side, write);
    SlabPlanes& S = sl->S;
    if (write && ((side == 0 && S.row0 == 0) || (side == 1 && S.row0 + S.rows == S.ny)))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_halo: no halo row beyond the domain's %s edge",
                       side == 0 ? "top" : "bottom");
    CU(cudaSetDevice(sl->desc.device));
    const size_t es = field == EFL_SLAB_X ? 8 : 4;
    char* base = field == EFL_SLAB_X ? (char*)S.x : field == EFL_SLAB_D ? (char*)S.d : (char*)S.ls;
    // halo plane rows: 0 = halo above, 1 .. rows = own, rows + 1 = halo below
    const int row = write ? (side == 0 ? 0 : S.rows + 1) : (side == 0 ? 1 : S.rows);
    char* dev = base + (size_t)row * S.nx * es;
    if (write) CU(cudaMemcpyAsync(dev, buf, (size_t)S.nx * es, cudaMemcpyDefault, sl->stream));
    else CU(cudaMemcpyAsync(buf, dev, (size_t)S.nx * es, cudaMemcpyDefault, sl->stream));
    CU(cudaStreamSynchronize(sl->stream));
    return EFL_OK;
}

efl_status efl_slab_prepare(efl_slab* sl) {
    efl_sim* s = nullptr;
    if (!sl) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_prepare: null slab");
    CU(cudaSetDevice(sl->desc.device));
    k_slab_coeffs<<<grid2d(sl->S.nx, sl->S.rows, kBlock), kBlock, count_launch(), sl->stream>>>(sl->S);
    return slab_finish(sl);
}

efl_status efl_slab_residual(efl_slab* sl, double* row_partials) {
    efl_sim* s = nullptr;
    if (!sl || !row_partials) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_residual: null argument");
    CU(cudaSetDevice(sl->desc.device));
    const efl_slab_desc& d = sl->desc;
    const double dx = (double)d.dx;
    const double cdiv = dx * dx * (double)d.rho / (double)d.dt;
    const double factor = (double)d.dt / (double)d.rho / dx / dx;
    k_slab_residual<<<sl->S.rows, kSlabRowThreads, count_launch(), sl->stream>>>(sl->S, factor, cdiv);
    LAUNCH_CHECK();
    CU(cudaMemcpyAsync(sl->h_part, sl->S.rowpart, (size_t)sl->S.rows * 16, cudaMemcpyDeviceToHost, sl->stream));
    CU(cudaStreamSynchronize(sl->stream));
    std::memcpy(row_partials, sl->h_part, (size_t)sl->S.rows * 16);
    return EFL_OK;
}

efl_status efl_slab_sweep(efl_slab* sl, int32_t color) {
    efl_sim* s = nullptr;
    if (!sl || (color != 0 && color != 1))
        return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_sweep: null slab or color %d", color);
    CU(cudaSetDevice(sl->desc.device));
    const SlabPlanes& S = sl->S;
    k_slab_sweep<<<grid2d((S.nx + 1) / 2, S.rows, kBlock), kBlock, count_launch(), sl->stream>>>(
        S, color, sl->desc.sor_weight);
    return slab_finish(sl);
}

efl_status efl_slab_apply(efl_slab* sl) {
    efl_sim* s = nullptr;
    if (!sl) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_apply: null slab");
    CU(cudaSetDevice(sl->desc.device));
    k_slab_apply<<<grid2d(sl->S.nx, sl->S.rows, kBlock), kBlock, count_launch(), sl->stream>>>(sl->S);
    return slab_finish(sl);
}

efl_status efl_slab_read(efl_slab* sl, double* x) {
    efl_sim* s = nullptr;
    if (!sl || !x) return set_err(s, EFL_ERR_INVALID_ARGUMENT, "efl_slab_read: null argument");
    CU(cudaSetDevice(sl->desc.device));
    const SlabPlanes& S = sl->S;
    CU(cudaMemcpyAsync(x, S.x + S.nx, (size_t)S.nx * S.rows * 8, cudaMemcpyDefault, sl->stream));
    CU(cudaStreamSynchronize(sl->stream));
    return EFL_OK;
}

}  // extern "C"
