// ctx.cu — the C ABI (include/sr_cuda.h): one context per world, owning its device buffers and one stream, and the
// step driver that runs the reference's pass order P1 → P2 → P4 → P5 → P8 → P9 (reference/mod.rs:264-297) as kernel
// launches on that stream. Δt lives on the device (the P9 → P1 hand-off never visits the host); the host reads back
// only at the end of sr_step (the non-finite guard) and in the report calls.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <string>
#include <vector>

#include "box.cuh"
#include "grav.cuh"
#include "heat.cuh"
#include "hydro.cuh"
#include "hydro_ref.cuh"
#include "learned.cuh"

#include <atomic>

namespace {
thread_local std::string g_create_error;
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void sr_set_global_error(const std::string& message) { g_create_error = message; }
void sr_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void sr_note_launches(long long n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long sr_launches() { return g_launches.load(std::memory_order_relaxed); }

struct sr_learner {
    Learner* L = nullptr;
    cudaStream_t stream = nullptr;  // training and weight uploads
};

struct sr_ctx {
    sr_config cfg{};
    HydroConst H{};
    int w = 0, h = 0;
    size_t n = 0;
    cudaStream_t stream = nullptr;
    float* U[2] = {nullptr, nullptr};
    int cur = 0;
    float *phi = nullptr, *gx = nullptr, *gy = nullptr;             // P2's field of the step's start state
    float *src = nullptr, *phim = nullptr, *gxm = nullptr, *gym = nullptr;  // the half step's source and field
    float* kappa = nullptr;
    // reference mode (14 channels)
    int nc = 4;                   // channels of the state
    RefConst R{};
    float* table = nullptr;       // the cold pressures' u(x) tables
    uint8_t* held = nullptr;      // the hold's mask
    float *src_free = nullptr, *phip = nullptr, *gxp = nullptr, *gyp = nullptr;  // the pull on the held cells
    float* push = nullptr;        // each cell's radiation push
    float *radx = nullptr, *rady = nullptr;  // the last P5's cell-centred flux, the next P4's radiation force
    double* rpart = nullptr;      // the reference-mode P4's per-CTA partials and their reduction
    float* rbest = nullptr;
    int* ridx = nullptr;
    double* rfin = nullptr;
    GravPlan grav;
    bool grav_ready = false;
    double* part_d = nullptr;
    float* part_best = nullptr;
    int* part_idx = nullptr;
    double* hreport = nullptr;  // 7 doubles
    int* herr = nullptr;        // the hydro kernels' error flag (a bounded wait gave up)
    DtRecord* rec = nullptr;
    float *part_rate = nullptr, *part_g = nullptr;
    long long* part_nf = nullptr;
    HeatSolver* heat = nullptr;
    sr_learner* learner = nullptr;  // attached learned preconditioner (not owned)
    sr_heat_report heat_report{};
    bool uploaded = false;
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};  // a whole step from state buffer 0 / 1, captured on first use
    long long step_launches = 0;
    unsigned generation = 0;  // counts the invalidations of captured steps (a batch's graph checks it)
    // the active box: the crop of the world's gas stepped as a world of its own (a context per box size met)
    bool use_box = false;
    BoxRec box{};                 // the box `sub` steps
    sr_ctx* sub = nullptr;        // the crop's context while the box is active
    std::vector<sr_ctx*> subs;    // the crop contexts made so far (owned)
    int* box_part = nullptr;      // the fit's per-CTA partials
    int* box_rec = nullptr;       // the fitted box (device)
    unsigned long long box_steps = 0;  // steps since the upload (or the restored step index): the refit cadence
    float* plane32 = nullptr;          // a W*H f32 staging plane (the rate's f32 form), made on first use
    unsigned long long box_fits = 0;
    // timing
    int timing = 0;  // 0 off; 1 each step's device time (captured steps); 2 per pass (passes launched one by one)
    std::vector<cudaEvent_t> events;
    sr_cost cost{};
    std::string error;
};

static void validate(const sr_config& c) {
    SR_REQUIRE(c.struct_size == sizeof(sr_config), "sr_config.struct_size does not match this library's sr_config");
    SR_REQUIRE(c.width >= 16 && c.width <= 4096 && c.width % 8 == 0,
               "world width must be a multiple of 8 in 16..4096 (got " + std::to_string(c.width) + ")");
    SR_REQUIRE(c.height >= 16 && c.height <= 4096 && c.height % 8 == 0,
               "world height must be a multiple of 8 in 16..4096 (got " + std::to_string(c.height) + ")");
    SR_REQUIRE(c.channels == 4 || c.channels == kRefChannels,
               "channels must be 4 (Σ, Σu, Σv, E) or 14 (reference mode: the ten mass fractions after them)");
    if (c.channels == kRefChannels) {
        SR_REQUIRE(!c.opacity_plane, "reference mode (14 channels) takes κ from each cell's species: no opacity plane");
        SR_REQUIRE(c.k1e >= 0.0 && c.k2e >= 0.0 && c.k1n >= 0.0 && c.k2n >= 0.0, "the cold pairs' K must be >= 0");
        SR_REQUIRE((c.k1e > 0.0) == (c.k2e > 0.0) && (c.k1n > 0.0) == (c.k2n > 0.0),
                   "a cold pair is on or off as a whole (k1e/k2e, k1n/k2n)");
        SR_REQUIRE(c.r_hold >= 0.0 && c.r_hold <= 64.0, "r_hold must be in 0..64 cells");
    }
    SR_REQUIRE(c.edge <= SR_EDGE_LEAVE, "unknown edge mode");
    SR_REQUIRE(c.limiter <= SR_LIMITER_MINMOD, "unknown limiter");
    SR_REQUIRE(c.kernel <= SR_KERNEL_SOFTENED, "unknown gravity kernel");
    SR_REQUIRE(c.precond <= SR_PRECOND_LEARNED, "unknown preconditioner");
    SR_REQUIRE(c.gamma > 1.0, "gamma must exceed 1");
    SR_REQUIRE(c.mu > 0.0, "mu must be positive");
    SR_REQUIRE(c.t_floor > 0.0, "t_floor must be positive");
    SR_REQUIRE(c.sigma_vac > 0.0 && c.sigma_floor > 0.0, "sigma_vac and sigma_floor must be positive");
    SR_REQUIRE(c.cfl > 0.0 && c.eta_g > 0.0, "cfl and eta_g must be positive");
    SR_REQUIRE(!(c.kernel == SR_KERNEL_SOFTENED && !(c.softening > 0.0)), "the softened kernel needs softening > 0");
    SR_REQUIRE(c.dt_fixed >= 0.0 && c.dt_cap >= 0.0, "dt_fixed and dt_cap must be >= 0");
}

static HydroConst hydro_const(const sr_config& c) {
    HydroConst H;
    H.w = (int)c.width;
    H.h = (int)c.height;
    H.edge = (int)c.edge;
    H.limiter = (int)c.limiter;
    H.bracket = (int)c.thermal_bracket;
    H.gamma = (float)c.gamma;
    H.gm1 = (float)(c.gamma - 1.0);
    H.inv_gm1 = (float)(1.0 / (c.gamma - 1.0));
    H.eps_floor = (float)(c.t_floor / c.mu / (c.gamma - 1.0));
    H.sigma_vac = (float)c.sigma_vac;
    H.sigma_floor = (float)c.sigma_floor;
    return H;
}

template <class T>
static void dalloc(T** p, size_t count) {
    SR_CUDA_TRY(cudaMalloc((void**)p, sizeof(T) * (count ? count : 1)));
    SR_CUDA_TRY(cudaMemset(*p, 0, sizeof(T) * (count ? count : 1)));
}

static void drop_step_graphs(sr_ctx* c) {
    c->generation++;
    for (auto& g : c->step_graph)
        if (g) {
            cudaStreamSynchronize(c->stream);
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

static void ctx_free(sr_ctx* c);

static void ctx_free(sr_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->U[0]);
    cudaFree(c->U[1]);
    cudaFree(c->phi); cudaFree(c->gx); cudaFree(c->gy);
    cudaFree(c->src); cudaFree(c->phim); cudaFree(c->gxm); cudaFree(c->gym);
    cudaFree(c->kappa);
    for (sr_ctx* s : c->subs) ctx_free(s);
    cudaFree(c->box_part); cudaFree(c->box_rec); cudaFree(c->plane32);
    cudaFree(c->table); cudaFree(c->held); cudaFree(c->src_free); cudaFree(c->phip); cudaFree(c->gxp);
    cudaFree(c->gyp); cudaFree(c->push); cudaFree(c->radx); cudaFree(c->rady); cudaFree(c->rpart); cudaFree(c->rbest); cudaFree(c->ridx); cudaFree(c->rfin);
    if (c->grav_ready) c->grav.destroy();
    cudaFree(c->part_d); cudaFree(c->part_best); cudaFree(c->part_idx); cudaFree(c->hreport); cudaFree(c->herr);
    cudaFree(c->rec); cudaFree(c->part_rate); cudaFree(c->part_g); cudaFree(c->part_nf);
    drop_step_graphs(c);
    if (c->heat) heat_destroy(c->heat);
    for (auto e : c->events) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// Runs `body`, turning an SrError or a CUDA error into a status and the context's message.
template <class F>
static sr_status guarded(sr_ctx* c, F body) {
    if (!c) return SR_E_INVALID;
    try {
        body();
        return SR_OK;
    } catch (const SrError& e) {
        c->error = e.message;
        return e.status;
    } catch (const std::exception& e) {
        c->error = e.what();
        return SR_E_CUDA;
    }
}

// The same for calls without a context (the message goes where sr_last_error(NULL) reads it).
template <class F>
static sr_status guarded_free(F body) {
    try {
        body();
        return SR_OK;
    } catch (const SrError& e) {
        g_create_error = e.message;
        return e.status;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return SR_E_CUDA;
    }
}

static float* planes(sr_ctx* c) { return c->U[c->cur]; }

static bool ref_mode(const sr_ctx* c) { return c->nc == kRefChannels; }

// Reference mode's constants, tables and buffers.
static void ref_setup(sr_ctx* c) {
    const sr_config& k = c->cfg;
    const size_t n = c->n;
    RefConst& R = c->R;
    R.w = c->w;
    R.h = c->h;
    R.edge = (int)k.edge;
    R.limiter = (int)k.limiter;
    R.bracket = (int)k.thermal_bracket;
    R.cold_e = k.k1e > 0.0 && k.k2e > 0.0;
    R.cold_n = k.k1n > 0.0 && k.k2n > 0.0;
    R.k1e = (float)k.k1e;
    R.k1e_k2e = R.cold_e ? (float)(k.k1e / k.k2e) : 0.0f;
    R.k1n = (float)k.k1n;
    R.k1n_k2n = R.cold_n ? (float)(k.k1n / k.k2n) : 0.0f;
    R.sigma_vac = (float)k.sigma_vac;
    R.sigma_floor = (float)k.sigma_floor;
    R.t_floor = (float)k.t_floor;
    R.kappa0 = (float)k.kappa0;
    R.inv_c_sb = (float)(1.0 / k.c_sb);
    R.kappa_dust = (float)k.kappa_dust;
    R.t_dust = (float)k.t_dust;
    R.sigma_hold = (float)k.sigma_hold;
    R.eta_hold = (float)k.eta_hold;
    R.r_hold = (float)k.r_hold;
    R.m_tov = (float)k.m_tov;
    std::vector<float> tab(4 * kColdPoints);
    ref_cold_tables(k, tab.data());
    dalloc(&c->table, tab.size());
    SR_CUDA_TRY(cudaMemcpy(c->table, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice));
    R.table = c->table;
    dalloc(&c->held, n);
    dalloc(&c->push, 2 * n);
    if (k.heat) {
        dalloc(&c->radx, n);
        dalloc(&c->rady, n);
    }
    if (k.gravity) {
        dalloc(&c->src_free, n);
        dalloc(&c->phip, n);
        dalloc(&c->gxp, n);
        dalloc(&c->gyp, n);
    }
    const int rb = ref_hydro_blocks(c->w, c->h);
    dalloc(&c->rpart, (size_t)rb * 5);
    dalloc(&c->rbest, (size_t)rb);
    dalloc(&c->ridx, (size_t)rb);
    dalloc(&c->rfin, 6);
}

static RefArgs ref_args(sr_ctx* c, int cur) {
    RefArgs A{};
    A.R = c->R;
    A.dt = &c->rec->dt;
    A.U = c->U[cur];
    A.Uout = c->U[1 - cur];
    A.held = c->held;
    A.gx = c->cfg.gravity ? c->gx : nullptr;
    A.gy = c->cfg.gravity ? c->gy : nullptr;
    A.src = c->src;
    A.src_free = c->src_free;
    A.phim = c->phim;
    A.gxm = c->gxm;
    A.gym = c->gym;
    A.gxp = c->gxp;
    A.gyp = c->gyp;
    A.radx = c->radx;  // the last P5's cell-centred flux (zero before the first P5: no force), or none without P5
    A.rady = c->rady;
    A.push = c->push;
    A.part = c->rpart;
    A.part_best = c->rbest;
    A.part_idx = c->ridx;
    A.fin = c->rfin;
    return A;
}

// P2 on the current state, then P9 (no floors) — what Twin::new does before step 0 (reference/mod.rs:129-177).
static void initial_reductions(sr_ctx* c) {
    DtRecord rec{};
    SR_CUDA_TRY(cudaMemcpyAsync(c->rec, &rec, sizeof rec, cudaMemcpyHostToDevice, c->stream));
    SR_CUDA_TRY(cudaMemsetAsync(c->hreport, 0, 7 * sizeof(double), c->stream));
    const sr_config& k = c->cfg;
    if (ref_mode(c)) {
        // reference/mod.rs:129-177: the hold's rule on the initial state, P2, then Δt_0
        ref_hold_dt_launch(c->R, planes(c), c->held, nullptr, nullptr, 1, 0, c->part_rate, c->part_g, c->part_nf,
                           k.cfl, k.eta_g, k.dt_fixed, k.dt_cap, c->rec, c->stream);
        if (k.gravity) c->grav.solve(planes(c), c->phi, c->gx, c->gy, c->stream);
        ref_hold_dt_launch(c->R, planes(c), c->held, k.gravity ? c->gx : nullptr, k.gravity ? c->gy : nullptr, 0, 1,
                           c->part_rate, c->part_g, c->part_nf, k.cfl, k.eta_g, k.dt_fixed, k.dt_cap, c->rec,
                           c->stream);
        SR_CUDA_TRY(cudaGetLastError());
        return;
    }
    if (c->cfg.gravity) c->grav.solve(planes(c), c->phi, c->gx, c->gy, c->stream);
    floors_dt_launch(c->H, planes(c), k.gravity ? c->gx : nullptr, k.gravity ? c->gy : nullptr, 0, c->part_rate,
                     c->part_g, c->part_nf, k.cfl, k.eta_g, k.dt_fixed, k.dt_cap, c->rec, c->stream);
    SR_CUDA_TRY(cudaGetLastError());
}

static cudaEvent_t event_at(sr_ctx* c, size_t i) {
    while (c->events.size() <= i) {
        cudaEvent_t e;
        SR_CUDA_TRY(cudaEventCreate(&e));
        c->events.push_back(e);
    }
    return c->events[i];
}

static HydroArgs hydro_args(sr_ctx* c, int cur) {
    HydroArgs A{};
    A.H = c->H;
    A.dt = &c->rec->dt;
    A.U = c->U[cur];
    A.Uout = c->U[1 - cur];
    A.gx = c->cfg.gravity ? c->gx : nullptr;
    A.gy = c->cfg.gravity ? c->gy : nullptr;
    A.src = c->src;
    A.phim = c->phim;
    A.gxm = c->gxm;
    A.gym = c->gym;
    A.part_d = c->part_d;
    A.part_best = c->part_best;
    A.part_idx = c->part_idx;
    A.report = c->hreport;
    A.err = c->herr;
    return A;
}

// One step's launches on `s` from state buffer `cur`, in the reference's pass order P1 → P2 → P4 → P5 → P8 → P9
// (reference/mod.rs:264-297). With `root` the launches are captured into that graph and P5 is the device-controlled
// step (heat_capture_step); otherwise they run now, P5 by heat_step. `mark(slot)` is called at the pass boundaries
// (0 start, 1 after P2, 2 hydro update start, 3 its end, 4 after P4, 5 after P5, 6 after P8/P9).
template <class Mark>
static long long enqueue_step(sr_ctx* c, int cur, cudaStream_t s, cudaGraph_t root, Mark mark) {
    long long heat_top = 0;  // kernels of a captured implicit step outside its loops
    const sr_config& k = c->cfg;
    float* U = c->U[cur];
    mark(0);
    dt_advance_launch(c->rec, s);
    if (k.gravity) c->grav.solve(U, c->phi, c->gx, c->gy, s);
    mark(1);
    if (ref_mode(c)) {
        // reference mode: P4 (step_held), P8's floors, the hold and P9 (reference/mod.rs:264-297; P5 is off)
        if (k.hydro) {
            RefArgs A = ref_args(c, cur);
            if (k.gravity) {
                ref_hydro_source_launch(A, s);
                c->grav.solve(c->src, c->phim, c->gxm, c->gym, s);
                c->grav.solve(c->src_free, c->phip, c->gxp, c->gyp, s);
            }
            mark(2);
            ref_hydro_update_launch(A, k.gravity, s);
            mark(3);
            ref_hydro_finalize_launch(A, s);
            U = c->U[1 - cur];
        } else {
            mark(2);
            mark(3);
        }
        mark(4);
        if (k.heat) {
            if (root) heat_top = heat_capture_step(c->heat, U, nullptr, &c->rec->dt, s, root);
            else heat_step(c->heat, U, nullptr, &c->rec->dt, s, &c->heat_report);
            const float *fx, *fy;
            heat_flux_planes(c->heat, &fx, &fy);
            ref_cell_flux_launch(fx, fy, c->radx, c->rady, c->w, c->h, s);
        }
        mark(5);
        ref_floors_launch(c->R, U, s);
        ref_hold_dt_launch(c->R, U, c->held, k.gravity ? c->gx : nullptr, k.gravity ? c->gy : nullptr, 1, 1,
                           c->part_rate, c->part_g, c->part_nf, k.cfl, k.eta_g, k.dt_fixed, k.dt_cap, c->rec, s);
        mark(6);
        return heat_top;
    }
    if (k.hydro) {
        HydroArgs A = hydro_args(c, cur);
        if (k.gravity) {
            hydro_launch(kHydroSource, A, s);
            c->grav.solve(c->src, c->phim, c->gxm, c->gym, s);
            mark(2);
            hydro_launch(kHydroUpdateGrav, A, s);
            mark(3);
            hydro_finalize_launch(A, 1, s);
        } else {
            mark(2);
            hydro_launch(kHydroUpdate, A, s);
            mark(3);
            hydro_finalize_launch(A, 0, s);
        }
        U = c->U[1 - cur];
    } else {
        mark(2);
        mark(3);
    }
    mark(4);
    if (k.heat) {
        const float* kappa = k.opacity_plane ? c->kappa : nullptr;
        if (root) heat_top = heat_capture_step(c->heat, U, kappa, &c->rec->dt, s, root);
        else heat_step(c->heat, U, kappa, &c->rec->dt, s, &c->heat_report);
    }
    mark(5);
    floors_dt_launch(c->H, U, k.gravity ? c->gx : nullptr, k.gravity ? c->gy : nullptr, 1, c->part_rate, c->part_g,
                     c->part_nf, k.cfl, k.eta_g, k.dt_fixed, k.dt_cap, c->rec, s);
    mark(6);
    return heat_top;
}

// Whether a whole step can run as one captured graph: P5 (when on) must run under device control.
static bool capturable(sr_ctx* c) { return !c->cfg.heat || heat_capturable(c->heat); }

// Appends one whole step from state buffer `cur` to the capture in progress on `s` (root graph `root`); returns the
// kernels one replay launches outside the implicit step's loops.
long long sr_ctx_capture_step(sr_ctx* c, int cur, cudaStream_t s, cudaGraph_t root) {
    const long long before = (long long)sr_launches();
    const long long heat_top = enqueue_step(c, cur, s, root, [](int) {});
    const long long n = (long long)sr_launches() - before;
    sr_note_launches(-n);  // captured, not launched
    return n + heat_top;
}

// Readies `c` for captures of its whole step (the implicit step's control block); false when it cannot be captured.
bool sr_ctx_prepare_capture(sr_ctx* c) {
    if (!capturable(c)) return false;
    if (c->cfg.heat) heat_prepare_capture(c->heat, c->stream);
    return true;
}

// After `steps` whole steps ran as graphs: the state buffer, the implicit step's pending report, the launch count.
void sr_ctx_graph_steps_done(sr_ctx* c, uint32_t steps, long long launches_per_step) {
    if (c->cfg.hydro && (steps & 1)) c->cur = 1 - c->cur;
    if (c->cfg.heat && steps) heat_graph_launched(c->heat);
    sr_note_launches(launches_per_step * (long long)steps);
}

// ---- the active box (crates/sr-engine/src/step/boxfit.rs): the crop of the world around its gas, stepped as a world
// of its own. Cells outside the box hold vacuum that no pass changes (the reference's box passes leave it alone), and
// with 8 cells of vacuum inside the box's edge the crop's edge cells are empty, so its edge mode changes no flux; its
// FFT is sized to the box, as the reference's is.

// Copies `count` planes of the box's cells between the world (W x H planes) and a crop (bw x bh planes).
static void box_copy(void* dst, int dst_pitch, size_t dst_plane, const void* src, int src_pitch, size_t src_plane,
                     int count, int bw, int bh, size_t elem, cudaStream_t s) {
    for (int k = 0; k < count; k++)
        SR_CUDA_TRY(cudaMemcpy2DAsync((char*)dst + k * dst_plane * elem, dst_pitch * elem,
                                      (const char*)src + k * src_plane * elem, src_pitch * elem, bw * elem, bh,
                                      cudaMemcpyDeviceToDevice, s));
}

// The world's cells of the box into the crop context `s` (its planes and what the next step reads beside them).
static void crop_in(sr_ctx* c, sr_ctx* s, const BoxRec& b, bool with_record) {
    SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    const size_t off = (size_t)b.y0 * c->w + b.x0;
    box_copy(s->U[s->cur], b.w, s->n, planes(c) + off, c->w, c->n, c->nc, b.w, b.h, sizeof(float), s->stream);
    if (c->kappa) box_copy(s->kappa, b.w, s->n, c->kappa + off, c->w, c->n, 1, b.w, b.h, sizeof(float), s->stream);
    if (c->held) box_copy(s->held, b.w, s->n, c->held + off, c->w, c->n, 1, b.w, b.h, 1, s->stream);
    if (c->radx) {
        box_copy(s->radx, b.w, s->n, c->radx + off, c->w, c->n, 1, b.w, b.h, sizeof(float), s->stream);
        box_copy(s->rady, b.w, s->n, c->rady + off, c->w, c->n, 1, b.w, b.h, sizeof(float), s->stream);
    }
    if (c->heat && s->heat)
        box_copy(heat_rate_plane(s->heat), b.w, s->n, heat_rate_plane(c->heat) + off, c->w, c->n, 1, b.w, b.h,
                 sizeof(double), s->stream);
    if (with_record) SR_CUDA_TRY(cudaMemcpyAsync(s->rec, c->rec, sizeof(DtRecord), cudaMemcpyDeviceToDevice, s->stream));
    s->uploaded = true;
}

// The crop's cells back into the world, and its Δt record (the guard's cell in world coordinates).
static void crop_out(sr_ctx* c, sr_ctx* s, const BoxRec& b) {
    SR_CUDA_TRY(cudaStreamSynchronize(s->stream));
    const size_t off = (size_t)b.y0 * c->w + b.x0;
    box_copy(planes(c) + off, c->w, c->n, s->U[s->cur], b.w, s->n, c->nc, b.w, b.h, sizeof(float), c->stream);
    if (c->held) box_copy(c->held + off, c->w, c->n, s->held, b.w, s->n, 1, b.w, b.h, 1, c->stream);
    if (c->radx) {
        box_copy(c->radx + off, c->w, c->n, s->radx, b.w, s->n, 1, b.w, b.h, sizeof(float), c->stream);
        box_copy(c->rady + off, c->w, c->n, s->rady, b.w, s->n, 1, b.w, b.h, sizeof(float), c->stream);
    }
    if (c->heat && s->heat)
        box_copy(heat_rate_plane(c->heat) + off, c->w, c->n, heat_rate_plane(s->heat), b.w, s->n, 1, b.w, b.h,
                 sizeof(double), c->stream);
    DtRecord rec;
    SR_CUDA_TRY(cudaMemcpyAsync(&rec, s->rec, sizeof rec, cudaMemcpyDeviceToHost, c->stream));
    SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (rec.non_finite)
        rec.nf_cell = (rec.nf_cell / b.w + b.y0) * (long long)c->w + rec.nf_cell % b.w + b.x0;
    SR_CUDA_TRY(cudaMemcpyAsync(c->rec, &rec, sizeof rec, cudaMemcpyHostToDevice, c->stream));
    SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
}

// The box of the state as it stands: over the crop while one is stepped (the vacuum outside it holds no gas).
static BoxRec fit_box(sr_ctx* c) {
    const float* sig = c->sub ? c->sub->U[c->sub->cur] : planes(c);
    const int w = c->sub ? c->sub->w : c->w, h = c->sub ? c->sub->h : c->h;
    const int ox = c->sub ? c->box.x0 : 0, oy = c->sub ? c->box.y0 : 0;
    cudaStream_t st = c->sub ? c->sub->stream : c->stream;
    box_fit_launch(sig, w, h, ox, oy, c->w, c->h, (float)c->cfg.sigma_vac, c->box_part, c->box_rec, st);
    int r[4];
    SR_CUDA_TRY(cudaMemcpyAsync(r, c->box_rec, sizeof r, cudaMemcpyDeviceToHost, st));
    SR_CUDA_TRY(cudaStreamSynchronize(st));
    c->box_fits++;
    BoxRec b{r[0], r[1], r[2], r[3]};
    if (b.w == 0 || b.h == 0) b = BoxRec{0, 0, c->w, c->h};  // no gas: the whole world runs the step
    return b;
}

// The crop context for a box of this size (made on first use, kept for the boxes that follow).
static sr_ctx* sub_for(sr_ctx* c, int w, int h) {
    for (sr_ctx* s : c->subs)
        if (s->w == w && s->h == h) return s;
    sr_config k = c->cfg;
    k.width = (uint32_t)w;
    k.height = (uint32_t)h;
    k.active_box = 0;
    sr_ctx* s = nullptr;
    const sr_status st = sr_create(&k, &s);
    if (st != SR_OK) throw SrError{st, "the active box's context: " + g_create_error};
    s->timing = c->timing;
    if (c->learner && s->heat) {
        heat_attach_learned(s->heat, c->learner->L);
        s->learner = c->learner;
    }
    c->subs.push_back(s);
    return s;
}

// A refit (reference: before step 0, and after P9 at step indices ≡ 0 mod 16): the crop follows the gas.
static void refit(sr_ctx* c) {
    const BoxRec b = fit_box(c);
    if (c->sub && b.x0 == c->box.x0 && b.y0 == c->box.y0 && b.w == c->box.w && b.h == c->box.h) return;
    if (c->sub) crop_out(c, c->sub, c->box);
    sr_ctx* s = sub_for(c, b.w, b.h);
    crop_in(c, s, b, true);
    c->sub = s;
    c->box = b;
}

// Makes the world's buffers current (the crop's state copied back) before a read of the world.
static void box_sync(sr_ctx* c) {
    if (c->sub) crop_out(c, c->sub, c->box);
}

static void run_steps(sr_ctx* c, uint32_t steps);

static void run_box_steps(sr_ctx* c, uint32_t steps) {
    constexpr unsigned long long kRefitEvery = 16;  // boxfit.rs REFIT_EVERY
    sr_cost total{};
    uint32_t done = 0;
    while (done < steps) {
        const unsigned long long s0 = c->box_steps;
        // the next refit follows the step of index ≡ 0 (mod 16): after 1, 17, 33, ... steps
        const unsigned long long next = s0 < 1 ? 1 : ((s0 - 1) / kRefitEvery + 1) * kRefitEvery + 1;
        const uint32_t k = (uint32_t)std::min<unsigned long long>(steps - done, next - s0);
        sr_ctx* s = c->sub;
        run_steps(s, k);
        if (c->timing) {
            total.steps += s->cost.steps;
            total.gravity_ms += s->cost.gravity_ms;
            total.hydro_ms += s->cost.hydro_ms;
            total.heat_ms += s->cost.heat_ms;
            total.floors_ms += s->cost.floors_ms;
            total.dt_ms += s->cost.dt_ms;
            total.total_ms += s->cost.total_ms;
            total.hydro_update_ms += s->cost.hydro_update_ms;
            total.hydro_update_launches += s->cost.hydro_update_launches;
            total.kernel_launches += s->cost.kernel_launches;
        }
        c->box_steps += k;
        done += k;
        if (c->box_steps == next) refit(c);
    }
    SR_CUDA_TRY(cudaStreamSynchronize(c->sub->stream));
    if (c->timing) c->cost = total;
}

// Captures the whole step from the current state buffer as a graph (once per buffer).
static void capture_step_graph(sr_ctx* c) {
    sr_ctx_prepare_capture(c);
    cudaGraph_t g;
    SR_CUDA_TRY(cudaGraphCreate(&g, 0));
    SR_CUDA_TRY(cudaStreamBeginCaptureToGraph(c->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    long long n = 0;
    try {
        n = sr_ctx_capture_step(c, c->cur, c->stream, g);
    } catch (...) {
        cudaGraph_t dead;
        cudaStreamEndCapture(c->stream, &dead);
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraph_t out;
    SR_CUDA_TRY(cudaStreamEndCapture(c->stream, &out));
    const cudaError_t e = cudaGraphInstantiate(&c->step_graph[c->cur], g, 0);
    cudaGraphDestroy(g);
    SR_CUDA_TRY(e);
    c->step_launches = n;
}

static void run_steps(sr_ctx* c, uint32_t steps) {
    if (c->use_box) {
        run_box_steps(c, steps);
        return;
    }
    const unsigned long long launches0 = sr_launches();
    // after the first step (which tunes the multigrid) every step is one captured graph, unless the per-pass timing
    // (2) asks for the passes launched one by one; timing 1 records the device time of each step's graph
    if (c->timing != 2 && steps && capturable(c)) {
        for (uint32_t s = 0; s < steps; s++) {
            if (!c->step_graph[c->cur]) capture_step_graph(c);  // before the step's start event
            if (c->timing) SR_CUDA_TRY(cudaEventRecord(event_at(c, 2 * (size_t)s), c->stream));
            SR_CUDA_TRY(cudaGraphLaunch(c->step_graph[c->cur], c->stream));
            if (c->timing) SR_CUDA_TRY(cudaEventRecord(event_at(c, 2 * (size_t)s + 1), c->stream));
            sr_ctx_graph_steps_done(c, 1, c->step_launches);
        }
        if (c->timing) {
            SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
            if (c->heat) heat_account_launches(c->heat, c->stream);
            sr_cost& t = c->cost;
            memset(&t, 0, sizeof t);
            t.steps = steps;
            for (uint32_t s = 0; s < steps; s++) {
                float ms = 0.0f;
                SR_CUDA_TRY(cudaEventElapsedTime(&ms, c->events[2 * (size_t)s], c->events[2 * (size_t)s + 1]));
                t.total_ms += ms;
            }
            t.kernel_launches = sr_launches() - launches0;
        }
        return;
    }
    // event slots per step: 0 start, 1 after P2, 2 hydro update start, 3 hydro update end, 4 after P4, 5 after P5,
    // 6 after P8/P9
    const int E = 7;
    for (uint32_t s = 0; s < steps; s++) {
        auto mark = [&](int slot) {
            if (c->timing) SR_CUDA_TRY(cudaEventRecord(event_at(c, (size_t)s * E + slot), c->stream));
        };
        enqueue_step(c, c->cur, c->stream, nullptr, mark);
        if (c->cfg.hydro) c->cur = 1 - c->cur;
        SR_CUDA_TRY(cudaGetLastError());
    }
    if (c->timing && steps) {
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (c->heat) heat_account_launches(c->heat, c->stream);
        sr_cost& t = c->cost;
        memset(&t, 0, sizeof t);
        t.steps = steps;
        for (uint32_t s = 0; s < steps; s++) {
            float ms[6];
            for (int q = 0; q < 6; q++) {
                int a = q, b = q + 1;
                SR_CUDA_TRY(cudaEventElapsedTime(&ms[q], c->events[(size_t)s * E + a], c->events[(size_t)s * E + b]));
            }
            t.gravity_ms += ms[0];
            t.hydro_ms += ms[1] + ms[2] + ms[3];
            t.hydro_update_ms += ms[2];
            t.heat_ms += ms[4];
            t.dt_ms += ms[5];
            float total;
            SR_CUDA_TRY(cudaEventElapsedTime(&total, c->events[(size_t)s * E], c->events[(size_t)s * E + 6]));
            t.total_ms += total;
        }
        t.hydro_update_launches = c->cfg.hydro ? steps : 0;
        t.kernel_launches = sr_launches() - launches0;
    }
}

// The world's buffers made current from the crop (with the active box), written by `write`, then the crop made current
// from them again: the resume calls write the world and let the box's crop follow.
template <class F>
static void write_world(sr_ctx* c, bool with_record, F write) {
    box_sync(c);
    write();
    SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->sub) {
        crop_in(c, c->sub, c->box, with_record);
        SR_CUDA_TRY(cudaStreamSynchronize(c->sub->stream));
    }
}

static float* staging_plane(sr_ctx* c) {
    if (!c->plane32) dalloc(&c->plane32, c->n);
    return c->plane32;
}

extern "C" {

void sr_config_default(sr_config* c) {
    memset(c, 0, sizeof *c);
    c->struct_size = sizeof(sr_config);
    c->width = 64;
    c->height = 64;
    c->channels = 4;
    c->edge = SR_EDGE_BOUNCE;
    c->limiter = SR_LIMITER_MC;
    c->thermal_bracket = 1;
    c->hydro = 1;
    c->kernel = SR_KERNEL_SELF_CELL;
    c->precond = SR_PRECOND_MG;
    c->flux_limiter = 1;
    c->mg_pre = 4;  // V(4,4): the fewest rounds for the least time at 2048² (more sweeps ride the same loads)
    c->mg_post = 4;
    c->max_passes = 128;
    c->max_rounds = 4096;
    c->gamma = 2.0;
    c->mu = 1.0;
    c->t_floor = 0.05;
    c->sigma_vac = 1e-6;
    c->sigma_floor = 1e-8;
    c->cfl = 0.4;
    c->eta_g = 0.3;
    c->G = 1.0;
    c->softening = 1.0;
    c->a_r = 6.25e-7;
    c->c_sb = 12800.0;
    c->kappa0 = 1.0;
    c->k_cond = 0.0;
    c->chi = 0.0;
    c->solve_tol = 1e-8;
    c->newton_heat = 1e-6;  // the reference GPU path's Newton stop (crates/sr-engine/shaders/heat.wgsl:355-357)
    c->newton_cell = 1e-3;
    c->k1e = 21.3;  // assets/physics.json's cold pairs and hold; m_tov_sb of assets/calibration.json
    c->k2e = 134.0;
    c->k1n = 2.67;
    c->k2n = 58.2;
    c->sigma_hold = 10.0;
    c->eta_hold = 0.1;
    c->r_hold = 24.0;
    c->m_tov = 4853.169981814195;
}

uint32_t sr_abi_version(void) { return SR_ABI_VERSION; }

sr_status sr_create(const sr_config* cfg, sr_ctx** out) {
    if (!cfg || !out) {
        g_create_error = "sr_create: null argument";
        return SR_E_INVALID;
    }
    *out = nullptr;
    sr_ctx* c = new sr_ctx();
    try {
        validate(*cfg);
        c->cfg = *cfg;
        c->H = hydro_const(*cfg);
        c->w = (int)cfg->width;
        c->h = (int)cfg->height;
        c->n = (size_t)c->w * c->h;
        const size_t n = c->n;
        SR_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->nc = (int)cfg->channels;
        dalloc(&c->U[0], (size_t)c->nc * n);
        dalloc(&c->U[1], (size_t)c->nc * n);
        dalloc(&c->phi, n);
        dalloc(&c->gx, n);
        dalloc(&c->gy, n);
        if (cfg->gravity) {
            dalloc(&c->src, n);
            dalloc(&c->phim, n);
            dalloc(&c->gxm, n);
            dalloc(&c->gym, n);
            c->grav.create(c->w, c->h, (int)cfg->kernel, cfg->G, cfg->softening, (float)cfg->sigma_vac);
            c->grav_ready = true;
        }
        if (cfg->opacity_plane) dalloc(&c->kappa, n);
        int hb = hydro_blocks(c->w, c->h);
        dalloc(&c->part_d, (size_t)hb * 6);
        dalloc(&c->part_best, (size_t)hb);
        dalloc(&c->part_idx, (size_t)hb);
        dalloc(&c->hreport, 7);
        dalloc(&c->herr, 1);
        dalloc(&c->rec, 1);
        int fb = floors_dt_blocks(c->w, c->h);
        if (c->nc == kRefChannels) {
            fb = 148 * 8;  // the reference-mode Δt partials' grid at most
            ref_setup(c);
        }
        dalloc(&c->part_rate, (size_t)fb);
        dalloc(&c->part_g, (size_t)fb);
        dalloc(&c->part_nf, (size_t)fb);
        if (cfg->heat) c->heat = heat_create(*cfg, c->stream);
        c->use_box = cfg->active_box != 0;
        if (c->use_box) {
            dalloc(&c->box_part, 4 * (size_t)kBoxMaxBlocks);
            dalloc(&c->box_rec, 4);
        }
        if (c->heat && ref_mode(c)) {
            HeatRef hr;
            hr.on = 1;
            hr.table = c->table;
            hr.cold_e = c->R.cold_e;
            hr.cold_n = c->R.cold_n;
            hr.kappa_dust = cfg->kappa_dust;
            hr.t_dust = cfg->t_dust;
            heat_set_reference(c->heat, hr);
        }
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    } catch (const SrError& e) {
        g_create_error = e.message;
        ctx_free(c);
        return e.status;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        ctx_free(c);
        return SR_E_CUDA;
    }
    *out = c;
    return SR_OK;
}

void sr_destroy(sr_ctx* ctx) { ctx_free(ctx); }

sr_status sr_upload(sr_ctx* c, const float* p, uint32_t nplanes) {
    return guarded(c, [&] {
        SR_REQUIRE(p, "sr_upload: null planes");
        SR_REQUIRE((int)nplanes == c->nc, "sr_upload: the context carries " + std::to_string(c->nc) + " planes");
        SR_CUDA_TRY(cudaMemcpyAsync(planes(c), p, sizeof(float) * c->nc * c->n, cudaMemcpyHostToDevice, c->stream));
        if (c->held) SR_CUDA_TRY(cudaMemsetAsync(c->held, 0, c->n, c->stream));  // a new state: none held yet
        if (c->radx) {  // nor a flux: the first step takes no radiation force (reference/mod.rs:122-123)
            SR_CUDA_TRY(cudaMemsetAsync(c->radx, 0, sizeof(float) * c->n, c->stream));
            SR_CUDA_TRY(cudaMemsetAsync(c->rady, 0, sizeof(float) * c->n, c->stream));
        }
        if (c->heat) heat_reset(c->heat, c->stream);
        c->uploaded = true;
        if (c->use_box) {
            // the box fit to the new state, its crop the world that steps; P2 and Δt_0 over it (boxfit.rs: before
            // step 0, ahead of the initial Δt reduction)
            c->sub = nullptr;
            c->box_steps = 0;
            const BoxRec b = fit_box(c);
            sr_ctx* s = sub_for(c, b.w, b.h);
            crop_in(c, s, b, false);
            if (s->heat) heat_reset(s->heat, s->stream);
            initial_reductions(s);
            SR_CUDA_TRY(cudaStreamSynchronize(s->stream));
            c->sub = s;
            c->box = b;
            return;
        }
        initial_reductions(c);
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    });
}

sr_status sr_readback(sr_ctx* c, float* p, uint32_t nplanes) {
    return guarded(c, [&] {
        SR_REQUIRE(p, "sr_readback: null planes");
        SR_REQUIRE((int)nplanes == c->nc, "sr_readback: the context carries " + std::to_string(c->nc) + " planes");
        box_sync(c);
        SR_CUDA_TRY(cudaMemcpyAsync(p, planes(c), sizeof(float) * c->nc * c->n, cudaMemcpyDeviceToHost, c->stream));
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    });
}

sr_status sr_upload_held(sr_ctx* c, const uint32_t* mask) {
    return guarded(c, [&] {
        SR_REQUIRE(mask, "sr_upload_held: null mask");
        SR_REQUIRE(c->held, "sr_upload_held: the hold is reference mode's (a context of 14 channels)");
        std::vector<uint8_t> m(c->n);
        for (size_t i = 0; i < c->n; i++) m[i] = mask[i] != 0;
        SR_CUDA_TRY(cudaMemcpyAsync(c->held, m.data(), c->n, cudaMemcpyHostToDevice, c->stream));
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (c->sub) {
            const BoxRec& b = c->box;
            box_copy(c->sub->held, b.w, c->sub->n, c->held + (size_t)b.y0 * c->w + b.x0, c->w, c->n, 1, b.w, b.h, 1,
                     c->sub->stream);
            SR_CUDA_TRY(cudaStreamSynchronize(c->sub->stream));
        }
    });
}

sr_status sr_read_held(sr_ctx* c, uint32_t* mask) {
    return guarded(c, [&] {
        SR_REQUIRE(mask, "sr_read_held: null mask");
        SR_REQUIRE(c->held, "sr_read_held: the hold is reference mode's (a context of 14 channels)");
        box_sync(c);
        std::vector<uint8_t> m(c->n);
        SR_CUDA_TRY(cudaMemcpyAsync(m.data(), c->held, c->n, cudaMemcpyDeviceToHost, c->stream));
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < c->n; i++) mask[i] = m[i];
    });
}

sr_status sr_upload_opacity(sr_ctx* c, const float* kappa) {
    return guarded(c, [&] {
        SR_REQUIRE(kappa, "sr_upload_opacity: null plane");
        SR_REQUIRE(c->cfg.opacity_plane, "sr_upload_opacity: the context was made without opacity_plane");
        SR_CUDA_TRY(cudaMemcpyAsync(c->kappa, kappa, sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (c->sub) {
            const BoxRec& b = c->box;
            box_copy(c->sub->kappa, b.w, c->sub->n, c->kappa + (size_t)b.y0 * c->w + b.x0, c->w, c->n, 1, b.w, b.h,
                     sizeof(float), c->sub->stream);
            SR_CUDA_TRY(cudaStreamSynchronize(c->sub->stream));
        }
    });
}

sr_status sr_set_clock(sr_ctx* c, uint64_t steps, double sim_time, double dt, double dt_next) {
    return guarded(c, [&] {
        SR_REQUIRE(c->uploaded, "sr_set_clock: no state uploaded");
        SR_REQUIRE(std::isfinite(sim_time) && sim_time >= 0.0, "sr_set_clock: sim_time must be finite and >= 0");
        SR_REQUIRE(std::isfinite(dt) && dt >= 0.0 && std::isfinite(dt_next) && dt_next > 0.0,
                   "sr_set_clock: dt must be finite and >= 0, dt_next finite and > 0");
        SR_REQUIRE(steps <= 0xffffffffull, "sr_set_clock: a step index past the GPU's u32 count");
        write_world(c, true, [&] {
            DtRecord rec{};  // the guard's finding cleared (latch.rs:496-510)
            rec.dt = dt;
            rec.dt_next = dt_next;
            rec.sim_time = sim_time;
            rec.steps = steps;
            SR_CUDA_TRY(cudaMemcpyAsync(c->rec, &rec, sizeof rec, cudaMemcpyHostToDevice, c->stream));
        });
        c->box_steps = steps;  // refits follow the restored step index
    });
}

sr_status sr_read_heat_rate(sr_ctx* c, float* rate) {
    return guarded(c, [&] {
        SR_REQUIRE(rate, "sr_read_heat_rate: null plane");
        SR_REQUIRE(c->heat, "sr_read_heat_rate: the context runs no heat pass");
        box_sync(c);
        float* d = staging_plane(c);
        heat_rate_to_f32(c->heat, d, c->stream);
        SR_CUDA_TRY(cudaMemcpyAsync(rate, d, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    });
}

sr_status sr_set_heat_rate(sr_ctx* c, const float* rate) {
    return guarded(c, [&] {
        SR_REQUIRE(c->heat, "sr_set_heat_rate: the context runs no heat pass");
        write_world(c, false, [&] {
            float* d = nullptr;
            if (rate) {
                d = staging_plane(c);
                SR_CUDA_TRY(cudaMemcpyAsync(d, rate, sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
            }
            heat_rate_from_f32(c->heat, d, c->stream);
        });
    });
}

sr_status sr_read_side_flux(sr_ctx* c, float* fx, float* fy) {
    return guarded(c, [&] {
        SR_REQUIRE(fx && fy, "sr_read_side_flux: null plane");
        SR_REQUIRE(c->radx && c->heat, "sr_read_side_flux: the side flux is reference mode's P5 output (14 channels, heat on)");
        box_sync(c);
        SR_CUDA_TRY(cudaMemcpyAsync(fx, c->radx, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
        SR_CUDA_TRY(cudaMemcpyAsync(fy, c->rady, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->stream));
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    });
}

sr_status sr_set_side_flux(sr_ctx* c, const float* fx, const float* fy) {
    return guarded(c, [&] {
        SR_REQUIRE(fx && fy, "sr_set_side_flux: null plane");
        SR_REQUIRE(c->radx && c->heat, "sr_set_side_flux: the side flux is reference mode's P5 output (14 channels, heat on)");
        write_world(c, false, [&] {
            SR_CUDA_TRY(cudaMemcpyAsync(c->radx, fx, sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
            SR_CUDA_TRY(cudaMemcpyAsync(c->rady, fy, sizeof(float) * c->n, cudaMemcpyHostToDevice, c->stream));
        });
    });
}

// The checks after steps ran (the stream idle): a bounded wait that gave up, then the non-finite guard.
static sr_status after_steps(sr_ctx* c) {
    if (c->sub) {
        const sr_status ss = after_steps(c->sub);
        if (ss == SR_OK) return SR_OK;
        c->error = c->sub->error;
        if (ss == SR_E_NONFINITE) {  // the cell in world coordinates
            DtRecord rec;
            sr_status st2 = guarded(c, [&] { SR_CUDA_TRY(cudaMemcpy(&rec, c->sub->rec, sizeof rec, cudaMemcpyDeviceToHost)); });
            if (st2 != SR_OK) return st2;
            const BoxRec& b = c->box;
            const long long cell = (rec.nf_cell / b.w + b.y0) * (long long)c->w + rec.nf_cell % b.w + b.x0;
            c->error = "non-finite value at cell " + std::to_string(cell) + " channel " +
                       std::to_string(rec.nf_channel) + " after step " + std::to_string(rec.nf_step);
        }
        return ss;
    }
    sr_status st = guarded(c, [&] {
        int herr = 0;
        SR_CUDA_TRY(cudaMemcpy(&herr, c->herr, sizeof herr, cudaMemcpyDeviceToHost));
        if (herr) {
            SR_CUDA_TRY(cudaMemset(c->herr, 0, sizeof herr));
            throw SrError{SR_E_TIMEOUT, "a TMA wait of the hydro kernel gave up"};
        }
        if (c->cfg.precond == SR_PRECOND_LEARNED && c->learner && learned_error(c->learner->L, c->stream))
            throw SrError{SR_E_TIMEOUT, "a tensor-core wait of the learned preconditioner gave up"};
        if (c->heat && heat_wait_error(c->heat, c->stream))
            throw SrError{SR_E_TIMEOUT, "a TMA wait of the multigrid smoother gave up"};
    });
    if (st != SR_OK) return st;
    DtRecord rec;
    st = guarded(c, [&] { SR_CUDA_TRY(cudaMemcpy(&rec, c->rec, sizeof rec, cudaMemcpyDeviceToHost)); });
    if (st != SR_OK) return st;
    if (rec.non_finite) {
        c->error = "non-finite value at cell " + std::to_string(rec.nf_cell) + " channel " +
                   std::to_string(rec.nf_channel) + " after step " + std::to_string(rec.nf_step);
        return SR_E_NONFINITE;
    }
    return SR_OK;
}

sr_status sr_step(sr_ctx* c, uint32_t steps) {
    sr_status st = guarded(c, [&] {
        SR_REQUIRE(c->uploaded, "sr_step: no state uploaded");
        run_steps(c, steps);
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
    });
    if (st != SR_OK) return st;
    return after_steps(c);
}

sr_status sr_read_dt(sr_ctx* c, sr_dt_report* out) {
    return guarded(c, [&] {
        SR_REQUIRE(out, "sr_read_dt: null report");
        DtRecord rec;
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (c->sub) {
            SR_CUDA_TRY(cudaStreamSynchronize(c->sub->stream));
            SR_CUDA_TRY(cudaMemcpy(&rec, c->sub->rec, sizeof rec, cudaMemcpyDeviceToHost));
            if (rec.non_finite)
                rec.nf_cell = (rec.nf_cell / c->box.w + c->box.y0) * (long long)c->w + rec.nf_cell % c->box.w + c->box.x0;
        } else {
            SR_CUDA_TRY(cudaMemcpy(&rec, c->rec, sizeof rec, cudaMemcpyDeviceToHost));
        }
        out->dt = rec.dt;
        out->dt_next = rec.dt_next;
        out->steps = rec.steps;
        out->sim_time = rec.sim_time;
        out->non_finite = rec.non_finite;
        out->nf_channel = rec.nf_channel;
        out->nf_cell = rec.nf_cell;
    });
}

sr_status sr_read_heat(sr_ctx* c, sr_heat_report* out) {
    return guarded(c, [&] {
        SR_REQUIRE(out, "sr_read_heat: null report");
        SR_REQUIRE(c->cfg.heat, "sr_read_heat: the context runs no heat pass");
        sr_ctx* h = c->sub ? c->sub : c;
        heat_report(h->heat, h->stream, &h->heat_report);
        *out = h->heat_report;
    });
}

sr_status sr_gravity_field(sr_ctx* c, float* gx, float* gy, float* phi) {
    return guarded(c, [&] {
        SR_REQUIRE(c->cfg.gravity, "sr_gravity_field: the context runs no gravity pass");
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (c->sub) {
            // the box's P2 (the field of the last step's start state over the box, as the reference's box-sized P2
            // leaves it), 0 outside the box
            sr_ctx* s = c->sub;
            const BoxRec& b = c->box;
            SR_CUDA_TRY(cudaStreamSynchronize(s->stream));
            std::vector<float> crop(s->n);
            float* outs[3] = {gx, gy, phi};
            const float* srcs[3] = {s->gx, s->gy, s->phi};
            for (int k = 0; k < 3; k++) {
                if (!outs[k]) continue;
                SR_CUDA_TRY(cudaMemcpy(crop.data(), srcs[k], sizeof(float) * s->n, cudaMemcpyDeviceToHost));
                std::fill(outs[k], outs[k] + c->n, 0.0f);
                for (int y = 0; y < b.h; y++)
                    std::copy(crop.data() + (size_t)y * b.w, crop.data() + (size_t)(y + 1) * b.w,
                              outs[k] + (size_t)(y + b.y0) * c->w + b.x0);
            }
            return;
        }
        if (gx) SR_CUDA_TRY(cudaMemcpy(gx, c->gx, sizeof(float) * c->n, cudaMemcpyDeviceToHost));
        if (gy) SR_CUDA_TRY(cudaMemcpy(gy, c->gy, sizeof(float) * c->n, cudaMemcpyDeviceToHost));
        if (phi) SR_CUDA_TRY(cudaMemcpy(phi, c->phi, sizeof(float) * c->n, cudaMemcpyDeviceToHost));
    });
}

sr_status sr_heat_flux(sr_ctx* c, float* fx, float* fy) {
    return guarded(c, [&] {
        SR_REQUIRE(c->cfg.heat, "sr_heat_flux: the context runs no heat pass");
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (!c->sub) {
            heat_read_flux(c->heat, fx, fy);
            return;
        }
        // the crop's faces at the box's place in the world's face planes; no flux crosses a face outside the box
        sr_ctx* s = c->sub;
        const BoxRec& b = c->box;
        SR_CUDA_TRY(cudaStreamSynchronize(s->stream));
        std::vector<float> sx((size_t)(b.w + 1) * b.h), sy((size_t)b.w * (b.h + 1));
        heat_read_flux(s->heat, sx.data(), sy.data());
        if (fx) {
            std::fill(fx, fx + (size_t)(c->w + 1) * c->h, 0.0f);
            for (int y = 0; y < b.h; y++)
                for (int x = 0; x <= b.w; x++)
                    fx[(size_t)(y + b.y0) * (c->w + 1) + x + b.x0] = sx[(size_t)y * (b.w + 1) + x];
        }
        if (fy) {
            std::fill(fy, fy + (size_t)c->w * (c->h + 1), 0.0f);
            for (int y = 0; y <= b.h; y++)
                for (int x = 0; x < b.w; x++) fy[(size_t)(y + b.y0) * c->w + x + b.x0] = sy[(size_t)y * b.w + x];
        }
    });
}

sr_status sr_set_edge_mode(sr_ctx* c, uint32_t edge) {
    return guarded(c, [&] {
        SR_REQUIRE(edge <= SR_EDGE_LEAVE, "unknown edge mode");
        drop_step_graphs(c);  // the captured steps hold the edge mode
        c->cfg.edge = edge;
        c->H.edge = (int)edge;
        c->R.edge = (int)edge;
        for (sr_ctx* s : c->subs) {
            drop_step_graphs(s);
            s->cfg.edge = edge;
            s->H.edge = (int)edge;
            s->R.edge = (int)edge;
        }
    });
}

sr_status sr_set_heat_precond(sr_ctx* c, uint32_t precond) {
    return guarded(c, [&] {
        SR_REQUIRE(precond <= SR_PRECOND_LEARNED, "unknown preconditioner");
        SR_REQUIRE(c->cfg.heat, "sr_set_heat_precond: the context runs no heat pass");
        drop_step_graphs(c);
        c->cfg.precond = precond;
        heat_set_precond(c->heat, precond);
        for (sr_ctx* s : c->subs) {
            drop_step_graphs(s);
            s->cfg.precond = precond;
            heat_set_precond(s->heat, precond);
        }
    });
}

sr_status sr_set_heat_limits(sr_ctx* c, uint32_t max_passes, uint32_t max_rounds) {
    return guarded(c, [&] {
        SR_REQUIRE(max_passes >= 1 && max_rounds >= 1, "heat limits must be >= 1");
        SR_REQUIRE(c->cfg.heat, "sr_set_heat_limits: the context runs no heat pass");
        drop_step_graphs(c);
        c->cfg.max_passes = max_passes;
        c->cfg.max_rounds = max_rounds;
        heat_set_limits(c->heat, max_passes, max_rounds);
        for (sr_ctx* s : c->subs) {
            drop_step_graphs(s);
            s->cfg.max_passes = max_passes;
            s->cfg.max_rounds = max_rounds;
            heat_set_limits(s->heat, max_passes, max_rounds);
        }
    });
}

sr_status sr_read_box(sr_ctx* c, sr_box_report* out) {
    return guarded(c, [&] {
        SR_REQUIRE(out, "sr_read_box: null report");
        sr_ctx* g = c->sub ? c->sub : c;
        out->x0 = c->sub ? (uint32_t)c->box.x0 : 0;
        out->y0 = c->sub ? (uint32_t)c->box.y0 : 0;
        out->w = (uint32_t)g->w;
        out->h = (uint32_t)g->h;
        out->fft_w = g->grav_ready ? (uint32_t)g->grav.px : 0;
        out->fft_h = g->grav_ready ? (uint32_t)g->grav.py : 0;
        out->fits = c->box_fits;
    });
}

sr_status sr_set_timing(sr_ctx* c, int32_t on) {
    return guarded(c, [&] {
        c->timing = on <= 0 ? 0 : (on == 1 ? 1 : 2);
        for (sr_ctx* s : c->subs) s->timing = c->timing;
    });
}

sr_status sr_read_cost(sr_ctx* c, sr_cost* out) {
    return guarded(c, [&] {
        SR_REQUIRE(out, "sr_read_cost: null report");
        *out = c->cost;
    });
}

sr_status sr_heat_first_solve(sr_ctx* c, double dt, uint32_t precond, double* ms, uint32_t* rounds,
                              double* rel_residual, double* x, uint32_t* fallback) {
    return guarded(c, [&] {
        SR_REQUIRE(c->cfg.heat, "sr_heat_first_solve: the context runs no heat pass");
        SR_REQUIRE(c->uploaded, "sr_heat_first_solve: no state uploaded");
        SR_REQUIRE(dt > 0.0, "sr_heat_first_solve: dt must be positive");
        SR_REQUIRE(precond <= SR_PRECOND_LEARNED, "unknown preconditioner");
        heat_first_solve(c->heat, planes(c), c->cfg.opacity_plane ? c->kappa : nullptr, dt, precond, c->stream, ms,
                         rounds, rel_residual, x, fallback);
        if (precond == SR_PRECOND_LEARNED && c->learner && learned_error(c->learner->L, c->stream))
            throw SrError{SR_E_TIMEOUT, "a tensor-core wait of the learned preconditioner gave up"};
    });
}

sr_status sr_time_smoother(sr_ctx* c, uint32_t reps, double* pre_ms, double* post_ms) {
    return guarded(c, [&] {
        SR_REQUIRE(c->cfg.heat, "sr_time_smoother: the context runs no heat pass");
        SR_REQUIRE(pre_ms && post_ms && reps >= 1, "sr_time_smoother: bad arguments");
        heat_time_smoother(c->heat, (int)reps, c->stream, pre_ms, post_ms);
    });
}

// ---- the learned preconditioner
sr_status sr_learner_create(uint32_t crop, uint32_t capacity, uint64_t seed, sr_learner** out) {
    return guarded_free([&] {
        SR_REQUIRE(out, "sr_learner_create: null argument");
        *out = nullptr;
        sr_learner* l = new sr_learner();
        try {
            SR_CUDA_TRY(cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking));
            l->L = learned_create((int)crop, (int)capacity, seed);
        } catch (...) {
            if (l->stream) cudaStreamDestroy(l->stream);
            delete l;
            throw;
        }
        *out = l;
    });
}

void sr_learner_destroy(sr_learner* l) {
    if (!l) return;
    cudaStreamSynchronize(l->stream);
    learned_destroy(l->L);
    cudaStreamDestroy(l->stream);
    delete l;
}

uint32_t sr_learner_param_count(void) { return (uint32_t)learned_param_count(); }

sr_status sr_learner_get_params(sr_learner* l, float* theta) {
    return guarded_free([&] {
        SR_REQUIRE(l && theta, "sr_learner_get_params: null argument");
        learned_get_params(l->L, theta);
    });
}

sr_status sr_learner_set_params(sr_learner* l, const float* theta) {
    return guarded_free([&] {
        SR_REQUIRE(l && theta, "sr_learner_set_params: null argument");
        learned_set_params(l->L, theta);
    });
}

sr_status sr_learner_collect(sr_learner* l, sr_ctx* c, double dt, uint32_t crops, uint64_t seed, uint32_t* samples) {
    return guarded(c, [&] {
        SR_REQUIRE(l, "sr_learner_collect: null learner");
        SR_REQUIRE(c->cfg.heat && c->uploaded, "sr_learner_collect: the context has no implicit step to solve");
        SR_REQUIRE(dt > 0.0, "sr_learner_collect: dt must be positive");
        SR_REQUIRE(crops >= 1 && crops <= 4096, "sr_learner_collect: crops must be in 1..4096");
        const int got = heat_collect(c->heat, l->L, planes(c), c->cfg.opacity_plane ? c->kappa : nullptr, dt,
                                     (int)crops, seed, c->stream);
        if (samples) *samples = (uint32_t)got;
    });
}

sr_status sr_learner_train(sr_learner* l, uint32_t iterations, uint32_t batch, double lr, uint64_t seed,
                           double* loss) {
    return guarded_free([&] {
        SR_REQUIRE(l, "sr_learner_train: null learner");
        SR_REQUIRE(batch >= 1 && batch <= 4096, "sr_learner_train: batch must be in 1..4096");
        SR_REQUIRE(lr > 0.0 && lr < 1.0, "sr_learner_train: lr must be in (0, 1)");
        const double v = learned_train(l->L, (int)iterations, (int)batch, lr, seed, l->stream);
        if (learned_error(l->L, l->stream))
            throw SrError{SR_E_TIMEOUT, "a tensor-core wait of the learned preconditioner gave up"};
        if (loss) *loss = v;
    });
}

sr_status sr_learner_loss_grad(sr_learner* l, const float* feats, const float* target, uint32_t n, double* loss,
                               float* grad, float* out) {
    return guarded_free([&] {
        SR_REQUIRE(l && feats && target, "sr_learner_loss_grad: null argument");
        SR_REQUIRE(n >= 1 && n <= 4096, "sr_learner_loss_grad: n must be in 1..4096");
        const double v = learned_loss_grad(l->L, feats, target, (int)n, grad, out, l->stream);
        if (learned_error(l->L, l->stream))
            throw SrError{SR_E_TIMEOUT, "a tensor-core wait of the learned preconditioner gave up"};
        if (loss) *loss = v;
    });
}

sr_status sr_attach_learner(sr_ctx* c, sr_learner* l) {
    return guarded(c, [&] {
        SR_REQUIRE(c->cfg.heat, "sr_attach_learner: the context runs no heat pass");
        drop_step_graphs(c);
        SR_CUDA_TRY(cudaStreamSynchronize(c->stream));
        heat_attach_learned(c->heat, l ? l->L : nullptr);
        c->learner = l;
        for (sr_ctx* s : c->subs) {
            drop_step_graphs(s);
            SR_CUDA_TRY(cudaStreamSynchronize(s->stream));
            heat_attach_learned(s->heat, l ? l->L : nullptr);
            s->learner = l;
            if (!l && s->cfg.precond == SR_PRECOND_LEARNED) s->cfg.precond = SR_PRECOND_MG;
        }
        if (!l && c->cfg.precond == SR_PRECOND_LEARNED) c->cfg.precond = SR_PRECOND_MG;
    });
}

const char* sr_last_error(const sr_ctx* c) { return c ? c->error.c_str() : g_create_error.c_str(); }

}  // extern "C"

// ---- for the batch (batch.cu): one captured graph over many contexts' whole steps
sr_status sr_ctx_after_steps(sr_ctx* c) { return after_steps(c); }
unsigned sr_ctx_generation(const sr_ctx* c) { return c->generation; }
int sr_ctx_state(const sr_ctx* c) { return c->cur; }
bool sr_ctx_uploaded(const sr_ctx* c) { return c->uploaded; }
sr_status sr_ctx_guard(sr_ctx* c, const std::function<void()>& body) { return guarded(c, body); }

extern "C" {

cudaStream_t sr_ctx_stream(sr_ctx* c) { return c->stream; }

}  // extern "C"
