/*
 * sr_cuda.h — the C ABI of the B200 field update (hydro + FFT gravity + implicit FLD) of sandbox_reactions.
 *
 * This is the drop-in boundary for the reference's `sr-engine` step API (Rust over wgpu). Every entry point below names
 * the reference interface it replaces (paths relative to the reference project). A thin Rust `extern "C"` crate maps
 * 1:1 onto these functions; Python reaches them through ctypes.
 *
 * Conventions (the reference's canonical layout, crates/sr-engine/src/state.rs:1-38):
 *   - planes are f32, channel-major, row-major inside a plane: value (c, x, y) at c*W*H + y*W + x, y down;
 *   - channels: 0 Σ (surface density), 1 Σu, 2 Σv, 3 E (energy per area), then, with `channels` 14 (reference mode),
 *     the ten species' mass fractions X_H, X_He, X_C, X_O, X_Ne, X_Mg, X_Si, X_S, X_Fe, X_n (state.rs:29-35);
 *   - x faces: (W+1)*H values, face (x, y) between cells (x-1, y) and (x, y); y faces: W*(H+1) values, face (x, y)
 *     between (x, y-1) and (x, y); a flux is positive toward +x / +y (crates/sr-physics/src/reference/heat.rs:94-101).
 *
 * Ownership and threading: a context owns all of its device memory and one CUDA stream; host buffers are borrowed for
 * the duration of a call only. One host thread per context (the reference's Step is !Sync). No callbacks.
 *
 * Errors: every call returns an sr_status. An unconverged implicit solve is a report flag, not an error
 * (crates/sr-engine/src/step/heat.rs:215-235). sr_last_error() gives the message of the last failed call.
 */
#ifndef SR_CUDA_H
#define SR_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SR_ABI_VERSION 3u

typedef enum sr_status {
    SR_OK = 0,
    SR_E_INVALID = 1,   /* refused arguments: the FftError / StateError / TwinError analogue */
    SR_E_NONFINITE = 2, /* a non-finite value in the state: the CLI's exit 5 (reduce.wgsl guard) */
    SR_E_TIMEOUT = 3,   /* a bounded device-side wait expired */
    SR_E_CUDA = 4,      /* a CUDA runtime error */
    SR_E_NOMEM = 5,     /* device allocation failed */
    SR_E_UNSUPPORTED = 6
} sr_status;

/* Edge modes (crates/sr-physics/src/reference/hydro.rs:183-188; scene "edge"). */
enum { SR_EDGE_BOUNCE = 0, SR_EDGE_LEAVE = 1 };
/* Slope limiters: the reference's monotonised central (hydro.rs:283-289) and minmod. */
enum { SR_LIMITER_MC = 0, SR_LIMITER_MINMOD = 1 };
/* Gravity kernels: the reference's exact self cell K(0,0) = -4 ln(1+sqrt 2) G (reference/grav.rs:25-34), or
 * Plummer-softened -G / sqrt(r^2 + eps^2). */
enum { SR_KERNEL_SELF_CELL = 0, SR_KERNEL_SOFTENED = 1 };
/* Preconditioners of the implicit FLD solve (crates/sr-engine/src/step/heat.rs:137-141), plus the learned one. */
enum { SR_PRECOND_MG = 0, SR_PRECOND_JACOBI = 1, SR_PRECOND_LEARNED = 2 };

/*
 * The run's configuration: the world, the scene's switches, the scheme's choices and physics.json's constants
 * (assets/physics.json; crates/sr-engine/src/step/mod.rs:399-527 takes them as &Physics/&Passes/&HeatSetup).
 * Fill with sr_config_default() and override fields.
 */
typedef struct sr_config {
    uint32_t struct_size;     /* sizeof(sr_config): guards against a header/library mismatch */
    uint32_t width, height;   /* multiples of 8, 8..4096 */
    uint32_t channels;        /* 4: Σ, Σu, Σv, E under the config-mode EOS (γ, μ); 14: reference mode — the reference's
                                 own EOS (γ = 2, μ and Y_e of each cell's species, the cold pressures of the K pairs),
                                 species advected, the hold (held cells behind reflecting walls) */
    uint32_t edge;            /* SR_EDGE_* */
    uint32_t limiter;         /* SR_LIMITER_* */
    uint32_t thermal_bracket; /* 1: the reference's HOT_FACE bracket on Σ and Π slopes (hydro.rs:310-331) */
    uint32_t gravity;         /* switches (reference/mod.rs:46-56) */
    uint32_t hydro;
    uint32_t heat;
    uint32_t kernel;          /* SR_KERNEL_* */
    uint32_t precond;         /* SR_PRECOND_* */
    uint32_t flux_limiter;    /* 1: Levermore-Pomraning λ(R); 0: λ = 1/3 (heat.rs TestFlags) */
    uint32_t opacity_plane;   /* 1: κ per cell from sr_upload_opacity; 0: κ = kappa0 everywhere */
    uint32_t mg_pre, mg_post; /* red-black sweeps before / after the coarse correction: V(mg_pre, mg_post), 1..4 */
    uint32_t max_passes;      /* Newton passes per implicit step (reference heat.rs:51 MAX_PASSES = 128) */
    uint32_t max_rounds;      /* PCG rounds over all passes (heat.rs:52 MAX_ROUNDS = 4096) */
    uint32_t pin_temperature; /* heat.rs TestFlags::pin_temperature */
    uint32_t active_box;      /* 1: the active box (crates/sr-engine/src/step/boxfit.rs, BoxMode::Fit): only the bounding
                                 box of the cells with Σ >= Σ_vac, grown by 8 and rounded out to multiples of 8, is
                                 stepped, its FFT sized to it, refit before step 0 and after every 16th step's P9; the
                                 vacuum outside is left as it is. 0: the whole world (BoxMode::WholeWorld) */
    uint32_t reserved[3];
    double gamma;             /* adiabatic index: Π = (γ-1) Σ ε_th, c² = γΠ/Σ (the reference hardwires γ = 2) */
    double mu;                /* mean molecular weight: T = μ (γ-1) ε_th (the reference's T = μ ε_th at γ = 2) */
    double t_floor;           /* physics.json t_floor */
    double sigma_vac;         /* physics.json sigma_vac */
    double sigma_floor;       /* physics.json sigma_floor */
    double cfl;               /* physics.json cfl */
    double eta_g;             /* physics.json eta_g */
    double G;                 /* gravitational constant (1 in sandbox units) */
    double softening;         /* ε of SR_KERNEL_SOFTENED, in cells */
    double a_r;               /* radiation constant */
    double c_sb;              /* c in the flux law */
    double kappa0;            /* opacity when no plane is given */
    double k_cond;            /* conduction coefficient */
    double chi;               /* > 0: the constant-diffusivity test flag (u = T, D_f = χ C_f) */
    double solve_tol;         /* FP64 relative residual the last Newton pass's solve reaches (1e-8); earlier passes
                                 are solved only as far as the Newton iteration needs */
    double newton_heat;       /* Newton stop: Σ C|ΔT| <= newton_heat Σ C T⁰ (1e-6) ... */
    double newton_cell;       /* ... and every |ΔT| <= newton_cell T (1e-3): the reference GPU path's rule */
    double dt_fixed;          /* > 0: every step runs on this Δt instead of the CFL/gravity one */
    double dt_cap;            /* > 0: Δt_{n+1} = min(Δt_{n+1}, dt_cap) (reference/mod.rs:213-216) */
    double mg_omega;          /* weight of the multigrid's coarse correction (0: the library's default) */
    double inner_tol;         /* smallest residual reduction asked of one FP32 inner solve (0: default 1e-5) */
    double reserved_d[2];
    /* reference mode (channels 14): physics.json's constants the 4-channel field update does not read */
    double k1e, k2e;          /* the electrons' cold-pressure pair K₁, K₂; both 0: off (eos.rs:150-190) */
    double k1n, k2n;          /* neutron matter's pair */
    double kappa_dust, t_dust; /* the dust opacity stand-in of the radiation force (reference/hydro.rs:365-382) */
    double sigma_hold, eta_hold, r_hold; /* the hold's Σ, ε_th/ε_cold and gate radius (reference/floors.rs:94-110) */
    double m_tov;             /* m_tov_sb: the hold's disk-mass gate (floors.rs:90-92; assets/calibration.json) */
} sr_config;

/* Δt record (crates/sr-engine/src/step/dt.rs:51-61). */
typedef struct sr_dt_report {
    double dt;          /* Δt_n of the last step run */
    double dt_next;     /* Δt_{n+1} */
    uint64_t steps;     /* steps run since the context was made */
    double sim_time;    /* Σ Δt in step order, f64 */
    int32_t non_finite; /* 1 when the guard found a non-finite value */
    int32_t nf_channel; /* its channel */
    int64_t nf_cell;    /* its cell index y*W+x */
} sr_dt_report;

/* Implicit-step report (crates/sr-engine/src/step/heat.rs:215-235, reference/heat.rs:106-124). */
typedef struct sr_heat_report {
    double dt;            /* Δt the step covered; 0 when P5 did not run */
    uint32_t passes;      /* Newton passes */
    uint32_t rounds;      /* preconditioned CG rounds over all passes */
    uint32_t refinements; /* FP64 outer refinement sweeps over all passes */
    uint32_t converged;   /* 0: ceiling reached, committed by limited fluxes */
    double delta;         /* heat-balance closure δ */
    double radiated;      /* heat lost to vacuum and through the edges */
    double rel_residual;  /* FP64 ||b - A u|| / ||b|| of the last pass's solve */
    uint32_t fallback_used; /* 1: the learned preconditioner stalled and plain MG-PCG finished the solve */
    uint32_t precond;       /* SR_PRECOND_* that finished the last solve */
} sr_heat_report;

/* Per-pass device time of the last sr_step call with timing on (crates/sr-engine/src/step/mod.rs:171-350). */
typedef struct sr_cost {
    uint32_t steps;
    uint32_t pad;
    double gravity_ms;   /* P2 */
    double hydro_ms;     /* P4, its mid-step gravity solve included */
    double heat_ms;      /* P5 */
    double floors_ms;    /* P8 */
    double dt_ms;        /* P9 */
    double total_ms;
    double hydro_update_ms; /* the fused hydro update kernel alone (the roofline kernel) */
    uint32_t hydro_update_launches;
    uint32_t pad2;
    uint64_t kernel_launches; /* this library's kernel launches during the call */
} sr_cost;

/* Fills `cfg` with physics.json's shipped constants and the reference's scheme (MC, bounce, γ = 2, self-cell kernel). */
void sr_config_default(sr_config* cfg);

/* Returns SR_ABI_VERSION. */
uint32_t sr_abi_version(void);

typedef struct sr_ctx sr_ctx;

/* Step::with_heat / with_passes / with_neutrino_heating (crates/sr-engine/src/step/mod.rs:399-527): validates `cfg`
 * (World 8..4096 per axis, multiple of 8; the reference's WorldConfig::validate, state.rs:72-90) and allocates every
 * buffer of the step on the current device. */
sr_status sr_create(const sr_config* cfg, sr_ctx** out);
void sr_destroy(sr_ctx* ctx);

/* State::upload (crates/sr-engine/src/state.rs:251): `nplanes` canonical f32 planes. Resets the step count and the
 * clock, solves P2 on the state and reduces Δt_0 from it (reference/mod.rs:129-177, Twin::new). */
sr_status sr_upload(sr_ctx* ctx, const float* planes, uint32_t nplanes);
/* State::readback (state.rs:273). */
sr_status sr_readback(sr_ctx* ctx, float* planes, uint32_t nplanes);
/* State::upload_held / read_held (crates/sr-engine/src/state.rs:198-250): the hold's mask, one word per cell, row-major,
 * nonzero where a cell is held — reference mode only (channels 14). sr_upload clears the mask and applies the hold's
 * rule to the new state (reference/mod.rs:129-177); sr_upload_held then replaces the mask (a dump's, resumed). */
sr_status sr_upload_held(sr_ctx* ctx, const uint32_t* mask);
sr_status sr_read_held(sr_ctx* ctx, uint32_t* mask);
/* The opacity plane κ (W*H f32) read when cfg.opacity_plane is 1. */
sr_status sr_upload_opacity(sr_ctx* ctx, const float* kappa);

/* Step::run (step/mod.rs:703-718): `steps` steps in the reference's order P1 → P2 → P4 → P5 → P8 → P9
 * (reference/mod.rs:264-297). Returns SR_E_NONFINITE when the guard finds a non-finite value. */
sr_status sr_step(sr_ctx* ctx, uint32_t steps);

/* Step::read_dt (step/dt.rs:173). */
sr_status sr_read_dt(sr_ctx* ctx, sr_dt_report* out);
/* Step::read_heat (step/heat.rs:499-512). */
sr_status sr_read_heat(sr_ctx* ctx, sr_heat_report* out);
/* Step::gravity_field (step/mod.rs:532-534): P2's field of the state the last step started from; W*H each. With the
 * active box, P2 runs over the box: its field inside the box, 0 outside. */
sr_status sr_gravity_field(sr_ctx* ctx, float* gx, float* gy, float* phi);
/* Step::read_heat_flux (step/heat.rs:542-548): the last implicit step's solved face fluxes, (W+1)*H and W*(H+1). */
sr_status sr_heat_flux(sr_ctx* ctx, float* fx, float* fy);

/* The records a state dump carries beyond the cells, for resuming a run where it stopped (dump_state / load_dump,
 * crates/sr-engine/src/dump.rs:355-410). sr_set_clock is Step::restore (step/latch.rs:493-510): the next step's index
 * is `steps`, the sim time goes on from `sim_time`, Δt_n = dt and the next step's Δt = dt_next, the guard's finding
 * cleared. sr_upload resets the clock, so the resume calls follow it. With the active box the box stays the one fit at
 * the upload and the refits follow the restored step index. */
sr_status sr_set_clock(sr_ctx* ctx, uint64_t steps, double sim_time, double dt, double dt_next);
/* Step::heat_rate / set_heat_rate (step/heat.rs:550-582): each cell's P5 rate (T − T⁰)/Δt in the last step, W*H f32
 * row-major — the next step's first iterate is T⁰ + rate·Δt. sr_upload zeroes it; sr_set_heat_rate after the upload
 * restores a dump's (NULL: zeros). The context must run P5. */
sr_status sr_read_heat_rate(sr_ctx* ctx, float* rate);
sr_status sr_set_heat_rate(sr_ctx* ctx, const float* rate);
/* Step::side_flux (step/heat.rs:584-589): the cell-centred F (F_x and F_y, W*H f32 each) that the next step's P4
 * pushes with — reference mode with P5 only (channels 14, heat on). sr_upload zeroes it (the first step takes no
 * radiation force, reference/mod.rs:122-123); sr_set_side_flux after the upload restores a dump's. */
sr_status sr_read_side_flux(sr_ctx* ctx, float* fx, float* fy);
sr_status sr_set_side_flux(sr_ctx* ctx, const float* fx, const float* fy);

/* Step::set_edge_mode (step/mod.rs:544-548). */
sr_status sr_set_edge_mode(sr_ctx* ctx, uint32_t edge);
/* Step::set_heat_precond (step/heat.rs:595-599). */
sr_status sr_set_heat_precond(sr_ctx* ctx, uint32_t precond);
/* Step::set_heat_rounds (step/heat.rs:529-533): the ceilings of the implicit step. */
sr_status sr_set_heat_limits(sr_ctx* ctx, uint32_t max_passes, uint32_t max_rounds);
/* BoxFit::read (crates/sr-engine/src/step/boxfit.rs:33-53, 152-172): the active box as it stands — origin and size
 * in cells (the whole world when the box is off or no cell holds gas), the FFT size per axis the step's gravity runs
 * on, and the fits made since the upload. */
typedef struct sr_box_report {
    uint32_t x0, y0, w, h;
    uint32_t fft_w, fft_h;
    uint64_t fits;
} sr_box_report;
sr_status sr_read_box(sr_ctx* ctx, sr_box_report* out);

/* Step::set_timing / read_cost (step/mod.rs:722-777). `on`: 0 off; 1 each step's device time (total_ms) as the steps
 * normally run — after the first step, one captured graph per step — with the per-pass fields left 0; 2 the per-pass
 * breakdown, the passes launched one by one (the implicit step still one captured graph after the first step). */
sr_status sr_set_timing(sr_ctx* ctx, int32_t on);
sr_status sr_read_cost(sr_ctx* ctx, sr_cost* out);

/* The first Newton pass's linear system of one implicit step on the uploaded state, solved alone to cfg.solve_tol
 * with `precond` — the reference's heat_first_system / apply_heat_precond test hooks (step/heat.rs:609-672).
 * `ms` gets the device time of the solve, `rounds` its preconditioned CG rounds; `x` (optional, W*H f64) the solution;
 * `fallback` (optional) 1 when the learned preconditioner stalled and MG-PCG finished the solve. */
sr_status sr_heat_first_solve(sr_ctx* ctx, double dt, uint32_t precond, double* ms, uint32_t* rounds,
                              double* rel_residual, double* x, uint32_t* fallback);

/* A benchmark hook with no counterpart in the reference: the device time of one launch of the multigrid's level-0
 * pre-smoother and post-smoother (the step's dominant kernels) on the last solved implicit system, each averaged over
 * `reps` launches timed with CUDA events on the context's stream, a 256 MB buffer rewritten before each launch so the
 * level's planes come from HBM. 0 when the world is small enough that the coarse tail covers level 0. */
sr_status sr_time_smoother(sr_ctx* ctx, uint32_t reps, double* pre_ms, double* post_ms);

/* ---- The learned preconditioner — no counterpart in the reference (its preconditioners are MG and Jacobi,
 * step/heat.rs:137-141). A 4-level convolutional U-Net (widths 8/16/32/64, 110,153 parameters) maps the
 * Jacobi-scaled, rms-normalised residual left by one MG V-cycle, with three operator features, to the error that
 * cycle leaves; the preconditioner is the V-cycle plus the network's correction, applied inside flexible CG. The 3x3
 * convolutions run as BF16 implicit GEMMs on the tcgen05 tensor cores with FP32 accumulation; the network is trained on
 * the GPU on (residual, error) pairs that plain MG-PCG generates. When it stalls (less than a 100x residual reduction
 * after 24 rounds, or a breakdown) plain MG-PCG finishes the solve and the report's fallback_used is set. A learner
 * owns its weights, sample store and stream; several contexts may share one (one host thread at a time). */
typedef struct sr_learner sr_learner;
/* `crop` (a multiple of 8 in 16..512): the side of the training crops; `capacity`: samples held. */
sr_status sr_learner_create(uint32_t crop, uint32_t capacity, uint64_t seed, sr_learner** out);
void sr_learner_destroy(sr_learner* learner);
uint32_t sr_learner_param_count(void);
/* Parameters, per layer W[cout][3][3][cin] then b[cout], f32. */
sr_status sr_learner_get_params(sr_learner* learner, float* theta);
sr_status sr_learner_set_params(sr_learner* learner, const float* theta);
/* Solves the first Newton pass's system of ctx's implicit step with dt by MG-PCG from zero and stores `crops` random
 * crops of every round's (residual left by the V-cycle, error remaining) as samples; `samples` gets how many. */
sr_status sr_learner_collect(sr_learner* learner, sr_ctx* ctx, double dt, uint32_t crops, uint64_t seed,
                             uint32_t* samples);
/* `iterations` Adam steps on random batches of `batch` samples; `loss` the mean loss of the last 10 batches. The loss
 * of a crop is the energy δᵀÂδ left by the correction (δ = target − output, Â the crop's Jacobi-scaled operator) as a
 * fraction of the target's energy. */
sr_status sr_learner_train(sr_learner* learner, uint32_t iterations, uint32_t batch, double lr, uint64_t seed,
                           double* loss);
/* The network's loss on host features (n, 4, crop, crop) against targets (n, crop, crop), the loss gradient
 * (param_count floats) and the output (n, crop, crop) — a hook for checking the kernels against a CPU network. */
sr_status sr_learner_loss_grad(sr_learner* learner, const float* feats, const float* target, uint32_t n, double* loss,
                               float* grad, float* out);
/* Makes `learner` ctx's SR_PRECOND_LEARNED (NULL detaches it; a learned context then falls back to MG). The learner
 * must outlive the attachment. */
sr_status sr_attach_learner(sr_ctx* ctx, sr_learner* learner);

/* ---- Batches: many independent worlds of uneven sizes advanced together (the reference runs one world per Step,
 * crates/sr-engine/src/step/mod.rs:367-718; a batch is N such Steps whose kernels overlap on one GPU). Each world keeps
 * its own context and stream; sr_batch_step hands the worlds to a pool of host threads balanced by cell count, so the
 * worlds' kernels (and their implicit solves' host decisions) interleave on the device. */
typedef struct sr_batch sr_batch;
/* `count` configurations; `threads` host threads (0: one per world, at most 16). */
sr_status sr_batch_create(const sr_config* cfgs, uint32_t count, uint32_t threads, sr_batch** out);
void sr_batch_destroy(sr_batch* b);
/* World `index`: its planes (as sr_upload) and, when its configuration asks for one, its opacity plane. */
sr_status sr_batch_upload(sr_batch* b, uint32_t index, const float* planes, const float* kappa);
/* Every world `steps` steps. `device_ms` (optional) gets the device time from the first world's start to the last
 * world's end. */
sr_status sr_batch_step(sr_batch* b, uint32_t steps, double* device_ms);
sr_status sr_batch_readback(sr_batch* b, uint32_t index, float* planes);
/* The context of world `index` (for its reports); owned by the batch. */
sr_ctx* sr_batch_ctx(sr_batch* b, uint32_t index);

/* P2's gravity solve (φ and g = -∇φ of Σ, as a context's) with no device allocation — no counterpart in the
 * reference. For callers that cannot allocate device memory: hosts that own every byte of device memory and hand their
 * plug-ins buffers (no cudaMalloc allowed), or loops that cannot afford cudaMalloc's device-wide synchronisation. The
 * caller passes device buffers: `sigma` (W*H) in, `phi`, `gx`, `gy` (W*H each) out, and the CUDA stream (NULL: the
 * default stream) as `stream`. The scratch lives in static device arrays sized for worlds up to 256 x 256 cells, held
 * by every GPU that loads the library until exit; a larger world is refused with SR_E_INVALID. The first call on a
 * device looks up the arrays and uploads the kernel's spectrum; so does every call whose padded FFT size, kernel, G or
 * (softened kernel only) softening differs from the previous call's on that device. Such a call copies from the host
 * and waits for `stream`, blocking the host: it must not be made during a stream capture. Calls share the arrays:
 * calls whose work overlaps on the GPU race. Uses cfg's width, height, kernel, G, softening and sigma_vac. */
sr_status sr_gravity_solve_static(const sr_config* cfg, const float* sigma, float* phi, float* gx, float* gy,
                                  void* stream);

/* The message of the last failed call on `ctx` (or of the last failed sr_create when ctx is NULL). */
const char* sr_last_error(const sr_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* SR_CUDA_H */
