// heat.cuh — P5, the implicit flux-limited diffusion step: Newton passes, each an SPD 5-point system solved by
// multigrid-preconditioned CG in FP32 inside an FP64 iterative-refinement loop.
#pragma once

#include "common.cuh"

struct HeatSolver;

// Reference mode's sides (reference/heat.rs:215-231): T from the reference's EOS (the cold energy of the K pairs'
// tables taken off), C = Σ/μ and κ = κ₀(1 + X_H) (+ κ_dust Z_met below T_dust) of each cell's species, read from the
// 14-plane state.
struct HeatRef {
    int on = 0;
    const float* table = nullptr;  // device: u_e, Δ ln u_e, u_n, Δ ln u_n at the 512 nodes
    int cold_e = 0, cold_n = 0;
    double kappa_dust = 0.0, t_dust = 0.0;
};

HeatSolver* heat_create(const sr_config& cfg, cudaStream_t s);
void heat_set_reference(HeatSolver* hs, const HeatRef& R);
// The last step's face fluxes on the device ((W+1)*H and W*(H+1) floats).
void heat_flux_planes(const HeatSolver* hs, const float** fx, const float** fy);
// Each cell's rate of the last step (W*H doubles on the device), the next step's first iterate.
double* heat_rate_plane(HeatSolver* hs);
// Whether a bounded device wait of the solver's multigrid gave up since the last call (clears the flag).
bool heat_wait_error(HeatSolver* hs, cudaStream_t s);
void heat_destroy(HeatSolver* hs);
// One implicit step of length *dt_dev on the 4 planes U (E changes), κ from `kappa` (W*H) or cfg.kappa0.
void heat_step(HeatSolver* hs, float* U, const float* kappa, const double* dt_dev, cudaStream_t s, sr_heat_report* rep);
void heat_read_flux(HeatSolver* hs, float* fx, float* fy);
// The last implicit step's report (waits for it when the step ran as a captured graph).
void heat_report(HeatSolver* hs, cudaStream_t s, sr_heat_report* rep);
// Adds the kernels the captured steps launched since the last count to the library's launch count (waits for them).
void heat_account_launches(HeatSolver* hs, cudaStream_t s);
// The implicit step as part of a larger captured graph (a context's whole step, a batch's): possible once the solver
// runs under device control (MG or Jacobi, after its first step tuned the multigrid). heat_prepare_capture (outside any
// capture) writes the control block; heat_capture_step appends the step to the capture in progress on `s` (root: the
// graph being captured; returns its top-level kernel count); heat_graph_launched marks its report as pending.
bool heat_capturable(const HeatSolver* hs);
void heat_prepare_capture(HeatSolver* hs, cudaStream_t s);
long long heat_capture_step(HeatSolver* hs, float* U, const float* kappa, const double* dt_dev, cudaStream_t s,
                            cudaGraph_t root);
void heat_graph_launched(HeatSolver* hs);
// Forgets the last step's rates (a new state was uploaded).
void heat_reset(HeatSolver* hs, cudaStream_t s);
// The last step's rates as f32 into `dst` (W*H floats on the device), or set from `src` (nullptr: zeros): the rate a
// dump carries (crates/sr-engine/src/step/heat.rs:550-582).
void heat_rate_to_f32(HeatSolver* hs, float* dst, cudaStream_t s);
void heat_rate_from_f32(HeatSolver* hs, const float* src, cudaStream_t s);
void heat_set_precond(HeatSolver* hs, uint32_t precond);
void heat_set_limits(HeatSolver* hs, uint32_t max_passes, uint32_t max_rounds);
// The first Newton pass's system of a step of length dt, solved alone (timed on the device); `fallback` gets 1 when
// the learned preconditioner stalled and MG-PCG finished.
void heat_first_solve(HeatSolver* hs, const float* U, const float* kappa, double dt, uint32_t precond, cudaStream_t s,
                      double* ms, uint32_t* rounds, double* rel_residual, double* x, uint32_t* fallback);

struct Learner;
// Makes `L` (or nothing, when null) the solver's SR_PRECOND_LEARNED: one V-cycle plus the network's correction.
void heat_attach_learned(HeatSolver* hs, Learner* L);
// Training samples for `L` from an MG-PCG solve of the first Newton pass's system of a step of length dt; returns how
// many were added.
int heat_collect(HeatSolver* hs, Learner* L, const float* U, const float* kappa, double dt, int crops, uint64_t seed,
                 cudaStream_t s);
// The level-0 smoothers of the last solved system, timed alone (mg.cuh time_level0): a benchmark hook.
void heat_time_smoother(HeatSolver* hs, int reps, cudaStream_t s, double* pre_ms, double* post_ms);
