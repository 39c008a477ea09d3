// learned.cuh — the learned preconditioner: a 4-level convolutional U-Net (110,153 parameters) mapping the
// Jacobi-scaled, rms-normalised residual and three operator features to the scaled error. Its 3x3 convolutions run as
// BF16 implicit GEMMs on the tcgen05 tensor cores with FP32 accumulation in TMEM (forward and data gradient); it is
// trained on the GPU by this file's kernels (weight gradients on the CUDA cores, Adam on FP32 master weights) on
// residual/error pairs that plain MG-PCG generates, and applied inside flexible PCG.
//
// The preconditioner is multiplicative: one MG V-cycle z₁ = M_mg r, then the network's estimate of the error that
// cycle leaves, z = z₁ + N(r − A z₁). The network therefore learns what the V-cycle misses (the samples are the
// V-cycle's remaining errors along MG-PCG solves), and with its head's weights at zero (the initial state) the
// preconditioner is exactly the V-cycle.
#pragma once

#include "common.cuh"
#include "mg.cuh"

struct Learner;
struct LearnedApply;

Learner* learned_create(int crop, int capacity, uint64_t seed);
void learned_destroy(Learner* L);
int learned_param_count();
void learned_get_params(Learner* L, float* theta);
void learned_set_params(Learner* L, const float* theta);

// Training pairs: begin on a w x h system (random crop positions), snapshot (r, e) every round of an MG-PCG solve of
// A e = r_0 from e = 0 — r the residual the round's V-cycle leaves, r_k − A z_k, and e the iterate it reaches, e_k + z_k
// — then end with the converged e: each snapshot's crops become samples (features of r, target e_final − e).
void learned_begin_collect(Learner* L, int w, int h, int crops, uint64_t seed);
void learned_snapshot(Learner* L, const MgLevel& level0, const float* r, const float* e, cudaStream_t s);
void learned_end_collect(Learner* L, const MgLevel& level0, const float* e_final, cudaStream_t s);
int learned_samples(Learner* L);

// `iterations` Adam steps on random batches of `batch` samples (the energy-norm loss below); returns the mean loss of
// the last 10 batches.
double learned_train(Learner* L, int iterations, int batch, double lr, uint64_t seed, cudaStream_t s);
// The loss — per crop the energy δᵀÂδ left by the correction (δ = target − output, Â the crop's Jacobi-scaled
// operator from the features) as a fraction of the target's — of the network on host features (n, 4, crop, crop)
// against targets (n, crop, crop), its gradient (param_count floats) and the output (n, crop, crop); for checks
// against the f64 CPU network.
double learned_loss_grad(Learner* L, const float* feats, const float* target, int n, float* grad, float* out,
                         cudaStream_t s);

// Inference inside the solve on a w x h world: z = z_base + N(r_in) on the gas cells (z_base optional; z may alias it),
// and <r_dot, z> into *rz_out.
LearnedApply* learned_apply_create(Learner* L, int w, int h);
void learned_apply_destroy(LearnedApply* A);
void learned_apply(LearnedApply* A, const MgLevel& level0, const float* r_in, const float* z_base, const float* r_dot,
                   float* z, double* part, unsigned* counter, double* rz_out, cudaStream_t s);
// Nonzero when a tensor-core wait of the learner's kernels gave up (its bound expired).
int learned_error(Learner* L, cudaStream_t s);
