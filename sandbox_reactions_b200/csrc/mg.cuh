// mg.cuh — the multigrid V-cycle preconditioner of the implicit FLD solve (FP32).
//
// Levels: level 0 is the 5-point SPD system of a Newton pass (diagonal, coupling to the +x and +y neighbour, a gas
// mask); level l+1 aggregates 2x2 cells of level l (the reference's tile-MG aggregates the same way,
// crates/sr-engine/shaders/heat.wgsl:1315-1398, with constant weights). Level 1 is level 0's plain aggregation; from
// level 1 on, each aggregate's basis function is weighted: the fine weights t come from two red-black Gauss-Seidel
// sweeps on A t = 0 from t = 1, scaled per aggregate to a largest weight of 1, so that cells the mass term dominates
// (whose error the smoother removes) weigh little in the coarse space. The aggregates do not overlap, so the Galerkin operator P^T A P stays 5-point: a coarse coupling sums
// t_j t_k d_jk over the two fine couplings crossing the aggregates' shared side, the coarse mass term is (P^T A t)_I.
// Restriction is P^T (r_c = sum t_j r_j), prolongation P (x_j += t_j x_c). Smoothing is red-black Gauss-Seidel
// (global parity), V(pre, post), the post-smoother sweeping the colours in reverse so the cycle is symmetric. Big
// levels run as tile kernels that do all of a smoother's half-sweeps in shared memory (temporal blocking: the tile's
// halo is as deep as the half-sweeps); every level of at most kMgTailCells cells runs inside one CTA (the coarse tail,
// the reference's mg_coarse), and the coarsest level (at most 4 x 4) is solved exactly by its inverse, built once per
// Newton pass.
#pragma once

#include "common.cuh"

constexpr int kMgTailCells = 4096;   // levels at most this large are solved inside one CTA
constexpr int kMgMaxLevels = 16;

struct MgLevel {
    int w = 0, h = 0;
    float* c = nullptr;     // A_ii less the cell's couplings (1 where masked out): the diagonal is c + Σ couplings
    float* dx = nullptr;    // -A_{i,i+1}: coupling to the +x neighbour (0 at the edge or to a masked cell)
    float* dy = nullptr;    // -A_{i,i+w}
    uint8_t* mask = nullptr;  // 1: a cell of the system (a gas cell, or an aggregate holding one)
    float* b = nullptr;
    float* x = nullptr;   // the pre-smoother's iterate
    float* x2 = nullptr;  // the post-smoother's result (a second buffer: neighbouring tiles read x's halo meanwhile)
    float* t = nullptr;   // the cell's weight in its aggregate's basis function (null: 1, level 0)
    int* err = nullptr;   // set to 1 when a bounded wait of a smoother gave up (its TMA boxes never landed)
};

// At most this many CTAs in one smoother launch on a w x h level (each writes one grid-sum partial at level 0).
size_t mg_smooth_ctas(int w, int h);

struct Multigrid {
    int nlevels = 0;
    int tail = 0;  // first level handled by the tail kernel
    int pre = 2, post = 2;
    float omega = 1.0f;  // coarse-correction weight
    MgLevel L[kMgMaxLevels];
    float* coarse_inv = nullptr;  // the coarsest level's operator inverted (at most 64 x 64), per Newton pass
    float* tail_img = nullptr;    // the coarse tail's shared-memory image (coefficients, inverse diagonals, weights,
                                  // masks, the coarsest inverse), packed once per Newton pass
    int* err = nullptr;           // the smoothers' error flag (MgLevel::err of every level)

    void create(int w, int h, int pre, int post);
    void destroy();
    size_t bytes() const;
    // Level 0's couplings (fixed within a step): dx, dy and mask, from the f64 face coefficients and the gas mask.
    void set_couplings(const double* kx, const double* ky, const uint8_t* gas, cudaStream_t s);
    // Every coarse level's operator, once level 0's c (written by the caller, per Newton pass) is in place.
    void coarsen(cudaStream_t s);
    // z = M r (level-0 b := r, x2 := z), and <r, z> into *rz_out (a one-launch grid sum over `part` and `counter`).
    void apply(const float* r, float* z, double* part, unsigned* counter, double* rz_out, cudaStream_t s);
    // Picks each level's smoother tile by timing (after the first coarsening, outside any stream capture).
    void autotune(cudaStream_t s);
    int tile[kMgMaxLevels] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    bool tuned = false;
    // The device time (ms) of one launch of level 0's pre- and post-smoother on the last applied system, each
    // averaged over `reps` launches with `flush` (flush_bytes, larger than L2) rewritten before each: a timing hook.
    void time_level0(int reps, void* flush, size_t flush_bytes, cudaStream_t s, double* pre_ms, double* post_ms);
    // Whether a smoother's bounded wait gave up since the last call (reads and clears the flag; waits for `s`).
    bool error(cudaStream_t s);
};
