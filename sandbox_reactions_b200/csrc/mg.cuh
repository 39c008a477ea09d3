// mg.cuh — the multigrid V-cycle preconditioner of the implicit FLD solve (FP32).
//
// Levels: level 0 is the 5-point SPD system of a Newton pass (diagonal, coupling to the +x and +y neighbour, a gas
// mask); level l+1 aggregates 2x2 cells of level l with the Galerkin operator of piecewise-constant prolongation, which
// stays 5-point: the coarse diagonal sums the aggregate's diagonals less twice its internal couplings, a coarse
// coupling sums the two fine couplings crossing the aggregates' shared side (the reference's tile-MG does the same,
// crates/sr-engine/shaders/heat.wgsl:1315-1398). Smoothing is red-black Gauss-Seidel (global parity), V(pre, post),
// the post-smoother sweeping the colours in reverse so the cycle is symmetric. Big levels run as tile kernels that do
// all of a smoother's half-sweeps in shared memory (temporal blocking: the tile's halo is as deep as the half-sweeps);
// every level of at most kMgTailCells cells runs inside one CTA (the coarse tail, the reference's mg_coarse), and the
// coarsest level (at most 8 x 8) is solved exactly by its inverse, built once per Newton pass.
#pragma once

#include "common.cuh"

constexpr int kMgTailCells = 4096;   // levels at most this large are solved inside one CTA
constexpr int kMgMaxLevels = 16;

struct MgLevel {
    int w = 0, h = 0;
    float* c = nullptr;     // A_ii less the cell's couplings (>= 0; 1 where masked out): the diagonal is c + Σ couplings
    float* dx = nullptr;    // -A_{i,i+1}: coupling to the +x neighbour (0 at the edge or to a masked cell)
    float* dy = nullptr;    // -A_{i,i+w}
    uint8_t* mask = nullptr;  // 1: a cell of the system (a gas cell, or an aggregate holding one)
    float* b = nullptr;
    float* x = nullptr;   // the pre-smoother's iterate
    float* x2 = nullptr;  // the post-smoother's result (a second buffer: neighbouring tiles read x's halo meanwhile)
};

// CTAs of one smoother launch on a w x h level (each writes one grid-sum partial at level 0).
size_t mg_smooth_ctas(int w, int h);

struct Multigrid {
    int nlevels = 0;
    int tail = 0;  // first level handled by the tail kernel
    int pre = 2, post = 2;
    float omega = 1.0f;  // coarse-correction weight
    MgLevel L[kMgMaxLevels];
    float* coarse_inv = nullptr;  // the coarsest level's operator inverted (at most 64 x 64), per Newton pass

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
};
