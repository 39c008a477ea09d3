// hydro_ref.cuh — reference mode (14 channels): P4 with the reference's own EOS, species and held cells; P8's floors
// and the hold; P9's Δt terms. The 4-channel kernels of hydro.cuh stay the config-mode path.
#pragma once

#include "common.cuh"
#include "hydro.cuh"

constexpr int kRefSpecies = 10;
constexpr int kRefChannels = 4 + kRefSpecies;
constexpr int kColdPoints = 512;  // eos.rs:15

// The run's reference-mode constants (f32 on the device, as the reference's GPU passes upload them).
struct RefConst {
    int w, h, edge, limiter, bracket;
    int cold_e, cold_n;            // the electrons' / neutrons' K pair on
    float k1e, k1e_k2e;            // K₁ₑ and K₁ₑ/K₂ₑ: P = K₁x² / (1 + (K₁/K₂)√x)
    float k1n, k1n_k2n;
    float sigma_vac, sigma_floor, t_floor;
    float kappa0, inv_c_sb, kappa_dust, t_dust;
    float sigma_hold, eta_hold, r_hold, m_tov;
    const float* table;            // 4 x 512: u_e(node), Δ ln u_e, u_n(node), Δ ln u_n (eos.rs:81-131)
};

// The u(x) tables of a run's K pairs in the device layout above, built on the host in f64 (eos.rs:81-98).
void ref_cold_tables(const sr_config& cfg, float* host4x512);

struct RefArgs {
    RefConst R;
    const double* dt;      // device Δt_n
    const float* U;        // 14 planes in
    float* Uout;           // 14 planes out
    const uint8_t* held;   // the hold's mask (1: held)
    const float* gx;       // P2's field of the start state (nullptr: no gravity)
    const float* gy;
    float* src;            // the half step's Σ_src (source pass out, update in)
    float* src_free;       // the same with the held cells emptied
    const float* phim;     // the half step's field
    const float* gxm;
    const float* gym;
    const float* gxp;      // the half step's field of the free cells (the pull on the held ones)
    const float* gyp;
    const float* radx;     // the cell-centred flux of the radiation force (nullptr: none)
    const float* rady;
    float* push;           // 2 planes: each cell's radiation push (for the take-back)
    double* part;          // per CTA: kick x, kick y, push x, push y, |push|
    float* part_best;      // per CTA: the densest free Σ_src and its cell
    int* part_idx;
    double* fin;           // [kick x, kick y, densest, push x, push y, |push|]
};

int ref_hydro_blocks(int w, int h);
void ref_hydro_source_launch(const RefArgs& A, cudaStream_t s);
void ref_hydro_update_launch(const RefArgs& A, int gravity, cudaStream_t s);
// The take-backs (the radiation force's net push, gravity's net kick) and the sticky wall on the updated state.
void ref_hydro_finalize_launch(const RefArgs& A, cudaStream_t s);

// The cell-centred flux the next step's radiation force reads: the mean of a cell's two faces on each axis
// (reference/heat.rs:100-112).
void ref_cell_flux_launch(const float* fx, const float* fy, float* radx, float* rady, int w, int h, cudaStream_t s);

// P8's floors (floors.rs:124-175) in place.
void ref_floors_launch(const RefConst& R, float* U, cudaStream_t s);
// The hold (floors.rs:196-243) and/or P9's per-CTA Δt terms with the 14-channel guard; then, with `do_dt`, the
// finalize into `rec`.
void ref_hold_dt_launch(const RefConst& R, float* U, uint8_t* held, const float* gx, const float* gy, int do_hold,
                        int do_dt, float* part_rate, float* part_g, long long* part_nf, double cfl, double eta_g,
                        double dt_fixed, double dt_cap, DtRecord* rec, cudaStream_t s);
