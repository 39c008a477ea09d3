// hydro.cuh — P4 (hydro), P8 (floors) and P1/P9 (Δt) kernel entry points.
#pragma once

#include "common.cuh"

enum { kHydroUpdate = 0, kHydroSource = 1, kHydroUpdateGrav = 2 };

// The Δt record kept on the device (crates/sr-engine/src/step/dt.rs:51-61): steps never wait on the host for it.
struct DtRecord {
    double dt;        // Δt_n of the last step
    double dt_next;   // Δt_{n+1}
    double sim_time;  // Σ Δt, f64
    unsigned long long steps;
    int non_finite;
    int nf_channel;
    long long nf_cell;
    unsigned long long nf_step;
};

struct HydroArgs {
    HydroConst H;
    const double* dt;          // device Δt_n
    const float* U;            // state in: 4 planes
    float* Uout;               // state out: 4 planes (kHydroUpdate*)
    const float* gx;           // P2's field of the start state (nullptr: no gravity)
    const float* gy;
    float* src;                // kHydroSource: out; kHydroUpdateGrav: in (Σ_src,mid)
    const float* phim;         // the half step's φ, g (kHydroUpdateGrav)
    const float* gxm;
    const float* gym;
    double* part_d;            // per-CTA partials: 6 doubles (kick x, y, escaped Σ, Σu, Σv, E)
    float* part_best;          // per-CTA densest Σ_src,mid and its cell
    int* part_idx;
    double* report;            // [kick x, kick y, densest, escaped Σ, Σu, Σv, E]
    int* err;                  // set to 1 when a bounded wait of the kernel gave up (its TMA box never landed)
};

size_t hydro_smem_bytes();
int hydro_blocks(int w, int h);
void hydro_launch(int mode, const HydroArgs& A, cudaStream_t s);
void hydro_finalize_launch(const HydroArgs& A, int take_back, cudaStream_t s);

int floors_dt_blocks(int w, int h);
void floors_dt_launch(const HydroConst& H, float* U, const float* gx, const float* gy, int do_floors, float* part_rate,
                      float* part_g, long long* part_nf, double cfl, double eta_g, double dt_fixed, double dt_cap,
                      DtRecord* rec, cudaStream_t s);
void dt_advance_launch(DtRecord* rec, cudaStream_t s);
// Δt_{n+1} and the guard from per-CTA partials (the guard's codes are cell * channels + channel).
void dt_finalize_launch(int nblocks, int channels, const float* part_rate, const float* part_g,
                        const long long* part_nf, double cfl, double eta_g, double dt_fixed, double dt_cap,
                        DtRecord* rec, cudaStream_t s);
