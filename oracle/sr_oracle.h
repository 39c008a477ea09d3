/*
 * sr_oracle.h — TEST INFRASTRUCTURE ONLY. A CPU f64 restatement of the reference's own CPU twin
 * (the crates/sr-physics/src/reference/ files of Feynstein/sandbox_reactions), used to check the CUDA path and to time the
 * CPU baseline. Nothing in the product links or calls it; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline do.
 *
 * Parity pins: the reference's own known-answer tests (padded sizes, FFT vs direct DFT, delta/wave, Parseval,
 * convolution vs direct sum, SELF_CELL, LP λ, Sod vs the exact Riemann solution) run against these functions in
 * tests/test_oracle_*.py. The config-mode extensions (γ ≠ 2, minmod, the softened kernel, a κ plane) are not pinned by
 * any reference test; they reduce to the reference's formulas at γ = 2 / MC / self cell / uniform κ.
 */
#ifndef SR_ORACLE_H
#define SR_ORACLE_H

#include <stdint.h>
#include "../include/sr_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FFT and convolution (reference/fft.rs) ---- */
/* Smallest power of two >= 2*len, at least 32; 0 when len is 0 or the result exceeds `cap` (fft.rs:92-101). */
int64_t or_padded_size(int64_t len, int64_t cap);
/* In-place radix-2 complex FFT, forward unnormalised, inverse conjugated and /N (fft.rs:137-172). Returns 0, or -1
 * when n is not a power of two. */
int or_fft(int64_t n, double* re, double* im, int inverse);
/* Rows with nx, then columns with ny (fft.rs:174-196). */
int or_fft2(int64_t nx, int64_t ny, double* re, double* im, int inverse);
/* φ = K * s zero-padded, on the box grown by `ring` (fft.rs:238-282). `ktab` holds K at padded index (i, j) of a
 * px*py grid (signed offsets i<px/2 → i, else i-px); px = or_padded_size(w, cap). Returns 0 or -1. */
int or_convolve_ringed(const double* field, int64_t w, int64_t h, int64_t ring, const double* ktab, int64_t px,
                       int64_t py, double* out);
/* Fills the px*py kernel table for cfg's gravity kernel (grav.rs:25-34, or the softened one). */
void or_kernel_table(const sr_config* cfg, int64_t px, int64_t py, double* ktab);
/* P2: φ, g over the w*h world from Σ (vacuum masked) (grav.rs:96-129). Returns 0 or -1. */
int or_grav_field(const sr_config* cfg, const double* sigma, int64_t w, int64_t h, double* phi, double* gx,
                  double* gy);
/* Direct sum of cfg's kernel over every source, at `n` target cells (the potential oracle). OpenMP. */
void or_direct_potential(const sr_config* cfg, const double* src, int64_t w, int64_t h, int64_t n,
                         const int64_t* tx, const int64_t* ty, double* out);

/* ---- Hydro (reference/hydro.rs) ---- */
typedef struct or_hydro_report {
    double kick_net[2]; /* gravity's net kick on the gas's own field, taken back at the densest cell */
    int64_t densest;    /* that cell, -1 when none */
    double escaped[4];  /* what left through the world's edge: Σ, Σu, Σv, E */
} or_hydro_report;
/* One P4 step in place on 4 f64 planes (hydro.rs:657-1025 without held cells, sinks or radiation). `gx`, `gy`:
 * P2's field of the start state, or NULL without gravity. */
void or_hydro_step(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, const double* gx,
                   const double* gy, or_hydro_report* rep);
/* Δt of the state (hydro.rs:618-634); `gx`/`gy` NULL without gravity. */
double or_hydro_dt(const sr_config* cfg, const double* planes, int64_t w, int64_t h, const double* gx,
                   const double* gy);
/* P8's vacuum reset and thermal floor (reference/floors.rs:124-196, config mode: no species). */
void or_floors(const sr_config* cfg, double* planes, int64_t w, int64_t h);

/* ---- Heat / FLD (reference/heat.rs) ---- */
typedef struct or_heat_report {
    int64_t passes, rounds;
    double delta;
    int32_t converged;
    int32_t pad;
    double radiated;
} or_heat_report;
double or_lambda(double r);
/* One implicit FLD step in place (heat.rs:453-536, commit_limited 538-592). `kappa`: W*H plane or NULL (κ0).
 * `fx` ((w+1)*h) and `fy` (w*(h+1)) receive the solved face fluxes when not NULL. `tol`: the solve's measures
 * (heat.rs SOLVE_TOL = 1e-12), `newton_heat`/`newton_cell` the pass rules (1e-12 / 1e-10 in the twin). */
void or_heat_step(const sr_config* cfg, double* planes, const double* kappa, int64_t w, int64_t h, double dt,
                  double tol, double newton_heat, double newton_cell, or_heat_report* rep, double* fx, double* fy);
/* The same step on per-cell sides (reference mode): T⁰, κ and 1/μ of every cell (T_floor off the gas); C = Σ/μ. */
void or_heat_step_sides(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, double tol,
                        double newton_heat, double newton_cell, const double* t0, const double* kappa,
                        const double* inv_mu, or_heat_report* rep, double* fxo, double* fyo);
/* The frozen law's flux on the start state (heat.rs:303-309). */
void or_heat_law(const sr_config* cfg, const double* planes, const double* kappa, int64_t w, int64_t h, double* fx,
                 double* fy);
/* The first Newton pass's SPD system of a step (heat.rs:476-489): diag, rhs (W*H), face coefficients kx
 * ((w+1)*h), ky (w*(h+1)), and gas mask. Non-gas cells: diag 1, rhs 0. */
void or_heat_system(const sr_config* cfg, const double* planes, const double* kappa, int64_t w, int64_t h,
                    double dt, double* diag, double* rhs, double* kx, double* ky, uint8_t* gas);
/* y = A x for such a system. */
void or_heat_matvec(int64_t w, int64_t h, const double* diag, const double* kx, const double* ky,
                    const uint8_t* gas, const double* x, double* y);
/* Jacobi-PCG to ||b - A x||/||b|| <= rel (x in/out), returns rounds (-1 on breakdown). */
int64_t or_heat_pcg(int64_t w, int64_t h, const double* diag, const double* rhs, const double* kx, const double* ky,
                    const uint8_t* gas, double rel, int64_t max_rounds, double* x);

/* ---- Exact Riemann solution, γ parameter (reference/riemann.rs:72-210) ---- */
/* sol[0..9]: p*, u*, ρ*L, ρ*R, left kind (0 shock / 1 fan), left s1, left s2, right kind, right s1, right s2.
 * Returns 0, 1 bad state, 2 vacuum, 3 no convergence. */
int or_riemann_solve(double gamma, double rl, double ul, double pl, double rr, double ur, double pr, double* sol);
void or_riemann_sample(double gamma, double rl, double ul, double pl, double rr, double ur, double pr,
                       const double* sol, double xi, double* out /* rho, u, p */);

/* ---- The twin's step driver (reference/mod.rs:94-297) ---- */
typedef struct or_twin or_twin;
or_twin* or_twin_new(const sr_config* cfg, const double* planes, const double* kappa);
void or_twin_free(or_twin* t);
void or_twin_step(or_twin* t);
void or_twin_state(const or_twin* t, double* planes);
/* [dt, dt_next, sim_time, steps] */
void or_twin_clock(const or_twin* t, double* out4);
/* The last P2 field (φ, gx, gy), W*H each. */
void or_twin_field(const or_twin* t, double* phi, double* gx, double* gy);
/* The last P5 report and solved fluxes. */
void or_twin_heat(const or_twin* t, or_heat_report* rep, double* fx, double* fy);

/* Number of OpenMP threads the oracle uses (0: the runtime's default). */
void or_set_threads(int n);
int or_get_threads(void);

/* ---- Reference mode (sr_oracle_ref.c): 14 channels, the reference's own EOS, species and the hold ---- */
/* The cold pressure P(x; K₁, K₂) (eos.rs:22-29), its energy per area in closed form (eos.rs:49-65), the 512-node
 * table of ln u (eos.rs:81-98) and the table's u(x) (eos.rs:118-131). */
double or_cold_pressure(double x, double k1, double k2);
double or_cold_energy_exact(double x, double k1, double k2);
void or_cold_table(double k1, double k2, double* ln_u);
double or_cold_table_u(const double* ln_u, double x);
/* 1/μ, Y_e, Z_met of ten mass fractions (registry.rs:145-154). */
void or_composition(const double* x, double* out3);
typedef struct or_ref_hydro_report {
    double spared[2];   /* momentum booked `held`: the held cells' spared impulses and the sticky walls' stops */
    double kick_net[2]; /* gravity's net kick on the gas's own field, taken back at the densest free cell */
    int64_t densest;
    double push_net[2]; /* the radiation force's net push, taken back */
    double push_abs;    /* Σ |push| */
} or_ref_hydro_report;
/* One P4 step in place on 14 f64 planes (hydro.rs:657-1025, step_held): `gx`/`gy` P2's field of the start state or
 * NULL; `held` the hold's mask or NULL; `radx`/`rady` the cell-centred flux of the radiation force or NULL. */
void or_ref_hydro_step(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, const double* gx,
                       const double* gy, const uint8_t* held, const double* radx, const double* rady,
                       or_ref_hydro_report* rep);
/* Δt of a 14-channel state (hydro.rs:618-634). */
double or_ref_dt(const sr_config* cfg, const double* planes, int64_t w, int64_t h, const double* gx,
                 const double* gy);
/* P8's floors (floors.rs:124-175); booked2 = [vacuum_reset, floor_added]. */
void or_ref_floors(const sr_config* cfg, double* planes, int64_t w, int64_t h, double* booked2);
/* The mass of the disk r about (x, y) (sinks.rs:117-125). */
double or_ref_disk_mass(const double* sigma, int64_t w, int64_t h, int64_t x, int64_t y, double r);
/* The hold (floors.rs:196-243): `held` in/out; taken2 = the newly held cells' momentum. */
void or_ref_hold(const sr_config* cfg, double* planes, int64_t w, int64_t h, uint8_t* held, double* taken2);
/* The reference-mode twin (mod.rs:129-297 without P5): P1, P2, P4, P8 + hold, P9. `mask`: the initial hold or NULL. */
typedef struct or_ref_twin or_ref_twin;
or_ref_twin* or_ref_twin_new(const sr_config* cfg, const double* planes, const uint8_t* mask);
void or_ref_twin_free(or_ref_twin* t);
void or_ref_twin_set_flux(or_ref_twin* t, const double* fx, const double* fy);
void or_ref_twin_step(or_ref_twin* t);
void or_ref_twin_state(const or_ref_twin* t, double* planes, uint8_t* mask);
/* [dt, dt_next, sim_time, steps] */
void or_ref_twin_clock(const or_ref_twin* t, double* out4);
/* [held x, held y, vacuum_reset, floor_added] booked since the twin was made */
void or_ref_twin_books(const or_ref_twin* t, double* out4);
/* The last P5's report and face fluxes. */
void or_ref_twin_heat(const or_ref_twin* t, or_heat_report* rep, double* fx, double* fy);
/* P5's sides of a 14-channel state (heat.rs:215-231) and one reference-mode implicit step on them. */
void or_ref_heat_sides(const sr_config* cfg, const double* planes, int64_t w, int64_t h, double* t0, double* kappa,
                       double* inv_mu);
void or_ref_heat_step(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, double tol,
                      double newton_heat, double newton_cell, or_heat_report* rep, double* fx, double* fy);

#ifdef __cplusplus
}
#endif
#endif
