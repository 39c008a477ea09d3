/*
 * sr_oracle_ref.c — TEST INFRASTRUCTURE ONLY: reference mode of the CPU f64 oracle, the reference twin's own
 * 14-channel field update (crates/sr-physics/src/{eos.rs, registry.rs} and reference/{hydro,floors,mod}.rs of
 * Feynstein/sandbox_reactions): the γ = 2 EOS with μ and Y_e from each cell's ten species and the cold pressures of
 * the two K pairs read from their u(x) tables, species slopes sharing one limiter factor and upwinded by the mass flux,
 * held cells behind reflecting walls with their sticky wall, the radiation force of a given cell-centred flux with its
 * cap and net take-back, P8's species renormalisation, vacuum reset and thermal floor, and the hold's rule. Only
 * tests/ use it; the product never links it. Each function names the reference lines it follows.
 *
 * Planes: 14 f64 planes of w*h, channel-major (Σ, Σu, Σv, E, then the mass fractions in the registry's order H, He,
 * C, O, Ne, Mg, Si, S, Fe, n). The hold's mask: one byte per cell, 1 where held. Sums the reference takes cell by cell
 * are taken in the same index order here (this file runs its loops on one thread unless a loop is order-free).
 */
#define _GNU_SOURCE
#include "sr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NS 10
#define NC 14
#define TABLE_POINTS 512 /* eos.rs:15 */
#define X_MIN 1e-8       /* eos.rs:17-18 */
#define X_MAX 1e8
#define QUAD_STEPS 64 /* eos.rs:21 */
#define HOT_FACE 2.0  /* reference/hydro.rs:301 */
#define IRON_TRACE 1e-3   /* reference/floors.rs:34-36 */
#define NEUTRON_RICH 0.5  /* floors.rs:38 */
enum { ID_H = 0, ID_HE = 1, ID_FE = 8, ID_N = 9 };

/* elements.json's species in id order: mass number A and charge Z (registry.rs:45-153) */
static const double SP_A[NS] = {1, 4, 12, 16, 20, 24, 28, 32, 56, 1};
static const double SP_Z[NS] = {1, 2, 6, 8, 10, 12, 14, 16, 26, 0};

/* ======================================================================= EOS (eos.rs) */

double or_cold_pressure(double x, double k1, double k2) {
    /* eos.rs:22-29 */
    if (x <= 0.0 || k1 <= 0.0 || k2 <= 0.0) return 0.0;
    return 1.0 / (1.0 / (k1 * x * x) + 1.0 / (k2 * pow(x, 1.5)));
}

static double quad_segment(double k1, double k2, double t0, double t1, int n) {
    /* eos.rs:31-47: Simpson's rule for ∫ P(s)/s² · 2t dt, s = t² */
#define QF(t) ((t) <= 0.0 ? 0.0 : or_cold_pressure((t) * (t), k1, k2) / (((t) * (t)) * ((t) * (t))) * 2.0 * (t))
    double h = (t1 - t0) / n;
    double sum = QF(t0) + QF(t1);
    for (int i = 1; i < n; i++) {
        double t = t0 + h * i;
        sum += QF(t) * (i % 2 == 1 ? 4.0 : 2.0);
    }
#undef QF
    return sum * h / 3.0;
}

double or_cold_energy_exact(double x, double k1, double k2) {
    /* eos.rs:49-65: u(x) in closed form, the table's check */
    if (x <= 0.0 || k1 <= 0.0 || k2 <= 0.0) return 0.0;
    double y = k1 / k2 * sqrt(x);
    double g;
    if (y < 1e-3) {
        g = 0.0;
        for (int k = 2; k < 10; k++) g += (k % 2 == 0 ? 1.0 : -1.0) * pow(y, k) / k;
    } else {
        g = y - log1p(y);
    }
    return x * 2.0 * k2 * k2 / k1 * g;
}

static double node_x(int i) { /* eos.rs:100-104 */
    double frac = (double)i / (TABLE_POINTS - 1);
    return exp(log(X_MIN) + frac * (log(X_MAX) - log(X_MIN)));
}

static double table_step(void) { return (log(X_MAX) - log(X_MIN)) / (TABLE_POINTS - 1); } /* eos.rs:106-109 */

void or_cold_table(double k1, double k2, double* ln_u) {
    /* eos.rs:81-98: J(x_i) accumulated segment by segment in t = √s, ln u = ln(x J) */
    double t_prev = 0.0, j = 0.0;
    for (int i = 0; i < TABLE_POINTS; i++) {
        double t = sqrt(node_x(i));
        int steps = i == 0 ? QUAD_STEPS * 8 : QUAD_STEPS;
        j += quad_segment(k1, k2, t_prev, t, steps);
        ln_u[i] = log(node_x(i) * j);
        t_prev = t;
    }
}

typedef struct {
    int on;
    double k1, k2;
    double ln_u[TABLE_POINTS];
} cold_table;

static double table_u(const cold_table* t, double x) {
    /* eos.rs:118-131: log-log interpolation, K₁x² below the first node, the last segment's slope past the end */
    if (x <= 0.0) return 0.0;
    double pos = (log(x) - log(X_MIN)) / table_step();
    if (pos < 0.0) return exp(t->ln_u[0]) * (x / X_MIN) * (x / X_MIN);
    int64_t i = (int64_t)floor(fmax(pos, 0.0));
    if (i > TABLE_POINTS - 2) i = TABLE_POINTS - 2;
    double frac = pos - (double)i;
    return exp(t->ln_u[i] + frac * (t->ln_u[i + 1] - t->ln_u[i]));
}

double or_cold_table_u(const double* ln_u, double x) {
    cold_table t;
    t.on = 1;
    memcpy(t.ln_u, ln_u, sizeof t.ln_u);
    return table_u(&t, x);
}

typedef struct {
    cold_table e, n;
    double t_floor;
} eos_t;

static void eos_init(eos_t* E, const sr_config* cfg) {
    /* eos.rs:175-187: a pair is on when both of its K are > 0 */
    E->e.on = cfg->k1e > 0.0 && cfg->k2e > 0.0;
    E->n.on = cfg->k1n > 0.0 && cfg->k2n > 0.0;
    E->e.k1 = cfg->k1e;
    E->e.k2 = cfg->k2e;
    E->n.k1 = cfg->k1n;
    E->n.k2 = cfg->k2n;
    if (E->e.on) or_cold_table(cfg->k1e, cfg->k2e, E->e.ln_u);
    if (E->n.on) or_cold_table(cfg->k1n, cfg->k2n, E->n.ln_u);
    E->t_floor = cfg->t_floor;
}

static double eos_pi_e(const eos_t* E, double s, double ye) { /* eos.rs:222-225 */
    return E->e.on ? or_cold_pressure(ye * s, E->e.k1, E->e.k2) : 0.0;
}
static double eos_pi_n(const eos_t* E, double s, double xn) { /* eos.rs:227-230 */
    return E->n.on ? or_cold_pressure(xn * s, E->n.k1, E->n.k2) : 0.0;
}
static double eos_pi(const eos_t* E, double s, double eps_th, double ye, double xn) { /* eos.rs:232-235 */
    return s * eps_th + eos_pi_e(E, s, ye) + eos_pi_n(E, s, xn);
}
static double eos_eps_cold(const eos_t* E, double s, double ye, double xn) { /* eos.rs:237-242 */
    double ue = E->e.on ? table_u(&E->e, ye * s) : 0.0;
    double un = E->n.on ? table_u(&E->n, xn * s) : 0.0;
    return (ue + un) / s;
}
/* eos.rs:250-262: ε_th recovered from E and floored at T_floor/μ; the floor's energy per area returned */
static double eos_thermal(const eos_t* E, double energy, double s, double mx, double my, double ye, double xn,
                          double mu, double* floor_added) {
    double kinetic = 0.5 * (mx * mx + my * my) / (s * s);
    double raw = energy / s - kinetic - eos_eps_cold(E, s, ye, xn);
    double floor = E->t_floor / mu;
    if (raw < floor) {
        if (floor_added) *floor_added = s * (floor - raw);
        return floor;
    }
    if (floor_added) *floor_added = 0.0;
    return raw;
}

typedef struct {
    double inv_mu, y_e, z_met;
} comp_t;

static comp_t composition(const double* x) {
    /* registry.rs:145-154: fully ionised 1/μ = Σ X(Z+1)/A, Y_e = Σ X Z/A, Z_met = 1 - X_H - X_He - X_n */
    comp_t c = {0.0, 0.0, 0.0};
    for (int s = 0; s < NS; s++) {
        c.inv_mu += x[s] * (SP_Z[s] + 1.0) / SP_A[s];
        c.y_e += x[s] * SP_Z[s] / SP_A[s];
    }
    c.z_met = 1.0 - x[ID_H] - x[ID_HE] - x[ID_N];
    return c;
}

void or_composition(const double* x, double* out3) {
    comp_t c = composition(x);
    out3[0] = c.inv_mu;
    out3[1] = c.y_e;
    out3[2] = c.z_met;
}

/* ======================================================================= P4 (reference/hydro.rs) */

typedef struct {
    double s, u, v, p;
    double x[NS];
} rprim; /* hydro.rs:226-233 */
typedef struct {
    double U[NC];
    rprim p;
} rface; /* hydro.rs:277-281 */

typedef struct {
    eos_t eos;
    double sigma_vac, sigma_floor, cfl, eta_g, kappa0, c_sb, kappa_dust, t_dust;
    int limiter, bracket, edge;
} rhyd;

static void rhyd_init(rhyd* H, const sr_config* cfg) {
    eos_init(&H->eos, cfg);
    H->sigma_vac = cfg->sigma_vac;
    H->sigma_floor = cfg->sigma_floor;
    H->cfl = cfg->cfl;
    H->eta_g = cfg->eta_g;
    H->kappa0 = cfg->kappa0;
    H->c_sb = cfg->c_sb;
    H->kappa_dust = cfg->kappa_dust;
    H->t_dust = cfg->t_dust;
    H->limiter = (int)cfg->limiter;
    H->bracket = (int)cfg->thermal_bracket;
    H->edge = (int)cfg->edge;
}

static rprim r_read(const rhyd* H, const double* planes, int64_t n, int64_t i) {
    /* hydro.rs:424-441: the floor state below Σ_vac (the cell's fractions kept), else ε_th recovered and floored */
    rprim p;
    for (int s = 0; s < NS; s++) p.x[s] = planes[(4 + s) * n + i];
    comp_t c = composition(p.x);
    double mu = 1.0 / c.inv_mu, xn = p.x[NS - 1];
    double s = planes[i];
    if (s < H->sigma_vac) {
        p.s = H->sigma_floor;
        p.u = 0.0;
        p.v = 0.0;
        p.p = eos_pi(&H->eos, p.s, H->eos.t_floor / mu, c.y_e, xn);
        return p;
    }
    double mx = planes[n + i], my = planes[2 * n + i];
    double eps = eos_thermal(&H->eos, planes[3 * n + i], s, mx, my, c.y_e, xn, mu, NULL);
    p.s = s;
    p.u = mx / s;
    p.v = my / s;
    p.p = eos_pi(&H->eos, s, eps, c.y_e, xn);
    return p;
}

static void r_cons(const rhyd* H, const rprim* p, double* U) {
    /* hydro.rs:443-460 */
    comp_t c = composition(p->x);
    double xn = p->x[NS - 1];
    double thermal = (p->p - eos_pi_e(&H->eos, p->s, c.y_e) - eos_pi_n(&H->eos, p->s, xn)) / p->s;
    double eps_th = fmax(thermal, H->eos.t_floor * c.inv_mu);
    U[0] = p->s;
    U[1] = p->s * p->u;
    U[2] = p->s * p->v;
    U[3] = p->s * (eps_th + eos_eps_cold(&H->eos, p->s, c.y_e, xn)) + 0.5 * p->s * (p->u * p->u + p->v * p->v);
    for (int s = 0; s < NS; s++) U[4 + s] = p->s * p->x[s];
}

static int r_prim(const rhyd* H, const double* U, rprim* out) {
    /* hydro.rs:462-478: none when Σ <= 0, a component not finite, or no thermal energy left */
    double s = U[0];
    if (isnan(s) || s <= 0.0) return 0;
    for (int k = 0; k < NC; k++)
        if (!isfinite(U[k])) return 0;
    for (int k = 0; k < NS; k++) out->x[k] = U[4 + k] / s;
    comp_t c = composition(out->x);
    double xn = out->x[NS - 1];
    double raw = U[3] / s - 0.5 * (U[1] * U[1] + U[2] * U[2]) / (s * s) - eos_eps_cold(&H->eos, s, c.y_e, xn);
    if (isnan(raw) || raw <= 0.0) return 0;
    double eps = fmax(raw, H->eos.t_floor * c.inv_mu);
    out->s = s;
    out->u = U[1] / s;
    out->v = U[2] / s;
    out->p = eos_pi(&H->eos, s, eps, c.y_e, xn);
    return 1;
}

static double r_sound(const rprim* p) { return sqrt(fmax(2.0 * p->p / p->s, 0.0)); } /* hydro.rs:480-483 */

static void r_flux(const rprim* p, double energy, int dir, double* f) {
    /* hydro.rs:485-499 */
    double un = dir == 0 ? p->u : p->v, ut = dir == 0 ? p->v : p->u;
    double mass = p->s * un;
    f[0] = mass;
    f[1 + dir] = mass * un + p->p;
    f[2 - dir] = mass * ut;
    f[3] = (energy + p->p) * un;
    for (int s = 0; s < NS; s++) f[4 + s] = mass * p->x[s];
}

static double lim_mc(double l, double c, double r) { /* hydro.rs:283-289 */
    double a = c - l, b = r - c;
    if (a * b <= 0.0) return 0.0;
    return copysign(fmin(fmin(fabs(0.5 * (a + b)), 2.0 * fabs(a)), 2.0 * fabs(b)), a);
}

static double lim_minmod(double l, double c, double r) {
    double a = c - l, b = r - c;
    if (a * b <= 0.0) return 0.0;
    return copysign(fmin(fabs(a), fabs(b)), a);
}

static rprim r_slope(const rhyd* H, const rprim* l, const rprim* c, const rprim* r) {
    /* hydro.rs:293-331: limited slopes of Σ, u, v, Π; the species' central differences scaled by the one factor the
     * most limited needs (species_slopes); Σ and Π flat where the thermal bracket refuses a face */
    double (*lim)(double, double, double) = H->limiter == SR_LIMITER_MINMOD ? lim_minmod : lim_mc;
    rprim s;
    s.s = lim(l->s, c->s, r->s);
    s.u = lim(l->u, c->u, r->u);
    s.v = lim(l->v, c->v, r->v);
    s.p = lim(l->p, c->p, r->p);
    double central[NS], theta = 1.0;
    for (int i = 0; i < NS; i++) {
        central[i] = 0.5 * (r->x[i] - l->x[i]);
        if (central[i] != 0.0) theta = fmin(theta, lim(l->x[i], c->x[i], r->x[i]) / central[i]);
    }
    for (int i = 0; i < NS; i++) s.x[i] = theta * central[i];
    if (H->bracket) {
        double hottest = fmax(fmax(l->p / l->s, c->p / c->s), r->p / r->s);
        int hot = 0;
        for (int k = 0; k < 2; k++) {
            double f = k ? 0.5 : -0.5;
            double pif = c->p + f * s.p, bound = HOT_FACE * hottest * (c->s + f * s.s);
            if (!(pif <= bound)) hot = 1; /* greater, or not a number */
        }
        if (hot) {
            s.s = 0.0;
            s.p = 0.0;
        }
    }
    return s;
}

static rprim r_offset(const rprim* c, const rprim* s, double f) { /* hydro.rs:236-250 */
    rprim o;
    o.s = c->s + f * s->s;
    o.u = c->u + f * s->u;
    o.v = c->v + f * s->v;
    o.p = c->p + f * s->p;
    for (int k = 0; k < NS; k++) o.x[k] = c->x[k] + f * s->x[k];
    return o;
}

static rface r_evolved(const rhyd* H, const rprim* base, const double* delta) {
    /* hydro.rs:501-513 */
    rface F;
    double U0[NC], U[NC];
    r_cons(H, base, U0);
    for (int k = 0; k < NC; k++) U[k] = U0[k] + delta[k];
    rprim p;
    if (r_prim(H, U, &p)) {
        memcpy(F.U, U, sizeof U);
        F.p = p;
    } else {
        memcpy(F.U, U0, sizeof U0);
        F.p = *base;
    }
    return F;
}

static void r_predicted(const rhyd* H, const rprim* grid, int64_t pw, int64_t gi, double half, int has_g, double gx,
                        double gy, rface* out4, double* mid3) {
    /* hydro.rs:587-614 */
    const rprim* c = &grid[gi];
    rprim sx = r_slope(H, &grid[gi - 1], c, &grid[gi + 1]);
    rprim sy = r_slope(H, &grid[gi - pw], c, &grid[gi + pw]);
    rprim wf[4] = {r_offset(c, &sx, -0.5), r_offset(c, &sx, 0.5), r_offset(c, &sy, -0.5), r_offset(c, &sy, 0.5)};
    double uf[4][NC];
    for (int k = 0; k < 4; k++) r_cons(H, &wf[k], uf[k]);
    double fxl[NC], fxr[NC], fyl[NC], fyr[NC];
    r_flux(&wf[0], uf[0][3], 0, fxl);
    r_flux(&wf[1], uf[1][3], 0, fxr);
    r_flux(&wf[2], uf[2][3], 1, fyl);
    r_flux(&wf[3], uf[3][3], 1, fyr);
    double delta[NC];
    for (int k = 0; k < NC; k++) delta[k] = half * ((fxl[k] - fxr[k]) + (fyl[k] - fyr[k]));
    mid3[0] = c->s + delta[0];
    mid3[1] = c->s * c->u + delta[1];
    mid3[2] = c->s * c->v + delta[2];
    if (!has_g) {
        for (int k = 0; k < 4; k++) out4[k] = r_evolved(H, &wf[k], delta);
        return;
    }
    mid3[1] += half * c->s * gx;
    mid3[2] += half * c->s * gy;
    for (int k = 0; k < 4; k++) {
        const rprim* p = &wf[k];
        double d[NC];
        memcpy(d, delta, sizeof d);
        d[1] += half * p->s * gx;
        d[2] += half * p->s * gy;
        d[3] += half * p->s * ((p->u + 0.5 * half * gx) * gx + (p->v + 0.5 * half * gy) * gy);
        out4[k] = r_evolved(H, p, d);
    }
}

static void r_hll(const rface* l, const rface* r, int dir, double* f) {
    /* hydro.rs:516-540: HLL with Davis speeds; the species by the mass flux's upwind side */
    double unl = dir == 0 ? l->p.u : l->p.v, unr = dir == 0 ? r->p.u : r->p.v;
    double cl = r_sound(&l->p), cr = r_sound(&r->p);
    double s_l = fmin(unl - cl, unr - cr);
    double s_r = fmax(unl + cl, unr + cr);
    double fl[NC], fr[NC];
    r_flux(&l->p, l->U[3], dir, fl);
    r_flux(&r->p, r->U[3], dir, fr);
    if (s_l >= 0.0) {
        memcpy(f, fl, sizeof fl);
    } else if (s_r <= 0.0) {
        memcpy(f, fr, sizeof fr);
    } else {
        for (int k = 0; k < NC; k++) f[k] = 0.0;
        for (int k = 0; k < 4; k++) f[k] = (s_r * fl[k] - s_l * fr[k] + s_l * s_r * (r->U[k] - l->U[k])) / (s_r - s_l);
    }
    const rprim* up = f[0] > 0.0 ? &l->p : &r->p;
    for (int s = 0; s < NS; s++) f[4 + s] = f[0] * up->x[s];
}

static void r_held_wall(const rface* face, int dir, int low, double* f) {
    /* hydro.rs:542-554: HLL against the free side's mirror, mass, energy and species exactly 0 */
    rface m = *face;
    if (dir == 0) m.p.u = -m.p.u;
    else m.p.v = -m.p.v;
    m.U[1 + dir] = -m.U[1 + dir];
    if (low) r_hll(face, &m, dir, f);
    else r_hll(&m, face, dir, f);
    f[0] = 0.0;
    f[3] = 0.0;
    for (int k = 4; k < NC; k++) f[k] = 0.0;
}

static void r_wall(const rface* own, int dir, double* f) { /* hydro.rs:556-562 */
    for (int k = 0; k < NC; k++) f[k] = 0.0;
    f[1 + dir] = own->p.p;
}

static void face_work(double q, double sl, double sh, double pl, double ph, double d, double dt, double* out3) {
    /* hydro.rs:1042-1067 */
    double a = fmax(sl, 0.0), b = fmax(sh, 0.0);
    double w = a + b > 0.0 ? a / (a + b) : 0.5;
    double extra = dt * (q - 0.5 * (pl + ph)) * d;
    double c = 0.0, kick = 0.0, el = 0.0, eh = 0.0;
    if (extra < 0.0 && a > 0.0 && b > 0.0) {
        double ul = pl / a, uh = ph / b;
        double du = ul - uh;
        double inv = 1.0 / a + 1.0 / b;
        c = fmin(-extra, 0.25 * du * du / inv);
        if (c > 0.0) {
            double disc = sqrt(fmax(du * du - 2.0 * inv * c, 0.0));
            kick = -2.0 * c / (du + copysign(1.0, du) * disc);
            el = ul * kick + 0.5 * kick * kick / a;
            eh = -uh * kick + 0.5 * kick * kick / b;
        }
    }
    double rest = extra + c;
    out3[0] = kick;
    out3[1] = 0.5 * dt * pl * d + w * rest + el;
    out3[2] = 0.5 * dt * ph * d + (1.0 - w) * rest + eh;
}

static void radiation_force(const rhyd* H, const double* planes, int64_t n, int64_t i, double fx, double fy,
                            double* out2) {
    /* hydro.rs:365-382: f = κΣF/c_sb, κ = κ₀(1 + X_H) plus κ_dust Z_met below T_dust; 0 below Σ_vac */
    double s = planes[i];
    out2[0] = out2[1] = 0.0;
    if (s < H->sigma_vac) return;
    double x[NS];
    for (int k = 0; k < NS; k++) x[k] = planes[(4 + k) * n + i];
    double kappa = H->kappa0 * (1.0 + x[ID_H]);
    if (H->kappa_dust != 0.0) {
        comp_t c = composition(x);
        double mu = 1.0 / c.inv_mu;
        double eps = eos_thermal(&H->eos, planes[3 * n + i], s, planes[n + i], planes[2 * n + i], c.y_e, x[ID_N], mu,
                                 NULL);
        if (mu * eps < H->t_dust) kappa += H->kappa_dust * c.z_met;
    }
    out2[0] = kappa * s * fx / H->c_sb;
    out2[1] = kappa * s * fy / H->c_sb;
}

static double push_share(const rhyd* H, const double* u, const double* d) {
    /* hydro.rs:384-405: the share of the impulse the cell's heat above its floor pays for */
    double d2 = d[0] * d[0] + d[1] * d[1];
    if (d2 == 0.0) return 1.0;
    double s = u[0];
    double x[NS];
    for (int k = 0; k < NS; k++) x[k] = u[4 + k] / s;
    comp_t c = composition(x);
    double added;
    double eps = eos_thermal(&H->eos, u[3], s, u[1], u[2], c.y_e, x[ID_N], 1.0 / c.inv_mu, &added);
    double raw = eps - added / s;
    double a = s * (raw - H->eos.t_floor * c.inv_mu);
    if (isnan(a) || a <= 0.0) return 0.0;
    double q = u[1] * d[0] + u[2] * d[1];
    double disc = sqrt(q * q + 2.0 * s * a * d2);
    double root = q >= 0.0 ? 2.0 * s * a / (q + disc) : (disc - q) / d2;
    return fmin(root, 1.0);
}

void or_ref_hydro_step(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, const double* gx,
                       const double* gy, const uint8_t* held, const double* radx, const double* rady,
                       or_ref_hydro_report* rep) {
    /* hydro.rs:657-1025 (step_held): gravity when `gx` is given (P2's field of the start state), the hold's `held`
     * mask (NULL: none held), the radiation force of the cell-centred flux (radx, rady; NULL: none) */
    rhyd H;
    rhyd_init(&H, cfg);
    const int64_t n = w * h, G2 = 2, pw = w + 4, ph = h + 4;
    const double* S = planes;
    const int has_g = gx != NULL;
#define AT(x, y) (((y) + G2) * pw + (x) + G2)
#define HELD(i) (held && held[i])
    rprim* grid = (rprim*)malloc(sizeof(rprim) * (size_t)(pw * ph));
    for (int64_t i = 0; i < pw * ph; i++) {
        memset(&grid[i], 0, sizeof(rprim));
        grid[i].s = 1.0;
        grid[i].p = 1.0;
    }
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) grid[AT(x, y)] = r_read(&H, planes, n, y * w + x);
    /* ghosts (hydro.rs:686-709): columns first, then rows over the padded width */
    for (int64_t y = 0; y < h; y++)
        for (int64_t k = 1; k <= G2; k++) {
            rprim a, b;
            if (H.edge == SR_EDGE_BOUNCE) {
                a = grid[AT(k - 1, y)];
                a.u = -a.u;
                b = grid[AT(w - k, y)];
                b.u = -b.u;
            } else {
                a = grid[AT(0, y)];
                a.u = fmin(a.u, 0.0);
                b = grid[AT(w - 1, y)];
                b.u = fmax(b.u, 0.0);
            }
            grid[(y + G2) * pw + G2 - k] = a;
            grid[(y + G2) * pw + G2 + w - 1 + k] = b;
        }
    for (int64_t px = 0; px < pw; px++)
        for (int64_t k = 1; k <= G2; k++) {
            rprim a, b;
            if (H.edge == SR_EDGE_BOUNCE) {
                a = grid[(G2 + k - 1) * pw + px];
                a.v = -a.v;
                b = grid[(G2 + h - k) * pw + px];
                b.v = -b.v;
            } else {
                a = grid[G2 * pw + px];
                a.v = fmin(a.v, 0.0);
                b = grid[(G2 + h - 1) * pw + px];
                b.v = fmax(b.v, 0.0);
            }
            grid[(G2 - k) * pw + px] = a;
            grid[(G2 + h - 1 + k) * pw + px] = b;
        }
    const double half = 0.5 * dt;
    rface* faces = (rface*)malloc(sizeof(rface) * 4 * (size_t)n);
    double* mids = (double*)malloc(sizeof(double) * 3 * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            int64_t i = y * w + x;
            r_predicted(&H, grid, pw, AT(x, y), half, has_g, has_g ? gx[i] : 0.0, has_g ? gy[i] : 0.0, faces + 4 * i,
                        mids + 3 * i);
        }
    /* the boundary faces (hydro.rs:564-582): bounce → wall; leave → HLL against the ghost's predicted face,
     * inflow → wall; a ghost's g is its edge cell's */
#define BOUNDARY(side, own, gcell, e, out)                                                                    \
    do {                                                                                                      \
        int dir_ = (side) / 2, high_ = (side) % 2;                                                            \
        if (H.edge == SR_EDGE_BOUNCE) {                                                                       \
            r_wall((own), dir_, (out));                                                                       \
        } else {                                                                                              \
            rface gf_[4];                                                                                     \
            double gm_[3];                                                                                    \
            r_predicted(&H, grid, pw, (gcell), half, has_g, has_g ? gx[e] : 0.0, has_g ? gy[e] : 0.0, gf_, gm_); \
            if (high_) r_hll((own), &gf_[(side) - 1], dir_, (out));                                           \
            else r_hll(&gf_[(side) + 1], (own), dir_, (out));                                                 \
            int inflow_ = high_ ? (out)[0] < 0.0 : (out)[0] > 0.0;                                            \
            if (inflow_) r_wall((own), dir_, (out));                                                          \
        }                                                                                                     \
    } while (0)
    double* fx = (double*)malloc(sizeof(double) * NC * (size_t)((w + 1) * h));
    double* fy = (double*)malloc(sizeof(double) * NC * (size_t)(w * (h + 1)));
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t i = 0; i <= w; i++) {
            double* f = fx + NC * (y * (w + 1) + i);
            if (i == 0) {
                int64_t e = y * w;
                BOUNDARY(0, &faces[4 * e + 0], AT(0, y) - 1, e, f);
            } else if (i == w) {
                int64_t e = y * w + w - 1;
                BOUNDARY(1, &faces[4 * e + 1], AT(w - 1, y) + 1, e, f);
            } else {
                r_hll(&faces[4 * (y * w + i - 1) + 1], &faces[4 * (y * w + i) + 0], 0, f);
            }
        }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j <= h; j++)
        for (int64_t x = 0; x < w; x++) {
            double* f = fy + NC * (j * w + x);
            if (j == 0) {
                int64_t e = x;
                BOUNDARY(2, &faces[4 * e + 2], AT(x, 0) - pw, e, f);
            } else if (j == h) {
                int64_t e = (h - 1) * w + x;
                BOUNDARY(3, &faces[4 * e + 3], AT(x, h - 1) + pw, e, f);
            } else {
                r_hll(&faces[4 * ((j - 1) * w + x) + 3], &faces[4 * (j * w + x) + 2], 1, f);
            }
        }
#undef BOUNDARY
    /* held cells' faces (hydro.rs:780-812): nothing between two held cells or at a held cell's edge, a reflecting
     * wall between a held and a free cell; `still` marks them (no gravitational work across) */
    uint8_t* still_x = (uint8_t*)calloc((size_t)((w + 1) * h), 1);
    uint8_t* still_y = (uint8_t*)calloc((size_t)(w * (h + 1)), 1);
    if (held) {
        for (int64_t y = 0; y < h; y++)
            for (int64_t i = 0; i <= w; i++) {
                int64_t a = i > 0 ? y * w + i - 1 : -1, b = i < w ? y * w + i : -1;
                int ha = a >= 0 && held[a], hb = b >= 0 && held[b];
                if (!ha && !hb) continue;
                double* f = fx + NC * (y * (w + 1) + i);
                if (a >= 0 && b >= 0 && ha != hb) {
                    if (ha) r_held_wall(&faces[4 * b + 0], 0, 0, f);
                    else r_held_wall(&faces[4 * a + 1], 0, 1, f);
                } else {
                    for (int k = 0; k < NC; k++) f[k] = 0.0;
                }
                still_x[y * (w + 1) + i] = 1;
            }
        for (int64_t j = 0; j <= h; j++)
            for (int64_t x = 0; x < w; x++) {
                int64_t a = j > 0 ? (j - 1) * w + x : -1, b = j < h ? j * w + x : -1;
                int ha = a >= 0 && held[a], hb = b >= 0 && held[b];
                if (!ha && !hb) continue;
                double* f = fy + NC * (j * w + x);
                if (a >= 0 && b >= 0 && ha != hb) {
                    if (ha) r_held_wall(&faces[4 * b + 2], 1, 0, f);
                    else r_held_wall(&faces[4 * a + 3], 1, 1, f);
                } else {
                    for (int k = 0; k < NC; k++) f[k] = 0.0;
                }
                still_y[j * w + x] = 1;
            }
    }
    free(faces);
#define VAC(x, y) (S[(y) * w + (x)] < H.sigma_vac)
#define EMPTY(x, y)                                                                                         \
    (VAC(x, y) && ((x) == 0 || VAC((x) - 1, y)) && ((x) + 1 == w || VAC((x) + 1, y)) && ((y) == 0 || VAC(x, (y) - 1)) && \
     ((y) + 1 == h || VAC(x, (y) + 1)))
    /* the half step's field (hydro.rs:815-856): Σ_src,mid = ½(Σⁿ + Σⁿ⁺¹), a held cell's own Σ, masked; solved, and
     * with a held cell the same with the held cells emptied (the pull on them). The given field's sinks' part
     * (the given field less P2's solve of the same Σⁿ) is exactly 0 without sinks. */
    double *src = NULL, *phim = NULL, *gxm = NULL, *gym = NULL, *gxp = NULL, *gyp = NULL;
    int any_held = 0;
    if (held)
        for (int64_t i = 0; i < n; i++) any_held |= held[i] != 0;
    if (has_g) {
        src = (double*)malloc(sizeof(double) * (size_t)n);
        phim = (double*)malloc(sizeof(double) * (size_t)n);
        gxm = (double*)malloc(sizeof(double) * (size_t)n);
        gym = (double*)malloc(sizeof(double) * (size_t)n);
        for (int64_t y = 0; y < h; y++)
            for (int64_t x = 0; x < w; x++) {
                int64_t i = y * w + x;
                double s;
                if (HELD(i)) {
                    s = S[i];
                } else if (EMPTY(x, y)) {
                    s = 0.0;
                } else {
                    double start;
                    if (VAC(x, y)) {
                        double U0[NC];
                        r_cons(&H, &grid[AT(x, y)], U0);
                        start = U0[0];
                    } else {
                        start = S[i];
                    }
                    double div = (fx[NC * (y * (w + 1) + x + 1)] - fx[NC * (y * (w + 1) + x)]) +
                                 (fy[NC * ((y + 1) * w + x)] - fy[NC * (y * w + x)]);
                    s = 0.5 * (S[i] + (start - dt * div));
                }
                src[i] = s >= H.sigma_vac ? s : 0.0;
            }
        or_grav_field(cfg, src, w, h, phim, gxm, gym);
        if (any_held) {
            double* freed = (double*)malloc(sizeof(double) * (size_t)n);
            double* php = (double*)malloc(sizeof(double) * (size_t)n);
            gxp = (double*)malloc(sizeof(double) * (size_t)n);
            gyp = (double*)malloc(sizeof(double) * (size_t)n);
            for (int64_t i = 0; i < n; i++) freed[i] = held[i] ? 0.0 : src[i];
            or_grav_field(cfg, freed, w, h, php, gxp, gyp);
            free(freed);
            free(php);
        }
    }
    double spared[2] = {0.0, 0.0};
    double* push = (double*)calloc(2 * (size_t)n, sizeof(double));
    double kick_net[2] = {0.0, 0.0};
    int64_t densest = -1;
    double best = 0.0;
    double* next = (double*)malloc(sizeof(double) * NC * (size_t)n);
    memcpy(next, planes, sizeof(double) * NC * (size_t)n);
    /* the update (hydro.rs:871-1003), in index order (the spared, kick and push sums are sequential) */
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            if (EMPTY(x, y)) continue;
            int64_t i = y * w + x;
            double u[NC];
            if (VAC(x, y)) {
                r_cons(&H, &grid[AT(x, y)], u);
            } else {
                for (int k = 0; k < 4; k++) u[k] = planes[k * n + i];
                for (int s = 0; s < NS; s++) u[4 + s] = u[0] * planes[(4 + s) * n + i];
            }
            const int held_here = HELD(i);
            const double* fr = fx + NC * (y * (w + 1) + x + 1);
            const double* fl = fx + NC * (y * (w + 1) + x);
            const double* fd = fy + NC * ((y + 1) * w + x);
            const double* fu = fy + NC * (y * w + x);
            for (int k = 0; k < NC; k++) {
                double d = dt * ((fr[k] - fl[k]) + (fd[k] - fu[k]));
                if (held_here && (k == 1 || k == 2)) spared[k - 1] -= d;
                else u[k] -= d;
            }
            if (has_g) {
                const double* m = mids + 3 * i;
                double kick[2] = {dt * src[i] * gxm[i], dt * src[i] * gym[i]};
                const double* ogx = held_here && gxp ? gxp : gxm;
                const double* ogy = held_here && gyp ? gyp : gym;
                kick_net[0] += dt * src[i] * ogx[i];
                kick_net[1] += dt * src[i] * ogy[i];
                if (!held_here && src[i] > 0.0 && (densest < 0 || src[i] > best)) {
                    densest = i;
                    best = src[i];
                }
                double p = phim[i];
                double pr = p, pl = p, pd = p, pu = p;
                const double *mr = m, *ml = m, *md = m, *mu = m;
                if (x + 1 < w) { pr = phim[i + 1]; mr = mids + 3 * (i + 1); }
                if (x > 0) { pl = phim[i - 1]; ml = mids + 3 * (i - 1); }
                if (y + 1 < h) { pd = phim[i + w]; md = mids + 3 * (i + w); }
                if (y > 0) { pu = phim[i - w]; mu = mids + 3 * (i - w); }
                const int64_t kr = y * (w + 1) + x + 1, kl = y * (w + 1) + x, kd = (y + 1) * w + x, ku = y * w + x;
                double r[3] = {0, 0, 0}, l[3] = {0, 0, 0}, dn[3] = {0, 0, 0}, up[3] = {0, 0, 0};
                if (!still_x[kr]) face_work(fr[0], m[0], mr[0], m[1], mr[1], p - pr, dt, r);
                if (!still_x[kl]) face_work(fl[0], ml[0], m[0], ml[1], m[1], pl - p, dt, l);
                if (!still_y[kd]) face_work(fd[0], m[0], md[0], m[2], md[2], p - pd, dt, dn);
                if (!still_y[ku]) face_work(fu[0], mu[0], m[0], mu[2], m[2], pu - p, dt, up);
                kick[0] += r[0] - l[0];
                kick[1] += dn[0] - up[0];
                if (held_here) {
                    if (gxp) {
                        kick[0] = dt * src[i] * gxp[i];
                        kick[1] = dt * src[i] * gyp[i];
                    }
                    spared[0] += kick[0];
                    spared[1] += kick[1];
                } else {
                    u[1] += kick[0];
                    u[2] += kick[1];
                }
                u[3] += r[1] + l[2] + dn[1] + up[2];
            }
            if (radx && !held_here) {
                double a[2], d[2];
                radiation_force(&H, planes, n, i, radx[i], rady[i], a);
                d[0] = dt * a[0];
                d[1] = dt * a[1];
                double s = push_share(&H, u, d);
                push[2 * i] = s * d[0];
                push[2 * i + 1] = s * d[1];
                u[1] += push[2 * i];
                u[2] += push[2 * i + 1];
            }
            for (int k = 0; k < 4; k++) next[k * n + i] = u[k];
            for (int s = 0; s < NS; s++) next[(4 + s) * n + i] = u[4 + s] / u[0];
        }
    /* the radiation force's net push taken back in proportion to each cell's (hydro.rs:975-985) */
    double net[3] = {0.0, 0.0, 0.0};
    for (int64_t i = 0; i < n; i++) {
        double px = push[2 * i], py = push[2 * i + 1];
        net[0] += px;
        net[1] += py;
        net[2] += sqrt(px * px + py * py);
    }
    if (net[2] > 0.0)
        for (int64_t i = 0; i < n; i++) {
            double px = push[2 * i], py = push[2 * i + 1], m = sqrt(px * px + py * py);
            next[n + i] -= m * net[0] / net[2];
            next[2 * n + i] -= m * net[1] / net[2];
        }
    /* gravity's net kick taken back from the densest free cell (hydro.rs:986-991) */
    if (densest >= 0) {
        next[n + densest] -= kick_net[0];
        next[2 * n + densest] -= kick_net[1];
    }
    /* the sticky wall (hydro.rs:992-1012) */
    if (held)
        for (int64_t i = 0; i < n; i++) {
            if (held[i] || next[i] < H.sigma_vac) continue;
            int64_t x = i % w, y = i / w;
            double ux = next[n + i], uy = next[2 * n + i];
            int into[2] = {(x > 0 && held[i - 1] && ux < 0.0) || (x + 1 < w && held[i + 1] && ux > 0.0),
                           (y > 0 && held[i - w] && uy < 0.0) || (y + 1 < h && held[i + w] && uy > 0.0)};
            for (int k = 0; k < 2; k++)
                if (into[k]) {
                    spared[k] += next[(1 + k) * n + i];
                    next[(1 + k) * n + i] = 0.0;
                }
        }
    if (rep) {
        rep->spared[0] = spared[0];
        rep->spared[1] = spared[1];
        rep->kick_net[0] = kick_net[0];
        rep->kick_net[1] = kick_net[1];
        rep->densest = densest;
        rep->push_net[0] = net[0];
        rep->push_net[1] = net[1];
        rep->push_abs = net[2];
    }
    memcpy(planes, next, sizeof(double) * NC * (size_t)n);
    free(next);
    free(push);
    free(src);
    free(phim);
    free(gxm);
    free(gym);
    free(gxp);
    free(gyp);
    free(still_x);
    free(still_y);
    free(mids);
    free(fx);
    free(fy);
    free(grid);
#undef VAC
#undef EMPTY
#undef HELD
#undef AT
}

double or_ref_dt(const sr_config* cfg, const double* planes, int64_t w, int64_t h, const double* gx,
                 const double* gy) {
    /* hydro.rs:618-634 */
    rhyd H;
    rhyd_init(&H, cfg);
    const int64_t n = w * h;
    double rate = 0.0, gmax = 0.0;
    for (int64_t i = 0; i < n; i++) {
        rprim p = r_read(&H, planes, n, i);
        double c = r_sound(&p);
        rate = fmax(rate, (fabs(p.u) + c) + (fabs(p.v) + c));
        if (gx) gmax = fmax(gmax, hypot(gx[i], gy[i]));
    }
    double dt = cfg->cfl / rate;
    if (gmax > 0.0) dt = fmin(dt, cfg->eta_g / sqrt(gmax));
    return dt;
}

/* ======================================================================= P8 (reference/floors.rs) */

static void renormalised(const double* raw, double* out) {
    /* floors.rs:45-58: clamped >= 0 and divided by their sum, pure hydrogen when none is positive */
    double sum = 0.0, c[NS];
    for (int k = 0; k < NS; k++) {
        c[k] = fmax(raw[k], 0.0);
        sum += c[k];
    }
    for (int k = 0; k < NS; k++) out[k] = 0.0;
    if (sum > 0.0)
        for (int k = 0; k < NS; k++) out[k] = c[k] / sum;
    else
        out[0] = 1.0;
}

void or_ref_floors(const sr_config* cfg, double* planes, int64_t w, int64_t h, double* booked2) {
    /* floors.rs:124-175: Σ_vac and Σ_floor compared and written as f32; a cell with a non-finite fraction left as
     * read; booked2: vacuum_reset, floor_added */
    eos_t E;
    eos_init(&E, cfg);
    const int64_t n = w * h;
    const double svac = (double)(float)cfg->sigma_vac, sfloor = (double)(float)cfg->sigma_floor;
    double vac_reset = 0.0, floor_added = 0.0;
    for (int64_t i = 0; i < n; i++) {
        double raw[NS], x[NS];
        int finite = 1;
        for (int k = 0; k < NS; k++) {
            raw[k] = planes[(4 + k) * n + i];
            finite &= isfinite(raw[k]) != 0;
        }
        if (!finite) continue;
        renormalised(raw, x);
        comp_t c = composition(x);
        double mu = 1.0 / c.inv_mu;
        double s = planes[i], energy = planes[3 * n + i];
        if (s < svac) {
            double e = sfloor * (E.t_floor / mu + eos_eps_cold(&E, sfloor, c.y_e, x[ID_N]));
            vac_reset += s - sfloor;
            floor_added += e - energy;
            planes[i] = sfloor;
            planes[n + i] = 0.0;
            planes[2 * n + i] = 0.0;
            planes[3 * n + i] = e;
        } else {
            double added;
            eos_thermal(&E, energy, s, planes[n + i], planes[2 * n + i], c.y_e, x[ID_N], mu, &added);
            planes[3 * n + i] = energy + added;
            floor_added += added;
        }
        for (int k = 0; k < NS; k++) planes[(4 + k) * n + i] = x[k];
    }
    if (booked2) {
        booked2[0] = vac_reset;
        booked2[1] = floor_added;
    }
}

double or_ref_disk_mass(const double* sigma, int64_t w, int64_t h, int64_t x, int64_t y, double r) {
    /* sinks.rs:117-125: the cells of the disk r about (x, y), centre to centre, clipped, row-major */
    int64_t k = (int64_t)r;
    double m = 0.0;
    for (int64_t dy = -k; dy <= k; dy++)
        for (int64_t dx = -k; dx <= k; dx++) {
            int64_t cx = x + dx, cy = y + dy;
            if (cx >= 0 && cy >= 0 && cx < w && cy < h && (double)(dx * dx + dy * dy) <= r * r) m += sigma[cy * w + cx];
        }
    return m;
}

void or_ref_hold(const sr_config* cfg, double* planes, int64_t w, int64_t h, uint8_t* held, double* taken2) {
    /* floors.rs:213-243 (hold) with floors.rs:196-211 (holds): the mask after P8; a newly held cell's momentum
     * zeroed and returned summed */
    eos_t E;
    eos_init(&E, cfg);
    const int64_t n = w * h;
    double taken[2] = {0.0, 0.0};
    for (int64_t i = 0; i < n; i++) {
        double raw[NS], x[NS];
        int finite = 1;
        for (int k = 0; k < NS; k++) {
            raw[k] = planes[(4 + k) * n + i];
            finite &= isfinite(raw[k]) != 0;
        }
        if (!finite) continue;
        renormalised(raw, x);
        comp_t c = composition(x);
        double s = planes[i], mx = planes[n + i], my = planes[2 * n + i], energy = planes[3 * n + i];
        double cold = eos_eps_cold(&E, s, c.y_e, x[ID_N]);
        double eps_th = energy / s - 0.5 * (mx * mx + my * my) / (s * s) - cold;
        int kind = x[ID_FE] < IRON_TRACE || x[ID_N] >= NEUTRON_RICH;
        int was = held[i] != 0, rest;
        if (was) rest = !(eps_th > 2.0 * cfg->eta_hold * cold || s < 0.5 * cfg->sigma_hold || !kind);
        else rest = s >= cfg->sigma_hold && eps_th <= cfg->eta_hold * cold && kind;
        int now = rest && or_ref_disk_mass(planes, w, h, i % w, i / w, cfg->r_hold) < cfg->m_tov;
        if (now && !was) {
            taken[0] += mx;
            taken[1] += my;
            planes[n + i] = 0.0;
            planes[2 * n + i] = 0.0;
        }
        held[i] = (uint8_t)now;
    }
    if (taken2) {
        taken2[0] = taken[0];
        taken2[1] = taken[1];
    }
}

/* ======================================================================= P5 (reference/heat.rs) */

void or_ref_heat_sides(const sr_config* cfg, const double* planes, int64_t w, int64_t h, double* t0, double* kappa,
                       double* inv_mu) {
    /* heat.rs:215-231: each cell's T⁰ (T_floor below Σ_vac), κ = κ₀(1 + X_H) plus κ_dust Z_met below T_dust, 1/μ */
    eos_t E;
    eos_init(&E, cfg);
    const int64_t n = w * h;
    for (int64_t i = 0; i < n; i++) {
        double x[NS];
        for (int k = 0; k < NS; k++) x[k] = planes[(4 + k) * n + i];
        comp_t c = composition(x);
        double mu = 1.0 / c.inv_mu, s = planes[i], t;
        if (s < cfg->sigma_vac) {
            t = E.t_floor;
        } else {
            double eps = eos_thermal(&E, planes[3 * n + i], s, planes[n + i], planes[2 * n + i], c.y_e, x[ID_N], mu,
                                     NULL);
            t = mu * eps;
        }
        t0[i] = t;
        kappa[i] = cfg->kappa0 * (1.0 + x[ID_H]) + (t < cfg->t_dust ? cfg->kappa_dust * c.z_met : 0.0);
        inv_mu[i] = c.inv_mu;
    }
}

void or_ref_heat_step(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, double tol,
                      double newton_heat, double newton_cell, or_heat_report* rep, double* fx, double* fy) {
    /* heat.rs:453-592 on the reference's own sides: C = Σ/μ, T from the EOS with the cold energy, κ of the species */
    const int64_t n = w * h;
    double* t0 = (double*)malloc(sizeof(double) * (size_t)n);
    double* kappa = (double*)malloc(sizeof(double) * (size_t)n);
    double* inv_mu = (double*)malloc(sizeof(double) * (size_t)n);
    or_ref_heat_sides(cfg, planes, w, h, t0, kappa, inv_mu);
    or_heat_step_sides(cfg, planes, w, h, dt, tol, newton_heat, newton_cell, t0, kappa, inv_mu, rep, fx, fy);
    free(t0);
    free(kappa);
    free(inv_mu);
}

/* ======================================================================= the twin (reference/mod.rs) */

struct or_ref_twin {
    sr_config cfg;
    int64_t w, h;
    double* planes;
    uint8_t* mask;
    double *gx, *gy, *phi;
    double* radx;  /* the cell-centred flux the radiation force reads (NULL: none) */
    double* rady;
    double held[2], booked[2];
    double dt, dt_next, sim_time;
    int64_t steps;
    or_heat_report heat;  /* the last P5's report */
    double *hfx, *hfy;    /* the last P5's face fluxes */
};

static void ref_twin_gravity(or_ref_twin* t) {
    if (t->cfg.gravity) or_grav_field(&t->cfg, t->planes, t->w, t->h, t->phi, t->gx, t->gy);
}

static double ref_twin_dt(or_ref_twin* t) {
    double dt = or_ref_dt(&t->cfg, t->planes, t->w, t->h, t->cfg.gravity ? t->gx : NULL, t->cfg.gravity ? t->gy : NULL);
    if (t->cfg.dt_fixed > 0.0) dt = t->cfg.dt_fixed;
    if (t->cfg.dt_cap > 0.0) dt = fmin(dt, t->cfg.dt_cap);
    return dt;
}

static void ref_twin_hold(or_ref_twin* t) {
    double taken[2];
    or_ref_hold(&t->cfg, t->planes, t->w, t->h, t->mask, taken);
    t->held[0] += taken[0];
    t->held[1] += taken[1];
}

or_ref_twin* or_ref_twin_new(const sr_config* cfg, const double* planes, const uint8_t* mask) {
    /* mod.rs:129-177: the hold's rule on the initial state (from `mask`, or none held), P2, Δt_0 */
    or_ref_twin* t = (or_ref_twin*)calloc(1, sizeof(or_ref_twin));
    t->cfg = *cfg;
    t->w = cfg->width;
    t->h = cfg->height;
    const int64_t n = t->w * t->h;
    t->planes = (double*)malloc(sizeof(double) * NC * (size_t)n);
    memcpy(t->planes, planes, sizeof(double) * NC * (size_t)n);
    t->mask = (uint8_t*)calloc((size_t)n, 1);
    if (mask) memcpy(t->mask, mask, (size_t)n);
    t->phi = (double*)calloc((size_t)n, sizeof(double));
    t->gx = (double*)calloc((size_t)n, sizeof(double));
    t->gy = (double*)calloc((size_t)n, sizeof(double));
    ref_twin_hold(t);
    ref_twin_gravity(t);
    t->dt_next = ref_twin_dt(t);
    return t;
}

void or_ref_twin_free(or_ref_twin* t) {
    if (!t) return;
    free(t->planes);
    free(t->mask);
    free(t->phi);
    free(t->gx);
    free(t->gy);
    free(t->radx);
    free(t->rady);
    free(t->hfx);
    free(t->hfy);
    free(t);
}

void or_ref_twin_set_flux(or_ref_twin* t, const double* fx, const double* fy) {
    /* the cell-centred flux the next step's radiation force reads (mod.rs:276-279: the last P5's F) */
    const int64_t n = t->w * t->h;
    if (!t->radx) {
        t->radx = (double*)malloc(sizeof(double) * (size_t)n);
        t->rady = (double*)malloc(sizeof(double) * (size_t)n);
    }
    memcpy(t->radx, fx, sizeof(double) * (size_t)n);
    memcpy(t->rady, fy, sizeof(double) * (size_t)n);
}

void or_ref_twin_step(or_ref_twin* t) {
    /* mod.rs:264-297: P1, P2, P4 (step_held), P5 (its F the next step's radiation force), P8 (floors, then the hold),
     * P9 */
    double dt = t->dt_next;
    t->dt = dt;
    t->sim_time += dt;
    ref_twin_gravity(t);
    if (t->cfg.hydro) {
        or_ref_hydro_report rep;
        or_ref_hydro_step(&t->cfg, t->planes, t->w, t->h, dt, t->cfg.gravity ? t->gx : NULL,
                          t->cfg.gravity ? t->gy : NULL, t->mask, t->radx, t->rady, &rep);
        t->held[0] += rep.spared[0];
        t->held[1] += rep.spared[1];
    }
    if (t->cfg.heat) {
        const int64_t w = t->w, h = t->h, n = w * h;
        if (!t->hfx) {
            t->hfx = (double*)malloc(sizeof(double) * (size_t)((w + 1) * h));
            t->hfy = (double*)malloc(sizeof(double) * (size_t)(w * (h + 1)));
            t->radx = (double*)malloc(sizeof(double) * (size_t)n);
            t->rady = (double*)malloc(sizeof(double) * (size_t)n);
        }
        /* the twin's tolerances (heat.rs:59-62) */
        or_ref_heat_step(&t->cfg, t->planes, w, h, dt, 1e-12, 1e-12, 1e-10, &t->heat, t->hfx, t->hfy);
        /* heat.rs:100-112: the cell-centred F, the mean of a cell's two faces on each axis */
        for (int64_t y = 0; y < h; y++)
            for (int64_t x = 0; x < w; x++) {
                t->radx[y * w + x] = 0.5 * (t->hfx[y * (w + 1) + x] + t->hfx[y * (w + 1) + x + 1]);
                t->rady[y * w + x] = 0.5 * (t->hfy[y * w + x] + t->hfy[(y + 1) * w + x]);
            }
    }
    double booked[2];
    or_ref_floors(&t->cfg, t->planes, t->w, t->h, booked);
    t->booked[0] += booked[0];
    t->booked[1] += booked[1];
    ref_twin_hold(t);
    t->dt_next = ref_twin_dt(t);
    t->steps++;
}

void or_ref_twin_state(const or_ref_twin* t, double* planes, uint8_t* mask) {
    const int64_t n = t->w * t->h;
    if (planes) memcpy(planes, t->planes, sizeof(double) * NC * (size_t)n);
    if (mask) memcpy(mask, t->mask, (size_t)n);
}

void or_ref_twin_clock(const or_ref_twin* t, double* out4) {
    out4[0] = t->dt;
    out4[1] = t->dt_next;
    out4[2] = t->sim_time;
    out4[3] = (double)t->steps;
}

void or_ref_twin_heat(const or_ref_twin* t, or_heat_report* rep, double* fx, double* fy) {
    if (rep) *rep = t->heat;
    const int64_t w = t->w, h = t->h;
    if (fx && t->hfx) memcpy(fx, t->hfx, sizeof(double) * (size_t)((w + 1) * h));
    if (fy && t->hfy) memcpy(fy, t->hfy, sizeof(double) * (size_t)(w * (h + 1)));
}

void or_ref_twin_books(const or_ref_twin* t, double* out4) {
    out4[0] = t->held[0];
    out4[1] = t->held[1];
    out4[2] = t->booked[0];
    out4[3] = t->booked[1];
}
