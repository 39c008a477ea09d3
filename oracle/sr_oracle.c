/*
 * sr_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU f64 restatement of the reference's twin
 * (crates/sr-physics/src/reference/{fft,grav,hydro,heat,riemann,floors,mod}.rs). Only tests/, the smoke check and
 * bench.py's CPU baseline use it; the product never links it. Each function names the reference lines it follows.
 *
 * Config mode generalises three of the reference's fixed choices, each reducing to the reference's arithmetic at the
 * reference's value: γ (Π = (γ-1)Σε, c² = γΠ/Σ, T = μ(γ-1)ε; the reference's γ = 2 gives Π = Σε, c² = 2Π/Σ,
 * T = με), the limiter (minmod beside MC) and the gravity kernel (softened beside the exact self cell). The cold
 * pressures and the ten species of the reference EOS are not carried (4 channels). Sums the reference takes cell by
 * cell in index order are taken here as per-row partials added in row order, so that results do not depend on the
 * thread count; they differ from a strictly sequential sum by rounding only.
 */
#define _GNU_SOURCE
#include "sr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SELF_CELL 3.525494348078172 /* reference/grav.rs:24-25: 4 ln(1 + sqrt 2) */
#define HOT_FACE 2.0                /* reference/hydro.rs:301 */

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ======================================================================= FFT (reference/fft.rs) */

int64_t or_padded_size(int64_t len, int64_t cap) {
    /* fft.rs:92-101: smallest power of two >= 2 len, at least MIN_PADDED = 32, refused past the cap. */
    if (len <= 0) return 0;
    int64_t n = 1;
    while (n < 2 * len) n <<= 1;
    if (n < 32) n = 32;
    if (n > cap) return 0;
    return n;
}

static int is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

int or_fft(int64_t n, double* re, double* im, int inverse) {
    /* fft.rs:106-172: twiddles e^{-2πik/N} each from its own sin/cos; bit reversal; iterative butterflies. */
    if (!is_pow2(n)) return -1;
    int bits = 0;
    while ((1LL << bits) < n) bits++;
    for (int64_t i = 0; i < n; i++) {
        int64_t j = 0;
        for (int b = 0; b < bits; b++)
            if (i & (1LL << b)) j |= 1LL << (bits - 1 - b);
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    int64_t halfn = n / 2;
    double* tc = (double*)malloc(sizeof(double) * (size_t)(halfn > 0 ? halfn : 1));
    double* ts = (double*)malloc(sizeof(double) * (size_t)(halfn > 0 ? halfn : 1));
    for (int64_t k = 0; k < halfn; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        tc[k] = cos(a);
        ts[k] = sin(a);
    }
    for (int64_t half = 1; half < n; half *= 2) {
        int64_t step = n / (2 * half);
        for (int64_t start = 0; start < n; start += 2 * half) {
            for (int64_t k = 0; k < half; k++) {
                double wr = tc[k * step], wi = inverse ? -ts[k * step] : ts[k * step];
                int64_t a = start + k, b = start + k + half;
                double br = re[b] * wr - im[b] * wi;
                double bi = re[b] * wi + im[b] * wr;
                double ar = re[a], ai = im[a];
                re[a] = ar + br; im[a] = ai + bi;
                re[b] = ar - br; im[b] = ai - bi;
            }
        }
    }
    free(tc);
    free(ts);
    if (inverse) {
        double scale = 1.0 / (double)n;
        for (int64_t i = 0; i < n; i++) { re[i] *= scale; im[i] *= scale; }
    }
    return 0;
}

int or_fft2(int64_t nx, int64_t ny, double* re, double* im, int inverse) {
    /* fft.rs:174-196: every row with plan_x, then every column with plan_y. */
    if (!is_pow2(nx) || !is_pow2(ny)) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < ny; y++) or_fft(nx, re + y * nx, im + y * nx, inverse);
#pragma omp parallel
    {
        double* cr = (double*)malloc(sizeof(double) * (size_t)ny);
        double* ci = (double*)malloc(sizeof(double) * (size_t)ny);
#pragma omp for schedule(static)
        for (int64_t x = 0; x < nx; x++) {
            for (int64_t y = 0; y < ny; y++) { cr[y] = re[y * nx + x]; ci[y] = im[y * nx + x]; }
            or_fft(ny, cr, ci, inverse);
            for (int64_t y = 0; y < ny; y++) { re[y * nx + x] = cr[y]; im[y * nx + x] = ci[y]; }
        }
        free(cr);
        free(ci);
    }
    return 0;
}

static int64_t signed_offset(int64_t i, int64_t n) { return i < n / 2 ? i : i - n; } /* fft.rs:198-207 */

static double kernel_value(const sr_config* cfg, int64_t dx, int64_t dy) {
    /* reference/grav.rs:27-34 (exact self cell) or the Plummer-softened kernel of the configs. */
    double r2 = (double)(dx * dx + dy * dy);
    if (cfg->kernel == SR_KERNEL_SOFTENED) return -cfg->G / sqrt(r2 + cfg->softening * cfg->softening);
    if (dx == 0 && dy == 0) return -cfg->G * SELF_CELL;
    return -cfg->G / sqrt(r2);
}

void or_kernel_table(const sr_config* cfg, int64_t px, int64_t py, double* ktab) {
    for (int64_t j = 0; j < py; j++)
        for (int64_t i = 0; i < px; i++) ktab[j * px + i] = kernel_value(cfg, signed_offset(i, px), signed_offset(j, py));
}

static int convolve_spectrum(const double* field, int64_t w, int64_t h, int64_t ring, const double* kre,
                             const double* kim, int64_t px, int64_t py, double* out) {
    /* fft.rs:238-282: zero-pad, forward, multiply by the kernel's spectrum, inverse, read the ringed box. */
    size_t np = (size_t)(px * py);
    double* re = (double*)calloc(np, sizeof(double));
    double* im = (double*)calloc(np, sizeof(double));
    if (!re || !im) { free(re); free(im); return -1; }
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) re[y * px + x] = field[y * w + x];
    or_fft2(px, py, re, im, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)np; i++) {
        double ar = re[i], ai = im[i];
        re[i] = ar * kre[i] - ai * kim[i];
        im[i] = ar * kim[i] + ai * kre[i];
    }
    or_fft2(px, py, re, im, 1);
    int64_t rw = w + 2 * ring, rh = h + 2 * ring;
    for (int64_t y = 0; y < rh; y++)
        for (int64_t x = 0; x < rw; x++) {
            int64_t sx = (x + px - ring) % px, sy = (y + py - ring) % py;
            out[y * rw + x] = re[sy * px + sx];
        }
    free(re);
    free(im);
    return 0;
}

int or_convolve_ringed(const double* field, int64_t w, int64_t h, int64_t ring, const double* ktab, int64_t px,
                       int64_t py, double* out) {
    if (!is_pow2(px) || !is_pow2(py)) return -1;
    size_t np = (size_t)(px * py);
    double* kre = (double*)malloc(np * sizeof(double));
    double* kim = (double*)calloc(np, sizeof(double));
    memcpy(kre, ktab, np * sizeof(double));
    or_fft2(px, py, kre, kim, 0);
    int rc = convolve_spectrum(field, w, h, ring, kre, kim, px, py, out);
    free(kre);
    free(kim);
    return rc;
}

/* The kernel spectrum cache of the gravity pass (fft.rs:230-236 caches per padded size). */
static struct {
    int64_t px, py;
    int kind;
    double G, eps;
    double *re, *im;
} kcache = {0, 0, -1, 0, 0, NULL, NULL};

static void kernel_spectrum(const sr_config* cfg, int64_t px, int64_t py, double** kre, double** kim) {
    if (kcache.re && kcache.px == px && kcache.py == py && kcache.kind == (int)cfg->kernel && kcache.G == cfg->G &&
        kcache.eps == cfg->softening) {
        *kre = kcache.re;
        *kim = kcache.im;
        return;
    }
    free(kcache.re);
    free(kcache.im);
    size_t np = (size_t)(px * py);
    kcache.re = (double*)malloc(np * sizeof(double));
    kcache.im = (double*)calloc(np, sizeof(double));
    or_kernel_table(cfg, px, py, kcache.re);
    or_fft2(px, py, kcache.re, kcache.im, 0);
    kcache.px = px;
    kcache.py = py;
    kcache.kind = (int)cfg->kernel;
    kcache.G = cfg->G;
    kcache.eps = cfg->softening;
    *kre = kcache.re;
    *kim = kcache.im;
}

int or_grav_field(const sr_config* cfg, const double* sigma, int64_t w, int64_t h, double* phi, double* gx,
                  double* gy) {
    /* grav.rs:115-121 field(): source mask (37-40), convolve_ringed with RING = 1, acceleration (55-70). The
     * reference caps padded axes at 2048; this restatement lifts the cap to 8192. */
    int64_t px = or_padded_size(w, 8192), py = or_padded_size(h, 8192);
    if (!px || !py) return -1;
    double* src = (double*)malloc(sizeof(double) * (size_t)(w * h));
    for (int64_t i = 0; i < w * h; i++) src[i] = sigma[i] >= cfg->sigma_vac ? sigma[i] : 0.0;
    int64_t rw = w + 2, rh = h + 2;
    double* ringed = (double*)malloc(sizeof(double) * (size_t)(rw * rh));
    double *kre, *kim;
    kernel_spectrum(cfg, px, py, &kre, &kim);
    int rc = convolve_spectrum(src, w, h, 1, kre, kim, px, py, ringed);
    free(src);
    if (rc) { free(ringed); return rc; }
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            /* the box's (x, y) sits at (x + 1, y + 1) of the ringed field */
            gx[y * w + x] = -(ringed[(y + 1) * rw + x + 2] - ringed[(y + 1) * rw + x]) / 2.0;
            gy[y * w + x] = -(ringed[(y + 2) * rw + x + 1] - ringed[y * rw + x + 1]) / 2.0;
            phi[y * w + x] = ringed[(y + 1) * rw + x + 1];
        }
    free(ringed);
    return 0;
}

void or_direct_potential(const sr_config* cfg, const double* src, int64_t w, int64_t h, int64_t n,
                         const int64_t* tx, const int64_t* ty, double* out) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t t = 0; t < n; t++) {
        double sum = 0.0;
        for (int64_t sy = 0; sy < h; sy++)
            for (int64_t sx = 0; sx < w; sx++) {
                double s = src[sy * w + sx];
                if (s != 0.0) sum += kernel_value(cfg, tx[t] - sx, ty[t] - sy) * s;
            }
        out[t] = sum;
    }
}

/* ======================================================================= Hydro (reference/hydro.rs) */

typedef struct { double s, u, v, p; } prim; /* Σ, u, v, Π (hydro.rs:226-233, no species) */
typedef struct { double U[4]; prim p; } face; /* hydro.rs:277-281 */

typedef struct {
    double gamma, gm1, eps_floor, sigma_vac, sigma_floor;
    int limiter, bracket, edge;
} hyd;

static hyd hyd_of(const sr_config* cfg) {
    hyd H;
    H.gamma = cfg->gamma;
    H.gm1 = cfg->gamma - 1.0;
    /* T = μ(γ-1)ε: the floor ε is T_floor/(μ(γ-1)) (eos.rs:250-263's T_floor/μ at γ = 2) */
    H.eps_floor = cfg->t_floor / cfg->mu / H.gm1;
    H.sigma_vac = cfg->sigma_vac;
    H.sigma_floor = cfg->sigma_floor;
    H.limiter = (int)cfg->limiter;
    H.bracket = (int)cfg->thermal_bracket;
    H.edge = (int)cfg->edge;
    return H;
}

static double h_pi(const hyd* H, double s, double eps) { return H->gm1 * s * eps; } /* eos.rs:207-210 */

static prim h_read(const hyd* H, double s, double mx, double my, double E) {
    /* hydro.rs:424-441: the floor state below Σ_vac; else ε_th recovered and floored (eos.rs:250-263) */
    prim p;
    if (s < H->sigma_vac) {
        p.s = H->sigma_floor;
        p.u = 0.0;
        p.v = 0.0;
        p.p = h_pi(H, H->sigma_floor, H->eps_floor);
        return p;
    }
    double kinetic = 0.5 * (mx * mx + my * my) / (s * s);
    double raw = E / s - kinetic;
    double eps = raw < H->eps_floor ? H->eps_floor : raw;
    p.s = s;
    p.u = mx / s;
    p.v = my / s;
    p.p = h_pi(H, s, eps);
    return p;
}

static void h_cons(const hyd* H, const prim* p, double* U) {
    /* hydro.rs:443-460 */
    double thermal = p->p / p->s / H->gm1;
    double eps = fmax(thermal, H->eps_floor);
    U[0] = p->s;
    U[1] = p->s * p->u;
    U[2] = p->s * p->v;
    U[3] = p->s * eps + 0.5 * p->s * (p->u * p->u + p->v * p->v);
}

static int h_prim(const hyd* H, const double* U, prim* out) {
    /* hydro.rs:462-478: None when Σ <= 0, not finite, or no thermal energy left */
    double s = U[0];
    if (isnan(s) || s <= 0.0) return 0;
    for (int k = 0; k < 4; k++)
        if (!isfinite(U[k])) return 0;
    double raw = U[3] / s - 0.5 * (U[1] * U[1] + U[2] * U[2]) / (s * s);
    if (isnan(raw) || raw <= 0.0) return 0;
    double eps = fmax(raw, H->eps_floor);
    out->s = s;
    out->u = U[1] / s;
    out->v = U[2] / s;
    out->p = h_pi(H, s, eps);
    return 1;
}

static double h_sound(const hyd* H, const prim* p) { /* hydro.rs:480-483, eos.rs:244-247 with γ */
    double c2 = H->gamma * p->p / p->s;
    return sqrt(fmax(c2, 0.0));
}

static void h_flux(const prim* p, double energy, int dir, double* f) {
    /* hydro.rs:485-499 */
    double un = dir == 0 ? p->u : p->v, ut = dir == 0 ? p->v : p->u;
    double mass = p->s * un;
    f[0] = mass;
    f[1 + dir] = mass * un + p->p;
    f[2 - dir] = mass * ut;
    f[3] = (energy + p->p) * un;
}

static double lim_mc(double l, double c, double r) { /* hydro.rs:283-289 */
    double a = c - l, b = r - c;
    if (a * b <= 0.0) return 0.0;
    double m = fmin(fmin(fabs(0.5 * (a + b)), 2.0 * fabs(a)), 2.0 * fabs(b));
    return copysign(m, a);
}

static double lim_minmod(double l, double c, double r) {
    double a = c - l, b = r - c;
    if (a * b <= 0.0) return 0.0;
    return copysign(fmin(fabs(a), fabs(b)), a);
}

static prim h_slope(const hyd* H, const prim* l, const prim* c, const prim* r) {
    /* hydro.rs:310-331: per-component limited slopes, Σ and Π flat where the thermal bracket refuses a face */
    double (*lim)(double, double, double) = H->limiter == SR_LIMITER_MINMOD ? lim_minmod : lim_mc;
    prim s;
    s.s = lim(l->s, c->s, r->s);
    s.u = lim(l->u, c->u, r->u);
    s.v = lim(l->v, c->v, r->v);
    s.p = lim(l->p, c->p, r->p);
    if (H->bracket) {
        double hottest = fmax(fmax(l->p / l->s, c->p / c->s), r->p / r->s);
        int hot = 0;
        for (int k = 0; k < 2; k++) {
            double f = k ? 0.5 : -0.5;
            double pif = c->p + f * s.p, bound = HOT_FACE * hottest * (c->s + f * s.s);
            if (!(pif <= bound)) hot = 1; /* greater, or not a number */
        }
        if (hot) { s.s = 0.0; s.p = 0.0; }
    }
    return s;
}

static prim p_offset(const prim* c, const prim* s, double f) {
    prim o = {c->s + f * s->s, c->u + f * s->u, c->v + f * s->v, c->p + f * s->p};
    return o;
}

static face h_evolved(const hyd* H, const prim* base, const double* delta) {
    /* hydro.rs:501-513 */
    face F;
    double U0[4];
    h_cons(H, base, U0);
    double U[4];
    for (int k = 0; k < 4; k++) U[k] = U0[k] + delta[k];
    prim p;
    if (h_prim(H, U, &p)) {
        memcpy(F.U, U, sizeof U);
        F.p = p;
    } else {
        memcpy(F.U, U0, sizeof U0);
        F.p = *base;
    }
    return F;
}

static void h_predicted(const hyd* H, const prim* grid, int64_t pw, int64_t gi, double half, int has_g, double gx,
                        double gy, face* out4, double* mid3) {
    /* hydro.rs:587-614: slopes on both axes, four face states, the Hancock half step of both axes' flux differences,
     * each face kicked by half a step of g */
    const prim* c = &grid[gi];
    prim sx = h_slope(H, &grid[gi - 1], c, &grid[gi + 1]);
    prim sy = h_slope(H, &grid[gi - pw], c, &grid[gi + pw]);
    prim wf[4] = {p_offset(c, &sx, -0.5), p_offset(c, &sx, 0.5), p_offset(c, &sy, -0.5), p_offset(c, &sy, 0.5)};
    double uf[4][4];
    for (int k = 0; k < 4; k++) h_cons(H, &wf[k], uf[k]);
    double fxl[4], fxr[4], fyl[4], fyr[4];
    h_flux(&wf[0], uf[0][3], 0, fxl);
    h_flux(&wf[1], uf[1][3], 0, fxr);
    h_flux(&wf[2], uf[2][3], 1, fyl);
    h_flux(&wf[3], uf[3][3], 1, fyr);
    double delta[4];
    for (int k = 0; k < 4; k++) delta[k] = half * ((fxl[k] - fxr[k]) + (fyl[k] - fyr[k]));
    mid3[0] = c->s + delta[0];
    mid3[1] = c->s * c->u + delta[1];
    mid3[2] = c->s * c->v + delta[2];
    if (!has_g) {
        for (int k = 0; k < 4; k++) out4[k] = h_evolved(H, &wf[k], delta);
        return;
    }
    mid3[1] += half * c->s * gx;
    mid3[2] += half * c->s * gy;
    for (int k = 0; k < 4; k++) {
        const prim* p = &wf[k];
        double d[4] = {delta[0], delta[1], delta[2], delta[3]};
        d[1] += half * p->s * gx;
        d[2] += half * p->s * gy;
        d[3] += half * p->s * ((p->u + 0.5 * half * gx) * gx + (p->v + 0.5 * half * gy) * gy);
        out4[k] = h_evolved(H, p, d);
    }
}

static void h_hll(const hyd* H, const face* l, const face* r, int dir, double* f) {
    /* hydro.rs:516-540: HLL with Davis speeds */
    double unl = dir == 0 ? l->p.u : l->p.v, unr = dir == 0 ? r->p.u : r->p.v;
    double cl = h_sound(H, &l->p), cr = h_sound(H, &r->p);
    double s_l = fmin(unl - cl, unr - cr);
    double s_r = fmax(unl + cl, unr + cr);
    double fl[4], fr[4];
    h_flux(&l->p, l->U[3], dir, fl);
    h_flux(&r->p, r->U[3], dir, fr);
    if (s_l >= 0.0) {
        memcpy(f, fl, sizeof fl);
    } else if (s_r <= 0.0) {
        memcpy(f, fr, sizeof fr);
    } else {
        for (int k = 0; k < 4; k++) f[k] = (s_r * fl[k] - s_l * fr[k] + s_l * s_r * (r->U[k] - l->U[k])) / (s_r - s_l);
    }
}

static void h_wall(const face* own, int dir, double* f) { /* hydro.rs:556-562 */
    f[0] = f[1] = f[2] = f[3] = 0.0;
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
            double sg = copysign(1.0, du); /* f64::signum */
            kick = -2.0 * c / (du + sg * disc);
            el = ul * kick + 0.5 * kick * kick / a;
            eh = -uh * kick + 0.5 * kick * kick / b;
        }
    }
    double rest = extra + c;
    out3[0] = kick;
    out3[1] = 0.5 * dt * pl * d + w * rest + el;
    out3[2] = 0.5 * dt * ph * d + (1.0 - w) * rest + eh;
}

void or_hydro_step(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, const double* gx,
                   const double* gy, or_hydro_report* rep) {
    /* hydro.rs:657-1025 (step_held with no held cells, no sinks, no radiation force) */
    hyd H = hyd_of(cfg);
    const int64_t n = w * h, G2 = 2, pw = w + 4, ph = h + 4;
    const double* S = planes;
    const double* MX = planes + n;
    const double* MY = planes + 2 * n;
    const double* EN = planes + 3 * n;
    int has_g = gx != NULL;
#define AT(x, y) (((y) + G2) * pw + (x) + G2)
    prim* grid = (prim*)malloc(sizeof(prim) * (size_t)(pw * ph));
    for (int64_t i = 0; i < pw * ph; i++) { grid[i].s = 1.0; grid[i].u = 0.0; grid[i].v = 0.0; grid[i].p = 1.0; }
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            int64_t i = y * w + x;
            grid[AT(x, y)] = h_read(&H, S[i], MX[i], MY[i], EN[i]);
        }
    /* ghosts (hydro.rs:686-709): columns first, then rows over the full padded width */
    for (int64_t y = 0; y < h; y++)
        for (int64_t k = 1; k <= G2; k++) {
            prim a, b;
            if (H.edge == SR_EDGE_BOUNCE) {
                a = grid[AT(k - 1, y)]; a.u = -a.u;
                b = grid[AT(w - k, y)]; b.u = -b.u;
            } else {
                a = grid[AT(0, y)]; a.u = fmin(a.u, 0.0);
                b = grid[AT(w - 1, y)]; b.u = fmax(b.u, 0.0);
            }
            grid[(y + G2) * pw + G2 - k] = a;
            grid[(y + G2) * pw + G2 + w - 1 + k] = b;
        }
    for (int64_t px = 0; px < pw; px++)
        for (int64_t k = 1; k <= G2; k++) {
            prim a, b;
            if (H.edge == SR_EDGE_BOUNCE) {
                a = grid[(G2 + k - 1) * pw + px]; a.v = -a.v;
                b = grid[(G2 + h - k) * pw + px]; b.v = -b.v;
            } else {
                a = grid[G2 * pw + px]; a.v = fmin(a.v, 0.0);
                b = grid[(G2 + h - 1) * pw + px]; b.v = fmax(b.v, 0.0);
            }
            grid[(G2 - k) * pw + px] = a;
            grid[(G2 + h - 1 + k) * pw + px] = b;
        }
    const double half = 0.5 * dt;
    face* faces = (face*)malloc(sizeof(face) * 4 * (size_t)n);
    double* mids = (double*)malloc(sizeof(double) * 3 * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            int64_t i = y * w + x;
            h_predicted(&H, grid, pw, AT(x, y), half, has_g, has_g ? gx[i] : 0.0, has_g ? gy[i] : 0.0, faces + 4 * i,
                        mids + 3 * i);
        }
    /* boundary faces (hydro.rs:564-582): bounce → wall; leave → HLL against the ghost's predicted face, inflow → wall */
#define BOUNDARY(side, own, gcell, gxv, gyv, out)                                                          \
    do {                                                                                                   \
        int dir_ = (side) / 2, high_ = (side) % 2;                                                         \
        if (H.edge == SR_EDGE_BOUNCE) {                                                                    \
            h_wall((own), dir_, (out));                                                                    \
        } else {                                                                                           \
            face gf_[4];                                                                                   \
            double gm_[3];                                                                                 \
            h_predicted(&H, grid, pw, (gcell), half, has_g, (gxv), (gyv), gf_, gm_);                       \
            if (high_) h_hll(&H, (own), &gf_[(side) - 1], dir_, (out));                                    \
            else h_hll(&H, &gf_[(side) + 1], (own), dir_, (out));                                          \
            int inflow_ = high_ ? (out)[0] < 0.0 : (out)[0] > 0.0;                                         \
            if (inflow_) h_wall((own), dir_, (out));                                                       \
        }                                                                                                  \
    } while (0)
    double* fx = (double*)malloc(sizeof(double) * 4 * (size_t)((w + 1) * h));
    double* fy = (double*)malloc(sizeof(double) * 4 * (size_t)(w * (h + 1)));
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t i = 0; i <= w; i++) {
            double* f = fx + 4 * (y * (w + 1) + i);
            if (i == 0) {
                int64_t e = y * w;
                BOUNDARY(0, &faces[4 * e + 0], AT(0, y) - 1, has_g ? gx[e] : 0.0, has_g ? gy[e] : 0.0, f);
            } else if (i == w) {
                int64_t e = y * w + w - 1;
                BOUNDARY(1, &faces[4 * e + 1], AT(w - 1, y) + 1, has_g ? gx[e] : 0.0, has_g ? gy[e] : 0.0, f);
            } else {
                h_hll(&H, &faces[4 * (y * w + i - 1) + 1], &faces[4 * (y * w + i) + 0], 0, f);
            }
        }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j <= h; j++)
        for (int64_t x = 0; x < w; x++) {
            double* f = fy + 4 * (j * w + x);
            if (j == 0) {
                int64_t e = x;
                BOUNDARY(2, &faces[4 * e + 2], AT(x, 0) - pw, has_g ? gx[e] : 0.0, has_g ? gy[e] : 0.0, f);
            } else if (j == h) {
                int64_t e = (h - 1) * w + x;
                BOUNDARY(3, &faces[4 * e + 3], AT(x, h - 1) + pw, has_g ? gx[e] : 0.0, has_g ? gy[e] : 0.0, f);
            } else {
                h_hll(&H, &faces[4 * ((j - 1) * w + x) + 3], &faces[4 * (j * w + x) + 2], 1, f);
            }
        }
#undef BOUNDARY
    free(faces);
    /* vacuum / empty (hydro.rs:733-742) */
#define VAC(x, y) (S[(y) * w + (x)] < H.sigma_vac)
#define EMPTY(x, y)                                                                                         \
    (VAC(x, y) && ((x) == 0 || VAC((x) - 1, y)) && ((x) + 1 == w || VAC((x) + 1, y)) && ((y) == 0 || VAC(x, (y) - 1)) && \
     ((y) + 1 == h || VAC(x, (y) + 1)))
    /* the half step's field (hydro.rs:815-856): Σ_src,mid = ½(Σⁿ + Σⁿ⁺¹), masked, solved by P2's convolution */
    double *src = NULL, *phim = NULL, *gxm = NULL, *gym = NULL;
    if (has_g) {
        src = (double*)malloc(sizeof(double) * (size_t)n);
        phim = (double*)malloc(sizeof(double) * (size_t)n);
        gxm = (double*)malloc(sizeof(double) * (size_t)n);
        gym = (double*)malloc(sizeof(double) * (size_t)n);
#pragma omp parallel for schedule(static)
        for (int64_t y = 0; y < h; y++)
            for (int64_t x = 0; x < w; x++) {
                int64_t i = y * w + x;
                double s;
                if (EMPTY(x, y)) {
                    s = 0.0;
                } else {
                    double start = VAC(x, y) ? grid[AT(x, y)].s : S[i];
                    double div = (fx[4 * (y * (w + 1) + x + 1)] - fx[4 * (y * (w + 1) + x)]) +
                                 (fy[4 * ((y + 1) * w + x)] - fy[4 * (y * w + x)]);
                    s = 0.5 * (S[i] + (start - dt * div));
                }
                src[i] = s >= H.sigma_vac ? s : 0.0;
            }
        or_grav_field(cfg, src, w, h, phim, gxm, gym);
    }
    /* the update (hydro.rs:871-1003) */
    double* next = (double*)malloc(sizeof(double) * 4 * (size_t)n);
    memcpy(next, planes, sizeof(double) * 4 * (size_t)n);
    double* kick_cell = has_g ? (double*)calloc(2 * (size_t)n, sizeof(double)) : NULL;
    double* esc_cell = (double*)calloc(4 * (size_t)n, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            if (EMPTY(x, y)) continue;
            int64_t i = y * w + x;
            double u[4];
            if (VAC(x, y)) {
                h_cons(&H, &grid[AT(x, y)], u);
            } else {
                u[0] = S[i]; u[1] = MX[i]; u[2] = MY[i]; u[3] = EN[i];
            }
            const double* fr = fx + 4 * (y * (w + 1) + x + 1);
            const double* fl = fx + 4 * (y * (w + 1) + x);
            const double* fd = fy + 4 * ((y + 1) * w + x);
            const double* fu = fy + 4 * (y * w + x);
            for (int k = 0; k < 4; k++) u[k] -= dt * ((fr[k] - fl[k]) + (fd[k] - fu[k]));
            if (has_g) {
                const double* m = mids + 3 * i;
                double kick[2] = {dt * src[i] * gxm[i], dt * src[i] * gym[i]};
                kick_cell[2 * i] = kick[0];
                kick_cell[2 * i + 1] = kick[1];
                double p = phim[i];
                double pr = p, pl = p, pd = p, pu = p;
                const double *mr = m, *ml = m, *md = m, *mu = m;
                if (x + 1 < w) { pr = phim[i + 1]; mr = mids + 3 * (i + 1); }
                if (x > 0) { pl = phim[i - 1]; ml = mids + 3 * (i - 1); }
                if (y + 1 < h) { pd = phim[i + w]; md = mids + 3 * (i + w); }
                if (y > 0) { pu = phim[i - w]; mu = mids + 3 * (i - w); }
                double r[3], l[3], dn[3], up[3];
                face_work(fr[0], m[0], mr[0], m[1], mr[1], p - pr, dt, r);
                face_work(fl[0], ml[0], m[0], ml[1], m[1], pl - p, dt, l);
                face_work(fd[0], m[0], md[0], m[2], md[2], p - pd, dt, dn);
                face_work(fu[0], mu[0], m[0], mu[2], m[2], pu - p, dt, up);
                kick[0] += r[0] - l[0];
                kick[1] += dn[0] - up[0];
                u[1] += kick[0];
                u[2] += kick[1];
                u[3] += r[1] + l[2] + dn[1] + up[2];
            }
            /* escaped (hydro.rs:948-973): each boundary face's flux as the cell took it */
            double phi_edge = has_g ? phim[i] : 0.0;
            double* esc = esc_cell + 4 * i;
            if (x == 0) { for (int k = 0; k < 4; k++) esc[k] += -dt * fl[k]; esc[3] += -dt * fl[0] * phi_edge; }
            if (x + 1 == w) { for (int k = 0; k < 4; k++) esc[k] += dt * fr[k]; esc[3] += dt * fr[0] * phi_edge; }
            if (y == 0) { for (int k = 0; k < 4; k++) esc[k] += -dt * fu[k]; esc[3] += -dt * fu[0] * phi_edge; }
            if (y + 1 == h) { for (int k = 0; k < 4; k++) esc[k] += dt * fd[k]; esc[3] += dt * fd[0] * phi_edge; }
            for (int k = 0; k < 4; k++) next[k * n + i] = u[k];
        }
    /* the net kick taken back from the densest free cell, the lowest index on a tie (hydro.rs:1008-1012) */
    double kn[2] = {0.0, 0.0};
    int64_t densest = -1;
    double best = 0.0;
    if (has_g) {
        for (int64_t y = 0; y < h; y++) {
            double rowk[2] = {0.0, 0.0};
            for (int64_t x = 0; x < w; x++) {
                int64_t i = y * w + x;
                if (EMPTY(x, y)) continue;
                rowk[0] += kick_cell[2 * i];
                rowk[1] += kick_cell[2 * i + 1];
                if (src[i] > 0.0 && (densest < 0 || src[i] > best)) { densest = i; best = src[i]; }
            }
            kn[0] += rowk[0];
            kn[1] += rowk[1];
        }
        if (densest >= 0) {
            next[n + densest] -= kn[0];
            next[2 * n + densest] -= kn[1];
        }
    }
    if (rep) {
        rep->kick_net[0] = kn[0];
        rep->kick_net[1] = kn[1];
        rep->densest = densest;
        for (int k = 0; k < 4; k++) {
            double t = 0.0;
            for (int64_t i = 0; i < n; i++) t += esc_cell[4 * i + k];
            rep->escaped[k] = t;
        }
    }
    memcpy(planes, next, sizeof(double) * 4 * (size_t)n);
    free(next);
    free(esc_cell);
    free(kick_cell);
    free(src);
    free(phim);
    free(gxm);
    free(gym);
    free(mids);
    free(fx);
    free(fy);
    free(grid);
#undef VAC
#undef EMPTY
#undef AT
}

double or_hydro_dt(const sr_config* cfg, const double* planes, int64_t w, int64_t h, const double* gx,
                   const double* gy) {
    /* hydro.rs:618-634 */
    hyd H = hyd_of(cfg);
    int64_t n = w * h;
    double rate = 0.0, gmax = 0.0;
#pragma omp parallel for reduction(max : rate, gmax) schedule(static)
    for (int64_t i = 0; i < n; i++) {
        prim p = h_read(&H, planes[i], planes[n + i], planes[2 * n + i], planes[3 * n + i]);
        double c = h_sound(&H, &p);
        double r = (fabs(p.u) + c) + (fabs(p.v) + c);
        if (r > rate) rate = r;
        if (gx) {
            double g = hypot(gx[i], gy[i]);
            if (g > gmax) gmax = g;
        }
    }
    double dt = cfg->cfl / rate;
    if (gmax > 0.0) dt = fmin(dt, cfg->eta_g / sqrt(gmax));
    return dt;
}

void or_floors(const sr_config* cfg, double* planes, int64_t w, int64_t h) {
    /* floors.rs:124-196: Σ_vac and Σ_floor as the f32 the planes hold; vacuum reset, then the thermal floor */
    int64_t n = w * h;
    double svac = (double)(float)cfg->sigma_vac, sfloor = (double)(float)cfg->sigma_floor;
    double eps_floor = cfg->t_floor / cfg->mu / (cfg->gamma - 1.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        double s = planes[i];
        if (s < svac) {
            planes[i] = sfloor;
            planes[n + i] = 0.0;
            planes[2 * n + i] = 0.0;
            planes[3 * n + i] = sfloor * eps_floor;
            continue;
        }
        double mx = planes[n + i], my = planes[2 * n + i], e = planes[3 * n + i];
        double kinetic = 0.5 * (mx * mx + my * my) / (s * s);
        double raw = e / s - kinetic;
        if (raw < eps_floor) planes[3 * n + i] = e + s * (eps_floor - raw);
    }
}

/* ======================================================================= Heat / FLD (reference/heat.rs) */

double or_lambda(double r) { return (2.0 + r) / (6.0 + 3.0 * r + r * r); } /* heat.rs:132-134 */

typedef struct { int gas; double t, s, kappa, inv_c; } side; /* heat.rs:136-154; C = Σ inv_c, inv_c = 1/(μ(γ-1)) */

/* Reference mode's sides, per cell: T⁰ (T_floor off the gas), κ and 1/μ from the cell's species (heat.rs:215-226) */
typedef struct {
    const double *t, *kappa, *inv_mu;
} ref_sides;

typedef struct {
    const sr_config* cfg;
    const ref_sides* rs;
    double gm1, mu, t_floor, sigma_vac, sigma_floor, a_r, c_sb, k_cond, chi;
    int limiter_on;
    int64_t w, h;
    uint8_t* gas;
    double *c, *kx, *ky, vac;
} net;

/* C = Σ/(μ(γ-1)); reference mode: Σ/μ of the side's own species */
static double cap_of(const net* N, const side* s) { return N->rs ? s->s * s->inv_c : s->s / (N->mu * N->gm1); }

static side side_of(const net* N, const double* planes, const double* kappa, int64_t i) {
    /* heat.rs:215-226: the floor state below Σ_vac, else T from the thermal energy (floored) */
    int64_t n = N->w * N->h;
    double s = planes[i];
    side o;
    if (N->rs) {
        o.gas = s >= N->sigma_vac;
        o.t = N->rs->t[i];
        o.s = o.gas ? s : N->sigma_floor;
        o.kappa = N->rs->kappa[i];
        o.inv_c = N->rs->inv_mu[i];
        return o;
    }
    double k = kappa ? kappa[i] : N->cfg->kappa0;
    o.inv_c = 1.0 / (N->mu * N->gm1);
    if (s < N->sigma_vac) {
        o.gas = 0;
        o.t = N->t_floor;
        o.s = N->sigma_floor;
        o.kappa = k;
        return o;
    }
    double mx = planes[n + i], my = planes[2 * n + i], e = planes[3 * n + i];
    double kinetic = 0.5 * (mx * mx + my * my) / (s * s);
    double raw = e / s - kinetic;
    double floor = N->t_floor / N->mu / N->gm1;
    double eps = raw < floor ? floor : raw;
    o.gas = 1;
    o.t = N->mu * N->gm1 * eps;
    o.s = s;
    o.kappa = k;
    return o;
}

static side vacuum_beyond(const net* N, const side* g) { /* heat.rs:234-237: the gas side's κ and μ */
    side o = {0, N->t_floor, N->sigma_floor, g->kappa, g->inv_c};
    return o;
}

static double u_of(const net* N, double t) { return N->chi > 0.0 ? t : N->a_r * ((t * t) * (t * t)); }
static double t_of(const net* N, double u) { return N->chi > 0.0 ? u : sqrt(sqrt(u / N->a_r)); }
static double dt_du(const net* N, double t) { return N->chi > 0.0 ? 1.0 : 1.0 / (4.0 * N->a_r * ((t * t) * t)); }

static double diffusivity(const net* N, const side* a, const side* b) {
    /* heat.rs:263-279 */
    if (!a->gas && !b->gas) return 0.0;
    if (N->chi > 0.0) return N->chi * (0.5 * (cap_of(N, a) + cap_of(N, b)));
    double ta2 = a->t * a->t, tb2 = b->t * b->t;
    double era = N->a_r * (ta2 * ta2), erb = N->a_r * (tb2 * tb2);
    double face_er = 0.5 * (era + erb);
    double ks = 0.5 * (a->kappa * a->s + b->kappa * b->s);
    double r = face_er > 0.0 ? fabs(erb - era) / (ks * face_er) : 0.0;
    double lam = N->limiter_on ? or_lambda(r) : 1.0 / 3.0;
    double radiative = N->c_sb * lam / ks;
    double conduction = N->k_cond != 0.0 ? N->k_cond / (N->a_r * (a->t + b->t) * (a->t * a->t + b->t * b->t)) : 0.0;
    return radiative + conduction;
}

static double face_coef(const net* N, const side* a, const side* b) {
    /* heat.rs:285-294: the far side of a gas cell's vacuum or edge face is the vacuum state */
    side A, B;
    if (a && b) {
        if (a->gas || b->gas) {
            A = a->gas ? *a : vacuum_beyond(N, b);
            B = b->gas ? *b : vacuum_beyond(N, a);
        } else {
            A = *a;
            B = *a;
        }
    } else if (a) {
        A = *a;
        B = vacuum_beyond(N, a);
    } else {
        A = vacuum_beyond(N, b);
        B = *b;
    }
    return diffusivity(N, &A, &B);
}

static void net_build(net* N, const sr_config* cfg, const double* planes, const double* kappa, int64_t w, int64_t h,
                      side** sides_out, const ref_sides* rs) {
    N->cfg = cfg;
    N->rs = rs;
    N->gm1 = cfg->gamma - 1.0;
    N->mu = cfg->mu;
    N->t_floor = cfg->t_floor;
    N->sigma_vac = cfg->sigma_vac;
    N->sigma_floor = cfg->sigma_floor;
    N->a_r = cfg->a_r;
    N->c_sb = cfg->c_sb;
    N->k_cond = cfg->k_cond;
    N->chi = cfg->chi;
    N->limiter_on = cfg->flux_limiter != 0;
    N->w = w;
    N->h = h;
    int64_t n = w * h;
    side* sides = (side*)malloc(sizeof(side) * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) sides[i] = side_of(N, planes, kappa, i);
    N->gas = (uint8_t*)malloc((size_t)n);
    N->c = (double*)malloc(sizeof(double) * (size_t)n);
    N->kx = (double*)malloc(sizeof(double) * (size_t)((w + 1) * h));
    N->ky = (double*)malloc(sizeof(double) * (size_t)(w * (h + 1)));
    for (int64_t i = 0; i < n; i++) {
        N->gas[i] = (uint8_t)sides[i].gas;
        N->c[i] = cap_of(N, &sides[i]);
    }
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x <= w; x++)
            N->kx[y * (w + 1) + x] = face_coef(N, x > 0 ? &sides[y * w + x - 1] : NULL, x < w ? &sides[y * w + x] : NULL);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y <= h; y++)
        for (int64_t x = 0; x < w; x++)
            N->ky[y * w + x] = face_coef(N, y > 0 ? &sides[(y - 1) * w + x] : NULL, y < h ? &sides[y * w + x] : NULL);
    N->vac = u_of(N, cfg->t_floor);
    *sides_out = sides;
}

static void net_free(net* N) {
    free(N->gas);
    free(N->c);
    free(N->kx);
    free(N->ky);
}

static void net_flux(const net* N, const double* v, double* fx, double* fy) {
    /* heat.rs:338-361 */
    int64_t w = N->w, h = N->h;
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x <= w; x++) {
            double k = N->kx[y * (w + 1) + x];
            double va = (x > 0 && N->gas[y * w + x - 1]) ? v[y * w + x - 1] : N->vac;
            double vb = (x < w && N->gas[y * w + x]) ? v[y * w + x] : N->vac;
            fx[y * (w + 1) + x] = k == 0.0 ? 0.0 : -k * (vb - va);
        }
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y <= h; y++)
        for (int64_t x = 0; x < w; x++) {
            double k = N->ky[y * w + x];
            double va = (y > 0 && N->gas[(y - 1) * w + x]) ? v[(y - 1) * w + x] : N->vac;
            double vb = (y < h && N->gas[y * w + x]) ? v[y * w + x] : N->vac;
            fy[y * w + x] = k == 0.0 ? 0.0 : -k * (vb - va);
        }
}

static void k_sums(const net* N, int64_t i, double* ksum, double* kvac) {
    /* heat.rs:363-371: Σ_f k over the four faces, and over the vacuum/edge ones */
    int64_t w = N->w, h = N->h, x = i % w, y = i / w;
    double k[4] = {N->kx[y * (w + 1) + x], N->kx[y * (w + 1) + x + 1], N->ky[y * w + x], N->ky[(y + 1) * w + x]};
    int64_t nb[4] = {x > 0 ? i - 1 : -1, x + 1 < w ? i + 1 : -1, y > 0 ? i - w : -1, y + 1 < h ? i + w : -1};
    double s = 0.0, v = 0.0;
    for (int f = 0; f < 4; f++) {
        s += k[f];
        if (!(nb[f] >= 0 && N->gas[nb[f]])) v += k[f];
    }
    *ksum = s;
    *kvac = v;
}

void or_heat_matvec(int64_t w, int64_t h, const double* diag, const double* kx, const double* ky,
                    const uint8_t* gas, const double* x, double* y) {
    /* heat.rs:373-392 */
#pragma omp parallel for schedule(static)
    for (int64_t yy = 0; yy < h; yy++)
        for (int64_t xx = 0; xx < w; xx++) {
            int64_t i = yy * w + xx;
            if (!gas[i]) { y[i] = 0.0; continue; }
            double s = diag[i] * x[i];
            if (xx > 0 && gas[i - 1]) s -= kx[yy * (w + 1) + xx] * x[i - 1];
            if (xx + 1 < w && gas[i + 1]) s -= kx[yy * (w + 1) + xx + 1] * x[i + 1];
            if (yy > 0 && gas[i - w]) s -= ky[yy * w + xx] * x[i - w];
            if (yy + 1 < h && gas[i + w]) s -= ky[(yy + 1) * w + xx] * x[i + w];
            y[i] = s;
        }
}

/* Σ_i a_i b_i as row partials added in row order. */
static double dot_rows(int64_t w, int64_t h, const double* a, const double* b) {
    double* part = (double*)malloc(sizeof(double) * (size_t)h);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++) {
        double s = 0.0;
        for (int64_t x = 0; x < w; x++) s += a[y * w + x] * b[y * w + x];
        part[y] = s;
    }
    double t = 0.0;
    for (int64_t y = 0; y < h; y++) t += part[y];
    free(part);
    return t;
}

typedef struct {
    const net* N;
    double *diag, *rhs, *heat, *slope;
    double u_bound, t_bound;
} sys_t;

static int64_t sys_solve(const sys_t* S, double* x, int64_t max_rounds, int* fail) {
    /* heat.rs:413-447: Jacobi-PCG checked before every round, the start included */
    const net* N = S->N;
    int64_t w = N->w, h = N->h, n = w * h;
    double* q = (double*)malloc(sizeof(double) * (size_t)n);
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* eh = (double*)malloc(sizeof(double) * (size_t)n);
    or_heat_matvec(w, h, S->diag, N->kx, N->ky, N->gas, x, q);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        r[i] = N->gas[i] ? S->rhs[i] - q[i] : 0.0;
        z[i] = N->gas[i] ? r[i] / S->diag[i] : 0.0;
        p[i] = z[i];
    }
    double rz = dot_rows(w, h, r, z);
    int64_t rounds = 0;
    *fail = 0;
    for (;;) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) {
            double e = N->gas[i] ? r[i] * S->slope[i] / S->diag[i] : 0.0;
            eh[i] = N->gas[i] ? S->heat[i] * e * e : 0.0;
        }
        double ones_dummy = 0.0;
        (void)ones_dummy;
        double e_heat = 0.0;
        {
            double* part = (double*)malloc(sizeof(double) * (size_t)h);
#pragma omp parallel for schedule(static)
            for (int64_t y = 0; y < h; y++) {
                double s = 0.0;
                for (int64_t xx = 0; xx < w; xx++) s += eh[y * w + xx];
                part[y] = s;
            }
            for (int64_t y = 0; y < h; y++) e_heat += part[y];
            free(part);
        }
        or_heat_matvec(w, h, S->diag, N->kx, N->ky, N->gas, p, q);
        double pq = dot_rows(w, h, p, q);
        if (!(isfinite(rz) && isfinite(e_heat) && isfinite(pq))) { *fail = 1; break; }
        if ((rz <= S->u_bound && e_heat <= S->t_bound) || rounds == max_rounds) break;
        double alpha = rz / pq;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            z[i] = N->gas[i] ? r[i] / S->diag[i] : 0.0;
        }
        double rz_next = dot_rows(w, h, r, z);
        double beta = rz_next / rz;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_next;
        rounds++;
    }
    free(q); free(r); free(z); free(p); free(eh);
    return rounds;
}

static void commit_limited(const net* N, double* planes, const double* u, const double* t0, double dt,
                           or_heat_report* rep, double* fxo, double* fyo) {
    /* heat.rs:545-592: F at the last iterate, each gas cell's outflow scaled to the heat it holds above its floor */
    int64_t w = N->w, h = N->h, n = w * h;
    double* fx = (double*)malloc(sizeof(double) * (size_t)((w + 1) * h));
    double* fy = (double*)malloc(sizeof(double) * (size_t)(w * (h + 1)));
    net_flux(N, u, fx, fy);
    double* scale = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; i++) {
        if (!N->gas[i]) { scale[i] = 1.0; continue; }
        int64_t x = i % w, y = i / w;
        double lv[4] = {-fx[y * (w + 1) + x], fx[y * (w + 1) + x + 1], -fy[y * w + x], fy[(y + 1) * w + x]};
        double out = 0.0;
        for (int f = 0; f < 4; f++) out += fmax(lv[f], 0.0);
        out *= dt;
        double held = N->c[i] * fmax(t0[i] - N->t_floor, 0.0);
        scale[i] = out > held ? held / out : 1.0;
    }
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x <= w; x++) {
            int64_t k = y * (w + 1) + x;
            int64_t from = fx[k] > 0.0 ? (x > 0 ? y * w + x - 1 : -1) : (x < w ? y * w + x : -1);
            fx[k] *= from >= 0 ? scale[from] : 1.0;
        }
    for (int64_t y = 0; y <= h; y++)
        for (int64_t x = 0; x < w; x++) {
            int64_t k = y * w + x;
            int64_t from = fy[k] > 0.0 ? (y > 0 ? (y - 1) * w + x : -1) : (y < h ? y * w + x : -1);
            fy[k] *= from >= 0 ? scale[from] : 1.0;
        }
    double radiated = 0.0;
    for (int64_t i = 0; i < n; i++) {
        if (!N->gas[i]) continue;
        int64_t x = i % w, y = i / w;
        double out[4] = {-fx[y * (w + 1) + x], fx[y * (w + 1) + x + 1], -fy[y * w + x], fy[(y + 1) * w + x]};
        int64_t nb[4] = {x > 0 ? i - 1 : -1, x + 1 < w ? i + 1 : -1, y > 0 ? i - w : -1, y + 1 < h ? i + w : -1};
        for (int f = 0; f < 4; f++)
            if (!(nb[f] >= 0 && N->gas[nb[f]])) radiated += dt * out[f];
        planes[3 * n + i] -= dt * (((out[0] + out[1]) + out[2]) + out[3]);
    }
    rep->delta = 0.0;
    rep->converged = 0;
    rep->radiated = radiated;
    if (fxo) memcpy(fxo, fx, sizeof(double) * (size_t)((w + 1) * h));
    if (fyo) memcpy(fyo, fy, sizeof(double) * (size_t)(w * (h + 1)));
    free(fx); free(fy); free(scale);
}

static void heat_step_impl(const sr_config* cfg, double* planes, const double* kappa, const ref_sides* rs, int64_t w,
                           int64_t h, double dt, double tol, double newton_heat, double newton_cell, or_heat_report* rep,
                           double* fxo, double* fyo);

void or_heat_step(const sr_config* cfg, double* planes, const double* kappa, int64_t w, int64_t h, double dt,
                  double tol, double newton_heat, double newton_cell, or_heat_report* rep, double* fxo, double* fyo) {
    heat_step_impl(cfg, planes, kappa, NULL, w, h, dt, tol, newton_heat, newton_cell, rep, fxo, fyo);
}

void or_heat_step_sides(const sr_config* cfg, double* planes, int64_t w, int64_t h, double dt, double tol,
                        double newton_heat, double newton_cell, const double* t0, const double* kappa,
                        const double* inv_mu, or_heat_report* rep, double* fxo, double* fyo) {
    ref_sides rs = {t0, kappa, inv_mu};
    heat_step_impl(cfg, planes, NULL, &rs, w, h, dt, tol, newton_heat, newton_cell, rep, fxo, fyo);
}

static void heat_step_impl(const sr_config* cfg, double* planes, const double* kappa, const ref_sides* rs, int64_t w,
                           int64_t h, double dt, double tol, double newton_heat, double newton_cell, or_heat_report* rep,
                           double* fxo, double* fyo) {
    /* heat.rs:453-536 */
    int64_t n = w * h;
    net N;
    side* sides;
    net_build(&N, cfg, planes, kappa, w, h, &sides, rs);
    double* t0 = (double*)malloc(sizeof(double) * (size_t)n);
    double* u0 = (double*)malloc(sizeof(double) * (size_t)n);
    int64_t ngas = 0;
    for (int64_t i = 0; i < n; i++) {
        t0[i] = sides[i].t;
        u0[i] = u_of(&N, t0[i]);
        ngas += N.gas[i];
    }
    free(sides);
    or_heat_report R = {0, 0, 0.0, 1, 0, 0.0};
    if (cfg->pin_temperature || ngas == 0 || isnan(dt) || dt <= 0.0) {
        if (fxo || fyo) {
            double* fx = (double*)malloc(sizeof(double) * (size_t)((w + 1) * h));
            double* fy = (double*)malloc(sizeof(double) * (size_t)(w * (h + 1)));
            net_flux(&N, u0, fx, fy);
            if (fxo) memcpy(fxo, fx, sizeof(double) * (size_t)((w + 1) * h));
            if (fyo) memcpy(fyo, fy, sizeof(double) * (size_t)(w * (h + 1)));
            free(fx); free(fy);
        }
        if (rep) *rep = R;
        free(t0); free(u0); net_free(&N);
        return;
    }
    double u_vac = N.vac;
    double heat0 = 0.0;
    for (int64_t i = 0; i < n; i++)
        if (N.gas[i]) heat0 += N.c[i] * t0[i];
    double* ksum = (double*)calloc((size_t)n, sizeof(double));
    double* kvac = (double*)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < n; i++)
        if (N.gas[i]) k_sums(&N, i, &ksum[i], &kvac[i]);
    double* t = (double*)malloc(sizeof(double) * (size_t)n);
    double* u = (double*)malloc(sizeof(double) * (size_t)n);
    memcpy(t, t0, sizeof(double) * (size_t)n);
    memcpy(u, u0, sizeof(double) * (size_t)n);
    sys_t S;
    S.N = &N;
    S.diag = (double*)malloc(sizeof(double) * (size_t)n);
    S.rhs = (double*)malloc(sizeof(double) * (size_t)n);
    S.heat = (double*)malloc(sizeof(double) * (size_t)n);
    S.slope = (double*)malloc(sizeof(double) * (size_t)n);
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    double* ub = (double*)malloc(sizeof(double) * (size_t)n);
    double* tb = (double*)malloc(sizeof(double) * (size_t)n);
    int64_t passes = 0, rounds = 0;
    int converged = 0;
    int64_t max_passes = cfg->max_passes ? cfg->max_passes : 128, max_rounds = cfg->max_rounds ? cfg->max_rounds : 4096;
    while (passes < max_passes && rounds < max_rounds) {
        passes++;
        for (int64_t i = 0; i < n; i++) {
            S.heat[i] = N.gas[i] ? N.c[i] / dt : 0.0;
            S.slope[i] = N.gas[i] ? dt_du(&N, t[i]) : 0.0;
            double ci = S.heat[i] * S.slope[i];
            S.diag[i] = N.gas[i] ? ci + ksum[i] : 1.0;
            S.rhs[i] = N.gas[i] ? ci * u[i] - S.heat[i] * (t[i] - t0[i]) + kvac[i] * u_vac : 0.0;
            ub[i] = N.gas[i] ? ci * u[i] * u[i] : 0.0;
            tb[i] = N.gas[i] ? S.heat[i] * t[i] * t[i] : 0.0;
            x[i] = N.gas[i] ? u[i] : 0.0;
        }
        double su = 0.0, st = 0.0;
        for (int64_t i = 0; i < n; i++) { su += ub[i]; st += tb[i]; }
        S.u_bound = tol * tol * su;
        S.t_bound = tol * tol * st;
        if (!(isfinite(S.u_bound) && isfinite(S.t_bound))) { passes--; break; }
        int fail = 0;
        rounds += sys_solve(&S, x, max_rounds - rounds, &fail);
        if (fail) break;
        double moved = 0.0;
        int every = 1;
        for (int64_t i = 0; i < n; i++) {
            if (!N.gas[i]) continue;
            double nx = t_of(&N, fmax(x[i], u_vac));
            double lo = 0.5 * t[i], hi = 2.0 * t[i];
            nx = nx < lo ? lo : (nx > hi ? hi : nx);
            double d = fabs(nx - t[i]);
            moved += N.c[i] * d;
            every &= d <= newton_cell * t[i];
            t[i] = nx;
            u[i] = u_of(&N, nx);
        }
        if (moved <= newton_heat * heat0 && every) { converged = 1; break; }
    }
    R.passes = passes;
    R.rounds = rounds;
    if (!converged) {
        commit_limited(&N, planes, u, t0, dt, &R, fxo, fyo);
    } else {
        double* fx = (double*)malloc(sizeof(double) * (size_t)((w + 1) * h));
        double* fy = (double*)malloc(sizeof(double) * (size_t)(w * (h + 1)));
        net_flux(&N, u, fx, fy);
        double radiated = 0.0, gained = 0.0, held = 0.0;
        for (int64_t i = 0; i < n; i++) {
            if (!N.gas[i]) continue;
            radiated += dt * kvac[i] * (u[i] - u_vac);
            gained += N.c[i] * (t[i] - t0[i]);
            held += N.c[i] * t[i];
        }
        double delta = -(gained + radiated) / held;
        for (int64_t i = 0; i < n; i++)
            if (N.gas[i]) planes[3 * n + i] += N.c[i] * ((1.0 + delta) * t[i] - t0[i]);
        R.delta = delta;
        R.converged = 1;
        R.radiated = radiated;
        if (fxo) memcpy(fxo, fx, sizeof(double) * (size_t)((w + 1) * h));
        if (fyo) memcpy(fyo, fy, sizeof(double) * (size_t)(w * (h + 1)));
        free(fx); free(fy);
    }
    if (rep) *rep = R;
    free(S.diag); free(S.rhs); free(S.heat); free(S.slope);
    free(x); free(ub); free(tb); free(t); free(u); free(t0); free(u0); free(ksum); free(kvac);
    net_free(&N);
}

void or_heat_law(const sr_config* cfg, const double* planes, const double* kappa, int64_t w, int64_t h, double* fx,
                 double* fy) {
    /* heat.rs:303-309 */
    net N;
    side* sides;
    net_build(&N, cfg, planes, kappa, w, h, &sides, NULL);
    int64_t n = w * h;
    double* u = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; i++) u[i] = u_of(&N, sides[i].t);
    net_flux(&N, u, fx, fy);
    free(u);
    free(sides);
    net_free(&N);
}

void or_heat_system(const sr_config* cfg, const double* planes, const double* kappa, int64_t w, int64_t h,
                    double dt, double* diag, double* rhs, double* kx, double* ky, uint8_t* gas) {
    /* heat.rs:476-489 at the first iterate (t = T⁰, u = u⁰) */
    net N;
    side* sides;
    net_build(&N, cfg, planes, kappa, w, h, &sides, NULL);
    int64_t n = w * h;
    for (int64_t i = 0; i < n; i++) {
        gas[i] = N.gas[i];
        if (!N.gas[i]) { diag[i] = 1.0; rhs[i] = 0.0; continue; }
        double ks, kv;
        k_sums(&N, i, &ks, &kv);
        double t = sides[i].t;
        double ci = N.c[i] / dt * dt_du(&N, t);
        diag[i] = ci + ks;
        rhs[i] = ci * u_of(&N, t) + kv * N.vac;
    }
    memcpy(kx, N.kx, sizeof(double) * (size_t)((w + 1) * h));
    memcpy(ky, N.ky, sizeof(double) * (size_t)(w * (h + 1)));
    free(sides);
    net_free(&N);
}

int64_t or_heat_pcg(int64_t w, int64_t h, const double* diag, const double* rhs, const double* kx, const double* ky,
                    const uint8_t* gas, double rel, int64_t max_rounds, double* x) {
    /* Jacobi-PCG to a relative residual (the reference's System::solve with the FP64 residual as its measure) */
    int64_t n = w * h;
    double* q = (double*)malloc(sizeof(double) * (size_t)n);
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    or_heat_matvec(w, h, diag, kx, ky, gas, x, q);
    for (int64_t i = 0; i < n; i++) {
        r[i] = gas[i] ? rhs[i] - q[i] : 0.0;
        z[i] = gas[i] ? r[i] / diag[i] : 0.0;
        p[i] = z[i];
    }
    double bb = dot_rows(w, h, rhs, rhs);
    double rz = dot_rows(w, h, r, z);
    int64_t rounds = 0;
    for (;;) {
        double rr = dot_rows(w, h, r, r);
        if (rr <= rel * rel * bb || rounds >= max_rounds) break;
        or_heat_matvec(w, h, diag, kx, ky, gas, p, q);
        double pq = dot_rows(w, h, p, q);
        if (!isfinite(pq) || pq <= 0.0) { rounds = -1; break; }
        double alpha = rz / pq;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            z[i] = gas[i] ? r[i] / diag[i] : 0.0;
        }
        double rz2 = dot_rows(w, h, r, z);
        double beta = rz2 / rz;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz2;
        rounds++;
    }
    free(q); free(r); free(z); free(p);
    return rounds;
}

/* ======================================================================= Exact Riemann (reference/riemann.rs) */

static void side_fn(double gamma, double p, double rk, double pk, double* f, double* df) {
    /* riemann.rs:72-85 (Toro's f_K) */
    double c = sqrt(gamma * pk / rk);
    if (p > pk) {
        double a = 2.0 / ((gamma + 1.0) * rk);
        double b = (gamma - 1.0) / (gamma + 1.0) * pk;
        double q = sqrt(a / (p + b));
        *f = (p - pk) * q;
        *df = q * (1.0 - (p - pk) / (2.0 * (b + p)));
    } else {
        double e = (gamma - 1.0) / (2.0 * gamma);
        double ratio = p / pk;
        *f = 2.0 * c / (gamma - 1.0) * (pow(ratio, e) - 1.0);
        *df = pow(ratio, -(gamma + 1.0) / (2.0 * gamma)) / (rk * c);
    }
}

int or_riemann_solve(double g, double rl, double ul, double pl, double rr, double ur, double pr, double* sol) {
    /* riemann.rs:88-165 */
    double st[6] = {rl, ul, pl, rr, ur, pr};
    for (int s = 0; s < 2; s++) {
        double rho = st[3 * s], u = st[3 * s + 1], p = st[3 * s + 2];
        if (!(isfinite(rho) && rho > 0.0 && isfinite(p) && p > 0.0 && isfinite(u))) return 1;
    }
    double du = ur - ul, f1, d1, f2, d2;
#define TOTAL(pp) (side_fn(g, (pp), rl, pl, &f1, &d1), side_fn(g, (pp), rr, pr, &f2, &d2), f1 + f2 + du)
    if (TOTAL(0.0) >= 0.0) return 2;
    double lo = 0.0, hi = 0.5 * (pl + pr);
    while (TOTAL(hi) < 0.0) {
        lo = hi;
        hi *= 2.0;
        if (!isfinite(hi)) return 3;
    }
    double p = 0.5 * (lo + hi), pstar = -1.0;
    for (int it = 0; it < 200; it++) {
        double f = TOTAL(p);
        if (f < 0.0) lo = p; else hi = p;
        double newton = p - f / (d1 + d2);
        double next = (newton > lo && newton < hi) ? newton : 0.5 * (lo + hi);
        if (fabs(next - p) <= 1e-15 * next) { pstar = next; break; }
        p = next;
    }
#undef TOTAL
    if (pstar < 0.0) return 3;
    double fl_, fr_, dd;
    side_fn(g, pstar, rr, pr, &fr_, &dd);
    side_fn(g, pstar, rl, pl, &fl_, &dd);
    double ustar = 0.5 * (ul + ur) + 0.5 * (fr_ - fl_);
    double mu = (g - 1.0) / (g + 1.0), e = (g - 1.0) / (2.0 * g);
    double cl = sqrt(g * pl / rl), cr = sqrt(g * pr / rr);
    sol[0] = pstar;
    sol[1] = ustar;
    if (pstar > pl) {
        sol[4] = 0.0;
        sol[5] = ul - cl * sqrt((g + 1.0) / (2.0 * g) * pstar / pl + e);
        sol[6] = sol[5];
        sol[2] = rl * ((pstar / pl + mu) / (mu * pstar / pl + 1.0));
    } else {
        double cs = cl * pow(pstar / pl, e);
        sol[4] = 1.0;
        sol[5] = ul - cl;
        sol[6] = ustar - cs;
        sol[2] = rl * pow(pstar / pl, 1.0 / g);
    }
    if (pstar > pr) {
        sol[7] = 0.0;
        sol[8] = ur + cr * sqrt((g + 1.0) / (2.0 * g) * pstar / pr + e);
        sol[9] = sol[8];
        sol[3] = rr * ((pstar / pr + mu) / (mu * pstar / pr + 1.0));
    } else {
        double cs = cr * pow(pstar / pr, e);
        sol[7] = 1.0;
        sol[8] = ur + cr;
        sol[9] = ustar + cs;
        sol[3] = rr * pow(pstar / pr, 1.0 / g);
    }
    return 0;
}

void or_riemann_sample(double g, double rl, double ul, double pl, double rr, double ur, double pr, const double* sol,
                       double xi, double* out) {
    /* riemann.rs:168-210 */
    double ps = sol[0], us = sol[1];
    if (xi <= us) {
        double c = sqrt(g * pl / rl);
        if (sol[4] == 0.0) {
            if (xi <= sol[5]) { out[0] = rl; out[1] = ul; out[2] = pl; }
            else { out[0] = sol[2]; out[1] = us; out[2] = ps; }
        } else {
            double head = sol[5], tail = sol[6];
            if (xi <= head) { out[0] = rl; out[1] = ul; out[2] = pl; }
            else if (xi > tail) { out[0] = sol[2]; out[1] = us; out[2] = ps; }
            else {
                double u = 2.0 / (g + 1.0) * (c + (g - 1.0) / 2.0 * ul + xi);
                double a = 2.0 / (g + 1.0) * (c + (g - 1.0) / 2.0 * (ul - xi));
                out[0] = rl * pow(a / c, 2.0 / (g - 1.0));
                out[1] = u;
                out[2] = pl * pow(a / c, 2.0 * g / (g - 1.0));
            }
        }
    } else {
        double c = sqrt(g * pr / rr);
        if (sol[7] == 0.0) {
            if (xi >= sol[8]) { out[0] = rr; out[1] = ur; out[2] = pr; }
            else { out[0] = sol[3]; out[1] = us; out[2] = ps; }
        } else {
            double head = sol[8], tail = sol[9];
            if (xi >= head) { out[0] = rr; out[1] = ur; out[2] = pr; }
            else if (xi < tail) { out[0] = sol[3]; out[1] = us; out[2] = ps; }
            else {
                double u = 2.0 / (g + 1.0) * (-c + (g - 1.0) / 2.0 * ur + xi);
                double a = 2.0 / (g + 1.0) * (c - (g - 1.0) / 2.0 * (ur - xi));
                out[0] = rr * pow(a / c, 2.0 / (g - 1.0));
                out[1] = u;
                out[2] = pr * pow(a / c, 2.0 * g / (g - 1.0));
            }
        }
    }
}

/* ======================================================================= Twin (reference/mod.rs) */

struct or_twin {
    sr_config cfg;
    int64_t w, h;
    double* planes;
    double* kappa;
    double *phi, *gx, *gy;
    int has_field;
    double dt, dt_next, sim_time;
    int64_t steps;
    or_heat_report heat;
    double *hfx, *hfy;
};

static void twin_gravity(or_twin* t) {
    if (!t->cfg.gravity) return;
    or_grav_field(&t->cfg, t->planes, t->w, t->h, t->phi, t->gx, t->gy);
    t->has_field = 1;
}

static double twin_reduce_dt(or_twin* t) {
    double d = or_hydro_dt(&t->cfg, t->planes, t->w, t->h, t->has_field ? t->gx : NULL, t->has_field ? t->gy : NULL);
    if (t->cfg.dt_fixed > 0.0) d = t->cfg.dt_fixed;
    if (t->cfg.dt_cap > 0.0) d = fmin(d, t->cfg.dt_cap);
    return d;
}

or_twin* or_twin_new(const sr_config* cfg, const double* planes, const double* kappa) {
    /* mod.rs:129-177: the state, P2 on it and Δt_0 reduced from it (the hold has nothing to hold without cold EOS) */
    or_twin* t = (or_twin*)calloc(1, sizeof(or_twin));
    t->cfg = *cfg;
    t->w = cfg->width;
    t->h = cfg->height;
    int64_t n = t->w * t->h;
    t->planes = (double*)malloc(sizeof(double) * 4 * (size_t)n);
    memcpy(t->planes, planes, sizeof(double) * 4 * (size_t)n);
    if (kappa && cfg->opacity_plane) {
        t->kappa = (double*)malloc(sizeof(double) * (size_t)n);
        memcpy(t->kappa, kappa, sizeof(double) * (size_t)n);
    }
    t->phi = (double*)calloc((size_t)n, sizeof(double));
    t->gx = (double*)calloc((size_t)n, sizeof(double));
    t->gy = (double*)calloc((size_t)n, sizeof(double));
    t->hfx = (double*)calloc((size_t)((t->w + 1) * t->h), sizeof(double));
    t->hfy = (double*)calloc((size_t)(t->w * (t->h + 1)), sizeof(double));
    twin_gravity(t);
    t->dt_next = twin_reduce_dt(t);
    return t;
}

void or_twin_free(or_twin* t) {
    if (!t) return;
    free(t->planes); free(t->kappa); free(t->phi); free(t->gx); free(t->gy); free(t->hfx); free(t->hfy);
    free(t);
}

void or_twin_step(or_twin* t) {
    /* mod.rs:264-297: P1 → P2 → P4 → P5 → P8 → P9 */
    double dt = t->dt_next;
    t->dt = dt;
    t->sim_time += dt;
    twin_gravity(t);
    if (t->cfg.hydro) {
        or_hydro_report rep;
        or_hydro_step(&t->cfg, t->planes, t->w, t->h, dt, t->has_field ? t->gx : NULL, t->has_field ? t->gy : NULL,
                      &rep);
    }
    if (t->cfg.heat) {
        /* the twin's own tolerances (heat.rs:53-55): SOLVE_TOL 1e-12, NEWTON_HEAT 1e-12, NEWTON_CELL 1e-10 */
        or_heat_step(&t->cfg, t->planes, t->kappa, t->w, t->h, dt, 1e-12, 1e-12, 1e-10, &t->heat, t->hfx, t->hfy);
    }
    or_floors(&t->cfg, t->planes, t->w, t->h);
    t->dt_next = twin_reduce_dt(t);
    t->steps++;
}

void or_twin_state(const or_twin* t, double* planes) {
    memcpy(planes, t->planes, sizeof(double) * 4 * (size_t)(t->w * t->h));
}

void or_twin_clock(const or_twin* t, double* out4) {
    out4[0] = t->dt;
    out4[1] = t->dt_next;
    out4[2] = t->sim_time;
    out4[3] = (double)t->steps;
}

void or_twin_field(const or_twin* t, double* phi, double* gx, double* gy) {
    size_t n = (size_t)(t->w * t->h);
    memcpy(phi, t->phi, n * sizeof(double));
    memcpy(gx, t->gx, n * sizeof(double));
    memcpy(gy, t->gy, n * sizeof(double));
}

void or_twin_heat(const or_twin* t, or_heat_report* rep, double* fx, double* fy) {
    if (rep) *rep = t->heat;
    if (fx) memcpy(fx, t->hfx, sizeof(double) * (size_t)((t->w + 1) * t->h));
    if (fy) memcpy(fy, t->hfy, sizeof(double) * (size_t)(t->w * (t->h + 1)));
}
