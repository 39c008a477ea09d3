// hydro_ref.cu — reference mode (14 channels): the reference twin's own P4 (crates/sr-physics/src/reference/hydro.rs,
// step_held), P8 (reference/floors.rs) and P9's Δt terms, in FP32 on the device.
//
// The EOS is the reference's (crates/sr-physics/src/eos.rs): γ = 2 (Π_th = Σ ε_th, c² = 2Π/Σ), μ and Y_e of each
// cell's ten mass fractions (registry.rs:145-154), the cold pressures of the electrons' and neutron matter's K pairs and
// their energies read from the 512-node u(x) tables. The tables live on the device as each node's u and the step of
// ln u to the next node, so a lookup is one logarithm (the node and its fraction) and u_i · exp(frac · Δ ln u): the
// exponential's argument stays below one node's step and adds no more than an ulp to the node's own value.
//
// P4 is one tile kernel run twice a step with gravity (the half step's source, then the update) and once without. A CTA
// owns a 16 x 16 tile: it reads the primitives of the tile and a 2-cell ring (ghosts by the edge mode) into shared
// memory, predicts the four face states of every tile cell and the one face of each ring cell that faces the tile
// (the Hancock half step of the cell's own four fluxes, the half kick of g), and each tile cell then takes the HLL
// fluxes of its four faces from those states — the held walls and the edge's walls where they apply — and updates.
// Gravity's net kick and the radiation force's net push are taken back, and the sticky wall applied, by a pass over the
// updated state after one CTA has reduced the per-CTA partials.
#include <limits.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "hydro_ref.cuh"

namespace {

constexpr int RT = 16;            // tile side
constexpr int RP = RT + 4;        // the primitives' region: the tile and a 2-cell ring
constexpr int RQ = RT + 2;        // the 1-cell ring's region (mids, φ_mid)
constexpr int RNT = RT * RT;      // threads: one per tile cell
constexpr int NS = kRefSpecies;
constexpr int NC = kRefChannels;
constexpr int FV = 5 + NS;        // a face state: Σ, Σu, Σv, E, Π and the ten fractions
constexpr double kXMin = 1e-8, kXMax = 1e8;  // eos.rs:17-18

// registry.rs:45-153 (elements.json, id order H He C O Ne Mg Si S Fe n): (Z+1)/A and Z/A
__constant__ float c_inv_mu[NS] = {2.0f, 0.75f, 7.0f / 12.0f, 9.0f / 16.0f, 11.0f / 20.0f, 13.0f / 24.0f,
                                   15.0f / 28.0f, 17.0f / 32.0f, 27.0f / 56.0f, 1.0f};
__constant__ float c_y_e[NS] = {1.0f, 0.5f, 0.5f, 0.5f, 0.5f, 0.5f, 0.5f, 0.5f, 26.0f / 56.0f, 0.0f};

struct RPrim {
    float s, u, v, p;
    float x[NS];
};

struct RShared {
    float tab[4][kColdPoints];
    float P[NC][RP * RP];       // primitives of the tile and its 2-cell ring
    float TF[FV][4][RNT];       // the tile cells' predicted faces [x-, x+, y-, y+]
    float RF[FV][4 * RT];       // the ring cells' faces toward the tile: left col x+, right col x-, top y+, bottom y-
    float MID[3][RQ * RQ];      // the cells' half-step Σ, Σu, Σv (tile and 1-ring)
    float PH[RQ * RQ];          // φ_mid (tile and 1-ring)
    uint8_t FL[RP * RP];        // bit 0: Σ < Σ_vac (in the world), bit 1: held
    double red[5][RNT / 32];
    float rbest[RNT / 32];
    int ridx[RNT / 32];
};

// ---------------------------------------------------------------------------------------------- the EOS (eos.rs)
__device__ __forceinline__ float cold_p(float x, float k1, float k1_k2) {
    // eos.rs:22-29: 1/(1/(K₁x²) + 1/(K₂x^{3/2})) = K₁x² / (1 + (K₁/K₂)√x); 0 for x <= 0
    return x > 0.0f ? k1 * x * x / (1.0f + k1_k2 * sqrtf(x)) : 0.0f;
}

__device__ __forceinline__ float cold_u(const float* u, const float* d, float x) {
    // eos.rs:118-131: log-log interpolation; K₁x² (u at the first node × (x/X_MIN)²) below the table
    if (!(x > 0.0f)) return 0.0f;
    const float ln_min = -18.420680743952367f;                      // ln 1e-8
    const float inv_step = 511.0f / 36.841361487904734f;            // (TABLE_POINTS - 1) / (ln X_MAX - ln X_MIN)
    const float pos = (logf(x) - ln_min) * inv_step;
    if (pos < 0.0f) {
        const float r = x * 1e8f;
        return u[0] * r * r;
    }
    int i = (int)pos;
    i = i > kColdPoints - 2 ? kColdPoints - 2 : i;
    return u[i] * expf((pos - (float)i) * d[i]);
}

struct Eos {
    const RefConst& R;
    const float* tab;  // shared copy
    __device__ float pi_cold(float s, float ye, float xn) const {
        float p = 0.0f;
        if (R.cold_e) p += cold_p(ye * s, R.k1e, R.k1e_k2e);
        if (R.cold_n) p += cold_p(xn * s, R.k1n, R.k1n_k2n);
        return p;
    }
    __device__ float eps_cold(float s, float ye, float xn) const {  // eos.rs:237-242
        float u = 0.0f;
        if (R.cold_e) u += cold_u(tab, tab + kColdPoints, ye * s);
        if (R.cold_n) u += cold_u(tab + 2 * kColdPoints, tab + 3 * kColdPoints, xn * s);
        return sr_div(u, s);
    }
};

__device__ __forceinline__ void composition(const float* x, float& inv_mu, float& ye) {
    inv_mu = 0.0f;
    ye = 0.0f;
#pragma unroll
    for (int k = 0; k < NS; k++) {
        inv_mu = fmaf(x[k], c_inv_mu[k], inv_mu);
        ye = fmaf(x[k], c_y_e[k], ye);
    }
}

// hydro.rs:424-441: a cell as primitives — the floor state below Σ_vac (its fractions kept), else ε_th recovered
// and floored at T_floor/μ.
__device__ RPrim ref_read(const Eos& E, float s, float mx, float my, float en, const float* x) {
    RPrim p;
#pragma unroll
    for (int k = 0; k < NS; k++) p.x[k] = x[k];
    float inv_mu, ye;
    composition(x, inv_mu, ye);
    const float xn = x[NS - 1], floor = E.R.t_floor * inv_mu;
    if (s < E.R.sigma_vac) {
        p.s = E.R.sigma_floor;
        p.u = 0.0f;
        p.v = 0.0f;
        p.p = p.s * floor + E.pi_cold(p.s, ye, xn);
        return p;
    }
    const float rs = sr_div(1.0f, s);
    p.s = s;
    p.u = mx * rs;
    p.v = my * rs;
    float raw = en * rs - 0.5f * (p.u * p.u + p.v * p.v) - E.eps_cold(s, ye, xn);
    const float eps = raw < floor ? floor : raw;
    p.p = s * eps + E.pi_cold(s, ye, xn);
    return p;
}

// hydro.rs:443-460: the conserved vector of primitives
__device__ void ref_cons(const Eos& E, const RPrim& p, float* U) {
    float inv_mu, ye;
    composition(p.x, inv_mu, ye);
    const float xn = p.x[NS - 1];
    const float thermal = sr_div(p.p - E.pi_cold(p.s, ye, xn), p.s);
    const float eps = fmaxf(thermal, E.R.t_floor * inv_mu);
    U[0] = p.s;
    U[1] = p.s * p.u;
    U[2] = p.s * p.v;
    U[3] = p.s * (eps + E.eps_cold(p.s, ye, xn)) + 0.5f * p.s * (p.u * p.u + p.v * p.v);
#pragma unroll
    for (int k = 0; k < NS; k++) U[4 + k] = p.s * p.x[k];
}

// hydro.rs:462-478: the primitives of a conserved vector; false when it is no state
__device__ bool ref_prim(const Eos& E, const float* U, RPrim& out) {
    const float s = U[0];
    if (!(s > 0.0f)) return false;
    bool finite = isfinite(s) && isfinite(U[1]) && isfinite(U[2]) && isfinite(U[3]);
    const float rs = sr_div(1.0f, s);
#pragma unroll
    for (int k = 0; k < NS; k++) {
        finite = finite && isfinite(U[4 + k]);
        out.x[k] = U[4 + k] * rs;
    }
    if (!finite) return false;
    float inv_mu, ye;
    composition(out.x, inv_mu, ye);
    const float xn = out.x[NS - 1];
    const float u = U[1] * rs, v = U[2] * rs;
    const float raw = U[3] * rs - 0.5f * (u * u + v * v) - E.eps_cold(s, ye, xn);
    if (!(raw > 0.0f)) return false;
    const float eps = fmaxf(raw, E.R.t_floor * inv_mu);
    out.s = s;
    out.u = u;
    out.v = v;
    out.p = s * eps + E.pi_cold(s, ye, xn);
    return true;
}

__device__ __forceinline__ float lim_mc(float l, float c, float r) {  // hydro.rs:283-289
    const float a = c - l, b = r - c;
    if (a * b <= 0.0f) return 0.0f;
    return copysignf(fminf(fminf(fabsf(0.5f * (a + b)), 2.0f * fabsf(a)), 2.0f * fabsf(b)), a);
}

__device__ __forceinline__ float lim_minmod(float l, float c, float r) {
    const float a = c - l, b = r - c;
    if (a * b <= 0.0f) return 0.0f;
    return copysignf(fminf(fabsf(a), fabsf(b)), a);
}

__device__ __forceinline__ float lim(int minmod, float l, float c, float r) {
    return minmod ? lim_minmod(l, c, r) : lim_mc(l, c, r);
}

__device__ __forceinline__ float pv(const RShared& S, int ch, int i) { return S.P[ch][i]; }

// hydro.rs:293-331: a cell's slope along one axis from the primitives at region indices l, c, r
__device__ RPrim ref_slope(const RefConst& R, const RShared& S, int l, int c, int r) {
    RPrim s;
    const int mm = R.limiter == SR_LIMITER_MINMOD;
    s.s = lim(mm, pv(S, 0, l), pv(S, 0, c), pv(S, 0, r));
    s.u = lim(mm, pv(S, 1, l), pv(S, 1, c), pv(S, 1, r));
    s.v = lim(mm, pv(S, 2, l), pv(S, 2, c), pv(S, 2, r));
    s.p = lim(mm, pv(S, 3, l), pv(S, 3, c), pv(S, 3, r));
    float theta = 1.0f;
#pragma unroll
    for (int k = 0; k < NS; k++) {
        const float xl = pv(S, 4 + k, l), xc = pv(S, 4 + k, c), xr = pv(S, 4 + k, r);
        const float central = 0.5f * (xr - xl);
        s.x[k] = central;
        if (central != 0.0f) theta = fminf(theta, lim(mm, xl, xc, xr) / central);
    }
#pragma unroll
    for (int k = 0; k < NS; k++) s.x[k] *= theta;
    if (R.bracket) {
        const float sl = pv(S, 0, l), sc = pv(S, 0, c), sr = pv(S, 0, r);
        const float hottest = fmaxf(fmaxf(pv(S, 3, l) / sl, pv(S, 3, c) / sc), pv(S, 3, r) / sr);
        bool hot = false;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const float f = q ? 0.5f : -0.5f;
            const float pif = pv(S, 3, c) + f * s.p, bound = 2.0f * hottest * (sc + f * s.s);
            hot = hot || !(pif <= bound);  // greater, or not a number (HOT_FACE = 2)
        }
        if (hot) {
            s.s = 0.0f;
            s.p = 0.0f;
        }
    }
    return s;
}

__device__ __forceinline__ RPrim offset_of(const RShared& S, int c, const RPrim& sl, float f) {
    RPrim o;
    o.s = pv(S, 0, c) + f * sl.s;
    o.u = pv(S, 1, c) + f * sl.u;
    o.v = pv(S, 2, c) + f * sl.v;
    o.p = pv(S, 3, c) + f * sl.p;
#pragma unroll
    for (int k = 0; k < NS; k++) o.x[k] = pv(S, 4 + k, c) + f * sl.x[k];
    return o;
}

// hydro.rs:485-499: the flux normal to `dir` of primitives whose energy per area is `energy`, added × `scale` to acc
__device__ __forceinline__ void add_flux(const RPrim& p, float energy, int dir, float scale, float* acc) {
    const float un = dir == 0 ? p.u : p.v, ut = dir == 0 ? p.v : p.u;
    const float mass = p.s * un;
    acc[0] += scale * mass;
    acc[1 + dir] += scale * (mass * un + p.p);
    acc[2 - dir] += scale * (mass * ut);
    acc[3] += scale * ((energy + p.p) * un);
#pragma unroll
    for (int k = 0; k < NS; k++) acc[4 + k] += scale * (mass * p.x[k]);
}

// The Hancock increment of the cell at region index c (both axes' flux differences × ½Δt) and its centre's half-step
// (Σ, Σu, Σv); the four face primitives are re-derived from the slopes when evolved.
struct Predict {
    RPrim sx, sy;
    float delta[NC];
    float mid[3];
};

__device__ void predict(const Eos& E, const RShared& S, int c, float half, bool has_g, float gx, float gy, Predict& P) {
    P.sx = ref_slope(E.R, S, c - 1, c, c + 1);
    P.sy = ref_slope(E.R, S, c - RP, c, c + RP);
#pragma unroll
    for (int k = 0; k < NC; k++) P.delta[k] = 0.0f;
#pragma unroll 1
    for (int f = 0; f < 4; f++) {
        const RPrim w = offset_of(S, c, f < 2 ? P.sx : P.sy, (f & 1) ? 0.5f : -0.5f);
        float U[NC];
        ref_cons(E, w, U);
        add_flux(w, U[3], f >> 1, (f & 1) ? -half : half, P.delta);  // ½Δt((F_l - F_r) + (G_l - G_r))
    }
    const float s = pv(S, 0, c);
    P.mid[0] = s + P.delta[0];
    P.mid[1] = s * pv(S, 1, c) + P.delta[1];
    P.mid[2] = s * pv(S, 2, c) + P.delta[2];
    if (has_g) {
        P.mid[1] += half * s * gx;
        P.mid[2] += half * s * gy;
    }
}

// hydro.rs:501-513 with the face's half kick (hydro.rs:600-610): face f of the predicted cell, as FV values at
// dst[v * stride]
__device__ void evolve_face(const Eos& E, const RShared& S, int c, const Predict& P, int f, float half, bool has_g,
                            float gx, float gy, float* dst, int stride) {
    const RPrim w = offset_of(S, c, f < 2 ? P.sx : P.sy, (f & 1) ? 0.5f : -0.5f);
    float U0[NC], U[NC];
    ref_cons(E, w, U0);
#pragma unroll
    for (int k = 0; k < NC; k++) U[k] = U0[k] + P.delta[k];
    if (has_g) {
        U[1] += half * w.s * gx;
        U[2] += half * w.s * gy;
        U[3] += half * w.s * ((w.u + 0.5f * half * gx) * gx + (w.v + 0.5f * half * gy) * gy);
    }
    RPrim p;
    if (ref_prim(E, U, p)) {
        dst[0] = U[0];
        dst[stride] = U[1];
        dst[2 * stride] = U[2];
        dst[3 * stride] = U[3];
        dst[4 * stride] = p.p;
#pragma unroll
        for (int k = 0; k < NS; k++) dst[(5 + k) * stride] = p.x[k];
    } else {
        dst[0] = U0[0];
        dst[stride] = U0[1];
        dst[2 * stride] = U0[2];
        dst[3 * stride] = U0[3];
        dst[4 * stride] = w.p;
#pragma unroll
        for (int k = 0; k < NS; k++) dst[(5 + k) * stride] = w.x[k];
    }
}

// A stored face state.
struct FaceRef {
    const float* base;
    int stride;
    __device__ float at(int v) const { return base[v * stride]; }
};

// hydro.rs:516-540: HLL with Davis speeds, the species by the mass flux's upwind side; `mirror_l`/`mirror_r` read
// that side as its mirror across the face (the normal velocity and momentum negated, hydro.rs:542-554)
__device__ void hll(FaceRef l, FaceRef r, int dir, bool mirror_l, bool mirror_r, float* f) {
    const float sl = l.at(0), sr = r.at(0);
    const float rl = sr_div(1.0f, sl), rr = sr_div(1.0f, sr);
    float Ul[4] = {sl, l.at(1), l.at(2), l.at(3)}, Ur[4] = {sr, r.at(1), r.at(2), r.at(3)};
    if (mirror_l) Ul[1 + dir] = -Ul[1 + dir];
    if (mirror_r) Ur[1 + dir] = -Ur[1 + dir];
    const float ul = Ul[1] * rl, vl = Ul[2] * rl, ur = Ur[1] * rr, vr = Ur[2] * rr;
    const float pl = l.at(4), pr = r.at(4);
    const float unl = dir == 0 ? ul : vl, unr = dir == 0 ? ur : vr;
    const float utl = dir == 0 ? vl : ul, utr = dir == 0 ? vr : ur;
    const float cl = sr_sqrt(2.0f * pl * rl), cr = sr_sqrt(2.0f * pr * rr);
    const float s_l = fminf(unl - cl, unr - cr), s_r = fmaxf(unl + cl, unr + cr);
    const float ml = sl * unl, mr = sr * unr;
    float fl[4], fr[4];
    fl[0] = ml;
    fl[1 + dir] = ml * unl + pl;
    fl[2 - dir] = ml * utl;
    fl[3] = (Ul[3] + pl) * unl;
    fr[0] = mr;
    fr[1 + dir] = mr * unr + pr;
    fr[2 - dir] = mr * utr;
    fr[3] = (Ur[3] + pr) * unr;
    if (s_l >= 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = fl[k];
    } else if (s_r <= 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = fr[k];
    } else {
        const float inv = sr_div(1.0f, s_r - s_l);
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = (s_r * fl[k] - s_l * fr[k] + s_l * s_r * (Ur[k] - Ul[k])) * inv;
    }
    const FaceRef up = f[0] > 0.0f ? l : r;
#pragma unroll
    for (int k = 0; k < NS; k++) f[4 + k] = f[0] * up.at(5 + k);
}

// ---------------------------------------------------------------------------------------------- the tile kernel
enum { kRefSource = 0, kRefUpdate = 1, kRefUpdateGrav = 2 };

__device__ __forceinline__ int mirror_coord(int g, int n, bool bounce, bool& flip, int& clamp) {
    // the ghost's source along one axis (hydro.rs:686-709): bounce mirrors (the normal velocity negated), leave copies
    // the edge cell (the normal velocity clamped outward: -1 to <= 0, +1 to >= 0)
    flip = false;
    clamp = 0;
    if (g < 0) {
        if (bounce) {
            flip = true;
            g = -g - 1;
        } else {
            clamp = -1;
            g = 0;
        }
    } else if (g >= n) {
        if (bounce) {
            flip = true;
            g = 2 * n - 1 - g;
        } else {
            clamp = 1;
            g = n - 1;
        }
    }
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

template <int MODE>
__global__ void __launch_bounds__(RNT, 2) ref_hydro_kernel(RefArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RShared& S = *reinterpret_cast<RShared*>(smem_raw);
    const RefConst& R = A.R;
    const int w = R.w, h = R.h;
    const size_t n = (size_t)w * h;
    const int x0 = blockIdx.x * RT, y0 = blockIdx.y * RT;
    const int tid = threadIdx.x;
    const bool bounce = R.edge == SR_EDGE_BOUNCE;
    const bool has_g = MODE != kRefUpdate && A.gx != nullptr;
    const float dt = (float)*A.dt, half = 0.5f * dt;

    for (int i = tid; i < 4 * kColdPoints; i += RNT) (&S.tab[0][0])[i] = R.table[i];
    const Eos E{R, &S.tab[0][0]};
    __syncthreads();

    // ---- the primitives of the tile and its 2-cell ring, ghosts by the edge mode
    for (int i = tid; i < RP * RP; i += RNT) {
        const int px = i % RP, py = i / RP;
        const int gxc = x0 + px - 2, gyc = y0 + py - 2;
        bool fu, fv;
        int cu, cv;
        const int sx = mirror_coord(gxc, w, bounce, fu, cu), sy = mirror_coord(gyc, h, bounce, fv, cv);
        const size_t c = (size_t)sy * w + sx;
        float x[NS];
#pragma unroll
        for (int k = 0; k < NS; k++) x[k] = A.U[(4 + k) * n + c];
        const float sig = A.U[c];
        RPrim p = ref_read(E, sig, A.U[n + c], A.U[2 * n + c], A.U[3 * n + c], x);
        if (fu) p.u = -p.u;
        if (fv) p.v = -p.v;
        if (cu < 0) p.u = fminf(p.u, 0.0f);
        if (cu > 0) p.u = fmaxf(p.u, 0.0f);
        if (cv < 0) p.v = fminf(p.v, 0.0f);
        if (cv > 0) p.v = fmaxf(p.v, 0.0f);
        S.P[0][i] = p.s;
        S.P[1][i] = p.u;
        S.P[2][i] = p.v;
        S.P[3][i] = p.p;
#pragma unroll
        for (int k = 0; k < NS; k++) S.P[4 + k][i] = p.x[k];
        const bool inside = gxc >= 0 && gxc < w && gyc >= 0 && gyc < h;
        uint8_t fl = 0;
        if (inside) {
            if (sig < R.sigma_vac) fl |= 1;
            if (A.held[c]) fl |= 2;
        }
        S.FL[i] = fl;
    }
    __syncthreads();

    // P2's g at a region cell: a ghost's is its edge cell's (hydro.rs:711-718)
    auto g_at = [&](int tx, int ty, float& gxv, float& gyv) {
        gxv = gyv = 0.0f;
        if (!has_g) return;
        int gxc = x0 + tx, gyc = y0 + ty;
        gxc = gxc < 0 ? 0 : (gxc >= w ? w - 1 : gxc);
        gyc = gyc < 0 ? 0 : (gyc >= h ? h - 1 : gyc);
        const size_t c = (size_t)gyc * w + gxc;
        gxv = A.gx[c];
        gyv = A.gy[c];
    };

    // ---- the tile cells' four predicted faces and mids
    {
        const int tx = tid % RT, ty = tid / RT;
        const int c = (ty + 2) * RP + tx + 2;
        float gxv, gyv;
        g_at(tx, ty, gxv, gyv);
        Predict P;
        predict(E, S, c, half, has_g, gxv, gyv, P);
        const int q = (ty + 1) * RQ + tx + 1;
        S.MID[0][q] = P.mid[0];
        S.MID[1][q] = P.mid[1];
        S.MID[2][q] = P.mid[2];
#pragma unroll 1
        for (int f = 0; f < 4; f++) evolve_face(E, S, c, P, f, half, has_g, gxv, gyv, &S.TF[0][f][tid], 4 * RNT);
    }
    // ---- the ring cells' faces toward the tile: left column (x+), right column (x-), top row (y+), bottom row (y-)
    if (tid < 4 * RT) {
        const int side = tid / RT, k = tid % RT;
        const int tx = side == 0 ? -1 : (side == 1 ? RT : k);
        const int ty = side == 2 ? -1 : (side == 3 ? RT : (side < 2 ? k : 0));
        const int f = side == 0 ? 1 : (side == 1 ? 0 : (side == 2 ? 3 : 2));
        const int c = (ty + 2) * RP + tx + 2;
        float gxv, gyv;
        g_at(tx, ty, gxv, gyv);
        Predict P;
        predict(E, S, c, half, has_g, gxv, gyv, P);
        const int q = (ty + 1) * RQ + tx + 1;
        S.MID[0][q] = P.mid[0];
        S.MID[1][q] = P.mid[1];
        S.MID[2][q] = P.mid[2];
        evolve_face(E, S, c, P, f, half, has_g, gxv, gyv, &S.RF[0][tid], 4 * RT);
    }
    if (MODE == kRefUpdateGrav) {
        for (int i = tid; i < RQ * RQ; i += RNT) {
            const int gxc = x0 + i % RQ - 1, gyc = y0 + i / RQ - 1;
            S.PH[i] = (gxc >= 0 && gxc < w && gyc >= 0 && gyc < h) ? A.phim[(size_t)gyc * w + gxc] : 0.0f;
        }
    }
    __syncthreads();

    const int tx = tid % RT, ty = tid / RT;
    const int gxc = x0 + tx, gyc = y0 + ty;
    const bool active = gxc < w && gyc < h;
    double kick[2] = {0.0, 0.0}, pushs[3] = {0.0, 0.0, 0.0};
    float best = 0.0f;
    int best_i = -1;
    if (active) {
        const size_t i = (size_t)gyc * w + gxc;
        const int pc = (ty + 2) * RP + tx + 2;
        auto flags = [&](int dx, int dy) { return S.FL[pc + dy * RP + dx]; };
        auto vac = [&](int dx, int dy) { return (flags(dx, dy) & 1) != 0; };
        const bool empty = vac(0, 0) && (gxc == 0 || vac(-1, 0)) && (gxc + 1 == w || vac(1, 0)) &&
                           (gyc == 0 || vac(0, -1)) && (gyc + 1 == h || vac(0, 1));
        const bool held_here = (flags(0, 0) & 2) != 0;
        // the stored face f of the region cell (tx + dx, ty + dy): a tile cell's, or the ring cell's one face
        auto face = [&](int cx, int cy, int f) -> FaceRef {
            if (cx >= 0 && cx < RT && cy >= 0 && cy < RT) return FaceRef{&S.TF[0][f][cy * RT + cx], 4 * RNT};
            const int r = cx < 0 ? cy : (cx >= RT ? RT + cy : (cy < 0 ? 2 * RT + cx : 3 * RT + cx));
            return FaceRef{&S.RF[0][r], 4 * RT};
        };
        // face `side` (0 x-, 1 x+, 2 y-, 3 y+) of this cell: its flux and whether it is still (a held side)
        float q[4];
        bool still[4];
        float acc[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) acc[k] = 0.0f;
#pragma unroll 1
        for (int side = 0; side < 4; side++) {
            const int dir = side >> 1, high = side & 1;
            const int dx = dir == 0 ? (high ? 1 : -1) : 0, dy = dir == 1 ? (high ? 1 : -1) : 0;
            const int nx = gxc + dx, ny = gyc + dy;
            const bool edge = nx < 0 || nx >= w || ny < 0 || ny >= h;
            const FaceRef own = face(tx, ty, side);
            float f[NC];
            // the low cell's high face against the high cell's low face
            if (!edge) {
                if (high) hll(own, face(tx + dx, ty + dy, side - 1), dir, false, false, f);
                else hll(face(tx + dx, ty + dy, side + 1), own, dir, false, false, f);
            } else if (bounce) {
#pragma unroll
                for (int k = 0; k < NC; k++) f[k] = 0.0f;
                f[1 + dir] = own.at(4);  // hydro.rs:556-562: the wall's flux, Π alone
            } else {
                // hydro.rs:564-582: leave — HLL against the ghost's facing face, a wall where the mass flows in
                if (high) hll(own, face(tx + dx, ty + dy, side - 1), dir, false, false, f);
                else hll(face(tx + dx, ty + dy, side + 1), own, dir, false, false, f);
                const bool inflow = high ? f[0] < 0.0f : f[0] > 0.0f;
                if (inflow) {
#pragma unroll
                    for (int k = 0; k < NC; k++) f[k] = 0.0f;
                    f[1 + dir] = own.at(4);
                }
            }
            // held faces (hydro.rs:780-812): nothing past a held cell's edge or between two held cells; a reflecting
            // wall (HLL against the free side's mirror, mass, energy and species 0) between a held and a free cell
            const bool hn = !edge && (flags(dx, dy) & 2) != 0;
            still[side] = held_here || hn;
            if (still[side]) {
                if (!edge && held_here != hn) {
                    if (held_here) {  // the free side is the neighbour: its face toward this cell
                        const FaceRef fr = face(tx + dx, ty + dy, high ? side - 1 : side + 1);
                        if (high) hll(fr, fr, dir, true, false, f);   // free cell on the high side: mirror | face
                        else hll(fr, fr, dir, false, true, f);        // free cell on the low side: face | mirror
                    } else {
                        if (high) hll(own, own, dir, false, true, f);  // this free cell is the low side
                        else hll(own, own, dir, true, false, f);
                    }
                    f[0] = 0.0f;
                    f[3] = 0.0f;
#pragma unroll
                    for (int k = 4; k < NC; k++) f[k] = 0.0f;
                } else {
#pragma unroll
                    for (int k = 0; k < NC; k++) f[k] = 0.0f;
                }
            }
            q[side] = f[0];
            const float sgn = high ? 1.0f : -1.0f;
#pragma unroll
            for (int k = 0; k < NC; k++) acc[k] += sgn * f[k];
        }
        const float sig = A.U[i];
        if (MODE == kRefSource) {
            float s;
            if (held_here) {
                s = sig;
            } else if (empty) {
                s = 0.0f;
            } else {
                const float start = vac(0, 0) ? R.sigma_floor : sig;
                const float div = (q[1] - q[0]) + (q[3] - q[2]);
                s = 0.5f * (sig + (start - dt * div));
            }
            s = s >= R.sigma_vac ? s : 0.0f;
            A.src[i] = s;
            A.src_free[i] = held_here ? 0.0f : s;
        } else if (empty) {
#pragma unroll 1
            for (int k = 0; k < NC; k++) A.Uout[k * n + i] = A.U[k * n + i];
            if (A.push) {
                A.push[i] = 0.0f;
                A.push[n + i] = 0.0f;
            }
        } else {
            float u[NC];
            if (vac(0, 0)) {
                RPrim p;
                p.s = S.P[0][pc];
                p.u = S.P[1][pc];
                p.v = S.P[2][pc];
                p.p = S.P[3][pc];
#pragma unroll
                for (int k = 0; k < NS; k++) p.x[k] = S.P[4 + k][pc];
                ref_cons(E, p, u);
            } else {
                u[0] = sig;
                u[1] = A.U[n + i];
                u[2] = A.U[2 * n + i];
                u[3] = A.U[3 * n + i];
#pragma unroll
                for (int k = 0; k < NS; k++) u[4 + k] = sig * A.U[(4 + k) * n + i];
            }
#pragma unroll
            for (int k = 0; k < NC; k++)
                if (!(held_here && (k == 1 || k == 2))) u[k] -= dt * acc[k];
            if (MODE == kRefUpdateGrav && has_g) {
                // gravity's source at the half step (hydro.rs:905-946)
                const float src = A.src[i];
                const float gxo = held_here ? A.gxp[i] : A.gxm[i], gyo = held_here ? A.gyp[i] : A.gym[i];
                kick[0] = (double)(dt * src * gxo);
                kick[1] = (double)(dt * src * gyo);
                if (!held_here && src > 0.0f) {
                    best = src;
                    best_i = (int)i;
                }
                if (!held_here) {
                    const int qc = (ty + 1) * RQ + tx + 1;
                    const float p = S.PH[qc];
                    const float m0 = S.MID[0][qc], m1 = S.MID[1][qc], m2 = S.MID[2][qc];
                    float kx = dt * src * A.gxm[i], ky = dt * src * A.gym[i], en = 0.0f;
                    // each face read as its low and its high cell read it (face_work, hydro.rs:1042-1067)
#pragma unroll 1
                    for (int side = 0; side < 4; side++) {
                        if (still[side]) continue;
                        const int dir = side >> 1, high = side & 1;
                        const int dx = dir == 0 ? (high ? 1 : -1) : 0, dy = dir == 1 ? (high ? 1 : -1) : 0;
                        const int nx = gxc + dx, ny = gyc + dy;
                        const bool edge = nx < 0 || nx >= w || ny < 0 || ny >= h;
                        const int qn = qc + dy * RQ + dx;
                        const float pn = edge ? p : S.PH[qn];
                        const float mn0 = edge ? m0 : S.MID[0][qn];
                        const float mnp = edge ? (dir ? m2 : m1) : S.MID[1 + dir][qn];
                        const float mp = dir ? m2 : m1;
                        float sl, sh, pl, ph, d;
                        if (high) {
                            sl = m0; sh = mn0; pl = mp; ph = mnp; d = p - pn;
                        } else {
                            sl = mn0; sh = m0; pl = mnp; ph = mp; d = pn - p;
                        }
                        const float a = fmaxf(sl, 0.0f), b = fmaxf(sh, 0.0f);
                        const float wl = a + b > 0.0f ? a / (a + b) : 0.5f;
                        const float extra = dt * (q[side] - 0.5f * (pl + ph)) * d;
                        float cc = 0.0f, kk = 0.0f, el = 0.0f, eh = 0.0f;
                        if (extra < 0.0f && a > 0.0f && b > 0.0f) {
                            const float ul = pl / a, uh = ph / b, du = ul - uh, inv = 1.0f / a + 1.0f / b;
                            cc = fminf(-extra, 0.25f * du * du / inv);
                            if (cc > 0.0f) {
                                const float disc = sqrtf(fmaxf(du * du - 2.0f * inv * cc, 0.0f));
                                kk = -2.0f * cc / (du + copysignf(1.0f, du) * disc);
                                el = ul * kk + 0.5f * kk * kk / a;
                                eh = -uh * kk + 0.5f * kk * kk / b;
                            }
                        }
                        const float rest = extra + cc;
                        if (high) {  // this cell is the face's low cell
                            en += 0.5f * dt * pl * d + wl * rest + el;
                            if (dir == 0) kx += kk;
                            else ky += kk;
                        } else {  // this cell is the face's high cell
                            en += 0.5f * dt * ph * d + (1.0f - wl) * rest + eh;
                            if (dir == 0) kx -= kk;
                            else ky -= kk;
                        }
                    }
                    u[1] += kx;
                    u[2] += ky;
                    u[3] += en;
                }
            }
            float px = 0.0f, py = 0.0f;
            if (A.radx && !held_here && sig >= R.sigma_vac) {
                // the radiation force from the cell as the step found it (hydro.rs:365-405, 947-956)
                float x[NS];
#pragma unroll
                for (int k = 0; k < NS; k++) x[k] = A.U[(4 + k) * n + i];
                float inv_mu, ye;
                composition(x, inv_mu, ye);
                float kappa = R.kappa0 * (1.0f + x[0]);
                if (R.kappa_dust != 0.0f) {
                    const float mx = A.U[n + i], my = A.U[2 * n + i];
                    float raw = A.U[3 * n + i] / sig - 0.5f * (mx * mx + my * my) / (sig * sig) -
                                E.eps_cold(sig, ye, x[NS - 1]);
                    const float eps = fmaxf(raw, R.t_floor * inv_mu);
                    if (eps / inv_mu < R.t_dust) kappa += R.kappa_dust * (1.0f - x[0] - x[1] - x[NS - 1]);
                }
                const float dx = dt * kappa * sig * A.radx[i] * R.inv_c_sb, dy = dt * kappa * sig * A.rady[i] * R.inv_c_sb;
                const float d2 = dx * dx + dy * dy;
                float share = 1.0f;
                if (d2 != 0.0f) {
                    const float s = u[0], rs = 1.0f / s;
                    float xs[NS];
#pragma unroll
                    for (int k = 0; k < NS; k++) xs[k] = u[4 + k] * rs;
                    float im, y2;
                    composition(xs, im, y2);
                    const float raw = u[3] * rs - 0.5f * (u[1] * u[1] + u[2] * u[2]) * rs * rs -
                                      E.eps_cold(s, y2, xs[NS - 1]);
                    const float a = s * (raw - R.t_floor * im);
                    if (!(a > 0.0f)) {
                        share = 0.0f;
                    } else {
                        const float qd = u[1] * dx + u[2] * dy;
                        const float disc = sqrtf(qd * qd + 2.0f * s * a * d2);
                        const float root = qd >= 0.0f ? 2.0f * s * a / (qd + disc) : (disc - qd) / d2;
                        share = fminf(root, 1.0f);
                    }
                }
                px = share * dx;
                py = share * dy;
                u[1] += px;
                u[2] += py;
                pushs[0] = px;
                pushs[1] = py;
                pushs[2] = sqrt((double)px * px + (double)py * py);
            }
            if (A.push) {
                A.push[i] = px;
                A.push[n + i] = py;
            }
            const float r0 = 1.0f / u[0];
#pragma unroll
            for (int k = 0; k < 4; k++) A.Uout[k * n + i] = u[k];
#pragma unroll
            for (int k = 0; k < NS; k++) A.Uout[(4 + k) * n + i] = u[4 + k] * r0;
        }
    }
    if (MODE == kRefSource) return;
    // ---- per-CTA partials: gravity's net kick, the densest free cell (lowest index on a tie), the net push
    double v[5] = {kick[0], kick[1], pushs[0], pushs[1], pushs[2]};
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 5; k++) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        const float ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, best_i, o);
        if (oi >= 0 && (best_i < 0 || ob > best || (ob == best && oi < best_i))) {
            best = ob;
            best_i = oi;
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 5; k++) S.red[k][warp] = v[k];
        S.rbest[warp] = best;
        S.ridx[warp] = best_i;
    }
    __syncthreads();
    if (tid == 0) {
        const int b = blockIdx.y * gridDim.x + blockIdx.x;
        for (int k = 0; k < 5; k++) {
            double t = 0.0;
            for (int q = 0; q < RNT / 32; q++) t += S.red[k][q];
            A.part[(size_t)b * 5 + k] = t;
        }
        float bb = 0.0f;
        int bi = -1;
        for (int q = 0; q < RNT / 32; q++)
            if (S.ridx[q] >= 0 && (bi < 0 || S.rbest[q] > bb || (S.rbest[q] == bb && S.ridx[q] < bi))) {
                bb = S.rbest[q];
                bi = S.ridx[q];
            }
        A.part_best[b] = bb;
        A.part_idx[b] = bi;
    }
}

// One CTA: the partials reduced in a fixed order into fin = [kick x, kick y, densest, push x, push y, |push|].
__global__ void ref_reduce_kernel(RefArgs A, int nblocks) {
    __shared__ double sd[5][256];
    __shared__ float sb[256];
    __shared__ int si[256];
    const int tid = threadIdx.x;
    double acc[5] = {0, 0, 0, 0, 0};
    float best = 0.0f;
    int bi = -1;
    const int per = (nblocks + 255) / 256;
    for (int b = tid * per; b < min(nblocks, (tid + 1) * per); b++) {
        for (int k = 0; k < 5; k++) acc[k] += A.part[(size_t)b * 5 + k];
        const int oi = A.part_idx[b];
        const float ob = A.part_best[b];
        if (oi >= 0 && (bi < 0 || ob > best || (ob == best && oi < bi))) {
            best = ob;
            bi = oi;
        }
    }
    for (int k = 0; k < 5; k++) sd[k][tid] = acc[k];
    sb[tid] = best;
    si[tid] = bi;
    __syncthreads();
    if (tid != 0) return;
    double t[5] = {0, 0, 0, 0, 0};
    for (int q = 0; q < 256; q++)
        for (int k = 0; k < 5; k++) t[k] += sd[k][q];
    float bb = 0.0f;
    int idx = -1;
    for (int q = 0; q < 256; q++)
        if (si[q] >= 0 && (idx < 0 || sb[q] > bb || (sb[q] == bb && si[q] < idx))) {
            bb = sb[q];
            idx = si[q];
        }
    A.fin[0] = t[0];
    A.fin[1] = t[1];
    A.fin[2] = (double)idx;
    A.fin[3] = t[2];
    A.fin[4] = t[3];
    A.fin[5] = t[4];
}

// hydro.rs:975-1012: the net push taken back in proportion to each cell's, the net kick from the densest free cell,
// then the sticky wall (a free gas cell's momentum into a held neighbour stopped).
__global__ void ref_apply_kernel(RefArgs A) {
    const RefConst& R = A.R;
    const int w = R.w, h = R.h;
    const size_t n = (size_t)w * h;
    const double nx = A.fin[3], ny = A.fin[4], sabs = A.fin[5];
    const long long densest = (long long)A.fin[2];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float mx = A.Uout[n + i], my = A.Uout[2 * n + i];
        bool changed = false;
        if (sabs > 0.0 && A.push) {
            const float px = A.push[i], py = A.push[n + i];
            const double m = sqrt((double)px * px + (double)py * py);
            if (m != 0.0) {
                mx = (float)((double)mx - m * nx / sabs);
                my = (float)((double)my - m * ny / sabs);
                changed = true;
            }
        }
        if ((long long)i == densest) {
            mx = (float)((double)mx - A.fin[0]);
            my = (float)((double)my - A.fin[1]);
            changed = true;
        }
        if (!A.held[i] && A.Uout[i] >= R.sigma_vac) {
            int x, y;
            split_index(i, w, x, y);
            const bool into_x = (x > 0 && A.held[i - 1] && mx < 0.0f) || (x + 1 < w && A.held[i + 1] && mx > 0.0f);
            const bool into_y = (y > 0 && A.held[i - w] && my < 0.0f) || (y + 1 < h && A.held[i + w] && my > 0.0f);
            if (into_x) {
                mx = 0.0f;
                changed = true;
            }
            if (into_y) {
                my = 0.0f;
                changed = true;
            }
        }
        if (changed) {
            A.Uout[n + i] = mx;
            A.Uout[2 * n + i] = my;
        }
    }
}

// ---------------------------------------------------------------------------------------------- P8 and P9
__device__ __forceinline__ bool renormalised(const float* raw, float* x) {
    // floors.rs:45-58; false when a fraction is not finite (the cell is left as read)
    float sum = 0.0f;
    bool finite = true;
#pragma unroll
    for (int k = 0; k < NS; k++) {
        finite = finite && isfinite(raw[k]);
        x[k] = fmaxf(raw[k], 0.0f);
        sum += x[k];
    }
    if (sum > 0.0f) {
        const float r = 1.0f / sum;
#pragma unroll
        for (int k = 0; k < NS; k++) x[k] *= r;
    } else {
#pragma unroll
        for (int k = 0; k < NS; k++) x[k] = 0.0f;
        x[0] = 1.0f;
    }
    return finite;
}

__global__ void ref_floors_kernel(RefConst R, float* __restrict__ U) {
    // floors.rs:124-175: species renormalised; below Σ_vac the floor state (Σ_floor, at rest, T_floor, its fractions
    // kept); else ε_th raised to T_floor/μ
    const Eos E{R, R.table};
    const size_t n = (size_t)R.w * R.h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float raw[NS], x[NS];
#pragma unroll
        for (int k = 0; k < NS; k++) raw[k] = U[(4 + k) * n + i];
        if (!renormalised(raw, x)) continue;
        float inv_mu, ye;
        composition(x, inv_mu, ye);
        const float s = U[i], floor = R.t_floor * inv_mu;
        if (s < R.sigma_vac) {
            const float sf = R.sigma_floor;
            U[i] = sf;
            U[n + i] = 0.0f;
            U[2 * n + i] = 0.0f;
            U[3 * n + i] = sf * (floor + E.eps_cold(sf, ye, x[NS - 1]));
        } else {
            const float mx = U[n + i], my = U[2 * n + i], en = U[3 * n + i];
            const float rs = 1.0f / s;
            const float raw_e = en * rs - 0.5f * (mx * mx + my * my) * rs * rs - E.eps_cold(s, ye, x[NS - 1]);
            if (raw_e < floor) U[3 * n + i] = en + s * (floor - raw_e);
        }
#pragma unroll
        for (int k = 0; k < NS; k++) U[(4 + k) * n + i] = x[k];
    }
}

// floors.rs:196-243 (the hold) and hydro.rs:618-634 (the Δt terms) with the guard over the 14 channels.
__global__ void ref_hold_dt_kernel(RefConst R, float* __restrict__ U, uint8_t* __restrict__ held,
                                   const float* __restrict__ gx, const float* __restrict__ gy, int do_hold, int do_dt,
                                   float* part_rate, float* part_g, long long* part_nf) {
    const Eos E{R, R.table};
    const int w = R.w, h = R.h;
    const size_t n = (size_t)w * h;
    float rate = 0.0f, gmax = 0.0f;
    long long nf = LLONG_MAX;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float raw[NS];
#pragma unroll
        for (int k = 0; k < NS; k++) raw[k] = U[(4 + k) * n + i];
        const float s = U[i];
        float mx = U[n + i], my = U[2 * n + i];
        const float en = U[3 * n + i];
        if (do_hold) {
            float x[NS];
            if (renormalised(raw, x)) {
                float inv_mu, ye;
                composition(x, inv_mu, ye);
                const float cold = E.eps_cold(s, ye, x[NS - 1]);
                const float eps_th = en / s - 0.5f * (mx * mx + my * my) / (s * s) - cold;
                const bool kind = x[8] < 1e-3f || x[NS - 1] >= 0.5f;  // no iron past a trace, or neutron-rich
                const bool was = held[i] != 0;
                const bool rest = was ? !(eps_th > 2.0f * R.eta_hold * cold || s < 0.5f * R.sigma_hold || !kind)
                                      : (s >= R.sigma_hold && eps_th <= R.eta_hold * cold && kind);
                bool now = false;
                if (rest) {
                    // the mass of the disk r <= r_hold about the cell, centre to centre, clipped (sinks.rs:117-125)
                    const int k = (int)R.r_hold;
                    int x0, y0;
                    split_index(i, w, x0, y0);
                    const float r2 = R.r_hold * R.r_hold;
                    double m = 0.0;
                    for (int dy = -k; dy <= k; dy++) {
                        const int cy = y0 + dy;
                        if (cy < 0 || cy >= h) continue;
                        for (int dx = -k; dx <= k; dx++) {
                            const int cx = x0 + dx;
                            if (cx >= 0 && cx < w && (float)(dx * dx + dy * dy) <= r2) m += U[(size_t)cy * w + cx];
                        }
                    }
                    now = m < (double)R.m_tov;
                }
                if (now && !was) {
                    mx = 0.0f;
                    my = 0.0f;
                    U[n + i] = 0.0f;
                    U[2 * n + i] = 0.0f;
                }
                held[i] = now ? 1 : 0;
            }
        }
        if (!do_dt) continue;
        if (!(isfinite(s) && isfinite(mx) && isfinite(my) && isfinite(en))) {
            const int c = !isfinite(s) ? 0 : (!isfinite(mx) ? 1 : (!isfinite(my) ? 2 : 3));
            nf = min(nf, (long long)i * NC + c);
        } else {
            for (int k = 0; k < NS; k++)
                if (!isfinite(raw[k])) {
                    nf = min(nf, (long long)i * NC + 4 + k);
                    break;
                }
        }
        const RPrim p = ref_read(E, s, mx, my, en, raw);
        const float c = sr_sqrt(2.0f * sr_div(p.p, p.s));
        rate = fmaxf(rate, (fabsf(p.u) + c) + (fabsf(p.v) + c));
        if (gx) gmax = fmaxf(gmax, hypotf(gx[i], gy[i]));
    }
    if (!do_dt) return;
    __shared__ float sr[32], sg[32];
    __shared__ long long sn[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rate = fmaxf(rate, __shfl_down_sync(0xffffffffu, rate, o));
        gmax = fmaxf(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
        const long long on = __shfl_down_sync(0xffffffffu, nf, o);
        nf = on < nf ? on : nf;
    }
    if (lane == 0) {
        sr[warp] = rate;
        sg[warp] = gmax;
        sn[warp] = nf;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x / 32); k++) {
            rate = fmaxf(rate, sr[k]);
            gmax = fmaxf(gmax, sg[k]);
            nf = sn[k] < nf ? sn[k] : nf;
        }
        part_rate[blockIdx.x] = rate;
        part_g[blockIdx.x] = gmax;
        part_nf[blockIdx.x] = nf;
    }
}

__global__ void ref_cell_flux_kernel(const float* __restrict__ fx, const float* __restrict__ fy, float* radx, float* rady,
                                     int w, int h) {
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t x = i % w, y = i / w;
        radx[i] = 0.5f * (fx[y * (w + 1) + x] + fx[y * (w + 1) + x + 1]);
        rady[i] = 0.5f * (fy[y * w + x] + fy[(y + 1) * w + x]);
    }
}

int ref_grid(size_t n) {
    const size_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

}  // namespace

// ---------------------------------------------------------------------------------------------- host
void ref_cold_tables(const sr_config& cfg, float* out) {
    // eos.rs:31-98 in f64: J(x_i) = ∫₀^{x_i} P(s)/s² ds by Simpson's rule in t = √s (the first segment 8x finer),
    // ln u_i = ln(x_i J); stored as u_i and ln u_{i+1} - ln u_i
    const double pairs[2][2] = {{cfg.k1e, cfg.k2e}, {cfg.k1n, cfg.k2n}};
    for (int q = 0; q < 2; q++) {
        float* u = out + 2 * q * kColdPoints;
        float* d = u + kColdPoints;
        const double k1 = pairs[q][0], k2 = pairs[q][1];
        if (!(k1 > 0.0 && k2 > 0.0)) {
            for (int i = 0; i < kColdPoints; i++) u[i] = d[i] = 0.0f;
            continue;
        }
        auto P = [&](double x) { return x <= 0.0 ? 0.0 : 1.0 / (1.0 / (k1 * x * x) + 1.0 / (k2 * pow(x, 1.5))); };
        auto f = [&](double t) {
            if (t <= 0.0) return 0.0;
            const double s = t * t;
            return P(s) / (s * s) * 2.0 * t;
        };
        auto node = [&](int i) {
            const double frac = (double)i / (kColdPoints - 1);
            return exp(log(kXMin) + frac * (log(kXMax) - log(kXMin)));
        };
        std::vector<double> ln_u(kColdPoints);
        double t_prev = 0.0, J = 0.0;
        for (int i = 0; i < kColdPoints; i++) {
            const double t = sqrt(node(i));
            const int steps = i == 0 ? 64 * 8 : 64;
            const double hq = (t - t_prev) / steps;
            double acc = f(t_prev) + f(t);
            for (int k = 1; k < steps; k++) acc += f(t_prev + hq * k) * (k % 2 == 1 ? 4.0 : 2.0);
            J += acc * hq / 3.0;
            ln_u[i] = log(node(i) * J);
            t_prev = t;
        }
        for (int i = 0; i < kColdPoints; i++) {
            u[i] = (float)exp(ln_u[i]);
            d[i] = i + 1 < kColdPoints ? (float)(ln_u[i + 1] - ln_u[i]) : 0.0f;
        }
    }
}

int ref_hydro_blocks(int w, int h) { return (int)(div_up(w, RT) * div_up(h, RT)); }

static void ref_launch(int mode, const RefArgs& A, cudaStream_t s) {
    const dim3 grid(div_up(A.R.w, RT), div_up(A.R.h, RT));
    const size_t smem = sizeof(RShared);
    static bool configured[3] = {false, false, false};
    if (mode == kRefSource) {
        if (!configured[0]) {
            SR_CUDA_TRY(cudaFuncSetAttribute(ref_hydro_kernel<kRefSource>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            configured[0] = true;
        }
        ref_hydro_kernel<kRefSource><<<grid, RNT, smem, s>>>(A);
    } else if (mode == kRefUpdate) {
        if (!configured[1]) {
            SR_CUDA_TRY(cudaFuncSetAttribute(ref_hydro_kernel<kRefUpdate>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            configured[1] = true;
        }
        ref_hydro_kernel<kRefUpdate><<<grid, RNT, smem, s>>>(A);
    } else {
        if (!configured[2]) {
            SR_CUDA_TRY(cudaFuncSetAttribute(ref_hydro_kernel<kRefUpdateGrav>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            configured[2] = true;
        }
        ref_hydro_kernel<kRefUpdateGrav><<<grid, RNT, smem, s>>>(A);
    }
    SR_CUDA_TRY(cudaGetLastError());
    sr_note_launch();
}

void ref_hydro_source_launch(const RefArgs& A, cudaStream_t s) { ref_launch(kRefSource, A, s); }

void ref_hydro_update_launch(const RefArgs& A, int gravity, cudaStream_t s) {
    ref_launch(gravity ? kRefUpdateGrav : kRefUpdate, A, s);
}

void ref_hydro_finalize_launch(const RefArgs& A, cudaStream_t s) {
    ref_reduce_kernel<<<1, 256, 0, s>>>(A, ref_hydro_blocks(A.R.w, A.R.h));
    sr_note_launch();
    ref_apply_kernel<<<ref_grid((size_t)A.R.w * A.R.h), 256, 0, s>>>(A);
    sr_note_launch();
}

void ref_cell_flux_launch(const float* fx, const float* fy, float* radx, float* rady, int w, int h, cudaStream_t s) {
    ref_cell_flux_kernel<<<ref_grid((size_t)w * h), 256, 0, s>>>(fx, fy, radx, rady, w, h);
    sr_note_launch();
}

void ref_floors_launch(const RefConst& R, float* U, cudaStream_t s) {
    ref_floors_kernel<<<ref_grid((size_t)R.w * R.h), 256, 0, s>>>(R, U);
    sr_note_launch();
}

void ref_hold_dt_launch(const RefConst& R, float* U, uint8_t* held, const float* gx, const float* gy, int do_hold,
                        int do_dt, float* part_rate, float* part_g, long long* part_nf, double cfl, double eta_g,
                        double dt_fixed, double dt_cap, DtRecord* rec, cudaStream_t s) {
    const int nb = ref_grid((size_t)R.w * R.h);
    ref_hold_dt_kernel<<<nb, 256, 0, s>>>(R, U, held, gx, gy, do_hold, do_dt, part_rate, part_g, part_nf);
    sr_note_launch();
    if (do_dt) dt_finalize_launch(nb, kRefChannels, part_rate, part_g, part_nf, cfl, eta_g, dt_fixed, dt_cap, rec, s);
}
