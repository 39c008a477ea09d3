// heat.cu — P5, the implicit flux-limited radiative diffusion step (crates/sr-physics/src/reference/heat.rs:453-592).
//
// One backward-Euler step in the heat potential u = a_r T⁴ with the Levermore–Pomraning law frozen at the pass start.
// Newton passes linearise T(u); each pass is one SPD 5-point system A u = b, solved here by iterative refinement:
// the residual r = b - A x and the update x += s e in FP64 (s the residual's rms scale), the correction from an FP32
// preconditioned CG on A e = r/s with FP64 dot products, preconditioned by the FP32 multigrid V-cycle (mg.cu) or
// Jacobi. The passes stop by the reference's two rules (the heat moved, the largest cell change); the commit closes the
// heat balance with δ (heat.rs:521-536), or past the ceiling commits by limited fluxes (heat.rs:545-592).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "heat.cuh"
#include "learned.cuh"
#include "mg.cuh"
#include "reduce.cuh"

namespace {

constexpr int RED_THREADS = 256;
constexpr double kFirstPassTol = 0.1;  // the first Newton pass's relative residual (and the loosest any pass asks)
constexpr double kTrustedPassTol = 1e-5;  // passes this loose end on their FP32 solve's own test
constexpr int kMaxRefinements = 16;    // FP64 refinement sweeps per Newton pass
constexpr int MAX_PART = 1184;    // most CTAs of a grid-stride heat kernel: one wave (148 SMs x 8), few partials to sum
constexpr int PART_CAP = 16384;   // partials per reduced value (the level-0 smoother's CTAs included)
// Device scalars. The kernels read Δt, the refinement's scale, δ and the PCG round's state from here (never from
// launch arguments), so a captured graph of the implicit step replays for any step. The fused MG/Jacobi rounds keep
// <r, z> of this round (S_RZC), of the last (S_RZP) and from the next preconditioner application (S_RZN), and which
// direction buffer is current (S_PAR); the flexible (learned) rounds use S_RZ0/S_RZ1.
enum Slot { S_HEAT0, S_NGAS, S_DT, S_RR, S_BB, S_GAM, S_HM, S_MOVED, S_VIOL, S_UB, S_TB, S_R32, S_PQ, S_RRI, S_RZ0, S_RZ1,
            S_ZRO, S_MGRZ, S_BETA, S_RAD, S_GAIN, S_HELD, S_RZC, S_RZP, S_RZN, S_PAR, S_SCALE, S_ISCALE, S_DELTA,
            S_COUNT };

// Where a kernel's grid sum goes: the partials buffer, the ticket counter and the device scalar(s).
struct Red {
    double* part;
    unsigned* counter;
    double* out;
};

struct HeatConst {
    int w, h;
    double gm1, mu, t_floor, sigma_vac, sigma_floor, a_r, c_sb, kappa0, k_cond, chi;
    int limiter_on;
    int ref;  // reference mode: the sides of heat_cells_kernel's reference branch (C = Σ/μ of each cell)
};

__device__ __forceinline__ double u_of(const HeatConst& K, double t) {
    return K.chi > 0.0 ? t : K.a_r * ((t * t) * (t * t));
}
__device__ __forceinline__ double t_of(const HeatConst& K, double u) {
    return K.chi > 0.0 ? u : sqrt(sqrt(u / K.a_r));
}
__device__ __forceinline__ double dt_du(const HeatConst& K, double t) {
    return K.chi > 0.0 ? 1.0 : 1.0 / (4.0 * K.a_r * ((t * t) * t));
}

// eos.rs:118-131 in f64 on the device tables (u at the node, Δ ln u to the next): u(x) = u_i exp(frac Δ_i)
__device__ __forceinline__ double cold_u64(const float* u, const float* d, double x) {
    if (!(x > 0.0)) return 0.0;
    const double pos = (log(x) + 18.420680743952367) * (511.0 / 36.841361487904734);
    if (pos < 0.0) {
        const double r = x * 1e8;
        return (double)u[0] * r * r;
    }
    int i = (int)pos;
    i = i > 510 ? 510 : i;
    return (double)u[i] * exp((pos - (double)i) * (double)d[i]);
}

// ---- step set-up: the sides (heat.rs:215-226), the faces' D_f (heat.rs:263-294), Σ_f k and its vacuum part
__global__ void heat_cells_kernel(HeatConst K, HeatRef RF, const float* __restrict__ U, const float* __restrict__ kappa,
                                  uint8_t* gas, double* t0, double* C, float* kap, float* sig, double* t, double* u,
                                  Red R) {
    const size_t n = (size_t)K.w * K.h;
    double acc = 0.0, ngas = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double s = U[i];
        if (RF.on) {
            // reference/heat.rs:215-231 with the registry's composition (registry.rs:145-154)
            const double za[10] = {2.0, 0.75, 7.0 / 12.0, 9.0 / 16.0, 11.0 / 20.0, 13.0 / 24.0, 15.0 / 28.0,
                                   17.0 / 32.0, 27.0 / 56.0, 1.0};
            const double ze[10] = {1.0, 0.5, 0.5, 0.5, 0.5, 0.5, 0.5, 0.5, 26.0 / 56.0, 0.0};
            double inv_mu = 0.0, ye = 0.0, x0 = 0.0, x1 = 0.0, xn = 0.0;
            for (int k = 0; k < 10; k++) {
                const double x = U[(4 + k) * n + i];
                inv_mu += x * za[k];
                ye += x * ze[k];
                if (k == 0) x0 = x;
                if (k == 1) x1 = x;
                if (k == 9) xn = x;
            }
            const double mu = 1.0 / inv_mu, z_met = 1.0 - x0 - x1 - xn;
            double T;
            const bool g = s >= K.sigma_vac;
            if (!g) {
                T = K.t_floor;
            } else {
                const double mx = U[n + i], my = U[2 * n + i], e = U[3 * n + i];
                double cold = 0.0;
                if (RF.cold_e) cold += cold_u64(RF.table, RF.table + 512, ye * s);
                if (RF.cold_n) cold += cold_u64(RF.table + 1024, RF.table + 1536, xn * s);
                const double raw = e / s - 0.5 * (mx * mx + my * my) / (s * s) - cold / s;
                const double floor = K.t_floor / mu;
                T = mu * (raw < floor ? floor : raw);
            }
            kap[i] = (float)(K.kappa0 * (1.0 + x0) + (T < RF.t_dust ? RF.kappa_dust * z_met : 0.0));
            gas[i] = g ? 1 : 0;
            t0[i] = T;
            sig[i] = g ? (float)s : (float)K.sigma_floor;
            C[i] = (g ? s : K.sigma_floor) * inv_mu;
            t[i] = T;
            u[i] = u_of(K, T);
            if (g) {
                acc += C[i] * T;
                ngas += 1.0;
            }
            continue;
        }
        const float k = kappa ? kappa[i] : (float)K.kappa0;
        kap[i] = k;
        if (s < K.sigma_vac) {
            gas[i] = 0;
            t0[i] = K.t_floor;
            sig[i] = (float)K.sigma_floor;
            C[i] = K.sigma_floor / (K.mu * K.gm1);
            t[i] = K.t_floor;
            u[i] = u_of(K, K.t_floor);
            continue;
        }
        const double mx = U[n + i], my = U[2 * n + i], e = U[3 * n + i];
        const double kinetic = 0.5 * (mx * mx + my * my) / (s * s);
        const double raw = e / s - kinetic;
        const double floor = K.t_floor / K.mu / K.gm1;
        const double eps = raw < floor ? floor : raw;
        const double T = K.mu * K.gm1 * eps;
        gas[i] = 1;
        t0[i] = T;
        sig[i] = (float)s;
        C[i] = s / (K.mu * K.gm1);
        t[i] = T;
        u[i] = u_of(K, T);
        acc += C[i] * T;
        ngas += 1.0;
    }
    const double v[2] = {acc, ngas};
    grid_sum_last<2>(v, R.part, R.counter, R.out);
}

struct Side {
    bool gas;
    double t, s, kappa, c;
};

__device__ __forceinline__ Side side_at(const HeatConst& K, const uint8_t* gas, const double* t0, const float* kap,
                                        const float* sig, const double* C, size_t i) {
    Side o;
    o.gas = gas[i];
    o.t = t0[i];
    o.s = sig[i];
    o.kappa = kap[i];
    o.c = C[i];
    return o;
}

__device__ __forceinline__ Side vacuum_beyond(const HeatConst& K, const Side& g) {
    Side o;
    o.gas = false;
    o.t = K.t_floor;
    o.s = K.sigma_floor;
    o.kappa = g.kappa;
    o.c = K.ref ? K.sigma_floor * (g.c / g.s) : K.sigma_floor / (K.mu * K.gm1);  // the gas side's μ
    return o;
}

__device__ __forceinline__ double diffusivity(const HeatConst& K, const Side& a, const Side& b) {
    if (!a.gas && !b.gas) return 0.0;
    if (K.chi > 0.0) return K.chi * (0.5 * (a.c + b.c));
    const double ta2 = a.t * a.t, tb2 = b.t * b.t;
    const double era = K.a_r * (ta2 * ta2), erb = K.a_r * (tb2 * tb2);
    const double face_er = 0.5 * (era + erb);
    const double ks = 0.5 * (a.kappa * a.s + b.kappa * b.s);
    const double r = face_er > 0.0 ? fabs(erb - era) / (ks * face_er) : 0.0;
    const double lam = K.limiter_on ? (2.0 + r) / (6.0 + 3.0 * r + r * r) : 1.0 / 3.0;
    const double radiative = K.c_sb * lam / ks;
    const double conduction =
        K.k_cond != 0.0 ? K.k_cond / (K.a_r * (a.t + b.t) * (a.t * a.t + b.t * b.t)) : 0.0;
    return radiative + conduction;
}

__device__ __forceinline__ double face_coef(const HeatConst& K, const Side* a, const Side* b) {
    Side A, B;
    if (a && b) {
        if (a->gas || b->gas) {
            A = a->gas ? *a : vacuum_beyond(K, *b);
            B = b->gas ? *b : vacuum_beyond(K, *a);
        } else {
            A = *a;
            B = *a;
        }
    } else if (a) {
        A = *a;
        B = vacuum_beyond(K, *a);
    } else {
        A = vacuum_beyond(K, *b);
        B = *b;
    }
    return diffusivity(K, A, B);
}

__global__ void heat_faces_kernel(HeatConst K, const uint8_t* __restrict__ gas, const double* __restrict__ t0,
                                  const float* __restrict__ kap, const float* __restrict__ sig,
                                  const double* __restrict__ C, double* kx, double* ky) {
    const int w = K.w, h = K.h;
    const size_t nx = (size_t)(w + 1) * h, ny = (size_t)w * (h + 1);
    for (size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x; f < nx + ny; f += (size_t)gridDim.x * blockDim.x) {
        Side a, b;
        bool ha, hb;
        if (f < nx) {
            int x, y;
            split_index(f, (w + 1), x, y);
            ha = x > 0;
            hb = x < w;
            if (ha) a = side_at(K, gas, t0, kap, sig, C, (size_t)y * w + x - 1);
            if (hb) b = side_at(K, gas, t0, kap, sig, C, (size_t)y * w + x);
            kx[f] = face_coef(K, ha ? &a : nullptr, hb ? &b : nullptr);
        } else {
            const size_t g = f - nx;
            int x, y;
            split_index(g, w, x, y);
            ha = y > 0;
            hb = y < h;
            if (ha) a = side_at(K, gas, t0, kap, sig, C, (size_t)(y - 1) * w + x);
            if (hb) b = side_at(K, gas, t0, kap, sig, C, (size_t)y * w + x);
            ky[g] = face_coef(K, ha ? &a : nullptr, hb ? &b : nullptr);
        }
    }
}

__global__ void heat_ksum_kernel(HeatConst K, const uint8_t* __restrict__ gas, const double* __restrict__ kx,
                                 const double* __restrict__ ky, double* ksum, double* kvac) {
    const int w = K.w, h = K.h;
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!gas[i]) {
            ksum[i] = 0.0;
            kvac[i] = 0.0;
            continue;
        }
        int x, y;
        split_index(i, w, x, y);
        const double k[4] = {kx[(size_t)y * (w + 1) + x], kx[(size_t)y * (w + 1) + x + 1], ky[(size_t)y * w + x],
                             ky[(size_t)(y + 1) * w + x]};
        const bool nb[4] = {x > 0 && gas[i - 1], x + 1 < w && gas[i + 1], y > 0 && gas[i - w],
                            y + 1 < h && gas[i + w]};
        double s = 0.0, v = 0.0;
        for (int f = 0; f < 4; f++) {
            s += k[f];
            if (!nb[f]) v += k[f];
        }
        ksum[i] = s;
        kvac[i] = v;
    }
}

// ---- a Newton pass's system at the iterate (heat.rs:476-489), kept as its mass term c = c_i + Σ_vac D_f (the
// diagonal less the couplings to gas neighbours, f64; FP32 copy as level 0's c) so that A x = c x + Σ D (x_i - x_j)
// is evaluated without cancellation; partials of the two measures' bounds, Σ c_i u² and Σ (C/Δt) T² (heat.rs:480-487).
__global__ void heat_system_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                   const double* __restrict__ C, const double* __restrict__ t,
                                   const double* __restrict__ u, const double* __restrict__ t0,
                                   const double* __restrict__ kvac, double* c64, double* rhs, float* c0, double* x,
                                   Red R) {
    const size_t n = (size_t)K.w * K.h;
    const double u_vac = u_of(K, K.t_floor);
    const double dt = scal[S_DT];
    double ub = 0.0, tb = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!gas[i]) {
            c64[i] = 1.0;
            rhs[i] = 0.0;
            c0[i] = 1.0f;
            x[i] = 0.0;
            continue;
        }
        const double heat = C[i] / dt;
        const double ci = heat * dt_du(K, t[i]);
        c64[i] = ci + kvac[i];
        rhs[i] = ci * u[i] - heat * (t[i] - t0[i]) + kvac[i] * u_vac;
        c0[i] = (float)(ci + kvac[i]);
        x[i] = u[i];
        ub += ci * u[i] * u[i];
        tb += heat * t[i] * t[i];
    }
    const double v[2] = {ub, tb};
    grid_sum_last<2>(v, R.part, R.counter, R.out);
}

// r = b - A x in FP64, A x = c x + Σ_gas D (x_i - x_j), with partials of <r, r>, <b, b> and the reference's two
// measures (heat.rs:413-447): rᵀD⁻¹r and the heat measure Σ (C/Δt)(r (dT/du) / D_ii)². Each thread takes ILP cells a
// grid stride apart and issues all of their loads before the arithmetic (the loads do not depend on the gas flags:
// the flags select afterwards), so a thread keeps several DRAM requests in flight.
constexpr int ILP = 4;

__global__ void heat_residual64_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                       const double* __restrict__ c64, const double* __restrict__ rhs,
                                       const double* __restrict__ kx, const double* __restrict__ ky,
                                       const double* __restrict__ C, const double* __restrict__ t,
                                       const double* __restrict__ x, double* __restrict__ r, Red R) {
    const int w = K.w, h = K.h;
    const size_t n = (size_t)w * h, stride = (size_t)gridDim.x * blockDim.x;
    const double dt = scal[S_DT];
    double rr = 0.0, bb = 0.0, gg = 0.0, hh = 0.0;
    for (size_t base = (size_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += 2 * stride) {
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const size_t i = base + u * stride;
            if (i >= n) break;
            int xx, y;
            split_index(i, w, xx, y);
            const bool gi = gas[i];
            const bool gl = xx > 0 && gas[i - 1], gr = xx + 1 < w && gas[i + 1];
            const bool gu = y > 0 && gas[i - w], gd = y + 1 < h && gas[i + w];
            const double xi = x[i], ci = c64[i], bi = rhs[i], Ci = C[i], ti = t[i];
            const double xl = xx > 0 ? x[i - 1] : 0.0, xr = xx + 1 < w ? x[i + 1] : 0.0;
            const double xu = y > 0 ? x[i - w] : 0.0, xd = y + 1 < h ? x[i + w] : 0.0;
            const double kl = kx[(size_t)y * (w + 1) + xx], kr = kx[(size_t)y * (w + 1) + xx + 1];
            const double ku = ky[(size_t)y * w + xx], kd = ky[(size_t)(y + 1) * w + xx];
            if (!gi) {
                r[i] = 0.0;
                continue;
            }
            double s = ci * xi, d = ci;
            if (gl) {
                s += kl * (xi - xl);
                d += kl;
            }
            if (gr) {
                s += kr * (xi - xr);
                d += kr;
            }
            if (gu) {
                s += ku * (xi - xu);
                d += ku;
            }
            if (gd) {
                s += kd * (xi - xd);
                d += kd;
            }
            const double ri = bi - s;
            r[i] = ri;
            rr += ri * ri;
            bb += bi * bi;
            gg += ri * ri / d;
            const double e = ri * dt_du(K, ti) / d;
            hh += Ci / dt * e * e;
        }
    }
    const double v[4] = {rr, bb, gg, hh};
    grid_sum_last<4>(v, R.part, R.counter, R.out);
}

__global__ void scale_kernel(size_t n, const double* __restrict__ r64, const double* __restrict__ scal, float* r32,
                             float* e32, Red R) {
    const double inv_scale = scal[S_ISCALE];
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = (float)(r64[i] * inv_scale);
        r32[i] = v;
        e32[i] = 0.0f;
        acc += (double)v * v;
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

// q = A p on level 0's FP32 operator in difference form, c p_i + Σ d (p_i - p_j); partials of <p, q>. ILP cells per
// thread, loads first (masked cells have c = 1 and no couplings; the mask selects afterwards).
__global__ void spmv_kernel(MgLevel L, const float* __restrict__ p, float* __restrict__ q, Red R) {
    const int w = L.w, h = L.h;
    const size_t n = (size_t)w * h, stride = (size_t)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (size_t base = (size_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += ILP * stride) {
        float pv[ILP], v[ILP];
#pragma unroll
        for (int u = 0; u < ILP; u++) {
            const size_t i = base + u * stride;
            pv[u] = 0.0f;
            v[u] = 0.0f;
            if (i < n) {
                int x, y;
                split_index(i, w, x, y);
                const float pi = p[i];
                const float pl = x > 0 ? p[i - 1] : pi, pr = x + 1 < w ? p[i + 1] : pi;
                const float pu = y > 0 ? p[i - w] : pi, pd = y + 1 < h ? p[i + w] : pi;
                const float dl = x > 0 ? L.dx[i - 1] : 0.0f, du = y > 0 ? L.dy[i - w] : 0.0f;
                const float dr = L.dx[i], dd = L.dy[i], c = L.c[i];
                const bool m = L.mask[i];
                float a = c * pi;
                a += dl * (pi - pl);
                a += dr * (pi - pr);
                a += du * (pi - pu);
                a += dd * (pi - pd);
                pv[u] = pi;
                v[u] = m ? a : 0.0f;
            }
        }
#pragma unroll
        for (int u = 0; u < ILP; u++) {
            const size_t i = base + u * stride;
            if (i < n) {
                q[i] = v[u];
                acc += (double)pv[u] * v[u];
            }
        }
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

// e += α p, r -= α q (α = <r,z>/<p,q> from the device scalars), partials of <r, r>.
__global__ void pcg_update_kernel(size_t n, const double* __restrict__ scal, int rz_slot, const float* __restrict__ p,
                                  const float* __restrict__ q, float* __restrict__ e, float* __restrict__ r, Red R) {
    const float alpha = (float)(scal[rz_slot] / scal[S_PQ]);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (size_t base = (size_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += ILP * stride) {
        float pv[ILP], qv[ILP], ev[ILP], rv[ILP];
#pragma unroll
        for (int u = 0; u < ILP; u++) {
            const size_t i = base + u * stride;
            if (i < n) {
                pv[u] = p[i];
                qv[u] = q[i];
                ev[u] = e[i];
                rv[u] = r[i];
            }
        }
#pragma unroll
        for (int u = 0; u < ILP; u++) {
            const size_t i = base + u * stride;
            if (i < n) {
                e[i] = ev[u] + alpha * pv[u];
                const float ri = rv[u] - alpha * qv[u];
                r[i] = ri;
                acc += (double)ri * ri;
            }
        }
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

// p = z + β p (β = <r,z>_new / <r,z>_old); the first direction (old slot < 0) is p = z.
__global__ void pcg_direction_kernel(size_t n, const double* __restrict__ scal, int old_slot, int new_slot,
                                     const float* __restrict__ z, float* __restrict__ p) {
    const float beta = old_slot < 0 ? 0.0f : (float)(scal[new_slot] / scal[old_slot]);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = (size_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += ILP * stride) {
        float zv[ILP], pv[ILP];
#pragma unroll
        for (int u = 0; u < ILP; u++) {
            const size_t i = base + u * stride;
            if (i < n) {
                zv[u] = z[i];
                pv[u] = old_slot < 0 ? 0.0f : p[i];
            }
        }
#pragma unroll
        for (int u = 0; u < ILP; u++) {
            const size_t i = base + u * stride;
            if (i < n) p[i] = old_slot < 0 ? zv[u] : zv[u] + beta * pv[u];
        }
    }
}

// The fused round head of (non-flexible) PCG: the search direction p_new = z + β p (β = <r,z>_cur / <r,z>_prev, or
// p_new = z while the S_BETA flag is 0: the first round) and q = A p_new in difference form, with partials of
// <p_new, q>; the last CTA sets the flag. Four consecutive cells of a row per thread with 16-byte loads (W is a
// multiple of 8); the neighbours' p_new are formed from their z and old p, so p_new goes to the other of the two
// direction buffers (S_PAR says which holds the old one).
__global__ void spmv_dir_kernel(MgLevel L, const double* __restrict__ scal, const float* __restrict__ z, float* pa,
                                float* pb, float* __restrict__ q, Red R, double* beta_flag) {
    const bool first = scal[S_BETA] == 0.0;  // p = z: the old direction is not read (it may hold anything)
    const float beta = first ? 0.0f : (float)(scal[S_RZC] / scal[S_RZP]);
    const bool par = scal[S_PAR] != 0.0;
    const float* __restrict__ p = par ? pb : pa;
    float* __restrict__ pnew = par ? pa : pb;
    const int w = L.w, h = L.h;
    const size_t n4 = (size_t)w * h / 4, stride = (size_t)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += stride) {
        const size_t i = 4 * t;
        int x, y;
        split_index(i, w, x, y);
        auto pn4 = [&](size_t j) {
            const float4 zz = *reinterpret_cast<const float4*>(z + j);
            if (first) return zz;
            const float4 pp = *reinterpret_cast<const float4*>(p + j);
            return make_float4(zz.x + beta * pp.x, zz.y + beta * pp.y, zz.z + beta * pp.z, zz.w + beta * pp.w);
        };
        auto pn1 = [&](size_t j) { return first ? z[j] : z[j] + beta * p[j]; };
        const float4 pc = pn4(i);
        const float4 pu = y > 0 ? pn4(i - w) : pc, pd = y + 1 < h ? pn4(i + w) : pc;
        const float pl = x > 0 ? pn1(i - 1) : pc.x;
        const float pr = x + 4 < w ? pn1(i + 4) : pc.w;
        const float4 c = *reinterpret_cast<const float4*>(L.c + i);
        const float4 dx = *reinterpret_cast<const float4*>(L.dx + i), dy = *reinterpret_cast<const float4*>(L.dy + i);
        const float dxl = x > 0 ? L.dx[i - 1] : 0.0f;
        const float4 dyu = y > 0 ? *reinterpret_cast<const float4*>(L.dy + i - w) : make_float4(0.f, 0.f, 0.f, 0.f);
        const uchar4 m = *reinterpret_cast<const uchar4*>(L.mask + i);
        const float P[6] = {pl, pc.x, pc.y, pc.z, pc.w, pr};
        const float U[4] = {pu.x, pu.y, pu.z, pu.w}, D[4] = {pd.x, pd.y, pd.z, pd.w};
        const float CC[4] = {c.x, c.y, c.z, c.w}, DXs[5] = {dxl, dx.x, dx.y, dx.z, dx.w};
        const float DYu[4] = {dyu.x, dyu.y, dyu.z, dyu.w}, DYd[4] = {dy.x, dy.y, dy.z, dy.w};
        const unsigned char M[4] = {m.x, m.y, m.z, m.w};
        float out[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float pi = P[k + 1];
            float a = CC[k] * pi;
            a += DXs[k] * (pi - P[k]);
            a += DXs[k + 1] * (pi - P[k + 2]);
            a += DYu[k] * (pi - U[k]);
            a += DYd[k] * (pi - D[k]);
            out[k] = M[k] ? a : 0.0f;
            acc += (double)pi * out[k];
        }
        *reinterpret_cast<float4*>(pnew + i) = pc;
        *reinterpret_cast<float4*>(q + i) = make_float4(out[0], out[1], out[2], out[3]);
    }
    // the last CTA raises the flag: every CTA read it before taking its ticket
    if (grid_sum_last1(acc, R.part, R.counter, R.out) && threadIdx.x == 0 && beta_flag) *beta_flag = 1.0;
}

// e += α p, r -= α q with 16-byte accesses (four cells per thread), p the round's new direction; partials of <r, r>.
__global__ void pcg_update4_kernel(size_t n, const double* __restrict__ scal, const float* pa, const float* pb,
                                   const float* __restrict__ q, float* __restrict__ e, float* __restrict__ r, Red R) {
    const float alpha = (float)(scal[S_RZC] / scal[S_PQ]);
    const float* __restrict__ p = scal[S_PAR] != 0.0 ? pa : pb;
    const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += stride) {
        const float4 pv = reinterpret_cast<const float4*>(p)[t], qv = reinterpret_cast<const float4*>(q)[t];
        float4 ev = reinterpret_cast<float4*>(e)[t], rv = reinterpret_cast<float4*>(r)[t];
        ev.x += alpha * pv.x; ev.y += alpha * pv.y; ev.z += alpha * pv.z; ev.w += alpha * pv.w;
        rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z; rv.w -= alpha * qv.w;
        reinterpret_cast<float4*>(e)[t] = ev;
        reinterpret_cast<float4*>(r)[t] = rv;
        acc += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

// Flexible CG (the learned preconditioner is not a fixed linear operator): the update keeps the residual it replaces,
// <z, r_old> is formed after the preconditioner, and β = (<z, r> - <z, r_old>) / <z_old, r_old> (Polak-Ribière).
__global__ void pcg_update_flex_kernel(size_t n, const double* __restrict__ scal, int rz_slot,
                                       const float* __restrict__ p, const float* __restrict__ q, float* e, float* r,
                                       float* r_old, Red R) {
    const float alpha = (float)(scal[rz_slot] / scal[S_PQ]);
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        e[i] += alpha * p[i];
        const float ro = r[i];
        const float ri = ro - alpha * q[i];
        r_old[i] = ro;
        r[i] = ri;
        acc += (double)ri * ri;
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

__global__ void dot_kernel(size_t n, const float* __restrict__ a, const float* __restrict__ b, Red R) {
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        acc += (double)a[i] * b[i];
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

__global__ void pcg_direction_flex_kernel(size_t n, const double* __restrict__ scal, int old_slot, int new_slot,
                                          const float* __restrict__ z, float* p) {
    const float beta = (float)((scal[new_slot] - scal[S_ZRO]) / scal[old_slot]);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// The residual a V-cycle leaves, r1 = r − A z (gas cells; 0 elsewhere), and optionally ez = e + z.
__global__ void vcycle_residual_kernel(MgLevel L, const float* __restrict__ r, const float* __restrict__ z,
                                       const float* __restrict__ e, float* r1, float* ez) {
    const int w = L.w, h = L.h;
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y;
        split_index(i, w, x, y);
        float v = 0.0f;
        const float zi = z[i];
        if (L.mask[i]) {
            float az = L.c[i] * zi;
            if (x > 0) az += L.dx[i - 1] * (zi - z[i - 1]);
            if (x + 1 < w) az += L.dx[i] * (zi - z[i + 1]);
            if (y > 0) az += L.dy[i - w] * (zi - z[i - w]);
            if (y + 1 < h) az += L.dy[i] * (zi - z[i + w]);
            v = r[i] - az;
        }
        r1[i] = v;
        if (ez) ez[i] = e[i] + zi;
    }
}

// z = r / diag (Jacobi), partials of <r, z>.
__global__ void jacobi_kernel(MgLevel L, const float* __restrict__ r, float* z, Red R) {
    const int w = L.w, h = L.h;
    const size_t n = (size_t)w * h;
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y;
        split_index(i, w, x, y);
        const float dl = x > 0 ? L.dx[i - 1] : 0.0f, du = y > 0 ? L.dy[i - w] : 0.0f;
        const float zi = L.mask[i] ? r[i] / (L.c[i] + dl + L.dx[i] + du + L.dy[i]) : 0.0f;
        z[i] = zi;
        acc += (double)r[i] * zi;
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

// z += v, and <r, z>.
__global__ void add_dot_kernel(size_t n, const float* __restrict__ r, const float* __restrict__ v, float* z, Red R) {
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float zi = z[i] + v[i];
        z[i] = zi;
        acc += (double)r[i] * zi;
    }
    grid_sum_last1(acc, R.part, R.counter, R.out);
}

__global__ void correction_kernel(size_t n, const uint8_t* __restrict__ gas, const float* __restrict__ e,
                                  const double* __restrict__ scal, double* x) {
    const double scale = scal[S_SCALE];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (gas[i]) x[i] += scale * (double)e[i];
}

// The pass's update (heat.rs:494-509: u >= u_vac, T within a factor 2) and the next pass's system at the new iterate
// (as heat_system_kernel builds it) in one sweep over the cells; partials of Σ C|ΔT|, the cells moved by more than
// newton_cell of their T, Σ c_i u² and Σ (C/Δt) T² (four consecutive slots from S_MOVED). When the passes end here
// the system goes unused.
__global__ void newton_system_kernel(HeatConst K, double cell_tol, const double* __restrict__ scal,
                                     const uint8_t* __restrict__ gas,
                                     const double* __restrict__ C, const double* __restrict__ t0,
                                     const double* __restrict__ kvac, double* t, double* u, double* x, double* c64,
                                     double* rhs, float* c0, Red R) {
    const size_t n = (size_t)K.w * K.h, stride = (size_t)gridDim.x * blockDim.x;
    const double u_vac = u_of(K, K.t_floor);
    const double dt = scal[S_DT];
    double moved = 0.0, viol = 0.0, ub = 0.0, tb = 0.0;
    // two cells a grid stride apart per iteration, all loads issued before the arithmetic
    for (size_t base = (size_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += 2 * stride) {
        const size_t i2 = base + stride;
        const bool g1 = gas[base], g2 = i2 < n && gas[i2];
        double tv[2], xv[2], Cv[2], t0v[2], kv[2];
        tv[0] = t[base];
        xv[0] = x[base];
        Cv[0] = C[base];
        t0v[0] = t0[base];
        kv[0] = kvac[base];
        if (i2 < n) {
            tv[1] = t[i2];
            xv[1] = x[i2];
            Cv[1] = C[i2];
            t0v[1] = t0[i2];
            kv[1] = kvac[i2];
        }
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const size_t i = e ? i2 : base;
            if (!(e ? g2 : g1)) continue;  // the system's masked rows (c = 1, b = 0, x = 0) are already in place
            const double ti = tv[e];
            double nx = t_of(K, fmax(xv[e], u_vac));
            nx = fmin(fmax(nx, 0.5 * ti), 2.0 * ti);
            const double d = fabs(nx - ti);
            moved += Cv[e] * d;
            if (!(d <= cell_tol * ti)) viol += 1.0;
            const double un = u_of(K, nx);
            t[i] = nx;
            u[i] = un;
            const double heat = Cv[e] / dt;
            const double ci = heat * dt_du(K, nx);
            c64[i] = ci + kv[e];
            rhs[i] = ci * un - heat * (nx - t0v[e]) + kv[e] * u_vac;
            c0[i] = (float)(ci + kv[e]);
            x[i] = un;
            ub += ci * un * un;
            tb += heat * nx * nx;
        }
    }
    const double v[4] = {moved, viol, ub, tb};
    grid_sum_last<4>(v, R.part, R.counter, R.out);
}

// F = -k (v_b - v_a) at every face (heat.rs:338-361), v = u on gas cells, u_vac elsewhere; FP32 out.
__device__ __forceinline__ double face_flux(const HeatConst& K, const uint8_t* gas, const double* u, double k,
                                            long a, long b, double u_vac) {
    if (k == 0.0) return 0.0;
    const double va = (a >= 0 && gas[a]) ? u[a] : u_vac;
    const double vb = (b >= 0 && gas[b]) ? u[b] : u_vac;
    return -k * (vb - va);
}

__global__ void heat_flux_kernel(HeatConst K, const uint8_t* __restrict__ gas, const double* __restrict__ kx,
                                 const double* __restrict__ ky, const double* __restrict__ u,
                                 const double* __restrict__ scale, float* fx, float* fy) {
    const int w = K.w, h = K.h;
    const size_t nx = (size_t)(w + 1) * h, ny = (size_t)w * (h + 1);
    const double u_vac = u_of(K, K.t_floor);
    for (size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x; f < nx + ny; f += (size_t)gridDim.x * blockDim.x) {
        long a, b;
        double k;
        if (f < nx) {
            int x, y;
            split_index(f, (w + 1), x, y);
            a = x > 0 ? (long)y * w + x - 1 : -1;
            b = x < w ? (long)y * w + x : -1;
            k = kx[f];
        } else {
            const size_t g = f - nx;
            int x, y;
            split_index(g, w, x, y);
            a = y > 0 ? (long)(y - 1) * w + x : -1;
            b = y < h ? (long)y * w + x : -1;
            k = ky[g];
        }
        double F = face_flux(K, gas, u, k, a, b, u_vac);
        if (scale) {
            const long from = F > 0.0 ? a : b;
            F *= from >= 0 ? scale[from] : 1.0;
        }
        if (f < nx) fx[f] = (float)F;
        else fy[f - nx] = (float)F;
    }
}

// The commit's sums (heat.rs:521-531): radiated, gained and held.
__global__ void commit_sums_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                   const double* __restrict__ C, const double* __restrict__ t,
                                   const double* __restrict__ t0, const double* __restrict__ u,
                                   const double* __restrict__ kvac, Red R) {
    const size_t n = (size_t)K.w * K.h;
    const double u_vac = u_of(K, K.t_floor);
    const double dt = scal[S_DT];
    double rad = 0.0, gain = 0.0, held = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!gas[i]) continue;
        rad += dt * kvac[i] * (u[i] - u_vac);
        gain += C[i] * (t[i] - t0[i]);
        held += C[i] * t[i];
    }
    const double v[3] = {rad, gain, held};
    grid_sum_last<3>(v, R.part, R.counter, R.out);
}

// E_i += C_i ((1 + δ) T_i - T_i⁰) (heat.rs:532-535), and the cell's rate (T - T⁰)/Δt kept for the next step's first
// iterate (heat.wgsl:1139-1155).
__global__ void commit_apply_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                    const double* __restrict__ C, const double* __restrict__ t,
                                    const double* __restrict__ t0, float* U, double* rate) {
    const size_t n = (size_t)K.w * K.h;
    const double delta = scal[S_DELTA], dt = scal[S_DT];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (gas[i]) U[3 * n + i] = (float)((double)U[3 * n + i] + C[i] * ((1.0 + delta) * t[i] - t0[i]));
        rate[i] = gas[i] ? (t[i] - t0[i]) / dt : 0.0;
    }
}

// The first iterate on the V-cycle (heat.wgsl:710-722): T⁰ + the last step's rate × Δt, T⁰ where that is off by more
// than a factor 2 or not finite, floored at T_floor.
__global__ void warm_start_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                  const double* __restrict__ t0, const double* __restrict__ rate, double* t, double* u) {
    const size_t n = (size_t)K.w * K.h;
    const double dt = scal[S_DT];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!gas[i]) continue;
        double tg = t0[i] + rate[i] * dt;
        if (!(tg >= 0.5 * t0[i] && tg <= 2.0 * t0[i])) tg = t0[i];
        tg = fmax(tg, K.t_floor);
        t[i] = tg;
        u[i] = u_of(K, tg);
    }
}

// Past the ceiling (heat.rs:545-564): each gas cell's outflow scaled to the heat it holds above its floor.
__global__ void limited_scale_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                     const double* __restrict__ kx, const double* __restrict__ ky,
                                     const double* __restrict__ u, const double* __restrict__ C,
                                     const double* __restrict__ t0, double* scale) {
    const int w = K.w, h = K.h;
    const size_t n = (size_t)w * h;
    const double u_vac = u_of(K, K.t_floor);
    const double dt = scal[S_DT];
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!gas[i]) {
            scale[i] = 1.0;
            continue;
        }
        int x, y;
        split_index(i, w, x, y);
        const long L = x > 0 ? (long)i - 1 : -1, R = x + 1 < w ? (long)i + 1 : -1;
        const long Uu = y > 0 ? (long)i - w : -1, D = y + 1 < h ? (long)i + w : -1;
        const double lv[4] = {-face_flux(K, gas, u, kx[(size_t)y * (w + 1) + x], L, (long)i, u_vac),
                              face_flux(K, gas, u, kx[(size_t)y * (w + 1) + x + 1], (long)i, R, u_vac),
                              -face_flux(K, gas, u, ky[(size_t)y * w + x], Uu, (long)i, u_vac),
                              face_flux(K, gas, u, ky[(size_t)(y + 1) * w + x], (long)i, D, u_vac)};
        double out = 0.0;
        for (int f = 0; f < 4; f++) out += fmax(lv[f], 0.0);
        out *= dt;
        const double held = C[i] * fmax(t0[i] - K.t_floor, 0.0);
        scale[i] = out > held ? held / out : 1.0;
    }
}

// E -= Δt Σ_f F_f with every face's F at the scale of the cell it leaves (heat.rs:565-592); partials of radiated.
__global__ void limited_apply_kernel(HeatConst K, const double* __restrict__ scal, const uint8_t* __restrict__ gas,
                                     const double* __restrict__ kx, const double* __restrict__ ky,
                                     const double* __restrict__ u, const double* __restrict__ scale, float* U,
                                     Red R) {
    const int w = K.w, h = K.h;
    const size_t n = (size_t)w * h;
    const double u_vac = u_of(K, K.t_floor);
    const double dt = scal[S_DT];
    double rad = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!gas[i]) continue;
        int x, y;
        split_index(i, w, x, y);
        const long nb[4] = {x > 0 ? (long)i - 1 : -1, x + 1 < w ? (long)i + 1 : -1, y > 0 ? (long)i - w : -1,
                            y + 1 < h ? (long)i + w : -1};
        double F[4] = {face_flux(K, gas, u, kx[(size_t)y * (w + 1) + x], nb[0], (long)i, u_vac),
                       face_flux(K, gas, u, kx[(size_t)y * (w + 1) + x + 1], (long)i, nb[1], u_vac),
                       face_flux(K, gas, u, ky[(size_t)y * w + x], nb[2], (long)i, u_vac),
                       face_flux(K, gas, u, ky[(size_t)(y + 1) * w + x], (long)i, nb[3], u_vac)};
        // the low cell of faces 0 and 2 is the neighbour, of faces 1 and 3 this cell
        const long low[4] = {nb[0], (long)i, nb[2], (long)i}, high[4] = {(long)i, nb[1], (long)i, nb[3]};
        double out[4];
        for (int f = 0; f < 4; f++) {
            const long from = F[f] > 0.0 ? low[f] : high[f];
            F[f] *= from >= 0 ? scale[from] : 1.0;
        }
        out[0] = -F[0];
        out[1] = F[1];
        out[2] = -F[2];
        out[3] = F[3];
        for (int f = 0; f < 4; f++)
            if (!(nb[f] >= 0 && gas[nb[f]])) rad += dt * out[f];
        U[3 * n + i] = (float)((double)U[3 * n + i] - dt * (((out[0] + out[1]) + out[2]) + out[3]));
    }
    grid_sum_last1(rad, R.part, R.counter, R.out);
}

__global__ void zero_kernel(double* a, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) a[i] = 0.0;
}

__global__ void f64_to_f32_kernel(float* dst, const double* __restrict__ src, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

__global__ void f32_to_f64_kernel(double* dst, const float* __restrict__ src, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

// One device scalar set by the host's launch (a value captured at launch time, so no staging buffer is reused).
__global__ void set_scalar_kernel(double* scal, int slot, double value) {
    if (threadIdx.x == 0 && blockIdx.x == 0) scal[slot] = value;
}

// A fused PCG solve's start, after its first preconditioner application: that <r, z> is the current one, the first
// direction is z, the direction buffers start at pa.
__global__ void pcg_start_kernel(double* scal) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    scal[S_RZC] = scal[S_RZN];
    scal[S_BETA] = 0.0;
    scal[S_PAR] = 0.0;
}

// A fused PCG round's end: the new <r, z> becomes the current one and the new direction buffer the old.
__global__ void pcg_rotate_kernel(double* scal) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    scal[S_RZP] = scal[S_RZC];
    scal[S_RZC] = scal[S_RZN];
    scal[S_PAR] = scal[S_PAR] != 0.0 ? 0.0 : 1.0;
}

// ---- the implicit step under device control (MG and Jacobi preconditioners)
//
// The host-driven step (heat_step's Newton loop, solve_pass's FP64 refinement, inner_pcg's rounds) decides from
// read-back scalars. Here the same decisions are taken by one-thread controller kernels that run between the step's
// kernels inside one captured CUDA graph and steer its conditional nodes: an IF around the step (no gas, pinned
// temperature or Δt <= 0 leave only the fluxes), a WHILE over the Newton passes, a WHILE over a pass's refinements, an
// IF around each inner solve, a WHILE over its PCG rounds (the residual tested after every round: no host round trip,
// no predicted cadence), an IF around the next pass's coarsening, and IFs choosing the commit. No launch argument
// changes from step to step: Δt, the scale, δ and the round state live in the device scalars.
struct HeatCtl {
    // configuration (host-written)
    double tol, nheat, ncell, inner_floor;
    int max_passes, max_rounds, pin;
    // the step
    double heat0, n_gas;
    int passes, rounds, refinements, converged, ok, skipped;
    double pass_tol, moved_prev, rel;
    // the pass's refinement and its inner solve
    int ref, reached, it, max_it;
    double prev, eta, rr0;
    // the commit
    double delta, radiated;
    // how often each body ran since the host last counted (for the launch count)
    unsigned long long runs[10];
};
enum CtlBody { B_MAIN, B_SKIP, B_PASS, B_REFINE, B_INNER, B_ROUND, B_NSYS, B_COARSEN, B_CONV, B_LIM, B_COUNT };

struct CtlHandles {
    cudaGraphConditionalHandle h[B_COUNT];
};

enum CtlPhase { C_BEGIN, C_NEWTON_BEGIN, C_PASS_BEGIN, C_REFINE, C_INNER_BEGIN, C_ROUND, C_AFTER_INNER, C_PASS_END,
                C_NEWTON, C_COMMIT, C_DELTA, C_LIMITED };

__device__ __forceinline__ void ctl_set(const CtlHandles& hd, HeatCtl* c, int body, bool on, bool count_entry) {
    cudaGraphSetConditional(hd.h[body], on ? 1u : 0u);
    if (on && count_entry) c->runs[body]++;
}

__global__ void heat_ctl_kernel(HeatCtl* c, double* scal, int phase, CtlHandles hd) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    switch (phase) {
        case C_BEGIN: {  // after the set-up: Σ C T⁰, the gas cells and Δt in the scalars
            c->heat0 = scal[S_HEAT0];
            c->n_gas = scal[S_NGAS];
            const bool skip = c->pin || c->n_gas == 0.0 || !(scal[S_DT] > 0.0);
            c->skipped = skip;
            c->passes = c->rounds = c->refinements = 0;
            c->converged = skip ? 1 : 0;
            c->ok = 1;
            c->rel = c->delta = c->radiated = 0.0;
            ctl_set(hd, c, B_MAIN, !skip, true);
            ctl_set(hd, c, B_SKIP, skip, true);
            break;
        }
        case C_NEWTON_BEGIN:  // after the first system (its two bounds in S_UB, S_TB)
            c->pass_tol = fmax(c->tol, kFirstPassTol);
            c->moved_prev = 0.0;
            ctl_set(hd, c, B_PASS, c->max_passes > 0 && c->max_rounds > 0, false);
            break;
        case C_PASS_BEGIN:
            c->runs[B_PASS]++;
            c->passes++;
            c->ref = 0;
            c->prev = INFINITY;
            ctl_set(hd, c, B_REFINE, true, false);
            break;
        case C_REFINE: {  // after the FP64 residual: stop, or scale the residual for an inner solve
            c->runs[B_REFINE]++;
            const double rr = scal[S_RR], bb = scal[S_BB], gam = scal[S_GAM], hm = scal[S_HM];
            bool go = false;
            if (!isfinite(rr) || !isfinite(bb) || !isfinite(gam) || !isfinite(hm)) {
                c->ok = 0;
            } else {
                c->rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
                const double tol = c->pass_tol, ub = scal[S_UB], tb = scal[S_TB];
                double worst = c->rel / tol;
                if (ub > 0.0) worst = fmax(worst, sqrt(gam / ub) / tol);
                if (tb > 0.0) worst = fmax(worst, sqrt(hm / tb) / tol);
                if (!(worst <= 1.0 || rr == 0.0) && !(worst > 0.5 * c->prev) && c->rounds < c->max_rounds) {
                    c->prev = worst;
                    const double scale = sqrt(rr / fmax(1.0, c->n_gas));
                    scal[S_SCALE] = scale;
                    scal[S_ISCALE] = 1.0 / scale;
                    c->eta = fmin(0.5, fmax(c->inner_floor, 0.5 / worst));
                    c->max_it = c->max_rounds - c->rounds;
                    go = true;
                }
            }
            ctl_set(hd, c, B_INNER, go, true);
            if (!go) ctl_set(hd, c, B_REFINE, false, false);
            break;
        }
        case C_INNER_BEGIN: {  // after the scaled residual and its first preconditioner application
            scal[S_RZC] = scal[S_RZN];
            scal[S_BETA] = 0.0;
            scal[S_PAR] = 0.0;
            c->rr0 = scal[S_R32];
            c->it = 0;
            c->reached = 0;
            ctl_set(hd, c, B_ROUND, c->rr0 > 0.0 && c->max_it > 0, false);
            break;
        }
        case C_ROUND: {  // after a round: rotate its state, test the residual
            c->runs[B_ROUND]++;
            c->it++;
            scal[S_RZP] = scal[S_RZC];
            scal[S_RZC] = scal[S_RZN];
            scal[S_PAR] = scal[S_PAR] != 0.0 ? 0.0 : 1.0;
            const double pq = scal[S_PQ], rr = scal[S_RRI];
            bool more = true;
            if (!(pq > 0.0) || !isfinite(pq) || !isfinite(rr)) {
                c->ok = 0;  // a breakdown: the solve's correction is dropped
                scal[S_SCALE] = 0.0;
                more = false;
            } else if (rr <= c->eta * c->eta * c->rr0) {
                c->reached = 1;
                more = false;
            } else if (c->it >= c->max_it) {
                more = false;
            }
            ctl_set(hd, c, B_ROUND, more, false);
            break;
        }
        case C_AFTER_INNER: {  // after the correction x += scale e
            bool more = c->ok != 0;
            if (c->ok) {
                c->rounds += c->it;
                c->refinements++;
                // an intermediate pass (its tolerance far above the FP32 solve's floor) trusts the solve that reached
                // its reduction; the final pass is always verified by another FP64 residual
                if (c->reached && c->pass_tol >= kTrustedPassTol) {
                    c->rel *= c->eta;
                    more = false;
                }
            }
            if (++c->ref >= kMaxRefinements) more = false;
            ctl_set(hd, c, B_REFINE, more, false);
            break;
        }
        case C_PASS_END:  // the pass's solve is done: its Newton update, unless the solve broke down
            ctl_set(hd, c, B_NSYS, c->ok != 0, true);
            if (!c->ok) ctl_set(hd, c, B_PASS, false, false);
            break;
        case C_NEWTON: {  // after the update and the next system: stop, or the next pass's tolerance and coarsening
            const double rel_moved = c->heat0 > 0.0 ? scal[S_MOVED] / c->heat0 : 0.0;
            bool more;
            if (rel_moved <= c->nheat && scal[S_VIOL] == 0.0 && c->pass_tol <= c->tol) {
                c->converged = 1;
                more = false;
            } else {
                // the next pass is solved to tol once it is expected to move less than nheat (the passes' observed
                // contraction times this pass's move), since only a pass solved to tol can end them
                const double ratio = c->moved_prev > 0.0 ? fmin(1.0, fmax(0.01, rel_moved / c->moved_prev)) : 0.1;
                c->moved_prev = rel_moved;
                c->pass_tol = fmax(c->tol, fmin(kFirstPassTol, rel_moved));
                if (ratio * rel_moved <= c->nheat) c->pass_tol = c->tol;
                more = c->passes < c->max_passes && c->rounds < c->max_rounds;
            }
            ctl_set(hd, c, B_COARSEN, more, true);
            ctl_set(hd, c, B_PASS, more, false);
            break;
        }
        case C_COMMIT:
            ctl_set(hd, c, B_CONV, c->converged != 0, true);
            ctl_set(hd, c, B_LIM, !c->converged, true);
            break;
        case C_DELTA: {  // after the commit's sums (heat.rs:521-531)
            const double rad = scal[S_RAD], gain = scal[S_GAIN], held = scal[S_HELD];
            c->delta = -(gain + rad) / held;
            c->radiated = rad;
            scal[S_DELTA] = c->delta;
            break;
        }
        case C_LIMITED:
            c->radiated = scal[S_RAD];
            break;
    }
}

int grid_for(size_t n) {
    size_t b = (n + RED_THREADS - 1) / RED_THREADS;
    return (int)(b < 1 ? 1 : (b > (size_t)MAX_PART ? (size_t)MAX_PART : b));
}

}  // namespace

struct RoundGraph {
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;  // kernel nodes in the graph
};

struct HeatSolver {
    sr_config cfg{};
    HeatConst K{};
    HeatRef ref{};
    int w = 0, h = 0;
    size_t n = 0;
    int grid = 0;
    uint32_t precond = SR_PRECOND_MG;
    uint32_t max_passes = 128, max_rounds = 4096;
    double inner_floor = 1e-5;  // the smallest residual reduction asked of one inner FP32 solve
    bool use_graphs = true;
    uint8_t* gas = nullptr;
    double *t0 = nullptr, *C = nullptr, *t = nullptr, *u = nullptr, *kx = nullptr, *ky = nullptr;
    double *ksum = nullptr, *kvac = nullptr, *c64 = nullptr, *rhs = nullptr, *x = nullptr, *r64 = nullptr;
    double* lscale = nullptr;
    double* rate = nullptr;      // each cell's P5 rate (T - T⁰)/Δt in the last step, for the next first iterate
    float *kap = nullptr, *sig = nullptr;
    float *r32 = nullptr, *e32 = nullptr, *p32 = nullptr, *q32 = nullptr, *z32 = nullptr;
    float* p2 = nullptr;  // the fused rounds' second direction buffer (rounds alternate p32 -> p2 -> p32)
    float *fx = nullptr, *fy = nullptr;
    double* part = nullptr;      // grid-sum partials: 4 x PART_CAP
    unsigned* counter = nullptr;  // grid-sum ticket
    double* scal = nullptr;       // S_COUNT device scalars
    double* hscal = nullptr;      // pinned host copy
    Multigrid mg;
    int n_gas = 0;
    RoundGraph graphs[3][2];      // one PCG round per preconditioner and <r,z> slot parity
    Learner* learner = nullptr;   // the learned preconditioner, when attached
    LearnedApply* lapply = nullptr;
    float* r_old = nullptr;       // flexible CG's previous residual
    float* ez = nullptr;          // sample collection: the iterate after each round's V-cycle
    float* vz = nullptr;          // the learned preconditioner's second V-cycle
    void* flush = nullptr;        // timing hook: a buffer larger than L2
    // the device-controlled step: its control block, the captured graphs (one per state buffer the step updates),
    // the extra streams its nested bodies are captured on, and each body's kernel count
    HeatCtl* ctl = nullptr;
    HeatCtl* hctl = nullptr;      // pinned host copy
    std::map<const float*, cudaGraphExec_t> step_graphs;
    cudaStream_t cap[6] = {};
    long long body_launches[B_COUNT + 1] = {};  // [B_COUNT]: the graph's own top-level kernels
    bool report_pending = false;  // the last step ran as a graph: its report is in ctl
    cudaStream_t stream = nullptr;  // the owning context's stream
    sr_heat_report report{};

    Red red(int slot) { return Red{part, counter, scal + slot}; }

    // Reads device scalars [first, first + count) into hscal (synchronises the stream).
    void read(int first, int count, cudaStream_t s) {
        SR_CUDA_TRY(cudaMemcpyAsync(hscal + first, scal + first, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
        SR_CUDA_TRY(cudaStreamSynchronize(s));
    }
};

namespace {

void set_scalar(HeatSolver* H, int slot, double value, cudaStream_t s) {
    set_scalar_kernel<<<1, 32, 0, s>>>(H->scal, slot, value);
    sr_note_launch();
}

void setup_step(HeatSolver* H, const float* U, const float* kappa, cudaStream_t s) {
    const HeatConst& K = H->K;
    heat_cells_kernel<<<H->grid, RED_THREADS, 0, s>>>(K, H->ref, U, kappa, H->gas, H->t0, H->C, H->kap, H->sig, H->t, H->u,
                                                      H->red(S_HEAT0));
    sr_note_launch();
    const size_t nf = (size_t)(H->w + 1) * H->h + (size_t)H->w * (H->h + 1);
    heat_faces_kernel<<<grid_for(nf), RED_THREADS, 0, s>>>(K, H->gas, H->t0, H->kap, H->sig, H->C, H->kx, H->ky);
    sr_note_launch();
    heat_ksum_kernel<<<H->grid, RED_THREADS, 0, s>>>(K, H->gas, H->kx, H->ky, H->ksum, H->kvac);
    sr_note_launch();
    H->mg.set_couplings(H->kx, H->ky, H->gas, s);
}

// z = M r, and <r, z> into scalar `rz_slot`.
void precondition(HeatSolver* H, uint32_t precond, int rz_slot, cudaStream_t s) {
    if (precond == SR_PRECOND_JACOBI) {
        jacobi_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->mg.L[0], H->r32, H->z32, H->red(rz_slot));
        sr_note_launch();
    } else if (precond == SR_PRECOND_LEARNED) {
        // V-cycle, network, V-cycle: z1 = M r; z2 = z1 + N(r − A z1); z = z2 + M (r − A z2). The network predicts the
        // smooth error the first cycle leaves; the second cycle removes the rounding noise of its BF16 output (high
        // frequencies, which the smoothers take out) and what remains of the smooth error.
        const MgLevel& L0 = H->mg.L[0];
        H->mg.apply(H->r32, H->z32, H->part, H->counter, H->scal + S_MGRZ, s);
        vcycle_residual_kernel<<<H->grid, RED_THREADS, 0, s>>>(L0, H->r32, H->z32, nullptr, H->q32, nullptr);
        sr_note_launch();
        learned_apply(H->lapply, L0, H->q32, H->z32, H->r32, H->z32, H->part, H->counter, H->scal + S_MGRZ, s);
        vcycle_residual_kernel<<<H->grid, RED_THREADS, 0, s>>>(L0, H->r32, H->z32, nullptr, H->q32, nullptr);
        sr_note_launch();
        H->mg.apply(H->q32, H->vz, H->part, H->counter, H->scal + S_MGRZ, s);
        add_dot_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->r32, H->vz, H->z32, H->red(rz_slot));
        sr_note_launch();
    } else {
        H->mg.apply(H->r32, H->z32, H->part, H->counter, H->scal + rz_slot, s);
    }
}

// One PCG round: q = A p, α, e += α p, r -= α q, z = M r, β, p = z + β p. `parity` picks the <r,z> slots.
void round_launches(HeatSolver* H, uint32_t precond, int parity, cudaStream_t s) {
    const int rz_old = parity ? S_RZ1 : S_RZ0, rz_new = parity ? S_RZ0 : S_RZ1;
    if (precond == SR_PRECOND_LEARNED) {
        spmv_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->mg.L[0], H->p32, H->q32, H->red(S_PQ));
        sr_note_launch();
        pcg_update_flex_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, rz_old, H->p32, H->q32, H->e32, H->r32,
                                                               H->r_old, H->red(S_RRI));
        sr_note_launch();
        precondition(H, precond, rz_new, s);
        dot_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->z32, H->r_old, H->red(S_ZRO));
        sr_note_launch();
        pcg_direction_flex_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, rz_old, rz_new, H->z32, H->p32);
        sr_note_launch();
        return;
    }
    // the fused round: the state (<r, z> slots, which direction buffer is current) lives in the device scalars, so
    // one captured graph serves every round
    (void)rz_old;
    (void)rz_new;
    spmv_dir_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->mg.L[0], H->scal, H->z32, H->p32, H->p2, H->q32,
                                                    H->red(S_PQ), H->scal + S_BETA);
    sr_note_launch();
    pcg_update4_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, H->p32, H->p2, H->q32, H->e32, H->r32,
                                                       H->red(S_RRI));
    sr_note_launch();
    precondition(H, precond, S_RZN, s);
    pcg_rotate_kernel<<<1, 32, 0, s>>>(H->scal);
    sr_note_launch();
}

// A round as one CUDA graph launch (captured once per preconditioner and parity; every pointer it reads is fixed).
void run_round(HeatSolver* H, uint32_t precond, int parity, cudaStream_t s) {
    if (!H->use_graphs) {
        round_launches(H, precond, parity, s);
        return;
    }
    RoundGraph& g = H->graphs[precond][precond == SR_PRECOND_LEARNED ? parity : 0];
    if (!g.exec) {
        const long long before = (long long)sr_launches();
        cudaGraph_t graph;
        SR_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        round_launches(H, precond, parity, s);
        SR_CUDA_TRY(cudaStreamEndCapture(s, &graph));
        cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        SR_CUDA_TRY(e);
        g.launches = (long long)sr_launches() - before;
        sr_note_launches(-g.launches);  // captured, not launched
    }
    SR_CUDA_TRY(cudaGraphLaunch(g.exec, s));
    sr_note_launches(g.launches);
}

struct SolveResult {
    int rounds = 0;
    int refinements = 0;
    double rel = 0.0;
    bool ok = true;
    bool fallback = false;  // the learned preconditioner stalled and MG-PCG finished
};

constexpr int kStallRounds = 24;  // learned: rounds after which a solve that has not gained 100x falls back

// PCG on A32 e = r32 from e = 0 to a residual reduction `eta` or `max_it` rounds. Returns the rounds, -1 on a
// breakdown (a non-positive or non-finite curvature), or with the learned preconditioner -2 - rounds when it stalls
// (a breakdown, or less than a 100x reduction after kStallRounds): plain MG-PCG then takes over.
int inner_pcg(HeatSolver* H, uint32_t precond, double eta, int max_it, cudaStream_t s, bool* reached = nullptr) {
    if (reached) *reached = false;
    if (precond == SR_PRECOND_LEARNED) {  // flexible CG forms its direction at the end of a round
        precondition(H, precond, S_RZ0, s);
        pcg_direction_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, -1, S_RZ0, H->z32, H->p32);
        sr_note_launch();
    } else {  // the first round's fused direction is p = z
        precondition(H, precond, S_RZN, s);
        pcg_start_kernel<<<1, 32, 0, s>>>(H->scal);
        sr_note_launch();
    }
    H->read(S_R32, 1, s);  // <r, r> of the scaled residual (written by scale_kernel)
    const double rr0 = H->hscal[S_R32];
    if (!(rr0 > 0.0)) return 0;
    int it = 0;
    int next_check = 1;
    while (it < max_it) {
        run_round(H, precond, it & 1, s);
        it++;
        if (it == next_check || it == max_it) {
            H->read(S_PQ, 2, s);  // S_PQ, S_RRI
            const double pq = H->hscal[S_PQ], rr = H->hscal[S_RRI];
            if (!(pq > 0.0) || !isfinite(pq) || !isfinite(rr)) return precond == SR_PRECOND_LEARNED ? -2 - it : -1;
            if (rr <= eta * eta * rr0) {
                if (reached) *reached = true;
                break;
            }
            if (precond == SR_PRECOND_LEARNED && it >= kStallRounds && rr > 1e-4 * rr0) return -2 - it;
            // after the first three rounds, the next check one round before the rate seen so far (the geometric mean
            // per round) reaches the target: each check costs a host round trip, each round past convergence a V-cycle
            int more = 1;
            const double ratio = pow(rr / rr0, 1.0 / it);
            if (ratio > 0.0 && ratio < 1.0) more = (int)ceil(log(eta * eta * rr0 / rr) / log(ratio)) - 1;
            next_check = it < 3 ? it + 1 : it + std::max(1, std::min(more, 8));
        }
    }
    return it;
}

// The pass's system by FP64 refinement around FP32 PCG, x starting at the iterate, until the plain relative residual
// ||b - A x|| / ||b|| and the reference's two measures (rᵀD⁻¹r against Σ c_i u², the heat measure against
// Σ (C/Δt) T², heat.rs:480-487 and 422-431) are all within `tol`; stops early when a refinement no longer halves the
// worst of the three ratios, or past `max_rounds`.
SolveResult solve_pass(HeatSolver* H, uint32_t precond, double tol, int max_rounds, double dt, cudaStream_t s) {
    SolveResult R;
    const HeatConst& K = H->K;
    double prev = INFINITY;
    const double ub = H->hscal[S_UB], tb = H->hscal[S_TB];
    for (int ref = 0; ref < 16; ref++) {
        heat_residual64_kernel<<<H->grid, RED_THREADS, 0, s>>>(K, H->scal, H->gas, H->c64, H->rhs, H->kx, H->ky, H->C,
                                                               H->t, H->x, H->r64, H->red(S_RR));
        sr_note_launch();
        H->read(S_RR, 4, s);
        const double rr = H->hscal[S_RR], bb = H->hscal[S_BB], gam = H->hscal[S_GAM], hm = H->hscal[S_HM];
        if (!isfinite(rr) || !isfinite(bb) || !isfinite(gam) || !isfinite(hm)) {
            R.ok = false;
            return R;
        }
        R.rel = bb > 0.0 ? sqrt(rr / bb) : 0.0;
        double worst = R.rel / tol;
        if (ub > 0.0) worst = std::max(worst, sqrt(gam / ub) / tol);
        if (tb > 0.0) worst = std::max(worst, sqrt(hm / tb) / tol);
        if (worst <= 1.0 || rr == 0.0) return R;
        if (worst > 0.5 * prev || R.rounds >= max_rounds) return R;  // stagnating, or out of rounds
        prev = worst;
        const double scale = sqrt(rr / (double)std::max(1, H->n_gas));
        set_scalar(H, S_SCALE, scale, s);
        set_scalar(H, S_ISCALE, 1.0 / scale, s);
        scale_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->r64, H->scal, H->r32, H->e32, H->red(S_R32));
        sr_note_launch();
        const double eta = std::min(0.5, std::max(H->inner_floor, 0.5 / worst));
        bool reached = false;
        int it = inner_pcg(H, precond, eta, max_rounds - R.rounds, s, &reached);
        if (it <= -2) {  // the learned preconditioner stalled: its inner solve is dropped, MG-PCG restarts from x
            R.rounds += -2 - it;
            R.fallback = true;
            precond = SR_PRECOND_MG;
            prev = INFINITY;
            continue;
        }
        if (it < 0) {
            R.ok = false;
            return R;
        }
        R.rounds += it;
        R.refinements++;
        correction_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->gas, H->e32, H->scal, H->x);
        sr_note_launch();
        // an intermediate Newton pass (its tolerance far above the FP32 solve's floor) trusts the FP32 solve that
        // reached its reduction: the next pass starts from a fresh residual anyway; the final pass is always verified
        if (reached && tol >= kTrustedPassTol) {
            R.rel *= eta;
            return R;
        }
    }
    return R;
}

// A pass's system and its measures' bounds (read to the host), then every coarse level and the coarsest inverse.
void build_system(HeatSolver* H, double dt, cudaStream_t s) {
    set_scalar(H, S_DT, dt, s);
    heat_system_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->C, H->t, H->u, H->t0, H->kvac, H->c64,
                                                       H->rhs, H->mg.L[0].c, H->x, H->red(S_UB));
    sr_note_launch();
    H->mg.coarsen(s);
    H->read(S_UB, 2, s);
}

// Appends a conditional node of `type` steered by `h` after everything captured so far on `s` (which is capturing),
// makes the stream's later work follow it, and returns its body graph.
cudaGraph_t capture_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    SR_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    SR_REQUIRE(st == cudaStreamCaptureStatusActive, "a conditional node outside a stream capture");
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    SR_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &p));
    SR_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return p.conditional.phGraph_out[0];
}

// Captures `body(stream)` into the body graph `g` on stream `cs`; returns the kernels it launched.
template <class F>
long long capture_body(cudaGraph_t g, cudaStream_t cs, F body) {
    const long long before = (long long)sr_launches();
    SR_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    body(cs);
    cudaGraph_t out;
    SR_CUDA_TRY(cudaStreamEndCapture(cs, &out));
    const long long n = (long long)sr_launches() - before;
    sr_note_launches(-n);  // captured, not launched
    return n;
}

void ctl_launch(HeatSolver* H, int phase, const CtlHandles& hd, cudaStream_t s) {
    heat_ctl_kernel<<<1, 32, 0, s>>>(H->ctl, H->scal, phase, hd);
    sr_note_launch();
}

// The whole implicit step (MG or Jacobi preconditioner) appended to the capture in progress on `s`, whose root graph
// is `root` (the conditional handles belong to it): set-up, Δt from the device record, the device-controlled Newton
// passes, refinements and PCG rounds, and the commit. The state buffer `U` and the opacity plane are fixed in it.
void capture_heat_step(HeatSolver* H, float* U, const float* kappa, const double* dt_dev, cudaStream_t s,
                       cudaGraph_t root) {
    CtlHandles hd;
    for (int b = 0; b < B_COUNT; b++) SR_CUDA_TRY(cudaGraphConditionalHandleCreate(&hd.h[b], root, 0, 0));
    const uint32_t precond = H->precond;
    const size_t nf = (size_t)(H->w + 1) * H->h + (size_t)H->w * (H->h + 1);
    long long* nb = H->body_launches;
    const long long top0 = (long long)sr_launches();
    setup_step(H, U, kappa, s);
    SR_CUDA_TRY(cudaMemcpyAsync(H->scal + S_DT, dt_dev, sizeof(double), cudaMemcpyDeviceToDevice, s));
    ctl_launch(H, C_BEGIN, hd, s);
    const long long top1 = (long long)sr_launches();
    nb[B_MAIN] = capture_body(capture_conditional(s, hd.h[B_MAIN], cudaGraphCondTypeIf), H->cap[0], [&](cudaStream_t s0) {
        if (precond != SR_PRECOND_JACOBI) {
            warm_start_kernel<<<H->grid, RED_THREADS, 0, s0>>>(H->K, H->scal, H->gas, H->t0, H->rate, H->t, H->u);
            sr_note_launch();
        }
        heat_system_kernel<<<H->grid, RED_THREADS, 0, s0>>>(H->K, H->scal, H->gas, H->C, H->t, H->u, H->t0, H->kvac,
                                                            H->c64, H->rhs, H->mg.L[0].c, H->x, H->red(S_UB));
        sr_note_launch();
        H->mg.coarsen(s0);
        ctl_launch(H, C_NEWTON_BEGIN, hd, s0);
        nb[B_PASS] = capture_body(capture_conditional(s0, hd.h[B_PASS], cudaGraphCondTypeWhile), H->cap[1],
                                  [&](cudaStream_t s1) {
            ctl_launch(H, C_PASS_BEGIN, hd, s1);
            nb[B_REFINE] = capture_body(capture_conditional(s1, hd.h[B_REFINE], cudaGraphCondTypeWhile), H->cap[2],
                                        [&](cudaStream_t s2) {
                heat_residual64_kernel<<<H->grid, RED_THREADS, 0, s2>>>(H->K, H->scal, H->gas, H->c64, H->rhs, H->kx,
                                                                         H->ky, H->C, H->t, H->x, H->r64, H->red(S_RR));
                sr_note_launch();
                ctl_launch(H, C_REFINE, hd, s2);
                nb[B_INNER] = capture_body(capture_conditional(s2, hd.h[B_INNER], cudaGraphCondTypeIf), H->cap[3],
                                           [&](cudaStream_t s3) {
                    scale_kernel<<<H->grid, RED_THREADS, 0, s3>>>(H->n, H->r64, H->scal, H->r32, H->e32, H->red(S_R32));
                    sr_note_launch();
                    precondition(H, precond, S_RZN, s3);
                    ctl_launch(H, C_INNER_BEGIN, hd, s3);
                    nb[B_ROUND] = capture_body(capture_conditional(s3, hd.h[B_ROUND], cudaGraphCondTypeWhile), H->cap[4],
                                               [&](cudaStream_t s4) {
                        spmv_dir_kernel<<<H->grid, RED_THREADS, 0, s4>>>(H->mg.L[0], H->scal, H->z32, H->p32, H->p2,
                                                                          H->q32, H->red(S_PQ), H->scal + S_BETA);
                        sr_note_launch();
                        pcg_update4_kernel<<<H->grid, RED_THREADS, 0, s4>>>(H->n, H->scal, H->p32, H->p2, H->q32,
                                                                             H->e32, H->r32, H->red(S_RRI));
                        sr_note_launch();
                        precondition(H, precond, S_RZN, s4);
                        ctl_launch(H, C_ROUND, hd, s4);
                    });
                    correction_kernel<<<H->grid, RED_THREADS, 0, s3>>>(H->n, H->gas, H->e32, H->scal, H->x);
                    sr_note_launch();
                    ctl_launch(H, C_AFTER_INNER, hd, s3);
                });
            });
            ctl_launch(H, C_PASS_END, hd, s1);
            nb[B_NSYS] = capture_body(capture_conditional(s1, hd.h[B_NSYS], cudaGraphCondTypeIf), H->cap[2],
                                      [&](cudaStream_t s2) {
                newton_system_kernel<<<H->grid, RED_THREADS, 0, s2>>>(H->K, H->cfg.newton_cell, H->scal, H->gas, H->C,
                                                                       H->t0, H->kvac, H->t, H->u, H->x, H->c64,
                                                                       H->rhs, H->mg.L[0].c, H->red(S_MOVED));
                sr_note_launch();
                ctl_launch(H, C_NEWTON, hd, s2);
                nb[B_COARSEN] = capture_body(capture_conditional(s2, hd.h[B_COARSEN], cudaGraphCondTypeIf), H->cap[3],
                                             [&](cudaStream_t s3) { H->mg.coarsen(s3); });
            });
        });
        ctl_launch(H, C_COMMIT, hd, s0);
        nb[B_CONV] = capture_body(capture_conditional(s0, hd.h[B_CONV], cudaGraphCondTypeIf), H->cap[1],
                                  [&](cudaStream_t s1) {
            heat_flux_kernel<<<grid_for(nf), RED_THREADS, 0, s1>>>(H->K, H->gas, H->kx, H->ky, H->u, nullptr, H->fx,
                                                                   H->fy);
            sr_note_launch();
            commit_sums_kernel<<<H->grid, RED_THREADS, 0, s1>>>(H->K, H->scal, H->gas, H->C, H->t, H->t0, H->u,
                                                                H->kvac, H->red(S_RAD));
            sr_note_launch();
            ctl_launch(H, C_DELTA, hd, s1);
            commit_apply_kernel<<<H->grid, RED_THREADS, 0, s1>>>(H->K, H->scal, H->gas, H->C, H->t, H->t0, U, H->rate);
            sr_note_launch();
        });
        nb[B_LIM] = capture_body(capture_conditional(s0, hd.h[B_LIM], cudaGraphCondTypeIf), H->cap[1],
                                 [&](cudaStream_t s1) {
            limited_scale_kernel<<<H->grid, RED_THREADS, 0, s1>>>(H->K, H->scal, H->gas, H->kx, H->ky, H->u, H->C,
                                                                  H->t0, H->lscale);
            sr_note_launch();
            heat_flux_kernel<<<grid_for(nf), RED_THREADS, 0, s1>>>(H->K, H->gas, H->kx, H->ky, H->u, H->lscale, H->fx,
                                                                   H->fy);
            sr_note_launch();
            limited_apply_kernel<<<H->grid, RED_THREADS, 0, s1>>>(H->K, H->scal, H->gas, H->kx, H->ky, H->u,
                                                                  H->lscale, U, H->red(S_RAD));
            sr_note_launch();
            zero_kernel<<<H->grid, RED_THREADS, 0, s1>>>(H->rate, H->n);
            sr_note_launch();
            ctl_launch(H, C_LIMITED, hd, s1);
        });
    });
    nb[B_SKIP] = capture_body(capture_conditional(s, hd.h[B_SKIP], cudaGraphCondTypeIf), H->cap[0],
                              [&](cudaStream_t s0) {
        heat_flux_kernel<<<grid_for(nf), RED_THREADS, 0, s0>>>(H->K, H->gas, H->kx, H->ky, H->u, nullptr, H->fx, H->fy);
        sr_note_launch();
    });
    nb[B_COUNT] = top1 - top0;
    sr_note_launches(-(top1 - top0));  // captured, not launched
}

// The control block's configuration for the next steps.
void ctl_configure(HeatSolver* H, cudaStream_t s) {
    HeatCtl c{};
    c.tol = H->cfg.solve_tol;
    c.nheat = H->cfg.newton_heat;
    c.ncell = H->cfg.newton_cell;
    c.inner_floor = H->inner_floor;
    c.max_passes = (int)H->max_passes;
    c.max_rounds = (int)H->max_rounds;
    c.pin = H->cfg.pin_temperature ? 1 : 0;
    *H->hctl = c;
    SR_CUDA_TRY(cudaMemcpyAsync(H->ctl, H->hctl, sizeof(HeatCtl), cudaMemcpyHostToDevice, s));
    SR_CUDA_TRY(cudaStreamSynchronize(s));
}

void drop_step_graphs(HeatSolver* H) {
    if (!H->step_graphs.empty() && H->stream) cudaStreamSynchronize(H->stream);  // none of them still running
    for (auto& kv : H->step_graphs) cudaGraphExecDestroy(kv.second);
    H->step_graphs.clear();
}

}  // namespace

HeatSolver* heat_create(const sr_config& cfg, cudaStream_t s) {
    HeatSolver* H = new HeatSolver();
    try {
        H->cfg = cfg;
        H->w = (int)cfg.width;
        H->h = (int)cfg.height;
        H->n = (size_t)H->w * H->h;
        SR_REQUIRE(cfg.precond != SR_PRECOND_LEARNED, "the learned preconditioner is loaded after creation");
        H->stream = s;
        H->precond = cfg.precond;
        H->max_passes = cfg.max_passes ? cfg.max_passes : 128;
        H->max_rounds = cfg.max_rounds ? cfg.max_rounds : 4096;
        HeatConst& K = H->K;
        K.w = H->w;
        K.h = H->h;
        K.gm1 = cfg.gamma - 1.0;
        K.mu = cfg.mu;
        K.t_floor = cfg.t_floor;
        K.sigma_vac = cfg.sigma_vac;
        K.sigma_floor = cfg.sigma_floor;
        K.a_r = cfg.a_r;
        K.c_sb = cfg.c_sb;
        K.kappa0 = cfg.kappa0;
        K.k_cond = cfg.k_cond;
        K.chi = cfg.chi;
        K.limiter_on = cfg.flux_limiter != 0;
        H->grid = grid_for(H->n);
        const size_t n = H->n, nx = (size_t)(H->w + 1) * H->h, ny = (size_t)H->w * (H->h + 1);
        SR_CUDA_TRY(cudaMalloc(&H->gas, n));
        double** d64[] = {&H->t0, &H->C, &H->t, &H->u, &H->ksum, &H->kvac, &H->c64, &H->rhs, &H->x, &H->r64,
                          &H->lscale, &H->rate};
        for (double** p : d64) SR_CUDA_TRY(cudaMalloc(p, sizeof(double) * n));
        SR_CUDA_TRY(cudaMemset(H->rate, 0, sizeof(double) * n));
        SR_CUDA_TRY(cudaMalloc(&H->kx, sizeof(double) * nx));
        SR_CUDA_TRY(cudaMalloc(&H->ky, sizeof(double) * ny));
        float** d32[] = {&H->kap, &H->sig, &H->r32, &H->e32, &H->p32, &H->q32, &H->z32, &H->p2};
        for (float** p : d32) SR_CUDA_TRY(cudaMalloc(p, sizeof(float) * n));
        SR_CUDA_TRY(cudaMalloc(&H->fx, sizeof(float) * nx));
        SR_CUDA_TRY(cudaMalloc(&H->fy, sizeof(float) * ny));
        SR_CUDA_TRY(cudaMemset(H->fx, 0, sizeof(float) * nx));
        SR_CUDA_TRY(cudaMemset(H->fy, 0, sizeof(float) * ny));
        SR_CUDA_TRY(cudaMalloc(&H->part, sizeof(double) * 4 * PART_CAP));
        SR_CUDA_TRY(cudaMalloc(&H->counter, sizeof(unsigned)));
        SR_CUDA_TRY(cudaMemset(H->counter, 0, sizeof(unsigned)));
        SR_CUDA_TRY(cudaMalloc(&H->scal, sizeof(double) * S_COUNT));
        SR_CUDA_TRY(cudaMemset(H->scal, 0, sizeof(double) * S_COUNT));
        SR_CUDA_TRY(cudaMallocHost(&H->hscal, sizeof(double) * S_COUNT));
        SR_CUDA_TRY(cudaMalloc(&H->ctl, sizeof(HeatCtl)));
        SR_CUDA_TRY(cudaMemset(H->ctl, 0, sizeof(HeatCtl)));
        SR_CUDA_TRY(cudaMallocHost(&H->hctl, sizeof(HeatCtl)));
        for (cudaStream_t& c : H->cap) SR_CUDA_TRY(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
        H->mg.create(H->w, H->h, (int)cfg.mg_pre, (int)cfg.mg_post);
        H->mg.omega = cfg.mg_omega > 0.0 ? (float)cfg.mg_omega : 1.0f;
        H->inner_floor = cfg.inner_tol > 0.0 ? cfg.inner_tol : 1e-5;
        SR_REQUIRE(mg_smooth_ctas(H->w, H->h) <= (size_t)PART_CAP, "world too large for the sums");
        (void)s;
    } catch (...) {
        heat_destroy(H);
        throw;
    }
    return H;
}

void heat_destroy(HeatSolver* H) {
    if (!H) return;
    for (auto& row : H->graphs)
        for (auto& g : row)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    drop_step_graphs(H);
    cudaFree(H->ctl);
    if (H->hctl) cudaFreeHost(H->hctl);
    for (cudaStream_t c : H->cap)
        if (c) cudaStreamDestroy(c);
    cudaFree(H->gas);
    double* d64[] = {H->t0, H->C, H->t, H->u, H->ksum, H->kvac, H->c64, H->rhs, H->x, H->r64, H->lscale, H->rate,
                     H->kx, H->ky};
    for (double* p : d64) cudaFree(p);
    float* d32[] = {H->kap, H->sig, H->r32, H->e32, H->p32, H->q32, H->z32, H->fx, H->fy, H->p2};
    for (float* p : d32) cudaFree(p);
    cudaFree(H->part);
    cudaFree(H->counter);
    cudaFree(H->scal);
    cudaFree(H->r_old);
    cudaFree(H->ez);
    cudaFree(H->vz);
    cudaFree(H->flush);
    learned_apply_destroy(H->lapply);
    if (H->hscal) cudaFreeHost(H->hscal);
    H->mg.destroy();
    delete H;
}

void heat_set_precond(HeatSolver* H, uint32_t precond) {
    if (precond == SR_PRECOND_LEARNED && !H->lapply)
        throw SrError{SR_E_UNSUPPORTED, "the learned preconditioner is not attached (sr_attach_learner)"};
    if (precond != H->precond) drop_step_graphs(H);  // a captured step holds its preconditioner
    H->precond = precond;
}

void heat_attach_learned(HeatSolver* H, Learner* L) {
    for (auto& g : H->graphs[SR_PRECOND_LEARNED])
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
    learned_apply_destroy(H->lapply);
    H->lapply = nullptr;
    H->learner = L;
    if (!L) {
        if (H->precond == SR_PRECOND_LEARNED) H->precond = SR_PRECOND_MG;
        return;
    }
    if (!H->r_old) SR_CUDA_TRY(cudaMalloc(&H->r_old, sizeof(float) * H->n));
    if (!H->vz) SR_CUDA_TRY(cudaMalloc(&H->vz, sizeof(float) * H->n));
    H->lapply = learned_apply_create(L, H->w, H->h);
}

int heat_collect(HeatSolver* H, Learner* L, const float* U, const float* kappa, double dt, int crops, uint64_t seed,
                 cudaStream_t s) {
    setup_step(H, U, kappa, s);
    H->read(S_HEAT0, 2, s);
    H->n_gas = (int)H->hscal[S_NGAS];
    build_system(H, dt, s);
    heat_residual64_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->c64, H->rhs, H->kx, H->ky, H->C,
                                                           H->t, H->x, H->r64, H->red(S_RR));
    sr_note_launch();
    H->read(S_RR, 1, s);
    const double rr = H->hscal[S_RR];
    if (!(rr > 0.0) || !isfinite(rr)) return 0;
    const double scale = sqrt(rr / (double)std::max(1, H->n_gas));
    set_scalar(H, S_SCALE, scale, s);
    set_scalar(H, S_ISCALE, 1.0 / scale, s);
    scale_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->r64, H->scal, H->r32, H->e32, H->red(S_R32));
    sr_note_launch();
    if (!H->ez) SR_CUDA_TRY(cudaMalloc(&H->ez, sizeof(float) * H->n));
    // after each V-cycle z_k = M_mg r_k: the sample (r_k − A z_k, e_k + z_k); q32 is free until the next round's SpMV
    auto snapshot = [&] {
        vcycle_residual_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->mg.L[0], H->r32, H->z32, H->e32, H->q32, H->ez);
        sr_note_launch();
        learned_snapshot(L, H->mg.L[0], H->q32, H->ez, s);
    };
    const int before = learned_samples(L);
    learned_begin_collect(L, H->w, H->h, crops, seed);
    precondition(H, SR_PRECOND_MG, S_RZ0, s);
    snapshot();
    pcg_direction_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, -1, S_RZ0, H->z32, H->p32);
    sr_note_launch();
    H->read(S_R32, 1, s);
    const double rr0 = H->hscal[S_R32];
    for (int it = 0; it < 200; it++) {
        const int rz_old = (it & 1) ? S_RZ1 : S_RZ0, rz_new = (it & 1) ? S_RZ0 : S_RZ1;
        spmv_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->mg.L[0], H->p32, H->q32, H->red(S_PQ));
        sr_note_launch();
        pcg_update_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, rz_old, H->p32, H->q32, H->e32, H->r32,
                                                          H->red(S_RRI));
        sr_note_launch();
        H->read(S_PQ, 2, s);
        // solve on to a 1e-6 residual reduction; samples only while the remaining error is large against that
        if (!(H->hscal[S_PQ] > 0.0) || H->hscal[S_RRI] <= 1e-12 * rr0) break;
        precondition(H, SR_PRECOND_MG, rz_new, s);
        if (H->hscal[S_RRI] > 1e-8 * rr0) snapshot();
        pcg_direction_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->n, H->scal, rz_old, rz_new, H->z32, H->p32);
        sr_note_launch();
    }
    learned_end_collect(L, H->mg.L[0], H->e32, s);
    return learned_samples(L) - before;
}

void heat_reset(HeatSolver* H, cudaStream_t s) { SR_CUDA_TRY(cudaMemsetAsync(H->rate, 0, sizeof(double) * H->n, s)); }

void heat_rate_to_f32(HeatSolver* H, float* dst, cudaStream_t s) {
    f64_to_f32_kernel<<<H->grid, RED_THREADS, 0, s>>>(dst, H->rate, H->n);
    sr_note_launch();
    SR_CUDA_TRY(cudaGetLastError());
}

void heat_rate_from_f32(HeatSolver* H, const float* src, cudaStream_t s) {
    if (!src) {
        heat_reset(H, s);
        return;
    }
    f32_to_f64_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->rate, src, H->n);
    sr_note_launch();
    SR_CUDA_TRY(cudaGetLastError());
}

void heat_set_reference(HeatSolver* H, const HeatRef& R) {
    H->ref = R;
    H->K.ref = R.on;
    drop_step_graphs(H);
}

void heat_flux_planes(const HeatSolver* H, const float** fx, const float** fy) {
    *fx = H->fx;
    *fy = H->fy;
}

double* heat_rate_plane(HeatSolver* H) { return H->rate; }

bool heat_wait_error(HeatSolver* H, cudaStream_t s) { return H->mg.error(s); }

void heat_set_limits(HeatSolver* H, uint32_t max_passes, uint32_t max_rounds) {
    H->max_passes = max_passes;
    H->max_rounds = max_rounds;
    drop_step_graphs(H);  // the next step captures again, with the new limits in its control block
}

void heat_read_flux(HeatSolver* H, float* fx, float* fy) {
    const size_t nx = (size_t)(H->w + 1) * H->h, ny = (size_t)H->w * (H->h + 1);
    if (fx) SR_CUDA_TRY(cudaMemcpy(fx, H->fx, sizeof(float) * nx, cudaMemcpyDeviceToHost));
    if (fy) SR_CUDA_TRY(cudaMemcpy(fy, H->fy, sizeof(float) * ny, cudaMemcpyDeviceToHost));
}

// Reads the device-controlled steps' control block: the last step's report, and the kernels its bodies launched since
// the last read (added to the library's launch count).
void heat_sync_report(HeatSolver* H, cudaStream_t s) {
    if (!H->report_pending) return;
    SR_CUDA_TRY(cudaMemcpyAsync(H->hctl, H->ctl, sizeof(HeatCtl), cudaMemcpyDeviceToHost, s));
    SR_CUDA_TRY(cudaMemsetAsync(H->ctl->runs, 0, sizeof(H->ctl->runs), s));
    SR_CUDA_TRY(cudaStreamSynchronize(s));
    const HeatCtl& c = *H->hctl;
    long long n = 0;
    for (int b = 0; b < B_COUNT; b++) n += (long long)c.runs[b] * H->body_launches[b];
    sr_note_launches(n);
    sr_heat_report R{};
    R.precond = H->precond;
    R.dt = c.skipped ? 0.0 : H->hscal[S_DT];
    R.passes = (uint32_t)c.passes;
    R.rounds = (uint32_t)c.rounds;
    R.refinements = (uint32_t)c.refinements;
    R.converged = (uint32_t)c.converged;
    R.delta = c.delta;
    R.radiated = c.radiated;
    R.rel_residual = c.rel;
    H->report = R;
    H->report_pending = false;
}

void heat_step(HeatSolver* H, float* U, const float* kappa, const double* dt_dev, cudaStream_t s,
               sr_heat_report* rep) {
    if (H->precond != SR_PRECOND_LEARNED && H->use_graphs && H->mg.tuned) {
        // the device-controlled step: captured once per state buffer, then replayed with no host round trip
        auto it = H->step_graphs.find(U);
        if (it == H->step_graphs.end()) {
            heat_sync_report(H, s);
            ctl_configure(H, s);
            cudaGraph_t g;
            SR_CUDA_TRY(cudaGraphCreate(&g, 0));
            SR_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            try {
                capture_heat_step(H, U, kappa, dt_dev, s, g);
            } catch (...) {
                cudaGraph_t dead;
                cudaStreamEndCapture(s, &dead);
                cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t out;
            SR_CUDA_TRY(cudaStreamEndCapture(s, &out));
            cudaGraphExec_t exec;
            const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            SR_CUDA_TRY(e);
            it = H->step_graphs.emplace(U, exec).first;
        }
        SR_CUDA_TRY(cudaGraphLaunch(it->second, s));
        sr_note_launches(H->body_launches[B_COUNT]);
        H->report_pending = true;
        (void)rep;
        return;
    }
    heat_sync_report(H, s);
    sr_heat_report R{};
    R.precond = H->precond;
    setup_step(H, U, kappa, s);
    SR_CUDA_TRY(cudaMemcpyAsync(H->scal + S_DT, dt_dev, sizeof(double), cudaMemcpyDeviceToDevice, s));
    H->read(S_HEAT0, 3, s);  // Σ C T⁰, gas cells, Δt
    H->n_gas = (int)H->hscal[S_NGAS];
    const double dt = H->hscal[S_DT];
    const double heat0 = H->hscal[S_HEAT0];
    const size_t nf = (size_t)(H->w + 1) * H->h + (size_t)H->w * (H->h + 1);
    if (H->cfg.pin_temperature || H->n_gas == 0 || !(dt > 0.0)) {
        heat_flux_kernel<<<grid_for(nf), RED_THREADS, 0, s>>>(H->K, H->gas, H->kx, H->ky, H->u, nullptr, H->fx,
                                                               H->fy);
        sr_note_launch();
        R.converged = 1;
        H->report = R;
        *rep = R;
        return;
    }
    R.dt = dt;
    if (H->precond != SR_PRECOND_JACOBI) {
        warm_start_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->t0, H->rate, H->t, H->u);
        sr_note_launch();
    }
    uint32_t passes = 0, rounds = 0;
    bool converged = false;
    // Inexact Newton: a pass's solve is asked for the last pass's relative heat moved (the first pass for
    // kFirstPassTol), never more than kFirstPassTol nor less than solve_tol; the passes end only on a pass solved to
    // solve_tol. Loose early passes cost fewer rounds in all than accurate ones: each pass's system is rebuilt at the
    // new iterate anyway, and the last pass meets the same tolerances.
    const double tol = H->cfg.solve_tol;
    double pass_tol = std::max(tol, kFirstPassTol);
    const double nheat = H->cfg.newton_heat, ncell = H->cfg.newton_cell;
    double moved_prev = 0.0;
    build_system(H, dt, s);
    while (passes < H->max_passes && rounds < H->max_rounds) {
        passes++;
        SolveResult S = solve_pass(H, H->precond, pass_tol, (int)(H->max_rounds - rounds), dt, s);
        rounds += (uint32_t)S.rounds;
        R.refinements += (uint32_t)S.refinements;
        R.rel_residual = S.rel;
        if (S.fallback) R.fallback_used = 1;
        if (!S.ok) break;
        newton_system_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, ncell, H->scal, H->gas, H->C, H->t0,
                                                              H->kvac, H->t, H->u, H->x, H->c64, H->rhs,
                                                              H->mg.L[0].c, H->red(S_MOVED));
        sr_note_launch();
        H->read(S_MOVED, 4, s);  // moved, violations, and the next system's two bounds
        const double rel_moved = heat0 > 0.0 ? H->hscal[S_MOVED] / heat0 : 0.0;
        if (rel_moved <= nheat && H->hscal[S_VIOL] == 0.0 && pass_tol <= tol) {
            converged = true;
            break;
        }
        // the next pass is solved to solve_tol once it is expected to move less than newton_heat (the passes' observed
        // contraction times this pass's move), since only a pass solved to solve_tol can end them
        const double ratio = moved_prev > 0.0 ? std::min(1.0, std::max(0.01, rel_moved / moved_prev)) : 0.1;
        moved_prev = rel_moved;
        pass_tol = std::max(tol, std::min(kFirstPassTol, rel_moved));
        if (ratio * rel_moved <= nheat) pass_tol = tol;
        H->mg.coarsen(s);  // the next pass's coarse levels (its level-0 c is in place)
    }
    R.passes = passes;
    R.rounds = rounds;
    if (converged) {
        heat_flux_kernel<<<grid_for(nf), RED_THREADS, 0, s>>>(H->K, H->gas, H->kx, H->ky, H->u, nullptr, H->fx, H->fy);
        sr_note_launch();
        commit_sums_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->C, H->t, H->t0, H->u, H->kvac,
                                                           H->red(S_RAD));
        sr_note_launch();
        H->read(S_RAD, 3, s);
        const double rad = H->hscal[S_RAD], gain = H->hscal[S_GAIN], held = H->hscal[S_HELD];
        const double delta = -(gain + rad) / held;
        set_scalar(H, S_DELTA, delta, s);
        commit_apply_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->C, H->t, H->t0, U, H->rate);
        sr_note_launch();
        R.converged = 1;
        R.delta = delta;
        R.radiated = rad;
    } else {
        limited_scale_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->kx, H->ky, H->u, H->C, H->t0,
                                                             H->lscale);
        sr_note_launch();
        heat_flux_kernel<<<grid_for(nf), RED_THREADS, 0, s>>>(H->K, H->gas, H->kx, H->ky, H->u, H->lscale, H->fx,
                                                               H->fy);
        sr_note_launch();
        limited_apply_kernel<<<H->grid, RED_THREADS, 0, s>>>(H->K, H->scal, H->gas, H->kx, H->ky, H->u, H->lscale, U,
                                                             H->red(S_RAD));
        sr_note_launch();
        SR_CUDA_TRY(cudaMemsetAsync(H->rate, 0, sizeof(double) * H->n, s));
        H->read(S_RAD, 1, s);
        R.converged = 0;
        R.delta = 0.0;
        R.radiated = H->hscal[S_RAD];
    }
    SR_CUDA_TRY(cudaGetLastError());
    H->report = R;
    *rep = R;
}

void heat_report(HeatSolver* H, cudaStream_t s, sr_heat_report* rep) {
    heat_sync_report(H, s);
    *rep = H->report;
}

void heat_account_launches(HeatSolver* H, cudaStream_t s) { heat_sync_report(H, s); }

bool heat_capturable(const HeatSolver* H) {
    return H->precond != SR_PRECOND_LEARNED && H->use_graphs && H->mg.tuned;
}

void heat_prepare_capture(HeatSolver* H, cudaStream_t s) {
    heat_sync_report(H, s);
    ctl_configure(H, s);
}

long long heat_capture_step(HeatSolver* H, float* U, const float* kappa, const double* dt_dev, cudaStream_t s,
                            cudaGraph_t root) {
    capture_heat_step(H, U, kappa, dt_dev, s, root);
    return H->body_launches[B_COUNT];
}

void heat_graph_launched(HeatSolver* H) { H->report_pending = true; }

void heat_first_solve(HeatSolver* H, const float* U, const float* kappa, double dt, uint32_t precond, cudaStream_t s,
                      double* ms, uint32_t* rounds, double* rel_residual, double* x, uint32_t* fallback) {
    if (precond == SR_PRECOND_LEARNED && !H->lapply)
        throw SrError{SR_E_UNSUPPORTED, "the learned preconditioner is not attached (sr_attach_learner)"};
    setup_step(H, U, kappa, s);
    H->read(S_HEAT0, 2, s);
    H->n_gas = (int)H->hscal[S_NGAS];
    build_system(H, dt, s);
    cudaEvent_t a, b;
    SR_CUDA_TRY(cudaEventCreate(&a));
    SR_CUDA_TRY(cudaEventCreate(&b));
    SR_CUDA_TRY(cudaEventRecord(a, s));
    SolveResult S = solve_pass(H, precond, H->cfg.solve_tol, (int)H->max_rounds, dt, s);
    SR_CUDA_TRY(cudaEventRecord(b, s));
    SR_CUDA_TRY(cudaEventSynchronize(b));
    float t = 0.0f;
    SR_CUDA_TRY(cudaEventElapsedTime(&t, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms) *ms = t;
    if (rounds) *rounds = (uint32_t)S.rounds;
    if (rel_residual) *rel_residual = S.rel;
    if (fallback) *fallback = S.fallback ? 1u : 0u;
    if (x) SR_CUDA_TRY(cudaMemcpy(x, H->x, sizeof(double) * H->n, cudaMemcpyDeviceToHost));
    SR_CUDA_TRY(cudaGetLastError());
}

void heat_time_smoother(HeatSolver* H, int reps, cudaStream_t s, double* pre_ms, double* post_ms) {
    constexpr size_t kFlush = (size_t)256 << 20;  // twice the L2
    if (!H->flush) SR_CUDA_TRY(cudaMalloc(&H->flush, kFlush));
    H->mg.time_level0(reps, H->flush, kFlush, s, pre_ms, post_ms);
}
