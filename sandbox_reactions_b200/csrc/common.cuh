// common.cuh — shared device/host helpers of the B200 field update: error plumbing, the scheme's parameters and the
// per-cell physics of the config-mode EOS (Π = (γ-1)Σε, c² = γΠ/Σ, T = μ(γ-1)ε), in FP32.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/sr_cuda.h"

#define SR_HOST_DEVICE __host__ __device__ __forceinline__

// ------------------------------------------------------------------------------------------------ error plumbing
struct SrError {
    sr_status status;
    std::string message;
};

#define SR_CUDA_TRY(expr)                                                                                     \
    do {                                                                                                      \
        cudaError_t e_ = (expr);                                                                              \
        if (e_ != cudaSuccess)                                                                                \
            throw SrError{e_ == cudaErrorMemoryAllocation ? SR_E_NOMEM : SR_E_CUDA,                           \
                          std::string(#expr) + ": " + cudaGetErrorString(e_)};                               \
    } while (0)

#define SR_REQUIRE(cond, msg)                                      \
    do {                                                           \
        if (!(cond)) throw SrError{SR_E_INVALID, std::string(msg)}; \
    } while (0)

// ------------------------------------------------------------------------------------------------ scheme constants
// The hydro scheme's scalars, passed by value to every hydro kernel.
struct HydroConst {
    int w, h;
    int edge, limiter, bracket;
    float gamma, gm1, eps_floor, sigma_vac, sigma_floor;
    float inv_gm1;  // 1 / (γ - 1)
};

struct Prim {
    float s, u, v, p;  // Σ, u, v, Π
};

struct Face {
    float U[4];  // conserved Σ, Σu, Σv, E
    Prim p;      // the primitives it stands for
};

// Division and the square root of a non-negative value at the hardware's approximate rate on the device (one
// reciprocal or reciprocal square root and a product, within 2 ulp; the FP32 physics is held to 1e-5 of the f64
// twin), exact on the host.
SR_HOST_DEVICE float sr_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
SR_HOST_DEVICE float sr_sqrt(float x) {
#ifdef __CUDA_ARCH__
    return x > 0.0f ? x * rsqrtf(x) : 0.0f;
#else
    return x > 0.0f ? sqrtf(x) : 0.0f;
#endif
}

SR_HOST_DEVICE float eos_pi(const HydroConst& H, float s, float eps) { return H.gm1 * s * eps; }

// A cell as primitives (reference hydro.rs:424-441): the floor state below Σ_vac, else ε_th floored at T_floor/(μ(γ-1)).
SR_HOST_DEVICE Prim eos_read(const HydroConst& H, float s, float mx, float my, float E) {
    Prim p;
    if (s < H.sigma_vac) {
        p.s = H.sigma_floor;
        p.u = 0.0f;
        p.v = 0.0f;
        p.p = eos_pi(H, H.sigma_floor, H.eps_floor);
        return p;
    }
    const float rs = sr_div(1.0f, s);  // one division per cell: the velocities and ε by products
    p.u = mx * rs;
    p.v = my * rs;
    float raw = E * rs - 0.5f * (p.u * p.u + p.v * p.v);
    float eps = raw < H.eps_floor ? H.eps_floor : raw;
    p.s = s;
    p.p = eos_pi(H, s, eps);
    return p;
}

// The conserved vector of primitives (hydro.rs:443-460).
SR_HOST_DEVICE void eos_cons(const HydroConst& H, const Prim& p, float* U) {
    float thermal = sr_div(p.p, p.s) * H.inv_gm1;
    float eps = fmaxf(thermal, H.eps_floor);
    U[0] = p.s;
    U[1] = p.s * p.u;
    U[2] = p.s * p.v;
    U[3] = p.s * eps + 0.5f * p.s * (p.u * p.u + p.v * p.v);
}

// The primitives of a conserved vector, false when it is no state (hydro.rs:462-478): Σ not positive, any component
// not finite, or no thermal energy left. The finiteness test rides on the derived values: a non-finite Σu or Σv makes
// u or v, hence the thermal energy, -inf or NaN; a non-finite E makes it ±inf or NaN; Σ = +inf makes every velocity 0
// (or NaN) and the thermal energy 0 (or NaN) — so "thermal energy positive and finite" rejects the states with a
// non-finite component, as the reference's test of all four does (and, beyond it, a state whose thermal energy per mass
// alone overflows FP32, which no FP32 cell can hold anyway).
SR_HOST_DEVICE bool eos_prim(const HydroConst& H, const float* U, Prim& out) {
    float s = U[0];
    if (!(s > 0.0f)) return false;  // NaN or <= 0
    const float rs = sr_div(1.0f, s);  // one division per state: the velocities and ε by products
    const float u = U[1] * rs, v = U[2] * rs;
    float raw = U[3] * rs - 0.5f * (u * u + v * v);
    if (!(raw > 0.0f) || raw == INFINITY) return false;
    float eps = fmaxf(raw, H.eps_floor);
    out.s = s;
    out.u = u;
    out.v = v;
    out.p = eos_pi(H, s, eps);
    return true;
}

SR_HOST_DEVICE float eos_sound(const HydroConst& H, const Prim& p) {
    return sr_sqrt(H.gamma * sr_div(p.p, p.s));
}

// The Euler flux through a face normal to `dir` (hydro.rs:485-499).
SR_HOST_DEVICE void euler_flux(const Prim& p, float energy, int dir, float* f) {
    float un = dir == 0 ? p.u : p.v, ut = dir == 0 ? p.v : p.u;
    float mass = p.s * un;
    f[0] = mass;
    f[1 + dir] = mass * un + p.p;
    f[2 - dir] = mass * ut;
    f[3] = (energy + p.p) * un;
}

// x = i mod w, y = i / w for a cell or face index below 2^32 (every world here), by 32-bit division: the 64-bit
// division of a size_t index costs an emulated sequence per element in the grid-stride kernels.
SR_HOST_DEVICE void split_index(size_t i, int w, int& x, int& y) {
    const unsigned u = (unsigned)i, uw = (unsigned)w;
    y = (int)(u / uw);
    x = (int)(u - (unsigned)y * uw);
}

// ------------------------------------------------------------------------------------------------ launch helpers
// Every kernel launch of the library is counted (sr_cost.kernel_launches reports the count of an sr_step call).
// The message sr_last_error(NULL) returns (calls without a context).
void sr_set_global_error(const std::string& message);
void sr_note_launch();
void sr_note_launches(long long n);
unsigned long long sr_launches();
static inline unsigned div_up(unsigned a, unsigned b) { return (a + b - 1) / b; }
