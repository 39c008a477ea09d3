// grav.cuh — P2, the FFT-convolution gravity solve.
#pragma once

#include "common.cuh"

struct GravArgs {
    int w, h, px, py;
    size_t ld;  // column stride of the spectrum buffer, in complex values (h + 2)
    float sigma_vac;
    const float* src;
    float2* spec;
    const float* khat;
    const float2* tw_x;
    const float2* tw_y;
    float* phi_ring;
    float* phi;
    float* gx;
    float* gy;
};

// The smallest power of two >= 2 len, at least 32, at most 8192 (0: refused).
int grav_padded_size(int len);

// One world's solve: its spectrum work buffer, ringed potential, K̂ quarter and twiddle tables.
struct GravPlan {
    int w = 0, h = 0, px = 0, py = 0;
    size_t ld = 0;
    float sigma_vac = 0.0f;
    float2* spec = nullptr;
    float* phi_ring = nullptr;
    float* khat = nullptr;
    float2* tw_x = nullptr;
    float2* tw_y = nullptr;

    void create(int w, int h, int kernel, double G, double eps, float sigma_vac);
    void destroy();
    size_t bytes() const;
    // φ = K * Σ_src (Σ below Σ_vac not a source) and g = -∇φ, W*H each.
    void solve(const float* src, float* phi, float* gx, float* gy, cudaStream_t s) const;
};
