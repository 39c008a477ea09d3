// hydro.cu — P4, the MUSCL-Hancock/HLL gas step, as one shared-memory tiled stencil kernel per pass (sm_100a, FP32).
//
// One CTA owns a TX x TY tile of output cells. It stages the primitives of the tile grown by two cells (the
// reconstruction's reach, ghosts of the world's edges included) in shared memory once, runs the Hancock predictor for
// the tile and for the one-cell strips around it, exchanges the predicted faces through shared memory for the HLL
// fluxes, and finishes with the per-cell epilogue of its pass:
//   - kHydroUpdate:     U' = U - Δt ΔF (no gravity);
//   - kHydroSource:     the half step's gravity source ½(Σⁿ + Σⁿ⁺¹), masked (reference hydro.rs:815-836);
//   - kHydroUpdateGrav: U' with gravity's half-step kick and the faces' work across φ_mid (hydro.rs:871-947).
// The scheme follows crates/sr-physics/src/reference/hydro.rs (step_held without held cells, sinks or radiation).
#include "hydro.cuh"

namespace {

constexpr int TX = kHydroTileX, TY = kHydroTileY;
constexpr int EX = TX + 4, EY = TY + 4;  // the staged region: the tile grown by 2
constexpr int NT = TX * TY;              // threads per CTA: one per tile cell

__device__ __forceinline__ float lim_mc(float l, float c, float r) {
    float a = c - l, b = r - c;
    if (a * b <= 0.0f) return 0.0f;
    return copysignf(fminf(fminf(fabsf(0.5f * (a + b)), 2.0f * fabsf(a)), 2.0f * fabsf(b)), a);
}

__device__ __forceinline__ float lim_minmod(float l, float c, float r) {
    float a = c - l, b = r - c;
    if (a * b <= 0.0f) return 0.0f;
    return copysignf(fminf(fabsf(a), fabsf(b)), a);
}

__device__ __forceinline__ float lim(int which, float l, float c, float r) {
    return which == SR_LIMITER_MINMOD ? lim_minmod(l, c, r) : lim_mc(l, c, r);
}

// Limited slopes of (Σ, u, v, Π) along one axis; Σ and Π flat where the thermal bracket refuses a face
// (hydro.rs:293-331, HOT_FACE = 2).
__device__ __forceinline__ Prim slope(const HydroConst& H, const Prim& l, const Prim& c, const Prim& r, float ql,
                                      float qc, float qr) {
    Prim s;
    s.s = lim(H.limiter, l.s, c.s, r.s);
    s.u = lim(H.limiter, l.u, c.u, r.u);
    s.v = lim(H.limiter, l.v, c.v, r.v);
    s.p = lim(H.limiter, l.p, c.p, r.p);
    if (H.bracket) {
        float hottest = fmaxf(fmaxf(ql, qc), qr);  // Π/Σ of the three cells, staged once per cell
        float plo = c.p - 0.5f * s.p, blo = 2.0f * hottest * (c.s - 0.5f * s.s);
        float phi = c.p + 0.5f * s.p, bhi = 2.0f * hottest * (c.s + 0.5f * s.s);
        if (!(plo <= blo) || !(phi <= bhi)) {
            s.s = 0.0f;
            s.p = 0.0f;
        }
    }
    return s;
}

__device__ __forceinline__ Prim offset(const Prim& c, const Prim& s, float f) {
    Prim o;
    o.s = c.s + f * s.s;
    o.u = c.u + f * s.u;
    o.v = c.v + f * s.v;
    o.p = c.p + f * s.p;
    return o;
}

// A face advanced by the Hancock increment, or the unevolved face when the advanced one is no state (hydro.rs:501-513).
__device__ __forceinline__ void evolved(const HydroConst& H, const Prim& base, const float* u0, const float* d, Face& F) {
    float U[4] = {u0[0] + d[0], u0[1] + d[1], u0[2] + d[2], u0[3] + d[3]};
    Prim p;
    if (eos_prim(H, U, p)) {
        F.U[0] = U[0]; F.U[1] = U[1]; F.U[2] = U[2]; F.U[3] = U[3];
        F.p = p;
    } else {
        F.U[0] = u0[0]; F.U[1] = u0[1]; F.U[2] = u0[2]; F.U[3] = u0[3];
        F.p = base;
    }
}

// The four predicted faces [x-, x+, y-, y+] of a cell and its centre's (Σ, Σu, Σv) half a step on (hydro.rs:587-614).
// `want` is a bit mask of the faces the caller keeps.
__device__ __forceinline__ void predict(const HydroConst& H, const Prim& l, const Prim& c, const Prim& r,
                                        const Prim& up, const Prim& dn, const float* q, float half, bool grav,
                                        float gx, float gy, int want, Face* out, float* mid) {
    // q: Π/Σ of l, c, r, up, dn
    Prim sx = slope(H, l, c, r, q[0], q[1], q[2]);
    Prim sy = slope(H, up, c, dn, q[3], q[1], q[4]);
    Prim wf[4] = {offset(c, sx, -0.5f), offset(c, sx, 0.5f), offset(c, sy, -0.5f), offset(c, sy, 0.5f)};
    float uf[4][4];
#pragma unroll
    for (int k = 0; k < 4; k++) eos_cons(H, wf[k], uf[k]);
    float fxl[4], fxr[4], fyl[4], fyr[4];
    euler_flux(wf[0], uf[0][3], 0, fxl);
    euler_flux(wf[1], uf[1][3], 0, fxr);
    euler_flux(wf[2], uf[2][3], 1, fyl);
    euler_flux(wf[3], uf[3][3], 1, fyr);
    float delta[4];
#pragma unroll
    for (int k = 0; k < 4; k++) delta[k] = half * ((fxl[k] - fxr[k]) + (fyl[k] - fyr[k]));
    mid[0] = c.s + delta[0];
    mid[1] = c.s * c.u + delta[1];
    mid[2] = c.s * c.v + delta[2];
    if (grav) {
        mid[1] += half * c.s * gx;
        mid[2] += half * c.s * gy;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (!(want & (1 << k))) continue;
        float d[4] = {delta[0], delta[1], delta[2], delta[3]};
        if (grav) {
            const Prim& p = wf[k];
            d[1] += half * p.s * gx;
            d[2] += half * p.s * gy;
            d[3] += half * p.s * ((p.u + 0.5f * half * gx) * gx + (p.v + 0.5f * half * gy) * gy);
        }
        evolved(H, wf[k], uf[k], d, out[k]);
    }
}

// HLL with Davis speeds across a face normal to `dir` (hydro.rs:516-540).
__device__ __forceinline__ void hll(const HydroConst& H, const Face& l, const Face& r, int dir, float* f) {
    float unl = dir == 0 ? l.p.u : l.p.v, unr = dir == 0 ? r.p.u : r.p.v;
    float cl = eos_sound(H, l.p), cr = eos_sound(H, r.p);
    float s_l = fminf(unl - cl, unr - cr);
    float s_r = fmaxf(unl + cl, unr + cr);
    float fl[4], fr[4];
    euler_flux(l.p, l.U[3], dir, fl);
    euler_flux(r.p, r.U[3], dir, fr);
    if (s_l >= 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = fl[k];
    } else if (s_r <= 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = fr[k];
    } else {
        float inv = 1.0f / (s_r - s_l);
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = (s_r * fl[k] - s_l * fr[k] + s_l * s_r * (r.U[k] - l.U[k])) * inv;
    }
}

__device__ __forceinline__ void wall(const Face& own, int dir, float* f) {  // hydro.rs:556-562
    f[0] = 0.0f; f[1] = 0.0f; f[2] = 0.0f; f[3] = 0.0f;
    f[1 + dir] = own.p.p;
}

// Gravity's source at one face over the step (hydro.rs:1042-1067): [impulse to the low cell, low energy, high energy].
__device__ __forceinline__ void face_work(float q, float sl, float sh, float pl, float ph, float d, float dt, float* o) {
    float a = fmaxf(sl, 0.0f), b = fmaxf(sh, 0.0f);
    float w = a + b > 0.0f ? a / (a + b) : 0.5f;
    float extra = dt * (q - 0.5f * (pl + ph)) * d;
    float c = 0.0f, kick = 0.0f, el = 0.0f, eh = 0.0f;
    if (extra < 0.0f && a > 0.0f && b > 0.0f) {
        float ul = pl / a, uh = ph / b;
        float du = ul - uh;
        float inv = 1.0f / a + 1.0f / b;
        c = fminf(-extra, 0.25f * du * du / inv);
        if (c > 0.0f) {
            float disc = sqrtf(fmaxf(du * du - 2.0f * inv * c, 0.0f));
            kick = -2.0f * c / (du + copysignf(1.0f, du) * disc);
            el = ul * kick + 0.5f * kick * kick / a;
            eh = -uh * kick + 0.5f * kick * kick / b;
        }
    }
    float rest = extra + c;
    o[0] = kick;
    o[1] = 0.5f * dt * pl * d + w * rest + el;
    o[2] = 0.5f * dt * ph * d + (1.0f - w) * rest + eh;
}

struct __align__(16) Shared {
    float4 P[EY][EX];         // primitives (Σ, u, v, Π) of the staged region, ghosts included
    float S[EY][EX];          // raw Σ of the staged region (out-of-world: -1, read as vacuum)
    float Q[EY][EX];          // Π/Σ of the staged region (the thermal bracket's temperatures)
    Face F[4][TY][TX];        // the tile's predicted faces
    Face FL[TY], FR[TY];      // x+ faces of the column left of the tile, x- faces of the column right of it
    Face FT[TX], FB[TX];      // y+ faces of the row above, y- faces of the row below
    float M[TY + 2][TX + 2][3];  // half-step (Σ, Σu, Σv) of the tile and its ring
    float FX[TY][TX + 1][4];  // x-face fluxes
    float FY[TY + 1][TX][4];  // y-face fluxes
};

// The primitives at world position (x, y), a ghost past the world's edge (hydro.rs:686-709): bounce mirrors the
// cells beyond with the normal velocity negated, leave copies the edge cell with it clamped outward.
__device__ __forceinline__ Prim ghosted(const HydroConst& H, const float* __restrict__ U, int x, int y, float& raw) {
    const int w = H.w, h = H.h;
    const size_t n = (size_t)w * h;
    bool xo = x < 0 || x >= w, yo = y < 0 || y >= h;
    int cx, cy;
    if (H.edge == SR_EDGE_BOUNCE) {
        cx = x < 0 ? -x - 1 : (x >= w ? 2 * w - 1 - x : x);
        cy = y < 0 ? -y - 1 : (y >= h ? 2 * h - 1 - y : y);
    } else {
        cx = min(max(x, 0), w - 1);
        cy = min(max(y, 0), h - 1);
    }
    size_t i = (size_t)cy * w + cx;
    float s = U[i];
    Prim p = eos_read(H, s, U[n + i], U[2 * n + i], U[3 * n + i]);
    raw = (xo || yo) ? -1.0f : s;
    if (H.edge == SR_EDGE_BOUNCE) {
        if (xo) p.u = -p.u;
        if (yo) p.v = -p.v;
    } else {
        if (x < 0) p.u = fminf(p.u, 0.0f);
        if (x >= w) p.u = fmaxf(p.u, 0.0f);
        if (y < 0) p.v = fminf(p.v, 0.0f);
        if (y >= h) p.v = fmaxf(p.v, 0.0f);
    }
    return p;
}

__device__ __forceinline__ Prim P_at(const Shared& sh, int ly, int lx) {
    float4 q = sh.P[ly][lx];
    Prim p;
    p.s = q.x; p.u = q.y; p.v = q.z; p.p = q.w;
    return p;
}

template <int MODE>
__global__ void __launch_bounds__(NT, 3) hydro_tile_kernel(HydroArgs A) {  // 3 CTAs per SM: 80 registers, ~15 B spilled
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Shared& sh = *reinterpret_cast<Shared*>(smem_raw);
    const HydroConst H = A.H;
    const int w = H.w, h = H.h;
    const size_t n = (size_t)w * h;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.x;
    const float dt = (float)(*A.dt);
    const float half = 0.5f * dt;
    const bool grav = A.gx != nullptr;

    // ---- stage: primitives of the tile grown by 2 (world cells or ghosts), raw Σ for the vacuum tests
    for (int k = tid; k < EX * EY; k += NT) {
        int ly = k / EX, lx = k % EX;
        int x = x0 + lx - 2, y = y0 + ly - 2;
        float raw = -1.0f;
        Prim p;
        if (x >= -2 && x <= w + 1 && y >= -2 && y <= h + 1) {
            p = ghosted(H, A.U, x, y, raw);
        } else {
            p.s = 1.0f; p.u = 0.0f; p.v = 0.0f; p.p = 1.0f;  // past every ghost: never reaches a kept cell
        }
        sh.P[ly][lx] = make_float4(p.s, p.u, p.v, p.p);
        sh.S[ly][lx] = raw;
        sh.Q[ly][lx] = p.p / p.s;
    }
    __syncthreads();

    // ---- predict: the tile's cells (all four faces) and the strips around it (the face toward the tile)
    for (int k = tid; k < NT + 2 * TY + 2 * TX; k += NT) {
        int lx, ly, want;  // local tile coordinates of the cell, -1..TX / -1..TY
        if (k < NT) {
            lx = k % TX; ly = k / TX; want = 15;
        } else if (k < NT + TY) {
            lx = -1; ly = k - NT; want = 2;
        } else if (k < NT + 2 * TY) {
            lx = TX; ly = k - NT - TY; want = 1;
        } else if (k < NT + 2 * TY + TX) {
            lx = k - NT - 2 * TY; ly = -1; want = 8;
        } else {
            lx = k - NT - 2 * TY - TX; ly = TY; want = 4;
        }
        int sx = lx + 2, sy = ly + 2;
        float gxv = 0.0f, gyv = 0.0f;
        if (grav) {
            int cx = min(max(x0 + lx, 0), w - 1), cy = min(max(y0 + ly, 0), h - 1);  // a ghost takes its edge cell's g
            size_t i = (size_t)cy * w + cx;
            gxv = A.gx[i];
            gyv = A.gy[i];
        }
        Face f[4];
        float mid[3];
        const float q[5] = {sh.Q[sy][sx - 1], sh.Q[sy][sx], sh.Q[sy][sx + 1], sh.Q[sy - 1][sx], sh.Q[sy + 1][sx]};
        predict(H, P_at(sh, sy, sx - 1), P_at(sh, sy, sx), P_at(sh, sy, sx + 1), P_at(sh, sy - 1, sx),
                P_at(sh, sy + 1, sx), q, half, grav, gxv, gyv, want, f, mid);
        if (k < NT) {
#pragma unroll
            for (int q = 0; q < 4; q++) sh.F[q][ly][lx] = f[q];
        } else if (lx == -1) {
            sh.FL[ly] = f[1];
        } else if (lx == TX) {
            sh.FR[ly] = f[0];
        } else if (ly == -1) {
            sh.FT[lx] = f[3];
        } else {
            sh.FB[lx] = f[2];
        }
        sh.M[ly + 1][lx + 1][0] = mid[0];
        sh.M[ly + 1][lx + 1][1] = mid[1];
        sh.M[ly + 1][lx + 1][2] = mid[2];
    }
    __syncthreads();

    // ---- fluxes: x faces then y faces; the world's edge faces by the edge mode (hydro.rs:564-582, 744-775)
    for (int k = tid; k < (TX + 1) * TY + TX * (TY + 1); k += NT) {
        float f[4];
        if (k < (TX + 1) * TY) {
            int i = k % (TX + 1), j = k / (TX + 1);
            int X = x0 + i;
            const Face& L = i == 0 ? sh.FL[j] : sh.F[1][j][i - 1];
            const Face& R = i == TX ? sh.FR[j] : sh.F[0][j][i];
            if (X > w || y0 + j >= h) {
                f[0] = f[1] = f[2] = f[3] = 0.0f;
            } else if (X == 0) {
                if (H.edge == SR_EDGE_BOUNCE) {
                    wall(R, 0, f);
                } else {
                    hll(H, L, R, 0, f);
                    if (f[0] > 0.0f) wall(R, 0, f);
                }
            } else if (X == w) {
                if (H.edge == SR_EDGE_BOUNCE) {
                    wall(L, 0, f);
                } else {
                    hll(H, L, R, 0, f);
                    if (f[0] < 0.0f) wall(L, 0, f);
                }
            } else {
                hll(H, L, R, 0, f);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) sh.FX[j][i][q] = f[q];
        } else {
            int kk = k - (TX + 1) * TY;
            int i = kk % TX, j = kk / TX;
            int Y = y0 + j;
            const Face& L = j == 0 ? sh.FT[i] : sh.F[3][j - 1][i];
            const Face& R = j == TY ? sh.FB[i] : sh.F[2][j][i];
            if (Y > h || x0 + i >= w) {
                f[0] = f[1] = f[2] = f[3] = 0.0f;
            } else if (Y == 0) {
                if (H.edge == SR_EDGE_BOUNCE) {
                    wall(R, 1, f);
                } else {
                    hll(H, L, R, 1, f);
                    if (f[0] > 0.0f) wall(R, 1, f);
                }
            } else if (Y == h) {
                if (H.edge == SR_EDGE_BOUNCE) {
                    wall(L, 1, f);
                } else {
                    hll(H, L, R, 1, f);
                    if (f[0] < 0.0f) wall(L, 1, f);
                }
            } else {
                hll(H, L, R, 1, f);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) sh.FY[j][i][q] = f[q];
        }
    }
    __syncthreads();

    // ---- epilogue: one thread per tile cell
    const int lx = tid % TX, ly = tid / TX;
    const int X = x0 + lx, Y = y0 + ly;
    const bool inside = X < w && Y < h;
    const size_t i = (size_t)Y * w + X;
    // a cell with no gas around it stays empty (hydro.rs:733-742); out-of-world neighbours read as vacuum
    const int sx = lx + 2, sy = ly + 2;
    const float sv = H.sigma_vac;
    const bool vac = sh.S[sy][sx] < sv;
    const bool empty = vac && sh.S[sy][sx - 1] < sv && sh.S[sy][sx + 1] < sv && sh.S[sy - 1][sx] < sv &&
                       sh.S[sy + 1][sx] < sv;
    const float* fl = sh.FX[ly][lx];
    const float* fr = sh.FX[ly][lx + 1];
    const float* fu = sh.FY[ly][lx];
    const float* fd = sh.FY[ly + 1][lx];

    if (MODE == kHydroSource) {
        if (!inside) return;
        float s;
        if (empty) {
            s = 0.0f;
        } else {
            float start = vac ? sh.P[sy][sx].x : sh.S[sy][sx];
            float div = (fr[0] - fl[0]) + (fd[0] - fu[0]);
            s = 0.5f * (sh.S[sy][sx] + (start - dt * div));
        }
        A.src[i] = s >= sv ? s : 0.0f;
        return;
    }

    double kick_acc[2] = {0.0, 0.0};
    float best = 0.0f;
    int best_i = -1;
    double esc[4] = {0.0, 0.0, 0.0, 0.0};
    if (inside) {
        float u[4];
        if (empty) {
            u[0] = A.U[i]; u[1] = A.U[n + i]; u[2] = A.U[2 * n + i]; u[3] = A.U[3 * n + i];
        } else {
            if (vac) {
                eos_cons(H, P_at(sh, sy, sx), u);
            } else {
                u[0] = A.U[i]; u[1] = A.U[n + i]; u[2] = A.U[2 * n + i]; u[3] = A.U[3 * n + i];
            }
#pragma unroll
            for (int q = 0; q < 4; q++) u[q] -= dt * ((fr[q] - fl[q]) + (fd[q] - fu[q]));
            if (MODE == kHydroUpdateGrav) {
                const float* m = sh.M[ly + 1][lx + 1];
                float src = A.src[i];
                float kick[2] = {dt * src * A.gxm[i], dt * src * A.gym[i]};
                kick_acc[0] = (double)kick[0];
                kick_acc[1] = (double)kick[1];
                if (src > 0.0f) {
                    best = src;
                    best_i = (int)i;
                }
                float p = A.phim[i];
                float pr = p, pl = p, pd = p, pu = p;
                const float *mr = m, *ml = m, *md = m, *mu = m;
                if (X + 1 < w) { pr = A.phim[i + 1]; mr = sh.M[ly + 1][lx + 2]; }
                if (X > 0) { pl = A.phim[i - 1]; ml = sh.M[ly + 1][lx]; }
                if (Y + 1 < h) { pd = A.phim[i + w]; md = sh.M[ly + 2][lx + 1]; }
                if (Y > 0) { pu = A.phim[i - w]; mu = sh.M[ly][lx + 1]; }
                float r[3], l[3], dn[3], up[3];
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
            // escaped (hydro.rs:948-973): the boundary faces' fluxes as the cell took them
            float phi_edge = MODE == kHydroUpdateGrav ? A.phim[i] : 0.0f;
            if (X == 0) { for (int q = 0; q < 4; q++) esc[q] -= (double)(dt * fl[q]); esc[3] -= (double)(dt * fl[0] * phi_edge); }
            if (X + 1 == w) { for (int q = 0; q < 4; q++) esc[q] += (double)(dt * fr[q]); esc[3] += (double)(dt * fr[0] * phi_edge); }
            if (Y == 0) { for (int q = 0; q < 4; q++) esc[q] -= (double)(dt * fu[q]); esc[3] -= (double)(dt * fu[0] * phi_edge); }
            if (Y + 1 == h) { for (int q = 0; q < 4; q++) esc[q] += (double)(dt * fd[q]); esc[3] += (double)(dt * fd[0] * phi_edge); }
        }
        A.Uout[i] = u[0];
        A.Uout[n + i] = u[1];
        A.Uout[2 * n + i] = u[2];
        A.Uout[3 * n + i] = u[3];
    }

    // ---- per-CTA partials in a fixed order: Σ kicks (FP64), the densest cell (max src, lowest index), Σ escaped
    __shared__ double red_d[6][NT / 32];
    __shared__ float red_best[NT / 32];
    __shared__ int red_idx[NT / 32];
    const int lane = tid & 31, warp = tid >> 5;
    double vals[6] = {kick_acc[0], kick_acc[1], esc[0], esc[1], esc[2], esc[3]};
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double v = vals[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red_d[q][warp] = v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ob = __shfl_down_sync(0xffffffffu, best, o);
        int oi = __shfl_down_sync(0xffffffffu, best_i, o);
        if (oi >= 0 && (best_i < 0 || ob > best || (ob == best && oi < best_i))) {
            best = ob;
            best_i = oi;
        }
    }
    if (lane == 0) {
        red_best[warp] = best;
        red_idx[warp] = best_i;
    }
    __syncthreads();
    if (tid == 0) {
        const int b = blockIdx.y * gridDim.x + blockIdx.x;
        for (int q = 0; q < 6; q++) {
            double t = 0.0;
            for (int k = 0; k < NT / 32; k++) t += red_d[q][k];
            A.part_d[(size_t)b * 6 + q] = t;
        }
        float bb = 0.0f;
        int bi = -1;
        for (int k = 0; k < NT / 32; k++) {
            int oi = red_idx[k];
            float ob = red_best[k];
            if (oi >= 0 && (bi < 0 || ob > bb || (ob == bb && oi < bi))) {
                bb = ob;
                bi = oi;
            }
        }
        A.part_best[b] = bb;
        A.part_idx[b] = bi;
    }
}

// The net kick on the gas's own field taken back from the densest cell (hydro.rs:1004-1012), and the escaped totals,
// summed over the CTAs' partials in CTA order by one CTA.
__global__ void hydro_finalize_kernel(HydroArgs A, int nblocks, int take_back) {
    __shared__ double sd[6][256];
    __shared__ float sb[256];
    __shared__ int si[256];
    const int tid = threadIdx.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    float best = 0.0f;
    int bi = -1;
    // each thread sums a contiguous run of CTAs, so the order is fixed
    int per = (nblocks + 255) / 256;
    for (int b = tid * per; b < min(nblocks, (tid + 1) * per); b++) {
        for (int q = 0; q < 6; q++) acc[q] += A.part_d[(size_t)b * 6 + q];
        int oi = A.part_idx[b];
        float ob = A.part_best[b];
        if (oi >= 0 && (bi < 0 || ob > best || (ob == best && oi < bi))) {
            best = ob;
            bi = oi;
        }
    }
    for (int q = 0; q < 6; q++) sd[q][tid] = acc[q];
    sb[tid] = best;
    si[tid] = bi;
    __syncthreads();
    if (tid == 0) {
        double t[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 256; k++)
            for (int q = 0; q < 6; q++) t[q] += sd[q][k];
        float bb = 0.0f;
        int idx = -1;
        for (int k = 0; k < 256; k++) {
            int oi = si[k];
            float ob = sb[k];
            if (oi >= 0 && (idx < 0 || ob > bb || (ob == bb && oi < idx))) {
                bb = ob;
                idx = oi;
            }
        }
        const size_t n = (size_t)A.H.w * A.H.h;
        if (take_back && idx >= 0) {
            A.Uout[n + idx] -= (float)t[0];
            A.Uout[2 * n + idx] -= (float)t[1];
        }
        A.report[0] = t[0];
        A.report[1] = t[1];
        A.report[2] = (double)idx;
        for (int q = 0; q < 4; q++) A.report[3 + q] += t[2 + q];  // escaped accumulates over steps
    }
}

}  // namespace

size_t hydro_smem_bytes() { return sizeof(Shared); }

int hydro_blocks(int w, int h) { return (int)(div_up(w, TX) * div_up(h, TY)); }

void hydro_launch(int mode, const HydroArgs& A, cudaStream_t s) {
    dim3 grid(div_up(A.H.w, TX), div_up(A.H.h, TY));
    size_t smem = sizeof(Shared);
    switch (mode) {
        case kHydroUpdate:
            cudaFuncSetAttribute(hydro_tile_kernel<kHydroUpdate>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            hydro_tile_kernel<kHydroUpdate><<<grid, NT, smem, s>>>(A);
    sr_note_launch();
            break;
        case kHydroSource:
            cudaFuncSetAttribute(hydro_tile_kernel<kHydroSource>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            hydro_tile_kernel<kHydroSource><<<grid, NT, smem, s>>>(A);
    sr_note_launch();
            break;
        default:
            cudaFuncSetAttribute(hydro_tile_kernel<kHydroUpdateGrav>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            hydro_tile_kernel<kHydroUpdateGrav><<<grid, NT, smem, s>>>(A);
    sr_note_launch();
            break;
    }
}

void hydro_finalize_launch(const HydroArgs& A, int take_back, cudaStream_t s) {
    hydro_finalize_kernel<<<1, 256, 0, s>>>(A, hydro_blocks(A.H.w, A.H.h), take_back);
    sr_note_launch();
}

// ------------------------------------------------------------------------------------------------ P8 + P9
// P8's vacuum reset and thermal floor (reference/floors.rs:124-196, Σ_vac and Σ_floor as the planes' f32), then P9's
// per-cell Δt terms (hydro.rs:618-634): the wave rate (|u|+c)+(|v|+c) of the floored state and |g| of the step's P2
// field, reduced per CTA with the non-finite guard (reduce.wgsl's exit-5 scan: the first (cell, channel) not finite).
__global__ void floors_dt_kernel(HydroConst H, float* __restrict__ U, const float* __restrict__ gx,
                                 const float* __restrict__ gy, int do_floors, float* part_rate, float* part_g,
                                 long long* part_nf) {
    const size_t n = (size_t)H.w * H.h;
    float rate = 0.0f, gmax = 0.0f;
    long long nf = LLONG_MAX;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float s = U[i], mx = U[n + i], my = U[2 * n + i], e = U[3 * n + i];
        if (do_floors) {
            if (s < H.sigma_vac) {
                s = H.sigma_floor;
                mx = 0.0f;
                my = 0.0f;
                e = H.sigma_floor * H.eps_floor;
                U[i] = s; U[n + i] = mx; U[2 * n + i] = my; U[3 * n + i] = e;
            } else {
                float kinetic = 0.5f * (mx * mx + my * my) / (s * s);
                float raw = e / s - kinetic;
                if (raw < H.eps_floor) {
                    e = e + s * (H.eps_floor - raw);
                    U[3 * n + i] = e;
                }
            }
        }
        if (!(isfinite(s) && isfinite(mx) && isfinite(my) && isfinite(e))) {
            int c = !isfinite(s) ? 0 : (!isfinite(mx) ? 1 : (!isfinite(my) ? 2 : 3));
            long long code = (long long)i * 4 + c;
            nf = code < nf ? code : nf;
        }
        Prim p = eos_read(H, s, mx, my, e);
        float c = eos_sound(H, p);
        float r = (fabsf(p.u) + c) + (fabsf(p.v) + c);
        rate = fmaxf(rate, r);
        if (gx) gmax = fmaxf(gmax, hypotf(gx[i], gy[i]));
    }
    __shared__ float sr[32], sg[32];
    __shared__ long long sn[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rate = fmaxf(rate, __shfl_down_sync(0xffffffffu, rate, o));
        gmax = fmaxf(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
        long long on = __shfl_down_sync(0xffffffffu, nf, o);
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

// Δt_{n+1} = min(C / max rate, η_g / sqrt(max |g|)) (hydro.rs:618-634), the configured fixed Δt or cap, and the guard.
__global__ void dt_finalize_kernel(int nblocks, const float* part_rate, const float* part_g, const long long* part_nf,
                                   double cfl, double eta_g, double dt_fixed, double dt_cap, DtRecord* rec) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float rate = 0.0f, gmax = 0.0f;
    long long nf = LLONG_MAX;
    for (int b = 0; b < nblocks; b++) {
        rate = fmaxf(rate, part_rate[b]);
        gmax = fmaxf(gmax, part_g[b]);
        nf = part_nf[b] < nf ? part_nf[b] : nf;
    }
    double dt = cfl / (double)rate;
    if (gmax > 0.0f) dt = fmin(dt, eta_g / sqrt((double)gmax));
    if (dt_fixed > 0.0) dt = dt_fixed;
    if (dt_cap > 0.0) dt = fmin(dt, dt_cap);
    rec->dt_next = dt;
    if (nf != LLONG_MAX && !rec->non_finite) {
        rec->non_finite = 1;
        rec->nf_cell = nf / 4;
        rec->nf_channel = (int)(nf % 4);
        rec->nf_step = rec->steps;
    }
}

// P1: this step runs on Δt_n = the last P9's Δt_{n+1} and adds it to the sim time (f64).
__global__ void dt_advance_kernel(DtRecord* rec) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    rec->dt = rec->dt_next;
    rec->sim_time += rec->dt;
    rec->steps += 1;
}

int floors_dt_blocks(int w, int h) {
    size_t n = (size_t)w * h;
    int b = (int)div_up((unsigned)((n + 3) / 4), 256u);
    return b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b);
}

void floors_dt_launch(const HydroConst& H, float* U, const float* gx, const float* gy, int do_floors, float* part_rate,
                      float* part_g, long long* part_nf, double cfl, double eta_g, double dt_fixed, double dt_cap,
                      DtRecord* rec, cudaStream_t s) {
    int nb = floors_dt_blocks(H.w, H.h);
    floors_dt_kernel<<<nb, 256, 0, s>>>(H, U, gx, gy, do_floors, part_rate, part_g, part_nf);
    sr_note_launch();
    dt_finalize_kernel<<<1, 32, 0, s>>>(nb, part_rate, part_g, part_nf, cfl, eta_g, dt_fixed, dt_cap, rec);
    sr_note_launch();
}

void dt_advance_launch(DtRecord* rec, cudaStream_t s) { dt_advance_kernel<<<1, 32, 0, s>>>(rec);
    sr_note_launch(); }
