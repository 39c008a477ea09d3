// hydro.cu — P4, the MUSCL-Hancock/HLL gas step, as one tiled stencil kernel per pass (sm_100a, FP32).
//
// One CTA owns a tile of output cells; the tile grown by two cells (the reconstruction's reach) arrives in shared
// memory by one TMA box, the world's ghosts are formed there, every lane runs the Hancock predictor for one cell (the
// tile's and the one-cell ring around it), the faces meet for the HLL fluxes by warp shuffles (x) and shared memory
// (y), and the per-cell epilogue of the pass finishes:
//   - kHydroUpdate:     U' = U - Δt ΔF (no gravity);
//   - kHydroSource:     the half step's gravity source ½(Σⁿ + Σⁿ⁺¹), masked (reference hydro.rs:815-836);
//   - kHydroUpdateGrav: U' with gravity's half-step kick and the faces' work across φ_mid (hydro.rs:871-947).
// The scheme follows crates/sr-physics/src/reference/hydro.rs (step_held without held cells, sinks or radiation).
#include "hydro.cuh"

#include <cudaTypedefs.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "tma.cuh"

namespace {

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

template <int LIM>
__device__ __forceinline__ float lim(float l, float c, float r) {
    return LIM == SR_LIMITER_MINMOD ? lim_minmod(l, c, r) : lim_mc(l, c, r);
}

// Limited slopes of (Σ, u, v, Π) along one axis; Σ and Π flat where the thermal bracket refuses a face
// (hydro.rs:293-331, HOT_FACE = 2). The limiter and the bracket are the kernel's template parameters.
template <int LIM, bool BRACKET>
__device__ __forceinline__ Prim slope(const Prim& l, const Prim& c, const Prim& r, float ql, float qc, float qr) {
    Prim s;
    s.s = lim<LIM>(l.s, c.s, r.s);
    s.u = lim<LIM>(l.u, c.u, r.u);
    s.v = lim<LIM>(l.v, c.v, r.v);
    s.p = lim<LIM>(l.p, c.p, r.p);
    if (BRACKET) {
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

// Gravity's source at one face over the step (hydro.rs:1042-1067): [impulse to the low cell, low energy, high energy].
__device__ __forceinline__ void face_work(float q, float sl, float sh, float pl, float ph, float d, float dt, float* o) {
    float a = fmaxf(sl, 0.0f), b = fmaxf(sh, 0.0f);
    float w = a + b > 0.0f ? sr_div(a, a + b) : 0.5f;
    float extra = dt * (q - 0.5f * (pl + ph)) * d;
    float c = 0.0f, kick = 0.0f, el = 0.0f, eh = 0.0f;
    if (extra < 0.0f && a > 0.0f && b > 0.0f) {
        float ul = sr_div(pl, a), uh = sr_div(ph, b);
        float du = ul - uh;
        float inv = sr_div(1.0f, a) + sr_div(1.0f, b);
        c = fminf(-extra, sr_div(0.25f * du * du, inv));
        if (c > 0.0f) {
            float disc = sr_sqrt(du * du - 2.0f * inv * c);
            kick = sr_div(-2.0f * c, du + copysignf(1.0f, du) * disc);
            el = ul * kick + sr_div(0.5f * kick * kick, a);
            eh = -uh * kick + sr_div(0.5f * kick * kick, b);
        }
    }
    float rest = extra + c;
    o[0] = kick;
    o[1] = 0.5f * dt * pl * d + w * rest + el;
    o[2] = 0.5f * dt * ph * d + (1.0f - w) * rest + eh;
}

// ---- the band kernel: one warp per row of the tile, one lane per cell
//
// A CTA covers HB_TX x HB_TY output cells with HB_W = HB_TY + 2 warps of 32 lanes: warp r is the row y0 - 1 + r and
// lane l the column x0 - 1 + l, so the ring of cells around the tile (whose faces toward the tile the fluxes need) is
// computed by the same straight-line code as the tile itself: lanes 0 and 31 and warps 0 and HB_W - 1 predict but
// write nothing. The four planes of the tile grown by two cells (the reconstruction's reach) arrive in one TMA box;
// the world's ghosts (hydro.rs:686-709) are formed from it in shared memory. Each lane predicts its cell's four faces
// (hydro.rs:587-614); the x faces meet by warp shuffles (a lane's x+ face against the next lane's x- face), the y faces
// through shared memory (a row's y+ faces against the next row's y- faces); the fluxes go back the same ways.
constexpr int HB_TX = 30, HB_TY = 14, HB_W = HB_TY + 2, HB_NT = 32 * HB_W;
constexpr int HB_SX = HB_TX + 4, HB_SY = HB_TY + 4;  // the staged region: the tile grown by 2
constexpr int HB_BX = 40, HB_BY = HB_SY;             // the TMA box: from a 16-byte aligned column, wide enough
constexpr uint32_t kHydroWaitPolls = 1u << 24;       // an mbarrier wait gives up after this many polls

// A predicted face: its conserved vector and the primitives it stands for (Σ is U0).
struct FaceS {
    float U0, U1, U2, U3, u, v, P;
};

struct __align__(128) BandShared {
    float raw[4][HB_BY][HB_BX];  // the TMA box of Σ, Σu, Σv, E (first: 128-byte aligned)
    float4 P[HB_SY][HB_SX];      // primitives (Σ, u, v, Π) of the staged region, ghosts included
    float Q[HB_SY][HB_SX];       // Π/Σ (the thermal bracket's temperatures)
    float S[HB_SY][HB_SX];       // raw Σ (out of the world: -1, read as vacuum)
    float M[3][HB_W][32];        // half-step (Σ, Σu, Σv) of each lane's cell
    float YF[7][HB_W][32];       // each lane's y+ face
    float FY[4][HB_W][32];       // the flux through each lane's top face
    double red_d[6][HB_W];
    float red_best[HB_W];
    int red_idx[HB_W];
    uint64_t mbar;
};

__device__ __forceinline__ Prim prim_at(const BandShared& sh, int y, int x) {
    const float4 q = sh.P[y][x];
    Prim p;
    p.s = q.x; p.u = q.y; p.v = q.z; p.p = q.w;
    return p;
}

// The Euler flux of the unevolved face c + f s normal to `dir` (the Hancock increment's terms).
__device__ __forceinline__ void face_flux(const HydroConst& H, const Prim& c, const Prim& s, float f, int dir,
                                          float* out) {
    const Prim wf = offset(c, s, f);
    float uf[4];
    eos_cons(H, wf, uf);
    euler_flux(wf, uf[3], dir, out);
}

// The face c + f s advanced by the Hancock increment and gravity's half-kick, or unevolved when the advanced one is no
// state (hydro.rs:501-513, 587-614).
__device__ __forceinline__ FaceS face_state(const HydroConst& H, const Prim& c, const Prim& s, float f,
                                            const float* delta, float half, bool grav, float gx, float gy) {
    const Prim wf = offset(c, s, f);
    float uf[4];
    eos_cons(H, wf, uf);
    float d[4] = {delta[0], delta[1], delta[2], delta[3]};
    if (grav) {
        d[1] += half * wf.s * gx;
        d[2] += half * wf.s * gy;
        d[3] += half * wf.s * ((wf.u + 0.5f * half * gx) * gx + (wf.v + 0.5f * half * gy) * gy);
    }
    const float U[4] = {uf[0] + d[0], uf[1] + d[1], uf[2] + d[2], uf[3] + d[3]};
    Prim p;
    FaceS F;
    if (eos_prim(H, U, p)) {
        F.U0 = U[0]; F.U1 = U[1]; F.U2 = U[2]; F.U3 = U[3];
        F.u = p.u; F.v = p.v; F.P = p.p;
    } else {
        F.U0 = uf[0]; F.U1 = uf[1]; F.U2 = uf[2]; F.U3 = uf[3];
        F.u = wf.u; F.v = wf.v; F.P = wf.p;
    }
    return F;
}

__device__ __forceinline__ FaceS shfl_face_down(const FaceS& F) {
    FaceS R;
    R.U0 = __shfl_down_sync(0xffffffffu, F.U0, 1);
    R.U1 = __shfl_down_sync(0xffffffffu, F.U1, 1);
    R.U2 = __shfl_down_sync(0xffffffffu, F.U2, 1);
    R.U3 = __shfl_down_sync(0xffffffffu, F.U3, 1);
    R.u = __shfl_down_sync(0xffffffffu, F.u, 1);
    R.v = __shfl_down_sync(0xffffffffu, F.v, 1);
    R.P = __shfl_down_sync(0xffffffffu, F.P, 1);
    return R;
}

__device__ __forceinline__ void flux_of(const FaceS& F, int dir, float* f) {
    Prim p;
    p.s = F.U0; p.u = F.u; p.v = F.v; p.p = F.P;
    euler_flux(p, F.U3, dir, f);
}

// HLL with Davis speeds across a face normal to `dir` (hydro.rs:516-540).
__device__ __forceinline__ void hll_s(const HydroConst& H, const FaceS& l, const FaceS& r, int dir, float* f) {
    const float unl = dir == 0 ? l.u : l.v, unr = dir == 0 ? r.u : r.v;
    const float cl = sr_sqrt(H.gamma * sr_div(l.P, l.U0)), cr = sr_sqrt(H.gamma * sr_div(r.P, r.U0));
    const float s_l = fminf(unl - cl, unr - cr);
    const float s_r = fmaxf(unl + cl, unr + cr);
    float fl[4], fr[4];
    flux_of(l, dir, fl);
    flux_of(r, dir, fr);
    if (s_l >= 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = fl[k];
    } else if (s_r <= 0.0f) {
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = fr[k];
    } else {
        const float inv = sr_div(1.0f, s_r - s_l);
        const float dU[4] = {r.U0 - l.U0, r.U1 - l.U1, r.U2 - l.U2, r.U3 - l.U3};
#pragma unroll
        for (int k = 0; k < 4; k++) f[k] = (s_r * fl[k] - s_l * fr[k] + s_l * s_r * dU[k]) * inv;
    }
}

__device__ __forceinline__ void wall_s(const FaceS& own, int dir, float* f) {  // hydro.rs:556-562
    f[0] = 0.0f; f[1] = 0.0f; f[2] = 0.0f; f[3] = 0.0f;
    f[1 + dir] = own.P;
}

// The flux through face `at` (along `dir`) of the world (0 and `edge` are its walls; hydro.rs:564-582, 744-775),
// between the faces L and R; zero for a face outside the world (`inside` false).
__device__ __forceinline__ void face_flux_at(const HydroConst& H, const FaceS& L, const FaceS& R, int dir, int at,
                                             int edge, bool inside, float* f) {
    if (!inside || at < 0 || at > edge) {
        f[0] = f[1] = f[2] = f[3] = 0.0f;
    } else if (at == 0) {
        if (H.edge == SR_EDGE_BOUNCE) {
            wall_s(R, dir, f);
        } else {
            hll_s(H, L, R, dir, f);
            if (f[0] > 0.0f) wall_s(R, dir, f);
        }
    } else if (at == edge) {
        if (H.edge == SR_EDGE_BOUNCE) {
            wall_s(L, dir, f);
        } else {
            hll_s(H, L, R, dir, f);
            if (f[0] < 0.0f) wall_s(L, dir, f);
        }
    } else {
        hll_s(H, L, R, dir, f);
    }
}

template <int MODE, int LIM, bool BRACKET>
__global__ void __launch_bounds__(HB_NT, 2) hydro_band_kernel(const __grid_constant__ CUtensorMap map, HydroArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BandShared& sh = *reinterpret_cast<BandShared*>(smem_raw);
    const HydroConst H = A.H;
    const int w = H.w, h = H.h;
    const size_t n = (size_t)w * h;
    const int tid = threadIdx.x, lane = tid & 31, row = tid >> 5;
    const int x0 = blockIdx.x * HB_TX, y0 = blockIdx.y * HB_TY;
    const int xs = (x0 - 2) & ~3, ys = y0 - 2;  // the box's origin: x on a 16-byte boundary
    const float dt = (float)(*A.dt);
    const float half = 0.5f * dt;
    const bool grav = A.gx != nullptr;

    // ---- the four planes of the staged region by one TMA box; every wait is bounded
    if (tid == 0) {
        tc::mbar_init(&sh.mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        tma::expect_tx(&sh.mbar, (uint32_t)sizeof(sh.raw));
        tma::load_3d(&sh.raw[0][0][0], &map, xs, ys, 0, &sh.mbar);
    }
    const bool landed = tc::mbar_wait(&sh.mbar, 0, kHydroWaitPolls);
    if (__syncthreads_or(!landed)) {
        if (tid == 0) atomicOr(A.err, 1);
        tc::mbar_wait(&sh.mbar, 0, kHydroWaitPolls);  // the copy still in flight lands before the CTA leaves
        return;
    }

    // ---- primitives of the staged region: world cells, or ghosts past the edges (bounce mirrors the cells beyond
    // with the normal velocity negated, leave copies the edge cell with it clamped outward)
    for (int k = tid; k < HB_SY * HB_SX; k += HB_NT) {
        const int ly = k / HB_SX, lx = k - ly * HB_SX;
        const int x = x0 - 2 + lx, y = y0 - 2 + ly;
        Prim p;
        float raw = -1.0f;
        if (x >= -2 && x <= w + 1 && y >= -2 && y <= h + 1) {
            const bool xo = x < 0 || x >= w, yo = y < 0 || y >= h;
            int cx, cy;
            if (H.edge == SR_EDGE_BOUNCE) {
                cx = x < 0 ? -x - 1 : (x >= w ? 2 * w - 1 - x : x);
                cy = y < 0 ? -y - 1 : (y >= h ? 2 * h - 1 - y : y);
            } else {
                cx = min(max(x, 0), w - 1);
                cy = min(max(y, 0), h - 1);
            }
            const int bx = cx - xs, by = cy - ys;
            const float s = sh.raw[0][by][bx];
            p = eos_read(H, s, sh.raw[1][by][bx], sh.raw[2][by][bx], sh.raw[3][by][bx]);
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
        } else {
            p.s = 1.0f; p.u = 0.0f; p.v = 0.0f; p.p = 1.0f;  // past every ghost: never reaches a kept cell
        }
        sh.P[ly][lx] = make_float4(p.s, p.u, p.v, p.p);
        sh.Q[ly][lx] = sr_div(p.p, p.s);
        sh.S[ly][lx] = raw;
    }
    __syncthreads();

    // ---- this lane's cell: slopes, the Hancock increment and the half-step centre (hydro.rs:587-614)
    const int sx = lane + 1, sy = row + 1;  // the cell in the staged region
    const int X = x0 - 1 + lane, Y = y0 - 1 + row;
    const Prim c = prim_at(sh, sy, sx);
    const Prim slx = slope<LIM, BRACKET>(prim_at(sh, sy, sx - 1), c, prim_at(sh, sy, sx + 1), sh.Q[sy][sx - 1],
                                         sh.Q[sy][sx], sh.Q[sy][sx + 1]);
    const Prim sly = slope<LIM, BRACKET>(prim_at(sh, sy - 1, sx), c, prim_at(sh, sy + 1, sx), sh.Q[sy - 1][sx],
                                         sh.Q[sy][sx], sh.Q[sy + 1][sx]);
    float gxv = 0.0f, gyv = 0.0f;
    if (grav) {  // a ghost takes its edge cell's g
        const size_t gi = (size_t)min(max(Y, 0), h - 1) * w + min(max(X, 0), w - 1);
        gxv = A.gx[gi];
        gyv = A.gy[gi];
    }
    float delta[4];
    {
        float a[4], b[4], dxs[4];
        face_flux(H, c, slx, -0.5f, 0, a);
        face_flux(H, c, slx, 0.5f, 0, b);
#pragma unroll
        for (int k = 0; k < 4; k++) dxs[k] = a[k] - b[k];
        face_flux(H, c, sly, -0.5f, 1, a);
        face_flux(H, c, sly, 0.5f, 1, b);
#pragma unroll
        for (int k = 0; k < 4; k++) delta[k] = half * (dxs[k] + (a[k] - b[k]));
    }
    {
        float m1 = c.s * c.u + delta[1], m2 = c.s * c.v + delta[2];
        if (grav) {
            m1 += half * c.s * gxv;
            m2 += half * c.s * gyv;
        }
        sh.M[0][row][lane] = c.s + delta[0];
        sh.M[1][row][lane] = m1;
        sh.M[2][row][lane] = m2;
    }

    // ---- x faces: this lane's x+ face against the next lane's x- face; the left face's flux from the lane before
    float fr[4], fl[4];
    {
        const FaceS R = shfl_face_down(face_state(H, c, slx, -0.5f, delta, half, grav, gxv, gyv));
        const FaceS L = face_state(H, c, slx, 0.5f, delta, half, grav, gxv, gyv);
        face_flux_at(H, L, R, 0, X + 1, w, Y >= 0 && Y < h, fr);
#pragma unroll
        for (int k = 0; k < 4; k++) fl[k] = __shfl_up_sync(0xffffffffu, fr[k], 1);
    }
    // ---- y faces: the row above's y+ faces against this row's y- faces, through shared memory
    {
        const FaceS T = face_state(H, c, sly, 0.5f, delta, half, grav, gxv, gyv);
        sh.YF[0][row][lane] = T.U0;
        sh.YF[1][row][lane] = T.U1;
        sh.YF[2][row][lane] = T.U2;
        sh.YF[3][row][lane] = T.U3;
        sh.YF[4][row][lane] = T.u;
        sh.YF[5][row][lane] = T.v;
        sh.YF[6][row][lane] = T.P;
    }
    const FaceS B = face_state(H, c, sly, -0.5f, delta, half, grav, gxv, gyv);
    __syncthreads();
    if (row >= 1) {
        FaceS L;
        L.U0 = sh.YF[0][row - 1][lane];
        L.U1 = sh.YF[1][row - 1][lane];
        L.U2 = sh.YF[2][row - 1][lane];
        L.U3 = sh.YF[3][row - 1][lane];
        L.u = sh.YF[4][row - 1][lane];
        L.v = sh.YF[5][row - 1][lane];
        L.P = sh.YF[6][row - 1][lane];
        float ft[4];
        face_flux_at(H, L, B, 1, Y, h, X >= 0 && X < w, ft);
#pragma unroll
        for (int k = 0; k < 4; k++) sh.FY[k][row][lane] = ft[k];
    }
    __syncthreads();

    // ---- epilogue: the tile's cells
    const bool inside = lane >= 1 && lane <= HB_TX && row >= 1 && row <= HB_TY && X < w && Y < h;
    const size_t i = inside ? (size_t)Y * w + X : 0;
    float fu[4], fd[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        fu[k] = row >= 1 ? sh.FY[k][row][lane] : 0.0f;
        fd[k] = row + 1 < HB_W ? sh.FY[k][row + 1][lane] : 0.0f;
    }
    // a cell with no gas around it stays empty (hydro.rs:733-742); out-of-world neighbours read as vacuum
    const float sv = H.sigma_vac;
    const bool vac = sh.S[sy][sx] < sv;
    const bool empty = vac && sh.S[sy][sx - 1] < sv && sh.S[sy][sx + 1] < sv && sh.S[sy - 1][sx] < sv &&
                       sh.S[sy + 1][sx] < sv;

    if (MODE == kHydroSource) {
        if (!inside) return;
        float s;
        if (empty) {
            s = 0.0f;
        } else {
            const float start = vac ? sh.P[sy][sx].x : sh.S[sy][sx];
            const float div = (fr[0] - fl[0]) + (fd[0] - fu[0]);
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
        const int bx = X - xs, by = Y - ys;
        float u[4];
        if (empty || !vac) {
            u[0] = sh.raw[0][by][bx]; u[1] = sh.raw[1][by][bx]; u[2] = sh.raw[2][by][bx]; u[3] = sh.raw[3][by][bx];
        } else {
            eos_cons(H, c, u);
        }
        if (!empty) {
#pragma unroll
            for (int q = 0; q < 4; q++) u[q] -= dt * ((fr[q] - fl[q]) + (fd[q] - fu[q]));
            if (MODE == kHydroUpdateGrav) {
                const float m[3] = {sh.M[0][row][lane], sh.M[1][row][lane], sh.M[2][row][lane]};
                const float src = A.src[i];
                float kick[2] = {dt * src * A.gxm[i], dt * src * A.gym[i]};
                kick_acc[0] = (double)kick[0];
                kick_acc[1] = (double)kick[1];
                if (src > 0.0f) {
                    best = src;
                    best_i = (int)i;
                }
                const float p = A.phim[i];
                float pr = p, pl = p, pd = p, pu = p;
                float mr[3] = {m[0], m[1], m[2]}, ml[3] = {m[0], m[1], m[2]}, md[3] = {m[0], m[1], m[2]},
                      mu[3] = {m[0], m[1], m[2]};
                if (X + 1 < w) {
                    pr = A.phim[i + 1];
#pragma unroll
                    for (int q = 0; q < 3; q++) mr[q] = sh.M[q][row][lane + 1];
                }
                if (X > 0) {
                    pl = A.phim[i - 1];
#pragma unroll
                    for (int q = 0; q < 3; q++) ml[q] = sh.M[q][row][lane - 1];
                }
                if (Y + 1 < h) {
                    pd = A.phim[i + w];
#pragma unroll
                    for (int q = 0; q < 3; q++) md[q] = sh.M[q][row + 1][lane];
                }
                if (Y > 0) {
                    pu = A.phim[i - w];
#pragma unroll
                    for (int q = 0; q < 3; q++) mu[q] = sh.M[q][row - 1][lane];
                }
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
            const float phi_edge = MODE == kHydroUpdateGrav ? A.phim[i] : 0.0f;
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
    // a warp whose lanes hold no term skips its tree (interior rows hold no escaped flux; only the gravity pass kicks)
    double vals[6] = {kick_acc[0], kick_acc[1], esc[0], esc[1], esc[2], esc[3]};
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double v = vals[q];
        if (__any_sync(0xffffffffu, v != 0.0)) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        }
        if (lane == 0) sh.red_d[q][row] = v;
    }
    if (__any_sync(0xffffffffu, best_i >= 0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, best_i, o);
            if (oi >= 0 && (best_i < 0 || ob > best || (ob == best && oi < best_i))) {
                best = ob;
                best_i = oi;
            }
        }
    }
    if (lane == 0) {
        sh.red_best[row] = best;
        sh.red_idx[row] = best_i;
    }
    __syncthreads();
    if (tid == 0) {
        const int b = blockIdx.y * gridDim.x + blockIdx.x;
        for (int q = 0; q < 6; q++) {
            double t = 0.0;
            for (int k = 0; k < HB_W; k++) t += sh.red_d[q][k];
            A.part_d[(size_t)b * 6 + q] = t;
        }
        float bb = 0.0f;
        int bi = -1;
        for (int k = 0; k < HB_W; k++) {
            const int oi = sh.red_idx[k];
            const float ob = sh.red_best[k];
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


size_t hydro_smem_bytes() { return sizeof(BandShared); }

int hydro_blocks(int w, int h) { return (int)(div_up(w, HB_TX) * div_up(h, HB_TY)); }

void tma_encode_planes(CUtensorMap* map, const float* base, int w, int h, int planes, int bx, int by) {
    // encoded maps are kept by their arguments: a launch on the same planes (every launch of a step, every smoother
    // launch of a level) copies its map instead of paying the driver call before the launch
    static std::mutex mu;
    static std::map<std::tuple<const float*, int, int, int, int, int>, CUtensorMap> cache;
    const auto key = std::make_tuple(base, w, h, planes, bx, by);
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto it = cache.find(key);
        if (it != cache.end()) {
            *map = it->second;
            return;
        }
    }
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SR_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        SR_REQUIRE(q == cudaDriverEntryPointSuccess && fn, "the driver has no cuTensorMapEncodeTiled");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    SR_REQUIRE(w % 4 == 0 && ((uintptr_t)base & 15) == 0, "a TMA plane needs 16-byte rows and a 16-byte base");
    const cuuint64_t dims[3] = {(cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)w * sizeof(float), (cuuint64_t)w * h * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)planes};
    const cuuint32_t unit[3] = {1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                              unit, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw SrError{SR_E_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r)};
    std::lock_guard<std::mutex> lock(mu);
    if (cache.size() > 4096) cache.clear();
    cache[key] = *map;
}

template <int MODE, int LIM, bool BRACKET>
void hydro_launch_t(const CUtensorMap& map, const HydroArgs& A, cudaStream_t s) {
    static bool attr = false;  // the attribute of this instance, once per process
    if (!attr) {
        SR_CUDA_TRY(cudaFuncSetAttribute(hydro_band_kernel<MODE, LIM, BRACKET>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BandShared)));
        attr = true;
    }
    const dim3 grid(div_up(A.H.w, HB_TX), div_up(A.H.h, HB_TY));
    hydro_band_kernel<MODE, LIM, BRACKET><<<grid, HB_NT, sizeof(BandShared), s>>>(map, A);
    sr_note_launch();
}

template <int MODE>
void hydro_launch_m(const CUtensorMap& map, const HydroArgs& A, cudaStream_t s) {
    const bool mc = A.H.limiter != SR_LIMITER_MINMOD, br = A.H.bracket != 0;
    if (mc && br) hydro_launch_t<MODE, SR_LIMITER_MC, true>(map, A, s);
    else if (mc) hydro_launch_t<MODE, SR_LIMITER_MC, false>(map, A, s);
    else if (br) hydro_launch_t<MODE, SR_LIMITER_MINMOD, true>(map, A, s);
    else hydro_launch_t<MODE, SR_LIMITER_MINMOD, false>(map, A, s);
}

void hydro_launch(int mode, const HydroArgs& A, cudaStream_t s) {
    CUtensorMap map;
    tma_encode_planes(&map, A.U, A.H.w, A.H.h, 4, HB_BX, HB_BY);
    if (mode == kHydroUpdate) hydro_launch_m<kHydroUpdate>(map, A, s);
    else if (mode == kHydroSource) hydro_launch_m<kHydroSource>(map, A, s);
    else hydro_launch_m<kHydroUpdateGrav>(map, A, s);
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
// One CTA: each thread takes a strided share of the partials, then a shuffle and shared-memory tree (max and min are
// exact in any order, so the result does not depend on the split).
__global__ void dt_finalize_kernel(int nblocks, int channels, const float* part_rate, const float* part_g,
                                   const long long* part_nf, double cfl, double eta_g, double dt_fixed, double dt_cap,
                                   DtRecord* rec) {
    float rate = 0.0f, gmax = 0.0f;
    long long nf = LLONG_MAX;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        rate = fmaxf(rate, part_rate[b]);
        gmax = fmaxf(gmax, part_g[b]);
        nf = part_nf[b] < nf ? part_nf[b] : nf;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rate = fmaxf(rate, __shfl_down_sync(0xffffffffu, rate, o));
        gmax = fmaxf(gmax, __shfl_down_sync(0xffffffffu, gmax, o));
        const long long on = __shfl_down_sync(0xffffffffu, nf, o);
        nf = on < nf ? on : nf;
    }
    __shared__ float sr[32], sg[32];
    __shared__ long long sn[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sr[warp] = rate;
        sg[warp] = gmax;
        sn[warp] = nf;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int k = 1; k < (int)(blockDim.x / 32); k++) {
        rate = fmaxf(rate, sr[k]);
        gmax = fmaxf(gmax, sg[k]);
        nf = sn[k] < nf ? sn[k] : nf;
    }
    double dt = cfl / (double)rate;
    if (gmax > 0.0f) dt = fmin(dt, eta_g / sqrt((double)gmax));
    if (dt_fixed > 0.0) dt = dt_fixed;
    if (dt_cap > 0.0) dt = fmin(dt, dt_cap);
    rec->dt_next = dt;
    if (nf != LLONG_MAX && !rec->non_finite) {
        rec->non_finite = 1;
        rec->nf_cell = nf / channels;
        rec->nf_channel = (int)(nf % channels);
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
    dt_finalize_launch(nb, 4, part_rate, part_g, part_nf, cfl, eta_g, dt_fixed, dt_cap, rec, s);
}

void dt_finalize_launch(int nblocks, int channels, const float* part_rate, const float* part_g,
                        const long long* part_nf, double cfl, double eta_g, double dt_fixed, double dt_cap,
                        DtRecord* rec, cudaStream_t s) {
    dt_finalize_kernel<<<1, 256, 0, s>>>(nblocks, channels, part_rate, part_g, part_nf, cfl, eta_g, dt_fixed, dt_cap,
                                         rec);
    sr_note_launch();
}

void dt_advance_launch(DtRecord* rec, cudaStream_t s) { dt_advance_kernel<<<1, 32, 0, s>>>(rec);
    sr_note_launch(); }
