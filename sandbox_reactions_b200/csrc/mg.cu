// mg.cu — the multigrid V-cycle (FP32) of the implicit FLD solve; see mg.cuh for the scheme.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "mg.cuh"
#include "reduce.cuh"
#include "tma.cuh"

namespace {

// Smoother tiles (outputs; even, so a tile's 2x2 aggregates stay inside it): 64 x 32 with 512 threads on big levels,
// 32 x 16 with 256 threads where the big tile leaves fewer than 2 CTAs per SM (a quarter of the work per CTA: the
// small levels are bound by one CTA's latency).
constexpr int BIG_SX = 64, BIG_SY = 32, BIG_NT = 512;
constexpr int SMALL_SX = 32, SMALL_SY = 16, SMALL_NT = 256;
constexpr int TAIL_THREADS = 1024;
constexpr int TAIL_ROWS = TAIL_THREADS / 32;  // the tail's threads as 32 columns x TAIL_ROWS rows

// A tail level's arrays as offsets into the tail's shared memory (floats for the seven arrays, bytes for the mask).
struct TailLevel {
    int w, h;
    int c, dx, dy, b, x, inv, t;  // float offsets; inv: the inverse diagonal (0 on masked cells); t: the weights towards
                                  // the next coarser level
    int m;                        // byte offset of the mask
};

struct TailArgs {
    int t, nl, pre, post;
    float omega;
    int sinv;                 // float offset of the coarsest level's inverse (nc x nc)
    const float4* img;        // the tail's shared memory image (everything but the top level's b), per Newton pass
    int img_f4;               // its size in 16-byte words
    double* out;              // non-null when the tail's top level is level 0: <b, x2> written here
    MgLevel L[kMgMaxLevels];
    TailLevel T[kMgMaxLevels];
};

// Level 0's couplings to the +x / +y neighbours from the f64 faces, zero unless both cells are gas.
__global__ void mg_couplings0_kernel(MgLevel L, const double* __restrict__ kx, const double* __restrict__ ky,
                                     const uint8_t* __restrict__ gas) {
    const int w = L.w, h = L.h;
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y;
        split_index(i, w, x, y);
        const bool g = gas[i];
        L.mask[i] = g;
        L.dx[i] = (g && x + 1 < w && gas[i + 1]) ? (float)kx[(size_t)y * (w + 1) + x + 1] : 0.0f;
        L.dy[i] = (g && y + 1 < h && gas[i + w]) ? (float)ky[(size_t)(y + 1) * w + x] : 0.0f;
    }
}

// Level 1 from level 0: Galerkin aggregation of 2x2 cells with constant weights (mg.cuh). The mass term c sums over
// the aggregate's system cells; a coarse coupling sums the two fine couplings across the aggregates' shared side.
__global__ void mg_aggregate_kernel(MgLevel F, MgLevel C) {
    const int wc = C.w, hc = C.h, wf = F.w, hf = F.h;
    const size_t nc = (size_t)wc * hc;
    for (size_t I = (size_t)blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += (size_t)gridDim.x * blockDim.x) {
        const int X = (int)(I % wc), Y = (int)(I / wc);
        const int fx0 = 2 * X, fy0 = 2 * Y;
        const bool has_x1 = fx0 + 1 < wf, has_y1 = fy0 + 1 < hf;
        float c = 0.0f;
        bool any = false;
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int a = 0; a < 2; a++) {
                if ((a && !has_x1) || (b && !has_y1)) continue;
                size_t j = (size_t)(fy0 + b) * wf + fx0 + a;
                if (F.mask[j]) {
                    c += F.c[j];
                    any = true;
                }
            }
        float dxc = 0.0f, dyc = 0.0f;
        if (X + 1 < wc) {
            dxc = F.dx[(size_t)fy0 * wf + fx0 + 1];
            if (has_y1) dxc += F.dx[(size_t)(fy0 + 1) * wf + fx0 + 1];
        }
        if (Y + 1 < hc) {
            dyc = F.dy[(size_t)(fy0 + 1) * wf + fx0];
            if (has_x1) dyc += F.dy[(size_t)(fy0 + 1) * wf + fx0 + 1];
        }
        C.c[I] = any ? c : 1.0f;
        C.dx[I] = dxc;
        C.dy[I] = dyc;
        C.mask[I] = any;
    }
}

// Level l+1 from level l >= 1 (mg.cuh): each 2x2 aggregate's basis function is the fine weight vector t restricted to
// the aggregate, t from two red-black Gauss-Seidel sweeps on A t = 0 from t = 1 (masked cells 0), scaled so that its
// largest value in the aggregate is 1; the coarse operator is the Galerkin product, still 5-point:
//   coarse coupling to +x  = sum over the two fine couplings crossing the shared side of t_j t_k d_jk,
//   coarse c (diagonal less couplings) = sum_j t_j (A t)_j over the aggregate = (P^T A t)_I,
// with (A t)_j = c_j t_j + sum_k d_jk (t_j - t_k) in difference form, summed in f64 from the f32 weights the
// restriction and prolongation use. One tile of CO_S x CO_S fine cells per CTA, all four half-sweeps in shared
// memory: the tile's halo is as deep as the half-sweeps plus the two rings whose aggregates' scale the Galerkin sums
// read (t of the cells next to the tile's aggregates).
constexpr int CO_S = 32, CO_H = 6, CO_R = CO_S + 2 * CO_H, CO_N = CO_R * CO_R, CO_NT = 256;

__global__ void __launch_bounds__(CO_NT) mg_coarsen_kernel(MgLevel F, MgLevel C) {
    __shared__ float sc[CO_N], sdx[CO_N], sdy[CO_N], st[CO_N];
    __shared__ uint8_t sm[CO_N];
    const int wf = F.w, hf = F.h;
    const int X0 = blockIdx.x * CO_S - CO_H, Y0 = blockIdx.y * CO_S - CO_H;  // even: local parity = global parity
    for (int k = threadIdx.x; k < CO_N; k += CO_NT) {
        const int gx = X0 + k % CO_R, gy = Y0 + k / CO_R;
        float c = 1.0f, dx = 0.0f, dy = 0.0f, t = 0.0f;
        uint8_t m = 0;
        if (gx >= 0 && gx < wf && gy >= 0 && gy < hf) {
            const int i = gy * wf + gx;
            c = F.c[i];
            dx = F.dx[i];
            dy = F.dy[i];
            m = F.mask[i];
            t = m ? 1.0f : 0.0f;
        }
        sm[k] = m;
        sc[k] = c;
        sdx[k] = dx;
        sdy[k] = dy;
        st[k] = t;
    }
    __syncthreads();
    // four half-sweeps, colour 0 first, over the region less its outermost ring (a cell's value is exact once it
    // lies as many rings inside as half-sweeps were taken)
    for (int sweep = 0; sweep < 4; sweep++) {
        const int col = sweep & 1;
        for (int k = threadIdx.x; k < CO_N / 2; k += CO_NT) {
            const int ly = k / (CO_R / 2), lx = 2 * (k - ly * (CO_R / 2)) + ((ly + col) & 1);
            if (lx < 1 || lx > CO_R - 2 || ly < 1 || ly > CO_R - 2) continue;
            const int q = ly * CO_R + lx;
            // a masked or outside cell has c = 1 and no couplings (nor do its neighbours towards it): it stays 0
            const float dl = sdx[q - 1], dr = sdx[q], du = sdy[q - CO_R], dd = sdy[q];
            const float num = dl * st[q - 1] + dr * st[q + 1] + du * st[q - CO_R] + dd * st[q + CO_R];
            st[q] = num / (sc[q] + dl + dr + du + dd);
        }
        __syncthreads();
    }
    // each aggregate of the tile and of the two rings around it, scaled to a largest weight of 1 (an aggregate whose
    // weights all vanished takes 1 on its system cells, as plain aggregation would)
    constexpr int AG = (CO_S + 4) / 2;
    for (int k = threadIdx.x; k < AG * AG; k += CO_NT) {
        const int ay = k / AG, ax = k - ay * AG;
        const int lx = CO_H - 2 + 2 * ax, ly = CO_H - 2 + 2 * ay;
        const int q = ly * CO_R + lx;
        const float m = fmaxf(fmaxf(st[q], st[q + 1]), fmaxf(st[q + CO_R], st[q + CO_R + 1]));
        const int offs[4] = {0, 1, CO_R, CO_R + 1};
        for (int e = 0; e < 4; e++) {
            const int j = q + offs[e];
            st[j] = !sm[j] ? 0.0f : (m > 1e-30f ? st[j] / m : 1.0f);  // outside the level: mask 0
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < CO_S * CO_S; k += CO_NT) {
        const int gx = X0 + CO_H + k % CO_S, gy = Y0 + CO_H + k / CO_S;
        if (gx < wf && gy < hf) F.t[gy * wf + gx] = st[(k / CO_S + CO_H) * CO_R + k % CO_S + CO_H];
    }
    const int wc = C.w, hc = C.h;
    for (int k = threadIdx.x; k < (CO_S / 2) * (CO_S / 2); k += CO_NT) {
        const int cy = k / (CO_S / 2), cx = k - cy * (CO_S / 2);
        const int X = blockIdx.x * (CO_S / 2) + cx, Y = blockIdx.y * (CO_S / 2) + cy;
        if (X >= wc || Y >= hc) continue;
        const int lx0 = CO_H + 2 * cx, ly0 = CO_H + 2 * cy;
        double csum = 0.0;
        bool any = false;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                const int q = (ly0 + b) * CO_R + lx0 + a;
                if (!sm[q]) continue;
                any = true;
                const double tj = st[q];
                const double at = (double)sc[q] * tj + (double)sdx[q - 1] * (tj - st[q - 1]) +
                                  (double)sdx[q] * (tj - st[q + 1]) + (double)sdy[q - CO_R] * (tj - st[q - CO_R]) +
                                  (double)sdy[q] * (tj - st[q + CO_R]);
                csum += tj * at;
            }
        double dxc = 0.0, dyc = 0.0;
        if (X + 1 < wc)
            for (int b = 0; b < 2; b++) {
                const int q = (ly0 + b) * CO_R + lx0 + 1;
                dxc += (double)st[q] * st[q + 1] * sdx[q];
            }
        if (Y + 1 < hc)
            for (int a = 0; a < 2; a++) {
                const int q = (ly0 + 1) * CO_R + lx0 + a;
                dyc += (double)st[q] * st[q + CO_R] * sdy[q];
            }
        const size_t I = (size_t)Y * wc + X;
        C.c[I] = any ? (float)csum : 1.0f;
        C.dx[I] = any ? (float)dxc : 0.0f;
        C.dy[I] = any ? (float)dyc : 0.0f;
        C.mask[I] = any;
    }
}

// One smoother on a big level, all NS half-sweeps of a tile in shared memory (the tile's halo as deep as the
// half-sweeps, so the tile's result is exactly the global red-black sweeps'). PRE: from x = 0, red first, into L.x,
// then the residual summed over each 2x2 aggregate into the coarse level's b (one more halo ring keeps the residual's
// neighbours exact). POST: from x = L.x + ω P xc, black first, into L.x2; at level 0 `out` gets <b, x2>.
//
// The tile is stored split by colour (cell (lx, ly) of colour (lx + ly) & 1 at ly * HX + lx / 2 of its colour's
// arrays), so that a half-sweep's consecutive threads update consecutive cells of one colour and read their
// neighbours, all of the other colour, at consecutive addresses: no bank conflicts. Per cell: x, b, the inverse
// diagonal, the couplings to +x and +y, and for PRE the mass term c (the residual is taken in difference form,
// c x + Σ d (x − x_j), which keeps its FP32 accuracy when c is far below the couplings). The mask is not read: a
// masked cell has b = 0, c = 1 and no couplings (nor do its neighbours towards it), so its update is 0 and it
// influences nobody; the cells outside the world get the same values. Each thread's cells of a half-sweep are the
// same in every half-sweep of a colour: their indices and validity are computed once.
constexpr int A_X = 0, A_B = 1, A_INV = 2, A_DX = 3, A_DY = 4, A_C = 5;

template <int NS, bool PRE, int SX, int SY>
constexpr size_t smooth_smem() {
    constexpr int H = PRE ? NS + 1 : NS;
    constexpr int RN = (SX + 2 * H) * (SY + 2 * H);
    return (size_t)RN * (PRE ? 6 : 5) * sizeof(float);
}

template <int NS, bool PRE, int SX, int SY, int NT, bool VEC, bool WT>
__global__ void __launch_bounds__(NT) mg_smooth_kernel(MgLevel L, MgLevel C, const float* __restrict__ xc,
                                                                    float omega, double* part, unsigned* counter,
                                                                    double* out) {
    constexpr int H = PRE ? NS + 1 : NS;
    constexpr int RX = SX + 2 * H, RY = SY + 2 * H, RN = RX * RY, HX = RX / 2, HN = HX * RY;
    static_assert(RX % 2 == 0, "the tile's rows split evenly by colour");
    extern __shared__ __align__(16) float smem_f[];
    auto arr = [&](int a, int k) { return smem_f + (2 * a + k) * HN; };
    const int w = L.w, h = L.h;
    const int X0 = blockIdx.x * SX - H, Y0 = blockIdx.y * SY - H;  // X0 + Y0 even: local colour = global colour
    const int tid = threadIdx.x;
    if constexpr (VEC) {
        // rows in 16-byte chunks from the 4-aligned column at or left of X0 (the level's width is a multiple of 4, so a
        // chunk lies wholly inside or wholly outside the level): 4 cells' b, c, dx, dy, the row above's dy, and for
        // POST x and the two coarse corrections, in 6-7 loads
        constexpr int OFF = (4 - H % 4) % 4, NCH = (OFF + RX + 3) / 4, NV = RY * NCH;
        const int X0a = X0 - OFF;
        constexpr int NVL = (NV + NT - 1) / NT;
#pragma unroll
        for (int it = 0; it < NVL; it++) {
            const int k = tid + it * NT;
            if (k >= NV) break;
            const int ly = k / NCH, ch = k - ly * NCH;
            const int gx0 = X0a + 4 * ch, gy = Y0 + ly;
            float4 b4 = make_float4(0.f, 0.f, 0.f, 0.f), c4 = make_float4(1.f, 1.f, 1.f, 1.f), dx4 = b4, dy4 = b4,
                   dyu4 = b4, x4 = b4;
            float dxl = 0.0f;
            float2 xc2 = make_float2(0.f, 0.f);
            float4 t4 = b4;
            const bool in = gy >= 0 && gy < h && gx0 >= 0 && gx0 < w;
            if (in) {
                const size_t i = (size_t)gy * w + gx0;
                b4 = *reinterpret_cast<const float4*>(L.b + i);
                c4 = *reinterpret_cast<const float4*>(L.c + i);
                dx4 = *reinterpret_cast<const float4*>(L.dx + i);
                dy4 = *reinterpret_cast<const float4*>(L.dy + i);
                if (gy > 0) dyu4 = *reinterpret_cast<const float4*>(L.dy + i - w);
                if (gx0 > 0) dxl = L.dx[i - 1];
                if (!PRE) {
                    x4 = *reinterpret_cast<const float4*>(L.x + i);
                    if constexpr (WT) t4 = *reinterpret_cast<const float4*>(L.t + i);
                    xc2 = *reinterpret_cast<const float2*>(xc + (size_t)(gy >> 1) * C.w + (gx0 >> 1));
                }
            }
            const float bb[4] = {b4.x, b4.y, b4.z, b4.w}, cc[4] = {c4.x, c4.y, c4.z, c4.w};
            const float dxa[5] = {dxl, dx4.x, dx4.y, dx4.z, dx4.w}, dya[4] = {dy4.x, dy4.y, dy4.z, dy4.w};
            const float dyua[4] = {dyu4.x, dyu4.y, dyu4.z, dyu4.w}, xa[4] = {x4.x, x4.y, x4.z, x4.w};
            const float xcv[2] = {xc2.x, xc2.y}, ta[4] = {t4.x, t4.y, t4.z, t4.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int lx = 4 * ch + e - OFF;
                if (lx < 0 || lx >= RX) continue;
                const float inv = in ? __fdividef(1.0f, cc[e] + dxa[e + 1] + dxa[e] + dya[e] + dyua[e]) : 0.0f;
                const float x = (!PRE && in) ? xa[e] + omega * (WT ? ta[e] : 1.0f) * xcv[e >> 1] : 0.0f;
                const int col = (lx + ly) & 1, q = ly * HX + (lx >> 1);
                arr(A_X, col)[q] = x;
                arr(A_B, col)[q] = bb[e];
                arr(A_INV, col)[q] = inv;
                arr(A_DX, col)[q] = dxa[e + 1];
                arr(A_DY, col)[q] = dya[e];
                if (PRE) arr(A_C, col)[q] = cc[e];
            }
        }
    } else {
    constexpr int NLOAD = (RN + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < NLOAD; it++) {
        const int k = tid + it * NT;
        if (k >= RN) break;
        const int lx = k % RX, ly = k / RX;
        const int gx = X0 + lx, gy = Y0 + ly;
        float b = 0.0f, c = 1.0f, dx = 0.0f, dy = 0.0f, x = 0.0f, inv = 0.0f;
        if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
            const int i = gy * w + gx;  // a level holds fewer than 2^31 cells
            b = L.b[i];
            c = L.c[i];
            dx = L.dx[i];
            dy = L.dy[i];
            const float dxl = gx > 0 ? L.dx[i - 1] : 0.0f, dyu = gy > 0 ? L.dy[i - w] : 0.0f;
            if (!PRE) x = L.x[i] + omega * (WT ? L.t[i] : 1.0f) * xc[(size_t)(gy >> 1) * C.w + (gx >> 1)];
            inv = __fdividef(1.0f, c + dx + dxl + dy + dyu);  // the smoother's diagonal: an approximate reciprocal
        }
        const int col = (lx + ly) & 1, q = ly * HX + (lx >> 1);
        arr(A_X, col)[q] = x;
        arr(A_B, col)[q] = b;
        arr(A_INV, col)[q] = inv;
        arr(A_DX, col)[q] = dx;
        arr(A_DY, col)[q] = dy;
        if (PRE) arr(A_C, col)[q] = c;
    }
    }
    __syncthreads();
    constexpr int NSWEEP = (HN + NT - 1) / NT;
    int qinfo[NSWEEP];  // per cell slot: q | o of colour 0 << 28 | updatable in colour 0 << 29 | in colour 1 << 30
#pragma unroll
    for (int it = 0; it < NSWEEP; it++) {
        const int q = tid + it * NT;
        int info = -1;
        if (q < HN) {
            const int ly = q / HX, j = q - ly * HX;
            const bool yok = ly >= 1 && ly <= RY - 2;
            const int o0 = ly & 1, lx0 = 2 * j + o0, lx1 = 2 * j + 1 - o0;
            const int ok0 = yok && lx0 >= 1 && lx0 <= RX - 2, ok1 = yok && lx1 >= 1 && lx1 <= RX - 2;
            info = q | (o0 << 28) | (ok0 << 29) | (ok1 << 30);
        }
        qinfo[it] = info;
    }
#pragma unroll 1
    for (int s = 0; s < NS; s++) {
        const int col = PRE ? (s & 1) : 1 - (s & 1), oth = 1 - col;
        float* x = arr(A_X, col);
        const float* b = arr(A_B, col);
        const float* inv = arr(A_INV, col);
        const float* dx = arr(A_DX, col);
        const float* dy = arr(A_DY, col);
        const float* xo = arr(A_X, oth);
        const float* dxo = arr(A_DX, oth);
        const float* dyo = arr(A_DY, oth);
#pragma unroll
        for (int it = 0; it < NSWEEP; it++) {
            const int info = qinfo[it];
            if (info < 0 || !((info >> (29 + col)) & 1)) continue;
            const int q = info & 0x0FFFFFFF, o = ((info >> 28) & 1) ^ col;
            const int left = q - 1 + o, right = q + o;  // the other colour's cells at lx - 1 and lx + 1
            x[q] = (b[q] + dxo[left] * xo[left] + dx[q] * xo[right] + dyo[q - HX] * xo[q - HX] + dy[q] * xo[q + HX]) *
                   inv[q];
        }
        __syncthreads();
    }
    double acc = 0.0;
    float* dst = PRE ? L.x : L.x2;
    for (int k = tid; k < SX * SY; k += NT) {
        const int ox = k % SX, oy = k / SX;
        const int gx = X0 + H + ox, gy = Y0 + H + oy;
        if (gx < w && gy < h) {
            const int lx = ox + H, ly = oy + H, col = (lx + ly) & 1, q = ly * HX + (lx >> 1);
            const float xv = arr(A_X, col)[q];
            dst[(size_t)gy * w + gx] = xv;
            if (!PRE && out) acc += (double)arr(A_B, col)[q] * (double)xv;
        }
    }
    if (PRE) {
        // the coarse right-hand side: the residual, in difference form, weighted by t and summed over each aggregate of
        // the tile
        for (int k = tid; k < (SX / 2) * (SY / 2); k += NT) {
            const int cxl = k % (SX / 2), cyl = k / (SX / 2);
            const int X = (X0 + H) / 2 + cxl, Y = (Y0 + H) / 2 + cyl;
            if (X >= C.w || Y >= C.h) continue;
            float sum = 0.0f;
#pragma unroll
            for (int bb = 0; bb < 2; bb++)
#pragma unroll
                for (int a = 0; a < 2; a++) {
                    const int lx = 2 * cxl + a + H, ly = 2 * cyl + bb + H;
                    const int col = (lx + ly) & 1, oth = 1 - col, q = ly * HX + (lx >> 1);
                    const int o = (col + ly) & 1, left = q - 1 + o, right = q + o;
                    const float xj = arr(A_X, col)[q];
                    const float* xo = arr(A_X, oth);
                    float ax = arr(A_C, col)[q] * xj;
                    ax += arr(A_DX, oth)[left] * (xj - xo[left]);
                    ax += arr(A_DX, col)[q] * (xj - xo[right]);
                    ax += arr(A_DY, oth)[q - HX] * (xj - xo[q - HX]);
                    ax += arr(A_DY, col)[q] * (xj - xo[q + HX]);
                    if constexpr (WT) {
                        const int gx = X0 + lx, gy = Y0 + ly;
                        sum += (gx < w && gy < h ? L.t[gy * w + gx] : 0.0f) * (arr(A_B, col)[q] - ax);
                    } else {
                        sum += arr(A_B, col)[q] - ax;
                    }
                }
            C.b[(size_t)Y * C.w + X] = C.mask[(size_t)Y * C.w + X] ? sum : 0.0f;
        }
    } else if (out) {
        grid_sum_last1(acc, part, counter, out);
    }
}

// The row-band smoother of the big levels of even width: the same smoother as mg_smooth_kernel (NS red-black
// half-sweeps of a tile whose halo is as deep as the half-sweeps, then the restriction or <b, x2>), with every cell's
// coefficients and iterate held in registers. A CTA covers a 64 x 64 region (RB_RX x RB_RY): warp w owns rows
// 4w .. 4w+3 (a band), lane j owns the cell pair (2j, 2j+1) of each of its rows. In a half-sweep a cell's horizontal
// neighbours are its pair partner (a register) and one cell of the next lane's pair (a shuffle), its vertical
// neighbours the same lane's rows above and below (registers), except across a band edge, whose rows go through shared
// memory once per half-sweep (double-buffered: one barrier per half-sweep). Which cell of a pair a colour updates is
// fixed by the row's parity (the region starts on an even column and row, so local parity = global parity), so the
// sweeps unroll into straight-line code. The halo is NS + 2 for the pre-smoother (NS + 1 keeps the restriction's
// neighbours exact; one more keeps the region on even columns, so pairs load as 8-byte words and sit inside one 2 x 2
// aggregate) and NS for the post-smoother. Cells outside the level: b = 0, c = 1, no couplings, inverse diagonal 0.
constexpr int RB_R = 4, RB_WARPS = 16, RB_NT = 32 * RB_WARPS, RB_RX = 64, RB_RY = RB_R * RB_WARPS;

template <int NS, bool PRE>
constexpr int rb_halo() { return PRE ? NS + 2 : NS; }

template <int NS, bool PRE, bool WT>
__global__ void __launch_bounds__(RB_NT, 2) mg_rowband_kernel(MgLevel L, MgLevel C, const float* __restrict__ xc,
                                                            float omega, double* part, unsigned* counter,
                                                            double* out) {
    constexpr int H = rb_halo<NS, PRE>(), SX = RB_RX - 2 * H, SY = RB_RY - 2 * H;
    static_assert(H % 2 == 0 && NS % 2 == 0, "the region starts on an even column and row");
    __shared__ float2 edge[2][2][RB_WARPS][32];  // [buffer][top row / bottom row][warp][lane]: (x of 2j, x of 2j+1)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int w = L.w, h = L.h;
    const int X0 = blockIdx.x * SX - H, Y0 = blockIdx.y * SY - H;
    const int gx = X0 + 2 * lane;             // the pair's first column (even)
    const bool xin = gx >= 0 && gx < w;        // w is even: both cells of the pair lie inside, or neither
    const int gy0 = Y0 + RB_R * warp;          // the band's first row (even)

    float bA[RB_R], bB[RB_R], iA[RB_R], iB[RB_R], dl[RB_R], dm[RB_R], dr[RB_R], dA[RB_R], dB[RB_R];
    float xA[RB_R], xB[RB_R], cA[RB_R], cB[RB_R];
    float uA = 0.0f, uB = 0.0f;  // the couplings of row 0 to the row above
#pragma unroll
    for (int r = 0; r < RB_R; r++) {
        const int gy = gy0 + r;
        const bool in = xin && gy >= 0 && gy < h;
        const size_t i = (size_t)gy * w + gx;
        float2 b2 = make_float2(0.f, 0.f), c2 = make_float2(1.f, 1.f), dx2 = b2, dy2 = b2;
        if (in) {
            b2 = *reinterpret_cast<const float2*>(L.b + i);
            c2 = *reinterpret_cast<const float2*>(L.c + i);
            dx2 = *reinterpret_cast<const float2*>(L.dx + i);
            dy2 = *reinterpret_cast<const float2*>(L.dy + i);
            if (r == 0 && gy > 0) {
                const float2 u2 = *reinterpret_cast<const float2*>(L.dy + i - w);
                uA = u2.x;
                uB = u2.y;
            }
        }
        bA[r] = b2.x;
        bB[r] = b2.y;
        cA[r] = c2.x;
        cB[r] = c2.y;
        dm[r] = dx2.x;
        dr[r] = dx2.y;
        dA[r] = dy2.x;
        dB[r] = dy2.y;
        // the coupling of cell 2j to 2j - 1 is the previous pair's right coupling (0 from a pair outside the level)
        dl[r] = __shfl_up_sync(0xffffffffu, dx2.y, 1);
        if (lane == 0) dl[r] = (in && gx > 0) ? L.dx[i - 1] : 0.0f;
        const float upA = r ? dA[r - 1] : uA, upB = r ? dB[r - 1] : uB;
        iA[r] = in ? __fdividef(1.0f, c2.x + dl[r] + dx2.x + upA + dy2.x) : 0.0f;
        iB[r] = in ? __fdividef(1.0f, c2.y + dx2.x + dx2.y + upB + dy2.y) : 0.0f;
        float x0 = 0.0f, x1 = 0.0f;
        if (!PRE && in) {
            const float2 xv = *reinterpret_cast<const float2*>(L.x + i);
            const float corr = omega * xc[(size_t)(gy >> 1) * C.w + (gx >> 1)];
            if constexpr (WT) {
                const float2 t2 = *reinterpret_cast<const float2*>(L.t + i);
                x0 = xv.x + corr * t2.x;
                x1 = xv.y + corr * t2.y;
            } else {
                x0 = xv.x + corr;
                x1 = xv.y + corr;
            }
        }
        xA[r] = x0;
        xB[r] = x1;
    }
    edge[0][0][warp][lane] = make_float2(xA[0], xB[0]);
    edge[0][1][warp][lane] = make_float2(xA[RB_R - 1], xB[RB_R - 1]);
    __syncthreads();
    const int wu = warp > 0 ? warp - 1 : warp, wd = warp + 1 < RB_WARPS ? warp + 1 : warp;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int col = PRE ? (s & 1) : 1 - (s & 1);
        const int rd = s & 1, wr = (s + 1) & 1;
        const float2 above = edge[rd][1][wu][lane], below = edge[rd][0][wd][lane];
#pragma unroll
        for (int r = 0; r < RB_R; r++) {
            if ((r & 1) == col) {  // the pair's first cell has this colour
                const float left = __shfl_up_sync(0xffffffffu, xB[r], 1);
                const float up = r ? xA[r - 1] : above.x, down = r + 1 < RB_R ? xA[r + 1] : below.x;
                const float cu = r ? dA[r - 1] : uA;
                xA[r] = (bA[r] + dl[r] * left + dm[r] * xB[r] + cu * up + dA[r] * down) * iA[r];
            } else {
                const float right = __shfl_down_sync(0xffffffffu, xA[r], 1);
                const float up = r ? xB[r - 1] : above.y, down = r + 1 < RB_R ? xB[r + 1] : below.y;
                const float cu = r ? dB[r - 1] : uB;
                xB[r] = (bB[r] + dm[r] * xA[r] + dr[r] * right + cu * up + dB[r] * down) * iB[r];
            }
        }
        edge[wr][0][warp][lane] = make_float2(xA[0], xB[0]);
        edge[wr][1][warp][lane] = make_float2(xA[RB_R - 1], xB[RB_R - 1]);
        __syncthreads();
    }
    const bool xout = xin && 2 * lane >= H && 2 * lane < RB_RX - H;
    if constexpr (PRE) {
        const float2 above = edge[NS & 1][1][wu][lane], below = edge[NS & 1][0][wd][lane];
        float ragg[RB_R / 2] = {};
#pragma unroll
        for (int r = 0; r < RB_R; r++) {
            const int gy = gy0 + r, ly = RB_R * warp + r;
            const bool o = xout && ly >= H && ly < RB_RY - H && gy < h;
            const size_t i = (size_t)gy * w + gx;
            if (o) *reinterpret_cast<float2*>(L.x + i) = make_float2(xA[r], xB[r]);
            // the residual in difference form, c x + Σ d (x - x_nb), for both cells
            const float left = __shfl_up_sync(0xffffffffu, xB[r], 1);
            const float right = __shfl_down_sync(0xffffffffu, xA[r], 1);
            const float upA = r ? xA[r - 1] : above.x, dnA = r + 1 < RB_R ? xA[r + 1] : below.x;
            const float upB = r ? xB[r - 1] : above.y, dnB = r + 1 < RB_R ? xB[r + 1] : below.y;
            const float cuA = r ? dA[r - 1] : uA, cuB = r ? dB[r - 1] : uB;
            float axA = cA[r] * xA[r];
            axA += dl[r] * (xA[r] - left);
            axA += dm[r] * (xA[r] - xB[r]);
            axA += cuA * (xA[r] - upA);
            axA += dA[r] * (xA[r] - dnA);
            float axB = cB[r] * xB[r];
            axB += dm[r] * (xB[r] - xA[r]);
            axB += dr[r] * (xB[r] - right);
            axB += cuB * (xB[r] - upB);
            axB += dB[r] * (xB[r] - dnB);
            float rA = bA[r] - axA, rB = bB[r] - axB;
            if constexpr (WT) {
                if (o) {
                    const float2 t2 = *reinterpret_cast<const float2*>(L.t + i);
                    rA *= t2.x;
                    rB *= t2.y;
                }
            }
            ragg[r >> 1] += rA + rB;
        }
#pragma unroll
        for (int k = 0; k < RB_R / 2; k++) {
            const int ly = RB_R * warp + 2 * k;
            const int X = gx >> 1, Y = (gy0 + 2 * k) >> 1;
            if (xout && ly >= H && ly < RB_RY - H && X < C.w && Y < C.h && gy0 + 2 * k >= 0) {
                const size_t I = (size_t)Y * C.w + X;
                C.b[I] = C.mask[I] ? ragg[k] : 0.0f;
            }
        }
    } else {
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < RB_R; r++) {
            const int gy = gy0 + r, ly = RB_R * warp + r;
            if (xout && ly >= H && ly < RB_RY - H && gy < h) {
                const size_t i = (size_t)gy * w + gx;
                *reinterpret_cast<float2*>(L.x2 + i) = make_float2(xA[r], xB[r]);
                if (out) acc += (double)bA[r] * (double)xA[r] + (double)bB[r] * (double)xB[r];
            }
        }
        if (out) grid_sum_last1(acc, part, counter, out);
    }
    (void)SX;
    (void)SY;
}

// The row-band smoother of level 0 with its region staged by TMA: the same smoother as mg_rowband_kernel (unweighted
// levels only), its coefficients (b, c, dx, dy) and, after the coarse correction, the iterate x read from shared memory
// where one thread's bulk tensor copies put them — the region's 64 rows and the row above it, 72 columns from a
// 16-byte boundary left of the region (the pair's left coupling included), zero past the level's edges — so a CTA's
// loads are all in flight at once instead of four row-dependent rounds per thread. Every wait is bounded: a wait that
// gives up sets the level's error flag and the CTA leaves without its stores.
constexpr int RB_TMA_X = 72, RB_TMA_Y = RB_RY + 1;
constexpr uint32_t kMgWaitPolls = 1u << 24;
// b, c, dx, dy, then x after the coarse correction (post) or the weights the restriction takes (pre, weighted levels);
// the post-smoother of a weighted level reads its weights while the boxes land
template <bool PRE, bool WT>
constexpr int rb_tma_arrays() { return PRE ? (WT ? 5 : 4) : 5; }
constexpr size_t rb_tma_array_bytes() { return ((size_t)RB_TMA_X * RB_TMA_Y * sizeof(float) + 127) / 128 * 128; }
template <bool PRE, bool WT>
constexpr size_t rb_tma_smem() {
    return rb_tma_arrays<PRE, WT>() * rb_tma_array_bytes() + sizeof(float2) * 2 * 2 * RB_WARPS * 32 + 16;
}

template <int NS, bool PRE, bool WT>
__global__ void __launch_bounds__(RB_NT, 2)
    mg_rowband_tma_kernel(const __grid_constant__ CUtensorMap mb, const __grid_constant__ CUtensorMap mc,
                          const __grid_constant__ CUtensorMap mdx, const __grid_constant__ CUtensorMap mdy,
                          const __grid_constant__ CUtensorMap mx, MgLevel L, MgLevel C, const float* __restrict__ xc,
                          float omega, double* part, unsigned* counter, double* out) {
    constexpr int H = rb_halo<NS, PRE>(), SX = RB_RX - 2 * H;
    constexpr int XO = (H % 4 == 2) ? 2 : 4;  // the region's first column within the box (X0 - XO on a 16-byte boundary)
    constexpr int NA = rb_tma_arrays<PRE, WT>();
    constexpr size_t AB = rb_tma_array_bytes() / sizeof(float);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* sarr = reinterpret_cast<float*>(smem_raw);
    float2(*edge)[2][RB_WARPS][32] = reinterpret_cast<float2(*)[2][RB_WARPS][32]>(smem_raw + NA * rb_tma_array_bytes());
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem_raw + NA * rb_tma_array_bytes() + sizeof(float2) * 2 * 2 * RB_WARPS * 32);
    const float* sb = sarr;
    const float* sc = sarr + AB;
    const float* sdx = sarr + 2 * AB;
    const float* sdy = sarr + 3 * AB;
    const float* sx = sarr + 4 * AB;  // post: the iterate; pre of a weighted level: the weights
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int w = L.w, h = L.h;
    const int X0 = blockIdx.x * SX - H, Y0 = blockIdx.y * (RB_RY - 2 * H) - H;
    if (tid == 0) {
        tc::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        tma::expect_tx(mbar, (uint32_t)(NA * RB_TMA_X * RB_TMA_Y * sizeof(float)));
        const int xs = X0 - XO, ys = Y0 - 1;
        tma::load_3d(sarr, &mb, xs, ys, 0, mbar);
        tma::load_3d(sarr + AB, &mc, xs, ys, 0, mbar);
        tma::load_3d(sarr + 2 * AB, &mdx, xs, ys, 0, mbar);
        tma::load_3d(sarr + 3 * AB, &mdy, xs, ys, 0, mbar);
        if constexpr (NA == 5) tma::load_3d(sarr + 4 * AB, &mx, xs, ys, 0, mbar);
    }
    const int gx = X0 + 2 * lane;
    const bool xin = gx >= 0 && gx < w;
    const int gy0 = Y0 + RB_R * warp;
    // read while the boxes land: the post-smoother's coarse correction, the pre-smoother's coarse mask (global, half
    // resolution)
    float corrA[RB_R], corrB[RB_R];
    uint8_t cmask[RB_R / 2];
#pragma unroll
    for (int r = 0; r < RB_R; r++) {
        const int gy = gy0 + r;
        const bool in = !PRE && xin && gy >= 0 && gy < h;
        const float cr = in ? omega * xc[(size_t)(gy >> 1) * C.w + (gx >> 1)] : 0.0f;
        corrA[r] = cr;
        corrB[r] = cr;
        if constexpr (WT && !PRE) {  // the prolongation's weights
            if (in) {
                const float2 t2 = *reinterpret_cast<const float2*>(L.t + (size_t)gy * w + gx);
                corrA[r] = cr * t2.x;
                corrB[r] = cr * t2.y;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < RB_R / 2; k++) {
        const int X = gx >> 1, Y = (gy0 + 2 * k) >> 1;
        cmask[k] = (PRE && xin && gy0 + 2 * k >= 0 && X < C.w && Y < C.h) ? C.mask[(size_t)Y * C.w + X] : 0;
    }
    const bool landed = tc::mbar_wait(mbar, 0, kMgWaitPolls);
    if (__syncthreads_or(!landed)) {
        if (tid == 0 && L.err) atomicOr(L.err, 1);
        tc::mbar_wait(mbar, 0, kMgWaitPolls);  // copies still in flight land before the CTA leaves
        return;
    }
    float bA[RB_R], bB[RB_R], iA[RB_R], iB[RB_R], dl[RB_R], dm[RB_R], dr[RB_R], dA[RB_R], dB[RB_R];
    float xA[RB_R], xB[RB_R], cA[RB_R], cB[RB_R];
    float uA = 0.0f, uB = 0.0f;
    const int col0 = XO + 2 * lane;  // the pair's first column within the box
#pragma unroll
    for (int r = 0; r < RB_R; r++) {
        const int gy = gy0 + r;
        const bool in = xin && gy >= 0 && gy < h;
        const int q = (RB_R * warp + r + 1) * RB_TMA_X + col0;  // the box's row 0 is the region's row -1
        float2 b2 = make_float2(0.f, 0.f), c2 = make_float2(1.f, 1.f), dx2 = b2, dy2 = b2;
        float left = 0.0f;
        if (in) {
            b2 = *reinterpret_cast<const float2*>(sb + q);
            c2 = *reinterpret_cast<const float2*>(sc + q);
            dx2 = *reinterpret_cast<const float2*>(sdx + q);
            dy2 = *reinterpret_cast<const float2*>(sdy + q);
            left = sdx[q - 1];  // zero past the level's left edge
            if (r == 0) {
                const float2 u2 = *reinterpret_cast<const float2*>(sdy + q - RB_TMA_X);  // zero above row 0
                uA = u2.x;
                uB = u2.y;
            }
        }
        bA[r] = b2.x;
        bB[r] = b2.y;
        cA[r] = c2.x;
        cB[r] = c2.y;
        dm[r] = dx2.x;
        dr[r] = dx2.y;
        dA[r] = dy2.x;
        dB[r] = dy2.y;
        dl[r] = left;
        const float upA = r ? dA[r - 1] : uA, upB = r ? dB[r - 1] : uB;
        iA[r] = in ? __fdividef(1.0f, c2.x + dl[r] + dx2.x + upA + dy2.x) : 0.0f;
        iB[r] = in ? __fdividef(1.0f, c2.y + dx2.x + dx2.y + upB + dy2.y) : 0.0f;
        float x0 = 0.0f, x1 = 0.0f;
        if (!PRE && in) {
            const float2 xv = *reinterpret_cast<const float2*>(sx + q);
            x0 = xv.x + corrA[r];
            x1 = xv.y + corrB[r];
        }
        xA[r] = x0;
        xB[r] = x1;
    }
    edge[0][0][warp][lane] = make_float2(xA[0], xB[0]);
    edge[0][1][warp][lane] = make_float2(xA[RB_R - 1], xB[RB_R - 1]);
    __syncthreads();
    const int wu = warp > 0 ? warp - 1 : warp, wd = warp + 1 < RB_WARPS ? warp + 1 : warp;
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const int col = PRE ? (s & 1) : 1 - (s & 1);
        const int rd = s & 1, wr = (s + 1) & 1;
        const float2 above = edge[rd][1][wu][lane], below = edge[rd][0][wd][lane];
#pragma unroll
        for (int r = 0; r < RB_R; r++) {
            if (PRE && s == 0) {  // the pre-smoother starts from x = 0: its first half-sweep is b times the inverse
                if ((r & 1) == col) xA[r] = bA[r] * iA[r];
                else xB[r] = bB[r] * iB[r];
                continue;
            }
            if ((r & 1) == col) {
                const float left = __shfl_up_sync(0xffffffffu, xB[r], 1);
                const float up = r ? xA[r - 1] : above.x, down = r + 1 < RB_R ? xA[r + 1] : below.x;
                const float cu = r ? dA[r - 1] : uA;
                xA[r] = (bA[r] + dl[r] * left + dm[r] * xB[r] + cu * up + dA[r] * down) * iA[r];
            } else {
                const float right = __shfl_down_sync(0xffffffffu, xA[r], 1);
                const float up = r ? xB[r - 1] : above.y, down = r + 1 < RB_R ? xB[r + 1] : below.y;
                const float cu = r ? dB[r - 1] : uB;
                xB[r] = (bB[r] + dm[r] * xA[r] + dr[r] * right + cu * up + dB[r] * down) * iB[r];
            }
        }
        edge[wr][0][warp][lane] = make_float2(xA[0], xB[0]);
        edge[wr][1][warp][lane] = make_float2(xA[RB_R - 1], xB[RB_R - 1]);
        __syncthreads();
    }
    const bool xout = xin && 2 * lane >= H && 2 * lane < RB_RX - H;
    if constexpr (PRE) {
        const float2 above = edge[NS & 1][1][wu][lane], below = edge[NS & 1][0][wd][lane];
        float ragg[RB_R / 2] = {};
#pragma unroll
        for (int r = 0; r < RB_R; r++) {
            const int gy = gy0 + r, ly = RB_R * warp + r;
            const bool o = xout && ly >= H && ly < RB_RY - H && gy < h;
            const size_t i = (size_t)gy * w + gx;
            if (o) *reinterpret_cast<float2*>(L.x + i) = make_float2(xA[r], xB[r]);
            const float left = __shfl_up_sync(0xffffffffu, xB[r], 1);
            const float right = __shfl_down_sync(0xffffffffu, xA[r], 1);
            const float upA = r ? xA[r - 1] : above.x, dnA = r + 1 < RB_R ? xA[r + 1] : below.x;
            const float upB = r ? xB[r - 1] : above.y, dnB = r + 1 < RB_R ? xB[r + 1] : below.y;
            const float cuA = r ? dA[r - 1] : uA, cuB = r ? dB[r - 1] : uB;
            float axA = cA[r] * xA[r];
            axA += dl[r] * (xA[r] - left);
            axA += dm[r] * (xA[r] - xB[r]);
            axA += cuA * (xA[r] - upA);
            axA += dA[r] * (xA[r] - dnA);
            float axB = cB[r] * xB[r];
            axB += dm[r] * (xB[r] - xA[r]);
            axB += dr[r] * (xB[r] - right);
            axB += cuB * (xB[r] - upB);
            axB += dB[r] * (xB[r] - dnB);
            float rA = bA[r] - axA, rB = bB[r] - axB;
            if constexpr (WT) {  // the restriction's weights, zero past the level (the box's fill)
                const float2 t2 = *reinterpret_cast<const float2*>(sx + (RB_R * warp + r + 1) * RB_TMA_X + col0);
                rA *= t2.x;
                rB *= t2.y;
            }
            ragg[r >> 1] += rA + rB;
        }
#pragma unroll
        for (int k = 0; k < RB_R / 2; k++) {
            const int ly = RB_R * warp + 2 * k;
            const int X = gx >> 1, Y = (gy0 + 2 * k) >> 1;
            if (xout && ly >= H && ly < RB_RY - H && X < C.w && Y < C.h && gy0 + 2 * k >= 0)
                C.b[(size_t)Y * C.w + X] = cmask[k] ? ragg[k] : 0.0f;
        }
    } else {
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < RB_R; r++) {
            const int gy = gy0 + r, ly = RB_R * warp + r;
            if (xout && ly >= H && ly < RB_RY - H && gy < h) {
                const size_t i = (size_t)gy * w + gx;
                *reinterpret_cast<float2*>(L.x2 + i) = make_float2(xA[r], xB[r]);
                if (out) acc += (double)bA[r] * (double)xA[r] + (double)bB[r] * (double)xB[r];
            }
        }
        if (out) grid_sum_last1(acc, part, counter, out);
    }
}

// The coarsest level's operator inverted by Gauss-Jordan elimination in f64 in one CTA (n <= 64 cells), masked-out
// cells as identity rows; stored f32. The operator is SPD, so no pivoting is needed. The augmented matrix [A | I] is
// kept twice and each elimination step reads one copy and writes the other, so a step is one pass and one barrier;
// at step p only columns p .. n + p change (to the left the pivot row is already 0, to the right of n + p it is still
// 0: untouched identity columns, the same in both copies).
__global__ void mg_coarse_inverse_kernel(MgLevel C, float* inv) {
    extern __shared__ double aug[];  // two n x 2n copies
    const int w = C.w, h = C.h, n = w * h, m = 2 * n;
    for (int k = threadIdx.x; k < n * m; k += blockDim.x) {
        const int i = k / m, j = k % m;
        double v = 0.0;
        if (j >= n) {
            v = (j - n == i) ? 1.0 : 0.0;
        } else if (!C.mask[i]) {
            v = (i == j) ? 1.0 : 0.0;
        } else {
            const int xi = i % w, yi = i / w;
            const double dl = xi > 0 ? C.dx[i - 1] : 0.0, dr = C.dx[i];
            const double du = yi > 0 ? C.dy[i - w] : 0.0, dd = C.dy[i];
            if (j == i) v = (double)C.c[i] + dl + dr + du + dd;
            else if (xi > 0 && j == i - 1) v = -dl;
            else if (xi + 1 < w && j == i + 1) v = -dr;
            else if (yi > 0 && j == i - w) v = -du;
            else if (yi + 1 < h && j == i + w) v = -dd;
        }
        aug[k] = v;
        aug[n * m + k] = v;
    }
    __syncthreads();
    // threads as 64 rows x 16 column lanes: thread (i, c) updates row i's active columns p + c, p + c + 16, ...
    // (n <= 64 rows; n + 1 <= 65 active columns), no index divisions in the loop; the thread that writes the next
    // step's pivot also leaves its reciprocal for every thread to read
    __shared__ double rpiv[2];
    if (threadIdx.x == 0) rpiv[0] = 1.0 / aug[0];
    __syncthreads();
    const int i = threadIdx.x >> 4, c = threadIdx.x & 15;
    for (int p = 0; p < n; p++) {
        const double* src = aug + (p & 1) * n * m;
        double* dst = aug + ((p + 1) & 1) * n * m;
        if (i < n) {
            const double rp = rpiv[p & 1];
            const double aip = src[i * m + p];
            for (int j = p + c; j <= n + p; j += 16) {
                const double apj = src[p * m + j] * rp;
                const double v = i == p ? apj : src[i * m + j] - aip * apj;
                dst[i * m + j] = v;
                if (i == p + 1 && j == p + 1) rpiv[(p + 1) & 1] = 1.0 / v;
            }
        }
        __syncthreads();
    }
    const double* fin = aug + (n & 1) * n * m;
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) inv[k] = (float)fin[(k / n) * m + n + (k % n)];
}

// ---- the coarse tail: every level from t on, inside one CTA
// The tail's levels live in its dynamic shared memory at the offsets of TailLevel: indexing the extern shared array
// itself keeps every access a shared-memory access.
extern __shared__ __align__(16) unsigned char tail_smem_raw[];
__device__ __forceinline__ float* tsf() { return reinterpret_cast<float*>(tail_smem_raw); }

// Threads of the tail run as 32 columns x TAIL_ROWS rows: thread (tx, ty) takes rows ty, ty + TAIL_ROWS, ... and, of
// a sweep's colour, the columns 2 tx + parity, 2 (tx + 32) + parity, ... (no index divisions).
__device__ __forceinline__ void tail_sweep(const TailLevel T, int color) {
    float* f = tsf();
    const float *b = f + T.b, *dx = f + T.dx, *dy = f + T.dy, *inv = f + T.inv;
    float* x = f + T.x;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int y = ty; y < T.h; y += TAIL_ROWS) {
        const int par = (y + color) & 1;
        for (int xx = 2 * tx + par; xx < T.w; xx += 64) {
            // masked cells: b = 0, no couplings, inv = 0, so they stay 0; couplings past the edges are 0
            const int i = y * T.w + xx;
            float s = b[i];
            if (xx > 0) s += dx[i - 1] * x[i - 1];
            if (xx + 1 < T.w) s += dx[i] * x[i + 1];
            if (y > 0) s += dy[i - T.w] * x[i - T.w];
            if (y + 1 < T.h) s += dy[i] * x[i + T.w];
            x[i] = s * inv[i];
        }
    }
    __syncthreads();
}

// `count` half-sweeps from colour `color` of a tail level of at most 64 x 64 cells, each thread holding one 2 x 2 block
// (warp v's rows 2v, 2v + 1, lane j's columns 2j, 2j + 1) with its coefficients and iterate in registers: a cell's
// neighbours inside the block are registers, across a column edge a shuffle, across a row edge one shared-memory load
// of the level's x (kept current after every half-sweep). Same arithmetic as tail_sweep.
__device__ __forceinline__ void tail_sweeps_reg(const TailLevel T, int color, int count) {
    float* f = tsf();
    const float *b = f + T.b, *dx = f + T.dx, *dy = f + T.dy, *inv = f + T.inv;
    float* x = f + T.x;
    const int lane = threadIdx.x & 31, x0 = 2 * lane, y0 = 2 * (threadIdx.x >> 5);
    float bb[4], iv[4], cl[4], cr[4], cu[4], cd[4], xv[4];
    bool ok[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int xx = x0 + (k & 1), yy = y0 + (k >> 1);
        ok[k] = xx < T.w && yy < T.h;
        const int i = ok[k] ? yy * T.w + xx : 0;
        bb[k] = ok[k] ? b[i] : 0.0f;
        iv[k] = ok[k] ? inv[i] : 0.0f;
        cl[k] = ok[k] && xx > 0 ? dx[i - 1] : 0.0f;
        cr[k] = ok[k] && xx + 1 < T.w ? dx[i] : 0.0f;
        cu[k] = ok[k] && yy > 0 ? dy[i - T.w] : 0.0f;
        cd[k] = ok[k] && yy + 1 < T.h ? dy[i] : 0.0f;
        xv[k] = ok[k] ? x[i] : 0.0f;
    }
    const int iu = y0 > 0 ? (y0 - 1) * T.w : 0, id = y0 + 2 < T.h ? (y0 + 2) * T.w : 0;
    const bool hu = y0 > 0 && ok[0], hd = y0 + 2 < T.h && ok[2];
    for (int s = 0; s < count; s++) {
        if (((color + s) & 1) == 0) {  // cells (2j, 2v) and (2j + 1, 2v + 1)
            const float left = __shfl_up_sync(0xffffffffu, xv[1], 1);
            const float right = __shfl_down_sync(0xffffffffu, xv[2], 1);
            const float up = hu ? x[iu + x0] : 0.0f;
            const float down = hd && ok[3] ? x[id + x0 + 1] : 0.0f;
            xv[0] = (bb[0] + cl[0] * left + cr[0] * xv[1] + cu[0] * up + cd[0] * xv[2]) * iv[0];
            xv[3] = (bb[3] + cl[3] * xv[2] + cr[3] * right + cu[3] * xv[1] + cd[3] * down) * iv[3];
            if (ok[0]) x[y0 * T.w + x0] = xv[0];
            if (ok[3]) x[(y0 + 1) * T.w + x0 + 1] = xv[3];
        } else {  // cells (2j + 1, 2v) and (2j, 2v + 1)
            const float right = __shfl_down_sync(0xffffffffu, xv[0], 1);
            const float left = __shfl_up_sync(0xffffffffu, xv[3], 1);
            const float up = hu && ok[1] ? x[iu + x0 + 1] : 0.0f;
            const float down = hd ? x[id + x0] : 0.0f;
            xv[1] = (bb[1] + cl[1] * xv[0] + cr[1] * right + cu[1] * up + cd[1] * xv[3]) * iv[1];
            xv[2] = (bb[2] + cl[2] * left + cr[2] * xv[3] + cu[2] * xv[0] + cd[2] * down) * iv[2];
            if (ok[1]) x[y0 * T.w + x0 + 1] = xv[1];
            if (ok[2]) x[(y0 + 1) * T.w + x0] = xv[2];
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void tail_restrict(const TailLevel F, const TailLevel C) {
    float* f = tsf();
    const float *fc = f + F.c, *fdx = f + F.dx, *fdy = f + F.dy, *fb = f + F.b, *fx = f + F.x, *ft = f + F.t;
    const uint8_t* fm = tail_smem_raw + F.m;
    const uint8_t* cm = tail_smem_raw + C.m;
    float *cb = f + C.b, *cx = f + C.x;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int Y = ty; Y < C.h; Y += TAIL_ROWS)
        for (int X = tx; X < C.w; X += 32) {
            const int I = Y * C.w + X;
            float sum = 0.0f;
            for (int bb = 0; bb < 2; bb++)
                for (int a = 0; a < 2; a++) {
                    const int x = 2 * X + a, y = 2 * Y + bb;
                    if (x >= F.w || y >= F.h) continue;
                    const int j = y * F.w + x;
                    if (!fm[j]) continue;
                    const float xj = fx[j];
                    float ax = fc[j] * xj;
                    if (x > 0) ax += fdx[j - 1] * (xj - fx[j - 1]);
                    if (x + 1 < F.w) ax += fdx[j] * (xj - fx[j + 1]);
                    if (y > 0) ax += fdy[j - F.w] * (xj - fx[j - F.w]);
                    if (y + 1 < F.h) ax += fdy[j] * (xj - fx[j + F.w]);
                    sum += ft[j] * (fb[j] - ax);
                }
            cb[I] = cm[I] ? sum : 0.0f;
            cx[I] = 0.0f;
        }
    __syncthreads();
}

__global__ void __launch_bounds__(TAIL_THREADS) mg_tail_kernel(TailArgs A) {
    float* f = tsf();
    __shared__ TailLevel T[kMgMaxLevels];  // indexed by a run-time level
    if (threadIdx.x < kMgMaxLevels) T[threadIdx.x] = A.T[threadIdx.x];
    // every level's coefficients, weights, inverse diagonal and mask, the iterates at 0 and the coarsest inverse, as
    // packed once per Newton pass: one 16-byte copy per word, all in flight together
    float4* dst = reinterpret_cast<float4*>(tail_smem_raw);
    for (int k = threadIdx.x; k < A.img_f4; k += TAIL_THREADS) dst[k] = A.img[k];
    __syncthreads();
    {
        const int n = T[A.t].w * T[A.t].h;
        const float* b = A.L[A.t].b;
        for (int i = threadIdx.x; i < n; i += TAIL_THREADS) f[T[A.t].b + i] = b[i];
    }
    const int nc = T[A.nl - 1].w * T[A.nl - 1].h;
    const float* sinv = f + A.sinv;
    __syncthreads();
    for (int l = A.t; l < A.nl - 1; l++) {
        const TailLevel Tl = T[l];
        if (Tl.w <= 64 && Tl.h <= 64) {
            tail_sweeps_reg(Tl, 0, 2 * A.pre);
        } else {
            for (int s = 0; s < A.pre; s++) {
                tail_sweep(Tl, 0);
                tail_sweep(Tl, 1);
            }
        }
        tail_restrict(Tl, T[l + 1]);
    }
    {
        // the coarsest level exactly: x = A⁻¹ b with the inverse built once per Newton pass (mg_coarse_inverse_kernel)
        // one warp per row, the lanes splitting the row and summing by shuffles
        const TailLevel Cs = T[A.nl - 1];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int i = warp; i < nc; i += TAIL_THREADS / 32) {
            float s = 0.0f;
            for (int k = lane; k < nc; k += 32) s += sinv[i * nc + k] * f[Cs.b + k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) f[Cs.x + i] = tail_smem_raw[Cs.m + i] ? s : 0.0f;
        }
        __syncthreads();
    }
    for (int l = A.nl - 2; l >= A.t; l--) {
        const TailLevel F = T[l];
        const TailLevel Cs = T[l + 1];
        {
            const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
            for (int y = ty; y < F.h; y += TAIL_ROWS)
                for (int x = tx; x < F.w; x += 32) {
                    const int i = y * F.w + x;
                    if (tail_smem_raw[F.m + i])
                        f[F.x + i] += A.omega * f[F.t + i] * f[Cs.x + (y >> 1) * Cs.w + (x >> 1)];
                }
        }
        __syncthreads();
        if (F.w <= 64 && F.h <= 64) {
            tail_sweeps_reg(F, 1, 2 * A.post);
        } else {
            for (int s = 0; s < A.post; s++) {
                tail_sweep(F, 1);
                tail_sweep(F, 0);
            }
        }
    }
    const TailLevel top = T[A.t];
    const int n = top.w * top.h;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += TAIL_THREADS) {
        const float xv = f[top.x + i];
        A.L[A.t].x2[i] = xv;
        acc += (double)f[top.b + i] * (double)xv;
    }
    if (A.out) {
        __shared__ double red[TAIL_THREADS / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int q = 0; q < TAIL_THREADS / 32; q++) t += red[q];
            *A.out = t;
        }
    }
}

// The tail's shared-memory layout: seven float arrays per level, the coarsest inverse, then the masks; the byte size
// rounded up to 16. Fills A.T, A.sinv and A.img_f4.
size_t tail_layout(const Multigrid& M, TailArgs& A) {
    int off = 0;  // floats
    for (int l = M.tail; l < M.nlevels; l++) {
        const int n = M.L[l].w * M.L[l].h;
        TailLevel& T = A.T[l];
        T.w = M.L[l].w;
        T.h = M.L[l].h;
        T.c = off;
        T.dx = off + n;
        T.dy = off + 2 * n;
        T.b = off + 3 * n;
        T.x = off + 4 * n;
        T.inv = off + 5 * n;
        T.t = off + 6 * n;
        off += 7 * n;
    }
    const int nc = M.L[M.nlevels - 1].w * M.L[M.nlevels - 1].h;
    A.sinv = off;
    off += nc * nc;
    int moff = off * (int)sizeof(float);
    for (int l = M.tail; l < M.nlevels; l++) {
        A.T[l].m = moff;
        moff += M.L[l].w * M.L[l].h;
    }
    const size_t bytes = ((size_t)moff + 15) & ~(size_t)15;
    A.img_f4 = (int)(bytes / 16);
    return bytes;
}

size_t tail_smem(const Multigrid& M) {
    TailArgs A;
    return tail_layout(M, A);
}

// Everything the tail kernel and its packing need but the output slot.
size_t tail_args(const Multigrid& M, TailArgs& T) {
    const size_t bytes = tail_layout(M, T);
    T.t = M.tail;
    T.nl = M.nlevels;
    T.pre = M.pre;
    T.post = M.post;
    T.omega = M.omega;
    T.img = reinterpret_cast<const float4*>(M.tail_img);
    T.out = nullptr;
    for (int l = 0; l < M.nlevels; l++) T.L[l] = M.L[l];
    return bytes;
}

// The tail's image for the next V-cycles (once per Newton pass, after the coarsening): each tail level's c, dx, dy,
// inverse diagonal, weights and mask at their offsets, b and x at 0, the coarsest inverse, and the padding after the
// masks at 0. Every byte of the image is written by exactly one thread.
__global__ void mg_tail_pack_kernel(TailArgs A, const float* __restrict__ coarse_inv, float* img) {
    unsigned char* bytes = reinterpret_cast<unsigned char*>(img);
    const int stride = gridDim.x * blockDim.x, tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int l = A.t; l < A.nl; l++) {
        const TailLevel T = A.T[l];
        const MgLevel& L = A.L[l];
        const int n = T.w * T.h;
        for (int i = tid; i < n; i += stride) {
            const int x = i % T.w, y = i / T.w;
            const float c = L.c[i], dx = L.dx[i], dy = L.dy[i];
            const float d = c + dx + dy + (x > 0 ? L.dx[i - 1] : 0.0f) + (y > 0 ? L.dy[i - T.w] : 0.0f);
            const uint8_t m = L.mask[i];
            img[T.c + i] = c;
            img[T.dx + i] = dx;
            img[T.dy + i] = dy;
            img[T.b + i] = 0.0f;
            img[T.x + i] = 0.0f;
            img[T.inv + i] = m ? 1.0f / d : 0.0f;
            img[T.t + i] = l + 1 < A.nl ? (L.t ? L.t[i] : 1.0f) : 0.0f;
            bytes[T.m + i] = m;
        }
    }
    const TailLevel last = A.T[A.nl - 1];
    const int nc = last.w * last.h;
    for (int k = tid; k < nc * nc; k += stride) img[A.sinv + k] = coarse_inv[k];
    const int end = last.m + nc;
    for (int k = end + tid; k < A.img_f4 * 16; k += stride) bytes[k] = 0;
}

template <int NS, bool PRE, int SX, int SY, int NT, bool VEC, bool WT>
void launch_one(const MgLevel& L, const MgLevel& C, const float* xc, float omega, double* part, unsigned* counter,
                double* out, cudaStream_t s) {
    const dim3 grid(div_up(L.w, SX), div_up(L.h, SY));
    mg_smooth_kernel<NS, PRE, SX, SY, NT, VEC, WT><<<grid, NT, smooth_smem<NS, PRE, SX, SY>(), s>>>(
        L, C, xc, omega, part, counter, out);
}

template <int NS, bool PRE, int SX, int SY, int NT>
void launch_smooth_t(const MgLevel& L, const MgLevel& C, const float* xc, float omega, double* part, unsigned* counter,
                     double* out, cudaStream_t s) {
    // 16-byte rows (and 8-byte coarse pairs) stay aligned; the pre-smoother's odd halo would load 8 % more columns, and
    // measured slower, so it keeps the per-cell loads. Level 0 has no weights (its kernels read none).
    const bool wt = L.t != nullptr;
    if constexpr (!PRE) {
        if (L.w % 4 == 0 && C.w % 2 == 0) {
            if (wt) launch_one<NS, PRE, SX, SY, NT, true, true>(L, C, xc, omega, part, counter, out, s);
            else launch_one<NS, PRE, SX, SY, NT, true, false>(L, C, xc, omega, part, counter, out, s);
            sr_note_launch();
            return;
        }
    }
    if (wt) launch_one<NS, PRE, SX, SY, NT, false, true>(L, C, xc, omega, part, counter, out, s);
    else launch_one<NS, PRE, SX, SY, NT, false, false>(L, C, xc, omega, part, counter, out, s);
    sr_note_launch();
}

bool small_tiles(const MgLevel& L) { return (size_t)div_up(L.w, BIG_SX) * div_up(L.h, BIG_SY) < 2 * 148; }

// A smoother's tile height: of the even heights from SY_MAX down to SY_MAX - 6, the one with the most output cells per
// sweep slot (a half-sweep gives each thread ceil(cells of one colour in the halo'd tile / NT) slots; the last slot
// round should be nearly full, or most threads wait at its barrier).
template <int NS, bool PRE, int SX, int SY_MAX, int NT>
constexpr int tile_sy() {
    constexpr int H = PRE ? NS + 1 : NS;
    int best = SY_MAX;
    double best_rate = 0.0;
    for (int sy = SY_MAX; sy >= SY_MAX - 6; sy -= 2) {
        const int hn = (SX + 2 * H) / 2 * (sy + 2 * H);
        const int slots = (hn + NT - 1) / NT;
        const double rate = (double)(SX * sy) / slots;
        if (rate > best_rate) {
            best_rate = rate;
            best = sy;
        }
    }
    return best;
}

template <int NS, bool PRE>
void launch_rowband(const MgLevel& L, const MgLevel& C, const float* xc, float omega, double* part, unsigned* counter,
                    double* out, cudaStream_t s) {
    constexpr int H = rb_halo<NS, PRE>();
    const dim3 grid(div_up(L.w, RB_RX - 2 * H), div_up(L.h, RB_RY - 2 * H));
    // rows of 16 bytes and 16-byte bases: the region staged by TMA
    auto aligned = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    if (L.w % 4 == 0 && aligned(L.b) && aligned(L.c) && aligned(L.dx) && aligned(L.dy) && aligned(L.x) &&
        (!L.t || aligned(L.t))) {
        CUtensorMap mb, mc, mdx, mdy, mx;
        tma_encode_planes(&mb, L.b, L.w, L.h, 1, RB_TMA_X, RB_TMA_Y);
        tma_encode_planes(&mc, L.c, L.w, L.h, 1, RB_TMA_X, RB_TMA_Y);
        tma_encode_planes(&mdx, L.dx, L.w, L.h, 1, RB_TMA_X, RB_TMA_Y);
        tma_encode_planes(&mdy, L.dy, L.w, L.h, 1, RB_TMA_X, RB_TMA_Y);
        if (!PRE) tma_encode_planes(&mx, L.x, L.w, L.h, 1, RB_TMA_X, RB_TMA_Y);
        else if (L.t) tma_encode_planes(&mx, L.t, L.w, L.h, 1, RB_TMA_X, RB_TMA_Y);
        else mx = mb;
        auto go = [&](auto kernel, size_t smem, bool& attr) {
            if (!attr) {  // the instance's shared-memory attribute, once per process
                SR_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                attr = true;
            }
            kernel<<<grid, RB_NT, smem, s>>>(mb, mc, mdx, mdy, mx, L, C, xc, omega, part, counter, out);
        };
        static bool attr_w = false, attr_u = false;
        if (L.t) go(mg_rowband_tma_kernel<NS, PRE, true>, rb_tma_smem<PRE, true>(), attr_w);
        else go(mg_rowband_tma_kernel<NS, PRE, false>, rb_tma_smem<PRE, false>(), attr_u);
        sr_note_launch();
        return;
    }
    if (L.t) mg_rowband_kernel<NS, PRE, true><<<grid, RB_NT, 0, s>>>(L, C, xc, omega, part, counter, out);
    else mg_rowband_kernel<NS, PRE, false><<<grid, RB_NT, 0, s>>>(L, C, xc, omega, part, counter, out);
    sr_note_launch();
}

template <int NS, bool PRE>
void launch_smooth(const MgLevel& L, const MgLevel& C, const float* xc, float omega, double* part, unsigned* counter,
                   double* out, int tile, cudaStream_t s) {
    if (tile < 0 ? small_tiles(L) : tile == 1)
        launch_smooth_t<NS, PRE, SMALL_SX, tile_sy<NS, PRE, SMALL_SX, SMALL_SY, SMALL_NT>(), SMALL_NT>(
            L, C, xc, omega, part, counter, out, s);
    else if (L.w % 2 == 0)  // the row-band kernel loads cell pairs as 8-byte words
        launch_rowband<NS, PRE>(L, C, xc, omega, part, counter, out, s);
    else
        launch_smooth_t<NS, PRE, BIG_SX, tile_sy<NS, PRE, BIG_SX, BIG_SY, BIG_NT>(), BIG_NT>(L, C, xc, omega, part,
                                                                                           counter, out, s);
}

// `tile`: 0 the big tile, 1 the small one, -1 by the CTA-count rule (small_tiles).
void smooth(int nu, bool pre, const MgLevel& L, const MgLevel& C, const float* xc, float omega, double* part,
            unsigned* counter, double* out, cudaStream_t s, int tile = -1) {
    if (pre) {
        if (nu == 1) launch_smooth<2, true>(L, C, xc, omega, part, counter, out, tile, s);
        else if (nu == 2) launch_smooth<4, true>(L, C, xc, omega, part, counter, out, tile, s);
        else if (nu == 3) launch_smooth<6, true>(L, C, xc, omega, part, counter, out, tile, s);
        else launch_smooth<8, true>(L, C, xc, omega, part, counter, out, tile, s);
    } else {
        if (nu == 1) launch_smooth<2, false>(L, C, xc, omega, part, counter, out, tile, s);
        else if (nu == 2) launch_smooth<4, false>(L, C, xc, omega, part, counter, out, tile, s);
        else if (nu == 3) launch_smooth<6, false>(L, C, xc, omega, part, counter, out, tile, s);
        else launch_smooth<8, false>(L, C, xc, omega, part, counter, out, tile, s);
    }
}

template <int NS, bool PRE, int SX, int SY, int NT, bool VEC, bool WT>
void set_attribute_one() {
    SR_CUDA_TRY(cudaFuncSetAttribute(mg_smooth_kernel<NS, PRE, SX, SY, NT, VEC, WT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smooth_smem<NS, PRE, SX, SY>()));
}

template <int NS, int SX, int SY, int NT>
void set_attributes_tile() {
    constexpr int PSY = tile_sy<NS, true, SX, SY, NT>(), QSY = tile_sy<NS, false, SX, SY, NT>();
    set_attribute_one<NS, true, SX, PSY, NT, false, false>();
    set_attribute_one<NS, true, SX, PSY, NT, false, true>();
    set_attribute_one<NS, false, SX, QSY, NT, false, false>();
    set_attribute_one<NS, false, SX, QSY, NT, false, true>();
    set_attribute_one<NS, false, SX, QSY, NT, true, false>();
    set_attribute_one<NS, false, SX, QSY, NT, true, true>();
}

template <int NS>
void set_attributes_ns() {
    set_attributes_tile<NS, BIG_SX, BIG_SY, BIG_NT>();
    set_attributes_tile<NS, SMALL_SX, SMALL_SY, SMALL_NT>();
}

int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

size_t mg_smooth_ctas(int w, int h) {
    MgLevel L;
    L.w = w;
    L.h = h;
    // a bound: the shortest tile tile_sy can pick, or the row-band kernel's smallest output tile (V(4,4)'s pre-smoother)
    const size_t rb = (size_t)div_up(w, RB_RX - 2 * rb_halo<8, true>()) * div_up(h, RB_RY - 2 * rb_halo<8, true>());
    return std::max(rb, small_tiles(L) ? (size_t)div_up(w, SMALL_SX) * div_up(h, SMALL_SY - 6)
                                       : (size_t)div_up(w, BIG_SX) * div_up(h, BIG_SY - 6));
}

void Multigrid::create(int w, int h, int pre_, int post_) {
    SR_REQUIRE(pre_ >= 1 && pre_ <= 4 && post_ >= 1 && post_ <= 4, "V-cycle sweeps must be 1..4");
    pre = pre_;
    post = post_;
    nlevels = 0;
    int lw = w, lh = h;
    for (;;) {
        MgLevel& L = this->L[nlevels];
        L.w = lw;
        L.h = lh;
        const size_t n = (size_t)lw * lh;
        SR_CUDA_TRY(cudaMalloc(&L.c, n * sizeof(float)));
        SR_CUDA_TRY(cudaMalloc(&L.dx, n * sizeof(float)));
        SR_CUDA_TRY(cudaMalloc(&L.dy, n * sizeof(float)));
        SR_CUDA_TRY(cudaMalloc(&L.mask, n));
        SR_CUDA_TRY(cudaMalloc(&L.x, n * sizeof(float)));
        if (nlevels > 0) {
            SR_CUDA_TRY(cudaMalloc(&L.t, n * sizeof(float)));
            SR_CUDA_TRY(cudaMalloc(&L.b, n * sizeof(float)));
            SR_CUDA_TRY(cudaMalloc(&L.x2, n * sizeof(float)));
        }
        nlevels++;
        if ((lw <= 4 && lh <= 4) || nlevels == kMgMaxLevels) break;
        lw = (lw + 1) / 2;
        lh = (lh + 1) / 2;
    }
    tail = 0;
    while ((size_t)L[tail].w * L[tail].h > (size_t)kMgTailCells) tail++;
    size_t ts = tail_smem(*this);
    SR_REQUIRE(ts <= 200 * 1024, "the coarse tail does not fit in shared memory");
    SR_CUDA_TRY(cudaFuncSetAttribute(mg_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ts));
    const size_t nc = (size_t)L[nlevels - 1].w * L[nlevels - 1].h;
    SR_REQUIRE(nc <= 64, "the coarsest level holds more than 64 cells");
    SR_CUDA_TRY(cudaMalloc(&coarse_inv, sizeof(float) * nc * nc));
    SR_CUDA_TRY(cudaMalloc(&tail_img, ts));
    SR_CUDA_TRY(cudaMalloc(&err, sizeof(int)));
    SR_CUDA_TRY(cudaMemset(err, 0, sizeof(int)));
    for (int l = 0; l < nlevels; l++) L[l].err = err;
    SR_CUDA_TRY(cudaFuncSetAttribute(mg_coarse_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(2 * nc * 2 * nc * sizeof(double))));
    set_attributes_ns<2>();
    set_attributes_ns<4>();
    set_attributes_ns<6>();
    set_attributes_ns<8>();
}

void Multigrid::destroy() {
    for (int l = 0; l < nlevels; l++) {
        cudaFree(L[l].c);
        cudaFree(L[l].dx);
        cudaFree(L[l].dy);
        cudaFree(L[l].mask);
        cudaFree(L[l].x);
        if (l > 0) {
            cudaFree(L[l].t);
            cudaFree(L[l].b);
            cudaFree(L[l].x2);
        }
        L[l] = MgLevel();
    }
    cudaFree(coarse_inv);
    coarse_inv = nullptr;
    cudaFree(tail_img);
    tail_img = nullptr;
    cudaFree(err);
    err = nullptr;
    nlevels = 0;
}

bool Multigrid::error(cudaStream_t s) {
    if (!err) return false;
    int v = 0;
    SR_CUDA_TRY(cudaMemcpyAsync(&v, err, sizeof v, cudaMemcpyDeviceToHost, s));
    SR_CUDA_TRY(cudaStreamSynchronize(s));
    if (v) SR_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
    return v != 0;
}

size_t Multigrid::bytes() const {
    size_t s = 0;
    for (int l = 0; l < nlevels; l++)
        s += (size_t)L[l].w * L[l].h * (l ? 7 * sizeof(float) + 1 : 4 * sizeof(float) + 1);
    return s;
}

void Multigrid::set_couplings(const double* kx, const double* ky, const uint8_t* gas, cudaStream_t s) {
    mg_couplings0_kernel<<<grid_for((size_t)L[0].w * L[0].h), 256, 0, s>>>(L[0], kx, ky, gas);
    sr_note_launch();
}

// The smoother tile of each level below 0 (level 0 keeps the CTA-count rule, which bounds its grid-sum partials),
// chosen by timing on the level's first operator: per candidate (the big and the small tile) one warm-up pre- and
// post-smoother, then the median of kTuneReps timed pairs; the rule's tile is kept unless the other is at least
// kTuneMargin faster, so that run-to-run noise does not flip a choice. Choices are kept per level size for the process
// (a batch's worlds of one size tune once).
constexpr int kTuneReps = 7;
constexpr float kTuneMargin = 0.95f;

void Multigrid::autotune(cudaStream_t s) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int>, int> chosen;  // (w, h, sweeps before, after) -> tile
    tuned = true;
    cudaEvent_t a, b;
    SR_CUDA_TRY(cudaEventCreate(&a));
    SR_CUDA_TRY(cudaEventCreate(&b));
    for (int l = 1; l < tail; l++) {
        const std::tuple<int, int, int, int> key(L[l].w, L[l].h, pre, post);
        {
            std::lock_guard<std::mutex> g(mu);
            auto it = chosen.find(key);
            if (it != chosen.end()) {
                tile[l] = it->second;
                continue;
            }
        }
        float med[2];
        for (int cand = 0; cand < 2; cand++) {
            float t[kTuneReps];
            for (int rep = -1; rep < kTuneReps; rep++) {  // rep -1 warms up
                SR_CUDA_TRY(cudaEventRecord(a, s));
                smooth(pre, true, L[l], L[l + 1], nullptr, omega, nullptr, nullptr, nullptr, s, cand);
                smooth(post, false, L[l], L[l + 1], L[l + 1].x2, omega, nullptr, nullptr, nullptr, s, cand);
                SR_CUDA_TRY(cudaEventRecord(b, s));
                SR_CUDA_TRY(cudaEventSynchronize(b));
                float ms = 0.0f;
                SR_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
                if (rep >= 0) t[rep] = ms;
            }
            std::sort(t, t + kTuneReps);
            med[cand] = t[kTuneReps / 2];
        }
        const int rule = small_tiles(L[l]) ? 1 : 0, other = 1 - rule;
        const int pick = med[other] < kTuneMargin * med[rule] ? other : rule;
        tile[l] = pick;
        std::lock_guard<std::mutex> g(mu);
        chosen[key] = pick;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}

void Multigrid::coarsen(cudaStream_t s) {
    for (int l = 1; l < nlevels; l++) {
        if (l == 1) {
            mg_aggregate_kernel<<<grid_for((size_t)L[1].w * L[1].h), 256, 0, s>>>(L[0], L[1]);
        } else {
            const dim3 grid(div_up(L[l - 1].w, CO_S), div_up(L[l - 1].h, CO_S));
            mg_coarsen_kernel<<<grid, CO_NT, 0, s>>>(L[l - 1], L[l]);
        }
        sr_note_launch();
    }
    const MgLevel& C = L[nlevels - 1];
    const size_t nc = (size_t)C.w * C.h;
    mg_coarse_inverse_kernel<<<1, 1024, 2 * nc * 2 * nc * sizeof(double), s>>>(C, coarse_inv);
    sr_note_launch();
    TailArgs T;
    tail_args(*this, T);
    mg_tail_pack_kernel<<<8, 256, 0, s>>>(T, coarse_inv, tail_img);
    sr_note_launch();
    if (!tuned) autotune(s);
}

void Multigrid::apply(const float* r, float* z, double* part, unsigned* counter, double* rz_out, cudaStream_t s) {
    L[0].b = const_cast<float*>(r);
    L[0].x2 = z;
    for (int l = 0; l < tail; l++)
        smooth(pre, true, L[l], L[l + 1], nullptr, omega, nullptr, nullptr, nullptr, s, tile[l]);
    TailArgs T;
    const size_t ts = tail_args(*this, T);
    T.out = tail == 0 ? rz_out : nullptr;
    mg_tail_kernel<<<1, TAIL_THREADS, ts, s>>>(T);
    sr_note_launch();
    for (int l = tail - 1; l >= 0; l--)
        smooth(post, false, L[l], L[l + 1], L[l + 1].x2, omega, l == 0 ? part : nullptr, l == 0 ? counter : nullptr,
               l == 0 ? rz_out : nullptr, s, tile[l]);
}

void Multigrid::time_level0(int reps, void* flush, size_t flush_bytes, cudaStream_t s, double* pre_ms,
                            double* post_ms) {
    *pre_ms = *post_ms = 0.0;
    if (tail == 0 || !L[0].b || !L[0].x2 || reps < 1) return;
    cudaEvent_t a, b;
    SR_CUDA_TRY(cudaEventCreate(&a));
    SR_CUDA_TRY(cudaEventCreate(&b));
    for (int which = 0; which < 2; which++) {
        double total = 0.0;
        for (int k = 0; k < reps; k++) {
            SR_CUDA_TRY(cudaMemsetAsync(flush, k & 0xff, flush_bytes, s));
            SR_CUDA_TRY(cudaEventRecord(a, s));
            if (which == 0)
                smooth(pre, true, L[0], L[1], nullptr, omega, nullptr, nullptr, nullptr, s);
            else
                smooth(post, false, L[0], L[1], L[1].x2, omega, nullptr, nullptr, nullptr, s);
            SR_CUDA_TRY(cudaEventRecord(b, s));
            SR_CUDA_TRY(cudaEventSynchronize(b));
            float t = 0.0f;
            SR_CUDA_TRY(cudaEventElapsedTime(&t, a, b));
            total += t;
        }
        (which ? *post_ms : *pre_ms) = total / reps;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}
