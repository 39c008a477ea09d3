// mg.cu — the multigrid V-cycle (FP32) of the implicit FLD solve; see mg.cuh for the scheme.
#include <vector>

#include "mg.cuh"

namespace {

constexpr int SX = 64, SY = 32;  // smoother tile (outputs)
constexpr int SMOOTH_THREADS = 512;
constexpr int TAIL_THREADS = 1024;

struct TailArgs {
    int t, nl, pre, post;
    float omega;
    MgLevel L[kMgMaxLevels];
    double* part;  // non-null when the tail's top level is level 0: partials of <b, x2>
};

// Level 0's couplings to the +x / +y neighbours from the f64 faces, zero unless both cells are gas.
__global__ void mg_couplings0_kernel(MgLevel L, const double* __restrict__ kx, const double* __restrict__ ky,
                                     const uint8_t* __restrict__ gas) {
    const int w = L.w, h = L.h;
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % w), y = (int)(i / w);
        const bool g = gas[i];
        L.mask[i] = g;
        L.dx[i] = (g && x + 1 < w && gas[i + 1]) ? (float)kx[(size_t)y * (w + 1) + x + 1] : 0.0f;
        L.dy[i] = (g && y + 1 < h && gas[i + w]) ? (float)ky[(size_t)(y + 1) * w + x] : 0.0f;
    }
}

// Level l+1 from level l: Galerkin aggregation of 2x2 cells (mg.cuh).
__global__ void mg_coarsen_kernel(MgLevel F, MgLevel C) {
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

// One smoother on a big level: all NS half-sweeps of a tile in shared memory. PRE: from x = 0, red first, into L.x.
// POST: from x = L.x + ω P xc (xc the coarse level's result), black first, into L.x2; `part` gets <b, x2> per CTA.
template <int NS, bool PRE>
__global__ void __launch_bounds__(SMOOTH_THREADS) mg_smooth_kernel(MgLevel L, const float* __restrict__ xc, int wc,
                                                                    float omega, double* part) {
    constexpr int H = NS;
    constexpr int RX = SX + 2 * H, RY = SY + 2 * H, RN = RX * RY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sx = reinterpret_cast<float*>(smem_raw);
    float* sb = sx + RN;
    float* sdx = sb + RN;
    float* sdy = sdx + RN;
    float* sinv = sdy + RN;
    uint8_t* sm = reinterpret_cast<uint8_t*>(sinv + RN);
    const int w = L.w, h = L.h;
    const int X0 = blockIdx.x * SX - H, Y0 = blockIdx.y * SY - H;
    const int tid = threadIdx.x;
    float* sc = sinv;  // c staged in the inverse-diagonal slot, replaced below
    for (int k = tid; k < RN; k += SMOOTH_THREADS) {
        const int lx = k % RX, ly = k / RX;
        const int gx = X0 + lx, gy = Y0 + ly;
        float b = 0.0f, c = 1.0f, dx = 0.0f, dy = 0.0f, x = 0.0f;
        uint8_t m = 0;
        if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
            const size_t i = (size_t)gy * w + gx;
            b = L.b[i];
            c = L.c[i];
            dx = L.dx[i];
            dy = L.dy[i];
            m = L.mask[i];
            if (!PRE) {
                x = L.x[i];
                if (m) x += omega * xc[(size_t)(gy >> 1) * wc + (gx >> 1)];
            }
        }
        sx[k] = x;
        sb[k] = b;
        sdx[k] = dx;
        sdy[k] = dy;
        sc[k] = c;
        sm[k] = m;
    }
    __syncthreads();
    // inverse diagonals of the interior (ring 0 is never updated)
    float inv_local[(RN + SMOOTH_THREADS - 1) / SMOOTH_THREADS];
#pragma unroll
    for (int q = 0; q < (RN + SMOOTH_THREADS - 1) / SMOOTH_THREADS; q++) {
        const int k = tid + q * SMOOTH_THREADS;
        inv_local[q] = 0.0f;
        if (k < RN) {
            const int lx = k % RX, ly = k / RX;
            if (lx > 0 && ly > 0 && lx < RX - 1 && ly < RY - 1)
                inv_local[q] = 1.0f / (sc[k] + sdx[k] + sdx[k - 1] + sdy[k] + sdy[k - RX]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < (RN + SMOOTH_THREADS - 1) / SMOOTH_THREADS; q++) {
        const int k = tid + q * SMOOTH_THREADS;
        if (k < RN) sinv[k] = inv_local[q];
    }
    __syncthreads();
    constexpr int HALF = RX / 2;
    for (int s = 0; s < NS; s++) {
        const int color = PRE ? (s & 1) : 1 - (s & 1);
        for (int k = tid; k < RY * HALF; k += SMOOTH_THREADS) {
            const int ly = k / HALF;
            const int lx = 2 * (k % HALF) + ((color + X0 + Y0 + ly) & 1);
            if (lx < 1 || lx >= RX - 1 || ly < 1 || ly >= RY - 1) continue;
            const int l = ly * RX + lx;
            if (!sm[l]) continue;
            sx[l] = (sb[l] + sdx[l - 1] * sx[l - 1] + sdx[l] * sx[l + 1] + sdy[l - RX] * sx[l - RX] +
                     sdy[l] * sx[l + RX]) *
                    sinv[l];
        }
        __syncthreads();
    }
    double acc = 0.0;
    float* out = PRE ? L.x : L.x2;
    for (int k = tid; k < SX * SY; k += SMOOTH_THREADS) {
        const int ox = k % SX, oy = k / SX;
        const int gx = X0 + H + ox, gy = Y0 + H + oy;
        if (gx < w && gy < h) {
            const int l = (oy + H) * RX + ox + H;
            out[(size_t)gy * w + gx] = sx[l];
            if (!PRE && part) acc += (double)sb[l] * (double)sx[l];
        }
    }
    if (!PRE && part) {
        __shared__ double red[SMOOTH_THREADS / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int q = 0; q < SMOOTH_THREADS / 32; q++) t += red[q];
            part[blockIdx.y * gridDim.x + blockIdx.x] = t;
        }
    }
}

// The residual of the pre-smoothed level summed over each 2x2 aggregate: the coarse right-hand side.
__global__ void mg_restrict_kernel(MgLevel F, MgLevel C) {
    const int wc = C.w, hc = C.h, wf = F.w, hf = F.h;
    const size_t nc = (size_t)wc * hc;
    for (size_t I = (size_t)blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += (size_t)gridDim.x * blockDim.x) {
        const int X = (int)(I % wc), Y = (int)(I / wc);
        float sum = 0.0f;
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int a = 0; a < 2; a++) {
                const int x = 2 * X + a, y = 2 * Y + b;
                if (x >= wf || y >= hf) continue;
                const size_t j = (size_t)y * wf + x;
                if (!F.mask[j]) continue;
                const float xl = x > 0 ? F.x[j - 1] : 0.0f, xr = x + 1 < wf ? F.x[j + 1] : 0.0f;
                const float xu = y > 0 ? F.x[j - wf] : 0.0f, xd = y + 1 < hf ? F.x[j + wf] : 0.0f;
                const float dl = x > 0 ? F.dx[j - 1] : 0.0f, du = y > 0 ? F.dy[j - wf] : 0.0f;
                const float dr = F.dx[j], dd = F.dy[j];
                const float diag = F.c[j] + dl + dr + du + dd;
                sum += F.b[j] - (diag * F.x[j] - dl * xl - dr * xr - du * xu - dd * xd);
            }
        C.b[I] = C.mask[I] ? sum : 0.0f;
    }
}

// ---- the coarse tail: every level from t on, inside one CTA
struct TailLevel {
    int w, h;
    float *c, *dx, *dy, *b, *x;
    uint8_t* m;
};

__device__ void tail_sweep(const TailLevel& T, int color) {
    const int n = T.w * T.h;
    for (int i = threadIdx.x; i < n; i += TAIL_THREADS) {
        const int x = i % T.w, y = i / T.w;
        if (((x + y) & 1) != color || !T.m[i]) continue;
        const float dl = x > 0 ? T.dx[i - 1] : 0.0f, du = y > 0 ? T.dy[i - T.w] : 0.0f;
        const float dr = T.dx[i], dd = T.dy[i];
        float s = T.b[i];
        if (x > 0) s += dl * T.x[i - 1];
        if (x + 1 < T.w) s += dr * T.x[i + 1];
        if (y > 0) s += du * T.x[i - T.w];
        if (y + 1 < T.h) s += dd * T.x[i + T.w];
        T.x[i] = s / (T.c[i] + dl + dr + du + dd);
    }
    __syncthreads();
}

__device__ void tail_restrict(const TailLevel& F, const TailLevel& C) {
    const int nc = C.w * C.h;
    for (int I = threadIdx.x; I < nc; I += TAIL_THREADS) {
        const int X = I % C.w, Y = I / C.w;
        float sum = 0.0f;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                const int x = 2 * X + a, y = 2 * Y + b;
                if (x >= F.w || y >= F.h) continue;
                const int j = y * F.w + x;
                if (!F.m[j]) continue;
                const float xl = x > 0 ? F.x[j - 1] : 0.0f, xr = x + 1 < F.w ? F.x[j + 1] : 0.0f;
                const float xu = y > 0 ? F.x[j - F.w] : 0.0f, xd = y + 1 < F.h ? F.x[j + F.w] : 0.0f;
                const float dl = x > 0 ? F.dx[j - 1] : 0.0f, du = y > 0 ? F.dy[j - F.w] : 0.0f;
                const float dr = F.dx[j], dd = F.dy[j];
                sum += F.b[j] - ((F.c[j] + dl + dr + du + dd) * F.x[j] - dl * xl - dr * xr - du * xu - dd * xd);
            }
        C.b[I] = C.m[I] ? sum : 0.0f;
        C.x[I] = 0.0f;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(TAIL_THREADS) mg_tail_kernel(TailArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TailLevel T[kMgMaxLevels];
    // carve shared memory: five float arrays per level, then the masks
    size_t off = 0;
    for (int l = A.t; l < A.nl; l++) {
        const int n = A.L[l].w * A.L[l].h;
        float* base = reinterpret_cast<float*>(smem_raw + off);
        T[l].w = A.L[l].w;
        T[l].h = A.L[l].h;
        T[l].c = base;
        T[l].dx = base + n;
        T[l].dy = base + 2 * n;
        T[l].b = base + 3 * n;
        T[l].x = base + 4 * n;
        off += sizeof(float) * 5 * (size_t)n;
    }
    for (int l = A.t; l < A.nl; l++) {
        T[l].m = reinterpret_cast<uint8_t*>(smem_raw + off);
        off += (size_t)A.L[l].w * A.L[l].h;
    }
    for (int l = A.t; l < A.nl; l++) {
        const int n = T[l].w * T[l].h;
        for (int i = threadIdx.x; i < n; i += TAIL_THREADS) {
            T[l].c[i] = A.L[l].c[i];
            T[l].dx[i] = A.L[l].dx[i];
            T[l].dy[i] = A.L[l].dy[i];
            T[l].m[i] = A.L[l].mask[i];
            T[l].x[i] = 0.0f;
            if (l == A.t) T[l].b[i] = A.L[l].b[i];
        }
    }
    __syncthreads();
    for (int l = A.t; l < A.nl - 1; l++) {
        for (int s = 0; s < A.pre; s++) {
            tail_sweep(T[l], 0);
            tail_sweep(T[l], 1);
        }
        tail_restrict(T[l], T[l + 1]);
    }
    {
        const TailLevel& C = T[A.nl - 1];
        tail_sweep(C, 0);
        for (int s = 0; s < kMgCoarsestSweeps; s++) {
            tail_sweep(C, 1);
            tail_sweep(C, 0);
        }
    }
    for (int l = A.nl - 2; l >= A.t; l--) {
        const TailLevel& F = T[l];
        const TailLevel& C = T[l + 1];
        const int n = F.w * F.h;
        for (int i = threadIdx.x; i < n; i += TAIL_THREADS) {
            const int x = i % F.w, y = i / F.w;
            if (F.m[i]) F.x[i] += A.omega * C.x[(y >> 1) * C.w + (x >> 1)];
        }
        __syncthreads();
        for (int s = 0; s < A.post; s++) {
            tail_sweep(F, 1);
            tail_sweep(F, 0);
        }
    }
    const TailLevel& top = T[A.t];
    const int n = top.w * top.h;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += TAIL_THREADS) {
        A.L[A.t].x2[i] = top.x[i];
        acc += (double)top.b[i] * (double)top.x[i];
    }
    if (A.part) {
        __shared__ double red[TAIL_THREADS / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int q = 0; q < TAIL_THREADS / 32; q++) t += red[q];
            A.part[0] = t;
        }
    }
}

size_t tail_smem(const Multigrid& M) {
    size_t s = 0;
    for (int l = M.tail; l < M.nlevels; l++) s += (size_t)M.L[l].w * M.L[l].h * (5 * sizeof(float) + 1);
    return (s + 15) & ~(size_t)15;
}

template <int NS>
size_t smooth_smem() {
    constexpr int RN = (SX + 2 * NS) * (SY + 2 * NS);
    return (size_t)RN * (5 * sizeof(float) + 1);
}

template <int NS, bool PRE>
void launch_smooth(const MgLevel& L, const float* xc, int wc, float omega, double* part, cudaStream_t s) {
    size_t smem = smooth_smem<NS>();
    cudaFuncSetAttribute(mg_smooth_kernel<NS, PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(div_up(L.w, SX), div_up(L.h, SY));
    mg_smooth_kernel<NS, PRE><<<grid, SMOOTH_THREADS, smem, s>>>(L, xc, wc, omega, part);
    sr_note_launch();
}

void smooth(int nu, bool pre, const MgLevel& L, const float* xc, int wc, float omega, double* part, cudaStream_t s) {
    if (pre) {
        if (nu == 1) launch_smooth<2, true>(L, xc, wc, omega, part, s);
        else if (nu == 2) launch_smooth<4, true>(L, xc, wc, omega, part, s);
        else launch_smooth<6, true>(L, xc, wc, omega, part, s);
    } else {
        if (nu == 1) launch_smooth<2, false>(L, xc, wc, omega, part, s);
        else if (nu == 2) launch_smooth<4, false>(L, xc, wc, omega, part, s);
        else launch_smooth<6, false>(L, xc, wc, omega, part, s);
    }
}

int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

void Multigrid::create(int w, int h, int pre_, int post_) {
    SR_REQUIRE(pre_ >= 1 && pre_ <= 3 && post_ >= 1 && post_ <= 3, "V-cycle sweeps must be 1..3");
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
            SR_CUDA_TRY(cudaMalloc(&L.b, n * sizeof(float)));
            SR_CUDA_TRY(cudaMalloc(&L.x2, n * sizeof(float)));
        }
        nlevels++;
        if ((lw <= 8 && lh <= 8) || nlevels == kMgMaxLevels) break;
        lw = (lw + 1) / 2;
        lh = (lh + 1) / 2;
    }
    tail = 0;
    while ((size_t)L[tail].w * L[tail].h > (size_t)kMgTailCells) tail++;
    part_count = tail == 0 ? 1 : (int)(div_up(w, SX) * div_up(h, SY));
    SR_CUDA_TRY(cudaMalloc(&part, sizeof(double) * part_count));
    size_t ts = tail_smem(*this);
    SR_REQUIRE(ts <= 200 * 1024, "the coarse tail does not fit in shared memory");
    SR_CUDA_TRY(cudaFuncSetAttribute(mg_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ts));
}

void Multigrid::destroy() {
    for (int l = 0; l < nlevels; l++) {
        cudaFree(L[l].c);
        cudaFree(L[l].dx);
        cudaFree(L[l].dy);
        cudaFree(L[l].mask);
        cudaFree(L[l].x);
        if (l > 0) {
            cudaFree(L[l].b);
            cudaFree(L[l].x2);
        }
        L[l] = MgLevel();
    }
    cudaFree(part);
    part = nullptr;
    nlevels = 0;
}

size_t Multigrid::bytes() const {
    size_t s = 0;
    for (int l = 0; l < nlevels; l++) s += (size_t)L[l].w * L[l].h * (l ? 6 * sizeof(float) + 1 : 4 * sizeof(float) + 1);
    return s;
}

void Multigrid::set_couplings(const double* kx, const double* ky, const uint8_t* gas, cudaStream_t s) {
    mg_couplings0_kernel<<<grid_for((size_t)L[0].w * L[0].h), 256, 0, s>>>(L[0], kx, ky, gas);
    sr_note_launch();
}

void Multigrid::coarsen(cudaStream_t s) {
    for (int l = 1; l < nlevels; l++)
        mg_coarsen_kernel<<<grid_for((size_t)L[l].w * L[l].h), 256, 0, s>>>(L[l - 1], L[l]);
    sr_note_launch();
}

void Multigrid::apply(const float* r, float* z, cudaStream_t s) {
    L[0].b = const_cast<float*>(r);
    L[0].x2 = z;
    for (int l = 0; l < tail; l++) {
        smooth(pre, true, L[l], nullptr, 0, omega, nullptr, s);
        mg_restrict_kernel<<<grid_for((size_t)L[l + 1].w * L[l + 1].h), 256, 0, s>>>(L[l], L[l + 1]);
    sr_note_launch();
    }
    TailArgs T;
    T.t = tail;
    T.nl = nlevels;
    T.pre = pre;
    T.post = post;
    T.omega = omega;
    for (int l = 0; l < nlevels; l++) T.L[l] = L[l];
    T.part = tail == 0 ? part : nullptr;
    mg_tail_kernel<<<1, TAIL_THREADS, tail_smem(*this), s>>>(T);
    sr_note_launch();
    for (int l = tail - 1; l >= 0; l--)
        smooth(post, false, L[l], L[l + 1].x2, L[l + 1].w, omega, l == 0 ? part : nullptr, s);
}
