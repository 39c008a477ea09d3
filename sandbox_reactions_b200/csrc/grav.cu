// grav.cu — P2, self-gravity by zero-padded FFT convolution (Hockney–Eastwood), FP32 on sm_100a.
//
// φ = K ∗ Σ_src over the w x h world padded to px x py (px the smallest power of two >= 2w, >= 32), then
// g = -∇φ by central differences, the outer ring reading the free-space φ one cell past the world
// (crates/sr-physics/src/reference/grav.rs, reference/fft.rs:238-282). Three FFT passes and a gradient pass:
//   1. rows: two real rows packed as one complex row, a px-point FFT in shared memory, unpacked to the half spectrum
//      kx = 0..px/2, written column-major (each spectrum column kx contiguous in y);
//   2. columns: each kx column zero-padded to py, forward FFT, times the kernel's real-even spectrum K̂ (the quarter
//      table, 1/(px py) folded in), inverse FFT, the world's rows and the two ring rows kept, in place;
//   3. inverse rows: two output rows packed through Hermitian symmetry into one complex inverse FFT, the world's
//      columns and the ring columns kept;
//   4. gradient: φ and g = -∇φ.
// The FFT is a Stockham autosort over radix-16 stages (a radix-2/4/8 stage last when log2 N is not a multiple of 4),
// each thread holding 16 points in registers between shared-memory exchanges; inter-stage twiddles come from a table
// built in f64 on the host.
#include <math.h>

#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "grav.cuh"

namespace {

__device__ __constant__ float kCos16[16] = {1.0f, 9.238795325e-01f, 7.071067812e-01f, 3.826834324e-01f, 0.0f,
                                             -3.826834324e-01f, -7.071067812e-01f, -9.238795325e-01f, -1.0f,
                                             -9.238795325e-01f, -7.071067812e-01f, -3.826834324e-01f, 0.0f,
                                             3.826834324e-01f, 7.071067812e-01f, 9.238795325e-01f};
__device__ __constant__ float kSin16[16] = {0.0f, 3.826834324e-01f, 7.071067812e-01f, 9.238795325e-01f, 1.0f,
                                             9.238795325e-01f, 7.071067812e-01f, 3.826834324e-01f, 0.0f,
                                             -3.826834324e-01f, -7.071067812e-01f, -9.238795325e-01f, -1.0f,
                                             -9.238795325e-01f, -7.071067812e-01f, -3.826834324e-01f};

// Shared-memory FFT buffers hold one float2 of padding after every 16 points: the radix-16 stages' scattered writes
// (stride Ns·16 elements in the first stage) and strided reads then fall on different banks.
__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }
template <int N>
constexpr int fft_len() {
    return N + N / 16;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-register DFT of R (<= 16) points, natural order in and out, by recursive decimation in time. Forward uses
// e^{-2πik/R}; inverse its conjugate (unscaled).
template <int R, bool INV>
struct Dft {
    __device__ __forceinline__ static void run(float2* v) {
        float2 e[R / 2], o[R / 2];
#pragma unroll
        for (int k = 0; k < R / 2; k++) {
            e[k] = v[2 * k];
            o[k] = v[2 * k + 1];
        }
        Dft<R / 2, INV>::run(e);
        Dft<R / 2, INV>::run(o);
#pragma unroll
        for (int k = 0; k < R / 2; k++) {
            const int m = k * (16 / R);
            float2 wk = make_float2(kCos16[m], INV ? kSin16[m] : -kSin16[m]);
            float2 t = k == 0 ? o[k] : cmul(o[k], wk);
            v[k] = make_float2(e[k].x + t.x, e[k].y + t.y);
            v[k + R / 2] = make_float2(e[k].x - t.x, e[k].y - t.y);
        }
    }
};
template <bool INV>
struct Dft<1, INV> {
    __device__ __forceinline__ static void run(float2*) {}
};

// One Stockham stage of radix R over an N-point sequence in shared memory, in place: every participating thread
// reads its butterflies' inputs into registers, the CTA synchronises, then every thread writes its outputs.
// `t` in [0, N/16) is the thread's index within this FFT; each thread owns N/(16 R) ... (16/R) butterflies so that it
// always holds 16 points.
template <int N, int R, bool INV>
__device__ __forceinline__ void stockham_stage(float2* buf, const float2* __restrict__ tw, int t, int Ns, bool active) {
    constexpr int B = 16 / R;  // butterflies per thread
    float2 v[B][R];
    if (active) {
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + b * (N / 16);
            const int k = j % Ns;
#pragma unroll
            for (int r = 0; r < R; r++) v[b][r] = buf[fpad(j + r * (N / R))];
            if (Ns > 1) {
                const int step = N / (Ns * R);
#pragma unroll
                for (int r = 1; r < R; r++) {
                    float2 wv = tw[(r * k * step) & (N - 1)];
                    if (INV) wv.y = -wv.y;
                    v[b][r] = cmul(v[b][r], wv);
                }
            }
            Dft<R, INV>::run(v[b]);
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int b = 0; b < B; b++) {
            const int j = t + b * (N / 16);
            const int k = j % Ns;
            const int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) buf[fpad(base + r * Ns)] = v[b][r];
        }
    }
    __syncthreads();
}

template <int N>
struct Log2 {
    static constexpr int value = 1 + Log2<N / 2>::value;
};
template <>
struct Log2<1> {
    static constexpr int value = 0;
};

// A full N-point FFT in shared memory by N/16 threads (`t` their index; `active` false for spare threads, which still
// take every barrier).
template <int N, bool INV>
__device__ __forceinline__ void fft_smem(float2* buf, const float2* __restrict__ tw, int t, bool active) {
    constexpr int L = Log2<N>::value;
    constexpr int full = L / 4, rest = L % 4;
    int Ns = 1;
#pragma unroll
    for (int s = 0; s < full; s++) {
        stockham_stage<N, 16, INV>(buf, tw, t, Ns, active);
        Ns *= 16;
    }
    if (rest == 1) stockham_stage<N, 2, INV>(buf, tw, t, Ns, active);
    if (rest == 2) stockham_stage<N, 4, INV>(buf, tw, t, Ns, active);
    if (rest == 3) stockham_stage<N, 8, INV>(buf, tw, t, Ns, active);
}

template <int N>
constexpr int fft_threads() {
    return N / 16 < 32 ? 32 : N / 16;
}

// ---- pass 1: two real rows per complex FFT, two FFTs per CTA (four rows)
template <int N>
__global__ void __launch_bounds__(2 * fft_threads<N>()) grav_rows_kernel(GravArgs A) {
    extern __shared__ float2 sm[];
    constexpr int T = fft_threads<N>();
    const int f = threadIdx.x / T, t = threadIdx.x % T;
    float2* buf = sm + f * fft_len<N>();
    const int ya = blockIdx.x * 4 + 2 * f, yb = ya + 1;
    const int w = A.w, h = A.h;
    const float sv = A.sigma_vac;
    for (int x = t; x < N; x += T) {
        float a = 0.0f, b = 0.0f;
        if (x < w) {
            if (ya < h) {
                float s = A.src[(size_t)ya * w + x];
                a = s >= sv ? s : 0.0f;
            }
            if (yb < h) {
                float s = A.src[(size_t)yb * w + x];
                b = s >= sv ? s : 0.0f;
            }
        }
        buf[fpad(x)] = make_float2(a, b);
    }
    __syncthreads();
    fft_smem<N, false>(buf, A.tw_x, t, t < N / 16);
    // unpack: X_a[k] = (Z[k] + conj Z[N-k]) / 2, X_b[k] = (Z[k] - conj Z[N-k]) / 2i, k = 0..N/2; column-major out
    const size_t ld = A.ld;
    for (int k = t; k <= N / 2; k += T) {
        float2 z = buf[fpad(k)], zc = buf[fpad((N - k) & (N - 1))];
        float2 xa = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
        float2 xb = make_float2(0.5f * (z.y + zc.y), 0.5f * (zc.x - z.x));
        if (ya < h) A.spec[(size_t)k * ld + 1 + ya] = xa;
        if (yb < h) A.spec[(size_t)k * ld + 1 + yb] = xb;
    }
}

// ---- pass 2: one spectrum column per CTA: forward, × K̂, inverse, rows -1..h kept
template <int N>
__global__ void __launch_bounds__(fft_threads<N>()) grav_columns_kernel(GravArgs A) {
    extern __shared__ float2 sm[];
    constexpr int T = fft_threads<N>();
    const int t = threadIdx.x;
    const int kx = blockIdx.x;
    const int h = A.h;
    const size_t ld = A.ld;
    float2* col = A.spec + (size_t)kx * ld;
    for (int y = t; y < N; y += T) sm[fpad(y)] = y < h ? col[1 + y] : make_float2(0.0f, 0.0f);
    __syncthreads();
    fft_smem<N, false>(sm, A.tw_y, t, t < N / 16);
    const float* kq = A.khat + (size_t)kx * (N / 2 + 1);
    for (int ky = t; ky < N; ky += T) {
        float k = kq[ky <= N / 2 ? ky : N - ky];
        float2 z = sm[fpad(ky)];
        sm[fpad(ky)] = make_float2(z.x * k, z.y * k);
    }
    __syncthreads();
    fft_smem<N, true>(sm, A.tw_y, t, t < N / 16);
    for (int r = t; r < h + 2; r += T) col[r] = sm[fpad((r - 1 + N) & (N - 1))];
}

// ---- pass 3: two output rows per complex inverse FFT, two FFTs per CTA; columns -1..w kept into φ_ring
template <int N>
__global__ void __launch_bounds__(2 * fft_threads<N>()) grav_rows_inverse_kernel(GravArgs A) {
    extern __shared__ float2 sm[];
    constexpr int T = fft_threads<N>();
    const int f = threadIdx.x / T, t = threadIdx.x % T;
    float2* buf = sm + f * fft_len<N>();
    const int rows = A.h + 2;
    const int ra = blockIdx.x * 4 + 2 * f, rb = ra + 1;
    const size_t ld = A.ld;
    for (int k = t; k <= N / 2; k += T) {
        float2 xa = ra < rows ? A.spec[(size_t)k * ld + ra] : make_float2(0.0f, 0.0f);
        float2 xb = rb < rows ? A.spec[(size_t)k * ld + rb] : make_float2(0.0f, 0.0f);
        // Z[k] = X_a[k] + i X_b[k]; Z[N-k] = conj X_a[k] + i conj X_b[k]
        buf[fpad(k)] = make_float2(xa.x - xb.y, xa.y + xb.x);
        if (k > 0 && k < N / 2) buf[fpad(N - k)] = make_float2(xa.x + xb.y, xb.x - xa.y);
    }
    __syncthreads();
    fft_smem<N, true>(buf, A.tw_x, t, t < N / 16);
    const int w = A.w, rw = w + 2;
    for (int c = t; c < rw; c += T) {
        float2 z = buf[fpad((c - 1 + N) & (N - 1))];
        if (ra < rows) A.phi_ring[(size_t)ra * rw + c] = z.x;
        if (rb < rows) A.phi_ring[(size_t)rb * rw + c] = z.y;
    }
}

// ---- pass 4: φ and g = -∇φ by central differences over the ringed potential (grav.rs:55-70)
__global__ void grav_gradient_kernel(GravArgs A) {
    const int w = A.w, h = A.h, rw = w + 2;
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int x, y;
        split_index(i, w, x, y);
        const float* r0 = A.phi_ring + (size_t)y * rw;
        const float* r1 = r0 + rw;
        const float* r2 = r1 + rw;
        A.gx[i] = -(r1[x + 2] - r1[x]) / 2.0f;
        A.gy[i] = -(r2[x + 1] - r0[x + 1]) / 2.0f;
        A.phi[i] = r1[x + 1];
    }
}

template <int N>
void launch_rows(const GravArgs& A, cudaStream_t s) {
    size_t smem = 2 * fft_len<N>() * sizeof(float2);
    cudaFuncSetAttribute(grav_rows_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    grav_rows_kernel<N><<<div_up(A.h, 4), 2 * fft_threads<N>(), smem, s>>>(A);
    sr_note_launch();
}

template <int N>
void launch_columns(const GravArgs& A, cudaStream_t s) {
    size_t smem = fft_len<N>() * sizeof(float2);
    cudaFuncSetAttribute(grav_columns_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    grav_columns_kernel<N><<<A.px / 2 + 1, fft_threads<N>(), smem, s>>>(A);
    sr_note_launch();
}

template <int N>
void launch_rows_inverse(const GravArgs& A, cudaStream_t s) {
    size_t smem = 2 * fft_len<N>() * sizeof(float2);
    cudaFuncSetAttribute(grav_rows_inverse_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    grav_rows_inverse_kernel<N><<<div_up(A.h + 2, 4), 2 * fft_threads<N>(), smem, s>>>(A);
    sr_note_launch();
}

#define SR_FFT_SIZES(X) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096) X(8192)

void dispatch_rows(int n, const GravArgs& A, cudaStream_t s) {
    switch (n) {
#define X(N) case N: launch_rows<N>(A, s); break;
        SR_FFT_SIZES(X)
#undef X
    }
}
void dispatch_columns(int n, const GravArgs& A, cudaStream_t s) {
    switch (n) {
#define X(N) case N: launch_columns<N>(A, s); break;
        SR_FFT_SIZES(X)
#undef X
    }
}
void dispatch_rows_inverse(int n, const GravArgs& A, cudaStream_t s) {
    switch (n) {
#define X(N) case N: launch_rows_inverse<N>(A, s); break;
        SR_FFT_SIZES(X)
#undef X
    }
}

// ------------------------------------------------------------------------------------------------ host: K̂ in f64
// A radix-2 complex FFT in f64 (forward, unnormalised), for the kernel's spectrum built once per padded size.
void fft_f64(std::vector<double>& re, std::vector<double>& im, size_t off, size_t stride, int n,
             const std::vector<double>& c, const std::vector<double>& s) {
    int bits = 0;
    while ((1 << bits) < n) bits++;
    for (int i = 0; i < n; i++) {
        int j = 0;
        for (int b = 0; b < bits; b++)
            if (i & (1 << b)) j |= 1 << (bits - 1 - b);
        if (i < j) {
            std::swap(re[off + i * stride], re[off + j * stride]);
            std::swap(im[off + i * stride], im[off + j * stride]);
        }
    }
    for (int half = 1; half < n; half *= 2) {
        int step = n / (2 * half);
        for (int start = 0; start < n; start += 2 * half)
            for (int k = 0; k < half; k++) {
                double wr = c[k * step], wi = s[k * step];
                size_t a = off + (start + k) * stride, b = off + (start + k + half) * stride;
                double br = re[b] * wr - im[b] * wi, bi = re[b] * wi + im[b] * wr;
                double ar = re[a], ai = im[a];
                re[a] = ar + br; im[a] = ai + bi;
                re[b] = ar - br; im[b] = ai - bi;
            }
    }
}

void parallel_for(int n, const std::function<void(int, int)>& body) {
    int nt = (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if (nt > 32) nt = 32;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++) {
        int a = (int)((long long)n * t / nt), b = (int)((long long)n * (t + 1) / nt);
        th.emplace_back([=, &body] { body(a, b); });
    }
    for (auto& x : th) x.join();
}

// K(dx, dy): the reference's exact self cell (grav.rs:25-34) or the softened kernel.
double kernel_value(int kind, double G, double eps, long dx, long dy) {
    double r2 = (double)(dx * dx + dy * dy);
    if (kind == SR_KERNEL_SOFTENED) return -G / sqrt(r2 + eps * eps);
    if (dx == 0 && dy == 0) return -G * 3.525494348078172;
    return -G / sqrt(r2);
}

std::mutex g_khat_mutex;
std::map<std::tuple<int, int, int, double, double>, std::vector<float>> g_khat_cache;

// The quarter (px/2+1) x (py/2+1) of K's real-even spectrum, in f64, scaled by 1/(px py) and stored f32
// (crates/sr-engine/src/step/grav.rs:76-130 builds the same quarter).
const std::vector<float>& khat_quarter(int px, int py, int kind, double G, double eps) {
    std::lock_guard<std::mutex> lock(g_khat_mutex);
    auto key = std::make_tuple(px, py, kind, G, eps);
    auto it = g_khat_cache.find(key);
    if (it != g_khat_cache.end()) return it->second;
    std::vector<double> re((size_t)px * py), im((size_t)px * py, 0.0);
    for (int j = 0; j < py; j++)
        for (int i = 0; i < px; i++) {
            long dx = i < px / 2 ? i : i - px, dy = j < py / 2 ? j : j - py;
            re[(size_t)j * px + i] = kernel_value(kind, G, eps, dx, dy);
        }
    auto twiddles = [](int n, std::vector<double>& c, std::vector<double>& s) {
        c.resize(n / 2 > 0 ? n / 2 : 1);
        s.resize(n / 2 > 0 ? n / 2 : 1);
        for (int k = 0; k < n / 2; k++) {
            double a = -2.0 * M_PI * (double)k / (double)n;
            c[k] = cos(a);
            s[k] = sin(a);
        }
    };
    std::vector<double> cx, sx, cy, sy;
    twiddles(px, cx, sx);
    twiddles(py, cy, sy);
    parallel_for(py, [&](int a, int b) {
        for (int j = a; j < b; j++) fft_f64(re, im, (size_t)j * px, 1, px, cx, sx);
    });
    parallel_for(px / 2 + 1, [&](int a, int b) {
        for (int i = a; i < b; i++) fft_f64(re, im, (size_t)i, (size_t)px, py, cy, sy);
    });
    std::vector<float> q((size_t)(px / 2 + 1) * (py / 2 + 1));
    const double scale = 1.0 / ((double)px * (double)py);
    for (int i = 0; i <= px / 2; i++)
        for (int j = 0; j <= py / 2; j++) q[(size_t)i * (py / 2 + 1) + j] = (float)(re[(size_t)j * px + i] * scale);
    return g_khat_cache.emplace(key, std::move(q)).first->second;
}

std::vector<float2> twiddle_table(int n) {
    std::vector<float2> t(n);
    for (int k = 0; k < n; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        t[k] = make_float2((float)cos(a), (float)sin(a));
    }
    return t;
}

}  // namespace

int grav_padded_size(int len) {
    // reference/fft.rs:92-101 with the cap lifted to 8192
    if (len <= 0) return 0;
    int n = 1;
    while (n < 2 * len) n <<= 1;
    if (n < 32) n = 32;
    return n > 8192 ? 0 : n;
}

void GravPlan::create(int w_, int h_, int kernel, double G, double eps, float sigma_vac_) {
    w = w_;
    h = h_;
    px = grav_padded_size(w);
    py = grav_padded_size(h);
    SR_REQUIRE(px && py, "a world axis pads past the FFT's 8192 points");
    sigma_vac = sigma_vac_;
    ld = (size_t)h + 2;
    SR_CUDA_TRY(cudaMalloc(&spec, sizeof(float2) * (size_t)(px / 2 + 1) * ld));
    SR_CUDA_TRY(cudaMalloc(&phi_ring, sizeof(float) * (size_t)(w + 2) * (h + 2)));
    const std::vector<float>& q = khat_quarter(px, py, kernel, G, eps);
    SR_CUDA_TRY(cudaMalloc(&khat, sizeof(float) * q.size()));
    SR_CUDA_TRY(cudaMemcpy(khat, q.data(), sizeof(float) * q.size(), cudaMemcpyHostToDevice));
    std::vector<float2> tx = twiddle_table(px), ty = twiddle_table(py);
    SR_CUDA_TRY(cudaMalloc(&tw_x, sizeof(float2) * px));
    SR_CUDA_TRY(cudaMalloc(&tw_y, sizeof(float2) * py));
    SR_CUDA_TRY(cudaMemcpy(tw_x, tx.data(), sizeof(float2) * px, cudaMemcpyHostToDevice));
    SR_CUDA_TRY(cudaMemcpy(tw_y, ty.data(), sizeof(float2) * py, cudaMemcpyHostToDevice));
}

void GravPlan::destroy() {
    cudaFree(spec);
    cudaFree(phi_ring);
    cudaFree(khat);
    cudaFree(tw_x);
    cudaFree(tw_y);
    spec = nullptr;
    phi_ring = nullptr;
    khat = nullptr;
    tw_x = tw_y = nullptr;
}

size_t GravPlan::bytes() const {
    return sizeof(float2) * (size_t)(px / 2 + 1) * ld + sizeof(float) * (size_t)(w + 2) * (h + 2) +
           sizeof(float) * (size_t)(px / 2 + 1) * (py / 2 + 1) + sizeof(float2) * (px + py);
}

void GravPlan::solve(const float* src, float* phi, float* gx, float* gy, cudaStream_t s) const {
    GravArgs A;
    A.w = w;
    A.h = h;
    A.px = px;
    A.py = py;
    A.ld = ld;
    A.sigma_vac = sigma_vac;
    A.src = src;
    A.spec = spec;
    A.khat = khat;
    A.tw_x = tw_x;
    A.tw_y = tw_y;
    A.phi_ring = phi_ring;
    A.phi = phi;
    A.gx = gx;
    A.gy = gy;
    dispatch_rows(px, A, s);
    dispatch_columns(py, A, s);
    dispatch_rows_inverse(px, A, s);
    size_t n = (size_t)w * h;
    int nb = (int)div_up((unsigned)((n + 3) / 4), 256u);
    nb = nb < 1 ? 1 : (nb > 148 * 8 ? 148 * 8 : nb);
    grav_gradient_kernel<<<nb, 256, 0, s>>>(A);
    sr_note_launch();
}
