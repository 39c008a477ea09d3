// learned.cu — the learned preconditioner (see learned.cuh): network, tcgen05 convolutions, training and inference.
//
// Tensors are FP32 NHWC with channels padded to a multiple of 8, images stacked along N. A 3x3 convolution is an
// implicit GEMM: M = 128 output pixels per CTA (a 16 x 8 tile, one TMEM lane each), N = the output channels, K = 9 taps
// x the input channels; the CTA stages its input halo once in shared memory as BF16 (applying the layer's input
// transform: pooling, upsampling, the skip addition, or for the data gradient the ReLU mask), builds its im2col rows
// from it in the canonical no-swizzle K-major layout, thread 0 issues tcgen05.mma (kind::f16, FP32 accumulator in
// TMEM) per 16 of K, commits to an mbarrier, and the four warps read their 32 TMEM lanes back for the epilogue (bias,
// ReLU, FP32 store). Every mbarrier wait is
// bounded; a wait that gives up sets the learner's error flag and the CTA skips its store.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "learned.cuh"
#include "reduce.cuh"
#include "tc.cuh"

namespace {

constexpr int NL = 15;
enum Mode { M_IN = 0, M_PREV = 1, M_POOL = 2, M_UP = 3, M_SKIP = 4 };
struct LayerDef {
    int cin, cout, mode, relu, skip, level;
};
// The network of oracle/unet.py: encoder 4-8-8 | 16-16 | 32-32 | 64-64, decoder with skip additions, 8 -> 1 head.
constexpr LayerDef kL[NL] = {{4, 8, M_IN, 1, -1, 0},    {8, 8, M_PREV, 1, -1, 0},   {8, 16, M_POOL, 1, -1, 1},
                             {16, 16, M_PREV, 1, -1, 1}, {16, 32, M_POOL, 1, -1, 2}, {32, 32, M_PREV, 1, -1, 2},
                             {32, 64, M_POOL, 1, -1, 3}, {64, 64, M_PREV, 1, -1, 3}, {64, 32, M_UP, 1, -1, 2},
                             {32, 32, M_SKIP, 1, 5, 2},  {32, 16, M_UP, 1, -1, 1},   {16, 16, M_SKIP, 1, 3, 1},
                             {16, 8, M_UP, 1, -1, 0},    {8, 8, M_SKIP, 1, 1, 0},    {8, 1, M_PREV, 0, -1, 0}};
constexpr int pad8(int c) { return c < 8 ? 8 : c; }
constexpr uint32_t kWaitLimit = 1u << 24;
constexpr int RT = 256;  // threads of the elementwise kernels

int kt_of(int cin_p) { return cin_p == 8 ? 80 : 9 * cin_p; }  // K of a weight image (a multiple of 16)

struct ConvArgs {
    int B, H, W;   // output dims per image
    int sH, sW;    // source dims (pooling: the finer level's, upsampling: the coarser level's)
    int mode;      // 0 same level, 1 pooled, 2 upsampled
    const float* src;
    const float* add;   // optional, added to the source (same level)
    const float* mask;  // optional, the source taken where mask > 0 (the ReLU of the forward output)
    const __nv_bfloat16* wimg;
    const float* bias;  // optional
    int cout_real;
    float* out;
    int relu;
    int* err;
};

__device__ __forceinline__ void load8(const float* p, float* v) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    const float4 b = *reinterpret_cast<const float4*>(p + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

// The convolution's input at (img, yy, xx), channels c0..c0+7, through the layer's input transform.
template <int CS>
__device__ __forceinline__ void conv_input(const ConvArgs& A, int img, int yy, int xx, int c0, float* v) {
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = 0.0f;
    if (yy < 0 || yy >= A.H || xx < 0 || xx >= A.W) return;
    if (A.mode == 0) {
        const size_t idx = (((size_t)img * A.H + yy) * A.W + xx) * CS + c0;
        load8(A.src + idx, v);
        if (A.add) {
            float w[8];
            load8(A.add + idx, w);
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] += w[q];
        }
        if (A.mask) {
            float m[8];
            load8(A.mask + idx, m);
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] = m[q] > 0.0f ? v[q] : 0.0f;
        }
    } else if (A.mode == 1) {
        int cnt = 0;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                const int fy = 2 * yy + b, fx = 2 * xx + a;
                if (fy >= A.sH || fx >= A.sW) continue;
                float w[8];
                load8(A.src + (((size_t)img * A.sH + fy) * A.sW + fx) * CS + c0, w);
#pragma unroll
                for (int q = 0; q < 8; q++) v[q] += w[q];
                cnt++;
            }
        const float inv = 1.0f / (float)cnt;
#pragma unroll
        for (int q = 0; q < 8; q++) v[q] *= inv;
    } else {
        load8(A.src + (((size_t)img * A.sH + (yy >> 1)) * A.sW + (xx >> 1)) * CS + c0, v);
    }
}

// A CTA's output tile: 16 x 8 pixels of one image (thread t <-> pixel (t % 16, t / 16) <-> TMEM lane t), and its input
// halo, 18 x 10 pixels, staged once in shared memory as BF16 (through the layer's input transform), from which each
// thread builds its im2col row with 16-byte shared-memory copies (8 channels = one core-matrix row).
constexpr int TW = 16, TH = 8, HW_ = TW + 2, HH_ = TH + 2, HP = HW_ * HH_;

template <int CIN_P, int COUT_P>
struct ConvShape {
    static constexpr int NC = CIN_P >= 32 ? 3 : 1;           // K chunks (3 taps each, or all 9 taps)
    static constexpr int KT = CIN_P == 8 ? 80 : 9 * CIN_P;   // K of the weight image (8 channels: 72 padded to 80)
    static constexpr int KC = NC == 1 ? KT : 3 * CIN_P;      // K of a chunk
    static constexpr int TAPS = NC == 1 ? 9 : 3;
    static constexpr int NBUF = (NC == 1 || CIN_P == 64) ? 1 : 2;  // one A buffer for 64 channels: 2 CTAs per SM
    static constexpr int NM = COUT_P < 16 ? 16 : COUT_P;     // MMA N (M = 128 takes N in multiples of 16)
    static constexpr int NCOLS = NM <= 32 ? 32 : 64;         // TMEM columns (a power of two >= 32)
    static constexpr size_t SBG = (size_t)COUT_P * KT * 2;   // the weight image in global memory
    static constexpr size_t SB = (size_t)NM * KT * 2;        // in shared memory, zero rows up to NM
    static constexpr size_t SA = (size_t)128 * KC * 2;
    static constexpr size_t SI = (size_t)HP * CIN_P * 2;     // the BF16 halo tile
    static constexpr size_t SMEM = SB + NBUF * SA + SI + 64;
};

template <int CIN_P, int COUT_P>
__global__ void __launch_bounds__(128) conv_tc_kernel(ConvArgs A) {
    using S = ConvShape<CIN_P, COUT_P>;
    constexpr int G = CIN_P / 8;  // channel groups of 16 bytes (BF16)
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sB = reinterpret_cast<__nv_bfloat16*>(smem);
    unsigned char* sA = smem + S::SB;
    uint4* sIn = reinterpret_cast<uint4*>(sA + S::NBUF * S::SA);  // [HP][G]
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sA + S::NBUF * S::SA + S::SI);
    uint32_t* tbase = reinterpret_cast<uint32_t*>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, S::NM);

    if (warp == 0) {
        tc::tmem_alloc(tbase, S::NCOLS);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&mbar[0], 1);
        tc::mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        const int4* g = reinterpret_cast<const int4*>(A.wimg);
        int4* d = reinterpret_cast<int4*>(sB);
        for (int i = tid; i < (int)(S::SB / 16); i += 128) d[i] = i < (int)(S::SBG / 16) ? g[i] : make_int4(0, 0, 0, 0);
    }
    const int img = blockIdx.z, X0 = blockIdx.x * TW, Y0 = blockIdx.y * TH;
    // the halo tile, through the input transform (zero outside the image), as BF16; a thread's items in batches of
    // four, all of a batch's loads issued before any conversion
    constexpr int NI = (HP * G + 127) / 128, NB = 4;
#pragma unroll
    for (int i0 = 0; i0 < NI; i0 += NB) {
        float v[NB][8];
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int e = tid + (i0 + u) * 128;
            if (i0 + u < NI && e < HP * G) {
                const int hp = e / G, g = e - hp * G;
                const int hy = hp / HW_, hx = hp - hy * HW_;
                conv_input<CIN_P>(A, img, Y0 + hy - 1, X0 + hx - 1, g * 8, v[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int e = tid + (i0 + u) * 128;
            if (i0 + u < NI && e < HP * G) {
                uint4 packed;
                __nv_bfloat162 h0 = __floats2bfloat162_rn(v[u][0], v[u][1]), h1 = __floats2bfloat162_rn(v[u][2], v[u][3]);
                __nv_bfloat162 h2 = __floats2bfloat162_rn(v[u][4], v[u][5]), h3 = __floats2bfloat162_rn(v[u][6], v[u][7]);
                packed.x = *reinterpret_cast<uint32_t*>(&h0);
                packed.y = *reinterpret_cast<uint32_t*>(&h1);
                packed.z = *reinterpret_cast<uint32_t*>(&h2);
                packed.w = *reinterpret_cast<uint32_t*>(&h3);
                sIn[e] = packed;
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tbase;

    const int px = tid % TW, py = tid / TW;
    const int x = X0 + px, y = Y0 + py;
    const bool valid = x < A.W && y < A.H;
    uint32_t par0 = 0u, par1 = 0u;
    bool ok = true;
    for (int c = 0; c < S::NC; c++) {
        const int buf = c % S::NBUF;
        if (c >= S::NBUF) {  // this buffer's previous MMAs must be done before it is rewritten
            const uint32_t par = buf ? par1 : par0;
            if (!tc::mbar_wait(&mbar[buf], par, kWaitLimit)) ok = false;
            if (buf) par1 ^= 1u; else par0 ^= 1u;
        }
        unsigned char* a = sA + buf * S::SA;
#pragma unroll
        for (int t = 0; t < S::TAPS; t++) {
            const int tap = S::NC == 1 ? t : c * 3 + t;
            const int hp = (py + tap / 3) * HW_ + px + tap % 3;  // the halo pixel of (x + dx, y + dy)
#pragma unroll
            for (int g = 0; g < G; g++) {
                const int k = t * CIN_P + g * 8;
                *reinterpret_cast<uint4*>(a + ((tid / 8) * (S::KC / 8) + k / 8) * 128 + (tid % 8) * 16) =
                    sIn[hp * G + g];
            }
        }
        if (CIN_P == 8)  // K 72..79: zero padding to a multiple of 16
            *reinterpret_cast<uint4*>(a + ((tid / 8) * (S::KC / 8) + 9) * 128 + (tid % 8) * 16) = make_uint4(0, 0, 0, 0);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_addr(a), b0 = tc::smem_addr(sB);
#pragma unroll
            for (int ks = 0; ks < S::KC / 16; ks++) {
                const uint64_t ad = tc::desc_kmajor(a0 + ks * 256, 128, S::KC * 16);
                const uint64_t bd = tc::desc_kmajor(b0 + (c * (S::KC / 8) + 2 * ks) * 128, 128, S::KT * 16);
                tc::mma_bf16(tmem, ad, bd, IDESC, c > 0 || ks > 0);
            }
            tc::mma_commit(&mbar[buf]);
        }
    }
    {
        const int buf = (S::NC - 1) % S::NBUF;
        if (!tc::mbar_wait(&mbar[buf], buf ? par1 : par0, kWaitLimit)) ok = false;
    }
    tc::fence_after_sync();
    float acc[COUT_P];
#pragma unroll
    for (int c0 = 0; c0 < COUT_P; c0 += 8) tc::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc + c0);
    tc::tmem_wait_ld();
    if (!ok) atomicExch(A.err, 1);
    if (valid && ok) {
        float* o = A.out + ((((size_t)img * A.H + y) * A.W) + x) * COUT_P;
#pragma unroll
        for (int c0 = 0; c0 < COUT_P; c0 += 4) {
            float4 q;
            float* qq = reinterpret_cast<float*>(&q);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int co = c0 + j;
                float v = acc[co] + ((A.bias && co < A.cout_real) ? A.bias[co] : 0.0f);
                if (A.relu) v = fmaxf(v, 0.0f);
                qq[j] = v;
            }
            *reinterpret_cast<float4*>(o + c0) = q;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, S::NCOLS);
}

template <int CI, int CO>
void conv_attr_t() {
    SR_CUDA_TRY(cudaFuncSetAttribute(conv_tc_kernel<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ConvShape<CI, CO>::SMEM));
}

// Shared-memory opt-in of every convolution, set once outside any launch (so that launches can be captured).
void conv_attributes() {
    conv_attr_t<8, 8>();
    conv_attr_t<8, 16>();
    conv_attr_t<16, 8>();
    conv_attr_t<16, 16>();
    conv_attr_t<16, 32>();
    conv_attr_t<32, 16>();
    conv_attr_t<32, 32>();
    conv_attr_t<32, 64>();
    conv_attr_t<64, 32>();
    conv_attr_t<64, 64>();
}

template <int CI, int CO>
void launch_conv_t(const ConvArgs& A, cudaStream_t s) {
    using S = ConvShape<CI, CO>;
    const dim3 grid((unsigned)((A.W + TW - 1) / TW), (unsigned)((A.H + TH - 1) / TH), (unsigned)A.B);
    conv_tc_kernel<CI, CO><<<grid, 128, S::SMEM, s>>>(A);
    sr_note_launch();
}

void launch_conv(int cin_p, int cout_p, const ConvArgs& A, cudaStream_t s) {
#define SR_CONV_CASE(CI, CO) \
    if (cin_p == CI && cout_p == CO) return launch_conv_t<CI, CO>(A, s);
    SR_CONV_CASE(8, 8) SR_CONV_CASE(8, 16) SR_CONV_CASE(16, 8) SR_CONV_CASE(16, 16) SR_CONV_CASE(16, 32)
    SR_CONV_CASE(32, 16) SR_CONV_CASE(32, 32) SR_CONV_CASE(32, 64) SR_CONV_CASE(64, 32) SR_CONV_CASE(64, 64)
#undef SR_CONV_CASE
    throw SrError{SR_E_INVALID, "no convolution for these channel counts"};
}

// ---- weight images: the forward B operand [cout_p/8][KT/8][8][8] with k = tap * cin_p + ci, and the data-gradient
// one, the convolution with the taps flipped and the channels swapped: n = ci, k = tap' * cout_p + co.
__global__ void pack_weights_kernel(const float* __restrict__ theta, int cin, int cout, int cin_p, int cout_p,
                                    __nv_bfloat16* fwd, __nv_bfloat16* bwd) {
    const int ktf = cin_p == 8 ? 80 : 9 * cin_p, ktb = cout_p == 8 ? 80 : 9 * cout_p;
    const int nf = cout_p * ktf, nb = cin_p * ktb;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nf + nb; e += gridDim.x * blockDim.x) {
        if (e < nf) {
            const int n = e / ktf, k = e % ktf;
            const int tap = k / cin_p, ci = k % cin_p;
            float v = 0.0f;
            if (n < cout && tap < 9 && ci < cin) v = theta[((size_t)n * 9 + tap) * cin + ci];
            fwd[((n / 8) * (ktf / 8) + k / 8) * 64 + (n % 8) * 8 + (k % 8)] = __float2bfloat16_rn(v);
        } else {
            const int f = e - nf;
            const int n = f / ktb, k = f % ktb;  // n: forward input channel, k: flipped tap x forward output channel
            const int tapf = k / cout_p, co = k % cout_p;
            float v = 0.0f;
            if (n < cin && tapf < 9 && co < cout) v = theta[((size_t)co * 9 + (8 - tapf)) * cin + n];
            bwd[((n / 8) * (ktb / 8) + k / 8) * 64 + (n % 8) * 8 + (k % 8)] = __float2bfloat16_rn(v);
        }
    }
}

// ---- weight gradient on the CUDA cores: dW[co][k] = Σ_p g[p][co] x[p][k], g the output gradient under the ReLU mask
// and x the convolution's input (through the input transform), per chunk of pixels; partials summed in chunk order.
constexpr int DW_PIX = 2048;  // pixels per CTA
constexpr int DW_SUB = 32;    // pixels staged at once
template <int CIN_P, int COUT_P>
__global__ void __launch_bounds__(256) dw_kernel(ConvArgs A, const float* __restrict__ gy, const float* __restrict__ y,
                                                 int relu, float* part) {
    constexpr int KT = 9 * CIN_P;
    __shared__ float sg[DW_SUB][COUT_P];
    __shared__ float sx[DW_SUB][64];
    const int tid = threadIdx.x;
    const int k0 = blockIdx.y * 64;
    const int kl = tid % 64, cg = tid / 64;  // this thread: k = k0 + kl, channels cg, cg + 4, ...
    constexpr int CPT = (COUT_P + 3) / 4;
    float acc[CPT];
#pragma unroll
    for (int j = 0; j < CPT; j++) acc[j] = 0.0f;
    const long long P = (long long)A.B * A.H * A.W;
    const long long p0 = (long long)blockIdx.x * DW_PIX;
    for (long long ps = p0; ps < p0 + DW_PIX && ps < P; ps += DW_SUB) {
        for (int e = tid; e < DW_SUB * COUT_P; e += 256) {
            const int q = e / COUT_P, co = e % COUT_P;
            const long long p = ps + q;
            float v = 0.0f;
            if (p < P) {
                v = gy[(size_t)p * COUT_P + co];
                if (relu && !(y[(size_t)p * COUT_P + co] > 0.0f)) v = 0.0f;
            }
            sg[q][co] = v;
        }
        for (int e = tid; e < DW_SUB * 8; e += 256) {  // 8 groups of 8 k per pixel
            const int q = e / 8, grp = e % 8;
            const long long p = ps + q;
            const int k = k0 + grp * 8;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) v[j] = 0.0f;
            if (p < P && k < KT) {
                const int tap = k / CIN_P, ci = k % CIN_P;
                const int img = (int)(p / ((long long)A.H * A.W));
                const int r = (int)(p - (long long)img * A.H * A.W);
                const int yy = r / A.W, xx = r - (r / A.W) * A.W;
                conv_input<CIN_P>(A, img, yy + tap / 3 - 1, xx + tap % 3 - 1, ci, v);
            }
#pragma unroll
            for (int j = 0; j < 8; j++) sx[q][grp * 8 + j] = v[j];
        }
        __syncthreads();
#pragma unroll 4
        for (int q = 0; q < DW_SUB; q++) {
            const float xv = sx[q][kl];
#pragma unroll
            for (int j = 0; j < CPT; j++) {
                const int co = cg + 4 * j;
                if (co < COUT_P) acc[j] += sg[q][co] * xv;
            }
        }
        __syncthreads();
    }
    const int k = k0 + kl;
    if (k < KT)
#pragma unroll
        for (int j = 0; j < CPT; j++) {
            const int co = cg + 4 * j;
            if (co < COUT_P) part[((size_t)blockIdx.x * COUT_P + co) * KT + k] = acc[j];
        }
}

// dW and db from the partials into the gradient vector (the parameter layout W[cout][3][3][cin], b[cout]).
__global__ void dw_reduce_kernel(const float* __restrict__ part, int chunks, int cin, int cout, int cin_p, int cout_p,
                                 float* gw, float* gb, const float* __restrict__ bpart) {
    const int kt = 9 * cin_p;
    const int n = cout * 9 * cin;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n + cout; e += gridDim.x * blockDim.x) {
        if (e < n) {
            const int co = e / (9 * cin), rem = e % (9 * cin), tap = rem / cin, ci = rem % cin;
            const int k = tap * cin_p + ci;
            double s = 0.0;
            for (int c = 0; c < chunks; c++) s += part[((size_t)c * cout_p + co) * kt + k];
            gw[e] = (float)s;
        } else {
            const int co = e - n;
            double s = 0.0;
            for (int c = 0; c < chunks; c++) s += bpart[(size_t)c * cout_p + co];
            gb[co] = (float)s;
        }
    }
}

// Bias gradient partials: Σ over a chunk of pixels of the masked output gradient.
template <int COUT_P>
__global__ void db_kernel(long long P, const float* __restrict__ gy, const float* __restrict__ y, int relu,
                          float* bpart) {
    __shared__ float red[COUT_P][8];
    const int co = threadIdx.x % COUT_P, lane = threadIdx.x / COUT_P;  // blockDim = COUT_P * 8
    const long long p0 = (long long)blockIdx.x * DW_PIX;
    float s = 0.0f;
    for (long long p = p0 + lane; p < p0 + DW_PIX && p < P; p += 8) {
        float v = gy[(size_t)p * COUT_P + co];
        if (relu && !(y[(size_t)p * COUT_P + co] > 0.0f)) v = 0.0f;
        s += v;
    }
    red[co][lane] = s;
    __syncthreads();
    if (lane == 0) {
        float t = 0.0f;
        for (int q = 0; q < 8; q++) t += red[co][q];
        bpart[(size_t)blockIdx.x * COUT_P + co] = t;
    }
}

// ---- input-transform adjoints and the elementwise pieces
__global__ void add_kernel(size_t n, const float* __restrict__ a, float* dst) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] += a[i];
}

// g_fine[fy][fx] += g_coarse[fy/2][fx/2] / (cells of that block)
__global__ void pool_adjoint_kernel(int B, int H, int W, int C, const float* __restrict__ gc, float* gf) {
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    const size_t n = (size_t)B * H * W * C;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(e % C);
        const size_t pix = e / C;
        const int x = (int)(pix % W), y = (int)((pix / W) % H), img = (int)(pix / ((size_t)W * H));
        const int Y = y >> 1, X = x >> 1;
        const int cnt = (2 * Y + 1 < H ? 2 : 1) * (2 * X + 1 < W ? 2 : 1);
        gf[e] += gc[(((size_t)img * Hc + Y) * Wc + X) * C + ch] / (float)cnt;
    }
}

// g_coarse[Y][X] += Σ over the fine cells of the block of g_fine
__global__ void up_adjoint_kernel(int B, int H, int W, int C, const float* __restrict__ gf, float* gc) {
    const int Hc = (H + 1) / 2, Wc = (W + 1) / 2;
    const size_t n = (size_t)B * Hc * Wc * C;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(e % C);
        const size_t pix = e / C;
        const int X = (int)(pix % Wc), Y = (int)((pix / Wc) % Hc), img = (int)(pix / ((size_t)Wc * Hc));
        float s = 0.0f;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                const int y = 2 * Y + b, x = 2 * X + a;
                if (y < H && x < W) s += gf[(((size_t)img * H + y) * W + x) * C + ch];
            }
        gc[e] += s;
    }
}

// The crop's Jacobi-scaled operator applied to v at pixel p of an H x W crop: unit diagonal, −d̂x / −d̂y (feature
// channels 1 and 2) to the +x / +y neighbour and symmetric, the couplings that leave the crop dropped.
template <class V>
__device__ __forceinline__ float crop_op(const float* __restrict__ feats, int H, int W, size_t p, V v) {
    const int x = (int)(p % W), y = (int)((p / W) % H);
    float a = v(p);
    if (x + 1 < W) a -= feats[p * 8 + 1] * v(p + 1);
    if (x > 0) a -= feats[(p - 1) * 8 + 1] * v(p - 1);
    if (y + 1 < H) a -= feats[p * 8 + 2] * v(p + W);
    if (y > 0) a -= feats[(p - W) * 8 + 2] * v(p - W);
    return a;
}

// E_b = t_bᵀ Â t_b, the energy of each crop's target (one CTA per crop).
__global__ void target_energy_kernel(int H, int W, const float* __restrict__ feats, const float* __restrict__ target,
                                     float* E) {
    const size_t per = (size_t)H * W, base = (size_t)blockIdx.x * per;
    double acc = 0.0;
    auto t = [&](size_t q) { return target[q]; };
    for (size_t q = threadIdx.x; q < per; q += blockDim.x)
        acc += (double)target[base + q] * crop_op(feats, H, W, base + q, t);
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double e = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) e += red[w];
        E[blockIdx.x] = (float)e;
    }
}

// The loss: the energy left after the correction as a fraction of the target's, averaged over the crops,
//   L = (1/B) Σ_b δ_bᵀ Â δ_b / (E_b + ε),  δ = t − y (y the head's channel 0),  ε = 10⁻³ · mean_b E_b,
// — what the error left by the V-cycle and the network costs conjugate gradients, each crop weighted alike. Its
// gradient ∂L/∂y = −2 Â δ_b / (B (E_b + ε)); the loss into *out. Crops with a non-finite energy get weight 0.
__global__ void energy_loss_kernel(int B, int H, int W, const float* __restrict__ y, const float* __restrict__ feats,
                                   const float* __restrict__ target, const float* __restrict__ E, float* gy,
                                   double* part, unsigned* counter, double* out) {
    __shared__ float s_eps;
    if (threadIdx.x == 0) {
        double m = 0.0;
        int k = 0;
        for (int b = 0; b < B; b++)
            if (isfinite(E[b])) {
                m += E[b];
                k++;
            }
        s_eps = k ? (float)(1e-3 * m / k) : 1.0f;
    }
    __syncthreads();
    const float eps = s_eps > 0.0f ? s_eps : 1e-30f;
    const size_t per = (size_t)H * W, P = (size_t)B * per;
    double acc = 0.0;
    auto delta = [&](size_t q) { return target[q] - y[q * 8]; };
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (size_t)gridDim.x * blockDim.x) {
        const float Eb = E[p / per];
        const float wgt = isfinite(Eb) ? 1.0f / ((float)B * (Eb + eps)) : 0.0f;
        float g = 0.0f;
        if (wgt > 0.0f) {
            const float ad = crop_op(feats, H, W, p, delta);
            acc += (double)wgt * delta(p) * ad;
            g = -2.0f * wgt * ad;
        }
        gy[p * 8] = g;
#pragma unroll
        for (int c = 1; c < 8; c++) gy[p * 8 + c] = 0.0f;
    }
    grid_sum_last1(acc, part, counter, out);
}

__global__ void adam_kernel(int n, float* theta, const float* __restrict__ g, float* m, float* v, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Samples (features NHWC 8-padded, targets) gathered into the batch tensors.
__global__ void gather_kernel(int C, const int* __restrict__ idx, int batch, const float* __restrict__ feats,
                              const float* __restrict__ targets, float* bf, float* bt) {
    const size_t per = (size_t)C * C;
    const size_t n = (size_t)batch * per;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(e / per);
        const size_t q = e % per;
        const size_t src = (size_t)idx[b] * per + q;
        reinterpret_cast<float4*>(bf)[e * 2] = reinterpret_cast<const float4*>(feats)[src * 2];
        reinterpret_cast<float4*>(bf)[e * 2 + 1] = reinterpret_cast<const float4*>(feats)[src * 2 + 1];
        bt[e] = targets[src];
    }
}

// Host features (n, 4, C, C) -> NHWC 8-padded.
__global__ void nchw_to_feats_kernel(int n, int C, const float* __restrict__ in, float* out) {
    const size_t per = (size_t)C * C;
    const size_t tot = (size_t)n * per;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const size_t b = e / per, q = e % per;
        for (int c = 0; c < 8; c++) out[e * 8 + c] = c < 4 ? in[(b * 4 + c) * per + q] : 0.0f;
    }
}

// ---- features of the operator at cell i of level 0: the diagonal, the scaled couplings and the mass share
struct CellOp {
    float d, dxs, dys, m;
};
__device__ __forceinline__ float diag_at(const MgLevel& L, int x, int y) {
    const size_t i = (size_t)y * L.w + x;
    float d = L.c[i] + L.dx[i] + L.dy[i];
    if (x > 0) d += L.dx[i - 1];
    if (y > 0) d += L.dy[i - L.w];
    return d;
}
__device__ __forceinline__ CellOp cell_op(const MgLevel& L, int x, int y) {
    const size_t i = (size_t)y * L.w + x;
    CellOp o;
    o.d = diag_at(L, x, y);
    o.dxs = (x + 1 < L.w) ? L.dx[i] * rsqrtf(o.d * diag_at(L, x + 1, y)) : 0.0f;
    o.dys = (y + 1 < L.h) ? L.dy[i] * rsqrtf(o.d * diag_at(L, x, y + 1)) : 0.0f;
    o.m = L.c[i] / o.d;
    return o;
}

// Σ r̂² (r̂ = r/sqrt(d)) and the gas cells over the world: the rms scale s of the features, in training and inference.
__global__ void apply_scale_kernel(MgLevel L, const float* __restrict__ r, double* part, unsigned* counter,
                                   double* out) {
    double s = 0.0, n = 0.0;
    const size_t N = (size_t)L.w * L.h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        if (!L.mask[i]) continue;
        const int x = (int)(i % L.w), y = (int)(i / L.w);
        const float rh = r[i] * rsqrtf(diag_at(L, x, y));
        s += (double)rh * rh;
        n += 1.0;
    }
    const double v[2] = {s, n};
    grid_sum_last<2>(v, part, counter, out);
}

// One CTA per crop: the crop's features (r̂/s, d̂x, d̂y, m) with s the world's rms of r̂ (gscale as apply_scale_kernel
// leaves it: the normalisation inference uses), and the stored t = sqrt(d) e / s (finished at the end of the solve).
__global__ void snapshot_kernel(MgLevel L, const float* __restrict__ r, const float* __restrict__ e, int C,
                                const int2* __restrict__ pos, int first_sample, const double* __restrict__ gscale,
                                float* feats, float* targets, float* scales) {
    const int j = blockIdx.x;
    const int sample = first_sample + j;
    const int2 o = pos[j];
    const double ss = gscale[1] > 0.0 ? sqrt(gscale[0] / gscale[1]) : 1.0;
    const float s = ss > 0.0 ? (float)ss : 1.0f;
    if (threadIdx.x == 0) scales[sample] = s;
    for (int q = threadIdx.x; q < C * C; q += blockDim.x) {
        const int x = o.x + q % C, y = o.y + q / C;
        const size_t i = (size_t)y * L.w + x;
        const CellOp op = cell_op(L, x, y);
        float* f = feats + ((size_t)sample * C * C + q) * 8;
        const float sq = sqrtf(op.d);
        f[0] = r[i] / sq / s;
        f[1] = op.dxs;
        f[2] = op.dys;
        f[3] = op.m;
        f[4] = f[5] = f[6] = f[7] = 0.0f;
        targets[(size_t)sample * C * C + q] = sq * e[i] / s;
    }
}

// target = sqrt(d) e_final / s - t for every sample of the system just solved.
__global__ void finish_targets_kernel(MgLevel L, const float* __restrict__ e, int C, const int2* __restrict__ pos,
                                      int crops, int first_sample, int count, float* targets,
                                      const float* __restrict__ scales) {
    const size_t per = (size_t)C * C;
    const size_t n = (size_t)count * per;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int sl = (int)(k / per);
        const int q = (int)(k % per);
        const int sample = first_sample + sl;
        const int2 o = pos[sl % crops];
        const int x = o.x + q % C, y = o.y + q / C;
        const float sq = sqrtf(diag_at(L, x, y));
        targets[(size_t)sample * per + q] = sq * e[(size_t)y * L.w + x] / scales[sample] - targets[(size_t)sample * per + q];
    }
}

__global__ void apply_features_kernel(MgLevel L, const float* __restrict__ r, const double* __restrict__ scale,
                                      float* feats) {
    const double ss = scale[1] > 0.0 ? sqrt(scale[0] / scale[1]) : 1.0;
    const float s = ss > 0.0 ? (float)ss : 1.0f;
    const size_t N = (size_t)L.w * L.h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % L.w), y = (int)(i / L.w);
        const CellOp op = cell_op(L, x, y);
        float4 a = make_float4(r[i] * rsqrtf(op.d) / s, op.dxs, op.dys, op.m);
        reinterpret_cast<float4*>(feats)[i * 2] = a;
        reinterpret_cast<float4*>(feats)[i * 2 + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// z = z_base + head · s / sqrt(d) on the gas cells (0 elsewhere), and <r_dot, z>.
__global__ void apply_output_kernel(MgLevel L, const float* __restrict__ r_dot, const float* zbase,
                                    const float* __restrict__ head, const double* __restrict__ scale, float* z,
                                    double* part, unsigned* counter, double* out) {
    const double ss = scale[1] > 0.0 ? sqrt(scale[0] / scale[1]) : 1.0;
    const float s = ss > 0.0 ? (float)ss : 1.0f;
    const size_t N = (size_t)L.w * L.h;
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        float zi = 0.0f;
        if (L.mask[i]) {
            const int x = (int)(i % L.w), y = (int)(i / L.w);
            zi = (zbase ? zbase[i] : 0.0f) + head[i * 8] * s * rsqrtf(diag_at(L, x, y));
        }
        z[i] = zi;
        acc += (double)r_dot[i] * zi;
    }
    grid_sum_last1(acc, part, counter, out);
}

int grid_of(size_t n) {
    size_t b = (n + RT - 1) / RT;
    return (int)std::max<size_t>(1, std::min<size_t>(b, 148 * 16));
}

// The network's activations and gradients for a batch of `B` images of H x W.
struct Net {
    int B = 0, H = 0, W = 0;
    int lh[4], lw[4];
    float* feats = nullptr;
    float* act[NL] = {};
    float* gact[NL] = {};
    float* gx = nullptr;      // a layer's input gradient, before its adjoint scatters it
    float* energy = nullptr;  // each crop's target energy
    float* wpart = nullptr;
    float* bpart = nullptr;
    bool train = false;

    size_t pix(int level) const { return (size_t)B * lh[level] * lw[level]; }

    void create(int B_, int H_, int W_, bool train_) {
        B = B_;
        H = H_;
        W = W_;
        train = train_;
        lh[0] = H;
        lw[0] = W;
        for (int l = 1; l < 4; l++) {
            lh[l] = (lh[l - 1] + 1) / 2;
            lw[l] = (lw[l - 1] + 1) / 2;
        }
        SR_CUDA_TRY(cudaMalloc(&feats, sizeof(float) * pix(0) * 8));
        size_t maxin = 0;
        for (int l = 0; l < NL; l++) {
            const size_t n = pix(kL[l].level) * pad8(kL[l].cout);
            SR_CUDA_TRY(cudaMalloc(&act[l], sizeof(float) * n));
            if (train) SR_CUDA_TRY(cudaMalloc(&gact[l], sizeof(float) * n));
            maxin = std::max(maxin, pix(kL[l].level) * (size_t)pad8(kL[l].cin));
        }
        if (train) {
            SR_CUDA_TRY(cudaMalloc(&gx, sizeof(float) * maxin));
            SR_CUDA_TRY(cudaMalloc(&energy, sizeof(float) * B));
            const size_t chunks = (pix(0) + DW_PIX - 1) / DW_PIX;
            SR_CUDA_TRY(cudaMalloc(&wpart, sizeof(float) * chunks * 64 * 9 * 64));
            SR_CUDA_TRY(cudaMalloc(&bpart, sizeof(float) * chunks * 64));
        }
    }
    void destroy() {
        cudaFree(feats);
        for (int l = 0; l < NL; l++) {
            cudaFree(act[l]);
            cudaFree(gact[l]);
        }
        cudaFree(gx);
        cudaFree(energy);
        cudaFree(wpart);
        cudaFree(bpart);
    }
};

}  // namespace

struct Learner {
    int crop = 0, capacity = 0, count = 0;
    int nparams = 0;
    int woff[NL], boff[NL];
    float* theta = nullptr;  // FP32 master weights
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    int adam_t = 0;
    __nv_bfloat16* wf[NL] = {};  // forward weight images
    __nv_bfloat16* wb[NL] = {};  // data-gradient weight images
    float* sfeats = nullptr;     // samples: capacity x crop² x 8
    float* stargets = nullptr;   // capacity x crop²
    float* sscales = nullptr;
    int2* pos = nullptr;         // crop positions of the system being collected
    int crops = 0, sys_first = 0;
    int* err = nullptr;
    double* red_part = nullptr;
    unsigned* red_counter = nullptr;
    double* scal = nullptr;      // [0] the loss, [2..3] the collection's scale sums
    Net train_net;
    int train_batch = 0;
    int* bidx = nullptr;
    float* btarget = nullptr;
    std::mt19937_64 rng;

    void pack(cudaStream_t s) {
        for (int l = 0; l < NL; l++) {
            pack_weights_kernel<<<64, RT, 0, s>>>(theta + woff[l], kL[l].cin, kL[l].cout, pad8(kL[l].cin),
                                                  pad8(kL[l].cout), wf[l], wb[l]);
            sr_note_launch();
        }
    }
};

struct LearnedApply {
    Learner* L = nullptr;
    Net net;
    double* scale = nullptr;  // [Σ r̂², gas cells]
};

namespace {

ConvArgs layer_args(const Learner* Lr, const Net& N, int l) {
    const LayerDef& d = kL[l];
    ConvArgs A{};
    A.B = N.B;
    A.H = N.lh[d.level];
    A.W = N.lw[d.level];
    A.sH = A.H;
    A.sW = A.W;
    A.mode = 0;
    A.src = l == 0 ? N.feats : N.act[l - 1];
    if (d.mode == M_POOL) {
        A.mode = 1;
        A.sH = N.lh[d.level - 1];
        A.sW = N.lw[d.level - 1];
    } else if (d.mode == M_UP) {
        A.mode = 2;
        A.sH = N.lh[d.level + 1];
        A.sW = N.lw[d.level + 1];
    } else if (d.mode == M_SKIP) {
        A.add = N.act[d.skip];
    }
    A.wimg = Lr->wf[l];
    A.bias = Lr->theta + Lr->boff[l];
    A.cout_real = d.cout;
    A.out = N.act[l];
    A.relu = d.relu;
    A.err = Lr->err;
    return A;
}

void forward(const Learner* Lr, const Net& N, cudaStream_t s) {
    for (int l = 0; l < NL; l++) launch_conv(pad8(kL[l].cin), pad8(kL[l].cout), layer_args(Lr, N, l), s);
}

template <int CI, int CO>
void launch_dw_t(const ConvArgs& A, const float* gy, const float* y, int relu, float* wpart, float* bpart,
                 cudaStream_t s) {
    const long long P = (long long)A.B * A.H * A.W;
    const int chunks = (int)((P + DW_PIX - 1) / DW_PIX);
    dim3 grid(chunks, (9 * CI + 63) / 64);
    dw_kernel<CI, CO><<<grid, 256, 0, s>>>(A, gy, y, relu, wpart);
    sr_note_launch();
    db_kernel<CO><<<chunks, CO * 8, 0, s>>>(P, gy, y, relu, bpart);
    sr_note_launch();
}

void launch_dw(int ci, int co, const ConvArgs& A, const float* gy, const float* y, int relu, float* wpart,
               float* bpart, cudaStream_t s) {
#define SR_DW_CASE(CI, CO) \
    if (ci == CI && co == CO) return launch_dw_t<CI, CO>(A, gy, y, relu, wpart, bpart, s);
    SR_DW_CASE(8, 8) SR_DW_CASE(8, 16) SR_DW_CASE(16, 16) SR_DW_CASE(16, 32) SR_DW_CASE(32, 32) SR_DW_CASE(32, 64)
    SR_DW_CASE(64, 64) SR_DW_CASE(64, 32) SR_DW_CASE(32, 16) SR_DW_CASE(16, 8)
#undef SR_DW_CASE
    throw SrError{SR_E_INVALID, "no weight gradient for these channel counts"};
}

// Loss gradient already in gact[NL-1]: every layer's weight gradient and the input gradients, last layer first.
void backward(Learner* Lr, Net& N, cudaStream_t s) {
    for (int l = 0; l < NL - 1; l++)
        SR_CUDA_TRY(cudaMemsetAsync(N.gact[l], 0, sizeof(float) * N.pix(kL[l].level) * pad8(kL[l].cout), s));
    for (int l = NL - 1; l >= 0; l--) {
        const LayerDef& d = kL[l];
        const int ci = pad8(d.cin), co = pad8(d.cout);
        ConvArgs A = layer_args(Lr, N, l);
        const long long P = (long long)A.B * A.H * A.W;
        const int chunks = (int)((P + DW_PIX - 1) / DW_PIX);
        launch_dw(ci, co, A, N.gact[l], N.act[l], d.relu, N.wpart, N.bpart, s);
        dw_reduce_kernel<<<grid_of((size_t)d.cout * 9 * d.cin + d.cout), RT, 0, s>>>(
            N.wpart, chunks, d.cin, d.cout, ci, co, Lr->grad + Lr->woff[l], Lr->grad + Lr->boff[l], N.bpart);
        sr_note_launch();
        if (l == 0) break;
        // the gradient of the convolution's input, at this layer's level
        ConvArgs G{};
        G.B = A.B;
        G.H = A.H;
        G.W = A.W;
        G.sH = A.H;
        G.sW = A.W;
        G.mode = 0;
        G.src = N.gact[l];
        G.mask = d.relu ? N.act[l] : nullptr;
        G.wimg = Lr->wb[l];
        G.bias = nullptr;
        G.cout_real = ci;
        G.out = N.gx;
        G.relu = 0;
        G.err = Lr->err;
        launch_conv(co, ci, G, s);
        const size_t nin = (size_t)P * ci;
        if (d.mode == M_PREV || d.mode == M_SKIP) {
            add_kernel<<<grid_of(nin), RT, 0, s>>>(nin, N.gx, N.gact[l - 1]);
            sr_note_launch();
            if (d.mode == M_SKIP) {
                add_kernel<<<grid_of(nin), RT, 0, s>>>(nin, N.gx, N.gact[d.skip]);
                sr_note_launch();
            }
        } else if (d.mode == M_POOL) {
            const int lv = d.level - 1;
            const size_t nf = N.pix(lv) * ci;
            pool_adjoint_kernel<<<grid_of(nf), RT, 0, s>>>(N.B, N.lh[lv], N.lw[lv], ci, N.gx, N.gact[l - 1]);
            sr_note_launch();
        } else if (d.mode == M_UP) {
            const int lv = d.level;
            const size_t nc = N.pix(lv + 1) * ci;
            up_adjoint_kernel<<<grid_of(nc), RT, 0, s>>>(N.B, N.lh[lv], N.lw[lv], ci, N.gx, N.gact[l - 1]);
            sr_note_launch();
        }
    }
}

}  // namespace

int learned_param_count() {
    int n = 0;
    for (int l = 0; l < NL; l++) n += kL[l].cout * 9 * kL[l].cin + kL[l].cout;
    return n;
}

Learner* learned_create(int crop, int capacity, uint64_t seed) {
    SR_REQUIRE(crop >= 16 && crop % 8 == 0 && crop <= 512, "training crops must be a multiple of 8 in 16..512");
    SR_REQUIRE(capacity >= 1, "a learner needs room for samples");
    Learner* L = new Learner();
    try {
        conv_attributes();
        L->crop = crop;
        L->capacity = capacity;
        L->rng.seed(seed);
        int k = 0;
        for (int l = 0; l < NL; l++) {
            L->woff[l] = k;
            k += kL[l].cout * 9 * kL[l].cin;
            L->boff[l] = k;
            k += kL[l].cout;
        }
        L->nparams = k;
        SR_CUDA_TRY(cudaMalloc(&L->theta, sizeof(float) * k));
        SR_CUDA_TRY(cudaMalloc(&L->grad, sizeof(float) * k));
        SR_CUDA_TRY(cudaMalloc(&L->m, sizeof(float) * k));
        SR_CUDA_TRY(cudaMalloc(&L->v, sizeof(float) * k));
        SR_CUDA_TRY(cudaMemset(L->m, 0, sizeof(float) * k));
        SR_CUDA_TRY(cudaMemset(L->v, 0, sizeof(float) * k));
        // He initialisation (std sqrt(2 / fan_in)), zero biases, and a zero head: the untrained network adds nothing
        std::vector<float> th(k, 0.0f);
        std::normal_distribution<float> nd(0.0f, 1.0f);
        for (int l = 0; l < NL - 1; l++) {
            const float std = sqrtf(2.0f / (9.0f * kL[l].cin));
            for (int i = 0; i < kL[l].cout * 9 * kL[l].cin; i++) th[L->woff[l] + i] = std * nd(L->rng);
        }
        SR_CUDA_TRY(cudaMemcpy(L->theta, th.data(), sizeof(float) * k, cudaMemcpyHostToDevice));
        for (int l = 0; l < NL; l++) {
            const int ci = pad8(kL[l].cin), co = pad8(kL[l].cout);
            SR_CUDA_TRY(cudaMalloc(&L->wf[l], 2 * (size_t)co * kt_of(ci)));
            SR_CUDA_TRY(cudaMalloc(&L->wb[l], 2 * (size_t)ci * kt_of(co)));
        }
        const size_t per = (size_t)crop * crop;
        SR_CUDA_TRY(cudaMalloc(&L->sfeats, sizeof(float) * per * 8 * capacity));
        SR_CUDA_TRY(cudaMalloc(&L->stargets, sizeof(float) * per * capacity));
        SR_CUDA_TRY(cudaMalloc(&L->sscales, sizeof(float) * capacity));
        SR_CUDA_TRY(cudaMalloc(&L->err, sizeof(int)));
        SR_CUDA_TRY(cudaMemset(L->err, 0, sizeof(int)));
        SR_CUDA_TRY(cudaMalloc(&L->red_part, sizeof(double) * 2 * 148 * 16));
        SR_CUDA_TRY(cudaMalloc(&L->red_counter, sizeof(unsigned)));
        SR_CUDA_TRY(cudaMemset(L->red_counter, 0, sizeof(unsigned)));
        SR_CUDA_TRY(cudaMalloc(&L->scal, sizeof(double) * 4));
        L->pack(0);
        SR_CUDA_TRY(cudaDeviceSynchronize());
    } catch (...) {
        learned_destroy(L);
        throw;
    }
    return L;
}

void learned_destroy(Learner* L) {
    if (!L) return;
    cudaFree(L->theta);
    cudaFree(L->grad);
    cudaFree(L->m);
    cudaFree(L->v);
    for (int l = 0; l < NL; l++) {
        cudaFree(L->wf[l]);
        cudaFree(L->wb[l]);
    }
    cudaFree(L->sfeats);
    cudaFree(L->stargets);
    cudaFree(L->sscales);
    cudaFree(L->pos);
    cudaFree(L->err);
    cudaFree(L->red_part);
    cudaFree(L->red_counter);
    cudaFree(L->scal);
    cudaFree(L->bidx);
    cudaFree(L->btarget);
    L->train_net.destroy();
    delete L;
}

void learned_get_params(Learner* L, float* theta) {
    SR_CUDA_TRY(cudaMemcpy(theta, L->theta, sizeof(float) * L->nparams, cudaMemcpyDeviceToHost));
}

void learned_set_params(Learner* L, const float* theta) {
    SR_CUDA_TRY(cudaMemcpy(L->theta, theta, sizeof(float) * L->nparams, cudaMemcpyHostToDevice));
    L->pack(0);
    SR_CUDA_TRY(cudaDeviceSynchronize());
}

int learned_error(Learner* L, cudaStream_t s) {
    int e = 0;
    SR_CUDA_TRY(cudaMemcpyAsync(&e, L->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    SR_CUDA_TRY(cudaStreamSynchronize(s));
    return e;
}

int learned_samples(Learner* L) { return L->count; }

void learned_begin_collect(Learner* L, int w, int h, int crops, uint64_t seed) {
    SR_REQUIRE(w >= L->crop && h >= L->crop, "the system is smaller than a training crop");
    std::mt19937_64 r(seed);
    std::vector<int2> pos(crops);
    for (auto& p : pos) {
        p.x = (int)(r() % (uint64_t)(w - L->crop + 1));
        p.y = (int)(r() % (uint64_t)(h - L->crop + 1));
    }
    cudaFree(L->pos);
    L->pos = nullptr;
    SR_CUDA_TRY(cudaMalloc(&L->pos, sizeof(int2) * crops));
    SR_CUDA_TRY(cudaMemcpy(L->pos, pos.data(), sizeof(int2) * crops, cudaMemcpyHostToDevice));
    L->crops = crops;
    L->sys_first = L->count;
}

void learned_snapshot(Learner* L, const MgLevel& level0, const float* r, const float* e, cudaStream_t s) {
    if (L->count + L->crops > L->capacity) return;  // full: later snapshots are dropped
    const size_t N = (size_t)level0.w * level0.h;
    apply_scale_kernel<<<grid_of(N), RT, 0, s>>>(level0, r, L->red_part, L->red_counter, L->scal + 2);
    sr_note_launch();
    snapshot_kernel<<<L->crops, 256, 0, s>>>(level0, r, e, L->crop, L->pos, L->count, L->scal + 2, L->sfeats,
                                             L->stargets, L->sscales);
    sr_note_launch();
    L->count += L->crops;
}

void learned_end_collect(Learner* L, const MgLevel& level0, const float* e_final, cudaStream_t s) {
    const int count = L->count - L->sys_first;
    if (count <= 0) return;
    finish_targets_kernel<<<grid_of((size_t)count * L->crop * L->crop), RT, 0, s>>>(
        level0, e_final, L->crop, L->pos, L->crops, L->sys_first, count, L->stargets, L->sscales);
    sr_note_launch();
    SR_CUDA_TRY(cudaStreamSynchronize(s));
}

namespace {
double loss_step(Learner* L, Net& N, const float* target, cudaStream_t s) {
    forward(L, N, s);
    const size_t P = N.pix(0);
    target_energy_kernel<<<N.B, RT, 0, s>>>(N.H, N.W, N.feats, target, N.energy);
    sr_note_launch();
    energy_loss_kernel<<<grid_of(P), RT, 0, s>>>(N.B, N.H, N.W, N.act[NL - 1], N.feats, target, N.energy,
                                                 N.gact[NL - 1], L->red_part, L->red_counter, L->scal);
    sr_note_launch();
    backward(L, N, s);
    double loss = 0.0;
    SR_CUDA_TRY(cudaMemcpyAsync(&loss, L->scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    SR_CUDA_TRY(cudaStreamSynchronize(s));
    return loss;
}

void ensure_train_net(Learner* L, int batch) {
    if (L->train_batch == batch) return;
    L->train_net.destroy();
    L->train_net = Net();
    L->train_batch = 0;
    cudaFree(L->bidx);
    cudaFree(L->btarget);
    L->bidx = nullptr;
    L->btarget = nullptr;
    L->train_net.create(batch, L->crop, L->crop, true);
    SR_CUDA_TRY(cudaMalloc(&L->bidx, sizeof(int) * batch));
    SR_CUDA_TRY(cudaMalloc(&L->btarget, sizeof(float) * (size_t)batch * L->crop * L->crop));
    L->train_batch = batch;
}
}  // namespace

double learned_train(Learner* L, int iterations, int batch, double lr, uint64_t seed, cudaStream_t s) {
    SR_REQUIRE(L->count > 0, "the learner holds no samples");
    SR_REQUIRE(batch >= 1, "batch must be >= 1");
    ensure_train_net(L, batch);
    std::mt19937_64 r(seed);
    std::vector<int> idx(batch);
    double tail = 0.0;
    int tail_n = 0;
    for (int it = 0; it < iterations; it++) {
        for (int& i : idx) i = (int)(r() % (uint64_t)L->count);
        SR_CUDA_TRY(cudaMemcpyAsync(L->bidx, idx.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, s));
        gather_kernel<<<grid_of((size_t)batch * L->crop * L->crop), RT, 0, s>>>(
            L->crop, L->bidx, batch, L->sfeats, L->stargets, L->train_net.feats, L->btarget);
        sr_note_launch();
        const double loss = loss_step(L, L->train_net, L->btarget, s);
        if (it >= iterations - 10) {
            tail += loss;
            tail_n++;
        }
        if (!std::isfinite(loss)) continue;  // a batch with a non-finite loss leaves the weights alone
        L->adam_t++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - powf(b1, (float)L->adam_t), c2 = 1.0f - powf(b2, (float)L->adam_t);
        adam_kernel<<<grid_of(L->nparams), RT, 0, s>>>(L->nparams, L->theta, L->grad, L->m, L->v, (float)lr, b1, b2,
                                                       1e-8f, c1, c2);
        sr_note_launch();
        L->pack(s);
    }
    SR_CUDA_TRY(cudaStreamSynchronize(s));
    return tail_n ? tail / tail_n : 0.0;
}

double learned_loss_grad(Learner* L, const float* feats, const float* target, int n, float* grad, float* out,
                         cudaStream_t s) {
    ensure_train_net(L, n);
    const size_t per = (size_t)L->crop * L->crop;
    float* hin = nullptr;
    SR_CUDA_TRY(cudaMalloc(&hin, sizeof(float) * per * 4 * n));
    try {
        SR_CUDA_TRY(cudaMemcpyAsync(hin, feats, sizeof(float) * per * 4 * n, cudaMemcpyHostToDevice, s));
        nchw_to_feats_kernel<<<grid_of(per * n), RT, 0, s>>>(n, L->crop, hin, L->train_net.feats);
        sr_note_launch();
        SR_CUDA_TRY(cudaMemcpyAsync(L->btarget, target, sizeof(float) * per * n, cudaMemcpyHostToDevice, s));
        const double loss = loss_step(L, L->train_net, L->btarget, s);
        if (grad) SR_CUDA_TRY(cudaMemcpy(grad, L->grad, sizeof(float) * L->nparams, cudaMemcpyDeviceToHost));
        if (out) {
            std::vector<float> head(per * n * 8);
            SR_CUDA_TRY(cudaMemcpy(head.data(), L->train_net.act[NL - 1], sizeof(float) * head.size(),
                                   cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < per * n; i++) out[i] = head[i * 8];
        }
        cudaFree(hin);
        return loss;
    } catch (...) {
        cudaFree(hin);
        throw;
    }
}

LearnedApply* learned_apply_create(Learner* L, int w, int h) {
    LearnedApply* A = new LearnedApply();
    try {
        A->L = L;
        A->net.create(1, h, w, false);
        SR_CUDA_TRY(cudaMalloc(&A->scale, sizeof(double) * 2));
    } catch (...) {
        learned_apply_destroy(A);
        throw;
    }
    return A;
}

void learned_apply_destroy(LearnedApply* A) {
    if (!A) return;
    A->net.destroy();
    cudaFree(A->scale);
    delete A;
}

void learned_apply(LearnedApply* A, const MgLevel& level0, const float* r_in, const float* z_base, const float* r_dot,
                   float* z, double* part, unsigned* counter, double* rz_out, cudaStream_t s) {
    const size_t N = (size_t)level0.w * level0.h;
    apply_scale_kernel<<<grid_of(N), RT, 0, s>>>(level0, r_in, part, counter, A->scale);
    sr_note_launch();
    apply_features_kernel<<<grid_of(N), RT, 0, s>>>(level0, r_in, A->scale, A->net.feats);
    sr_note_launch();
    forward(A->L, A->net, s);
    apply_output_kernel<<<grid_of(N), RT, 0, s>>>(level0, r_dot, z_base, A->net.act[NL - 1], A->scale, z, part,
                                                  counter, rz_out);
    sr_note_launch();
}
