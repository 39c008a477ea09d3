// grav_static.cu — P2's gravity solve for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory themselves (a game engine or plug-in host that hands its plug-ins
// buffers and forbids them cudaMalloc), and some cannot afford cudaMalloc's device-wide synchronisation inside a
// time-stepping loop. For them, sr_gravity_solve_static runs the same FFT-convolution kernels as a context's P2 on
// device buffers the caller passes in, with every scratch buffer the solve needs — the half spectrum, the ringed
// potential, the kernel's spectrum and the twiddle tables — held in file-scope static device arrays sized for worlds
// of at most kStaticMaxWorld cells a side. Every GPU that loads this library holds those arrays (about 1.1 MB) until
// the process exits.
//
// Host code never hands a static array's name to a kernel: a __device__ array's name is a host-side stand-in, not a
// device address. Once per device, with that device current, the first call looks up each array's device address with
// cudaGetSymbolAddress (checking every return code) and keeps them. That first call, and every later call whose
// padded size, gravity kernel, G or (for the softened kernel) softening differs from the previous call's on the same
// device, also builds the kernel's spectrum and twiddles on the host, copies them up and waits for the caller's stream
// (the host staging is reused), so such a call blocks the host and must not be made during a stream capture. Calls
// share the arrays: two calls whose work overlaps on the GPU race. No buffer needs clearing between calls: every value
// a kernel reads was written earlier in the same call.
#include <math.h>
#include <string.h>

#include <mutex>
#include <string>

#include "grav.cuh"

namespace {

constexpr int kStaticMaxWorld = 256;                // world axes up to 256 cells
constexpr int kStaticMaxPadded = 2 * kStaticMaxWorld;  // their padded FFT length
constexpr size_t kSpecCount = (size_t)(kStaticMaxPadded / 2 + 1) * (kStaticMaxWorld + 2);
constexpr size_t kRingCount = (size_t)(kStaticMaxWorld + 2) * (kStaticMaxWorld + 2);
constexpr size_t kKhatCount = (size_t)(kStaticMaxPadded / 2 + 1) * (kStaticMaxPadded / 2 + 1);

static __device__ __align__(256) float2 g_spec[kSpecCount];
static __device__ __align__(256) float g_ring[kRingCount];
static __device__ __align__(256) float g_khat[kKhatCount];
static __device__ __align__(256) float2 g_tw[2 * kStaticMaxPadded];

// Host-side staging, static too: the f64 work of the kernel's spectrum and the f32 tables copied up.
static double h_re[(size_t)kStaticMaxPadded * kStaticMaxPadded];
static double h_im[(size_t)kStaticMaxPadded * kStaticMaxPadded];
static double h_cos[kStaticMaxPadded / 2], h_sin[kStaticMaxPadded / 2];
static float h_khat[kKhatCount];
static float2 h_tw[2 * kStaticMaxPadded];

constexpr int kMaxDevices = 64;
struct DeviceSlot {
    bool ready = false;
    float2* spec = nullptr;
    float* ring = nullptr;
    float* khat = nullptr;
    float2* tw = nullptr;
    // what the uploaded tables were built for
    int px = 0, py = 0, kind = -1;
    double G = 0.0, eps = 0.0;
};
static DeviceSlot g_slots[kMaxDevices];
static std::mutex g_mutex;

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw SrError{SR_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

// In-place radix-2 f64 FFT of n points at stride `stride` from `off` (forward, unnormalised), on the static arrays.
void fft_f64_static(size_t off, size_t stride, int n) {
    int bits = 0;
    while ((1 << bits) < n) bits++;
    for (int k = 0; k < n / 2; k++) {
        const double a = -2.0 * M_PI * (double)k / (double)n;
        h_cos[k] = cos(a);
        h_sin[k] = sin(a);
    }
    for (int i = 0; i < n; i++) {
        int j = 0;
        for (int b = 0; b < bits; b++)
            if (i & (1 << b)) j |= 1 << (bits - 1 - b);
        if (i < j) {
            double t = h_re[off + i * stride];
            h_re[off + i * stride] = h_re[off + j * stride];
            h_re[off + j * stride] = t;
            t = h_im[off + i * stride];
            h_im[off + i * stride] = h_im[off + j * stride];
            h_im[off + j * stride] = t;
        }
    }
    for (int half = 1; half < n; half *= 2) {
        const int step = n / (2 * half);
        for (int start = 0; start < n; start += 2 * half)
            for (int k = 0; k < half; k++) {
                const double wr = h_cos[k * step], wi = h_sin[k * step];
                const size_t a = off + (start + k) * stride, b = off + (start + k + half) * stride;
                const double br = h_re[b] * wr - h_im[b] * wi, bi = h_re[b] * wi + h_im[b] * wr;
                const double ar = h_re[a], ai = h_im[a];
                h_re[a] = ar + br;
                h_im[a] = ai + bi;
                h_re[b] = ar - br;
                h_im[b] = ai - bi;
            }
    }
}

double kernel_at(int kind, double G, double eps, long dx, long dy) {
    const double r2 = (double)(dx * dx + dy * dy);
    if (kind == SR_KERNEL_SOFTENED) return -G / sqrt(r2 + eps * eps);
    if (dx == 0 && dy == 0) return -G * 3.525494348078172;  // reference/grav.rs:24-34
    return -G / sqrt(r2);
}

// The kernel's real-even spectrum quarter, scaled by 1/(px py), and the twiddle tables, built on the host in the
// static staging arrays and copied to the device's static arrays.
void upload_tables(DeviceSlot& d, int px, int py, int kind, double G, double eps, cudaStream_t s) {
    for (int j = 0; j < py; j++)
        for (int i = 0; i < px; i++) {
            const long dx = i < px / 2 ? i : i - px, dy = j < py / 2 ? j : j - py;
            h_re[(size_t)j * px + i] = kernel_at(kind, G, eps, dx, dy);
            h_im[(size_t)j * px + i] = 0.0;
        }
    for (int j = 0; j < py; j++) fft_f64_static((size_t)j * px, 1, px);
    for (int i = 0; i <= px / 2; i++) fft_f64_static((size_t)i, (size_t)px, py);
    const double scale = 1.0 / ((double)px * (double)py);
    for (int i = 0; i <= px / 2; i++)
        for (int j = 0; j <= py / 2; j++) h_khat[(size_t)i * (py / 2 + 1) + j] = (float)(h_re[(size_t)j * px + i] * scale);
    for (int k = 0; k < px; k++) {
        const double a = -2.0 * M_PI * (double)k / (double)px;
        h_tw[k] = make_float2((float)cos(a), (float)sin(a));
    }
    for (int k = 0; k < py; k++) {
        const double a = -2.0 * M_PI * (double)k / (double)py;
        h_tw[kStaticMaxPadded + k] = make_float2((float)cos(a), (float)sin(a));
    }
    const size_t kq = (size_t)(px / 2 + 1) * (py / 2 + 1);
    // forget what the arrays held before the copies start: if one of them fails, the next call uploads again
    d.kind = -1;
    d.px = d.py = 0;
    check(cudaMemcpyAsync(d.khat, h_khat, sizeof(float) * kq, cudaMemcpyHostToDevice, s), "copy K̂ to the static array");
    check(cudaMemcpyAsync(d.tw, h_tw, sizeof(float2) * 2 * kStaticMaxPadded, cudaMemcpyHostToDevice, s),
          "copy the twiddles to the static array");
    check(cudaStreamSynchronize(s), "wait for the table upload");  // the host staging is reused by the next call
    d.px = px;
    d.py = py;
    d.kind = kind;
    d.G = G;
    d.eps = eps;
}

}  // namespace

extern "C" sr_status sr_gravity_solve_static(const sr_config* cfg, const float* sigma, float* phi, float* gx,
                                             float* gy, void* stream) {
    try {
        SR_REQUIRE(cfg && sigma && phi && gx && gy, "sr_gravity_solve_static: null argument");
        SR_REQUIRE(cfg->struct_size == sizeof(sr_config), "sr_config.struct_size does not match this library");
        const int w = (int)cfg->width, h = (int)cfg->height;
        SR_REQUIRE(w >= 16 && h >= 16 && w % 8 == 0 && h % 8 == 0, "sr_gravity_solve_static: world axes must be "
                                                                    "multiples of 8, at least 16");
        SR_REQUIRE(w <= kStaticMaxWorld && h <= kStaticMaxWorld,
                   "sr_gravity_solve_static: a " + std::to_string(w) + "x" + std::to_string(h) +
                       " world exceeds the static scratch's " + std::to_string(kStaticMaxWorld) + "x" +
                       std::to_string(kStaticMaxWorld) + " cells");
        SR_REQUIRE(cfg->kernel <= SR_KERNEL_SOFTENED, "unknown gravity kernel");
        SR_REQUIRE(!(cfg->kernel == SR_KERNEL_SOFTENED && !(cfg->softening > 0.0)),
                   "the softened kernel needs softening > 0");
        cudaStream_t s = (cudaStream_t)stream;
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        SR_REQUIRE(dev >= 0 && dev < kMaxDevices, "device index past the static slots");
        std::lock_guard<std::mutex> lock(g_mutex);
        DeviceSlot& d = g_slots[dev];
        if (!d.ready) {
            // the device addresses of the static arrays, looked up with this device current
            check(cudaGetSymbolAddress((void**)&d.spec, g_spec), "cudaGetSymbolAddress(g_spec)");
            check(cudaGetSymbolAddress((void**)&d.ring, g_ring), "cudaGetSymbolAddress(g_ring)");
            check(cudaGetSymbolAddress((void**)&d.khat, g_khat), "cudaGetSymbolAddress(g_khat)");
            check(cudaGetSymbolAddress((void**)&d.tw, g_tw), "cudaGetSymbolAddress(g_tw)");
            d.ready = true;
        }
        const int px = grav_padded_size(w), py = grav_padded_size(h);
        // the self-cell kernel ignores the softening, so a change of it alone keeps the tables
        const double eps = cfg->kernel == SR_KERNEL_SOFTENED ? cfg->softening : 0.0;
        if (d.px != px || d.py != py || d.kind != (int)cfg->kernel || d.G != cfg->G || d.eps != eps)
            upload_tables(d, px, py, (int)cfg->kernel, cfg->G, eps, s);
        // the allocating path's kernels, their scratch pointed at the static arrays
        GravPlan plan;
        plan.w = w;
        plan.h = h;
        plan.px = px;
        plan.py = py;
        plan.ld = (size_t)h + 2;
        plan.sigma_vac = (float)cfg->sigma_vac;
        plan.spec = d.spec;
        plan.phi_ring = d.ring;
        plan.khat = d.khat;
        plan.tw_x = d.tw;
        plan.tw_y = d.tw + kStaticMaxPadded;
        plan.solve(sigma, phi, gx, gy, s);
        check(cudaGetLastError(), "gravity kernels");
        return SR_OK;
    } catch (const SrError& e) {
        sr_set_global_error(e.message);
        return e.status;
    }
}
