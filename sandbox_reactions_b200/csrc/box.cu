// box.cu — the active box (crates/sr-engine/src/step/boxfit.rs; shaders/reduce.wgsl:377-466): the bounding box of the
// cells with Σ >= Σ_vac, grown by 8 cells, rounded out to multiples of 8, clamped to the world. One grid-stride pass
// takes each CTA's (min x, min y, max x + 1, max y + 1) with shuffles and a shared-memory step; one CTA reduces the
// partials (integer min and max: the order does not matter) and writes the box. Nothing sizes a launch from the device
// record: the host reads it at the refits (the context steps the box's crop as a world of its own).
#include <limits.h>

#include "box.cuh"

namespace {

constexpr int kBoxThreads = 256;

__device__ __forceinline__ void warp_minmax(int& a, int& b, int& c, int& d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = min(a, __shfl_down_sync(0xffffffffu, a, o));
        b = min(b, __shfl_down_sync(0xffffffffu, b, o));
        c = max(c, __shfl_down_sync(0xffffffffu, c, o));
        d = max(d, __shfl_down_sync(0xffffffffu, d, o));
    }
}

__global__ void box_cells_kernel(const float* __restrict__ sigma, int w, int h, float sigma_vac, int* part) {
    const size_t n = (size_t)w * h;
    int x0 = INT_MAX, y0 = INT_MAX, x1 = INT_MIN, y1 = INT_MIN;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (sigma[i] >= sigma_vac) {
            int x, y;
            split_index(i, w, x, y);
            x0 = min(x0, x);
            y0 = min(y0, y);
            x1 = max(x1, x + 1);
            y1 = max(y1, y + 1);
        }
    }
    warp_minmax(x0, y0, x1, y1);
    __shared__ int s[4][kBoxThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s[0][warp] = x0;
        s[1][warp] = y0;
        s[2][warp] = x1;
        s[3][warp] = y1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kBoxThreads / 32; k++) {
            x0 = min(x0, s[0][k]);
            y0 = min(y0, s[1][k]);
            x1 = max(x1, s[2][k]);
            y1 = max(y1, s[3][k]);
        }
        int* p = part + 4 * (size_t)blockIdx.x;
        p[0] = x0;
        p[1] = y0;
        p[2] = x1;
        p[3] = y1;
    }
}

__global__ void box_fit_kernel(const int* part, int nblocks, int ox, int oy, int W, int H, int* rec) {
    int x0 = INT_MAX, y0 = INT_MAX, x1 = INT_MIN, y1 = INT_MIN;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        x0 = min(x0, part[4 * b]);
        y0 = min(y0, part[4 * b + 1]);
        x1 = max(x1, part[4 * b + 2]);
        y1 = max(y1, part[4 * b + 3]);
    }
    warp_minmax(x0, y0, x1, y1);
    __shared__ int s[4][kBoxThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s[0][warp] = x0;
        s[1][warp] = y0;
        s[2][warp] = x1;
        s[3][warp] = y1;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int k = 1; k < kBoxThreads / 32; k++) {
        x0 = min(x0, s[0][k]);
        y0 = min(y0, s[1][k]);
        x1 = max(x1, s[2][k]);
        y1 = max(y1, s[3][k]);
    }
    if (x0 == INT_MAX) {  // no cell holds gas: the empty box
        rec[0] = rec[1] = rec[2] = rec[3] = 0;
        return;
    }
    // in world coordinates, grown by 8, rounded out to multiples of 8, clamped to the world
    auto down8 = [](int v) { return v >= 0 ? v / 8 * 8 : -((-v + 7) / 8 * 8); };
    auto up8 = [](int v) { return (v + 7) / 8 * 8; };
    const int bx0 = max(0, down8(x0 + ox - 8)), by0 = max(0, down8(y0 + oy - 8));
    const int bx1 = min(W, up8(x1 + ox + 8)), by1 = min(H, up8(y1 + oy + 8));
    rec[0] = bx0;
    rec[1] = by0;
    rec[2] = bx1 - bx0;
    rec[3] = by1 - by0;
}

}  // namespace

int box_blocks(size_t n) {
    const size_t b = (n + kBoxThreads - 1) / kBoxThreads;
    return (int)(b < 1 ? 1 : (b > kBoxMaxBlocks ? kBoxMaxBlocks : b));
}

void box_fit_launch(const float* sigma, int w, int h, int ox, int oy, int W, int H, float sigma_vac, int* part,
                    int* rec, cudaStream_t s) {
    const int nb = box_blocks((size_t)w * h);
    box_cells_kernel<<<nb, kBoxThreads, 0, s>>>(sigma, w, h, sigma_vac, part);
    sr_note_launch();
    box_fit_kernel<<<1, kBoxThreads, 0, s>>>(part, nb, ox, oy, W, H, rec);
    sr_note_launch();
    SR_CUDA_TRY(cudaGetLastError());
}
