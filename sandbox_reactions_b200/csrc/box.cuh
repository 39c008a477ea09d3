// box.cuh — the active box's fit (crates/sr-engine/src/step/boxfit.rs).
#pragma once

#include "common.cuh"

constexpr int kBoxMaxBlocks = 148 * 8;  // the fit's partials: at most this many CTAs

// A box in world cells: origin and size, multiples of 8; w == 0 when no cell holds gas.
struct BoxRec {
    int x0, y0, w, h;
};

int box_blocks(size_t n);
// The box of the cells with Σ >= Σ_vac of `sigma` (a w x h plane whose origin is world cell (ox, oy)), grown by 8,
// rounded out to multiples of 8 and clamped to the W x H world, into rec[4] (device); `part` holds 4 ints per CTA.
void box_fit_launch(const float* sigma, int w, int h, int ox, int oy, int W, int H, float sigma_vac, int* part,
                    int* rec, cudaStream_t s);
