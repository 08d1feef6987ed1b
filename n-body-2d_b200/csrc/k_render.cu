// k_render.cu -- headless point-splat rendering of the bodies into an RGBA8
// buffer, the frame the reference draws with SFML/OpenGL
// (src/Graphics/src/Graphics.cpp:122-128), without a graphics stack.
//
// Mapping (ViewPort::coords_to_pos_on_viewport, src/Graphics/lib/ViewPort/src/
// ViewPort.cpp:90-93): relative = (p - rect.position) / rect.size in FP64,
// rounded to float, times the window resolution in float; pixel (i, j) has
// its centre at (i + 0.5, j + 0.5), row 0 at the top.
//
// Coverage (a GL point of diameter D, then the body shader's circle clip,
// Graphics.cpp:20-26): a pixel is covered when its centre c lies in the
// half-open square [p - D/2, p + D/2) on both axes and, for D > 1, when the
// point-sprite coordinate u = (c - (p - D/2)) / D - 1/2 has u.u <= 1/4
// (the shader discards length(u) > 1/2).
//
// Colour: every body is BODY_COLOR = (255, 255, 255, 120)
// (src/common_lib/Constants/include/Constants/Constants.hpp:39) blended over
// the black clear colour with alpha blending, so a pixel covered k times has
// the 8-bit value of k successive blends, c <- round(120 + c * 135 / 255),
// whatever the order; alpha stays 255.  The kernels count coverings with
// atomics and map counts through that table.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "nb_internal.cuh"

namespace nb {
namespace {

__global__ void render_count(const double2* __restrict__ pos, int64_t n, double rx, double ry,
                             double rw, double rh, float res_x, float res_y, int width,
                             int height, float diam, uint32_t* __restrict__ count) {
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= n) return;
    const double2 q = pos[b];
    const float px = __fmul_rn(res_x, (float)((q.x - rx) / rw));
    const float py = __fmul_rn(res_y, (float)((q.y - ry) / rh));
    const float half = __fmul_rn(diam, 0.5f);
    const float x0 = __fsub_rn(px, half), x1 = __fadd_rn(px, half);
    const float y0 = __fsub_rn(py, half), y1 = __fadd_rn(py, half);
    if (!(x1 > 0.f && y1 > 0.f && x0 < (float)width && y0 < (float)height)) return;
    const int i0 = max(0, (int)floorf(x0) - 1), i1 = min(width - 1, (int)ceilf(x1) + 1);
    const int j0 = max(0, (int)floorf(y0) - 1), j1 = min(height - 1, (int)ceilf(y1) + 1);
    for (int j = j0; j <= j1; ++j) {
        const float cy = __fadd_rn((float)j, 0.5f);
        if (!(y0 <= cy && cy < y1)) continue;
        for (int i = i0; i <= i1; ++i) {
            const float cx = __fadd_rn((float)i, 0.5f);
            if (!(x0 <= cx && cx < x1)) continue;
            if (diam > 1.f) {
                const float u = __fsub_rn(__fdiv_rn(__fsub_rn(cx, x0), diam), 0.5f);
                const float v = __fsub_rn(__fdiv_rn(__fsub_rn(cy, y0), diam), 0.5f);
                if (__fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)) > 0.25f) continue;
            }
            atomicAdd(count + (int64_t)j * width + i, 1u);
        }
    }
}

__global__ void render_resolve(const uint32_t* __restrict__ count, int64_t pixels,
                               const uint8_t* __restrict__ table, uchar4* __restrict__ rgba) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= pixels) return;
    const uint8_t c = table[min(count[k], 255u)];
    rgba[k] = make_uchar4(c, c, c, 255);
}

inline unsigned blocks_for(int64_t n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

}  // namespace

void launch_render(nb_ctx* c, const double2* pos, const nb_view& v, uint32_t* count,
                   const uint8_t* table, uchar4* rgba) {
    const int64_t pixels = (int64_t)v.res_x * v.res_y;
    c->launches += 2;
    cudaMemsetAsync(count, 0, sizeof(uint32_t) * pixels, c->stream);
    render_count<<<blocks_for(c->n, 256), 256, 0, c->stream>>>(
        pos, c->n, v.x, v.y, v.width, v.height, (float)v.res_x, (float)v.res_y, (int)v.res_x,
        (int)v.res_y, v.point_diameter, count);
    render_resolve<<<blocks_for(pixels, 256), 256, 0, c->stream>>>(count, pixels, table, rgba);
}

}  // namespace nb
