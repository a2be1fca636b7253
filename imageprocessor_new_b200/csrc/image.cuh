// Device views of the signal image and the background map, shared by the deblending kernels and
// the tail-family windows.
#pragma once

#include "common.cuh"

namespace spx {

// Background map: bg(y, x) = (1 - t[y]) rows[j1[y]-1][x] + t[y] rows[j1[y]][x] (ny > 1),
// rows[0][x] (ny == 1), or a constant.
__device__ __forceinline__ double bg_at(const spx_bgmap& m, int y, int x) {
    if (m.mode == SPX_BG_FIXED) return m.fixed;
    if (m.ny == 1) return m.rows[x];
    const int j = m.j1[y];
    const double t = m.t[y];
    return __dadd_rn(__dmul_rn(__dsub_rn(1.0, t), m.rows[(long long)(j - 1) * m.width + x]),
                     __dmul_rn(t, m.rows[(long long)j * m.width + x]));
}

struct Image {
    const void* data;
    int dtype;
    double sign;
    int H, W;
    __device__ __forceinline__ double at(int y, int x) const {
        const double v = load_px(data, dtype, (long long)y * W + x);
        return sign < 0 ? -v : v;
    }
};

}  // namespace spx
