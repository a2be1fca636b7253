// Inputs of the warm-start MLP and the synthetic pages it is trained on.
//
// A patch is the 32 x 32 window of the signal (image x sign) whose centre pixel (16, 16) is the
// cell seed rounded to the nearest pixel, edges replicated. In a stack of images (images x H rows;
// cell boxes in stack rows, seeds in their own image's rows) a patch replicates the edges of its
// cell's image, so a stacked cell's patch is the one it has in that image. It is normalised by its own level and
// scale: bg = the smallest mean of the 60 2 x 2 blocks along its border (robust to single noisy
// pixels), amp = max - bg, and x = (v - bg) / amp, stored as bf16. One warp per patch, lane c
// holding column c in registers, so the window is read once.
//
// Training pages are rendered here so that the training set comes from the same detection and
// plain-fit pipeline the warm start serves: every hole is a rotated superellipse
// |u / a|^n + |v / b|^n <= 1 whose pixel coverage is sampled on an s x s grid; the caller blurs
// the coverage (spx_gaussian_filter) and k_page_finish turns it into background + amplitude x
// coverage + Gaussian read noise (a counter-based hash generator, Box-Muller), rounded to uint16.

#include <cuda_bf16.h>

#include "common.cuh"

namespace spx {
namespace {

constexpr int kPatch = 32;
// Templated on the pixel type so that a lane's 32 loads are straight-line code, all in flight at
// once (a dtype switch per load can put each load behind its own branch).
template <typename Px>
__global__ void k_extract_patches(const Px* img, double sign, int images, int H, int W, const double* seeds,
                                  const int* boxes, int n, __nv_bfloat16* out, double* norm) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        // First row of the cell's image (a box's y is in stack rows).
        const int y0 = boxes ? min(max(boxes[4LL * i + 1], 0) / H, images - 1) * H : 0;
        const int ox = (int)rint(seeds[2LL * i]) - kPatch / 2, oy = (int)rint(seeds[2LL * i + 1]) - kPatch / 2;
        const int x = min(max(ox + lane, 0), W - 1);
        double col[kPatch];
        double mx = -dinf();
#pragma unroll
        for (int r = 0; r < kPatch; ++r) {
            const int y = y0 + min(max(oy + r, 0), H - 1);
            col[r] = sign * (double)img[(long long)y * W + x];
            mx = fmax(mx, col[r]);
        }
        mx = warp_max(mx);
        // 2 x 2 block sums along the border: this lane's column pair (lane, lane ^ 1) for the top and
        // bottom block rows, and the block rows in between for the outer column pairs.
        double lo = dinf();
        auto pair = [&](int r) { return col[r] + col[r + 1]; };
        const double top = pair(0), bottom = pair(kPatch - 2);
        const double top_b = top + __shfl_xor_sync(0xffffffffu, top, 1);
        const double bottom_b = bottom + __shfl_xor_sync(0xffffffffu, bottom, 1);
        lo = fmin(top_b, bottom_b);
#pragma unroll
        for (int br = 1; br < kPatch / 2 - 1; ++br) {
            const double v = pair(2 * br);
            const double blk = v + __shfl_xor_sync(0xffffffffu, v, 1);
            if (lane < 2 || lane >= kPatch - 2) lo = fmin(lo, blk);
        }
        const double bg = warp_min(lo) / 4.0;
        const double amp = fmax(mx - bg, 1e-12);
        const double inv = 1.0 / amp;
        __nv_bfloat16* o = out + (long long)i * kPatch * kPatch + lane;
#pragma unroll
        for (int r = 0; r < kPatch; ++r) o[r * kPatch] = __float2bfloat16_rn((float)((col[r] - bg) * inv));
        if (lane == 0) {
            norm[4LL * i] = ox;
            norm[4LL * i + 1] = y0 + oy;
            norm[4LL * i + 2] = bg;
            norm[4LL * i + 3] = amp;
        }
    }
}

// Fraction of the pixel's s x s sample points inside any hole of the 3 x 3 grid cells around it.
// Holes: (cx, cy, a, b, theta, n) rows; grid: cell size `cell`, CSR start[gh * gw + 1], ids.
__global__ void k_hole_coverage(int H, int W, const double* holes, const int* start, const int* ids, int gw, int gh,
                                double cell, int s, double* cov) {
    const long long total = (long long)H * W;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(t, W, &y, &x);
        const int gx = min(max((int)floor(x / cell), 0), gw - 1), gy = min(max((int)floor(y / cell), 0), gh - 1);
        int inside = 0;
        for (int sy = 0; sy < s; ++sy)
            for (int sx = 0; sx < s; ++sx) {
                const double X = x - 0.5 + (sx + 0.5) / s, Y = y - 0.5 + (sy + 0.5) / s;
                bool hit = false;
                for (int cy = max(gy - 1, 0); cy <= min(gy + 1, gh - 1) && !hit; ++cy)
                    for (int cx = max(gx - 1, 0); cx <= min(gx + 1, gw - 1) && !hit; ++cx)
                        for (int k = start[cy * gw + cx]; k < start[cy * gw + cx + 1] && !hit; ++k) {
                            const double* h = holes + 6LL * ids[k];
                            const double dx = X - h[0], dy = Y - h[1];
                            const double c = cos(h[4]), sn = sin(h[4]);
                            const double u = fabs((dx * c + dy * sn) / h[2]), v = fabs((-dx * sn + dy * c) / h[3]);
                            if (u <= 1.0 && v <= 1.0 && pow(u, h[5]) + pow(v, h[5]) <= 1.0) hit = true;
                        }
                inside += hit;
            }
        cov[t] = (double)inside / (double)(s * s);
    }
}

// splitmix64 finaliser as a counter-based hash.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void k_page_finish(const double* cov, long long n, double background, double amplitude, double noise,
                              unsigned long long seed, uint16_t* page) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long h1 = mix64(seed ^ (2 * (unsigned long long)i));
        const unsigned long long h2 = mix64(seed ^ (2 * (unsigned long long)i + 1));
        const double u1 = ((h1 >> 11) + 1) * (1.0 / 9007199254740993.0), u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
        const double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        const double v = rint(background + amplitude * cov[i] + noise * g);
        page[i] = (uint16_t)fmin(fmax(v, 0.0), 65535.0);
    }
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

int spx_extract_patches_stack(const void* img, int dtype, double sign, int images, int height, int width,
                              const double* seeds, const int* boxes, int n, void* out, double* norm, void* stream) {
    SPX_REQUIRE(images > 0 && height > 0 && width > 0 && n >= 0 && dtype >= SPX_U8 && dtype <= SPX_F64,
                "bad arguments");
    SPX_REQUIRE((long long)images * height <= 0x7fffffffLL, "stack too tall");
    SPX_REQUIRE(images == 1 || boxes, "a stack needs the cell boxes");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(img && seeds && out && norm, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = grid_for(n, 8, 148 * 32);
    auto* o = static_cast<__nv_bfloat16*>(out);
    switch (dtype) {
        case SPX_U8:
            k_extract_patches<<<grid, 256, 0, s>>>(static_cast<const uint8_t*>(img), sign, images, height, width,
                                                   seeds, boxes, n, o, norm);
            break;
        case SPX_U16:
            k_extract_patches<<<grid, 256, 0, s>>>(static_cast<const uint16_t*>(img), sign, images, height, width,
                                                   seeds, boxes, n, o, norm);
            break;
        case SPX_F32:
            k_extract_patches<<<grid, 256, 0, s>>>(static_cast<const float*>(img), sign, images, height, width,
                                                   seeds, boxes, n, o, norm);
            break;
        default:
            k_extract_patches<<<grid, 256, 0, s>>>(static_cast<const double*>(img), sign, images, height, width,
                                                   seeds, boxes, n, o, norm);
    }
    return check_launch("k_extract_patches");
}

int spx_extract_patches(const void* img, int dtype, double sign, int height, int width, const double* seeds, int n,
                        void* out, double* norm, void* stream) {
    return spx_extract_patches_stack(img, dtype, sign, 1, height, width, seeds, nullptr, n, out, norm, stream);
}

int spx_hole_coverage(int height, int width, const double* holes, const int* grid_start, const int* grid_ids,
                      int grid_w, int grid_h, double cell, int samples, double* coverage, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && grid_w > 0 && grid_h > 0 && cell > 0 && samples >= 1 && samples <= 16,
                "bad arguments");
    SPX_REQUIRE(holes && grid_start && grid_ids && coverage, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_hole_coverage<<<grid_for((long long)height * width, 256), 256, 0, s>>>(height, width, holes, grid_start,
                                                                            grid_ids, grid_w, grid_h, cell, samples,
                                                                            coverage);
    return check_launch("k_hole_coverage");
}

int spx_page_finish(const double* coverage, long long n, double background, double amplitude, double noise,
                    unsigned long long seed, uint16_t* page, void* stream) {
    SPX_REQUIRE(n > 0 && coverage && page, "bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_page_finish<<<grid_for(n, 256), 256, 0, s>>>(coverage, n, background, amplitude, noise, seed, page);
    return check_launch("k_page_finish");
}

}  // extern "C"
