// Image filters of the seed revision and the feature masks of the deblending driver.
//
// Reference: revise_seeds (subpx/_cpu/deblend.py:525-567): gaussian_filter(residual, sigma,
// mode="nearest") then maximum_filter(size 2r+1, mode="nearest"), peaks = local maxima above a
// level; _unmodelled_features (subpx/cd.py:411-421): thresholded pixels of components without a
// model, dilated twice with the 3x3 cross; the oversized-component exclusion (subpx/cd.py:489-491).
//
// The Gaussian filter is separable (axis 0, then axis 1) with scipy's symmetric correlate1d sum:
// centre term first, then the pairs (in[-k] + in[k]) * w[k] from the outermost inwards, edges
// replicated. The maximum filter is exact in any order.

#include "common.cuh"

namespace spx {
namespace {

// out[y][x] = sum_k w[k] in[y + (k - r) * dy][x + (k - r) * dx] (nearest edges), axis 0 when dy.
__global__ void k_gauss_1d(const double* in, int H, int W, const double* w, int r, int along_y, double* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i % W);
        auto at = [&](int o) {
            if (along_y) return in[(long long)min(max(y + o, 0), H - 1) * W + x];
            return in[(long long)y * W + min(max(x + o, 0), W - 1)];
        };
        double t = __dmul_rn(at(0), w[r]);
        for (int k = r; k >= 1; --k) t = __dadd_rn(t, __dmul_rn(__dadd_rn(at(-k), at(k)), w[r - k]));
        out[i] = t;
    }
}

__global__ void k_max_1d(const double* in, int H, int W, int r, int along_y, double* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i % W);
        double m = -dinf();
        for (int o = -r; o <= r; ++o) {
            const double v = along_y ? in[(long long)min(max(y + o, 0), H - 1) * W + x]
                                     : in[(long long)y * W + min(max(x + o, 0), W - 1)];
            m = fmax(m, v);
        }
        out[i] = m;
    }
}

// Pixels with smooth == maxf, smooth > level and not excluded, appended as (y, x) int pairs.
__global__ void k_peaks(const double* smooth, const double* maxf, const uint8_t* exclude, int H, int W,
                        double level, int* out, int capacity, int* count) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const double s = smooth[i];
        if (s == maxf[i] && s > level && !(exclude && exclude[i])) {
            const int slot = atomicAdd(count, 1);
            if (slot < capacity) {
                out[2 * slot] = (int)(i / W);
                out[2 * slot + 1] = (int)(i % W);
            }
        }
    }
}

// mask[i] = flags[labels[i]] (labels >= 0) — per-pixel lookup of a per-label flag.
__global__ void k_label_flags(const int* labels, const uint8_t* flags, long long n, uint8_t* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = labels[i];
        out[i] = l > 0 ? flags[l] : 0;
    }
}

// One dilation with the 3x3 cross, zero outside the image.
__global__ void k_dilate_cross(const uint8_t* in, int H, int W, uint8_t* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i % W);
        uint8_t v = in[i];
        if (!v) v = (y > 0 && in[i - W]) || (y < H - 1 && in[i + W]) || (x > 0 && in[i - 1]) || (x < W - 1 && in[i + 1]);
        out[i] = v;
    }
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

int spx_gaussian_filter(const double* in, int height, int width, const double* weights, int radius, double* tmp,
                        double* out, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && radius >= 0, "bad arguments");
    SPX_REQUIRE(in && weights && tmp && out && tmp != in && tmp != out, "null or aliased pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = (long long)height * width;
    k_gauss_1d<<<grid_for(n, 256), 256, 0, s>>>(in, height, width, weights, radius, 1, tmp);
    if (int e = check_launch("k_gauss_1d")) return e;
    k_gauss_1d<<<grid_for(n, 256), 256, 0, s>>>(tmp, height, width, weights, radius, 0, out);
    return check_launch("k_gauss_1d");
}

int spx_maximum_filter(const double* in, int height, int width, int radius, double* tmp, double* out, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && radius >= 0, "bad arguments");
    SPX_REQUIRE(in && tmp && out && tmp != in && tmp != out, "null or aliased pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = (long long)height * width;
    k_max_1d<<<grid_for(n, 256), 256, 0, s>>>(in, height, width, radius, 1, tmp);
    if (int e = check_launch("k_max_1d")) return e;
    k_max_1d<<<grid_for(n, 256), 256, 0, s>>>(tmp, height, width, radius, 0, out);
    return check_launch("k_max_1d");
}

int spx_find_peaks(const double* smooth, const double* maxf, const uint8_t* exclude, int height, int width,
                   double level, int* out_yx, int capacity, int* count, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && capacity >= 0, "bad arguments");
    SPX_REQUIRE(smooth && maxf && count && (out_yx || capacity == 0), "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SPX_CUDA(cudaMemsetAsync(count, 0, sizeof(int), s));
    const long long n = (long long)height * width;
    k_peaks<<<grid_for(n, 256), 256, 0, s>>>(smooth, maxf, exclude, height, width, level, out_yx, capacity, count);
    return check_launch("k_peaks");
}

int spx_label_mask(const int* labels, const uint8_t* flags, int height, int width, int dilations, uint8_t* out,
                   uint8_t* tmp, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && dilations >= 0, "bad arguments");
    SPX_REQUIRE(labels && flags && out && (dilations == 0 || tmp), "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = (long long)height * width;
    uint8_t* cur = dilations % 2 ? tmp : out;
    k_label_flags<<<grid_for(n, 256), 256, 0, s>>>(labels, flags, n, cur);
    if (int e = check_launch("k_label_flags")) return e;
    for (int d = 0; d < dilations; ++d) {
        uint8_t* nxt = cur == out ? tmp : out;
        k_dilate_cross<<<grid_for(n, 256), 256, 0, s>>>(cur, height, width, nxt);
        if (int e = check_launch("k_dilate_cross")) return e;
        cur = nxt;
    }
    return SPX_OK;
}

}  // extern "C"
