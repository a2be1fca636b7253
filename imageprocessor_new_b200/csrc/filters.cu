// Image filters of the seed revision and the feature masks of the deblending driver.
//
// Reference: revise_seeds (subpx/_cpu/deblend.py:525-567): gaussian_filter(residual, sigma,
// mode="nearest") then maximum_filter(size 2r+1, mode="nearest"), peaks = local maxima above a
// level; _unmodelled_features (subpx/cd.py:411-421): thresholded pixels of components without a
// model, dilated twice with the 3x3 cross; the oversized-component exclusion (subpx/cd.py:489-491).
//
// The Gaussian filter is separable (axis 0, then axis 1) with scipy's symmetric correlate1d sum:
// centre term first, then the pairs (in[-k] + in[k]) * w[k] from the outermost inwards, edges
// replicated. The maximum and minimum filters (also detect_peaks' prominence window,
// subpx/_cpu/deblend.py:620) are exact in any order.

#include "common.cuh"

namespace spx {
namespace {

// Separable 1-D passes through shared-memory tiles: a block stages its outputs' window plus the
// r-pixel halo on both sides (edges replicated, scipy's mode="nearest") once, then every output
// reads its 2r + 1 inputs from shared memory. Along x a block covers kRowTile pixels of one row;
// along y it covers 32 columns x kColTile rows.
constexpr int kRowTile = 1024;
constexpr int kColTile = 64;
constexpr int kFilterMaxR = 200;  // larger radii take the direct path

struct GaussOp {
    const double* w;
    int r;
    // scipy correlate1d with a symmetric kernel: centre first, then the pairs outermost inwards.
    __device__ __forceinline__ double operator()(const double* v, int stride) const {
        double t = __dmul_rn(v[0], w[r]);
        for (int k = r; k >= 1; --k) t = __dadd_rn(t, __dmul_rn(__dadd_rn(v[-k * stride], v[k * stride]), w[r - k]));
        return t;
    }
};

struct MaxOp {
    int r;
    __device__ __forceinline__ double operator()(const double* v, int stride) const {
        double m = -dinf();
        for (int o = -r; o <= r; ++o) m = fmax(m, v[o * stride]);
        return m;
    }
};

struct MinOp {
    int r;
    __device__ __forceinline__ double operator()(const double* v, int stride) const {
        double m = dinf();
        for (int o = -r; o <= r; ++o) m = fmin(m, v[o * stride]);
        return m;
    }
};

template <typename Op>
__global__ void __launch_bounds__(256) k_filter_x(const double* in, int H, int W, int r, Op op, double* out) {
    extern __shared__ double tile[];  // kRowTile + 2r
    const int y = blockIdx.y, x0 = blockIdx.x * kRowTile;
    const double* row = in + (long long)y * W;
    for (int i = threadIdx.x; i < kRowTile + 2 * r; i += blockDim.x)
        tile[i] = row[min(max(x0 - r + i, 0), W - 1)];
    __syncthreads();
    double* orow = out + (long long)y * W;
    for (int i = threadIdx.x; i < kRowTile; i += blockDim.x)
        if (x0 + i < W) orow[x0 + i] = op(tile + r + i, 1);
}

template <typename Op>
__global__ void __launch_bounds__(256) k_filter_y(const double* in, int H, int W, int r, Op op, double* out) {
    extern __shared__ double tile[];  // (kColTile + 2r) x 32
    const int x = blockIdx.x * 32 + (threadIdx.x & 31), y0 = blockIdx.y * kColTile;
    const int rows = kColTile + 2 * r;
    for (int i = threadIdx.x >> 5; i < rows; i += blockDim.x >> 5)
        tile[i * 32 + (threadIdx.x & 31)] = x < W ? in[(long long)min(max(y0 - r + i, 0), H - 1) * W + x] : 0.0;
    __syncthreads();
    if (x >= W) return;
    for (int i = threadIdx.x >> 5; i < kColTile; i += blockDim.x >> 5)
        if (y0 + i < H) out[(long long)(y0 + i) * W + x] = op(tile + (r + i) * 32 + (threadIdx.x & 31), 32);
}

// Direct passes for radii beyond the tiles' halo (nearest edges): out[y][x] from the clamped
// neighbours in global memory, axis 0 when along_y.
__global__ void k_gauss_1d(const double* in, int H, int W, const double* w, int r, int along_y, double* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(i, W, &y, &x);
        auto at = [&](int o) {
            if (along_y) return in[(long long)min(max(y + o, 0), H - 1) * W + x];
            return in[(long long)y * W + min(max(x + o, 0), W - 1)];
        };
        double t = __dmul_rn(at(0), w[r]);
        for (int k = r; k >= 1; --k) t = __dadd_rn(t, __dmul_rn(__dadd_rn(at(-k), at(k)), w[r - k]));
        out[i] = t;
    }
}

// Direct maximum (lowest = false) or minimum (lowest = true) pass.
__global__ void k_max_1d(const double* in, int H, int W, int r, int along_y, bool lowest, double* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(i, W, &y, &x);
        double m = lowest ? dinf() : -dinf();
        for (int o = -r; o <= r; ++o) {
            const double v = along_y ? in[(long long)min(max(y + o, 0), H - 1) * W + x]
                                     : in[(long long)y * W + min(max(x + o, 0), W - 1)];
            m = lowest ? fmin(m, v) : fmax(m, v);
        }
        out[i] = m;
    }
}

template <typename Op>
int filter_pass(const double* in, int H, int W, int r, int along_y, Op op, double* out, cudaStream_t s,
                const char* name) {
    if (along_y) {
        const size_t smem = (size_t)(kColTile + 2 * r) * 32 * sizeof(double);
        if (smem > 48 * 1024) SPX_CUDA(cudaFuncSetAttribute(k_filter_y<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_filter_y<Op><<<dim3((W + 31) / 32, (H + kColTile - 1) / kColTile), 256, smem, s>>>(in, H, W, r, op, out);
    } else {
        const size_t smem = (size_t)(kRowTile + 2 * r) * sizeof(double);
        k_filter_x<Op><<<dim3((W + kRowTile - 1) / kRowTile, H), 256, smem, s>>>(in, H, W, r, op, out);
    }
    return check_launch(name);
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
                int y, x;
                divmod_idx(i, W, &y, &x);
                out[2 * slot] = y;
                out[2 * slot + 1] = x;
            }
        }
    }
}

// mask[i] = flags[labels[i]] (labels >= 0) — per-pixel lookup of a per-label flag.
__global__ void k_label_flags(const int* labels, const uint8_t* flags, long long n, uint8_t* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = labels[i];
        out[i] = l > 0 && flags[l] ? 1 : 0;
    }
}

// One dilation with the 3x3 cross on 0/1 bytes, four per thread (W a multiple of 4, 4-byte
// aligned rows): the word's own bytes shifted by one byte left and right, the words above and
// below, and the edge bytes of the neighbouring words; zero outside the image.
__global__ void k_dilate_cross4(const uint32_t* in, int H, int W4, uint32_t* out) {
    const long long total = (long long)H * W4;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, xw;
        divmod_idx(i, W4, &y, &xw);
        const uint32_t v = in[i];
        uint32_t d = v | (v << 8) | (v >> 8);
        if (y > 0) d |= in[i - W4];
        if (y < H - 1) d |= in[i + W4];
        if (xw > 0) d |= in[i - 1] >> 24;
        if (xw < W4 - 1) d |= in[i + 1] << 24;
        out[i] = d;
    }
}

// One dilation with the 3x3 cross, zero outside the image.
__global__ void k_dilate_cross(const uint8_t* in, int H, int W, uint8_t* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(i, W, &y, &x);
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
    if (radius <= kFilterMaxR && height <= 65535) {
        const GaussOp op{weights, radius};
        if (int e = filter_pass(in, height, width, radius, 1, op, tmp, s, "k_filter_y<gauss>")) return e;
        return filter_pass(tmp, height, width, radius, 0, op, out, s, "k_filter_x<gauss>");
    }
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
    if (radius <= kFilterMaxR && height <= 65535) {
        const MaxOp op{radius};
        if (int e = filter_pass(in, height, width, radius, 1, op, tmp, s, "k_filter_y<max>")) return e;
        return filter_pass(tmp, height, width, radius, 0, op, out, s, "k_filter_x<max>");
    }
    k_max_1d<<<grid_for(n, 256), 256, 0, s>>>(in, height, width, radius, 1, false, tmp);
    if (int e = check_launch("k_max_1d")) return e;
    k_max_1d<<<grid_for(n, 256), 256, 0, s>>>(tmp, height, width, radius, 0, false, out);
    return check_launch("k_max_1d");
}

int spx_minimum_filter(const double* in, int height, int width, int radius, double* tmp, double* out, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && radius >= 0, "bad arguments");
    SPX_REQUIRE(in && tmp && out && tmp != in && tmp != out, "null or aliased pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = (long long)height * width;
    if (radius <= kFilterMaxR && height <= 65535) {
        const MinOp op{radius};
        if (int e = filter_pass(in, height, width, radius, 1, op, tmp, s, "k_filter_y<min>")) return e;
        return filter_pass(tmp, height, width, radius, 0, op, out, s, "k_filter_x<min>");
    }
    k_max_1d<<<grid_for(n, 256), 256, 0, s>>>(in, height, width, radius, 1, true, tmp);
    if (int e = check_launch("k_max_1d")) return e;
    k_max_1d<<<grid_for(n, 256), 256, 0, s>>>(tmp, height, width, radius, 0, true, out);
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
        if (width % 4 == 0 && reinterpret_cast<uintptr_t>(cur) % 4 == 0 && reinterpret_cast<uintptr_t>(nxt) % 4 == 0) {
            k_dilate_cross4<<<grid_for(n / 4, 256), 256, 0, s>>>(reinterpret_cast<const uint32_t*>(cur), height,
                                                                width / 4, reinterpret_cast<uint32_t*>(nxt));
            if (int e = check_launch("k_dilate_cross4")) return e;
        } else {
            k_dilate_cross<<<grid_for(n, 256), 256, 0, s>>>(cur, height, width, nxt);
            if (int e = check_launch("k_dilate_cross")) return e;
        }
        cur = nxt;
    }
    return SPX_OK;
}

}  // extern "C"
