// Shared device helpers and host error plumbing for libsubpx_b200 (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <math.h>

#include "subpx_b200.h"

namespace spx {

// ---------------------------------------------------------------------------------------------
// Host-side error reporting: every C entry point returns an int status and leaves a message that
// spx_last_error() returns (thread-local, like errno).
void set_error(const char* fmt, ...);
int check_launch(const char* what);

// Launch-shape knobs the autotuner sets (process-wide; none of them changes a result).
struct Tuning {
    int fit_warps = 4;          // warps (cells in flight) per block of the LM fit kernels: 2, 4 or 8
    int fit_blocks_per_sm = 8;  // persistent fit blocks per SM: 2..32
    int render_tile = 64;       // model render tile edge: 16, 32 or 64 pixels
    int radial_rays = 2;        // radial profiles, one ray per thread: 0 cached spline window, 2 window read per sample
};
Tuning& tuning();

#define SPX_REQUIRE(cond, ...)                 \
    do {                                       \
        if (!(cond)) {                         \
            ::spx::set_error(__VA_ARGS__);     \
            return SPX_ERR_ARGUMENT;           \
        }                                      \
    } while (0)

#define SPX_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            ::spx::set_error("%s failed: %s", #call, cudaGetErrorString(_e));           \
            return SPX_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

// Carves aligned pieces out of a caller-provided workspace. Used twice per entry point: once with
// a null base to size the workspace, once with the real pointer.
struct Arena {
    char* base;
    size_t used;
    explicit Arena(void* b) : base(static_cast<char*>(b)), used(0) {}
    template <typename T>
    T* take(size_t count) {
        used = (used + 255) & ~size_t(255);
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += count * sizeof(T);
        return p;
    }
};

inline int grid_for(long long n, int block, int cap = 148 * 64) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<int>(g);
}

// ---------------------------------------------------------------------------------------------
// Device helpers.

// Pixel value of an image in its own dtype, converted to double exactly (u8/u16/f32 widen exactly).
__device__ __forceinline__ double load_px(const void* img, int dtype, long long i) {
    switch (dtype) {
        case SPX_U8: return (double)static_cast<const uint8_t*>(img)[i];
        case SPX_U16: return (double)static_cast<const uint16_t*>(img)[i];
        case SPX_F32: return (double)static_cast<const float*>(img)[i];
        default: return static_cast<const double*>(img)[i];
    }
}

// Round-to-nearest arithmetic without FMA contraction: these keep sums and products rounded
// the way NumPy's element-wise operations round them.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// (i / d, i % d) of a non-negative pixel index: 32-bit division when the index fits in 31 bits
// (every image up to 2^31 pixels), 64-bit otherwise.
__device__ __forceinline__ void divmod_idx(long long i, int d, int* q, int* r) {
    if (i <= 0x7fffffffLL) {
        const int ii = (int)i, qq = ii / d;
        *q = qq;
        *r = ii - qq * d;
    } else {
        const long long qq = i / d;
        *q = (int)qq;
        *r = (int)(i - qq * d);
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7ff8000000000000LL); }
__device__ __forceinline__ double dinf() { return __longlong_as_double(0x7ff0000000000000LL); }

// Bitonic sort of n (a power of two, n <= 32 * 32) doubles in shared memory by one warp.
__device__ __forceinline__ void warp_bitonic_sort(double* keys, int n, int lane) {
    for (int len = 2; len <= n; len <<= 1) {
        for (int stride = len >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < n; i += 32) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & len) == 0;
                    const double u = keys[i], v = keys[j];
                    if (up ? u > v : u < v) { keys[i] = v; keys[j] = u; }
                }
            }
            __syncwarp();
        }
    }
}

// NumPy's 'linear' percentile of n sorted values (the rounding of numpy's _lerp).
__device__ __forceinline__ double sorted_percentile(const double* s, int n, double q) {
    if (n <= 0) return 0.0;
    const double virt = __dmul_rn((double)(n - 1), q);
    const double below = floor(virt);
    int lo = (int)below;
    if (lo < 0) lo = 0;
    if (lo > n - 1) lo = n - 1;
    const int hi = lo + 1 < n ? lo + 1 : n - 1;
    if (virt >= (double)(n - 1)) return s[n - 1];
    const double a = s[lo], b = s[hi];
    const double gamma = __dsub_rn(virt, below);
    const double diff = __dsub_rn(b, a);
    if (gamma >= 0.5) return __dsub_rn(b, __dmul_rn(diff, __dsub_rn(1.0, gamma)));
    return __dadd_rn(a, __dmul_rn(diff, gamma));
}

}  // namespace spx
