// Peak seeds for arrays too dense to threshold (measure_cds(seeds="peaks")).
//
// Reference: estimate_pitch and detect_peaks (subpx/_cpu/deblend.py:570-630), reached from
// subpx/cd.py:502-511. The pitch is the first ring of the radially averaged autocorrelation of a
// centred crop (at most max_size^2, mean removed, zero-padded to twice its size); the seeds are the
// maxima of the Gaussian-smoothed signal over a (2 floor(min_distance) + 1)^2 window whose
// prominence over the minimum of a (2 ceil(pitch) + 1)^2 window is positive and at least a fraction
// of the 90th percentile of all maxima's prominences, in row-major order, each moved by the clipped
// vertex of the parabola through its row and column neighbours.
//
// Here: the crop, the radial bins of the autocorrelation and the pick of the ring run as kernels
// (the transforms between them are the caller's FFT); the filters are spx_gaussian_filter /
// spx_maximum_filter / spx_minimum_filter; candidates are compacted per row in row-major order (a
// per-row count, an exclusive scan, a per-row ordered write), so the seed order is the reference's
// np.nonzero order without a sort, and the kept seeds are compacted by a scan of their flags.

#include <algorithm>

#include "common.cuh"
#include "scan.cuh"

namespace spx {
namespace {

constexpr int kRowThreads = 256;

// Sum of a CTA of kRowThreads threads in a fixed order (the same on every thread).
__device__ __forceinline__ double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < kRowThreads / 32; ++k) t += red[k];
    __syncthreads();
    return t;
}

__global__ void k_signal(const void* img, int dtype, double sign, long long n, double* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = sign * load_px(img, dtype, i);
}

// Row sums of the signed crop (one block per crop row, fixed order).
__global__ void __launch_bounds__(kRowThreads) k_crop_rows(const void* img, int dtype, double sign, int W, int y0,
                                                            int x0, int cw, double* rows) {
    __shared__ double red[kRowThreads / 32];
    const long long base = (long long)(y0 + blockIdx.x) * W + x0;
    double acc = 0.0;
    for (int x = threadIdx.x; x < cw; x += kRowThreads) acc += sign * load_px(img, dtype, base + x);
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) rows[blockIdx.x] = acc;
}

// mean = sum(rows) / (ch * cw), one block.
__global__ void __launch_bounds__(kRowThreads) k_crop_mean(const double* rows, int ch, int cw, double* mean) {
    __shared__ double red[kRowThreads / 32];
    double acc = 0.0;
    for (int y = threadIdx.x; y < ch; y += kRowThreads) acc += rows[y];
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) *mean = acc / ((double)ch * (double)cw);
}

// The crop minus its mean in the top-left corner of a zero (2 ch) x (2 cw) array.
__global__ void k_crop_pad(const void* img, int dtype, double sign, int W, int y0, int x0, int ch, int cw,
                           const double* mean, double* out) {
    const int W2 = 2 * cw;
    const long long total = 4LL * ch * cw;
    const double m = *mean;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(i, W2, &y, &x);
        out[i] = (y < ch && x < cw) ? sign * load_px(img, dtype, (long long)(y0 + y) * W + x0 + x) - m : 0.0;
    }
}

// Largest d >= 0 with 4 (d^2 + dy^2) < bound (or -1 if none), bound > 0.
__device__ __forceinline__ int max_dx_below(long long bound, int dy) {
    const long long rest = bound - 4LL * dy * dy;  // need 4 d^2 < rest
    if (rest <= 0) return -1;
    int d = (int)floor(sqrt((double)rest / 4.0));
    while (d > 0 && 4LL * d * d >= rest) --d;
    while (4LL * (d + 1) * (d + 1) < rest) ++d;
    return 4LL * d * d < rest ? d : -1;
}

// Radius bin k of the autocorrelation (period H2 x W2, zero lag at index 0): every lag (dy, dx)
// whose distance rounds to k, i.e. (2k - 1)^2 < 4 (dx^2 + dy^2) < (2k + 1)^2 (sqrt of an integer
// is never a half-integer, so np.rint has no ties here). One block per bin; each thread sums its
// rows' lags in order and the block adds the partial sums in a fixed order.
__global__ void __launch_bounds__(kRowThreads) k_radial_bins(const double* autoc, int H2, int W2, int rmax,
                                                              double* sums, int* counts) {
    __shared__ double red[kRowThreads / 32];
    __shared__ int redi[kRowThreads / 32];
    const int k = blockIdx.x;
    const long long outer = (long long)(2 * k + 1) * (2 * k + 1);       // 4 r^2 < outer
    const long long inner = k ? (long long)(2 * k - 1) * (2 * k - 1) : -1;  // 4 r^2 > inner
    double acc = 0.0;
    int cnt = 0;
    for (int dy = -k + (int)threadIdx.x; dy <= k; dy += kRowThreads) {
        const int hi = max_dx_below(outer, dy);   // |dx| <= hi
        if (hi < 0) continue;
        const int lo = inner < 0 ? 0 : max_dx_below(inner + 1, dy) + 1;  // |dx| >= lo: 4 r^2 >= inner + 1
        const double* row = autoc + (long long)((dy % H2 + H2) % H2) * W2;
        for (int dx = -hi; dx <= hi; ++dx) {
            const int a = dx < 0 ? -dx : dx;
            if (a < lo) {
                dx = lo - 1;  // jump over the hole of the annulus (next dx = lo)
                continue;
            }
            acc += row[(dx % W2 + W2) % W2];
            ++cnt;
        }
    }
    acc = block_sum(acc, red);
    cnt = warp_sum_i(cnt);
    if ((threadIdx.x & 31) == 0) redi[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0;
        for (int w = 0; w < kRowThreads / 32; ++w) c += redi[w];
        sums[k] = acc;
        counts[k] = c;
    }
}

// The first bin k >= 2 whose mean exceeds the previous one, is at least the next one and is
// positive, refined by the parabola through its neighbours; NaN when there is none.
__global__ void k_pitch_pick(const double* sums, const int* counts, int nbins, double* pitch) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    auto prof = [&](int k) { return sums[k] / (double)max(counts[k], 1); };
    double out = dnan();
    for (int k = 2; k < nbins - 1; ++k) {
        const double pm = prof(k - 1), p0 = prof(k), pp = prof(k + 1);
        if (p0 > pm && p0 >= pp && p0 > 0) {
            const double den = pm - 2 * p0 + pp;
            out = (double)k + (den < 0 ? 0.5 * (pm - pp) / den : 0.0);
            break;
        }
    }
    *pitch = out;
}

__device__ __forceinline__ bool is_candidate(const double* smooth, const double* maxf, const double* minf, long long i,
                                             double* prom) {
    const double s = smooth[i];
    *prom = __dsub_rn(s, minf[i]);
    return s == maxf[i] && *prom > 0.0;
}

// Candidates per row (one block per row).
__global__ void __launch_bounds__(kRowThreads) k_candidates_count(const double* smooth, const double* maxf,
                                                                   const double* minf, int W, int* row_counts) {
    __shared__ int red[kRowThreads / 32];
    const long long base = (long long)blockIdx.x * W;
    int cnt = 0;
    for (int x = threadIdx.x; x < W; x += kRowThreads) {
        double p;
        cnt += is_candidate(smooth, maxf, minf, base + x, &p);
    }
    cnt = warp_sum_i(cnt);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0;
        for (int w = 0; w < kRowThreads / 32; ++w) c += red[w];
        row_counts[blockIdx.x] = c;
    }
}

// Candidates of one row written from its offset in increasing x (block-wide ballot prefix per
// chunk of kRowThreads pixels).
__global__ void __launch_bounds__(kRowThreads) k_candidates_write(const double* smooth, const double* maxf,
                                                                   const double* minf, int W, const int* row_offsets,
                                                                   int* out_yx, double* out_prom, int capacity) {
    __shared__ int warp_base[kRowThreads / 32 + 1];
    const int y = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long base = (long long)y * W;
    int offset = row_offsets[y];
    for (int x0 = 0; x0 < W; x0 += kRowThreads) {
        const int x = x0 + threadIdx.x;
        double p = 0.0;
        const bool c = x < W && is_candidate(smooth, maxf, minf, base + x, &p);
        const unsigned bal = __ballot_sync(0xffffffffu, c);
        if (lane == 0) warp_base[warp] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            int run = 0;
            for (int w = 0; w < kRowThreads / 32; ++w) {
                const int v = warp_base[w];
                warp_base[w] = run;
                run += v;
            }
            warp_base[kRowThreads / 32] = run;
        }
        __syncthreads();
        if (c) {
            const int slot = offset + warp_base[warp] + __popc(bal & ((1u << lane) - 1u));
            if (slot < capacity) {
                out_yx[2LL * slot] = y;
                out_yx[2LL * slot + 1] = x;
                out_prom[slot] = p;
            }
        }
        offset += warp_base[kRowThreads / 32];
        __syncthreads();
    }
}

__global__ void k_keep_flags(const double* prom, int n, const double* level, double fraction, int* flags) {
    const double thr = __dmul_rn(fraction, level[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flags[i] = prom[i] >= thr;
}

// Kept candidates at their scanned slots, [x, y] moved by the clipped parabola vertex along each
// axis (zero where a neighbour is outside the image or the curvature is not negative).
__global__ void k_peak_refine(const int* yx, const double* prom, int n, const double* level, double fraction,
                              const int* offsets, const double* smooth, int H, int W, double* out_xy) {
    const double thr = __dmul_rn(fraction, level[0]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!(prom[i] >= thr)) continue;
        const int y = yx[2LL * i], x = yx[2LL * i + 1];
        const double mid = smooth[(long long)y * W + x];
        double sub[2] = {(double)x, (double)y};
        for (int axis = 0; axis < 2; ++axis) {
            const int dy = axis, dx = 1 - axis;
            const bool ok = y - dy >= 0 && y + dy < H && x - dx >= 0 && x + dx < W;
            const double left = smooth[(long long)min(max(y - dy, 0), H - 1) * W + min(max(x - dx, 0), W - 1)];
            const double right = smooth[(long long)min(max(y + dy, 0), H - 1) * W + min(max(x + dx, 0), W - 1)];
            const double curv = __dadd_rn(__dsub_rn(left, __dmul_rn(2.0, mid)), right);
            double delta = 0.0;
            if (ok && curv < 0) delta = __dmul_rn(0.5, __dsub_rn(left, right)) / curv;
            delta = fmin(fmax(delta, -0.5), 0.5);
            sub[axis] = __dadd_rn(sub[axis], delta);
        }
        const int slot = offsets[i];
        out_xy[2LL * slot] = sub[0];
        out_xy[2LL * slot + 1] = sub[1];
    }
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

int spx_signal_image(const void* img, int dtype, double sign, int height, int width, double* out, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && dtype >= SPX_U8 && dtype <= SPX_F64, "bad arguments");
    SPX_REQUIRE(img && out, "null pointer");
    const long long n = (long long)height * width;
    k_signal<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(img, dtype, sign, n, out);
    return check_launch("k_signal");
}

size_t spx_pitch_workspace_bytes(int height, int width, int max_size) {
    const int ch = std::min(height, max_size), cw = std::min(width, max_size);
    Arena a(nullptr);
    a.take<double>(std::max(ch, 1));                 // crop row sums
    a.take<double>(1);                               // mean
    a.take<double>(std::min(ch, cw) / 2 + 1);        // bin sums
    a.take<int>(std::min(ch, cw) / 2 + 1);           // bin counts
    return a.used + 256;
}

int spx_pitch_crop(const void* img, int dtype, double sign, int height, int width, int max_size, double* padded,
                   void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && max_size > 0 && dtype >= SPX_U8 && dtype <= SPX_F64, "bad arguments");
    SPX_REQUIRE(img && padded && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_pitch_workspace_bytes(height, width, max_size), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int ch = std::min(height, max_size), cw = std::min(width, max_size);
    const int y0 = std::max(0, (height - max_size) / 2), x0 = std::max(0, (width - max_size) / 2);
    Arena a(workspace);
    double* rows = a.take<double>(std::max(ch, 1));
    double* mean = a.take<double>(1);
    k_crop_rows<<<ch, kRowThreads, 0, s>>>(img, dtype, sign, width, y0, x0, cw, rows);
    if (int e = check_launch("k_crop_rows")) return e;
    k_crop_mean<<<1, kRowThreads, 0, s>>>(rows, ch, cw, mean);
    if (int e = check_launch("k_crop_mean")) return e;
    k_crop_pad<<<grid_for(4LL * ch * cw, 256), 256, 0, s>>>(img, dtype, sign, width, y0, x0, ch, cw, mean, padded);
    return check_launch("k_crop_pad");
}

int spx_pitch_from_autocorrelation(const double* autoc, int height2, int width2, int r_max, double* pitch,
                                   void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(height2 > 0 && width2 > 0 && r_max >= 0 && 2 * r_max < height2 && 2 * r_max < width2,
                "bad arguments");
    SPX_REQUIRE(autoc && pitch && workspace, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena a(workspace);
    a.take<double>(std::max(height2 / 2, 1));
    a.take<double>(1);
    double* sums = a.take<double>(r_max + 1);
    int* counts = a.take<int>(r_max + 1);
    SPX_REQUIRE(workspace_bytes >= a.used, "workspace too small");
    k_radial_bins<<<r_max + 1, kRowThreads, 0, s>>>(autoc, height2, width2, r_max, sums, counts);
    if (int e = check_launch("k_radial_bins")) return e;
    k_pitch_pick<<<1, 32, 0, s>>>(sums, counts, r_max + 1, pitch);
    return check_launch("k_pitch_pick");
}

size_t spx_peak_workspace_bytes(int height, int width) {
    Arena a(nullptr);
    a.take<int>(std::max(height, 1));
    a.take<int>(scan_scratch_ints(std::max(height, 1)));
    return a.used + 256;
}

int spx_peak_candidates(const double* smooth, const double* maxf, const double* minf, int height, int width,
                        int* out_yx, double* out_prom, int capacity, int* count, void* workspace,
                        size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && capacity >= 0, "bad arguments");
    SPX_REQUIRE(smooth && maxf && minf && count && workspace && ((out_yx && out_prom) || capacity == 0),
                "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_peak_workspace_bytes(height, width), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena a(workspace);
    int* rows = a.take<int>(height);
    int* scratch = a.take<int>(scan_scratch_ints(height));
    k_candidates_count<<<height, kRowThreads, 0, s>>>(smooth, maxf, minf, width, rows);
    if (int e = check_launch("k_candidates_count")) return e;
    if (int e = exclusive_scan(rows, height, rows, count, scratch, s)) return e;
    k_candidates_write<<<height, kRowThreads, 0, s>>>(smooth, maxf, minf, width, rows, out_yx, out_prom, capacity);
    return check_launch("k_candidates_write");
}

size_t spx_peak_select_workspace_bytes(int n) {
    Arena a(nullptr);
    a.take<int>(std::max(n, 1));
    a.take<int>(scan_scratch_ints(std::max(n, 1)));
    return a.used + 256;
}

int spx_peak_select(const int* yx, const double* prom, int n, const double* level, double fraction,
                    const double* smooth, int height, int width, double* out_xy, int* count, void* workspace,
                    size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && height > 0 && width > 0, "bad arguments");
    SPX_REQUIRE(count && workspace && (n == 0 || (yx && prom && level && smooth && out_xy)), "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_peak_select_workspace_bytes(n), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        SPX_CUDA(cudaMemsetAsync(count, 0, sizeof(int), s));
        return SPX_OK;
    }
    Arena a(workspace);
    int* flags = a.take<int>(n);
    int* scratch = a.take<int>(scan_scratch_ints(n));
    k_keep_flags<<<grid_for(n, 256), 256, 0, s>>>(prom, n, level, fraction, flags);
    if (int e = check_launch("k_keep_flags")) return e;
    if (int e = exclusive_scan(flags, n, flags, count, scratch, s)) return e;
    k_peak_refine<<<grid_for(n, 256), 256, 0, s>>>(yx, prom, n, level, fraction, flags, smooth, height, width, out_xy);
    return check_launch("k_peak_refine");
}

}  // extern "C"
