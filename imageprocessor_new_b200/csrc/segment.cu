// Segmentation: Otsu threshold, binarisation and connected-component labelling with stats.
//
// Replaces, for the subpx hot path:
//   cv2.threshold(..., THRESH_OTSU)            subpx/_cpu/centers.py:247-266, subpx/_gpu/centers.py:1789-1796
//   cv2.connectedComponentsWithStats           subpx/_cpu/components.py:18-32
//
// Otsu: a shared-memory histogram over the occupied value range, then OpenCV's published Otsu scan
// (between-class variance q1*q2*(mu1-mu2)^2, first maximum, bins skipped while min(q1,q2) <
// FLT_EPSILON). The scan's running sums are rounded sequentially by one thread so that the chosen
// bin is the one OpenCV chooses.
//
// CCL: union-find in two levels. Parents live in a canonical-order array: for 8-connectivity the
// pixels of each 2x2 block are contiguous and blocks follow the row-pair scan, for 4-connectivity
// canonical order is raster order. Unions always link the larger id under the smaller, so the root
// of a component is its first pixel in that order, and OpenCV's label numbering is the rank of the
// root among all roots: a bitmap of roots plus a prefix count of its words.
//   k_local_ccl     one CTA per 32x64 tile: binarise, union-find in shared memory, write parents
//   k_border_merge  unions across tile borders in global memory (lock-free atomicMin linking)
//   scan            popcount prefix of the root bitmap -> component count K
//   k_finish        final raster labels (rank of the root) + stats by warp run-length aggregation

#include "common.cuh"

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace spx {

static thread_local char g_error[1024];
static unsigned long long g_launches = 0;  // kernel launches issued by this library (all threads)

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

Tuning& tuning() {
    static Tuning t;
    return t;
}

int check_launch(const char* what) {
    __atomic_add_fetch(&g_launches, 1ull, __ATOMIC_RELAXED);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s launch failed: %s", what, cudaGetErrorString(e));
        return SPX_ERR_CUDA;
    }
    return SPX_OK;
}

namespace {

constexpr int kHistSmemBins = 16384;  // value ranges up to this use a shared-memory histogram
constexpr int kTileH = 32;            // CCL tile (even height keeps 2x2 blocks inside one tile)
constexpr int kTileW = 64;
constexpr int kTilePx = kTileH * kTileW;

// ------------------------------------------------------------------------------------------ Otsu

__device__ __forceinline__ unsigned int px_u(const void* img, int dtype, long long i) {
    return dtype == SPX_U8 ? (unsigned int)static_cast<const uint8_t*>(img)[i]
                           : (unsigned int)static_cast<const uint16_t*>(img)[i];
}

// range[0] = min, range[1] = max of the sampled pixels (range must be preset to {~0u, 0}).
__global__ void k_minmax(const void* img, int dtype, int height, int width, int step,
                         unsigned int* range) {
    const int hs = (int)(((long long)height + step - 1) / step), ws = (int)(((long long)width + step - 1) / step);
    const long long n = (long long)hs * ws;
    unsigned int lo = 0xffffffffu, hi = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        int yi, xi;
        divmod_idx(k, ws, &yi, &xi);
        const long long y = yi, x = xi;
        const unsigned int v = px_u(img, dtype, y * step * (long long)width + x * step);
        lo = min(lo, v);
        hi = max(hi, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&range[0], lo);
        atomicMax(&range[1], hi);
    }
}

// k_minmax for a contiguous, 16-byte aligned uint16 image: eight pixels per 16-byte load.
__global__ void k_minmax_dense(const uint16_t* img, long long n, unsigned int* range) {
    unsigned int lo = 0xffffffffu, hi = 0;
    const uint4* v4 = reinterpret_cast<const uint4*>(img);
    const long long n8 = n / 8;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n8;
         k += (long long)gridDim.x * blockDim.x) {
        const uint4 q = __ldg(v4 + k);
        const unsigned int w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const unsigned int a = w[j] & 0xffffu, b = w[j] >> 16;
            lo = min(lo, min(a, b));
            hi = max(hi, max(a, b));
        }
    }
    for (long long k = n8 * 8 + blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const unsigned int v = img[k];
        lo = min(lo, v);
        hi = max(hi, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&range[0], lo);
        atomicMax(&range[1], hi);
    }
}

// Histogram of the sampled pixels into hist[65536] (pre-zeroed, u32).
__global__ void k_histogram(const void* img, int dtype, int height, int width, int step,
                            int dense, const unsigned int* range, unsigned int* hist) {
    extern __shared__ unsigned int sh[];
    const unsigned int lo = range[0], hi = range[1];
    const unsigned int nb = hi >= lo ? hi - lo + 1 : 0;
    const bool in_smem = nb <= (unsigned int)kHistSmemBins;
    if (in_smem) {
        for (unsigned int i = threadIdx.x; i < nb; i += blockDim.x) sh[i] = 0;
        __syncthreads();
    }
    const int hs = (int)(((long long)height + step - 1) / step), ws = (int)(((long long)width + step - 1) / step);
    const long long n = (long long)hs * ws;
    if (dense) {
        // 16-byte loads of 8 pixels, then the ragged tail.
        const uint4* v4 = static_cast<const uint4*>(img);
        const long long n8 = n / 8;
        for (long long k = n8 * 8 + blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
             k += (long long)gridDim.x * blockDim.x) {
            const unsigned int v = static_cast<const uint16_t*>(img)[k];
            if (in_smem) atomicAdd(&sh[v - lo], 1u);
            else atomicAdd(&hist[v], 1u);
        }
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n8;
             k += (long long)gridDim.x * blockDim.x) {
            const uint4 q = __ldg(v4 + k);
            const unsigned int w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const unsigned int a = w[j] & 0xffffu, b = w[j] >> 16;
                if (in_smem) {
                    atomicAdd(&sh[a - lo], 1u);
                    atomicAdd(&sh[b - lo], 1u);
                } else {
                    atomicAdd(&hist[a], 1u);
                    atomicAdd(&hist[b], 1u);
                }
            }
        }
    } else {
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
             k += (long long)gridDim.x * blockDim.x) {
            int yi, xi;
        divmod_idx(k, ws, &yi, &xi);
        const long long y = yi, x = xi;
            const unsigned int v = px_u(img, dtype, y * step * (long long)width + x * step);
            if (in_smem) atomicAdd(&sh[v - lo], 1u);
            else atomicAdd(&hist[v], 1u);
        }
    }
    if (in_smem) {
        __syncthreads();
        for (unsigned int i = threadIdx.x; i < nb; i += blockDim.x)
            if (sh[i]) atomicAdd(&hist[lo + i], sh[i]);
    }
}

// Certified parallel Otsu: the bin that OpenCV's sequential FP64 scan chooses, found without the
// scan whenever the exact rational between-class variances single it out.
//
// For bin i with integer prefix sums Q = sum_{j<=i} h_j and S = sum_{j<=i} j h_j (N pixels, grey
// sum M), the exact variance is sigma2 = (S N - Q M)^2 / (N^2 Q (N - Q)), and mu1 - mu2 =
// (S N - Q M) / (Q (N - Q)). OpenCV's loop computes q1 as a running FP64 sum of h_j / N (relative
// error <= (n + 2) u for n bins, u = 2^-53), mu1 by a recurrence whose product mu1 q1 is a running
// sum of j h_j / N (relative error <= 4 (n + 2) u), mu2 = (mu - q1 mu1) / q2 and sigma2 = q1 q2
// (mu1 - mu2)^2. From these error terms every bin gets an interval [lo, hi] that holds OpenCV's
// rounded sigma2 (each term inflated four times), and the skip test min(q1, q2) < FLT_EPSILON is
// decided on the exact q1 = Q / N unless q1 or q2 lies within 1e-9 of FLT_EPSILON or of
// 1 - FLT_EPSILON (a bin that might go either way). When the bin i* with the largest lo among the
// surely unskipped bins has lo > 0 and lo above every other not-surely-skipped bin's hi, OpenCV's
// strict-maximum scan must choose i*: returns true with the threshold. Otherwise (near-ties,
// ambiguous skips) returns false and the caller runs the sequential scan. Block-uniform result;
// needs blockDim.x == 1024.
__device__ bool otsu_certified(const unsigned int* hist, int first, int n, long long total,
                               unsigned long long grey_sum, double* threshold) {
    constexpr int T = 1024;
    __shared__ unsigned long long s_q[T], s_m[T];
    __shared__ double s_val[32];
    __shared__ int s_idx[32];
    __shared__ double s_best_lo;
    __shared__ int s_best;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (n + T - 1) / T, b0 = min(n, t * per), b1 = min(n, b0 + per);
    unsigned long long cq = 0, cm = 0;
    for (int k = b0; k < b1; ++k) {
        const unsigned long long h = hist[first + k];
        cq += h;
        cm += h * (unsigned long long)(first + k);
    }
    s_q[t] = cq;
    s_m[t] = cm;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {  // inclusive scan of the chunk totals
        const unsigned long long aq = t >= o ? s_q[t - o] : 0ull, am = t >= o ? s_m[t - o] : 0ull;
        __syncthreads();
        s_q[t] += aq;
        s_m[t] += am;
        __syncthreads();
    }
    const unsigned long long q_start = s_q[t] - cq, m_start = s_m[t] - cm;
    const double Nd = (double)total, invN = 1.0 / Nd;
    const double u = 1.1102230246251565e-16;
    const double eps = 1.1920928955078125e-07, win = 1e-9;
    const double g = (double)(n + 2) * u;
    const double mu = (double)grey_sum * invN;
    // cls: 0 surely skipped, 1 surely unskipped, 2 either. lo / hi: the interval of OpenCV's sigma2.
    auto eval = [&](unsigned long long Q, unsigned long long S, double* lo, double* hi) -> int {
        const unsigned long long R = (unsigned long long)total - Q;
        const double q1 = (double)Q * invN, q2 = (double)R * invN;
        const bool amb = fabs(q1 - eps) <= win || fabs(q2 - eps) <= win || fabs(q1 - (1.0 - eps)) <= win ||
                         fabs(q2 - (1.0 - eps)) <= win;
        const bool skip = fmin(q1, q2) < eps || fmax(q1, q2) > 1.0 - eps;
        if (skip && !amb) return 0;
        if (Q == 0 || R == 0) {  // q1 or q2 exactly 0 cannot be unskipped (amb never holds here)
            *lo = *hi = 0.0;
            return 0;
        }
        const __int128 D = (__int128)S * (__int128)total - (__int128)Q * (__int128)grey_sum;
        const double qr = (double)Q * (double)R;
        const double d = (double)D / qr;                  // mu1 - mu2
        const double ad = fabs(d);
        const double mu1 = (double)S / (double)Q;
        const double mu2 = (double)(grey_sum - S) / (double)R;
        const double rel_q1 = 4.0 * g;
        const double rel_q2 = 4.0 * (g * q1 + u) / q2;
        const double num = q2 * mu2;                      // mu - q1 mu1, > 0 here
        const double rel_mu2 = (5.0 * g + u) * mu / fmax(num, 1e-300) + (g * q1 + u) / q2 + u;
        const double err_d = 4.0 * (4.0 * g * mu1 + mu2 * rel_mu2 + u * ad);
        const double base = q1 * q2;
        *hi = base * (1.0 + rel_q1) * (1.0 + rel_q2) * (ad + err_d) * (ad + err_d) * (1.0 + 16.0 * u);
        const double dl = fmax(ad - err_d, 0.0);
        *lo = rel_q2 >= 1.0 ? 0.0 : base * (1.0 - rel_q1) * (1.0 - rel_q2) * dl * dl * (1.0 - 16.0 * u);
        return amb ? 2 : 1;
    };
    // Pass 1: the surely unskipped bin with the largest lower bound (lowest index on ties).
    double best_lo = -1.0;
    int best = 0x7fffffff;
    {
        unsigned long long Q = q_start, S = m_start;
        for (int k = b0; k < b1; ++k) {
            const unsigned long long h = hist[first + k];
            Q += h;
            S += h * (unsigned long long)(first + k);
            double lo, hi;
            if (eval(Q, S, &lo, &hi) == 1 && lo > best_lo) {
                best_lo = lo;
                best = k;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best_lo, o);
        const int oi = __shfl_xor_sync(0xffffffffu, best, o);
        if (ov > best_lo || (ov == best_lo && oi < best)) { best_lo = ov; best = oi; }
    }
    if (lane == 0) { s_val[warp] = best_lo; s_idx[warp] = best; }
    __syncthreads();
    if (t == 0) {
        double v = -1.0;
        int i = 0x7fffffff;
        for (int w = 0; w < T / 32; ++w)
            if (s_val[w] > v || (s_val[w] == v && s_idx[w] < i)) { v = s_val[w]; i = s_idx[w]; }
        s_best_lo = v;
        s_best = i;
    }
    __syncthreads();
    const double star_lo = s_best_lo;
    const int star = s_best;
    // Pass 2: the largest upper bound of every other bin that may be unskipped.
    double other_hi = 0.0;
    {
        unsigned long long Q = q_start, S = m_start;
        for (int k = b0; k < b1; ++k) {
            const unsigned long long h = hist[first + k];
            Q += h;
            S += h * (unsigned long long)(first + k);
            double lo, hi;
            if (k != star && eval(Q, S, &lo, &hi) != 0) other_hi = fmax(other_hi, hi);
        }
    }
    other_hi = warp_max(other_hi);
    __syncthreads();  // s_val is reused
    if (lane == 0) s_val[warp] = other_hi;
    __syncthreads();
    double top = 0.0;
    for (int w = 0; w < T / 32; ++w) top = fmax(top, s_val[w]);
    const bool ok = star != 0x7fffffff && star_lo > 0.0 && star_lo > top;
    if (ok && t == 0) *threshold = (double)(first + star);
    return ok;
}

// OpenCV's Otsu scan (getThreshVal_Otsu) over bins [0, N), by one block in four phases:
//   A  p_i = h[i] * scale (parallel), then q1_i = q1_{i-1} + p_i by one thread (additions only);
//   B  y_i = RN(1 / q1_i) (parallel);
//   C  the mu1 recurrence by one thread: mu1 <- mu1 * q1_{i-1}; unless bin i is skipped,
//      mu1 <- RN((mu1 + i p_i) / q1_i), the quotient by Markstein's correction
//      (q = RN(a y); r = a - q q1 exactly by FMA; RN(q + r y) = RN(a / q1) when y = RN(1 / q1));
//   D  sigma_i = q1 q2 (mu1 - mu2)^2 for every unskipped bin and the first maximum (parallel).
// Every value is rounded exactly as OpenCV's sequential loop rounds it, so the chosen bin is OpenCV's.
__global__ void __launch_bounds__(1024) k_otsu_scan(const unsigned int* hist, int nbins,
                                                    const unsigned int* range, long long total,
                                                    double* p_buf, double* q1_buf, double* y_buf,
                                                    double* mu1_buf, double* threshold) {
    __shared__ unsigned long long s_mu[32];
    __shared__ double s_best[32];
    __shared__ int s_arg[32];
    unsigned long long mu_part = 0;
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) mu_part += (unsigned long long)i * hist[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mu_part += __shfl_xor_sync(0xffffffffu, mu_part, o);
    if ((threadIdx.x & 31) == 0) s_mu[threadIdx.x >> 5] = mu_part;
    const double scale = 1.0 / (double)total;
    int first = (int)range[0], last = (int)range[1];
    if (first < 0) first = 0;
    if (last > nbins - 1) last = nbins - 1;
    const int n = last - first + 1;
    // Bins below the first occupied one leave mu1 = q1 = 0 and are all skipped; bins above the last
    // occupied one have q2 < FLT_EPSILON and are skipped as well.
    for (int k = threadIdx.x; k < n; k += blockDim.x) p_buf[k] = __dmul_rn((double)hist[first + k], scale);
    __syncthreads();
    unsigned long long mu_int = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mu_int += s_mu[w];
    if (n > 0 && otsu_certified(hist, first, n, total, mu_int, threshold)) return;
    // The reference sums i*h[i] sequentially in double: every partial sum is an integer below 2^53,
    // hence exact, and equal to this integer sum.
    const double mu = __dmul_rn((double)mu_int, scale);
    // The sequential loops below load eight bins ahead, so the loads are not on the recurrence's
    // critical path.
    constexpr int kAhead = 8;
    if (threadIdx.x == 0) {
        double q1 = 0.0;
        for (int k0 = 0; k0 < n; k0 += kAhead) {
            double pb[kAhead];
#pragma unroll
            for (int j = 0; j < kAhead; ++j) pb[j] = k0 + j < n ? p_buf[k0 + j] : 0.0;
#pragma unroll
            for (int j = 0; j < kAhead; ++j) {
                q1 = __dadd_rn(q1, pb[j]);
                if (k0 + j < n) q1_buf[k0 + j] = q1;
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) y_buf[k] = __drcp_rn(q1_buf[k]);
    __syncthreads();
    const double eps = (double)1.1920928955078125e-07f;
    const double one_minus_eps = __dsub_rn(1.0, eps);
    if (threadIdx.x == 0) {
        double mu1 = 0.0, q1_prev = 0.0;
        for (int k0 = 0; k0 < n; k0 += kAhead) {
            double qb[kAhead], pb[kAhead], yb[kAhead];
#pragma unroll
            for (int j = 0; j < kAhead; ++j) {
                const bool in = k0 + j < n;
                qb[j] = in ? q1_buf[k0 + j] : 0.0;
                pb[j] = in ? p_buf[k0 + j] : 0.0;
                yb[j] = in ? y_buf[k0 + j] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < kAhead; ++j) {
                const int k = k0 + j;
                if (k >= n) break;
                const double q1 = qb[j], p_i = pb[j];
                mu1 = __dmul_rn(mu1, q1_prev);
                q1_prev = q1;
                const double q2 = __dsub_rn(1.0, q1);
                if (fmin(q1, q2) < eps || fmax(q1, q2) > one_minus_eps) {
                    mu1_buf[k] = dnan();
                    continue;
                }
                const double a = __dadd_rn(mu1, __dmul_rn((double)(first + k), p_i));
                const double y = yb[j];
                const double q = __dmul_rn(a, y);
                const double r = __fma_rn(-q, q1, a);
                mu1 = __fma_rn(r, y, q);
                mu1_buf[k] = mu1;
            }
        }
    }
    __syncthreads();
    double best = 0.0;
    int arg = 0x7fffffff;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double mu1 = mu1_buf[k];
        if (isnan(mu1)) continue;
        const double q1 = q1_buf[k], q2 = __dsub_rn(1.0, q1);
        const double mu2 = __ddiv_rn(__dsub_rn(mu, __dmul_rn(q1, mu1)), q2);
        const double d = __dsub_rn(mu1, mu2);
        const double sigma = __dmul_rn(__dmul_rn(__dmul_rn(q1, q2), d), d);
        // First maximum strictly above 0 (OpenCV starts from max_sigma = 0, bin 0).
        if (sigma > best) { best = sigma; arg = k; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oa = __shfl_xor_sync(0xffffffffu, arg, o);
        if (ob > best || (ob == best && oa < arg)) { best = ob; arg = oa; }
    }
    if ((threadIdx.x & 31) == 0) { s_best[threadIdx.x >> 5] = best; s_arg[threadIdx.x >> 5] = arg; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        int a = 0x7fffffff;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (s_best[w] > b || (s_best[w] == b && s_arg[w] < a)) { b = s_best[w]; a = s_arg[w]; }
        *threshold = (b > 0.0 && a != 0x7fffffff) ? (double)(first + a) : 0.0;
    }
}

// OpenCV's triangle threshold (getThreshVal_Triangle_8u) over a 256-bin histogram: the bin of
// maximum distance to the line from the histogram peak to the far end of the occupied range.
__global__ void k_triangle_scan(const unsigned int* hist, double* threshold) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int N = 256;
    long long h[256];
    for (int i = 0; i < N; ++i) h[i] = hist[i];
    int left = 0, right = 0, max_ind = 0;
    long long mx = 0;
    for (int i = 0; i < N; ++i)
        if (h[i] > 0) { left = i; break; }
    if (left > 0) left--;
    for (int i = N - 1; i > 0; --i)
        if (h[i] > 0) { right = i; break; }
    if (right < N - 1) right++;
    for (int i = 0; i < N; ++i)
        if (h[i] > mx) { mx = h[i]; max_ind = i; }
    bool flipped = false;
    if (max_ind - left < right - max_ind) {
        flipped = true;
        for (int i = 0, j = N - 1; i < j; ++i, --j) { const long long t = h[i]; h[i] = h[j]; h[j] = t; }
        left = N - 1 - right;
        max_ind = N - 1 - max_ind;
    }
    double thresh = left, dist = 0.0;
    const double a = (double)mx, b = (double)(left - max_ind);
    for (int i = left + 1; i <= max_ind; ++i) {
        const double d = __dadd_rn(__dmul_rn(a, (double)i), __dmul_rn(b, (double)h[i]));
        if (d > dist) { dist = d; thresh = i; }
    }
    thresh -= 1.0;
    if (flipped) thresh = (N - 1) - thresh;
    *threshold = thresh;
}

// -------------------------------------------------------------------------------------------- CCL

struct Geo {
    int H, W, Wb;   // image size; blocks per row pair (8-connectivity)
    int conn;       // 8 or 4
    __device__ __forceinline__ int canon(int y, int x) const {
        return conn == 8 ? ((((y >> 1) * Wb + (x >> 1)) << 2) | ((y & 1) << 1) | (x & 1)) : y * W + x;
    }
    // Foreground bitmap: bit x & 31 of word y * words_per_row + x / 32 (rows padded to 64 bits).
    // Only local roots and foreground pixels on tile edges have an entry in the parents array;
    // readers test the bitmap first.
    __device__ __forceinline__ int words_per_row() const { return (W + 63) / 64 * 2; }
    __device__ __forceinline__ bool fg(const unsigned* bits, int y, int x) const {
        return (bits[(long long)y * words_per_row() + (x >> 5)] >> (x & 31)) & 1u;
    }
};

__device__ __forceinline__ bool is_fg(double v, double t, int invert) { return invert ? v <= t : v > t; }

// Root of a, halving the path on the way (each visited node is re-pointed to its grandparent, an
// ancestor, so concurrent finds and unions stay valid).
__device__ __forceinline__ int find_root_volatile(volatile int* p, int a) {
    while (true) {
        const int b = p[a];
        if (b == a) return a;
        const int c = p[b];
        if (c == b) return b;
        p[a] = c;
        a = c;
    }
}

// Root of a without writing: safe to run while other threads overwrite entries with their roots.
__device__ __forceinline__ int find_root_readonly(const volatile int* p, int a) {
    int b = p[a];
    while (b != a) {
        a = b;
        b = p[a];
    }
    return a;
}

// Lock-free union (link the larger root under the smaller with atomicMin; retry from the value
// that was there when another thread won the race). Clears the root bit of a root that gets linked.
__device__ void unite(int* p, int a, int b, unsigned int* roots) {
    while (true) {
        a = find_root_volatile(p, a);
        b = find_root_volatile(p, b);
        if (a == b) return;
        if (a < b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicMin(&p[a], b);
        if (old == a) {
            if (roots) atomicAnd(&roots[a >> 5], ~(1u << (a & 31)));
            return;
        }
        a = old;
    }
}

// ---------------------------------------------------------------------- run-based tile union-find
//
// A 32 x 64 tile is 32 row masks (bit x of mask[r] = pixel (ty0 + r, tx0 + x) is foreground). The
// union-find runs over the row runs: a run's node is its first pixel, which has the smallest
// canonical id of the run (canonical order increases with x inside a row), so the root of every
// local component is its smallest canonical id, as in a pixel-level union by minimum. Each of 32
// threads takes one row and unites every run with the runs of the row above that touch it (their
// columns overlap, widened by one for 8-connectivity). Both CCL kernels rebuild the same tile
// forest from the bitmap; the result does not depend on the order of the unions.

constexpr int kCclThreads = 128;

__device__ __forceinline__ int tile_lidx(int conn, int yl, int xl) {
    return conn == 8 ? ((((yl >> 1) * (kTileW / 2) + (xl >> 1)) << 2) | ((yl & 1) << 1) | (xl & 1))
                     : yl * kTileW + xl;
}

// First column of the run of set bits of m that holds bit x.
__device__ __forceinline__ int run_first(unsigned long long m, int x) {
    const unsigned long long below = ~m & ((1ull << x) - 1ull);
    return below ? 64 - __clzll((long long)below) : 0;
}

// Last column of the run of set bits of m that holds bit x.
__device__ __forceinline__ int run_last(unsigned long long m, int x) {
    const unsigned long long above = ~m & ~((1ull << x) - 1ull);
    return above ? __ffsll((long long)above) - 2 : 63;
}

// Builds the tile forest in par[] (indexed by local canonical id; only run nodes are written) from
// mask[0..31] and leaves every run node pointing at its root. Called by all threads of the block.
__device__ void tile_forest(const unsigned long long* mask, int conn, int* par) {
    const int r = threadIdx.x;
    if (r < kTileH) {
        const unsigned long long m = mask[r];
        for (unsigned long long s = m & ~(m << 1); s; s &= s - 1) {
            const int a = __ffsll((long long)s) - 1;
            par[tile_lidx(conn, r, a)] = tile_lidx(conn, r, a);
        }
    }
    __syncthreads();
    if (r > 0 && r < kTileH) {
        const unsigned long long m = mask[r], mp = mask[r - 1];
        for (unsigned long long s = m & ~(m << 1); s && mp; s &= s - 1) {
            const int a = __ffsll((long long)s) - 1, b = run_last(m, a);
            const int lo = conn == 8 ? max(a - 1, 0) : a, hi = conn == 8 ? min(b + 1, 63) : b;
            unsigned long long touch = mp & ((2ull << hi) - 1ull) & ~((1ull << lo) - 1ull);
            const int me = tile_lidx(conn, r, a);
            while (touch) {
                const int c = __ffsll((long long)touch) - 1;
                unite(par, me, tile_lidx(conn, r - 1, run_first(mp, c)), nullptr);
                const int e = run_last(mp, c);
                touch = e >= 63 ? 0ull : touch & ~((2ull << e) - 1ull);
            }
        }
    }
    __syncthreads();
    // Point every run node at its root. The finds do not write (a path-halving find could put an
    // intermediate node back over an entry its owner has already set to the root); each entry is
    // written only by its own thread, with a value that is an ancestor of every value it had.
    if (r < kTileH) {
        const unsigned long long m = mask[r];
        for (unsigned long long s = m & ~(m << 1); s; s &= s - 1) {
            const int l = tile_lidx(conn, r, __ffsll((long long)s) - 1);
            par[l] = find_root_readonly(par, l);
        }
    }
    __syncthreads();
}

// Global canonical id of local canonical id l of the tile at (ty0, tx0).
__device__ __forceinline__ int tile_gid(const Geo& g, int ty0, int tx0, int l) {
    int ry, rx;
    if (g.conn == 8) {
        const int b = l >> 2;
        ry = (b / (kTileW / 2)) * 2 + ((l >> 1) & 1);
        rx = (b % (kTileW / 2)) * 2 + (l & 1);
    } else {
        ry = l / kTileW;
        rx = l % kTileW;
    }
    return g.canon(ty0 + ry, tx0 + rx);
}

// Binarises one 32 x 64 tile into the foreground bitmap and builds its forest. Writes parents only
// where the border merge reads them: each local root points at itself (and gets its root bit) and
// each foreground pixel on the tile's four edges points at its local root.
__global__ void __launch_bounds__(kCclThreads) k_local_ccl(const void* img, int dtype, Geo g,
                                                           const double* thr_dev, double thr_fixed,
                                                           int invert, int* parents, unsigned int* roots,
                                                           unsigned int* fgbits) {
    __shared__ int par[kTilePx];
    __shared__ unsigned int words[kTileH * 2];
    __shared__ unsigned long long mask[kTileH];
    const int tx0 = blockIdx.x * kTileW, ty0 = blockIdx.y * kTileH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double t = thr_dev ? *thr_dev : thr_fixed;
    // Half-rows of 32 pixels: one warp-wide ballot each.
    for (int hr = warp; hr < kTileH * 2; hr += kCclThreads / 32) {
        const int y = ty0 + (hr >> 1), x = tx0 + (hr & 1) * 32 + lane;
        bool f = false;
        if (y < g.H && x < g.W) f = is_fg(load_px(img, dtype, (long long)y * g.W + x), t, invert);
        const unsigned w = __ballot_sync(0xffffffffu, f);
        if (lane == 0) {
            words[hr] = w;
            if (y < g.H) fgbits[(long long)y * g.words_per_row() + (x >> 5)] = w;
        }
    }
    __syncthreads();
    if (threadIdx.x < kTileH)
        mask[threadIdx.x] = (unsigned long long)words[2 * threadIdx.x] |
                            ((unsigned long long)words[2 * threadIdx.x + 1] << 32);
    __syncthreads();
    tile_forest(mask, g.conn, par);
    if (threadIdx.x < kTileH) {
        const int r = threadIdx.x, y = ty0 + r;
        const unsigned long long m = mask[r];
        for (unsigned long long s = m & ~(m << 1); s; s &= s - 1) {
            const int l = tile_lidx(g.conn, r, __ffsll((long long)s) - 1);
            if (par[l] == l) {
                const int gid = tile_gid(g, ty0, tx0, l);
                parents[gid] = gid;
                atomicOr(&roots[gid >> 5], 1u << (gid & 31));
            }
        }
        // Left and right edge pixels of this row.
        if (m & 1ull) parents[g.canon(y, tx0)] = tile_gid(g, ty0, tx0, par[tile_lidx(g.conn, r, 0)]);
        if (m >> 63)
            parents[g.canon(y, tx0 + 63)] =
                tile_gid(g, ty0, tx0, par[tile_lidx(g.conn, r, run_first(m, 63))]);
    }
    // Top and bottom rows: one warp each, lanes over the 64 columns.
    if (warp < 2) {
        const int r = warp == 0 ? 0 : kTileH - 1;
        const unsigned long long m = mask[r];
        for (int x = lane; x < kTileW; x += 32)
            if ((m >> x) & 1ull)
                parents[g.canon(ty0 + r, tx0 + x)] =
                    tile_gid(g, ty0, tx0, par[tile_lidx(g.conn, r, run_first(m, x))]);
    }
}

// Unions across tile borders. One thread per border pixel of a tile: top row (neighbours above),
// left column (neighbours to the left), right column (the up-right neighbour in the next tile).
__global__ void k_border_merge(Geo g, int* parents, unsigned int* roots, const unsigned int* fgbits, int tiles_x,
                               int tiles_y) {
    const int per_tile = kTileW + 2 * kTileH;
    const long long total = (long long)tiles_x * tiles_y * per_tile;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        int tile, e;
        divmod_idx(k, per_tile, &tile, &e);
        const int tx0 = (tile % tiles_x) * kTileW, ty0 = (tile / tiles_x) * kTileH;
        int y, x;
        if (e < kTileW) { y = ty0; x = tx0 + e; }
        else if (e < kTileW + kTileH) { y = ty0 + (e - kTileW); x = tx0; }
        else { y = ty0 + (e - kTileW - kTileH); x = tx0 + kTileW - 1; }
        if (y >= g.H || x >= g.W) continue;
        if (!g.fg(fgbits, y, x)) continue;
        const int me = g.canon(y, x);
        auto link = [&](int yy, int xx) {
            if (yy < 0 || xx < 0 || xx >= g.W) return;
            // Only neighbours in another tile.
            if (yy >= ty0 && xx >= tx0 && xx < tx0 + kTileW) return;
            if (!g.fg(fgbits, yy, xx)) return;
            unite(parents, me, g.canon(yy, xx), roots);
        };
        if (e < kTileW) {  // top row: (y-1, x) and, for 8-connectivity, (y-1, x-1), (y-1, x+1)
            link(y - 1, x);
            if (g.conn == 8) { link(y - 1, x - 1); link(y - 1, x + 1); }
        } else if (e < kTileW + kTileH) {  // left column: (y, x-1) and (y-1, x-1)
            link(y, x - 1);
            if (g.conn == 8) link(y - 1, x - 1);
        } else {  // right column: (y-1, x+1) lies in the tile to the right (or up-right)
            if (g.conn == 8) link(y - 1, x + 1);
        }
    }
}

// ---------------------------------------------------------------------------- prefix of popcounts

__global__ void k_popc_block_sums(const unsigned int* words, long long n, int per_block,
                                  int* block_sums) {
    __shared__ int s[32];
    const long long start = (long long)blockIdx.x * per_block;
    int acc = 0;
    for (int i = threadIdx.x; i < per_block; i += blockDim.x) {
        const long long w = start + i;
        if (w < n) acc += __popc(words[w]);
    }
    acc = warp_sum_i(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0;
        v = warp_sum_i(v);
        if (threadIdx.x == 0) block_sums[blockIdx.x] = v;
    }
}

// Exclusive scan of block_sums in place by one block; writes the total to *total.
__global__ void k_scan_small(int* block_sums, int n, int* total) {
    __shared__ int s[1024];
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    int acc = 0;
    for (int i = 0; i < per; ++i)
        if (b0 + i < n) acc += block_sums[b0 + i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const int v = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int run = s[threadIdx.x] - acc;  // exclusive prefix of this thread's chunk
    for (int i = 0; i < per; ++i)
        if (b0 + i < n) {
            const int v = block_sums[b0 + i];
            block_sums[b0 + i] = run;
            run += v;
        }
    if (threadIdx.x == blockDim.x - 1) *total = s[threadIdx.x];
}

// prefix[w] = number of set bits in words[0..w).
__global__ void k_popc_prefix(const unsigned int* words, long long n, int per_block,
                              const int* block_offsets, int* prefix) {
    __shared__ int s[1024];
    const long long start = (long long)blockIdx.x * per_block;
    const int per = per_block / blockDim.x;  // words per thread (per_block is a multiple)
    const long long w0 = start + (long long)threadIdx.x * per;
    int acc = 0;
    for (int i = 0; i < per; ++i)
        if (w0 + i < n) acc += __popc(words[w0 + i]);
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const int v = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int run = block_offsets[blockIdx.x] + s[threadIdx.x] - acc;
    for (int i = 0; i < per; ++i)
        if (w0 + i < n) {
            prefix[w0 + i] = run;
            run += __popc(words[w0 + i]);
        }
}

// --------------------------------------------------------------------------------------- finish

__global__ void k_stats_init(int* stats, unsigned long long* sums, int k1) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k1; i += gridDim.x * blockDim.x) {
        stats[i * 5 + 0] = 0x7fffffff;  // min x
        stats[i * 5 + 1] = 0x7fffffff;  // min y
        stats[i * 5 + 2] = -1;          // max x (turned into width)
        stats[i * 5 + 3] = -1;          // max y (turned into height)
        stats[i * 5 + 4] = 0;           // area
        sums[2 * i] = 0;
        sums[2 * i + 1] = 0;
    }
}

// Final labels and stats of one 32 x 64 tile. The tile forest is rebuilt from the bitmap; each
// local root follows the merged parents to its global root once, whose label is the rank of that
// root among the roots (popcount prefix) + 1; every pixel then takes the label of its run's root.
// Warps write 32 consecutive pixels of a row, so equal labels form runs of lanes; a run's head lane
// adds the run's bbox, area and coordinate sums with one set of atomics. Background runs are
// reduced per block first.
__global__ void __launch_bounds__(kCclThreads) k_finish(Geo g, const int* parents, const unsigned int* roots,
                                                        const int* prefix, const unsigned int* fgbits,
                                                        int* labels, int* stats, unsigned long long* sums, int k1) {
    __shared__ int par[kTilePx];
    __shared__ int lab_of[kTilePx];
    __shared__ unsigned long long mask[kTileH];
    __shared__ long long s_bg[7];
    const int tx0 = blockIdx.x * kTileW, ty0 = blockIdx.y * kTileH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < kTileH) {
        const int y = ty0 + threadIdx.x;
        unsigned long long m = 0;
        if (y < g.H) {
            const unsigned* row = fgbits + (long long)y * g.words_per_row() + (tx0 >> 5);
            m = (unsigned long long)row[0] | ((unsigned long long)row[1] << 32);
        }
        mask[threadIdx.x] = m;
    }
    if (threadIdx.x == 0) {
        s_bg[0] = 0x7fffffff; s_bg[1] = 0x7fffffff; s_bg[2] = -1; s_bg[3] = -1; s_bg[4] = 0; s_bg[5] = 0; s_bg[6] = 0;
    }
    __syncthreads();
    tile_forest(mask, g.conn, par);
    if (threadIdx.x < kTileH) {
        const unsigned long long m = mask[threadIdx.x];
        for (unsigned long long s = m & ~(m << 1); s; s &= s - 1) {
            const int l = tile_lidx(g.conn, threadIdx.x, __ffsll((long long)s) - 1);
            if (par[l] != l) continue;
            int p = tile_gid(g, ty0, tx0, l);
            int q = parents[p];
            while (q != p) {
                p = q;
                q = parents[p];
            }
            lab_of[l] = prefix[p >> 5] + __popc(roots[p >> 5] & ((1u << (p & 31)) - 1u)) + 1;
        }
    }
    __syncthreads();
    for (int hr = warp; hr < kTileH * 2; hr += kCclThreads / 32) {
        const int r = hr >> 1, xl = (hr & 1) * 32 + lane;
        const int y = ty0 + r, x = tx0 + xl;
        const unsigned long long m = mask[r];
        int lab = -1;  // -1 outside the image
        if (x < g.W && y < g.H) {
            lab = ((m >> xl) & 1ull) ? lab_of[par[tile_lidx(g.conn, r, run_first(m, xl))]] : 0;
            labels[(long long)y * g.W + x] = lab;
        }
        const int prev = __shfl_up_sync(0xffffffffu, lab, 1);
        const bool head = lab >= 0 && (lane == 0 || prev != lab);
        const unsigned heads = __ballot_sync(0xffffffffu, head);
        const unsigned valid = __ballot_sync(0xffffffffu, lab >= 0);
        // Run end: lane before the next head (or the last valid lane).
        const unsigned later = heads & ~((2u << lane) - 1u);
        const int next = later ? __ffs(later) - 1 : 32;
        const int last_valid = 31 - __clz(valid | 1u);
        const int tail = min(next - 1, last_valid);
        if (head && lab > 0 && lab < k1) {  // labels beyond the component count cannot occur
            const int x0 = x, x1 = x + (tail - lane);
            const long long len = x1 - x0 + 1;
            const long long sx = (long long)(x0 + x1) * len / 2;
            int* st = stats + (long long)lab * 5;
            atomicMin(&st[0], x0);
            atomicMin(&st[1], y);
            atomicMax(&st[2], x1);
            atomicMax(&st[3], y);
            atomicAdd(&st[4], (int)len);
            atomicAdd(&sums[2LL * lab], (unsigned long long)sx);
            atomicAdd(&sums[2LL * lab + 1], (unsigned long long)((long long)y * len));
        }
        // Background (label 0): one ballot per warp row, block totals in shared memory.
        const unsigned bgm = __ballot_sync(0xffffffffu, lab == 0);
        const int bsum = warp_sum_i(lab == 0 ? x : 0);
        if (lane == 0 && bgm) {
            const int xs = tx0 + (hr & 1) * 32;
            atomicMin(&s_bg[0], (long long)(xs + __ffs(bgm) - 1));
            atomicMin(&s_bg[1], (long long)y);
            atomicMax(&s_bg[2], (long long)(xs + 31 - __clz(bgm)));
            atomicMax(&s_bg[3], (long long)y);
            atomicAdd(reinterpret_cast<unsigned long long*>(&s_bg[4]), (unsigned long long)__popc(bgm));
            atomicAdd(reinterpret_cast<unsigned long long*>(&s_bg[5]), (unsigned long long)bsum);
            atomicAdd(reinterpret_cast<unsigned long long*>(&s_bg[6]),
                      (unsigned long long)((long long)y * __popc(bgm)));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_bg[4] > 0) {
        atomicMin(&stats[0], (int)s_bg[0]);
        atomicMin(&stats[1], (int)s_bg[1]);
        atomicMax(&stats[2], (int)s_bg[2]);
        atomicMax(&stats[3], (int)s_bg[3]);
        atomicAdd(&stats[4], (int)s_bg[4]);
        atomicAdd(&sums[0], (unsigned long long)s_bg[5]);
        atomicAdd(&sums[1], (unsigned long long)s_bg[6]);
    }
}

// bbox max -> width/height; centroid = exact integer sum / area (as OpenCV).
__global__ void k_stats_final(int* stats, const unsigned long long* sums, double* centroids, int k1) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k1; i += gridDim.x * blockDim.x) {
        int* st = stats + (long long)i * 5;
        const int area = st[4];
        const unsigned long long sx = sums[2 * i], sy = sums[2 * i + 1];
        if (area > 0) {
            st[2] = st[2] - st[0] + 1;
            st[3] = st[3] - st[1] + 1;
            centroids[2 * i] = (double)sx / (double)area;
            centroids[2 * i + 1] = (double)sy / (double)area;
        } else {
            st[0] = st[1] = st[2] = st[3] = 0;
            centroids[2 * i] = dnan();
            centroids[2 * i + 1] = dnan();
        }
    }
}

struct CclLayout {
    long long canon_n;   // entries of the canonical parents array
    long long words;     // root bitmap words
    int scan_blocks;     // blocks of the popcount prefix
    int* parents;
    unsigned int* roots;
    int* prefix;
    int* block_sums;
    int* scratch_count;
    unsigned int* fgbits;  // foreground bitmap, H x words-per-row
};
constexpr int kScanPerBlock = 4096;  // bitmap words per prefix block (1024 threads x 4)

CclLayout ccl_layout(void* ws, int H, int W, size_t* bytes) {
    CclLayout L;
    const long long Hb = (H + 1) / 2, Wb = (W + 1) / 2;
    L.canon_n = Hb * Wb * 4;  // >= H*W; also covers raster order for 4-connectivity
    L.words = (L.canon_n + 31) / 32;
    L.scan_blocks = (int)((L.words + kScanPerBlock - 1) / kScanPerBlock);
    Arena a(ws);
    L.parents = a.take<int>(L.canon_n);
    L.roots = a.take<unsigned int>(L.words);
    L.prefix = a.take<int>(L.words);
    L.block_sums = a.take<int>(L.scan_blocks + 1);
    L.scratch_count = a.take<int>(4);
    L.fgbits = a.take<unsigned int>((long long)H * ((W + 63) / 64 * 2));
    if (bytes) *bytes = a.used;
    return L;
}

// ---------------------------------------------------------------------- allocation-free Otsu

// Scratch of spx_otsu_static: the same pieces as the Otsu workspace (histogram, value range, four
// per-bin arrays of the scan), in one file-scope device array. Every GPU that loads this library
// holds it (2.3 MiB) until the process exits.
constexpr size_t kOtsuStaticBytes = 65536 * sizeof(unsigned int) + 256 + 4 * 65536 * sizeof(double) + 256;
__device__ __align__(256) unsigned char g_otsu_static[kOtsuStaticBytes];

__global__ void k_range_init(unsigned int* range) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        range[0] = 0xffffffffu;
        range[1] = 0u;
    }
}

__global__ void k_zero_u32(unsigned int* p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0u;
}

// Device address of g_otsu_static for the current device, looked up once per device and kept for the
// life of the process: a cudaDeviceReset (which unloads this module's device copy) invalidates it,
// so the library must not be used across one.
int otsu_static_scratch(void** out) {
    static std::mutex mu;
    static void* cache[128] = {};
    int dev = 0;
    SPX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) {
        set_error("device index %d out of range", dev);
        return SPX_ERR_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!cache[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_otsu_static);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(g_otsu_static) failed: %s", cudaGetErrorString(e));
            return SPX_ERR_CUDA;
        }
        cache[dev] = p;
    }
    *out = cache[dev];
    return SPX_OK;
}


// ------------------------------------------------------------------------------ morphology

// bw = 255 where the pixel is foreground (img > t, or img <= t with invert), else 0: the 0/255
// image of cv2.threshold(THRESH_BINARY[_INV]).
__global__ void k_binarize(const void* img, int dtype, long long n, const double* t_dev, double t_fixed, int invert,
                           uint8_t* bw) {
    const double t = t_dev ? *t_dev : t_fixed;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        bw[i] = is_fg(load_px(img, dtype, i), t, invert) ? 255 : 0;
}

// One erosion (dilate = 0: minimum) or dilation (maximum) of a 0/255 image with the 3x3 cross
// (cv2.getStructuringElement(MORPH_ELLIPSE, (3, 3))); neighbours outside the image are ignored, as
// OpenCV's default morphology border does.
__global__ void k_morph_cross(const uint8_t* in, int H, int W, int dilate, uint8_t* out) {
    const long long total = (long long)H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(i, W, &y, &x);
        unsigned v = in[i];
        if (dilate) {
            if (y > 0) v = max(v, (unsigned)in[i - W]);
            if (y < H - 1) v = max(v, (unsigned)in[i + W]);
            if (x > 0) v = max(v, (unsigned)in[i - 1]);
            if (x < W - 1) v = max(v, (unsigned)in[i + 1]);
        } else {
            if (y > 0) v = min(v, (unsigned)in[i - W]);
            if (y < H - 1) v = min(v, (unsigned)in[i + W]);
            if (x > 0) v = min(v, (unsigned)in[i - 1]);
            if (x < W - 1) v = min(v, (unsigned)in[i + 1]);
        }
        out[i] = (uint8_t)v;
    }
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

const char* spx_last_error(void) { return spx::g_error; }

int spx_version(void) { return 1; }

int spx_tune_set(const char* knob, int value) {
    SPX_REQUIRE(knob, "null knob name");
    Tuning& t = tuning();
    if (!strcmp(knob, "fit_warps")) {
        SPX_REQUIRE(value == 2 || value == 4 || value == 8, "fit_warps must be 2, 4 or 8");
        t.fit_warps = value;
    } else if (!strcmp(knob, "fit_blocks_per_sm")) {
        SPX_REQUIRE(value >= 2 && value <= 32, "fit_blocks_per_sm must be in [2, 32]");
        t.fit_blocks_per_sm = value;
    } else if (!strcmp(knob, "render_tile")) {
        SPX_REQUIRE(value == 16 || value == 32 || value == 64, "render_tile must be 16, 32 or 64");
        t.render_tile = value;
    } else if (!strcmp(knob, "radial_rays")) {
        SPX_REQUIRE(value == 0 || value == 2, "radial_rays must be 0 or 2");
        t.radial_rays = value;
    } else {
        set_error("unknown tuning knob '%s'", knob);
        return SPX_ERR_ARGUMENT;
    }
    return SPX_OK;
}

int spx_tune_get(const char* knob, int* value) {
    SPX_REQUIRE(knob && value, "null pointer");
    const Tuning& t = tuning();
    if (!strcmp(knob, "fit_warps")) *value = t.fit_warps;
    else if (!strcmp(knob, "fit_blocks_per_sm")) *value = t.fit_blocks_per_sm;
    else if (!strcmp(knob, "render_tile")) *value = t.render_tile;
    else if (!strcmp(knob, "radial_rays")) *value = t.radial_rays;
    else {
        set_error("unknown tuning knob '%s'", knob);
        return SPX_ERR_ARGUMENT;
    }
    return SPX_OK;
}

unsigned long long spx_launch_count(void) { return __atomic_load_n(&spx::g_launches, __ATOMIC_RELAXED); }

}  // extern "C"

namespace spx {
namespace {
// Eight independent FP64 FMA chains per thread (no dependency between them, so the FP64 pipe, not
// the FMA latency, bounds the rate); the sums go to `sink` so nothing is optimised away.
__global__ void __launch_bounds__(256) k_fp64_fma_rate(int iters, double* sink) {
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = 1.0 + 1e-3 * (threadIdx.x + q);
    const double b = 0.9999999, c = 1e-7;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = __fma_rn(a[q], b, c);
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += a[q];
    sink[blockIdx.x * blockDim.x + threadIdx.x] = t;
}
}  // namespace
}  // namespace spx

extern "C" {

int spx_fp64_fma_rate(int blocks, int iters, double* sink, double* flops, void* stream) {
    SPX_REQUIRE(blocks >= 1 && iters >= 1 && sink && flops, "bad arguments");
    k_fp64_fma_rate<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(iters, sink);
    *flops = 2.0 * 8.0 * 256.0 * (double)blocks * (double)iters;
    return check_launch("k_fp64_fma_rate");
}

int spx_device_info(int* sm_count, int* is_sm100) {
    int dev = 0;
    SPX_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    SPX_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (sm_count) *sm_count = prop.multiProcessorCount;
    if (is_sm100) *is_sm100 = prop.major == 10 ? 1 : 0;
    return SPX_OK;
}

size_t spx_otsu_workspace_bytes(int dtype) {
    (void)dtype;
    Arena a(nullptr);
    a.take<unsigned int>(65536);
    a.take<unsigned int>(2);
    a.take<double>(4 * 65536);
    return a.used;
}

static int launch_minmax(const void* img, int dtype, int height, int width, int step, long long n, unsigned int* range,
                         cudaStream_t s) {
    if (step == 1 && dtype == SPX_U16 && (reinterpret_cast<uintptr_t>(img) % 16) == 0) {
        k_minmax_dense<<<grid_for(n / 8 + 1, 256, 148 * 8), 256, 0, s>>>(static_cast<const uint16_t*>(img), n, range);
        return check_launch("k_minmax_dense");
    }
    k_minmax<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(img, dtype, height, width, step, range);
    return check_launch("k_minmax");
}

int spx_otsu(const void* img, int dtype, int height, int width, int step, double* threshold,
             void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(dtype == SPX_U8 || dtype == SPX_U16, "Otsu thresholding needs a uint8 or uint16 image");
    SPX_REQUIRE(height > 0 && width > 0 && step >= 1, "bad image size or step");
    SPX_REQUIRE(img && threshold && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_otsu_workspace_bytes(dtype), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena a(workspace);
    unsigned int* hist = a.take<unsigned int>(65536);
    unsigned int* range = a.take<unsigned int>(2);
    const int nbins = dtype == SPX_U8 ? 256 : 65536;
    SPX_CUDA(cudaMemsetAsync(hist, 0, 65536 * sizeof(unsigned int), s));
    const unsigned int init[2] = {0xffffffffu, 0u};
    SPX_CUDA(cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int hs = (int)(((long long)height + step - 1) / step), ws = (int)(((long long)width + step - 1) / step);
    const long long n = (long long)hs * ws;
    if (int e = launch_minmax(img, dtype, height, width, step, n, range, s)) return e;
    const size_t smem = kHistSmemBins * sizeof(unsigned int);
    SPX_CUDA(cudaFuncSetAttribute(k_histogram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int dense = step == 1 && dtype == SPX_U16 && (reinterpret_cast<uintptr_t>(img) % 16) == 0;
    k_histogram<<<grid_for(n / 8 + 1, 512, 148 * 3), 512, smem, s>>>(img, dtype, height, width, step,
                                                                     dense, range, hist);
    if (int e = check_launch("k_histogram")) return e;
    double* bufs = a.take<double>(4 * 65536);
    k_otsu_scan<<<1, 1024, 0, s>>>(hist, nbins, range, n, bufs, bufs + 65536, bufs + 2 * 65536,
                                   bufs + 3 * 65536, threshold);
    return check_launch("k_otsu_scan");
}

int spx_histogram(const void* img, int dtype, int height, int width, int step, unsigned int* hist,
                  unsigned int* range, void* stream) {
    SPX_REQUIRE(dtype == SPX_U8 || dtype == SPX_U16, "histograms need a uint8 or uint16 image");
    SPX_REQUIRE(height > 0 && width > 0 && step >= 1, "bad image size or step");
    SPX_REQUIRE(img && hist && range, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SPX_CUDA(cudaMemsetAsync(hist, 0, 65536 * sizeof(unsigned int), s));
    const unsigned int init[2] = {0xffffffffu, 0u};
    SPX_CUDA(cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int hs = (int)(((long long)height + step - 1) / step), ws = (int)(((long long)width + step - 1) / step);
    const long long n = (long long)hs * ws;
    if (int e = launch_minmax(img, dtype, height, width, step, n, range, s)) return e;
    const size_t smem = kHistSmemBins * sizeof(unsigned int);
    SPX_CUDA(cudaFuncSetAttribute(k_histogram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int dense = step == 1 && dtype == SPX_U16 && (reinterpret_cast<uintptr_t>(img) % 16) == 0;
    k_histogram<<<grid_for(n / 8 + 1, 512, 148 * 3), 512, smem, s>>>(img, dtype, height, width, step, dense, range,
                                                                     hist);
    return check_launch("k_histogram");
}

int spx_otsu_from_histogram(const unsigned int* hist, int dtype, const unsigned int* range, long long total,
                            double* threshold, void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(dtype == SPX_U8 || dtype == SPX_U16, "Otsu thresholding needs a uint8 or uint16 histogram");
    SPX_REQUIRE(total > 0, "empty histogram");
    SPX_REQUIRE(hist && range && threshold && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_otsu_workspace_bytes(dtype), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena a(workspace);
    a.take<unsigned int>(65536);
    a.take<unsigned int>(2);
    double* bufs = a.take<double>(4 * 65536);
    k_otsu_scan<<<1, 1024, 0, s>>>(hist, dtype == SPX_U8 ? 256 : 65536, range, total, bufs, bufs + 65536,
                                   bufs + 2 * 65536, bufs + 3 * 65536, threshold);
    return check_launch("k_otsu_scan");
}

int spx_otsu_static(const void* img, int dtype, int height, int width, int step, double* threshold, void* stream) {
    SPX_REQUIRE(dtype == SPX_U8 || dtype == SPX_U16, "Otsu thresholding needs a uint8 or uint16 image");
    SPX_REQUIRE(height > 0 && width > 0 && step >= 1, "bad image size or step");
    const long long hs = ((long long)height + step - 1) / step, ws = ((long long)width + step - 1) / step;
    SPX_REQUIRE(hs * ws <= 0xffffffffLL,
                "spx_otsu_static: %lld sampled pixels exceed the maximum of 4294967295 (32-bit histogram counts)",
                hs * ws);
    SPX_REQUIRE(img && threshold, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* scratch = nullptr;
    if (int e = otsu_static_scratch(&scratch)) return e;
    Arena a(scratch);
    unsigned int* hist = a.take<unsigned int>(65536);
    unsigned int* range = a.take<unsigned int>(2);
    double* bufs = a.take<double>(4 * 65536);
    SPX_REQUIRE(a.used <= kOtsuStaticBytes, "static Otsu scratch too small");
    const int nbins = dtype == SPX_U8 ? 256 : 65536;
    const long long n = hs * ws;
    // The array keeps the previous call's contents: clear the histogram and reset the range first.
    k_zero_u32<<<64, 256, 0, s>>>(hist, 65536);
    if (int e = check_launch("k_zero_u32")) return e;
    k_range_init<<<1, 32, 0, s>>>(range);
    if (int e = check_launch("k_range_init")) return e;
    if (int e = launch_minmax(img, dtype, height, width, step, n, range, s)) return e;
    const size_t smem = kHistSmemBins * sizeof(unsigned int);
    SPX_CUDA(cudaFuncSetAttribute(k_histogram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int dense = step == 1 && dtype == SPX_U16 && (reinterpret_cast<uintptr_t>(img) % 16) == 0;
    k_histogram<<<grid_for(n / 8 + 1, 512, 148 * 3), 512, smem, s>>>(img, dtype, height, width, step, dense, range,
                                                                     hist);
    if (int e = check_launch("k_histogram")) return e;
    k_otsu_scan<<<1, 1024, 0, s>>>(hist, nbins, range, n, bufs, bufs + 65536, bufs + 2 * 65536, bufs + 3 * 65536,
                                   threshold);
    return check_launch("k_otsu_scan");
}

int spx_triangle(const void* img, int dtype, int height, int width, double* threshold,
                 void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(dtype == SPX_U8, "the triangle threshold needs a uint8 image");
    SPX_REQUIRE(height > 0 && width > 0, "bad image size");
    SPX_REQUIRE(img && threshold && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_otsu_workspace_bytes(dtype), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena a(workspace);
    unsigned int* hist = a.take<unsigned int>(65536);
    unsigned int* range = a.take<unsigned int>(2);
    SPX_CUDA(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), s));
    const unsigned int init[2] = {0u, 255u};
    SPX_CUDA(cudaMemcpyAsync(range, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const long long n = (long long)height * width;
    const size_t smem = kHistSmemBins * sizeof(unsigned int);
    SPX_CUDA(cudaFuncSetAttribute(k_histogram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_histogram<<<grid_for(n, 512, 148 * 3), 512, smem, s>>>(img, dtype, height, width, 1, 0, range, hist);
    if (int e = check_launch("k_histogram")) return e;
    k_triangle_scan<<<1, 32, 0, s>>>(hist, threshold);
    return check_launch("k_triangle_scan");
}

size_t spx_ccl_workspace_bytes(int height, int width) {
    size_t b = 0;
    ccl_layout(nullptr, height, width, &b);
    return b;
}

int spx_binarize(const void* img, int dtype, int height, int width, const double* threshold_dev,
                 double fixed_threshold, int invert, uint8_t* out, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && dtype >= SPX_U8 && dtype <= SPX_F64, "bad arguments");
    SPX_REQUIRE(img && out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = (long long)height * width;
    k_binarize<<<grid_for(n, 256), 256, 0, s>>>(img, dtype, n, threshold_dev, fixed_threshold, invert, out);
    return check_launch("k_binarize");
}

int spx_morphology(uint8_t* bw, int height, int width, int open_iterations, int close_iterations, uint8_t* tmp,
                   void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && open_iterations >= 0 && close_iterations >= 0, "bad arguments");
    SPX_REQUIRE(bw && tmp && bw != tmp, "null or aliased pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n = (long long)height * width;
    // MORPH_OPEN: erode then dilate, `open` times each; MORPH_CLOSE: dilate then erode. The number
    // of passes is even, so the result ends in bw.
    uint8_t* cur = bw;
    uint8_t* nxt = tmp;
    auto pass = [&](int dilate, int times) -> int {
        for (int k = 0; k < times; ++k) {
            k_morph_cross<<<grid_for(n, 256), 256, 0, s>>>(cur, height, width, dilate, nxt);
            if (int e = check_launch("k_morph_cross")) return e;
            uint8_t* t = cur;
            cur = nxt;
            nxt = t;
        }
        return SPX_OK;
    };
    if (int e = pass(0, open_iterations)) return e;
    if (int e = pass(1, open_iterations)) return e;
    if (int e = pass(1, close_iterations)) return e;
    return pass(0, close_iterations);
}

int spx_ccl_label(const void* img, int dtype, int height, int width, const double* threshold_dev,
                  double fixed_threshold, int invert, int connectivity, int* labels, int* count,
                  void* workspace, size_t workspace_bytes, void* stream) {
    (void)labels;
    SPX_REQUIRE(height > 0 && width > 0, "bad image size");
    SPX_REQUIRE((long long)((height + 1) / 2) * ((width + 1) / 2) * 4 < 0x7fffffffLL,
                "image too large for 32-bit labels");
    SPX_REQUIRE(connectivity == 8 || connectivity == 4, "connectivity must be 4 or 8");
    SPX_REQUIRE(dtype >= SPX_U8 && dtype <= SPX_F64, "bad dtype");
    SPX_REQUIRE(img && count && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_ccl_workspace_bytes(height, width), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CclLayout L = ccl_layout(workspace, height, width, nullptr);
    Geo g{height, width, (width + 1) / 2, connectivity};
    SPX_CUDA(cudaMemsetAsync(L.roots, 0, L.words * sizeof(unsigned int), s));
    const int tiles_x = (width + kTileW - 1) / kTileW, tiles_y = (height + kTileH - 1) / kTileH;
    k_local_ccl<<<dim3(tiles_x, tiles_y), kCclThreads, 0, s>>>(img, dtype, g, threshold_dev, fixed_threshold,
                                                       invert, L.parents, L.roots, L.fgbits);
    if (int e = check_launch("k_local_ccl")) return e;
    const long long border = (long long)tiles_x * tiles_y * (kTileW + 2 * kTileH);
    k_border_merge<<<grid_for(border, 256), 256, 0, s>>>(g, L.parents, L.roots, L.fgbits, tiles_x, tiles_y);
    if (int e = check_launch("k_border_merge")) return e;
    SPX_REQUIRE(L.scan_blocks <= 1024 * 64, "image too large for the label prefix");
    k_popc_block_sums<<<L.scan_blocks, 1024, 0, s>>>(L.roots, L.words, kScanPerBlock, L.block_sums);
    if (int e = check_launch("k_popc_block_sums")) return e;
    k_scan_small<<<1, 1024, 0, s>>>(L.block_sums, L.scan_blocks, count);
    if (int e = check_launch("k_scan_small")) return e;
    k_popc_prefix<<<L.scan_blocks, 1024, 0, s>>>(L.roots, L.words, kScanPerBlock, L.block_sums, L.prefix);
    return check_launch("k_popc_prefix");
}

int spx_ccl_finish(int* labels, int height, int width, int connectivity, int num_components,
                   int* stats, double* centroids, void* workspace, size_t workspace_bytes,
                   void* stream) {
    SPX_REQUIRE(labels && stats && centroids && workspace, "null pointer");
    SPX_REQUIRE(num_components >= 0, "bad component count");
    SPX_REQUIRE(workspace_bytes >= spx_ccl_workspace_bytes(height, width), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CclLayout L = ccl_layout(workspace, height, width, nullptr);
    Geo g{height, width, (width + 1) / 2, connectivity};
    const int k1 = num_components + 1;
    // The u64 coordinate sums live in the centroid array until the last kernel converts them.
    unsigned long long* sums = reinterpret_cast<unsigned long long*>(centroids);
    k_stats_init<<<grid_for(k1, 256), 256, 0, s>>>(stats, sums, k1);
    if (int e = check_launch("k_stats_init")) return e;
    k_finish<<<dim3((width + kTileW - 1) / kTileW, (height + kTileH - 1) / kTileH), kCclThreads, 0, s>>>(
        g, L.parents, L.roots, L.prefix, L.fgbits, labels, stats, sums, k1);
    if (int e = check_launch("k_finish")) return e;
    k_stats_final<<<grid_for(k1, 256), 256, 0, s>>>(stats, sums, centroids, k1);
    return check_launch("k_stats_final");
}

}  // extern "C"
