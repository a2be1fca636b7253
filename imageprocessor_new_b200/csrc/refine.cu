// Component selection and per-blob centre refinement, one warp per blob.
//
// Reference semantics (CPU estimators, the parity target):
//   area filter / refine="auto"      subpx/_cpu/centers.py:22-30, 376-391
//   _bg_from_border (2-px median)    subpx/_cpu/centers.py:31-42
//   weighted centroid                subpx/_cpu/centers.py:45-64
//   log-quadratic                    subpx/_cpu/centers.py:67-107
//   edge gradient-moment             subpx/_cpu/centers.py:111-223
//   "none" (mask mean)               subpx/_cpu/centers.py:239-243
//
// ROI = bbox +- pad clipped to the image; mask = labels == label. Sums whose terms are exact
// (integer images: g - median is a multiple of 1/2) are exact in FP64 whatever the order, so the
// weighted and edge estimators return NumPy's bits on integer images. The log-quadratic fit solves
// the normal equations in ROI-centred, scaled coordinates (the stationary point and cond(H) do not
// depend on that change of coordinates) instead of an SVD least-squares solve.

#include "common.cuh"
#include "scan.cuh"

namespace spx {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kSortCap = 1024;  // border values sorted in shared memory per warp

// ------------------------------------------------------------------------------------ selection

__global__ void k_select_flags(const int* stats, int k, int area_min, int area_max, int* flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const int area = stats[(long long)(i + 1) * 5 + 4];
        flags[i] = (area >= area_min && area <= area_max) ? 1 : 0;
    }
}

__global__ void k_select_rows(const int* stats, int k, int area_min, int area_max, int refine,
                              double small_feature_max, const int* offsets, int* rows,
                              uint8_t* methods) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const int* st = stats + (long long)(i + 1) * 5;
        const int area = st[4];
        if (!(area >= area_min && area <= area_max)) continue;
        const int o = offsets[i];
        rows[o * 5 + 0] = st[0];
        rows[o * 5 + 1] = st[1];
        rows[o * 5 + 2] = st[2];
        rows[o * 5 + 3] = st[3];
        rows[o * 5 + 4] = i + 1;
        int m = refine;
        if (refine == SPX_REFINE_AUTO) {
            const double size = (double)max(st[2], st[3]);
            m = size <= small_feature_max ? SPX_REFINE_LOGQUAD : SPX_REFINE_EDGE;
        }
        methods[o] = (uint8_t)m;
    }
}

// Cells of measure_cds: rows [x, y, w, h, cx, cy] (double) of the kept components in label order,
// their labels, whether the bbox stays off the image border, and per label whether it is too large.
__global__ void k_component_rows(const int* stats, const double* centroids, int k, int area_min, int area_max,
                                 int width, int height, const int* offsets, double* rows, int* ids,
                                 uint8_t* interior, uint8_t* oversized, int* n_oversized) {
    int over = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const int* st = stats + (long long)(i + 1) * 5;
        const int area = st[4];
        oversized[i + 1] = area > area_max;
        over += area > area_max;
        if (!(area >= area_min && area <= area_max)) continue;
        const int o = offsets[i];
        double* r = rows + (long long)o * 6;
        r[0] = st[0];
        r[1] = st[1];
        r[2] = st[2];
        r[3] = st[3];
        r[4] = centroids[2LL * (i + 1)];
        r[5] = centroids[2LL * (i + 1) + 1];
        ids[o] = i + 1;
        interior[o] = !(st[0] <= 0 || st[1] <= 0 || st[0] + st[2] >= width || st[1] + st[3] >= height);
    }
    over = warp_sum_i(over);
    if ((threadIdx.x & 31) == 0 && over) atomicAdd(n_oversized, over);
    if (blockIdx.x == 0 && threadIdx.x == 0) oversized[0] = 0;
}

// ------------------------------------------------------------------------------------- refiners

struct Roi {
    int x0, y0, w, h;  // ROI origin and size in the image
    int label;
};

__device__ __forceinline__ Roi make_roi(const int* row, int pad, int H, int W) {
    Roi r;
    const int x = row[0], y = row[1], bw = row[2], bh = row[3];
    r.x0 = max(0, x - pad);
    r.y0 = max(0, y - pad);
    const int x1 = min(W, x + bw + pad), y1 = min(H, y + bh + pad);
    r.w = x1 - r.x0;
    r.h = y1 - r.y0;
    r.label = row[4];
    return r;
}

// k-th smallest (0-based) of n 16-bit values value(i) by a warp: two 8-bit radix passes over a
// 256-bin shared-memory histogram, each digit found by a warp prefix sum of per-lane bin groups.
template <typename F>
__device__ int warp_select_u16(F value, int n, int k, int* hist, int lane) {
    int prefix = 0;
    for (int shift = 8; shift >= 0; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0;
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            const int v = value(i);
            if (shift == 0 ? (v >> 8) == (prefix >> 8) : true) atomicAdd(&hist[(v >> shift) & 255], 1);
        }
        __syncwarp();
        int c[8], mine = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = hist[lane * 8 + j];
            mine += c[j];
        }
        int incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        const int excl = incl - mine;
        const unsigned owner = __ballot_sync(0xffffffffu, excl <= k && k < incl);
        const int src = __ffs(owner) - 1;
        int digit = 0, rest = k - excl;
        if (lane == src) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (rest < c[j]) {
                    digit = lane * 8 + j;
                    break;
                }
                rest -= c[j];
            }
        }
        digit = __shfl_sync(0xffffffffu, digit, src);
        k = __shfl_sync(0xffffffffu, rest, src);
        prefix |= digit << shift;
        __syncwarp();
    }
    return prefix;
}

// Median of the ROI's top and bottom 2 rows and left and right 2 columns (full height, so the four
// 2x2 corners count twice), or of the whole ROI when it is too small, as _bg_from_border:
// np.median = mean of the two middle values for an even count.
__device__ double border_median(const void* img, int dtype, int W, const Roi& r, double* keys,
                                int lane) {
    const bool whole = r.h <= 4 || r.w <= 4;
    const int n = whole ? r.h * r.w : 4 * r.w + 4 * r.h;
    auto value = [&](int k) -> double {
        int yy, xx;
        if (whole) {
            yy = k / r.w;
            xx = k % r.w;
        } else if (k < 2 * r.w) {
            yy = k / r.w;
            xx = k % r.w;
        } else if (k < 4 * r.w) {
            yy = r.h - 2 + (k - 2 * r.w) / r.w;
            xx = (k - 2 * r.w) % r.w;
        } else if (k < 4 * r.w + 2 * r.h) {
            const int j = k - 4 * r.w;
            yy = j / 2;
            xx = j % 2;
        } else {
            const int j = k - 4 * r.w - 2 * r.h;
            yy = j / 2;
            xx = r.w - 2 + j % 2;
        }
        return load_px(img, dtype, (long long)(r.y0 + yy) * W + (r.x0 + xx));
    };
    if (dtype == SPX_U8 || dtype == SPX_U16) {
        // Integer images: the two middle order statistics by radix selection (exact).
        int* hist = reinterpret_cast<int*>(keys);
        auto iv = [&](int i) { return (int)value(i); };
        const int a = warp_select_u16(iv, n, (n - 1) / 2, hist, lane);
        const int b = (n & 1) ? a : warp_select_u16(iv, n, n / 2, hist, lane);
        return __ddiv_rn(__dadd_rn((double)a, (double)b), 2.0);
    }
    if (n <= kSortCap) {
        int m = 1;
        while (m < n) m <<= 1;
        for (int i = lane; i < m; i += 32) keys[i] = i < n ? value(i) : dinf();
        __syncwarp();
        warp_bitonic_sort(keys, m, lane);
        const double a = keys[(n - 1) / 2], b = keys[n / 2];
        __syncwarp();
        return __ddiv_rn(__dadd_rn(a, b), 2.0);
    }
    // Large frames: order statistics by counting (exact, O(n^2 / 32)).
    const int ka = (n - 1) / 2, kb = n / 2;
    double va = 0.0, vb = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double v = value(i);
        int less = 0, le = 0;
        for (int j = 0; j < n; ++j) {
            const double u = value(j);
            less += u < v;
            le += u <= v;
        }
        if (less <= ka && ka < le) va = v;
        if (less <= kb && kb < le) vb = v;
    }
    // Exactly the lanes that own the order statistics wrote them; take them by max over lanes of
    // a flag-selected value.
    int has_a = 0, has_b = 0;
    for (int i = lane; i < n; i += 32) {
        const double v = value(i);
        int less = 0, le = 0;
        for (int j = 0; j < n; ++j) {
            const double u = value(j);
            less += u < v;
            le += u <= v;
        }
        has_a |= (less <= ka && ka < le);
        has_b |= (less <= kb && kb < le);
    }
    const unsigned ma = __ballot_sync(0xffffffffu, has_a), mb = __ballot_sync(0xffffffffu, has_b);
    va = __shfl_sync(0xffffffffu, va, __ffs(ma) - 1);
    vb = __shfl_sync(0xffffffffu, vb, __ffs(mb) - 1);
    return __ddiv_rn(__dadd_rn(va, vb), 2.0);
}

__device__ __forceinline__ bool in_mask(const int* labels, int W, const Roi& r, int yy, int xx) {
    return labels[(long long)(r.y0 + yy) * W + (r.x0 + xx)] == r.label;
}

// Mask pixel count and exact integer coordinate sums (ROI-local), plus the mask bbox.
struct MaskSums {
    long long n, sx, sy;
    int xmin, xmax, ymin, ymax;
};

__device__ MaskSums mask_sums(const int* labels, int W, const Roi& r, int lane) {
    long long n = 0, sx = 0, sy = 0;
    int xmin = 0x7fffffff, xmax = -1, ymin = 0x7fffffff, ymax = -1;
    const int P = r.w * r.h;
    for (int k = lane; k < P; k += 32) {
        const int yy = k / r.w, xx = k % r.w;
        if (in_mask(labels, W, r, yy, xx)) {
            ++n;
            sx += xx;
            sy += yy;
            xmin = min(xmin, xx);
            xmax = max(xmax, xx);
            ymin = min(ymin, yy);
            ymax = max(ymax, yy);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
        xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
        ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
        ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
    }
    return {n, sx, sy, xmin, xmax, ymin, ymax};
}

__device__ void refine_weighted(const void* img, int dtype, const int* labels, int W, const Roi& r,
                                double* keys, int lane, double* cx, double* cy) {
    const MaskSums ms = mask_sums(labels, W, r, lane);
    if (ms.n == 0) {
        *cx = *cy = dnan();
        return;
    }
    const double bg = border_median(img, dtype, W, r, keys, lane);
    double s = 0.0, sx = 0.0, sy = 0.0;
    const int P = r.w * r.h;
    for (int k = lane; k < P; k += 32) {
        const int yy = k / r.w, xx = k % r.w;
        if (!in_mask(labels, W, r, yy, xx)) continue;
        double w = __dsub_rn(load_px(img, dtype, (long long)(r.y0 + yy) * W + (r.x0 + xx)), bg);
        if (w < 0.0) w = 0.0;
        s = __dadd_rn(s, w);
        sx = __dadd_rn(sx, __dmul_rn((double)xx, w));
        sy = __dadd_rn(sy, __dmul_rn((double)yy, w));
    }
    s = warp_sum(s);
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (s <= 0.0) {
        *cx = __ddiv_rn((double)ms.sx, (double)ms.n);
        *cy = __ddiv_rn((double)ms.sy, (double)ms.n);
        return;
    }
    *cx = __ddiv_rn(sx, s);
    *cy = __ddiv_rn(sy, s);
}

// Solves the n x n system A x = b (row-major, in place) by LU with partial pivoting; returns false
// when a pivot is zero or not finite.
template <int N>
__device__ bool solve_lu(double (&A)[N][N], double (&b)[N]) {
    for (int c = 0; c < N; ++c) {
        int p = c;
        double best = fabs(A[c][c]);
        for (int r = c + 1; r < N; ++r)
            if (fabs(A[r][c]) > best) { best = fabs(A[r][c]); p = r; }
        if (!(best > 0.0) || !isfinite(best)) return false;
        if (p != c) {
            for (int k = 0; k < N; ++k) { const double t = A[c][k]; A[c][k] = A[p][k]; A[p][k] = t; }
            const double t = b[c]; b[c] = b[p]; b[p] = t;
        }
        for (int r = c + 1; r < N; ++r) {
            const double f = A[r][c] / A[c][c];
            for (int k = c; k < N; ++k) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int c = N - 1; c >= 0; --c) {
        double v = b[c];
        for (int k = c + 1; k < N; ++k) v -= A[c][k] * b[k];
        b[c] = v / A[c][c];
    }
    for (int c = 0; c < N; ++c)
        if (!isfinite(b[c])) return false;
    return true;
}

// Eigen-decomposition of a symmetric 6x6 matrix by cyclic Jacobi rotations: A is destroyed, its
// diagonal ends up holding the eigenvalues, the columns of V the eigenvectors. Kept out of line:
// inlined into k_refine (nvcc 12.9, sm_100a) the rotations stopped being similarity transforms
// (the trace was not preserved), while the out-of-line copy and the same code on the host agree.
__device__ __noinline__ void jacobi6(double (&A)[6][6], double (&V)[6][6]) {
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) V[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 30; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < 6; ++i) {
            diag += A[i][i] * A[i][i];
            for (int j = i + 1; j < 6; ++j) off += A[i][j] * A[i][j];
        }
        if (off == 0.0 || off <= 1e-36 * diag) break;
        for (int p = 0; p < 5; ++p)
            for (int q = p + 1; q < 6; ++q) {
                const double apq = A[p][q];
                if (apq == 0.0) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < 6; ++k) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - sn * akq;
                    A[k][q] = sn * akp + c * akq;
                }
                for (int k = 0; k < 6; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - sn * aqk;
                    A[q][k] = sn * apk + c * aqk;
                }
                for (int k = 0; k < 6; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - sn * vkq;
                    V[k][q] = sn * vkp + c * vkq;
                }
            }
    }
}

// Coefficients in ROI pixel coordinates from coefficients in u = (x - xm) / s, v = (y - ym) / s
// (design [x^2, y^2, xy, x, y, 1] in both).
__device__ void unscale_coef(const double* c, double xm, double ym, double s, double* out) {
    const double s2 = s * s;
    out[0] = c[0] / s2;
    out[1] = c[1] / s2;
    out[2] = c[2] / s2;
    out[3] = (-2.0 * c[0] * xm - c[2] * ym) / s2 + c[3] / s;
    out[4] = (-2.0 * c[1] * ym - c[2] * xm) / s2 + c[4] / s;
    out[5] = (c[0] * xm * xm + c[1] * ym * ym + c[2] * xm * ym) / s2 - (c[3] * xm + c[4] * ym) / s + c[5];
}

__device__ void refine_logquad(const void* img, int dtype, const int* labels, int W, const Roi& r,
                               double* keys, int lane, double* cx, double* cy) {
    *cx = *cy = dnan();
    const MaskSums ms = mask_sums(labels, W, r, lane);
    if (ms.n < 6) return;
    const double bg = border_median(img, dtype, W, r, keys, lane);
    // Centred, scaled coordinates u = (x - xm) / s, v = (y - ym) / s.
    const double xm = 0.5 * (r.w - 1), ym = 0.5 * (r.h - 1), sc = 0.5 * max(r.w, r.h);
    const double inv = 1.0 / sc;
    double acc[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) acc[i] = 0.0;
    double vmax = -dinf();
    const int P = r.w * r.h;
    for (int k = lane; k < P; k += 32) {
        const int yy = k / r.w, xx = k % r.w;
        if (!in_mask(labels, W, r, yy, xx)) continue;
        const double v = load_px(img, dtype, (long long)(r.y0 + yy) * W + (r.x0 + xx)) - bg;
        vmax = fmax(vmax, v);
        const double z = log(fmax(v, 1e-9));
        const double u = (xx - xm) * inv, t = (yy - ym) * inv;
        const double d[6] = {u * u, t * t, u * t, u, t, 1.0};
        int q = 0;
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = a; b < 6; ++b) acc[q++] += d[a] * d[b];
#pragma unroll
        for (int a = 0; a < 6; ++a) acc[21 + a] += d[a] * z;
    }
#pragma unroll
    for (int i = 0; i < 27; ++i) acc[i] = warp_sum(acc[i]);
    vmax = warp_max(vmax);
    if (!(vmax > 0.0)) return;
    double A[6][6], b[6];
    int q = 0;
    for (int a = 0; a < 6; ++a)
        for (int c = a; c < 6; ++c) { A[a][c] = A[c][a] = acc[q++]; }
    for (int a = 0; a < 6; ++a) b[a] = acc[21 + a];
    double ca, cb, cc, cd, ce;
    const bool degenerate = (ms.xmax - ms.xmin) <= 1 || (ms.ymax - ms.ymin) <= 1;
    if (!degenerate) {
        if (!solve_lu<6>(A, b)) return;
        const double cf = b[5];
        ca = b[0]; cb = b[1]; cc = b[2]; cd = b[3]; ce = b[4];
        // A flat blob (log-values constant over the mask) has zero curvature: the reference's SVD
        // least squares then returns rounding noise for a..e and no meaningful stationary point.
        // Treat curvature below 1e-9 of the fitted level (in ROI-scaled units) as no fit.
        const double level = fmax(1.0, fabs(cf));
        if (fmax(fmax(fabs(ca), fabs(cb)), fabs(cc)) <= 1e-9 * level) return;
    } else {
        // Blobs one or two pixels thick: the design is rank-deficient (for two rows y1, y2,
        // y^2 - (y1 + y2) y + y1 y2 = 0 on every pixel). lstsq returns the minimum-norm solution in
        // pixel coordinates; build it from the scaled problem: pseudo-inverse solution there, mapped
        // to pixel coordinates, minus its component along the (mapped) null space.
        double V[6][6];
        jacobi6(A, V);
        double lmax = 0.0;
        for (int k = 0; k < 6; ++k) lmax = fmax(lmax, A[k][k]);
        double cs[6] = {0, 0, 0, 0, 0, 0};
        double nul[6][6];
        int nn = 0;
        for (int k = 0; k < 6; ++k) {
            const double lam = A[k][k];
            if (lam > 1e-11 * lmax) {
                double dot = 0.0;
                for (int r2 = 0; r2 < 6; ++r2) dot += V[r2][k] * b[r2];
                for (int r2 = 0; r2 < 6; ++r2) cs[r2] += V[r2][k] * (dot / lam);
            } else {
                double col[6];
                for (int r2 = 0; r2 < 6; ++r2) col[r2] = V[r2][k];
                unscale_coef(col, xm, ym, sc, nul[nn]);
                ++nn;
            }
        }
        double cp[6];
        unscale_coef(cs, xm, ym, sc, cp);
        // Orthonormalise the null directions (Gram-Schmidt) and project them out of cp.
        for (int k = 0; k < nn; ++k) {
            for (int j = 0; j < k; ++j) {
                double d = 0.0;
                for (int r2 = 0; r2 < 6; ++r2) d += nul[k][r2] * nul[j][r2];
                for (int r2 = 0; r2 < 6; ++r2) nul[k][r2] -= d * nul[j][r2];
            }
            double nrm = 0.0;
            for (int r2 = 0; r2 < 6; ++r2) nrm += nul[k][r2] * nul[k][r2];
            nrm = sqrt(nrm);
            if (!(nrm > 0.0)) continue;
            for (int r2 = 0; r2 < 6; ++r2) nul[k][r2] /= nrm;
            double d = 0.0;
            for (int r2 = 0; r2 < 6; ++r2) d += nul[k][r2] * cp[r2];
            for (int r2 = 0; r2 < 6; ++r2) cp[r2] -= d * nul[k][r2];
        }
        // Back to the scaled units of the code below (its cond test and centre map undo them).
        ca = cp[0] * sc * sc;
        cb = cp[1] * sc * sc;
        cc = cp[2] * sc * sc;
        cd = (cp[3] + 2.0 * cp[0] * xm + cp[2] * ym) * sc;
        ce = (cp[4] + 2.0 * cp[1] * ym + cp[2] * xm) * sc;
    }
    // H = [[2a, c], [c, 2b]] (in scaled units); cond(H) by its eigenvalues (symmetric).
    const double h00 = 2.0 * ca, h01 = cc, h11 = 2.0 * cb;
    const double mean = 0.5 * (h00 + h11), half = 0.5 * (h00 - h11);
    const double rad = sqrt(half * half + h01 * h01);
    const double l1 = fabs(mean + rad), l2 = fabs(mean - rad);
    const double smax = fmax(l1, l2), smin = fmin(l1, l2);
    if (!(smin > 0.0) || smax / smin > 1e8) return;
    const double det = h00 * h11 - h01 * h01;
    if (det == 0.0 || !isfinite(det)) return;
    // H (u, v) = -(d, e)
    const double uu = (-cd * h11 + ce * h01) / det;
    const double vv = (-ce * h00 + cd * h01) / det;
    const double px = xm + sc * uu, py = ym + sc * vv;
    if (!(px >= 0.0 && px < (double)r.w && py >= 0.0 && py < (double)r.h)) return;
    *cx = px;
    *cy = py;
}

// 2x binomial-5 smoothing with edge replication, in NumPy's operation order.
__device__ void smooth_binom5(double* p, int n) {
    double t[32];
    for (int i = 0; i < n; ++i) {
        const double xm2 = p[max(i - 2, 0)], xm1 = p[max(i - 1, 0)], x = p[i];
        const double xp1 = p[min(i + 1, n - 1)], xp2 = p[min(i + 2, n - 1)];
        double s = __dadd_rn(xm2, __dmul_rn(4.0, xm1));
        s = __dadd_rn(s, __dmul_rn(6.0, x));
        s = __dadd_rn(s, __dmul_rn(4.0, xp1));
        s = __dadd_rn(s, xp2);
        t[i] = __dmul_rn(s, 1.0 / 16.0);
    }
    for (int i = 0; i < n; ++i) p[i] = t[i];
}

// Edge position from a smoothed profile (_edge_from_profile_gradmoment_np); false when undefined.
__device__ bool edge_from_profile(const double* prof, int n, double base, double* out) {
    const int loc_rad = 3;
    if (n < 3) return false;
    double d[32];
    const int nd = n - 1;
    for (int i = 0; i < nd; ++i) d[i] = fabs(__dsub_rn(prof[i + 1], prof[i]));
    int ip = 0;
    double best = d[0];
    bool any_finite = isfinite(d[0]);
    for (int i = 1; i < nd; ++i) {
        any_finite |= isfinite(d[i]);
        if (d[i] > best || (isnan(best) && !isnan(d[i]))) { best = d[i]; ip = i; }
    }
    if (!any_finite) return false;
    const int hi = max(loc_rad, nd - 1 - loc_rad);
    const int ip0 = min(max(ip, loc_rad), hi);
    double sw = 0.0, swx = 0.0;
    for (int j = ip0 - loc_rad; j <= ip0 + loc_rad; ++j) {
        const int jj = min(max(j, 0), nd - 1);
        const double w = pow(fmax(d[jj], 0.0), 8.0);
        sw = __dadd_rn(sw, w);
        swx = __dadd_rn(swx, __dmul_rn(w, __dadd_rn(base, __dadd_rn((double)jj, 0.5))));
    }
    if (sw <= 1e-12) return false;
    *out = __ddiv_rn(swx, sw);
    return isfinite(*out);
}

__device__ void refine_edge(const void* img, int dtype, const int* labels, int W, const Roi& r,
                            double* prof_sh, int lane, double* cx, double* cy) {
    const int band_rad = 4, edge_rad = 10, n = 2 * edge_rad + 1;
    *cx = *cy = dnan();
    const MaskSums ms = mask_sums(labels, W, r, lane);
    if (ms.n == 0) return;
    const double w = (double)(ms.xmax - ms.xmin + 1), h = (double)(ms.ymax - ms.ymin + 1);
    double xc = __ddiv_rn((double)ms.sx, (double)ms.n), yc = __ddiv_rn((double)ms.sy, (double)ms.n);
    auto px = [&](int yy, int xx) {
        return load_px(img, dtype, (long long)(r.y0 + yy) * W + (r.x0 + xx));
    };
    for (int it = 0; it < 2; ++it) {
        const int xL0 = (int)rint(__dsub_rn(xc, __dmul_rn(0.5, __dsub_rn(w, 1.0))));
        const int xR0 = (int)rint(__dadd_rn(xc, __dmul_rn(0.5, __dsub_rn(w, 1.0))));
        const int yT0 = (int)rint(__dsub_rn(yc, __dmul_rn(0.5, __dsub_rn(h, 1.0))));
        const int yB0 = (int)rint(__dadd_rn(yc, __dmul_rn(0.5, __dsub_rn(h, 1.0))));
        const int ryc = (int)rint(yc), rxc = (int)rint(xc);
        // Lanes 0..20 build one sample of each of the four profiles.
        if (lane < n) {
            const int xs[2] = {xL0, xR0};
            for (int s = 0; s < 2; ++s) {  // x profiles: mean over 9 rows (axis 0: row by row)
                const int xx = min(max(xs[s] - edge_rad + lane, 0), r.w - 1);
                double acc = 0.0;
                for (int b = -band_rad; b <= band_rad; ++b) {
                    const int yy = min(max(ryc + b, 0), r.h - 1);
                    acc = __dadd_rn(acc, px(yy, xx));
                }
                prof_sh[s * 32 + lane] = __ddiv_rn(acc, 9.0);
            }
            const int ys[2] = {yT0, yB0};
            for (int s = 0; s < 2; ++s) {  // y profiles: mean over 9 columns (pairwise order of 9)
                const int yy = min(max(ys[s] - edge_rad + lane, 0), r.h - 1);
                double v[9];
                for (int b = 0; b < 9; ++b) v[b] = px(yy, min(max(rxc - band_rad + b, 0), r.w - 1));
                const double acc = __dadd_rn(
                    __dadd_rn(__dadd_rn(__dadd_rn(v[0], v[1]), __dadd_rn(v[2], v[3])),
                              __dadd_rn(__dadd_rn(v[4], v[5]), __dadd_rn(v[6], v[7]))),
                    v[8]);
                prof_sh[(2 + s) * 32 + lane] = __ddiv_rn(acc, 9.0);
            }
        }
        __syncwarp();
        // Lane s < 4 smooths profile s and finds its edge.
        int ok_s = 1;
        double e_s = 0.0;
        if (lane < 4) {
            const int base = lane == 0 ? xL0 : lane == 1 ? xR0 : lane == 2 ? yT0 : yB0;
            double p[32];
            for (int i = 0; i < n; ++i) p[i] = prof_sh[lane * 32 + i];
            smooth_binom5(p, n);
            smooth_binom5(p, n);
            ok_s = edge_from_profile(p, n, (double)(base - edge_rad), &e_s);
        }
        __syncwarp();
        if (__ballot_sync(0xffffffffu, lane < 4 && !ok_s)) return;
        double e[4];
        for (int s = 0; s < 4; ++s) e[s] = __shfl_sync(0xffffffffu, e_s, s);
        xc = __dmul_rn(0.5, __dadd_rn(e[0], e[1]));
        yc = __dmul_rn(0.5, __dadd_rn(e[2], e[3]));
    }
    if (!isfinite(xc) || !isfinite(yc)) return;
    *cx = xc;
    *cy = yc;
}

// One kernel per refiner M (each sized by its own register needs): it takes the rows whose
// method is M; the SPX_REFINE_NONE kernel also takes every other code and the rows past a device
// count (NaN).
template <int M>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
k_refine(const void* img, int dtype, int H, int W, const int* labels, const int* rows,
         const uint8_t* methods, int n, const int* n_dev, int pad, double* centers) {
    __shared__ double keys[kWarpsPerBlock][kSortCap];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int live = n_dev ? min(*n_dev, n) : n;  // rows past a device count are outputs of NaN
    for (int blob = blockIdx.x * kWarpsPerBlock + warp; blob < n; blob += gridDim.x * kWarpsPerBlock) {
        if (blob >= live) {
            if (M == SPX_REFINE_NONE && lane == 0) centers[2LL * blob] = centers[2LL * blob + 1] = dnan();
            continue;
        }
        const int m = methods[blob];
        const bool mine = M == SPX_REFINE_NONE
                              ? (m != SPX_REFINE_WEIGHTED && m != SPX_REFINE_LOGQUAD && m != SPX_REFINE_EDGE)
                              : m == M;
        if (!mine) continue;
        const Roi r = make_roi(rows + (long long)blob * 5, pad, H, W);
        double cx = dnan(), cy = dnan();
        if (r.w > 0 && r.h > 0) {
            if constexpr (M == SPX_REFINE_WEIGHTED) {
                refine_weighted(img, dtype, labels, W, r, keys[warp], lane, &cx, &cy);
            } else if constexpr (M == SPX_REFINE_LOGQUAD) {
                refine_logquad(img, dtype, labels, W, r, keys[warp], lane, &cx, &cy);
            } else if constexpr (M == SPX_REFINE_EDGE) {
                refine_edge(img, dtype, labels, W, r, keys[warp], lane, &cx, &cy);
            } else {
                const MaskSums ms = mask_sums(labels, W, r, lane);
                if (ms.n > 0) {
                    cx = __ddiv_rn((double)ms.sx, (double)ms.n);
                    cy = __ddiv_rn((double)ms.sy, (double)ms.n);
                }
            }
        }
        if (lane == 0) {
            centers[2LL * blob] = isfinite(cx) && isfinite(cy) ? __dadd_rn((double)r.x0, cx) : dnan();
            centers[2LL * blob + 1] = isfinite(cx) && isfinite(cy) ? __dadd_rn((double)r.y0, cy) : dnan();
        }
        __syncwarp();
    }
}

int launch_refine(const void* img, int dtype, int H, int W, const int* labels, const int* rows, const uint8_t* methods,
                  int n, const int* n_dev, int pad, double* centers, int blocks, cudaStream_t s) {
    const int grid = blocks < 148 * 16 ? blocks : 148 * 16;
    k_refine<SPX_REFINE_WEIGHTED><<<grid, kWarpsPerBlock * 32, 0, s>>>(img, dtype, H, W, labels, rows, methods, n,
                                                                        n_dev, pad, centers);
    if (int e = check_launch("k_refine")) return e;
    k_refine<SPX_REFINE_LOGQUAD><<<grid, kWarpsPerBlock * 32, 0, s>>>(img, dtype, H, W, labels, rows, methods, n,
                                                                       n_dev, pad, centers);
    if (int e = check_launch("k_refine")) return e;
    k_refine<SPX_REFINE_EDGE><<<grid, kWarpsPerBlock * 32, 0, s>>>(img, dtype, H, W, labels, rows, methods, n, n_dev,
                                                                    pad, centers);
    if (int e = check_launch("k_refine")) return e;
    k_refine<SPX_REFINE_NONE><<<grid, kWarpsPerBlock * 32, 0, s>>>(img, dtype, H, W, labels, rows, methods, n, n_dev,
                                                                    pad, centers);
    return check_launch("k_refine");
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

size_t spx_select_workspace_bytes(int num_components) {
    Arena a(nullptr);
    a.take<int>(num_components > 0 ? num_components : 1);
    a.take<int>(scan_scratch_ints(num_components > 0 ? num_components : 1));
    return a.used;
}

int spx_select_components(const int* stats, int num_components, int area_min, int area_max,
                          int refine, double small_feature_max, int* rows_out,
                          uint8_t* methods_out, int* kept, void* workspace,
                          size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(num_components >= 0, "bad component count");
    SPX_REQUIRE(refine >= SPX_REFINE_NONE && refine <= SPX_REFINE_AUTO, "bad refine method");
    SPX_REQUIRE(kept && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_select_workspace_bytes(num_components), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (num_components == 0) {
        SPX_CUDA(cudaMemsetAsync(kept, 0, sizeof(int), s));
        return SPX_OK;
    }
    SPX_REQUIRE(stats && rows_out && methods_out, "null pointer");
    Arena a(workspace);
    int* flags = a.take<int>(num_components);
    int* scratch = a.take<int>(scan_scratch_ints(num_components));
    k_select_flags<<<grid_for(num_components, 256), 256, 0, s>>>(stats, num_components, area_min,
                                                                  area_max, flags);
    if (int e = check_launch("k_select_flags")) return e;
    if (int e = exclusive_scan(flags, num_components, flags, kept, scratch, s)) return e;
    k_select_rows<<<grid_for(num_components, 256), 256, 0, s>>>(
        stats, num_components, area_min, area_max, refine, small_feature_max, flags, rows_out, methods_out);
    return check_launch("k_select_rows");
}

int spx_component_rows(const int* stats, const double* centroids, int num_components, int area_min, int area_max,
                       int width, int height, double* rows_out, int* ids_out, uint8_t* interior_out,
                       uint8_t* oversized_out, int* counts_out, void* workspace, size_t workspace_bytes,
                       void* stream) {
    SPX_REQUIRE(num_components >= 0 && width > 0 && height > 0, "bad arguments");
    SPX_REQUIRE(counts_out && oversized_out && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_select_workspace_bytes(num_components), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SPX_CUDA(cudaMemsetAsync(counts_out, 0, 2 * sizeof(int), s));
    if (num_components == 0) {
        SPX_CUDA(cudaMemsetAsync(oversized_out, 0, 1, s));
        return SPX_OK;
    }
    SPX_REQUIRE(stats && centroids && rows_out && ids_out && interior_out, "null pointer");
    Arena a(workspace);
    int* flags = a.take<int>(num_components);
    int* scratch = a.take<int>(scan_scratch_ints(num_components));
    k_select_flags<<<grid_for(num_components, 256), 256, 0, s>>>(stats, num_components, area_min, area_max, flags);
    if (int e = check_launch("k_select_flags")) return e;
    if (int e = exclusive_scan(flags, num_components, flags, counts_out, scratch, s)) return e;
    k_component_rows<<<grid_for(num_components, 256), 256, 0, s>>>(stats, centroids, num_components, area_min,
                                                                    area_max, width, height, flags, rows_out, ids_out,
                                                                    interior_out, oversized_out, counts_out + 1);
    return check_launch("k_component_rows");
}

int spx_refine_centers(const void* img, int dtype, int height, int width, const int* labels,
                       const int* rows, const uint8_t* methods, int n, int pad,
                       double* centers_out, void* stream) {
    SPX_REQUIRE(n >= 0 && pad >= 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(img && labels && rows && methods && centers_out, "null pointer");
    SPX_REQUIRE(dtype >= SPX_U8 && dtype <= SPX_F64, "bad dtype");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
    return launch_refine(img, dtype, height, width, labels, rows, methods, n, nullptr, pad, centers_out, blocks, s);
}

int spx_refine_centers_counted(const void* img, int dtype, int height, int width, const int* labels,
                               const int* rows, const uint8_t* methods, const int* n_dev, int capacity, int pad,
                               double* centers_out, void* stream) {
    SPX_REQUIRE(capacity >= 0 && pad >= 0, "bad arguments");
    if (capacity == 0) return SPX_OK;
    SPX_REQUIRE(img && labels && rows && methods && n_dev && centers_out, "null pointer");
    SPX_REQUIRE(dtype >= SPX_U8 && dtype <= SPX_F64, "bad dtype");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = (capacity + kWarpsPerBlock - 1) / kWarpsPerBlock;
    return launch_refine(img, dtype, height, width, labels, rows, methods, capacity, n_dev, pad, centers_out, blocks,
                         s);
}

}  // extern "C"
