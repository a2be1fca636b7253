// CD measurements of deblended cells, one warp per cell (every per-cell step on the device).
//
// Reference: subpx/_cpu/cd.py — _inside (19-25), _geometry (35-47), _logquad (50-89),
// _half_max_ellipse (92-107), _ellipse_geometry (131-141), gaussian_method (144-192),
// _radial_profiles (195-217), _radial_contour (220-264), measure_cells (267-322); the GPU
// reference's ray kernel subpx/_gpu/cd.py:31-131 for the streaming form of the ray rules.
//
// The symmetric 2x2 eigen-decomposition follows LAPACK's published dsyevd path for n = 2 (dsteqr:
// the deflation tests, then dlaev2, then ascending order), so eigenvector signs, and with them the
// contour vertex order and angle_deg, agree with numpy.linalg.eigh. The cubic B-spline profiles
// use Unser's recursive prefilter (pole sqrt(3) - 2) over the cell padded by 12 edge pixels, as
// scipy.ndimage.map_coordinates(order=3, mode="nearest") does, and scipy's cubic weights.

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "lm.cuh"
#include "select.cuh"

namespace spx {
namespace {

constexpr double kFwhmK = 1.1774100225154747;  // sqrt(2 ln 2)
constexpr double kPi = 3.141592653589793;
constexpr int kPad = 12;

// ------------------------------------------------------------------------------ 2x2 eigh

struct Eig2 {
    double w0, w1;          // ascending eigenvalues
    double v00, v10;        // eigenvector of w0 (column 0: axes[0][0], axes[1][0])
    double v01, v11;        // eigenvector of w1
};

// dlaev2(a, b, c): rt1 (larger in absolute value), rt2 and (cs1, sn1), the unit eigenvector of rt1.
__device__ void dlaev2(double a, double b, double c, double* rt1, double* rt2, double* cs1, double* sn1) {
    const double sm = __dadd_rn(a, c), df = __dsub_rn(a, c), adf = fabs(df);
    const double tb = __dadd_rn(b, b), ab = fabs(tb);
    double acmx, acmn;
    if (fabs(a) > fabs(c)) { acmx = a; acmn = c; } else { acmx = c; acmn = a; }
    double rt;
    if (adf > ab) { const double q = __ddiv_rn(ab, adf); rt = __dmul_rn(adf, sqrt(__dadd_rn(1.0, __dmul_rn(q, q)))); }
    else if (adf < ab) { const double q = __ddiv_rn(adf, ab); rt = __dmul_rn(ab, sqrt(__dadd_rn(1.0, __dmul_rn(q, q)))); }
    else rt = __dmul_rn(ab, sqrt(2.0));
    int sgn1;
    if (sm < 0.0) {
        *rt1 = __dmul_rn(0.5, __dsub_rn(sm, rt));
        sgn1 = -1;
        *rt2 = __dsub_rn(__dmul_rn(__ddiv_rn(acmx, *rt1), acmn), __dmul_rn(__ddiv_rn(b, *rt1), b));
    } else if (sm > 0.0) {
        *rt1 = __dmul_rn(0.5, __dadd_rn(sm, rt));
        sgn1 = 1;
        *rt2 = __dsub_rn(__dmul_rn(__ddiv_rn(acmx, *rt1), acmn), __dmul_rn(__ddiv_rn(b, *rt1), b));
    } else {
        *rt1 = __dmul_rn(0.5, rt);
        *rt2 = __dmul_rn(-0.5, rt);
        sgn1 = 1;
    }
    int sgn2;
    double cs;
    if (df >= 0.0) { cs = __dadd_rn(df, rt); sgn2 = 1; } else { cs = __dsub_rn(df, rt); sgn2 = -1; }
    const double acs = fabs(cs);
    if (acs > ab) {
        const double ct = __ddiv_rn(-tb, cs);
        *sn1 = __ddiv_rn(1.0, sqrt(__dadd_rn(1.0, __dmul_rn(ct, ct))));
        *cs1 = __dmul_rn(ct, *sn1);
    } else if (ab == 0.0) {
        *cs1 = 1.0;
        *sn1 = 0.0;
    } else {
        const double tn = __ddiv_rn(-cs, tb);
        *cs1 = __ddiv_rn(1.0, sqrt(__dadd_rn(1.0, __dmul_rn(tn, tn))));
        *sn1 = __dmul_rn(tn, *cs1);
    }
    if (sgn1 == sgn2) {
        const double tn = *cs1;
        *cs1 = -*sn1;
        *sn1 = tn;
    }
}

// numpy.linalg.eigh of [[a, b], [b, c]] (dsyevd, lower): eigenvalues ascending, columns of V.
__device__ Eig2 eigh2(double a, double b, double c) {
    const double eps = 1.1102230246251565e-16;      // dlamch('E')
    const double safmin = 2.2250738585072014e-308;  // dlamch('S')
    double d0 = a, d1 = c;
    double z00 = 1.0, z01 = 0.0, z10 = 0.0, z11 = 1.0;
    const double e = b;
    // Initial splitting test of dsteqr.
    bool split = e == 0.0 || fabs(e) <= __dmul_rn(__dmul_rn(sqrt(fabs(d0)), sqrt(fabs(d1))), eps);
    if (!split) {
        // QL when |d1| >= |d0|, QR otherwise; both test e^2 <= eps^2 |d_m| |d_m+1| + safmin and else
        // rotate the 2x2 block with dlaev2 into (rt1, rt2) with vectors (cs, sn), (-sn, cs).
        const double tst = __dmul_rn(fabs(e), fabs(e));
        const double bound = (fabs(d1) < fabs(d0))
                                 ? __dadd_rn(__dmul_rn(__dmul_rn(eps * eps, fabs(d1)), fabs(d0)), safmin)
                                 : __dadd_rn(__dmul_rn(__dmul_rn(eps * eps, fabs(d0)), fabs(d1)), safmin);
        if (!(tst <= bound)) {
            double rt1, rt2, cs, sn;
            dlaev2(d0, e, d1, &rt1, &rt2, &cs, &sn);
            d0 = rt1;
            d1 = rt2;
            z00 = cs; z10 = sn;    // column 0
            z01 = -sn; z11 = cs;   // column 1
        }
    }
    Eig2 r;
    if (d1 < d0) {  // selection sort: ascending, columns swapped with their values
        r.w0 = d1; r.w1 = d0;
        r.v00 = z01; r.v10 = z11; r.v01 = z00; r.v11 = z10;
    } else {
        r.w0 = d0; r.w1 = d1;
        r.v00 = z00; r.v10 = z10; r.v01 = z01; r.v11 = z11;
    }
    return r;
}

// ---------------------------------------------------------------------------- shared pieces

struct CellView {
    const double* roi;  // hm x wm cleaned cell (zero outside its mask)
    const int* vor;
    int4 box;
    int j;              // cell index in the Voronoi labels
    int W, hm, wm;
    __device__ __forceinline__ bool mask(int yy, int xx) const {
        return yy >= 0 && xx >= 0 && yy < box.w && xx < box.z && yy < hm && xx < wm &&
               vor[(long long)(box.y + yy) * W + (box.x + xx)] == j;
    }
};

// Output slots of one method (per cell arrays; null pointers are skipped).
struct MethodOut {
    double* centers;     // n x 2 global
    double* contours;    // n x (n_angles + 1) x 2 global, or null (metrics_only)
    uint8_t* status;     // n
    double* metrics;     // n x n_metrics, NaN where not measured
    double* center_local;  // n x 2 (radial, logquad)
    double* edge_px;     // n x n_angles (radial)
    double* eigenvalues; // n x 2 (ellipse methods)
    double* axes;        // n x 2 x 2 (ellipse methods)
    int n_metrics;
    long long col_stride;  // 0: row-major metrics; else metric q of cell i at metrics[i + q * col_stride]
    __device__ __forceinline__ struct MetricRow row(long long i) const;
};

// One cell's metrics, row-major or column-major.
struct MetricRow {
    double* p;
    long long step;
    __device__ __forceinline__ double& operator[](int q) const { return p[q * step]; }
};

__device__ __forceinline__ MetricRow MethodOut::row(long long i) const {
    return col_stride ? MetricRow{metrics + i, col_stride} : MetricRow{metrics + i * n_metrics, 1};
}

// Metric columns (same order as the Python side).
enum {
    M_AREA = 0, M_CD_EQ = 1, M_CD_X = 2, M_CD_Y = 3, M_PERIM = 4, M_BACKGROUND = 5, M_PEAK = 6,
    // ellipse methods
    M_SIG_MAJ = 7, M_SIG_MIN = 8, M_FWHM_MAJ = 9, M_FWHM_MIN = 10, M_ANGLE = 11, M_RMSE = 12,
    // area methods
    M_LOCAL_LEVEL = 7, M_THRESHOLD = 8, M_MEAN_SIGNAL = 9, M_STEEPEST = 10,
    // radial methods
    M_COVERAGE = 7
};

// Half-maximum ellipse: contour vertex k of center + (cos t_k, sin t_k) * (K sigma) @ axes^T.
__device__ __forceinline__ void ellipse_vertex(double cx, double cy, const Eig2& e, double s0, double s1, double ang,
                                               double* px, double* py) {
    const double u = __dmul_rn(cos(ang), __dmul_rn(kFwhmK, s0));
    const double v = __dmul_rn(sin(ang), __dmul_rn(kFwhmK, s1));
    // (u, v) @ axes^T: x = u axes[0][0] + v axes[0][1]; y = u axes[1][0] + v axes[1][1]
    *px = __dadd_rn(cx, __dadd_rn(__dmul_rn(u, e.v00), __dmul_rn(v, e.v01)));
    *py = __dadd_rn(cy, __dadd_rn(__dmul_rn(u, e.v10), __dmul_rn(v, e.v11)));
}

// Warp-wide polygon geometry of the closed contour (n_angles + 1 vertices): shoelace area about
// the first vertex, perimeter, x and y extents. Vertices come from `vertex(k, &x, &y)`.
template <typename V>
__device__ void polygon_geometry(int nv, V vertex, int lane, double* area, double* perim, double* ptpx,
                                 double* ptpy) {
    double x0, y0;
    vertex(0, &x0, &y0);
    double s = 0.0, p = 0.0, xmn = dinf(), xmx = -dinf(), ymn = dinf(), ymx = -dinf();
    for (int k = lane; k < nv - 1; k += 32) {
        double xa, ya, xb, yb;
        vertex(k, &xa, &ya);
        vertex(k + 1, &xb, &yb);
        const double ax = xa - x0, ay = ya - y0, bx = xb - x0, by = yb - y0;
        s += ax * by - bx * ay;
        p += sqrt((xb - xa) * (xb - xa) + (yb - ya) * (yb - ya));
        xmn = fmin(xmn, xa); xmx = fmax(xmx, xa); ymn = fmin(ymn, ya); ymx = fmax(ymx, ya);
    }
    if (lane == 0) {  // the closing vertex
        double xa, ya;
        vertex(nv - 1, &xa, &ya);
        xmn = fmin(xmn, xa); xmx = fmax(xmx, xa); ymn = fmin(ymn, ya); ymx = fmax(ymx, ya);
    }
    s = warp_sum(s);
    p = warp_sum(p);
    *area = fabs(s) / 2.0;
    *perim = p;
    *ptpx = warp_max(xmx) - warp_min(xmn);
    *ptpy = warp_max(ymx) - warp_min(ymn);
}

// map_coordinates(mask, order=1, mode='constant') >= 1 - 1e-8 (_inside).
__device__ __forceinline__ bool inside_bilinear(const CellView& c, bool eroded, double y, double x) {
    const double h1 = (double)(c.hm - 1), w1 = (double)(c.wm - 1);
    if (!(y >= 0.0 && y <= h1 && x >= 0.0 && x <= w1)) return false;
    const double fy = floor(y), fx = floor(x);
    const int y0 = (int)fy, x0 = (int)fx;
    const int ny = (y == fy) ? 1 : 2, nx = (x == fx) ? 1 : 2;
    double v = 0.0;
    for (int a = 0; a < ny; ++a) {
        const double wy = a == 0 ? (fy + 1.0) - y : y - fy;
        for (int b = 0; b < nx; ++b) {
            const double wx = b == 0 ? (fx + 1.0) - x : x - fx;
            bool m;
            const int yy = y0 + a, xx = x0 + b;
            if (eroded) {  // binary_erosion with the cross structure, border 0
                m = c.mask(yy, xx) && yy > 0 && xx > 0 && yy < c.hm - 1 && xx < c.wm - 1 && c.mask(yy - 1, xx) &&
                    c.mask(yy + 1, xx) && c.mask(yy, xx - 1) && c.mask(yy, xx + 1);
            } else {
                m = c.mask(yy, xx);
            }
            v += (m ? 1.0 : 0.0) * (wy * wx);
        }
    }
    return v >= 1.0 - 1e-8;
}

// The same test on a byte mask staged in shared memory (hm x wm).
__device__ __forceinline__ bool inside_bytes(const uint8_t* m, int hm, int wm, double y, double x) {
    if (!(y >= 0.0 && y <= (double)(hm - 1) && x >= 0.0 && x <= (double)(wm - 1))) return false;
    const double fy = floor(y), fx = floor(x);
    const int y0 = (int)fy, x0 = (int)fx;
    const int ny = (y == fy) ? 1 : 2, nx = (x == fx) ? 1 : 2;
    double v = 0.0;
    for (int a = 0; a < ny; ++a) {
        const double wy = a == 0 ? (fy + 1.0) - y : y - fy;
        for (int b = 0; b < nx; ++b) {
            const double wx = b == 0 ? (fx + 1.0) - x : x - fx;
            v += (m[(y0 + a) * wm + x0 + b] ? 1.0 : 0.0) * (wy * wx);
        }
    }
    return v >= 1.0 - 1e-8;
}

// ---------------------------------------------------------------------- gaussian method

// gaussian_method: params ROI-local; status in/out (non_gaussian_fit for eig0 <= 1e-10).
__global__ void k_gaussian_method(const double* params, const uint8_t* status_in, const double* cleaned,
                                  const int* vor, const int4* boxes, const int* which, int n, int hm, int wm,
                                  int W, int n_angles, MethodOut out) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int i = blockIdx.x * warps + (threadIdx.x >> 5); i < n; i += gridDim.x * warps) {
        const int j = which ? which[i] : i;
        const double* p = params + 6LL * j;
        const CellView c{cleaned + (long long)i * hm * wm, vor, boxes[j], j, W, hm, wm};
        // fit_rmse over the mask, untruncated model.
        const double e1 = exp(p[3]), e3 = exp(p[5]);
        double ss = 0.0;
        int cnt = 0;
        for (int k = lane; k < hm * wm; k += 32) {
            const int yy = k / wm, xx = k % wm;
            if (!c.mask(yy, xx)) continue;
            const GaussEval g = gauss_eval(p, e1, e3, (double)xx - p[1], (double)yy - p[2]);
            const double r = c.roi[k] - p[0] * g.shape;
            ss += r * r;
            ++cnt;
        }
        ss = warp_sum(ss);
        cnt = warp_sum_i(cnt);
        const MetricRow m = out.row(i);
        uint8_t st = status_in[j];
        bool finite = true;
        for (int q = 0; q < 6; ++q) finite = finite && isfinite(p[q]);
        const int nv = n_angles + 1;
        if (lane == 0) {
            for (int q = 0; q < out.n_metrics; ++q) m[q] = dnan();
            m[M_PEAK] = p[0];
            m[M_RMSE] = sqrt(ss / (double)max(cnt, 1));
            out.centers[2LL * i] = out.centers[2LL * i + 1] = dnan();
            if (out.eigenvalues) {
                out.eigenvalues[2LL * i] = out.eigenvalues[2LL * i + 1] = dnan();
                for (int q = 0; q < 4; ++q) out.axes[4LL * i + q] = dnan();
            }
        }
        if (out.contours)
            for (int k = lane; k < 2 * nv; k += 32) out.contours[(long long)i * 2 * nv + k] = dnan();
        if (!finite) {
            if (lane == 0) out.status[i] = st;
            continue;
        }
        const double cx = p[1] + c.box.x, cy = p[2] + c.box.y;
        // precision = L L^T.
        const double pa = e1 * e1, pb = e1 * p[4], pc = p[4] * p[4] + e3 * e3;
        const Eig2 e = eigh2(pa, pb, pc);
        if (lane == 0) { out.centers[2LL * i] = cx; out.centers[2LL * i + 1] = cy; }
        if (e.w0 <= 1e-10) {
            if (lane == 0) out.status[i] = SPX_ST_NON_GAUSSIAN_FIT;
            continue;
        }
        const double s0 = 1.0 / sqrt(e.w0), s1 = 1.0 / sqrt(e.w1);
        const double step = 2.0 * kPi / n_angles;
        auto vertex = [&](int k, double* x, double* y) {
            ellipse_vertex(cx, cy, e, s0, s1, (double)(k % n_angles) * step, x, y);
        };
        if (out.contours)
            for (int k = lane; k < nv; k += 32) {
                double x, y;
                vertex(k, &x, &y);
                out.contours[(long long)i * 2 * nv + 2 * k] = x;
                out.contours[(long long)i * 2 * nv + 2 * k + 1] = y;
            }
        double area = 0, perim = 0, px = 0, py = 0;
        if (out.contours) polygon_geometry(nv, vertex, lane, &area, &perim, &px, &py);
        if (lane == 0) {
            if (out.eigenvalues) {
                out.eigenvalues[2LL * i] = e.w0;
                out.eigenvalues[2LL * i + 1] = e.w1;
                out.axes[4LL * i + 0] = e.v00; out.axes[4LL * i + 1] = e.v01;
                out.axes[4LL * i + 2] = e.v10; out.axes[4LL * i + 3] = e.v11;
            }
            m[M_SIG_MAJ] = s0;
            m[M_SIG_MIN] = s1;
            m[M_FWHM_MAJ] = 2.0 * kFwhmK * s0;
            m[M_FWHM_MIN] = 2.0 * kFwhmK * s1;
            double ang = atan2(e.v10, e.v00) * (180.0 / kPi);
            ang = fmod(ang, 180.0);
            if (ang < 0) ang += 180.0;
            m[M_ANGLE] = ang;
            if (st == SPX_ST_OK) {
                const double ar = kPi * kFwhmK * kFwhmK * (s0 * s1);
                m[M_AREA] = ar;
                m[M_CD_EQ] = 2.0 * sqrt(ar / kPi);
                // covariance = axes diag(sigma^2) axes^T
                const double c00 = e.v00 * e.v00 * s0 * s0 + e.v01 * e.v01 * s1 * s1;
                const double c11 = e.v10 * e.v10 * s0 * s0 + e.v11 * e.v11 * s1 * s1;
                m[M_CD_X] = 2.0 * kFwhmK * sqrt(c00);
                m[M_CD_Y] = 2.0 * kFwhmK * sqrt(c11);
                m[M_PERIM] = out.contours ? perim : dnan();
            }
            out.status[i] = st;
        }
    }
}

// ------------------------------------------------------------------------------ logquad CD

__global__ void k_logquad_cd(const double* cleaned, const int* vor, const int4* boxes, const int* which,
                             const double* seeds, int n, int hm, int wm, int W, int n_angles, double fit_fraction,
                             MethodOut out) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    const double scale = 0.5 * (double)max(hm, wm), inv = 1.0 / scale;
    for (int i = blockIdx.x * warps + (threadIdx.x >> 5); i < n; i += gridDim.x * warps) {
        const int j = which ? which[i] : i;
        const CellView c{cleaned + (long long)i * hm * wm, vor, boxes[j], j, W, hm, wm};
        const double sx = seeds[2LL * j] - c.box.x, sy = seeds[2LL * j + 1] - c.box.y;
        const int nv = n_angles + 1;
        const MetricRow m = out.row(i);
        // Defaults: no_signal, seed centre, NaN geometry.
        if (lane == 0) {
            for (int q = 0; q < out.n_metrics; ++q) m[q] = dnan();
            out.status[i] = SPX_ST_NO_SIGNAL;
            out.centers[2LL * i] = out.centers[2LL * i + 1] = dnan();
            out.center_local[2LL * i] = out.center_local[2LL * i + 1] = dnan();
            out.eigenvalues[2LL * i] = out.eigenvalues[2LL * i + 1] = dnan();
            for (int q = 0; q < 4; ++q) out.axes[4LL * i + q] = dnan();
        }
        if (out.contours)
            for (int k = lane; k < 2 * nv; k += 32) out.contours[(long long)i * 2 * nv + k] = dnan();
        int cnt = 0;
        double peak = -dinf();
        for (int k = lane; k < hm * wm; k += 32) {
            if (!c.mask(k / wm, k % wm)) continue;
            ++cnt;
            peak = fmax(peak, c.roi[k]);
        }
        cnt = warp_sum_i(cnt);
        peak = warp_max(peak);
        if (cnt < 6) {
            if (lane == 0) out.status[i] = SPX_ST_INSUFFICIENT_CELL_PIXELS;
            continue;
        }
        if (!(peak > 0.0)) continue;  // measure_cells skips cells with no signal above the background
        if (lane == 0) {
            m[M_BACKGROUND] = 0.0;
            m[M_PEAK] = peak;
            out.center_local[2LL * i] = sx;
            out.center_local[2LL * i + 1] = sy;
            out.centers[2LL * i] = sx + c.box.x;
            out.centers[2LL * i + 1] = sy + c.box.y;
        }
        // Weighted sums of the log-quadratic least squares in seed-centred coordinates / scale.
        double acc[28];
#pragma unroll
        for (int q = 0; q < 28; ++q) acc[q] = 0.0;
        for (int k = lane; k < hm * wm; k += 32) {
            const int yy = k / wm, xx = k % wm;
            const double s = c.roi[k];
            if (!c.mask(yy, xx) || !(s > fit_fraction * peak)) continue;
            const double wt = s / peak, w2 = wt * wt, z = log(s);
            const double u = ((double)xx - sx) * inv, v = ((double)yy - sy) * inv;
            const double d[6] = {u * u, v * v, u * v, u, v, 1.0};
            int q = 1;
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int b = a; b < 6; ++b) acc[q++] += w2 * d[a] * d[b];
#pragma unroll
            for (int a = 0; a < 6; ++a) acc[22 + a] += w2 * d[a] * z;
            acc[0] += 1.0;
        }
#pragma unroll
        for (int q = 0; q < 28; ++q) acc[q] = warp_sum(acc[q]);
        if (acc[0] < 6.0) {
            if (lane == 0) out.status[i] = SPX_ST_INSUFFICIENT_FIT_PIXELS;
            continue;
        }
        // Cholesky of the normal matrix; a pivot below 1e-12 of the largest diagonal is rank
        // deficiency (lstsq rank < 6).
        double A[6][6], b[6];
        {
            int q = 1;
            for (int a = 0; a < 6; ++a)
                for (int bb = a; bb < 6; ++bb) { A[a][bb] = A[bb][a] = acc[q++]; }
            for (int a = 0; a < 6; ++a) b[a] = acc[22 + a];
        }
        double dmax = 0.0;
        for (int a = 0; a < 6; ++a) dmax = fmax(dmax, A[a][a]);
        bool singular = false;
        double L[6][6];
        for (int r = 0; r < 6; ++r)
            for (int col = 0; col <= r; ++col) {
                double v = A[r][col];
                for (int k = 0; k < col; ++k) v -= L[r][k] * L[col][k];
                if (r == col) {
                    if (!(v > 1e-12 * dmax)) singular = true;
                    L[r][r] = sqrt(fmax(v, 1e-300));
                } else {
                    L[r][col] = v / L[col][col];
                }
            }
        if (singular) {
            if (lane == 0) out.status[i] = SPX_ST_SINGULAR_FIT;
            continue;
        }
        double yv[6], cf[6];
        for (int r = 0; r < 6; ++r) {
            double v = b[r];
            for (int k = 0; k < r; ++k) v -= L[r][k] * yv[k];
            yv[r] = v / L[r][r];
        }
        for (int r = 5; r >= 0; --r) {
            double v = yv[r];
            for (int k = r + 1; k < 6; ++k) v -= L[k][r] * cf[k];
            cf[r] = v / L[r][r];
        }
        // Back to pixel units.
        const double ca = cf[0] / (scale * scale), cb = cf[1] / (scale * scale), cc = cf[2] / (scale * scale);
        const double cd = cf[3] / scale, ce = cf[4] / scale;
        const double pa = -2.0 * ca, pb = -cc, pc = -2.0 * cb;  // precision = -[[2a, c], [c, 2b]]
        const Eig2 e = eigh2(pa, pb, pc);
        if (e.w0 <= 1e-10 || e.w1 / e.w0 > 1e8) {
            if (lane == 0) out.status[i] = SPX_ST_NON_GAUSSIAN_FIT;
            continue;
        }
        // offset = solve(precision, [d, e]).
        const double det = pa * pc - pb * pb;
        const double ox = (cd * pc - pb * ce) / det, oy = (pa * ce - pb * cd) / det;
        const double lx = sx + ox, ly = sy + oy;
        const double gx = lx + c.box.x, gy = ly + c.box.y;
        const double s0 = 1.0 / sqrt(e.w0), s1 = 1.0 / sqrt(e.w1);
        const double step = 2.0 * kPi / n_angles;
        auto lvertex = [&](int k, double* x, double* y) {
            ellipse_vertex(lx, ly, e, s0, s1, (double)(k % n_angles) * step, x, y);
        };
        // log_fit_rmse (weights w^2) of the solved fit.
        double rr = 0.0, ww = 0.0;
        for (int k = lane; k < hm * wm; k += 32) {
            const int yy = k / wm, xx = k % wm;
            const double s = c.roi[k];
            if (!c.mask(yy, xx) || !(s > fit_fraction * peak)) continue;
            const double wt = s / peak, w2 = wt * wt;
            const double u = ((double)xx - sx) * inv, v = ((double)yy - sy) * inv;
            const double fit = cf[0] * u * u + cf[1] * v * v + cf[2] * u * v + cf[3] * u + cf[4] * v + cf[5];
            const double d = fit - log(s);
            rr += w2 * d * d;
            ww += w2;
        }
        rr = warp_sum(rr);
        ww = warp_sum(ww);
        // Centre and contour inside the cell mask.
        bool inside = true;
        for (int k = lane; k < nv; k += 32) {
            double x, y;
            lvertex(k, &x, &y);
            inside = inside && inside_bilinear(c, false, y, x);
        }
        inside = __all_sync(0xffffffffu, inside) && inside_bilinear(c, false, ly, lx);
        if (out.contours)
            for (int k = lane; k < nv; k += 32) {
                double x, y;
                lvertex(k, &x, &y);
                out.contours[(long long)i * 2 * nv + 2 * k] = x + c.box.x;
                out.contours[(long long)i * 2 * nv + 2 * k + 1] = y + c.box.y;
            }
        double area = 0, perim = 0, px = 0, py = 0;
        polygon_geometry(nv, lvertex, lane, &area, &perim, &px, &py);
        if (lane == 0) {
            out.center_local[2LL * i] = lx;
            out.center_local[2LL * i + 1] = ly;
            out.centers[2LL * i] = gx;
            out.centers[2LL * i + 1] = gy;
            out.eigenvalues[2LL * i] = e.w0;
            out.eigenvalues[2LL * i + 1] = e.w1;
            out.axes[4LL * i + 0] = e.v00; out.axes[4LL * i + 1] = e.v01;
            out.axes[4LL * i + 2] = e.v10; out.axes[4LL * i + 3] = e.v11;
            m[M_SIG_MAJ] = s0;
            m[M_SIG_MIN] = s1;
            m[M_FWHM_MAJ] = 2.0 * kFwhmK * s0;
            m[M_FWHM_MIN] = 2.0 * kFwhmK * s1;
            double ang = atan2(e.v10, e.v00) * (180.0 / kPi);
            ang = fmod(ang, 180.0);
            if (ang < 0) ang += 180.0;
            m[M_ANGLE] = ang;
            m[M_RMSE] = sqrt(rr / ww);
            if (!inside) {
                out.status[i] = SPX_ST_CONTOUR_OUTSIDE_CELL;
            } else {
                const double ar = kPi * kFwhmK * kFwhmK * (s0 * s1);
                m[M_AREA] = ar;
                m[M_CD_EQ] = 2.0 * sqrt(ar / kPi);
                const double c00 = e.v00 * e.v00 * s0 * s0 + e.v01 * e.v01 * s1 * s1;
                const double c11 = e.v10 * e.v10 * s0 * s0 + e.v11 * e.v11 * s1 * s1;
                m[M_CD_X] = 2.0 * kFwhmK * sqrt(c00);
                m[M_CD_Y] = 2.0 * kFwhmK * sqrt(c11);
                m[M_PERIM] = perim;
                out.status[i] = SPX_ST_OK;
            }
        }
    }
}

// ------------------------------------------------------------------------------ radial CD

// Unser's causal/anticausal recursion for the cubic B-spline (pole z = sqrt(3) - 2) over one line
// of n values with stride, the gain applied first, half-sample-symmetric initial conditions.
__device__ void spline_line(double* c, int n, int stride) {
    const double z = -0.2679491924311228;  // sqrt(3) - 2
    const double gain = (1.0 - z) * (1.0 - 1.0 / z);
    for (int i = 0; i < n; ++i) c[i * stride] *= gain;
    if (n == 1) return;
    // causal init
    {
        double zi = z;
        const double zn = pow(z, (double)n);
        const double c0 = c[0];
        double acc = c[0] + zn * c[(n - 1) * stride];
        for (int i = 1; i < n; ++i) {
            acc += zi * (c[i * stride] + zn * c[(n - 1 - i) * stride]);
            zi *= z;
        }
        acc *= z / (1.0 - zn * zn);
        c[0] = acc + c0;
    }
    for (int i = 1; i < n; ++i) c[i * stride] += z * c[(i - 1) * stride];
    c[(n - 1) * stride] *= z / (z - 1.0);
    for (int i = n - 2; i >= 0; --i) c[i * stride] = z * (c[(i + 1) * stride] - c[i * stride]);
}

// x / 6, correctly rounded, by Markstein's correction of x * RN(1/6) with one FMA (checked against
// exact rational division on 600k operands spanning the double range).
__device__ __forceinline__ double div6(double x) {
    const double c = 0.16666666666666666;  // RN(1/6)
    const double q = __dmul_rn(x, c);
    return __fma_rn(__fma_rn(-q, 6.0, x), c, q);
}

// scipy's order-3 interpolation weights at fractional offset t = v - floor(v).
__device__ __forceinline__ void cubic_weights_t(double t, double* w) {
    const double s = 1.0 - t;
    w[1] = div6(t * t * (t - 2.0) * 3.0 + 4.0);
    w[2] = div6(s * s * (s - 2.0) * 3.0 + 4.0);
    w[0] = div6(s * s * s);
    w[3] = 1.0 - w[0] - w[1] - w[2];
}

// scipy's order-3 interpolation weights and clamped ("nearest") indices at coordinate v.
__device__ __forceinline__ void cubic_weights(double v, int n, double* w, int* idx) {
    const double f = floor(v);
    cubic_weights_t(v - f, w);
    for (int k = 0; k < 4; ++k) idx[k] = min(max((int)f - 1 + k, 0), n - 1);
}

__device__ __forceinline__ double cubic_at(const double* coef, int hp, int wp, int pitch, double y, double x) {
    double wy[4], wx[4];
    int iy[4], ix[4];
    cubic_weights(y, hp, wy, iy);
    cubic_weights(x, wp, wx, ix);
    double out = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) out += coef[iy[a] * pitch + ix[b]] * wy[a] * wx[b];
    return out;
}

// cubic_at for a position whose 4 x 4 window lies inside the plane (no index clamps needed): the same
// weights, products and order of additions, so the same value.
__device__ __forceinline__ double cubic_at_inner(const double* coef, int pitch, double y, double x) {
    const double fy = floor(y), fx = floor(x);
    double wy[4], wx[4];
    cubic_weights_t(y - fy, wy);
    cubic_weights_t(x - fx, wx);
    const double* q = coef + ((int)fy - 1) * pitch + ((int)fx - 1);
    double out = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) out += q[a * pitch + b] * wy[a] * wx[b];
    return out;
}

// The same window evaluated in FP32 (weights, products and sums), the sampling precision the ray
// profiles use, from an FP32 copy of the coefficients: sample positions stay FP64 and only their
// fractional offsets inside the window are rounded to FP32, so a sample differs from the FP64
// evaluation by ~1e-7 relative. The caller passes the window's integer cell and the offsets.
struct SplineWindowF {
    int fy = -1 << 30, fx = -1 << 30;
    float c[16];
    __device__ __forceinline__ static void weights(float t, float* w) {
        const float s = 1.0f - t;
        const float k = 1.0f / 6.0f;
        w[1] = (t * t * (t - 2.0f) * 3.0f + 4.0f) * k;
        w[2] = (s * s * (s - 2.0f) * 3.0f + 4.0f) * k;
        w[0] = s * s * s * k;
        w[3] = 1.0f - w[0] - w[1] - w[2];
    }
    // (iy, ix): the sample's cell in box coordinates (0 <= iy < hm, 0 <= ix < wm); the window is the
    // four float4 rows quad[(iy + a) * wm + ix], a = 0..3 (radial_quad_offset).
    __device__ __forceinline__ float at(const float4* quad, int wm, int iy, int ix, float ty, float tx) {
        if (iy != fy || ix != fx) {
            fy = iy;
            fx = ix;
            const float4* q = quad + iy * wm + ix;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const float4 t = q[a * wm];
                c[a * 4 + 0] = t.x;
                c[a * 4 + 1] = t.y;
                c[a * 4 + 2] = t.z;
                c[a * 4 + 3] = t.w;
            }
        }
        float wy[4], wx[4];
        weights(ty, wy);
        weights(tx, wx);
        float out = 0.0f;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            float row = 0.0f;
#pragma unroll
            for (int b = 0; b < 4; ++b) row = fmaf(c[a * 4 + b], wx[b], row);
            out = fmaf(row, wy[a], out);
        }
        return out;
    }
};

// One FP32 spline sample from the window rows of box cell (iy, ix): the arithmetic of
// SplineWindowF::at without the cached window.
__device__ __forceinline__ float spline_sample_f(const float4* quad, int wm, int iy, int ix, float ty, float tx) {
    float wy[4], wx[4];
    SplineWindowF::weights(ty, wy);
    SplineWindowF::weights(tx, wx);
    const float4* q = quad + iy * wm + ix;
    float out = 0.0f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const float4 t = q[a * wm];
        float row = 0.0f;
        row = fmaf(t.x, wx[0], row);
        row = fmaf(t.y, wx[1], row);
        row = fmaf(t.z, wx[2], row);
        row = fmaf(t.w, wx[3], row);
        out = fmaf(row, wy[a], out);
    }
    return out;
}

// floor(y) for 0 <= y < 2^51 as an int and as a double, with FP64 additions only (no conversion
// instructions): y + 1.5 * 2^52 holds y rounded to an integer in its low mantissa bits, and one
// comparison turns the rounding into a floor.
__device__ __forceinline__ int floor_nonneg(double y, double* fl) {
    const double magic = 6755399441055744.0;
    const double t = __dadd_rn(y, magic);
    double r = __dsub_rn(t, magic);
    int n = __double2loint(t);
    if (r > y) {
        r -= 1.0;
        n -= 1;
    }
    *fl = r;
    return n;
}

constexpr int kRadialThreads = 128;
constexpr int kTrigMax = 256;  // ray angles with a cos / sin table in shared memory (4 KB)
constexpr int kRewalkQueue = 64;  // rays per cell queued for the warps' FP64 re-walk

// Shared (or scratch) memory of one radial CTA, in doubles: the FP64 spline coefficient plane, the
// FP32 sampling windows, a reduction area, then the cell mask and the eroded mask as bytes.
// Row pitch (in doubles) of the FP64 coefficient plane: the padded width made odd, so that the
// threads of the row pass of the spline prefilter (one row each, stepping along their rows) fall in
// different shared-memory banks.
__host__ __device__ inline int radial_pitch(int wm) { return (wm + 2 * kPad) | 1; }

// The FP32 sampling windows start after the FP64 plane, 16-byte aligned. A ray sample in box cell
// (iy, ix) (0 <= iy < hm, 0 <= ix < wm) reads the 4 x 4 coefficients of padded rows iy + kPad - 1 ..
// iy + kPad + 2 and columns ix + kPad - 1 .. ix + kPad + 2; quad[r * wm + ix] holds the four of padded
// row r + kPad - 1 as one float4, for r = 0 .. hm + 2, so a window is four 16-byte loads.
__host__ __device__ inline long long radial_quad_offset(int hm, int wm) {
    return ((long long)(hm + 2 * kPad) * radial_pitch(wm) + 1) & ~1LL;
}
__host__ __device__ inline long long radial_quad_doubles(int hm, int wm) { return 2LL * (hm + 3) * wm; }

// The masks are three byte planes (cell, eroded cell, and per pixel square whether its four corners
// are all in the eroded cell). With smoothing, three more hm x wm doubles follow (the two axis-0
// passes and the smoothed signal). The total is even, so every CTA's scratch stays 16-byte aligned.
__host__ __device__ inline long long radial_cta_doubles(int hm, int wm, bool smooth = false) {
    const long long t = radial_quad_offset(hm, wm) + radial_quad_doubles(hm, wm) + 32 + (3LL * hm * wm + 7) / 8 +
                        (smooth ? 3LL * hm * wm : 0);
    return (t + 1) & ~1LL;
}

// One output of scipy's correlate1d with a symmetric kernel (weights w[0..2r], centre w[r]) and
// mode="constant" (zero outside 0..n-1): the centre term first, then the pairs outermost inwards.
__device__ __forceinline__ double sym_correlate_zero(const double* v, int pos, int n, int stride, const double* w,
                                                     int r) {
    double t = __dmul_rn(v[pos * stride], w[r]);
    for (int k = r; k >= 1; --k) {
        const double a = pos - k >= 0 ? v[(pos - k) * stride] : 0.0;
        const double b = pos + k < n ? v[(pos + k) * stride] : 0.0;
        t = __dadd_rn(t, __dmul_rn(__dadd_rn(a, b), w[r - k]));
    }
    return t;
}

// Sum over the CTA's 4 warps in a fixed order (the same value on every thread). Slots of `red`
// must not be reused before the next __syncthreads that follows every read.
__device__ __forceinline__ double cta_sum(double v, double* red) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    return ((red[0] + red[1]) + red[2]) + red[3];
}

__device__ __forceinline__ double cta_max(double v, double* red) {
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    return fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
}

// NaN / no_signal defaults of one cell's radial outputs (the CTA's threads share the stores).
__device__ void radial_clear(const MethodOut out, int i, int n_angles) {
    if (!out.status) return;
    const int nv = n_angles + 1;
    if (threadIdx.x == 0) {
        const MetricRow m = out.row(i);
        for (int q = 0; q < out.n_metrics; ++q) m[q] = dnan();
        out.status[i] = SPX_ST_NO_SIGNAL;
        out.centers[2LL * i] = out.centers[2LL * i + 1] = dnan();
        out.center_local[2LL * i] = out.center_local[2LL * i + 1] = dnan();
    }
    for (int k = threadIdx.x; k < n_angles; k += blockDim.x) out.edge_px[(long long)i * n_angles + k] = dnan();
    if (out.contours)
        for (int k = threadIdx.x; k < 2 * nv; k += blockDim.x) out.contours[(long long)i * 2 * nv + k] = dnan();
}

// Contour, polygon geometry and metrics of one method from its edge radii (one warp).
// trig: cos and sin of the n_angles ray angles (interleaved), or null to evaluate them here.
__device__ __noinline__ void radial_finish(const MethodOut out, int found, int i, int n_angles, double cx, double cy,
                                           double peak, int4 box, const double* trig) {
    if (!out.status) return;
    const int lane = threadIdx.x & 31, nv = n_angles + 1;
    const double* edge = out.edge_px + (long long)i * n_angles;
    const double step = 2.0 * kPi / n_angles;
    auto vertex = [&](int k, double* x, double* y) {
        const int a = k % n_angles;
        double c, sn;
        if (trig) {
            c = trig[2 * a];
            sn = trig[2 * a + 1];
        } else {
            const double ang = (double)a * step;
            c = cos(ang);
            sn = sin(ang);
        }
        *x = cx + edge[a] * c;
        *y = cy + edge[a] * sn;
    };
    if (out.contours)
        for (int k = lane; k < nv; k += 32) {
            double x, y;
            vertex(k, &x, &y);
            out.contours[(long long)i * 2 * nv + 2 * k] = x + box.x;
            out.contours[(long long)i * 2 * nv + 2 * k + 1] = y + box.y;
        }
    double area = 0, perim = 0, px = 0, py = 0;
    if (found == n_angles) polygon_geometry(nv, vertex, lane, &area, &perim, &px, &py);
    if (lane == 0) {
        const MetricRow m = out.row(i);
        out.center_local[2LL * i] = cx;
        out.center_local[2LL * i + 1] = cy;
        out.centers[2LL * i] = cx + box.x;
        out.centers[2LL * i + 1] = cy + box.y;
        m[M_BACKGROUND] = 0.0;
        m[M_PEAK] = peak;
        m[M_COVERAGE] = (double)found / n_angles;
        if (found == n_angles) {
            m[M_AREA] = area;
            m[M_CD_EQ] = 2.0 * sqrt(area / kPi);
            m[M_CD_X] = px;
            m[M_CD_Y] = py;
            m[M_PERIM] = perim;
            out.status[i] = SPX_ST_OK;
        } else {
            out.status[i] = SPX_ST_INCOMPLETE_RAYS;
        }
    }
}

// FP64 sample k of a ray (k = 0: the peak): position centre + k step (cos, sin) rounded as the FP32
// walk computes it, and scipy's order-3 evaluation of the FP64 coefficient plane. Not inlined: every
// FP64 sample of the radial kernel runs this one copy of the code, which keeps the kernel's
// instruction footprint small (the walk's loop and this function stay in the instruction cache).
__device__ __noinline__ double ray_sample64(const double* coef, int hp, int wp, int dp, double cx, double cy,
                                            double ux, double uy, double step, int k, double peak) {
    if (k == 0) return peak;
    const double r = (double)k * step;
    const double x = __dadd_rn(cx, __dmul_rn(ux, r)), y = __dadd_rn(cy, __dmul_rn(uy, r));
    return cubic_at_inner(coef, dp, y + kPad, x + kPad);
}

// One ray walked again with FP64 samples (scipy's order-3 evaluation of the FP64 coefficient plane,
// as the peak) and the reference's own arithmetic (subpx/_cpu/cd.py:220-264): the first half-height
// crossing (p[j] >= half > p[j+1], radius j step + (p[j] - half) / (p[j] - p[j+1]) step) and the
// first maximum of the outward decrease grad(j) = -((p[j+1] - p[j-1]) / (2 step)) over the
// candidates, refined by the parabola through grad(j-1), grad(j), grad(j+1). Validity as in the FP32
// walk. Writes the edges asked for (NaN when none).
__device__ __noinline__ void ray_fp64(const double* coef, int hp, int wp, int dp, const uint8_t* emask, int hm, int wm,
                                      double cx, double cy, double ux, double uy, double step, int n_radii,
                                      int j_min, double peak, bool want_h, bool want_g, double* edge_h,
                                      double* edge_g) {
    const double half = peak / 2.0, two_step = 2.0 * step;
    const double ymax = (double)(hm - 1), xmax = (double)(wm - 1);
    double p1 = 0.0, p2 = 0.0;             // p[k-1], p[k-2]
    double ga = 0.0, gb = 0.0;             // grad(k-3), grad(k-2)
    double best = -INFINITY, bl = 0.0, bm = 0.0, br = 0.0;
    int best_j = -1, first_invalid = n_radii;
    double eh = dnan(), eg = dnan();
    bool crossed = false;
    for (int k = 0; k < n_radii; ++k) {
        const double r = (double)k * step;
        const double x = __dadd_rn(cx, __dmul_rn(ux, r)), y = __dadd_rn(cy, __dmul_rn(uy, r));
        if (!(y >= 0.0 && y <= ymax && x >= 0.0 && x <= xmax)) {
            first_invalid = k;
            break;
        }
        double fyd, fxd;
        const int iy = floor_nonneg(y, &fyd), ix = floor_nonneg(x, &fxd);
        const uint8_t* q = emask + iy * wm + ix;
        const bool full4 = iy + 1 < hm && ix + 1 < wm && q[0] && q[1] && q[wm] && q[wm + 1];
        if (!(full4 || inside_bytes(emask, hm, wm, y, x))) {
            first_invalid = k;
            break;
        }
        const double pk = ray_sample64(coef, hp, wp, dp, cx, cy, ux, uy, step, k, peak);
        if (k >= 1 && !crossed && p1 >= half && pk < half) {
            eh = __dadd_rn((double)(k - 1) * step, __dmul_rn(__ddiv_rn(__dsub_rn(p1, half), __dsub_rn(p1, pk)), step));
            crossed = true;
        }
        if (k >= 2) {
            const double gc = -__ddiv_rn(__dsub_rn(pk, p2), two_step);  // grad(k-1)
            const int j = k - 2;  // candidate: samples j-2 .. j+2 valid
            if (k >= 3 && j >= j_min && j <= n_radii - 3 && gb > best) {
                best = gb;
                best_j = j;
                bl = ga;
                bm = gb;
                br = gc;
            }
            ga = gb;
            gb = gc;
        }
        p2 = p1;
        p1 = pk;
    }
    if (best_j >= 0) {
        const int j = best_j;
        const bool left_ok = j - 1 >= j_min;
        const bool right_ok = j + 1 <= n_radii - 3 && j + 3 < first_invalid;
        const double curv = __dadd_rn(__dsub_rn(bl, __dmul_rn(2.0, bm)), br);
        if (left_ok && right_ok && bm >= bl && bm >= br && bm > __dmul_rn(0.01, peak) && curv < -1e-12) {
            double delta = __ddiv_rn(__dmul_rn(0.5, __dsub_rn(bl, br)), curv);
            delta = delta < -0.5 ? -0.5 : (delta > 0.5 ? 0.5 : delta);
            eg = __dadd_rn((double)j * step, __dmul_rn(delta, step));
        }
    }
    if (want_h) *edge_h = eh;
    if (want_g) *edge_g = eg;
}

// ray_fp64 by one warp: the lanes take 32 consecutive samples at a time into `buf` (the warp's part of
// the CTA's FP32 window rows, free once every ray's FP32 walk is done), then find the first
// half-height crossing by ballot and the first maximum of the outward decrease by a warp reduction
// (largest value, lowest index), with ray_fp64's arithmetic. Returns false (nothing written) when the
// valid samples do not fit `cap`; the caller then walks the ray on one thread.
__device__ __noinline__ bool ray_fp64_warp(const double* coef, int hp, int wp, int dp, const uint8_t* emask, int hm,
                                           int wm, double cx, double cy, double ux, double uy, double step,
                                           int n_radii, int j_min, double peak, bool want_h, bool want_g,
                                           double* buf, int cap, double* edge_h, double* edge_g) {
    const int lane = threadIdx.x & 31;
    const double half = peak / 2.0, two_step = 2.0 * step;
    const double ymax = (double)(hm - 1), xmax = (double)(wm - 1);
    int first_invalid = n_radii;
    for (int base = 0; base < n_radii; base += 32) {
        const int k = base + lane;
        bool valid = false;
        double x = 0.0, y = 0.0;
        if (k < n_radii) {
            const double r = (double)k * step;
            x = __dadd_rn(cx, __dmul_rn(ux, r));
            y = __dadd_rn(cy, __dmul_rn(uy, r));
            if (y >= 0.0 && y <= ymax && x >= 0.0 && x <= xmax) {
                double fyd, fxd;
                const int iy = floor_nonneg(y, &fyd), ix = floor_nonneg(x, &fxd);
                const uint8_t* q = emask + iy * wm + ix;
                const bool full4 = iy + 1 < hm && ix + 1 < wm && q[0] && q[1] && q[wm] && q[wm + 1];
                valid = full4 || inside_bytes(emask, hm, wm, y, x);
            }
        }
        const unsigned bad = __ballot_sync(0xffffffffu, !valid);
        const int stop = bad ? base + __ffs(bad) - 1 : n_radii;
        if (min(stop, base + 32) > cap) return false;  // this chunk's valid samples do not fit
        if (valid && k < stop) buf[k] = k == 0 ? peak : cubic_at(coef, hp, wp, dp, y + kPad, x + kPad);
        if (bad) {
            first_invalid = min(stop, n_radii);
            break;
        }
    }
    __syncwarp();
    if (want_h) {
        double e = dnan();
        for (int base = 1; base < first_invalid; base += 32) {
            const int k = base + lane;
            const bool cross = k < first_invalid && buf[k - 1] >= half && buf[k] < half;
            const unsigned hit = __ballot_sync(0xffffffffu, cross);
            if (hit) {
                const int kc = base + __ffs(hit) - 1;
                const double p1 = buf[kc - 1], pk = buf[kc];
                e = __dadd_rn((double)(kc - 1) * step, __dmul_rn(__ddiv_rn(__dsub_rn(p1, half), __dsub_rn(p1, pk)), step));
                break;
            }
        }
        *edge_h = e;
    }
    if (want_g) {
        // Candidates j: j >= max(j_min, 1), j <= n_radii - 3 and sample j + 2 valid.
        const int jlo = max(j_min, 1), jhi = min(n_radii - 3, first_invalid - 3);
        double best = -INFINITY;
        int best_j = 0x7fffffff;
        for (int j = jlo + lane; j <= jhi; j += 32) {
            const double g = -__ddiv_rn(__dsub_rn(buf[j + 1], buf[j - 1]), two_step);
            if (g > best) {
                best = g;
                best_j = j;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oj = __shfl_xor_sync(0xffffffffu, best_j, o);
            if (ob > best || (ob == best && oj < best_j)) {
                best = ob;
                best_j = oj;
            }
        }
        double e = dnan();
        if (best_j != 0x7fffffff) {
            const int j = best_j;
            const bool left_ok = j - 1 >= j_min;
            const bool right_ok = j + 1 <= n_radii - 3 && j + 3 < first_invalid;
            if (left_ok && right_ok) {
                const double bl = -__ddiv_rn(__dsub_rn(buf[j], buf[j - 2]), two_step);
                const double bm = best;
                const double br = -__ddiv_rn(__dsub_rn(buf[j + 2], buf[j]), two_step);
                const double curv = __dadd_rn(__dsub_rn(bl, __dmul_rn(2.0, bm)), br);
                if (bm >= bl && bm >= br && bm > __dmul_rn(0.01, peak) && curv < -1e-12) {
                    double delta = __ddiv_rn(__dmul_rn(0.5, __dsub_rn(bl, br)), curv);
                    delta = delta < -0.5 ? -0.5 : (delta > 0.5 ? 0.5 : delta);
                    e = __dadd_rn((double)j * step, __dmul_rn(delta, step));
                }
            }
        }
        *edge_g = e;
    }
    __syncwarp();
    return true;
}

// The edges of one ray from FP64 samples (scipy's order-3 evaluation of the FP64 coefficient plane)
// at the places the FP32 walk found, with the reference's arithmetic (subpx/_cpu/cd.py:220-264):
// * kc > 0: the half-height crossing between samples kc - 1 and kc (the walk has checked that no
//   earlier sample and neither of these is within its error bound of half height), at radius
//   (kc - 1) step + (p[kc-1] - half) / (p[kc-1] - p[kc]) step;
// * j >= 0: the gradient edge around j, the maximum of the FP32 outward decreases, when every
//   candidate three or more samples from j is clearly below it: candidates j-2 .. j+2 compete with
//   FP64 decreases grad(k) = -((p[k+1] - p[k-1]) / (2 step)) (first maximum wins) and the winner is
//   refined by the parabola through its neighbours, NaN when it fails a test.
// Samples j-3 .. j+3 and the crossing pair (usually among them) are taken once each in one rolled
// loop with the sampler inlined once (this function has one call site); when the winner is j-2 or
// j+2, the two samples of its outer neighbour's decrease are taken again (rare).
__device__ __forceinline__ void ray_edges64(const double* coef, int hp, int wp, int dp, double cx, double cy, double ux,
                                         double uy, double step, double peak, int kc, int j, int j_min, int n_radii,
                                         int first_invalid, double* edge_h, double* edge_g) {
    const double half = peak / 2.0, two_step = 2.0 * step;
    int lo = 1 << 30, hi = -(1 << 30);
    if (kc > 0) {
        lo = kc - 1;
        hi = kc;
    }
    if (j >= 0) {
        lo = min(lo, j - 3);
        hi = max(hi, j + 3);
    }
    double g1 = 0.0, g2 = 0.0, g3 = 0.0, g4 = 0.0, g5 = 0.0;  // grad(j-2) .. grad(j+2)
    double pm1 = 0.0, pm2 = 0.0;                              // p[k-1], p[k-2]
    double c0 = 0.0, c1 = 0.0;                                // p[kc-1], p[kc]
#pragma unroll 1
    for (int k = lo; k <= hi; ++k) {
        const bool in_g = j >= 0 && k >= j - 3 && k <= j + 3;
        const bool in_h = kc > 0 && (k == kc - 1 || k == kc);
        if (!in_g && !in_h) continue;
        double pk = 0.0;
        if (k == 0) {
            pk = peak;
        } else if (k > 0 && k < first_invalid) {
            const double r = (double)k * step;
            const double x = __dadd_rn(cx, __dmul_rn(ux, r)), y = __dadd_rn(cy, __dmul_rn(uy, r));
            pk = cubic_at_inner(coef, dp, y + kPad, x + kPad);
        }
        if (k == kc - 1) c0 = pk;
        if (k == kc) c1 = pk;
        if (in_g) {
            if (k >= j - 1) {  // grad(k - 1)
                g1 = g2;
                g2 = g3;
                g3 = g4;
                g4 = g5;
                g5 = -__ddiv_rn(__dsub_rn(pk, pm2), two_step);
            }
            pm2 = pm1;
            pm1 = pk;
        }
    }
    if (kc > 0) *edge_h = __dadd_rn((double)(kc - 1) * step, __dmul_rn(__ddiv_rn(__dsub_rn(c0, half), __dsub_rn(c0, c1)), step));
    if (j < 0) return;
    *edge_g = dnan();
    const double gs[5] = {g1, g2, g3, g4, g5};
    int tb = -1;
    double mid = 0.0;
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const int k = j - 2 + t;
        const bool cand = k >= j_min && k <= n_radii - 3 && k + 2 < first_invalid;
        if (cand && (tb < 0 || gs[t] > mid)) {
            tb = t;
            mid = gs[t];
        }
    }
    const int jb = j - 2 + tb;
    const bool left_ok = jb - 1 >= j_min;
    const bool right_ok = jb + 1 <= n_radii - 3 && jb + 3 < first_invalid;
    if (!(left_ok && right_ok)) return;
    double left, right;
    if (tb == 0) {  // grad(j - 3) needs samples j - 4 and j - 2
        const double pa = ray_sample64(coef, hp, wp, dp, cx, cy, ux, uy, step, j - 4, peak);
        const double pb = ray_sample64(coef, hp, wp, dp, cx, cy, ux, uy, step, j - 2, peak);
        left = -__ddiv_rn(__dsub_rn(pb, pa), two_step);
        right = g2;
    } else if (tb == 4) {  // grad(j + 3) needs samples j + 2 and j + 4
        const double pa = ray_sample64(coef, hp, wp, dp, cx, cy, ux, uy, step, j + 2, peak);
        const double pb = ray_sample64(coef, hp, wp, dp, cx, cy, ux, uy, step, j + 4, peak);
        left = g4;
        right = -__ddiv_rn(__dsub_rn(pb, pa), two_step);
    } else {
        left = tb == 1 ? g1 : (tb == 2 ? g2 : g3);
        right = tb == 1 ? g3 : (tb == 2 ? g4 : g5);
    }
    const double curv = __dadd_rn(__dsub_rn(left, __dmul_rn(2.0, mid)), right);
    if (!(mid >= left && mid >= right && mid > __dmul_rn(0.01, peak) && curv < -1e-12)) return;
    double delta = __ddiv_rn(__dmul_rn(0.5, __dsub_rn(left, right)), curv);
    delta = delta < -0.5 ? -0.5 : (delta > 0.5 ? 0.5 : delta);
    *edge_g = __dadd_rn((double)jb * step, __dmul_rn(delta, step));
}

// Radial profiles of each cell: weighted centroid of the pixels above 0.1 x max, cubic-spline
// samples every radial_step along n_angles rays until the eroded cell ends, first half-height
// crossing and the parabolic maximum of the outward decrease (halfmax / gradient methods).
// One 128-thread CTA per cell: the cell's masks and spline coefficients are staged once in
// shared memory and each thread walks its own rays.
// kSmooth: the mask-normalised Gaussian smoothing of subpx/_cpu/cd.py:206-208 (smooth_sigma > 0):
// the signal (zero outside the cell) and the mask are each filtered along y then x with zero edges
// (scipy's gaussian_filter, mode="constant"), and the spline is fitted to their ratio over the whole
// cell box; the centroid still comes from the unsmoothed signal.
// kRays: 0 one ray per thread with the 4 x 4 window cached in registers (reloaded when a ray enters
// another pixel), 2 one ray per thread reading the window's four float4 rows at every sample (no
// per-lane reload branch) and the precomputed corner plane; the same samples either way.
// The walk samples in FP32 and finds the first half-height crossing and the largest outward decrease;
// the edges come from FP64 samples at those places (the crossing pair; the decreases two samples
// either side of the maximum, grad_edge64), so they carry the reference's FP64 arithmetic. Where an
// FP32 sample leaves a decision elsewhere within its error bound (a sample near half height before
// the crossing; a candidate three or more samples from the maximum level with it), ray_fp64 walks
// the ray again with FP64 samples and that result is kept.
template <bool kSmooth, int kRays>
__global__ void __launch_bounds__(kRadialThreads, 6) k_radial_cd(
    const double* cleaned, const int* vor, const int4* boxes, const int* which, int n, int hm, int wm, int W,
    int n_angles, double radial_step, int n_radii, const double* smooth_w, int smooth_r, double* coef_scratch,
    MethodOut half_out, MethodOut grad_out) {
    extern __shared__ double sm[];
    __shared__ double trig_tab[2 * kTrigMax];  // cos, sin of the ray angles (n_angles <= kTrigMax)
    __shared__ int s_queue[kRewalkQueue], s_nq;  // rays to walk again in FP64, by warps
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int hp = hm + 2 * kPad, wp = wm + 2 * kPad, dp = radial_pitch(wm), area_px = hm * wm;
    const double* trig = n_angles <= kTrigMax ? trig_tab : nullptr;
    if (trig)
        for (int a = tid; a < n_angles; a += kRadialThreads) {
            const double ang = (double)a * (2.0 * kPi / n_angles);
            trig_tab[2 * a] = cos(ang);
            trig_tab[2 * a + 1] = sin(ang);
        }
    double* coef = coef_scratch ? coef_scratch + (long long)blockIdx.x * radial_cta_doubles(hm, wm, kSmooth) : sm;
    float4* quad = reinterpret_cast<float4*>(coef + radial_quad_offset(hm, wm));  // FP32 window rows
    double* red = coef + radial_quad_offset(hm, wm) + radial_quad_doubles(hm, wm);  // 32 doubles: 8 slots of 4
    uint8_t* mask = reinterpret_cast<uint8_t*>(red + 32);
    uint8_t* emask = mask + area_px;
    uint8_t* full = emask + area_px;  // square [iy, iy+1] x [ix, ix+1] inside the eroded cell
    const double thr = fmax(0.35, 2.0 * radial_step);
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int j = which ? which[i] : i;
        const CellView c{cleaned + (long long)i * area_px, vor, boxes[j], j, W, hm, wm};
        __syncthreads();  // the previous cell's shared-memory reads are done
        radial_clear(half_out, i, n_angles);
        radial_clear(grad_out, i, n_angles);
        int cnt = 0;
        double top = 0.0;  // max of the signal array (zeros outside the mask)
        for (int k = tid; k < area_px; k += kRadialThreads) {
            const bool m = c.mask(k / wm, k % wm);
            mask[k] = m;
            cnt += m;
            top = fmax(top, c.roi[k]);
        }
        const int total = (int)cta_sum((double)cnt, red);
        top = cta_max(top, red + 4);
        if (total < 6) {
            if (tid == 0) {
                if (half_out.status) half_out.status[i] = SPX_ST_INSUFFICIENT_CELL_PIXELS;
                if (grad_out.status) grad_out.status[i] = SPX_ST_INSUFFICIENT_CELL_PIXELS;
            }
            continue;
        }
        if (!(top > 0.0)) continue;
        // Weighted centroid of pixels above 0.1 x max.
        double sw = 0.0, swx = 0.0, swy = 0.0;
        for (int k = tid; k < area_px; k += kRadialThreads) {
            const double s = mask[k] ? c.roi[k] : 0.0;
            if (mask[k] && s > 0.1 * top) {
                sw += s;
                swx += s * (k % wm);
                swy += s * (k / wm);
            }
        }
        sw = cta_sum(sw, red + 8);
        const double cx = cta_sum(swx, red + 12) / sw, cy = cta_sum(swy, red + 16) / sw;
        // Spline coefficients (the cell padded by 12 edge pixels) and the eroded cell (cross
        // structure, zero outside the stack), where ray samples stay valid.
        if constexpr (kSmooth) {
            double* ts = reinterpret_cast<double*>(mask) + (3LL * area_px + 7) / 8;  // after the masks
            double* tm = ts + area_px;
            double* fs = tm + area_px;
            double* sig = coef;  // the masked signal, staged in the coefficient plane (hp * wp >= hm * wm)
            for (int k = tid; k < area_px; k += kRadialThreads) sig[k] = mask[k] ? c.roi[k] : 0.0;
            __syncthreads();
            for (int k = tid; k < area_px; k += kRadialThreads) {
                const int yy = k / wm, xx = k % wm;
                ts[k] = sym_correlate_zero(sig + xx, yy, hm, wm, smooth_w, smooth_r);
                double t = mask[k] ? smooth_w[smooth_r] : 0.0;
                for (int q = smooth_r; q >= 1; --q) {
                    const double a = yy - q >= 0 && mask[k - q * wm] ? 1.0 : 0.0;
                    const double b = yy + q < hm && mask[k + q * wm] ? 1.0 : 0.0;
                    t = __dadd_rn(t, __dmul_rn(__dadd_rn(a, b), smooth_w[smooth_r - q]));
                }
                tm[k] = t;
            }
            __syncthreads();
            for (int k = tid; k < area_px; k += kRadialThreads) {
                const int yy = k / wm, xx = k % wm;
                const double num = sym_correlate_zero(ts + yy * wm, xx, wm, 1, smooth_w, smooth_r);
                const double den = sym_correlate_zero(tm + yy * wm, xx, wm, 1, smooth_w, smooth_r);
                fs[k] = num / fmax(den, 1e-12);
            }
            __syncthreads();
            for (int k = tid; k < hp * wp; k += kRadialThreads) {
                const int r = k / wp, q = k % wp;
                const int yy = min(max(r - kPad, 0), hm - 1), xx = min(max(q - kPad, 0), wm - 1);
                coef[r * dp + q] = fs[yy * wm + xx];
            }
        } else {
            for (int k = tid; k < hp * wp; k += kRadialThreads) {
                const int r = k / wp, q = k % wp;
                const int yy = min(max(r - kPad, 0), hm - 1), xx = min(max(q - kPad, 0), wm - 1);
                coef[r * dp + q] = mask[yy * wm + xx] ? c.roi[yy * wm + xx] : 0.0;
            }
        }
        for (int k = tid; k < area_px; k += kRadialThreads) {
            const int yy = k / wm, xx = k % wm;
            emask[k] = mask[k] && yy > 0 && xx > 0 && yy < hm - 1 && xx < wm - 1 && mask[k - wm] && mask[k + wm] &&
                       mask[k - 1] && mask[k + 1];
        }
        __syncthreads();
        if constexpr (kRays != 0)
            for (int k = tid; k < area_px; k += kRadialThreads) {
                const int yy = k / wm, xx = k % wm;
                full[k] = yy + 1 < hm && xx + 1 < wm && emask[k] && emask[k + 1] && emask[k + wm] && emask[k + wm + 1];
            }
        for (int col = tid; col < wp; col += kRadialThreads) spline_line(coef + col, hp, dp);
        __syncthreads();
        for (int row = tid; row < hp; row += kRadialThreads) spline_line(coef + (long long)row * dp, wp, 1);
        __syncthreads();
        const double peak = cubic_at(coef, hp, wp, dp, cy + kPad, cx + kPad);
        float cmax = 0.0f;  // largest FP32 coefficient magnitude a sample can weigh
        for (int k = tid; k < (hm + 3) * wm; k += kRadialThreads) {
            const double* q = coef + (k / wm + kPad - 1) * dp + (k % wm + kPad - 1);
            const float4 f = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
            quad[k] = f;
            cmax = fmaxf(cmax, fmaxf(fmaxf(fabsf(f.x), fabsf(f.y)), fmaxf(fabsf(f.z), fabsf(f.w))));
        }
        // The window weights are non-negative and sum to one per axis, so an FP32 sample is within about
        // 45 ulps of cmax of the FP64 one (coefficient, offset and weight roundings, 20 FMAs); tol keeps
        // a margin of nearly 3 (2^-17 cmax). Also orders the quad writes before the rays read them.
        if (tid == 0) s_nq = 0;  // before the barrier in cta_max; read after the barrier that follows the rays
        const float tol = (float)cta_max((double)cmax, red + 28) * 7.62939453125e-06f;
        const double half = peak / 2.0;
        int j_min = 2;  // first gradient candidate: j >= 2 and j * step >= thr
        while ((double)j_min * radial_step < thr) ++j_min;
        int found_h = 0, found_g = 0;
        for (int ray = tid; ray < n_angles; ray += kRadialThreads) {
            double edge_h = dnan(), edge_g = dnan();
            bool pend_h = false, pend_g = false;  // queued for the warps' FP64 re-walk
            if (peak > 0.0) {
                const double ang = (double)ray * (2.0 * kPi / n_angles);
                const double ux = trig ? trig[2 * ray] : cos(ang), uy = trig ? trig[2 * ray + 1] : sin(ang);
                // Samples are FP32 (SplineWindowF) and the walk's decisions are FP32; the edges are then
                // computed from FP64 samples at the decisive positions.
                float h1 = 0, h2 = 0, h3 = 0;  // p[k-1] .. p[k-3]
                int kc = -1;                   // first FP32 crossing: p[kc-1] >= half > p[kc]
                bool amb_h = false;            // a sample up to kc within tol of half height
                // Largest outward decrease p[j-1] - p[j+1] (first maximum) and the largest of the
                // candidates three or more samples from it; d1, d2: the decreases at jj-1, jj-2, and
                // m3 the largest at or before jj-3, for the current candidate jj.
                float best = -INFINITY, far = -INFINITY, d1 = -INFINITY, d2 = -INFINITY, m3 = -INFINITY;
                int best_j = -1, first_invalid = n_radii;
                const float halff = (float)half;
                SplineWindowF win;
                int mfy = -1 << 30, mfx = -1 << 30;  // mask cell of the last sample and whether all
                bool mfull = false;                   // four of its corners are in the eroded cell
                const double ymax = (double)(hm - 1), xmax = (double)(wm - 1);
                double kd = 0.0;  // k as a double (exact), so r = k * step needs no conversion
                for (int k = 0; k < n_radii; ++k, kd += 1.0) {
                    const double r = kd * radial_step;
                    const double x = __dadd_rn(cx, __dmul_rn(ux, r)), y = __dadd_rn(cy, __dmul_rn(uy, r));
                    if (!(y >= 0.0 && y <= ymax && x >= 0.0 && x <= xmax)) { first_invalid = k; break; }
                    double fyd, fxd;
                    const int iy = floor_nonneg(y, &fyd), ix = floor_nonneg(x, &fxd);
                    float p;
                    if constexpr (kRays == 2) {
                        if (!(full[iy * wm + ix] || inside_bytes(emask, hm, wm, y, x))) { first_invalid = k; break; }
                        p = k == 0 ? (float)peak
                                   : spline_sample_f(quad, wm, iy, ix, (float)(y - fyd), (float)(x - fxd));
                    } else {
                        if (iy != mfy || ix != mfx) {
                            mfy = iy;
                            mfx = ix;
                            const uint8_t* q = emask + iy * wm + ix;
                            mfull = iy + 1 < hm && ix + 1 < wm && q[0] && q[1] && q[wm] && q[wm + 1];
                        }
                        if (!(mfull || inside_bytes(emask, hm, wm, y, x))) { first_invalid = k; break; }
                        p = k == 0 ? (float)peak : win.at(quad, wm, iy, ix, (float)(y - fyd), (float)(x - fxd));
                    }
                    if (k >= 1 && kc < 0) {
                        amb_h |= fabsf(p - halff) <= tol;
                        if (h1 >= halff && p < halff) kc = k;
                    }
                    // Sample k valid makes j = k - 2 a candidate (valid[j - 2] and valid[j + 2]); its
                    // outward decrease is (p[j-1] - p[j+1]) / (2 step).
                    const int jj = k - 2;
                    if (jj >= j_min && jj <= n_radii - 3) {
                        const float d = h3 - h1;
                        if (d > best) {
                            far = m3;
                            best = d;
                            best_j = jj;
                        } else if (jj >= best_j + 3) {
                            far = fmaxf(far, d);
                        }
                        m3 = fmaxf(m3, d2);
                        d2 = d1;
                        d1 = d;
                    }
                    h3 = h2;
                    h2 = h1;
                    h1 = p;
                }
                // FP64 samples settle the edges: the crossing pair, and the decreases around the FP32
                // maximum. A decision within the FP32 samples' error bound elsewhere on the ray (a
                // sample near half height before the crossing, a distant candidate level with the
                // maximum) walks the ray again in FP64.
                const bool redo_h = half_out.status && amb_h;
                const bool redo_g = grad_out.status && best_j >= 0 && far >= best - 4.0f * tol;
                const int fix_kc = half_out.status && !amb_h ? kc : -1;
                const int fix_j = grad_out.status && !redo_g ? best_j : -1;
                if (fix_kc > 0 || fix_j >= 0)
                    ray_edges64(coef, hp, wp, dp, cx, cy, ux, uy, radial_step, peak, fix_kc, fix_j, j_min, n_radii,
                                first_invalid, &edge_h, &edge_g);
                if (redo_h || redo_g) {
                    // Queued for a warp after the ray loop, or walked here when the queue is full.
                    const int slot = atomicAdd(&s_nq, 1);
                    if (slot < kRewalkQueue) {
                        s_queue[slot] = ray | (redo_h ? 1 << 16 : 0) | (redo_g ? 1 << 17 : 0);
                        pend_h = redo_h;
                        pend_g = redo_g;
                    } else {
                        ray_fp64(coef, hp, wp, dp, emask, hm, wm, cx, cy, ux, uy, radial_step, n_radii, j_min, peak,
                                 redo_h, redo_g, &edge_h, &edge_g);
                    }
                }
            }
            if (half_out.status && !pend_h) {
                half_out.edge_px[(long long)i * n_angles + ray] = edge_h;
                found_h += isfinite(edge_h);
            }
            if (grad_out.status && !pend_g) {
                grad_out.edge_px[(long long)i * n_angles + ray] = edge_g;
                found_g += isfinite(edge_g);
            }
        }
        // The queued rays, one warp each, 32 FP64 samples at a time (the FP32 window rows are free now).
        __syncthreads();
        const int nq = min(s_nq, kRewalkQueue);
        if (nq > 0) {
            const int cap = (int)(2LL * (hm + 3) * wm / (kRadialThreads / 32));
            double* buf = reinterpret_cast<double*>(quad) + (long long)warp * cap;
            for (int q = warp; q < nq; q += kRadialThreads / 32) {
                const int e = s_queue[q], ray = e & 0xffff;
                const bool wh = (e >> 16) & 1, wg = (e >> 17) & 1;
                const double ang = (double)ray * (2.0 * kPi / n_angles);
                const double ux = trig ? trig[2 * ray] : cos(ang), uy = trig ? trig[2 * ray + 1] : sin(ang);
                double eh = dnan(), eg = dnan();
                if (!ray_fp64_warp(coef, hp, wp, dp, emask, hm, wm, cx, cy, ux, uy, radial_step, n_radii, j_min, peak,
                                   wh, wg, buf, cap, &eh, &eg)) {
                    if (lane == 0)
                        ray_fp64(coef, hp, wp, dp, emask, hm, wm, cx, cy, ux, uy, radial_step, n_radii, j_min, peak,
                                 wh, wg, &eh, &eg);
                }
                if (lane == 0) {
                    if (wh) {
                        half_out.edge_px[(long long)i * n_angles + ray] = eh;
                        found_h += isfinite(eh);
                    }
                    if (wg) {
                        grad_out.edge_px[(long long)i * n_angles + ray] = eg;
                        found_g += isfinite(eg);
                    }
                }
            }
        }
        const int all_h = (int)cta_sum((double)found_h, red + 20);
        const int all_g = (int)cta_sum((double)found_g, red + 24);  // also orders the edge writes
        if (warp < 2)  // warp 0: halfmax, warp 1: gradient
            radial_finish(warp == 0 ? half_out : grad_out, warp == 0 ? all_h : all_g, i, n_angles, cx, cy, peak, c.box,
                          trig);
    }
}

// Contours of stored results from their geometry (the compact result files' rebuild), with the
// measurement kernels' own vertex arithmetic: kind 0 the deblended Gaussian's half-maximum ellipse
// about the global centre, kind 1 the log-quadratic ellipse about the local centre plus the origin,
// kind 2 the radial polygon center_local + edge * (cos, sin) plus the origin. NaN where the cell
// has no ellipse or, for kind 2, no centre.
__global__ void k_rebuild_contours(int kind, const double* centers, const double* center_local,
                                   const double* eigenvalues, const double* axes, const double* edge_px,
                                   const int* origins, int n, int n_angles, double* contours) {
    const int nv = n_angles + 1;
    const long long total = (long long)n * nv;
    const double step = 2.0 * kPi / n_angles;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / nv), k = (int)(t % nv), a = k % n_angles;
        double x = dnan(), y = dnan();
        if (kind == 2) {
            const double cx = center_local[2LL * i], cy = center_local[2LL * i + 1];
            const double ang = (double)a * (2.0 * kPi / n_angles);
            const double c = cos(ang), sn = sin(ang);
            const double e = edge_px[(long long)i * n_angles + a];
            const double vx = cx + e * c, vy = cy + e * sn;
            x = vx + origins[2LL * i];
            y = vy + origins[2LL * i + 1];
        } else {
            Eig2 e;
            e.w0 = eigenvalues[2LL * i];
            e.w1 = eigenvalues[2LL * i + 1];
            e.v00 = axes[4LL * i + 0];
            e.v01 = axes[4LL * i + 1];
            e.v10 = axes[4LL * i + 2];
            e.v11 = axes[4LL * i + 3];
            if (isfinite(e.w0) && isfinite(e.w1)) {
                const double s0 = 1.0 / sqrt(e.w0), s1 = 1.0 / sqrt(e.w1);
                const double* ctr = kind == 0 ? centers : center_local;
                ellipse_vertex(ctr[2LL * i], ctr[2LL * i + 1], e, s0, s1, (double)a * step, &x, &y);
                if (kind == 1) {
                    x = x + origins[2LL * i];
                    y = y + origins[2LL * i + 1];
                }
            }
        }
        contours[2 * t] = x;
        contours[2 * t + 1] = y;
    }
}

// ------------------------------------------------------------------------------ projection

// numpy's sum of n values a[k * stride] along a contiguous axis (pairwise_sum): in order below 8
// values; up to 128, eight running sums (a[j], a[j + 8], ...) combined as ((r0 + r1) + (r2 + r3)) +
// ((r4 + r5) + (r6 + r7)), then the values past the last full eight in order; above 128, the two
// halves (the first a multiple of 8 long) summed that way and added.
__device__ double np_pairwise_sum(const double* a, int n, int stride) {
    if (n < 8) {
        double r = 0.0;
        for (int i = 0; i < n; ++i) r = __dadd_rn(r, a[i * stride]);
        return r;
    }
    if (n <= 128) {
        double r[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = a[j * stride];
        int i = 8;
        for (; i < n - (n % 8); i += 8)
#pragma unroll
            for (int j = 0; j < 8; ++j) r[j] = __dadd_rn(r[j], a[(i + j) * stride]);
        double res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                               __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
        for (; i < n; ++i) res = __dadd_rn(res, a[i * stride]);
        return res;
    }
    int n2 = n / 2;
    n2 -= n2 % 8;
    return __dadd_rn(np_pairwise_sum(a, n2, stride), np_pairwise_sum(a + n2 * stride, n - n2, stride));
}

// np_pairwise_sum by one warp (every lane calls it; all lanes return the sum): lanes 0-7 run the
// eight running sums of a block of up to 128 values, every lane combines them in numpy's tree and
// adds the tail; above 128 values the same halves as numpy's.
__device__ double warp_np_sum(const double* a, int n) {
    if (n > 128) {
        int n2 = n / 2;
        n2 -= n2 % 8;
        const double left = warp_np_sum(a, n2);
        return __dadd_rn(left, warp_np_sum(a + n2, n - n2));
    }
    if (n < 8) {
        double r = 0.0;
        for (int i = 0; i < n; ++i) r = __dadd_rn(r, a[i]);
        return r;
    }
    const int lane = threadIdx.x & 31, full = n - n % 8;
    double r = 0.0;
    if (lane < 8) {
        r = a[lane];
        for (int i = 8; i < full; i += 8) r = __dadd_rn(r, a[i + lane]);
    }
    double q[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) q[j] = __shfl_sync(0xffffffffu, r, j);
    double res = __dadd_rn(__dadd_rn(__dadd_rn(q[0], q[1]), __dadd_rn(q[2], q[3])),
                           __dadd_rn(__dadd_rn(q[4], q[5]), __dadd_rn(q[6], q[7])));
    for (int i = full; i < n; ++i) res = __dadd_rn(res, a[i]);
    return res;
}

constexpr int kProjWarps = 4;

// The "projection" CD of each cell (subpx/_cpu/invariant_cd.py:365-421), one warp per cell: the x
// profile (the masked cell summed over its rows, in row order as numpy reduces a strided axis) and
// the y profile (summed along each row, numpy's pairwise order), each spline-interpolated with the
// host's not-a-knot operators (value_op / slope_op, size x G, the profile padded with zeros) at
// the G points k * step. Inside the profile's span [first, last] the highest value (first on ties)
// and, before / after it, the steepest rise and fall (first on ties) give the width (their
// distance) and the centre (their midpoint); the cell is "ok" when both axes rise and fall strictly
// inside their span. The result is the axis-aligned ellipse of the two widths (subpx/_cpu/
// invariant_cd.py:320-336): edge radii a b / sqrt((b cos)^2 + (a sin)^2), contour, area pi a b,
// equivalent CD a + b, Ramanujan's perimeter. Arithmetic in FP64 without contraction where numpy
// rounds each operation; the spline sums are FMA chains in profile order.
// Shared memory per warp: max(hm, wm) profile values, then max(Gx, Gy) slopes.
__global__ void __launch_bounds__(kProjWarps * 32) k_projection_cd(
    const double* cleaned, const int* vor, const int4* boxes, const int* which, int n, int hm, int wm, int W,
    int n_angles, double step, const double* vx, const double* sx, int gx, const double* vy, const double* sy,
    int gy, MethodOut out) {
    extern __shared__ double psm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int pmax = max(hm, wm), gmax = max(gx, gy);
    double* prof = psm + (long long)warp * (pmax + gmax);
    double* slope = prof + pmax;
    const int area_px = hm * wm;
    for (int i = blockIdx.x * kProjWarps + warp; i < n; i += gridDim.x * kProjWarps) {
        const int j = which ? which[i] : i;
        const CellView c{cleaned + (long long)i * area_px, vor, boxes[j], j, W, hm, wm};
        // Peak of the masked cell (-inf when the mask is empty).
        double peak = -INFINITY;
        for (int k = lane; k < area_px; k += 32)
            if (c.mask(k / wm, k % wm)) peak = fmax(peak, c.roi[k]);
        peak = warp_max(peak);
        double width[2], centre[2];
        bool good[2];
        for (int axis = 0; axis < 2; ++axis) {
            const int size = axis == 0 ? wm : hm;
            const int G = axis == 0 ? gx : gy;
            const double* vop = axis == 0 ? vx : vy;
            const double* sop = axis == 0 ? sx : sy;
            // Profile and the span of columns (rows) that hold mask pixels.
            int first = size, last = -1;
            for (int q = lane; q < size; q += 32) {
                double v = 0.0;
                bool any = false;
                if (axis == 0) {  // sum over rows, in row order
                    for (int y = 0; y < hm; ++y) {
                        const bool m = c.mask(y, q);
                        v = y == 0 ? (m ? c.roi[q] : 0.0) : __dadd_rn(v, m ? c.roi[y * wm + q] : 0.0);
                        any = any || m;
                    }
                } else {
                    for (int x = 0; x < wm; ++x) any = any || c.mask(q, x);
                }
                if (axis == 0) prof[q] = v;
                if (any) {
                    first = min(first, q);
                    last = max(last, q);
                }
            }
            __syncwarp();
            if (axis == 1) {
                // Row sums in numpy's pairwise order, the masked values staged first.
                for (int q = 0; q < size; ++q) {
                    for (int x = lane; x < wm; x += 32) slope[x] = c.mask(q, x) ? c.roi[q * wm + x] : 0.0;
                    __syncwarp();
                    if (lane == 0) prof[q] = np_pairwise_sum(slope, wm, 1);
                    __syncwarp();
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
                last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
            }
            width[axis] = centre[axis] = dnan();
            good[axis] = false;
            if (last < 0) continue;  // no mask pixels: the cell has no signal either
            const double lo = (double)first, hi = (double)last;
            // Values and slopes on the grid; the highest value inside the span (first on ties).
            double best = -INFINITY;
            int best_g = 0x7fffffff;
            for (int g = lane; g < G; g += 32) {
                double v = 0.0, d = 0.0;
                for (int q = 0; q < size; ++q) {
                    const double p = prof[q];
                    v = __fma_rn(p, vop[(long long)q * G + g], v);
                    d = __fma_rn(p, sop[(long long)q * G + g], d);
                }
                slope[g] = d;
                const double t = __dmul_rn((double)g, step);
                if (t >= lo && t <= hi && (v > best || best_g == 0x7fffffff)) {
                    if (v > best || best_g == 0x7fffffff) {
                        best = v;
                        best_g = g;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int og = __shfl_xor_sync(0xffffffffu, best_g, o);
                if (ob > best || (ob == best && og < best_g)) {
                    best = ob;
                    best_g = og;
                }
            }
            __syncwarp();
            // Steepest rise at or before the peak, steepest fall at or after it (first on ties).
            double up = -INFINITY, down = INFINITY;
            int up_g = 0x7fffffff, down_g = 0x7fffffff;
            for (int g = lane; g < G; g += 32) {
                const double t = __dmul_rn((double)g, step);
                if (!(t >= lo && t <= hi)) continue;
                const double d = slope[g];
                if (g <= best_g && (d > up || up_g == 0x7fffffff)) {
                    up = d;
                    up_g = g;
                }
                if (g >= best_g && (d < down || down_g == 0x7fffffff)) {
                    down = d;
                    down_g = g;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ou = __shfl_xor_sync(0xffffffffu, up, o);
                const int oug = __shfl_xor_sync(0xffffffffu, up_g, o);
                if (oug != 0x7fffffff && (up_g == 0x7fffffff || ou > up || (ou == up && oug < up_g))) {
                    up = ou;
                    up_g = oug;
                }
                const double od = __shfl_xor_sync(0xffffffffu, down, o);
                const int odg = __shfl_xor_sync(0xffffffffu, down_g, o);
                if (odg != 0x7fffffff && (down_g == 0x7fffffff || od < down || (od == down && odg < down_g))) {
                    down = od;
                    down_g = odg;
                }
            }
            const double xl = __dmul_rn((double)up_g, step), xr = __dmul_rn((double)down_g, step);
            width[axis] = __dsub_rn(xr, xl);
            centre[axis] = __dmul_rn(__dadd_rn(xl, xr), 0.5);
            good[axis] = !(xl <= lo || xr >= hi || !(up > 0.0) || !(down < 0.0));
            __syncwarp();
        }
        const bool signal = peak > 0.0;
        const bool ok = signal && good[0] && good[1];
        const MetricRow m = out.row(i);
        if (lane == 0) {
            for (int q = 0; q < out.n_metrics; ++q) m[q] = dnan();
            m[M_PEAK] = peak;
            out.status[i] = (uint8_t)(ok ? SPX_ST_OK : signal ? SPX_ST_EDGE_AT_CELL_BORDER : SPX_ST_NO_SIGNAL);
        }
        const double a = __dmul_rn(width[0], 0.5), b = __dmul_rn(width[1], 0.5);
        const double cx = centre[0], cy = centre[1];
        const int nv = n_angles + 1;
        const double ang_step = 2.0 * kPi / n_angles;
        for (int k = lane; k < nv; k += 32) {
            const int q = k % n_angles;
            double e = dnan(), x = dnan(), y = dnan();
            if (signal) {
                const double ang = __dmul_rn((double)q, ang_step);
                const double co = cos(ang), si = sin(ang);
                const double bc = __dmul_rn(b, co), as = __dmul_rn(a, si);
                e = __ddiv_rn(__dmul_rn(a, b), sqrt(__dadd_rn(__dmul_rn(bc, bc), __dmul_rn(as, as))));
                x = __dadd_rn(__dadd_rn(cx, __dmul_rn(e, co)), (double)c.box.x);
                y = __dadd_rn(__dadd_rn(cy, __dmul_rn(e, si)), (double)c.box.y);
            }
            if (k < n_angles && out.edge_px) out.edge_px[(long long)i * n_angles + k] = e;
            if (out.contours) {
                out.contours[((long long)i * nv + k) * 2] = x;
                out.contours[((long long)i * nv + k) * 2 + 1] = y;
            }
        }
        if (lane == 0) {
            const double gx_ = signal ? __dadd_rn(cx, (double)c.box.x) : dnan();
            const double gy_ = signal ? __dadd_rn(cy, (double)c.box.y) : dnan();
            out.centers[2LL * i] = gx_;
            out.centers[2LL * i + 1] = gy_;
            if (out.center_local) {
                out.center_local[2LL * i] = signal ? cx : dnan();
                out.center_local[2LL * i + 1] = signal ? cy : dnan();
            }
            if (ok) {
                m[M_CD_X] = width[0];
                m[M_CD_Y] = width[1];
                m[M_AREA] = __dmul_rn(__dmul_rn(kPi, a), b);
                const double ab = __dadd_rn(a, b);
                m[M_CD_EQ] = ab;
                const double r = __ddiv_rn(__dsub_rn(a, b), fmax(ab, 1e-300));
                const double h = __dmul_rn(r, r);
                const double h3 = __dmul_rn(3.0, h);
                m[M_PERIM] = __dmul_rn(__dmul_rn(kPi, ab),
                                       __dadd_rn(1.0, __ddiv_rn(h3, __dadd_rn(10.0, sqrt(__dsub_rn(4.0, h3))))));
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------ half_area family

constexpr int kHalfThreads = 256;
constexpr int kHalfLeavesMax = 1024;  // pairwise-sum leaves of one enlarged cell (<= 128 values each)
constexpr int kHalfCtas = 148 * 4;    // persistent CTAs (each with its own scratch)

// The leaves of numpy's pairwise sum of n values (blocks of at most 128, split at half rounded down to
// a multiple of 8), in order: starts and lengths; returns their number.
__device__ int np_pairwise_leaves(int start, int n, int* lo, int* len, int count) {
    if (n <= 128) {
        lo[count] = start;
        len[count] = n;
        return count + 1;
    }
    int n2 = n / 2;
    n2 -= n2 % 8;
    count = np_pairwise_leaves(start, n2, lo, len, count);
    return np_pairwise_leaves(start + n2, n - n2, lo, len, count);
}

// The pairwise sum's tree over its leaf sums (same splits as np_pairwise_leaves).
__device__ double np_pairwise_tree(const double* leaf, int n, int* next) {
    if (n <= 128) return leaf[(*next)++];
    int n2 = n / 2;
    n2 -= n2 % 8;
    const double a = np_pairwise_tree(leaf, n2, next);
    return __dadd_rn(a, np_pairwise_tree(leaf, n - n2, next));
}

// Doubles before the zoom operators in a half-area CTA's shared memory: cell, ring, leaf sums and
// small arrays (doubles), four bit planes, row / column counts and leaves (ints), the mask bytes.
__host__ __device__ inline long long half_ops_offset(int hm, int wm, int f, int n_angles) {
    const long long Hb = (long long)hm * f, Wb = (long long)wm * f, RW = (Wb + 31) / 32, area = (long long)hm * wm;
    const long long tmpn = Hb + Wb > 3LL * (n_angles + 1) ? Hb + Wb : 3LL * (n_angles + 1);
    const long long bytes = (2 * area + kHalfLeavesMax + tmpn) * 8 + 4 * Hb * RW * 4 + (Hb + Wb + 2 * kHalfLeavesMax) * 4 +
                            area;
    return (bytes + 7) / 8;
}

struct HalfArgs {
    const double* cleaned;
    const int* vor;
    const int4* boxes;
    const int* which;
    int n, hm, wm, W, n_angles;
    const double* zy;  // (hm * f) x hm enlargement along y
    const double* zx;  // (wm * f) x wm along x
    int factor;
    double level;
    int median;   // local level: 1 median, 0 minimum of the outermost mask pixels
    int n_top;    // sub-pixels of the averaged peak
    int outlines;
    double* scratch;  // per CTA: the (hm f) x (wm f) enlarged cell
    MethodOut single, averaged;  // highest-pixel peak, averaged peak (status null: not wanted)
};

struct HalfCtx {
    const uint8_t* mask;
    const double* big;
    const uint32_t* bmask;
    uint32_t* above;
    uint32_t* reg;
    uint32_t* reg2;
    int* rowcnt;
    int* colcnt;
    double* tmp;
    double* leafsum;
    const int* leaf_lo;
    const int* leaf_len;
    int n_leaves;
    int Hb, Wb, RW, N;
    double b;
    int top;
    int* s_int;
    double* s_dbl;
};

// Where an area output's positions go: centres and contours are the enlargement's local positions
// plus (ox, oy); center_local is the local position itself, or with a finite lx the global centre
// minus (lx, ly) (the tail windows report it relative to the hole's own cell).
struct AreaPlace {
    double ox, oy, lx, ly;
};

// One output of the area methods from the cell's enlargement: region above b + cut around the
// highest pixel, its metrics and outline (see k_half_area); steepest (foot_area) goes to the
// metric after mean_signal when the output has that column.
__device__ void half_output(const HalfArgs& a, const MethodOut& out, int i, double peak, double cut, double steepest,
                            const HalfCtx& h, const AreaPlace& at) {
    const int tid = threadIdx.x, Hb = h.Hb, Wb = h.Wb, RW = h.RW;
    const bool signal = peak > 0.0 && isfinite(cut) && cut < peak;
    const uint32_t last_bits = (Wb % 32) ? ((1u << (Wb % 32)) - 1u) : 0xffffffffu;
    const int lane = tid & 31;
    for (int t = tid >> 5; t < Hb * RW; t += kHalfThreads / 32) {
        const int Y = t / RW, X = (t % RW) * 32 + lane;
        const bool in = X < Wb && h.big[(long long)Y * Wb + X] > cut;  // -inf outside the mask
        const uint32_t word = __ballot_sync(0xffffffffu, in);
        if (lane == 0) {
            h.above[t] = word;
            h.reg[t] = 0u;
            h.reg2[t] = 0u;
        }
    }
    __syncthreads();
    if (tid == 0) {
        const int Y = h.top / Wb, X = h.top % Wb;
        const uint32_t bitv = 1u << (X % 32);
        if (h.above[Y * RW + X / 32] & bitv) h.reg[Y * RW + X / 32] = bitv;
    }
    __syncthreads();
    // Grow the region from the highest pixel, one 8-neighbour ring per step, inside the above-
    // threshold pixels, until it stops changing. After s steps the region lies within s rows of the
    // highest pixel's row, so step s + 1 only computes the rows within s + 1 of it (the others of both
    // planes stay zero).
    uint32_t* cur = h.reg;
    uint32_t* nxt = h.reg2;
    auto vert = [&](const uint32_t* p, int Y, int w) {
        uint32_t v = p[Y * RW + w];
        if (Y > 0) v |= p[(Y - 1) * RW + w];
        if (Y < Hb - 1) v |= p[(Y + 1) * RW + w];
        return v;
    };
    auto dilate = [&](const uint32_t* p, int t) {
        const int Y = t / RW, w = t % RW;
        const uint32_t v = vert(p, Y, w);
        const uint32_t vp = w > 0 ? vert(p, Y, w - 1) : 0u, vn = w < RW - 1 ? vert(p, Y, w + 1) : 0u;
        uint32_t d = v | (v << 1) | (v >> 1) | (vp >> 31) | (vn << 31);
        if (w == RW - 1) d &= last_bits;
        return d;
    };
    const int top_row = h.top / Wb;
    for (int step = 0; step < h.N; ++step) {
        int changed = 0;
        const int r0 = max(top_row - step - 1, 0), r1 = min(top_row + step + 1, Hb - 1);
        for (int t = r0 * RW + tid; t < (r1 + 1) * RW; t += kHalfThreads) {
            const uint32_t nw = dilate(cur, t) & h.above[t];
            nxt[t] = nw;
            changed |= nw != cur[t];
        }
        changed = __syncthreads_or(changed);
        uint32_t* sw = cur;
        cur = nxt;
        nxt = sw;
        if (!changed) break;
    }
    // Counts per row and column, and whether the region reaches outside the mask or the stack's edge.
    int touch = 0;
    for (int t = tid; t < Hb * RW; t += kHalfThreads) {
        const int Y = t / RW, w = t % RW;
        const uint32_t d = dilate(cur, t);
        const uint32_t valid = w == RW - 1 ? last_bits : 0xffffffffu;
        touch |= (d & ~h.bmask[t] & valid) != 0u;
        if ((Y == 0 || Y == Hb - 1) && cur[t]) touch = 1;
        if (w == 0 && (cur[t] & 1u)) touch = 1;
        if (w == (Wb - 1) / 32 && ((cur[t] >> ((Wb - 1) % 32)) & 1u)) touch = 1;
    }
    for (int Y = tid; Y < Hb; Y += kHalfThreads) {
        int cnt = 0;
        for (int w = 0; w < RW; ++w) cnt += __popc(cur[Y * RW + w]);
        h.rowcnt[Y] = cnt;
    }
    for (int X = tid; X < Wb; X += kHalfThreads) {
        int cnt = 0;
        for (int Y = 0; Y < Hb; ++Y) cnt += (cur[Y * RW + X / 32] >> (X % 32)) & 1u;
        h.colcnt[X] = cnt;
    }
    // Leaves of the region's brightness sum (numpy's pairwise order over the enlarged cell).
    for (int L = tid; L < h.n_leaves; L += kHalfThreads) {
        // The leaf's values in memory order (the order of numpy's running sums), (Y, X) stepped along.
        const int lo = h.leaf_lo[L], n = h.leaf_len[L];
        int Y = lo / Wb, X = lo - Y * Wb;
        auto next = [&]() {
            const double v = ((cur[Y * RW + (X >> 5)] >> (X & 31)) & 1u) ? h.big[(long long)Y * Wb + X] : 0.0;
            if (++X == Wb) {
                X = 0;
                ++Y;
            }
            return v;
        };
        double res;
        if (n < 8) {
            res = 0.0;
            for (int q = 0; q < n; ++q) res = __dadd_rn(res, next());
        } else {
            double r[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) r[j] = next();
            int q = 8;
            for (; q < n - (n % 8); q += 8)
#pragma unroll
                for (int j = 0; j < 8; ++j) r[j] = __dadd_rn(r[j], next());
            res = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                            __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
            for (; q < n; ++q) res = __dadd_rn(res, next());
        }
        h.leafsum[L] = res;
    }
    touch = __syncthreads_or(touch);
    __shared__ long long s_count;
    const int warp = tid >> 5;
    // Row / column moments (products first, by all threads; numpy's sums by one warp each).
    double* ty = h.tmp;       // rows
    double* tx = h.tmp + Hb;  // columns
    for (int Y = tid; Y < Hb; Y += kHalfThreads) ty[Y] = __dmul_rn((double)h.rowcnt[Y], (double)Y);
    for (int X = tid; X < Wb; X += kHalfThreads) tx[X] = __dmul_rn((double)h.colcnt[X], (double)X);
    __syncthreads();
    if (warp == 0) {
        long long count = 0;
        for (int Y = lane; Y < Hb; Y += 32) count += h.rowcnt[Y];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
        if (lane == 0) s_count = count;
    } else if (warp == 1) {
        if (lane == 0) {
            int next = 0;
            h.s_dbl[2] = np_pairwise_tree(h.leafsum, h.N, &next);
        }
    } else if (warp == 2) {
        const double v = warp_np_sum(ty, Hb);
        if (lane == 0) h.s_dbl[0] = v;  // sum of row counts x row
    } else if (warp == 3) {
        const double v = warp_np_sum(tx, Wb);
        if (lane == 0) h.s_dbl[1] = v;
    }
    __syncthreads();
    const long long count = s_count;
    const double weight = (double)(count > 1 ? count : 1);
    const double cy = __ddiv_rn(h.s_dbl[0], weight), cx = __ddiv_rn(h.s_dbl[1], weight);
    const double mean_signal = __ddiv_rn(h.s_dbl[2], weight);
    const double sx = 1.0 / a.factor, sy = sx;
    const bool pow2 = (a.factor & (a.factor - 1)) == 0;
    for (int X = tid; X < Wb; X += kHalfThreads) {
        const double d = __dsub_rn((double)X, cx);
        tx[X] = __dmul_rn((double)h.colcnt[X], __dmul_rn(d, d));
    }
    for (int Y = tid; Y < Hb; Y += kHalfThreads) {
        const double d = __dsub_rn((double)Y, cy);
        ty[Y] = __dmul_rn((double)h.rowcnt[Y], __dmul_rn(d, d));
    }
    __syncthreads();
    if (warp == 0) {
        const double v = warp_np_sum(tx, Wb);
        if (lane == 0) h.s_dbl[3] = __dmul_rn(__dmul_rn(__ddiv_rn(v, weight), sx), sx);  // var_x
    } else if (warp == 1) {
        const double v = warp_np_sum(ty, Hb);
        if (lane == 0) h.s_dbl[2] = __dmul_rn(__dmul_rn(__ddiv_rn(v, weight), sy), sy);  // var_y
    }
    __syncthreads();
    const double var_x = h.s_dbl[3], var_y = h.s_dbl[2];
    const double shift = (double)(a.factor - 1) / (2.0 * a.factor);
    const double cxl = __dsub_rn(__dmul_rn(cx, sx), shift), cyl = __dsub_rn(__dmul_rn(cy, sy), shift);
    const bool ok = signal && !touch;
    // Display outline: along each ray from the centroid, the last 1/8 px step still in the region.
    const int nv = a.n_angles + 1;
    double* vx = h.tmp;
    double* vy = h.tmp + nv;
    if (a.outlines && signal) {
        const int nr = (int)ceil(hypot((double)a.hm, (double)a.wm) / 0.125);
        const double ang_step = 2.0 * kPi / a.n_angles;
        for (int q = tid; q < a.n_angles; q += kHalfThreads) {
            const double ang = __dmul_rn((double)q, ang_step);
            const double co = cos(ang), si = sin(ang);
            int first_out = nr;
            for (int s = 0; s < nr; ++s) {
                const double st = __dmul_rn((double)s, 0.125);
                // (cos x step) / sx, a multiplication by the factor when it is a power of two (exact).
                const double ox = pow2 ? __dmul_rn(__dmul_rn(co, st), (double)a.factor) : __ddiv_rn(__dmul_rn(co, st), sx);
                const double oy = pow2 ? __dmul_rn(__dmul_rn(si, st), (double)a.factor) : __ddiv_rn(__dmul_rn(si, st), sy);
                const double fx = rint(__dadd_rn(cx, ox));
                const double fy = rint(__dadd_rn(cy, oy));
                bool hit = fx >= 0.0 && fx < (double)Wb && fy >= 0.0 && fy < (double)Hb;
                if (hit) {
                    const int X = (int)fx, Y = (int)fy;
                    hit = (cur[Y * RW + X / 32] >> (X % 32)) & 1u;
                }
                if (!hit) {
                    first_out = s;
                    break;
                }
            }
            const double e = __dadd_rn(__dmul_rn((double)max(first_out - 1, 0), 0.125), 0.0625);
            if (out.edge_px) out.edge_px[(long long)i * a.n_angles + q] = e;
            vx[q] = __dadd_rn(__dadd_rn(cxl, __dmul_rn(e, co)), at.ox);
            vy[q] = __dadd_rn(__dadd_rn(cyl, __dmul_rn(e, si)), at.oy);
        }
        __syncthreads();
        if (tid == 0) {
            vx[a.n_angles] = vx[0];
            vy[a.n_angles] = vy[0];
        }
        __syncthreads();
        if (out.contours)
            for (int k = tid; k < nv; k += kHalfThreads) {
                out.contours[((long long)i * nv + k) * 2] = vx[k];
                out.contours[((long long)i * nv + k) * 2 + 1] = vy[k];
            }
        // Perimeter: the closed polygon's side lengths, summed in numpy's order by one warp.
        double* side = h.tmp + 2 * nv;
        for (int q = tid; q < a.n_angles; q += kHalfThreads) {
            const double dx = __dsub_rn(vx[q + 1], vx[q]), dy = __dsub_rn(vy[q + 1], vy[q]);
            side[q] = sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
        }
        __syncthreads();
        if (warp == 0) {
            const double v = warp_np_sum(side, a.n_angles);
            if (lane == 0) h.s_dbl[3] = v;
        }
    } else {
        if (out.edge_px)
            for (int q = tid; q < a.n_angles; q += kHalfThreads) out.edge_px[(long long)i * a.n_angles + q] = dnan();
        if (out.contours)
            for (int k = tid; k < 2 * nv; k += kHalfThreads) out.contours[(long long)i * 2 * nv + k] = dnan();
    }
    __syncthreads();
    if (tid == 0) {
        const MetricRow m = out.row(i);
        for (int q = 0; q < out.n_metrics; ++q) m[q] = dnan();
        m[M_LOCAL_LEVEL] = h.b;
        out.status[i] = (uint8_t)(!signal ? SPX_ST_NO_SIGNAL : touch ? SPX_ST_REGION_AT_CELL_BORDER : SPX_ST_OK);
        const double nan = dnan();
        const double gcx = __dadd_rn(cxl, at.ox), gcy = __dadd_rn(cyl, at.oy);
        out.centers[2LL * i] = signal ? gcx : nan;
        out.centers[2LL * i + 1] = signal ? gcy : nan;
        if (out.center_local) {
            const bool rel = isfinite(at.lx);
            out.center_local[2LL * i] = signal ? (rel ? __dsub_rn(gcx, at.lx) : cxl) : nan;
            out.center_local[2LL * i + 1] = signal ? (rel ? __dsub_rn(gcy, at.ly) : cyl) : nan;
        }
        if (signal) {
            m[M_PEAK] = peak;
            m[M_THRESHOLD] = __dadd_rn(h.b, cut);
            m[M_MEAN_SIGNAL] = mean_signal;
            if (out.n_metrics > M_STEEPEST) m[M_STEEPEST] = steepest;
        }
        if (ok) {
            const double area = __dmul_rn((double)count, __dmul_rn(sx, sy));
            const double cd_eq = __dmul_rn(2.0, sqrt(__ddiv_rn(area, kPi)));
            const double ratio = sqrt(sqrt(__ddiv_rn(fmax(var_x, 1e-12), fmax(var_y, 1e-12))));
            m[M_AREA] = area;
            m[M_CD_EQ] = cd_eq;
            m[M_CD_X] = __dmul_rn(cd_eq, ratio);
            m[M_CD_Y] = __ddiv_rn(cd_eq, ratio);
            if (a.outlines) m[M_PERIM] = h.s_dbl[3];
        }
    }
    __syncthreads();
}

// The half_area family (subpx/_cpu/invariant_cd.py:551-799 with 802-875 for the level backgrounds):
// one CTA per cell. Local level b = median or minimum of the outermost mask pixels; the cell minus b
// (zero outside its mask) enlarged f times by the host's cubic zoom operators (Zy C Zx^T, FMA chains in
// the order of the inner index); peak = the highest enlarged pixel of the mask (or the mean of the
// n_top highest); threshold b + level x peak; the region = the 8-connected above-threshold pixels that
// hold the highest pixel (grown one ring per step over bit rows); area, centroid, x / y spreads (sums in
// numpy's pairwise order), the equal-area ellipse's diameters, and the display outline (the region's
// last pixel along each ray from the centroid, 1/8 px steps). Status no_signal / region_at_cell_border
// (the region reaches the mask's edge or the stack's) / ok.
__global__ void __launch_bounds__(kHalfThreads) k_half_area(HalfArgs a) {
    extern __shared__ double hsm[];
    __shared__ int hist[2048];
    __shared__ int warp_tot[32], s_pick[3];
    __shared__ unsigned long long s_keys[2];
    __shared__ double s_red[2 * (kHalfThreads / 32)];
    __shared__ int s_ired[kHalfThreads / 32];
    __shared__ int s_int[4];
    __shared__ double s_dbl[4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int hm = a.hm, wm = a.wm, f = a.factor;
    const int Hb = hm * f, Wb = wm * f, RW = (Wb + 31) / 32, N = Hb * Wb, area_px = hm * wm;
    // Shared layout: cell values, ring values, leaf sums, small arrays (doubles); bit planes, counts,
    // leaves (ints); mask bytes.
    double* cell = hsm;
    double* ring = cell + area_px;
    double* leafsum = ring + area_px;
    const int tmpn = max(Hb + Wb, 3 * (a.n_angles + 1));
    double* tmp = leafsum + kHalfLeavesMax;
    uint32_t* bmask = reinterpret_cast<uint32_t*>(tmp + tmpn);
    uint32_t* above = bmask + Hb * RW;
    uint32_t* reg = above + Hb * RW;
    uint32_t* reg2 = reg + Hb * RW;
    int* rowcnt = reinterpret_cast<int*>(reg2 + Hb * RW);
    int* colcnt = rowcnt + Hb;
    int* leaf_lo = colcnt + Wb;
    int* leaf_len = leaf_lo + kHalfLeavesMax;
    uint8_t* mask = reinterpret_cast<uint8_t*>(leaf_len + kHalfLeavesMax);
    // The zoom operators, staged once per CTA after the mask bytes (8-byte aligned).
    double* zy = reinterpret_cast<double*>(hsm) + half_ops_offset(hm, wm, f, a.n_angles);
    double* zxT = zy + (long long)Hb * hm;  // transposed: zxT[x * Wb + X] = zx[X * wm + x]
    double* T = zxT + (long long)Wb * wm;    // Hb x wm
    for (int t = tid; t < Hb * hm; t += kHalfThreads) zy[t] = a.zy[t];
    for (int t = tid; t < Wb * wm; t += kHalfThreads) zxT[(t % wm) * Wb + t / wm] = a.zx[t];
    double* big = a.scratch + (long long)blockIdx.x * (long long)N;
    if (tid == 0) s_int[3] = np_pairwise_leaves(0, N, leaf_lo, leaf_len, 0);
    __syncthreads();
    const int n_leaves = s_int[3];
    for (int i = blockIdx.x; i < a.n; i += gridDim.x) {
        const int j = a.which ? a.which[i] : i;
        const CellView c{a.cleaned + (long long)i * area_px, a.vor, a.boxes[j], j, a.W, hm, wm};
        __syncthreads();  // the previous cell's shared-memory reads are done
        if (tid == 0) s_int[0] = 0;
        for (int k = tid; k < area_px; k += kHalfThreads) {
            const bool m = c.mask(k / wm, k % wm);
            mask[k] = m;
            cell[k] = m ? c.roi[k] : 0.0;
        }
        __syncthreads();
        // Outermost mask pixels: a 4-neighbour outside the mask, or on the stack's edge.
        double lmin = INFINITY;
        for (int k = tid; k < area_px; k += kHalfThreads) {
            const int y = k / wm, x = k % wm;
            if (!mask[k]) continue;
            const bool inner = y > 0 && x > 0 && y < hm - 1 && x < wm - 1 && mask[k - wm] && mask[k + wm] &&
                               mask[k - 1] && mask[k + 1];
            if (!inner) {
                ring[atomicAdd(&s_int[0], 1)] = cell[k];
                lmin = fmin(lmin, cell[k]);
            }
        }
        lmin = warp_min(lmin);
        if (lane == 0) s_red[warp] = lmin;
        __syncthreads();
        const int r = s_int[0];
        double b;
        if (a.median) {
            // nanmedian: the middle value(s) by rank (ties ranked by position), their mean; NaN if none.
            const int k1 = (r - 1) / 2, k2 = r / 2;
            for (int t = tid; t < r; t += kHalfThreads) {
                const double v = ring[t];
                int rank = 0;
                for (int q = 0; q < r; ++q) rank += ring[q] < v || (ring[q] == v && q < t);
                if (rank == k1) s_dbl[0] = v;
                if (rank == k2) s_dbl[1] = v;
            }
            __syncthreads();
            b = r ? __ddiv_rn(__dadd_rn(s_dbl[0], s_dbl[1]), 2.0) : dnan();
        } else {
            b = s_red[0];
            for (int q = 1; q < kHalfThreads / 32; ++q) b = fmin(b, s_red[q]);
        }
        __syncthreads();
        for (int k = tid; k < area_px; k += kHalfThreads) cell[k] = mask[k] ? __dsub_rn(cell[k], b) : 0.0;
        __syncthreads();
        // Bit plane of the enlarged mask (each sub-pixel copies its pixel), one word per warp ballot.
        for (int t = warp; t < Hb * RW; t += kHalfThreads / 32) {
            const int Y = t / RW, X = (t % RW) * 32 + lane;
            const uint32_t word = __ballot_sync(0xffffffffu, X < Wb && mask[(Y / f) * wm + X / f]);
            if (lane == 0) bmask[t] = word;
        }
        // Enlargement: T = Zy C (Hb x wm), then big = T Zx^T (Hb x Wb), stored -inf outside the
        // mask (only sub-pixels of the mask take part in what follows).
        for (int t = tid; t < Hb * wm; t += kHalfThreads) {
            const int Y = t / wm, x = t % wm;
            double v = 0.0;
            for (int y = 0; y < hm; ++y) v = __fma_rn(zy[Y * hm + y], cell[y * wm + x], v);
            T[t] = v;
        }
        __syncthreads();
        // One warp per pair of enlarged rows: lane takes columns lane + 32 q, the rows' T values
        // broadcast, each column's operator values shared by the two rows.
        for (int Y0 = 2 * warp; Y0 < Hb; Y0 += 2 * (kHalfThreads / 32))
            for (int X0 = 0; X0 < Wb; X0 += 128) {
                const bool two = Y0 + 1 < Hb;
                double v0[4] = {0.0, 0.0, 0.0, 0.0}, v1[4] = {0.0, 0.0, 0.0, 0.0};
                for (int x = 0; x < wm; ++x) {
                    const double t0 = T[Y0 * wm + x], t1 = two ? T[(Y0 + 1) * wm + x] : 0.0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int X = X0 + lane + 32 * q;
                        if (X < Wb) {
                            const double z = zxT[x * Wb + X];
                            v0[q] = __fma_rn(t0, z, v0[q]);
                            v1[q] = __fma_rn(t1, z, v1[q]);
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int X = X0 + lane + 32 * q;
                    if (X >= Wb) continue;
                    const bool m0 = (bmask[Y0 * RW + (X >> 5)] >> (X & 31)) & 1u;
                    big[(long long)Y0 * Wb + X] = m0 ? v0[q] : -INFINITY;
                    if (two) {
                        const bool m1 = (bmask[(Y0 + 1) * RW + (X >> 5)] >> (X & 31)) & 1u;
                        big[(long long)(Y0 + 1) * Wb + X] = m1 ? v1[q] : -INFINITY;
                    }
                }
            }
        __syncthreads();
        // Highest enlarged pixel of the mask (first in row-major order on ties; index 0 when none).
        double best = -INFINITY;
        int best_i = 0x7fffffff;
        unsigned long long kmin = ~0ull, kmax = 0;
        for (int t = tid; t < N; t += kHalfThreads) {
            const double v = big[t];
            if (v > best || best_i == 0x7fffffff) {
                if (v > best || best_i == 0x7fffffff) {
                    best = v;
                    best_i = t;
                }
            }
            const unsigned long long key = order_key(v);
            kmin = min(kmin, key);
            kmax = max(kmax, key);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, best_i, o);
            if (ob > best || (ob == best && oi < best_i)) {
                best = ob;
                best_i = oi;
            }
        }
        kmin = warp_min_u64(kmin);
        kmax = warp_max_u64(kmax);
        if (lane == 0) {
            s_red[warp] = best;
            s_ired[warp] = best_i;
            s_red[kHalfThreads / 32 + warp] = 0.0;
            hist[warp] = 0;  // (overwritten by the select below)
        }
        __shared__ unsigned long long s_kmin, s_kmax;
        if (tid == 0) {
            s_kmin = ~0ull;
            s_kmax = 0;
        }
        __syncthreads();
        if (lane == 0) {
            atomicMin(&s_kmin, kmin);
            atomicMax(&s_kmax, kmax);
        }
        __syncthreads();
        double top_v = s_red[0];
        int top = s_ired[0];
        for (int q = 1; q < kHalfThreads / 32; ++q)
            if (s_red[q] > top_v || (s_red[q] == top_v && s_ired[q] < top)) {
                top_v = s_red[q];
                top = s_ired[q];
            }
        if (top == 0x7fffffff) top = 0;
        __syncthreads();
        HalfCtx ctx{mask, big, bmask, above, reg, reg2, rowcnt, colcnt, tmp, leafsum, leaf_lo, leaf_len, n_leaves,
                    Hb, Wb, RW, N, b, top, s_int, s_dbl};
        const AreaPlace at{(double)c.box.x, (double)c.box.y, dnan(), dnan()};
        if (a.single.status) half_output(a, a.single, i, top_v, __dmul_rn(a.level, top_v), dnan(), ctx, at);
        if (a.averaged.status) {
            // Mean of the n_top highest enlarged pixels (outside the mask -inf): the n_top-th highest key
            // by the CTA select, then the keys above it and as many copies of it as are missing.
            double peak = -1.0;
            if (a.n_top <= N) {
                auto for_keys = [&](auto&& fn) {
                    for (int t = tid; t < N; t += kHalfThreads) fn(order_key(big[t]));
                };
                unsigned long long kth, kth2;
                cta_select<kHalfThreads>(for_keys, N - a.n_top, false, s_kmin, s_kmax, hist, warp_tot, s_pick,
                                         s_keys, &kth, &kth2);
                double sum = 0.0;
                int cnt = 0;
                for_keys([&](unsigned long long key) {
                    if (key > kth) {
                        sum += key_value(key);
                        ++cnt;
                    }
                });
                sum = warp_sum(sum);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
                if (lane == 0) {
                    s_red[warp] = sum;
                    s_ired[warp] = cnt;
                }
                __syncthreads();
                double total = 0.0;
                int above_cnt = 0;
                for (int q = 0; q < kHalfThreads / 32; ++q) {
                    total += s_red[q];
                    above_cnt += s_ired[q];
                }
                total += (double)(a.n_top - above_cnt) * key_value(kth);
                const double mean = total / a.n_top;
                peak = isfinite(mean) ? mean : -1.0;
                __syncthreads();
            }
            half_output(a, a.averaged, i, peak, __dmul_rn(a.level, peak), dnan(), ctx, at);
        }
    }
}

// ------------------------------------------------------------------------------ tail family

// Two of numpy's pairwise sums over an enlargement's N sub-pixels in memory order (leaves of at most
// 128 values with eight running sums each, then the tree), of val(Y, X, &v0, &v1); the results on
// every thread. All threads call it.
template <class F>
__device__ void np_sums2(F&& val, int Wb, int N, const int* leaf_lo, const int* leaf_len, int n_leaves,
                         double* leafsum, double* s_out, double* r0, double* r1) {
    const int tid = threadIdx.x;
    for (int L = tid; L < n_leaves; L += kHalfThreads) {
        const int lo = leaf_lo[L], n = leaf_len[L];
        int Y = lo / Wb, X = lo - Y * Wb;
        auto next = [&](double* a, double* b) {
            val(Y, X, a, b);
            if (++X == Wb) {
                X = 0;
                ++Y;
            }
        };
        double res0, res1;
        if (n < 8) {
            res0 = res1 = 0.0;
            for (int q = 0; q < n; ++q) {
                double a, b;
                next(&a, &b);
                res0 = __dadd_rn(res0, a);
                res1 = __dadd_rn(res1, b);
            }
        } else {
            double u[8], w[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) next(&u[j], &w[j]);
            int q = 8;
            for (; q < n - (n % 8); q += 8)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    double a, b;
                    next(&a, &b);
                    u[j] = __dadd_rn(u[j], a);
                    w[j] = __dadd_rn(w[j], b);
                }
            res0 = __dadd_rn(__dadd_rn(__dadd_rn(u[0], u[1]), __dadd_rn(u[2], u[3])),
                             __dadd_rn(__dadd_rn(u[4], u[5]), __dadd_rn(u[6], u[7])));
            res1 = __dadd_rn(__dadd_rn(__dadd_rn(w[0], w[1]), __dadd_rn(w[2], w[3])),
                             __dadd_rn(__dadd_rn(w[4], w[5]), __dadd_rn(w[6], w[7])));
            for (; q < n; ++q) {
                double a, b;
                next(&a, &b);
                res0 = __dadd_rn(res0, a);
                res1 = __dadd_rn(res1, b);
            }
        }
        leafsum[L] = res0;
        leafsum[kHalfLeavesMax + L] = res1;
    }
    __syncthreads();
    if (tid == 0) {
        int next = 0;
        s_out[0] = np_pairwise_tree(leafsum, N, &next);
        next = 0;
        s_out[1] = np_pairwise_tree(leafsum + kHalfLeavesMax, N, &next);
    }
    __syncthreads();
    *r0 = s_out[0];
    *r1 = s_out[1];
    __syncthreads();
}

struct TailArgs {
    HalfArgs h;              // factor, level, n_top, outlines, n_angles; hm = wm = the window side
    const float* cells;      // (n, S, S) each hole's share of the light
    const uint8_t* inside;   // (n, S, S) the window inside the image: the mask
    const uint8_t* levelm;   // level pixels (tail_area's local level)
    const uint8_t* zone;     // own territory (foot_area)
    const int* win_org;      // (n, 2) window origins
    const int* cell_org;     // (n, 2) the holes' own cell origins (center_local)
    const double* zxT;       // (S, S f) the x zoom operator transposed
    const double* cuts;      // (n) foot_area_ratio's thresholds
    MethodOut med, norm, edge, foot, given;  // status null: not wanted
};

// Shared memory of a tail CTA: the window (doubles), leaf sums and small arrays, five bit planes,
// row / column counts, the three masks. The enlargement, its first product (whose space also holds
// the level pixels' values before it) and the pairwise-sum leaves live in the CTA's global scratch,
// so that two CTAs fit an SM for windows up to 59 px.
__host__ __device__ inline long long tail_smem_bytes(int S, int f, int n_angles) {
    const long long Hb = (long long)S * f, RW = (Hb + 31) / 32, area = (long long)S * S;
    const long long tmpn = 2 * Hb > 3LL * (n_angles + 1) ? 2 * Hb : 3LL * (n_angles + 1);
    return (area + 2 * kHalfLeavesMax + tmpn) * 8 + 5 * Hb * RW * 4 + 2 * Hb * 4 + 3 * area;
}

// Doubles of one tail CTA's global scratch: enlargement (Hb^2), first product (Hb S), leaves.
__host__ __device__ inline long long tail_scratch_doubles(int S, int f) {
    const long long Hb = (long long)S * f;
    return Hb * Hb + Hb * S + kHalfLeavesMax;
}

// The tail family on hole windows (subpx/_cpu/invariant_cd.py:551-875 with the windows of 878-964):
// one CTA per window. Local level b: the median of the level pixels (tail_area) or none (the others,
// which share one enlargement); the window minus b inside the image, enlarged f times by the host's
// zoom operators (read from global memory: windows are up to 64 px); averaged peak; the threshold
// per method: level x peak (tail_area, tail_area_norm), the steepness-weighted mean of the core
// sub-pixels (edge_area), the curvature-weighted mean below the steepest level inside the territory
// (foot_area), or given (foot_area_ratio). The region, its metrics and outline as the half_area
// family; positions in the image, center_local relative to the hole's own cell.
__global__ void __launch_bounds__(kHalfThreads, 2) k_tail_area(TailArgs t) {
    extern __shared__ double hsm[];
    __shared__ int hist[2048];
    __shared__ int warp_tot[32], s_pick[3];
    __shared__ unsigned long long s_keys[2], s_kmin, s_kmax;
    __shared__ double s_red[2 * (kHalfThreads / 32)];
    __shared__ int s_ired[kHalfThreads / 32];
    __shared__ int s_int[4];
    __shared__ double s_dbl[8];
    const HalfArgs& a = t.h;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int S = a.hm, f = a.factor;
    const int Hb = S * f, Wb = Hb, RW = (Wb + 31) / 32, N = Hb * Wb, area = S * S;
    const int tmpn = max(2 * Hb, 3 * (a.n_angles + 1));
    double* cell = hsm;
    double* leafsum = cell + area;
    double* tmp = leafsum + 2 * kHalfLeavesMax;
    uint32_t* bmask = reinterpret_cast<uint32_t*>(tmp + tmpn);
    uint32_t* above = bmask + Hb * RW;
    uint32_t* reg = above + Hb * RW;
    uint32_t* reg2 = reg + Hb * RW;
    uint32_t* zplane = reg2 + Hb * RW;
    int* rowcnt = reinterpret_cast<int*>(zplane + Hb * RW);
    int* colcnt = rowcnt + Hb;
    uint8_t* mask = reinterpret_cast<uint8_t*>(colcnt + Wb);
    uint8_t* lmask = mask + area;
    uint8_t* zmask = lmask + area;
    double* big = a.scratch + (long long)blockIdx.x * tail_scratch_doubles(S, f);
    double* T = big + N;
    double* lv = T;  // the level pixels' values, used before T is computed
    int* leaf_lo = reinterpret_cast<int*>(T + (long long)Hb * S);
    int* leaf_len = leaf_lo + kHalfLeavesMax;
    if (tid == 0) s_int[3] = np_pairwise_leaves(0, N, leaf_lo, leaf_len, 0);
    __syncthreads();
    const int n_leaves = s_int[3];
    __syncthreads();  // s_int is reused below
    const bool want_zero = t.norm.status || t.edge.status || t.foot.status || t.given.status;
    const double sy = 1.0 / f;
    const double den_g = __dmul_rn((double)(2 * f), sy);  // 2 d sy: central differences over +-d
    const double den_c = __dmul_rn(__dmul_rn((double)f, sy), __dmul_rn((double)f, sy));  // (d sy)^2
    auto bit = [&](const uint32_t* p, int Y, int X) { return (p[Y * RW + (X >> 5)] >> (X & 31)) & 1u; };
    for (int i = blockIdx.x; i < a.n; i += gridDim.x) {
        __syncthreads();  // the previous window's shared-memory reads are done
        const long long base = (long long)i * area;
        for (int k = tid; k < area; k += kHalfThreads) {
            const bool m = t.inside[base + k];
            mask[k] = m;
            cell[k] = m ? (double)t.cells[base + k] : 0.0;
            lmask[k] = t.levelm ? t.levelm[base + k] : 0;
            zmask[k] = t.zone ? t.zone[base + k] : 1;
        }
        __syncthreads();
        for (int w = warp; w < Hb * RW; w += kHalfThreads / 32) {
            const int Y = w / RW, X = (w % RW) * 32 + lane;
            const int src = (Y / f) * S + X / f;
            const uint32_t mw = __ballot_sync(0xffffffffu, X < Wb && mask[src]);
            const uint32_t zw = __ballot_sync(0xffffffffu, X < Wb && zmask[src]);
            if (lane == 0) {
                bmask[w] = mw;
                zplane[w] = zw;
            }
        }
        const AreaPlace at{(double)t.win_org[2LL * i], (double)t.win_org[2LL * i + 1],
                           (double)t.cell_org[2LL * i], (double)t.cell_org[2LL * i + 1]};
        for (int kind = 0; kind < 2; ++kind) {
            if (kind == 0 ? !t.med.status : !want_zero) continue;
            double b = 0.0;
            if (kind == 0) {
                // nanmedian of the level pixels inside the window (ranks, ties by position; NaN if none).
                if (tid == 0) s_int[0] = 0;
                __syncthreads();
                for (int k = tid; k < area; k += kHalfThreads)
                    if (mask[k] && lmask[k]) lv[atomicAdd(&s_int[0], 1)] = cell[k];
                __syncthreads();
                const int r = s_int[0], k1 = (r - 1) / 2, k2 = r / 2;
                for (int q0 = tid; q0 < r; q0 += kHalfThreads) {
                    const double v = lv[q0];
                    int rank = 0;
                    for (int q = 0; q < r; ++q) rank += lv[q] < v || (lv[q] == v && q < q0);
                    if (rank == k1) s_dbl[0] = v;
                    if (rank == k2) s_dbl[1] = v;
                }
                __syncthreads();
                b = r ? __ddiv_rn(__dadd_rn(s_dbl[0], s_dbl[1]), 2.0) : dnan();
                __syncthreads();
            }
            // T = Zy (window - b, zero outside the image) (Hb x S), then big = T Zx^T, -inf outside.
            for (int q = tid; q < Hb * S; q += kHalfThreads) {
                const int Y = q / S, x = q % S;
                const double* zr = a.zy + (long long)Y * S;
                double v = 0.0;
#pragma unroll 4
                for (int y = 0; y < S; ++y) {
                    const double c = mask[y * S + x] ? __dsub_rn(cell[y * S + x], b) : 0.0;
                    v = __fma_rn(__ldg(zr + y), c, v);
                }
                T[q] = v;
            }
            __syncthreads();
            // Four enlarged rows per warp step (each operator load feeds four rows), lanes across
            // columns, the products summed in the order of x as before.
            for (int Y0 = 4 * warp; Y0 < Hb; Y0 += 4 * (kHalfThreads / 32))
                for (int X0 = 0; X0 < Wb; X0 += 128) {
                    double v[4][4];
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int q = 0; q < 4; ++q) v[r][q] = 0.0;
#pragma unroll 2
                    for (int x = 0; x < S; ++x) {
                        double tr[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r) tr[r] = Y0 + r < Hb ? T[(long long)(Y0 + r) * S + x] : 0.0;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int X = X0 + lane + 32 * q;
                            if (X < Wb) {
                                const double z = __ldg(t.zxT + (long long)x * Wb + X);
#pragma unroll
                                for (int r = 0; r < 4; ++r) v[r][q] = __fma_rn(tr[r], z, v[r][q]);
                            }
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int X = X0 + lane + 32 * q;
                        if (X >= Wb) continue;
#pragma unroll
                        for (int r = 0; r < 4; ++r)
                            if (Y0 + r < Hb) big[(long long)(Y0 + r) * Wb + X] = bit(bmask, Y0 + r, X) ? v[r][q] : -INFINITY;
                    }
                }
            __syncthreads();
            // Highest enlarged pixel (first on ties) and the key range for the averaged peak.
            double best = -INFINITY;
            int best_i = 0x7fffffff;
            unsigned long long kmin = ~0ull, kmax = 0;
            for (int q = tid; q < N; q += kHalfThreads) {
                const double v = big[q];
                if (v > best || best_i == 0x7fffffff) {
                    best = v;
                    best_i = q;
                }
                const unsigned long long key = order_key(v);
                kmin = min(kmin, key);
                kmax = max(kmax, key);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, best_i, o);
                if (ob > best || (ob == best && oi < best_i)) {
                    best = ob;
                    best_i = oi;
                }
            }
            kmin = warp_min_u64(kmin);
            kmax = warp_max_u64(kmax);
            if (lane == 0) {
                s_red[warp] = best;
                s_ired[warp] = best_i;
            }
            if (tid == 0) {
                s_kmin = ~0ull;
                s_kmax = 0;
            }
            __syncthreads();
            if (lane == 0) {
                atomicMin(&s_kmin, kmin);
                atomicMax(&s_kmax, kmax);
            }
            __syncthreads();
            double top_v = s_red[0];
            int top = s_ired[0];
            for (int q = 1; q < kHalfThreads / 32; ++q)
                if (s_red[q] > top_v || (s_red[q] == top_v && s_ired[q] < top)) {
                    top_v = s_red[q];
                    top = s_ired[q];
                }
            if (top == 0x7fffffff) top = 0;
            __syncthreads();
            // Averaged peak: the mean of the n_top highest sub-pixels (-inf outside the mask).
            double peak = -1.0;
            if (a.n_top <= N) {
                auto for_keys = [&](auto&& fn) {
                    for (int q = tid; q < N; q += kHalfThreads) fn(order_key(big[q]));
                };
                unsigned long long kth, kth2;
                cta_select<kHalfThreads>(for_keys, N - a.n_top, false, s_kmin, s_kmax, hist, warp_tot, s_pick, s_keys,
                                         &kth, &kth2);
                double sum = 0.0;
                int cnt = 0;
                for_keys([&](unsigned long long key) {
                    if (key > kth) {
                        sum += key_value(key);
                        ++cnt;
                    }
                });
                sum = warp_sum(sum);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
                if (lane == 0) {
                    s_red[warp] = sum;
                    s_ired[warp] = cnt;
                }
                __syncthreads();
                double total = 0.0;
                int above_cnt = 0;
                for (int q = 0; q < kHalfThreads / 32; ++q) {
                    total += s_red[q];
                    above_cnt += s_ired[q];
                }
                total += (double)(a.n_top - above_cnt) * key_value(kth);
                const double mean = total / a.n_top;
                peak = isfinite(mean) ? mean : -1.0;
                __syncthreads();
            }
            HalfCtx ctx{mask, big, bmask, above, reg, reg2, rowcnt, colcnt, tmp, leafsum, leaf_lo, leaf_len, n_leaves,
                        Hb, Wb, RW, N, b, top, s_int, s_dbl};
            if (kind == 0) {
                half_output(a, t.med, i, peak, __dmul_rn(a.level, peak), dnan(), ctx, at);
                continue;
            }
            if (t.norm.status) half_output(a, t.norm, i, peak, __dmul_rn(a.level, peak), dnan(), ctx, at);
            // Core sub-pixels: inside the enlarged mask with their +-f stencil, none within f of the edge.
            auto core = [&](int Y, int X, bool zoned) {
                if (Y < f || Y >= Hb - f || X < f || X >= Wb - f) return false;
                if (!(bit(bmask, Y, X) && bit(bmask, Y - f, X) && bit(bmask, Y + f, X) && bit(bmask, Y, X - f) &&
                      bit(bmask, Y, X + f)))
                    return false;
                return !zoned || bit(zplane, Y, X) != 0u;
            };
            auto steep_at = [&](int Y, int X) {
                const double* r = big + (long long)Y * Wb + X;
                const double gy = __ddiv_rn(__dsub_rn(r[(long long)f * Wb], r[-(long long)f * Wb]), den_g);
                const double gx = __ddiv_rn(__dsub_rn(r[f], r[-f]), den_g);
                return sqrt(__dadd_rn(__dmul_rn(gy, gy), __dmul_rn(gx, gx)));
            };
            if (t.edge.status) {
                double total, num;
                np_sums2(
                    [&](int Y, int X, double* w, double* wb) {
                        if (core(Y, X, false)) {
                            const double s = steep_at(Y, X);
                            *w = s;
                            *wb = __dmul_rn(s, big[(long long)Y * Wb + X]);
                        } else {
                            *w = 0.0;
                            *wb = 0.0;
                        }
                    },
                    Wb, N, leaf_lo, leaf_len, n_leaves, leafsum, s_dbl + 4, &total, &num);
                const double cut = total > 0.0 ? __ddiv_rn(num, total) : INFINITY;
                half_output(a, t.edge, i, peak, cut, dnan(), ctx, at);
            }
            if (t.foot.status) {
                const bool zoned = t.zone != nullptr;
                double total, num;
                np_sums2(
                    [&](int Y, int X, double* w, double* wb) {
                        if (core(Y, X, zoned)) {
                            const double s = steep_at(Y, X);
                            *w = s;
                            *wb = __dmul_rn(s, big[(long long)Y * Wb + X]);
                        } else {
                            *w = 0.0;
                            *wb = 0.0;
                        }
                    },
                    Wb, N, leaf_lo, leaf_len, n_leaves, leafsum, s_dbl + 4, &total, &num);
                const double steepest = __ddiv_rn(num, total > 0.0 ? total : 1.0);
                double bend, num2;
                np_sums2(
                    [&](int Y, int X, double* c, double* cb) {
                        const double v = big[(long long)Y * Wb + X];
                        if (core(Y, X, zoned) && v < steepest) {
                            const double* r = big + (long long)Y * Wb + X;
                            const double v2 = __dmul_rn(2.0, v);
                            const double cy = __ddiv_rn(__dsub_rn(__dadd_rn(r[(long long)f * Wb], r[-(long long)f * Wb]), v2), den_c);
                            const double cx = __ddiv_rn(__dsub_rn(__dadd_rn(r[f], r[-f]), v2), den_c);
                            const double curve = __dadd_rn(cy, cx);
                            *c = curve;
                            *cb = __dmul_rn(curve, v);
                        } else {
                            *c = 0.0;
                            *cb = 0.0;
                        }
                    },
                    Wb, N, leaf_lo, leaf_len, n_leaves, leafsum, s_dbl + 4, &bend, &num2);
                const double cut = total > 0.0 && bend > 0.0 ? __ddiv_rn(num2, bend) : INFINITY;
                half_output(a, t.foot, i, peak, cut, steepest, ctx, at);
            }
            if (t.given.status) half_output(a, t.given, i, peak, t.cuts[i], dnan(), ctx, at);
        }
    }
}

// The status names, as the reference's result arrays spell them (numpy "U32": 32 UCS-4 code
// points per entry, zero-padded).
#define SPX_STATUS_NAMES(X)                                                                            \
    X("ok") X("no_signal") X("insufficient_cell_pixels") X("insufficient_fit_pixels") X("singular_fit") \
        X("non_gaussian_fit") X("contour_outside_cell") X("incomplete_rays") X("fit_diverged")         \
            X("center_outside_cell") X("edge_at_cell_border") X("region_at_cell_border")
#define SPX_NAME_ENTRY(s) s,
constexpr int kStatusCount = 12;
constexpr int kStatusChars = 32;
__constant__ char c_status_names[kStatusCount][kStatusChars] = {SPX_STATUS_NAMES(SPX_NAME_ENTRY)};
const char* const kStatusNamesHost[kStatusCount] = {SPX_STATUS_NAMES(SPX_NAME_ENTRY)};

// One thread per (cell, character): the UCS-4 text of each cell's status code.
__global__ void k_status_text(const uint8_t* codes, int n, uint32_t* out) {
    const long long total = (long long)n * kStatusChars;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / kStatusChars), c = (int)(t % kStatusChars);
        const int code = codes[i];
        out[t] = code < kStatusCount ? (uint32_t)(unsigned char)c_status_names[code][c] : 0u;
    }
}

MethodOut method_out(const spx_method_out* o) {
    MethodOut m;
    if (!o) {
        m = MethodOut{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0};
        return m;
    }
    m.centers = o->centers;
    m.contours = o->contours;
    m.status = o->status;
    m.metrics = o->metrics;
    m.center_local = o->center_local;
    m.edge_px = o->edge_px;
    m.eigenvalues = o->eigenvalues;
    m.axes = o->axes;
    m.n_metrics = o->n_metrics;
    m.col_stride = o->metric_col_stride;
    return m;
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

int spx_gaussian_method(const double* params, const uint8_t* status_in, const double* cleaned, const int* voronoi,
                        const int* boxes, const int* which, int n, int hm, int wm, int width, int n_angles,
                        const spx_method_out* out, void* stream) {
    SPX_REQUIRE(n >= 0 && n_angles >= 1, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(params && status_in && cleaned && voronoi && boxes && out && out->centers && out->status &&
                    out->metrics && out->n_metrics >= 13,
                "null pointer or too few metric columns");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_gaussian_method<<<grid_for(n, 8, 148 * 32), 256, 0, s>>>(params, status_in, cleaned, voronoi,
                                                              reinterpret_cast<const int4*>(boxes), which, n, hm,
                                                              wm, width, n_angles, method_out(out));
    return check_launch("k_gaussian_method");
}

const char* spx_status_name(int code) { return code >= 0 && code < kStatusCount ? kStatusNamesHost[code] : nullptr; }

int spx_status_text(const uint8_t* codes, int n, uint32_t* text, void* stream) {
    SPX_REQUIRE(n >= 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(codes && text, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_status_text<<<grid_for((long long)n * kStatusChars, 256), 256, 0, s>>>(codes, n, text);
    return check_launch("k_status_text");
}

int spx_logquad_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, const double* seeds,
                   int n, int hm, int wm, int width, int n_angles, double fit_fraction, const spx_method_out* out,
                   void* stream) {
    SPX_REQUIRE(n >= 0 && n_angles >= 1, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(cleaned && voronoi && boxes && seeds && out && out->centers && out->status && out->metrics &&
                    out->center_local && out->eigenvalues && out->axes && out->n_metrics >= 13,
                "null pointer or too few metric columns");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_logquad_cd<<<grid_for(n, 8, 148 * 32), 256, 0, s>>>(cleaned, voronoi, reinterpret_cast<const int4*>(boxes),
                                                         which, seeds, n, hm, wm, width, n_angles, fit_fraction,
                                                         method_out(out));
    return check_launch("k_logquad_cd");
}

int spx_projection_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                      int wm, int width, int n_angles, double step, const double* value_op_x,
                      const double* slope_op_x, int gx, const double* value_op_y, const double* slope_op_y, int gy,
                      const spx_method_out* out, void* stream) {
    SPX_REQUIRE(n >= 0 && n_angles >= 1 && hm >= 1 && wm >= 1 && gx >= 1 && gy >= 1 && step > 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(cleaned && voronoi && boxes && out && out->centers && out->status && out->metrics &&
                    value_op_x && slope_op_x && value_op_y && slope_op_y && out->n_metrics >= 7,
                "null pointer or too few metric columns");
    const size_t smem = (size_t)kProjWarps * (std::max(hm, wm) + std::max(gx, gy)) * sizeof(double);
    SPX_REQUIRE(smem <= 220 * 1024, "cell stack too large for the projection kernel");
    if (smem > 48 * 1024) SPX_CUDA(cudaFuncSetAttribute(k_projection_cd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)smem));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_projection_cd<<<grid_for(n, kProjWarps, 148 * 16), kProjWarps * 32, smem, s>>>(
        cleaned, voronoi, reinterpret_cast<const int4*>(boxes), which, n, hm, wm, width, n_angles, step, value_op_x,
        slope_op_x, gx, value_op_y, slope_op_y, gy, method_out(out));
    return check_launch("k_projection_cd");
}

// Shared memory of one half-area CTA (see the layout in k_half_area): the cell's arrays, then the
// two zoom operators and the first product.
static size_t half_smem(int hm, int wm, int f, int n_angles) {
    return (half_ops_offset(hm, wm, f, n_angles) + (size_t)hm * f * hm + (size_t)wm * f * wm + (size_t)hm * f * wm) *
           sizeof(double);
}

size_t spx_half_area_workspace_bytes(int hm, int wm, int factor) {
    const size_t Hb = (size_t)hm * factor, Wb = (size_t)wm * factor;
    return (size_t)kHalfCtas * Hb * Wb * sizeof(double) + 256;
}

int spx_half_area_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                     int wm, int width, int n_angles, const double* zoom_y, const double* zoom_x, int factor,
                     double level, int median, int n_top, int outlines, const spx_method_out* single,
                     const spx_method_out* averaged, void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && n_angles >= 1 && hm >= 1 && wm >= 1 && factor >= 1 && n_top >= 1, "bad arguments");
    SPX_REQUIRE(level > 0.0 && level < 1.0, "level must be between 0 and 1");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(cleaned && voronoi && boxes && zoom_y && zoom_x && workspace && (single || averaged), "null pointer");
    for (const spx_method_out* o : {single, averaged})
        if (o) SPX_REQUIRE(o->centers && o->status && o->metrics && o->n_metrics >= 10, "null pointer or too few metric columns");
    // Up to 32768 sub-pixels: numpy's pairwise-sum leaves (at least 57 values each) then fit kHalfLeavesMax.
    SPX_REQUIRE((long long)hm * factor * wm * factor <= 32768, "cell stack too large for the half-area kernel");
    SPX_REQUIRE(workspace_bytes >= spx_half_area_workspace_bytes(hm, wm, factor), "workspace too small");
    const size_t smem = half_smem(hm, wm, factor, n_angles);
    SPX_REQUIRE(smem <= 200 * 1024, "cell stack too large for the half-area kernel");
    if (smem > 48 * 1024)
        SPX_CUDA(cudaFuncSetAttribute(k_half_area, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uintptr_t base = (reinterpret_cast<uintptr_t>(workspace) + 255) & ~(uintptr_t)255;
    HalfArgs a{cleaned, voronoi, reinterpret_cast<const int4*>(boxes), which, n, hm, wm, width, n_angles, zoom_y,
               zoom_x, factor, level, median, n_top, outlines, reinterpret_cast<double*>(base), method_out(single),
               method_out(averaged)};
    if (!single) a.single.status = nullptr;
    if (!averaged) a.averaged.status = nullptr;
    k_half_area<<<std::min(n, kHalfCtas), kHalfThreads, smem, static_cast<cudaStream_t>(stream)>>>(a);
    return check_launch("k_half_area");
}

// Persistent CTAs of the tail kernel (each with its own enlargement scratch): up to four per SM as
// its shared memory allows.
static int tail_ctas(int side, int factor, int n_angles) {
    const size_t smem = (size_t)tail_smem_bytes(side, factor, n_angles);
    if (smem > 48 * 1024)
        if (cudaFuncSetAttribute(k_tail_area, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tail_area, kHalfThreads, smem) != cudaSuccess) return 0;
    return 148 * std::min(std::max(per_sm, 1), 4);
}

size_t spx_tail_area_workspace_bytes(int side, int factor, int n_angles) {
    if (side < 1 || factor < 1 || n_angles < 1) return 0;
    return (size_t)(148LL * 4 * tail_scratch_doubles(side, factor) * sizeof(double) + 256);
}

int spx_tail_area_cd(const float* cells, const uint8_t* inside, const uint8_t* level_pixels, const uint8_t* territory,
                     const int* window_origins, const int* cell_origins, int n, int side, int n_angles,
                     const double* zoom_y, const double* zoom_x_t, int factor, double level, int n_top, int outlines,
                     const double* cuts, const spx_method_out* tail, const spx_method_out* norm,
                     const spx_method_out* edge, const spx_method_out* foot, const spx_method_out* given,
                     void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && n_angles >= 1 && side >= 1 && factor >= 1 && n_top >= 1, "bad arguments");
    SPX_REQUIRE(level > 0.0 && level < 1.0, "level must be between 0 and 1");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(cells && inside && window_origins && cell_origins && zoom_y && zoom_x_t && workspace &&
                    (tail || norm || edge || foot || given),
                "null pointer");
    SPX_REQUIRE(!tail || level_pixels, "tail_area needs the level pixels");
    SPX_REQUIRE(!given || cuts, "foot_area_ratio needs its thresholds");
    for (const spx_method_out* o : {tail, norm, edge, given})
        if (o) SPX_REQUIRE(o->centers && o->status && o->metrics && o->n_metrics >= 10, "null pointer or too few metric columns");
    if (foot) SPX_REQUIRE(foot->centers && foot->status && foot->metrics && foot->n_metrics >= 11,
                          "null pointer or too few metric columns");
    // numpy's pairwise-sum leaves (at least 64 values each) of up to 65536 sub-pixels fit kHalfLeavesMax.
    SPX_REQUIRE((long long)side * factor * side * factor <= 65536, "tail window too large for the tail kernel");
    SPX_REQUIRE(tail_smem_bytes(side, factor, n_angles) <= 200 * 1024, "tail window too large for the tail kernel");
    SPX_REQUIRE(workspace_bytes >= spx_tail_area_workspace_bytes(side, factor, n_angles), "workspace too small");
    const int ctas = tail_ctas(side, factor, n_angles);
    SPX_REQUIRE(ctas > 0, "tail kernel launch configuration failed");
    const uintptr_t base = (reinterpret_cast<uintptr_t>(workspace) + 255) & ~(uintptr_t)255;
    HalfArgs h{nullptr, nullptr, nullptr, nullptr, n, side, side, 0, n_angles, zoom_y, nullptr, factor, level, 0, n_top,
               outlines, reinterpret_cast<double*>(base), method_out(nullptr), method_out(nullptr)};
    TailArgs t{h, cells, inside, level_pixels, territory, window_origins, cell_origins, zoom_x_t, cuts,
               method_out(tail), method_out(norm), method_out(edge), method_out(foot), method_out(given)};
    const size_t smem = (size_t)tail_smem_bytes(side, factor, n_angles);
    k_tail_area<<<std::min(n, ctas), kHalfThreads, smem, static_cast<cudaStream_t>(stream)>>>(t);
    return check_launch("k_tail_area");
}

// Shared memory of one radial CTA, or 0 when it does not fit and the CTAs use global scratch.
static size_t radial_smem(int hm, int wm, bool smooth) {
    const size_t bytes = (size_t)radial_cta_doubles(hm, wm, smooth) * sizeof(double);
    return bytes <= 220 * 1024 ? bytes : 0;
}

constexpr int kRadialScratchCtas = 148 * 4;

int spx_rebuild_contours(int kind, const double* centers, const double* center_local, const double* eigenvalues,
                         const double* axes, const double* edge_px, const int* origins, int n, int n_angles,
                         double* contours, void* stream) {
    SPX_REQUIRE(kind >= 0 && kind <= 2 && n >= 0 && n_angles >= 1, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(contours && (kind != 2 || (center_local && edge_px && origins)) &&
                    (kind == 2 || (eigenvalues && axes && (kind == 0 ? centers != nullptr : (center_local && origins)))),
                "null pointer");
    const long long total = (long long)n * (n_angles + 1);
    k_rebuild_contours<<<grid_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        kind, centers, center_local, eigenvalues, axes, edge_px, origins, n, n_angles, contours);
    return check_launch("k_rebuild_contours");
}

size_t spx_radial_workspace_bytes(int hm, int wm, int smooth) {
    if (radial_smem(hm, wm, smooth != 0)) return 256;
    return (size_t)kRadialScratchCtas * radial_cta_doubles(hm, wm, smooth != 0) * sizeof(double) + 256;
}

}  // extern "C"

template <bool kSmooth, int kRays>
static int launch_radial(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                         int wm, int width, int n_angles, double radial_step, int n_radii, const double* smooth_w,
                         int smooth_r, const spx_method_out* halfmax, const spx_method_out* gradient, void* workspace,
                         cudaStream_t s) {
    const size_t smem = radial_smem(hm, wm, kSmooth);
    double* scratch = nullptr;
    int blocks;
    if (smem) {
        if (smem + 2 * kTrigMax * sizeof(double) > 48 * 1024)  // with the static cos / sin table
            SPX_CUDA(cudaFuncSetAttribute(k_radial_cd<kSmooth, kRays>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        int per_sm = 0;
        SPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_radial_cd<kSmooth, kRays>, kRadialThreads,
                                                               smem));
        blocks = (int)std::min<long long>(n, 148LL * std::max(per_sm, 1));
    } else {
        SPX_REQUIRE((reinterpret_cast<uintptr_t>(workspace) & 15) == 0, "workspace must be 16-byte aligned");
        scratch = static_cast<double*>(workspace);
        blocks = std::min(n, kRadialScratchCtas);
    }
    k_radial_cd<kSmooth, kRays><<<blocks, kRadialThreads, smem, s>>>(
        cleaned, voronoi, reinterpret_cast<const int4*>(boxes), which, n, hm, wm, width, n_angles, radial_step, n_radii,
        smooth_w, smooth_r, scratch, method_out(halfmax), method_out(gradient));
    return check_launch("k_radial_cd");
}

extern "C" {

int spx_radial_cd(const double* cleaned, const int* voronoi, const int* boxes, const int* which, int n, int hm,
                  int wm, int width, int n_angles, double radial_step, const double* smooth_weights,
                  int smooth_radius, const spx_method_out* halfmax, const spx_method_out* gradient, void* workspace,
                  size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && n_angles >= 1 && radial_step > 0 && smooth_radius >= 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(cleaned && voronoi && boxes && (halfmax || gradient), "null pointer");
    const bool smooth = smooth_weights != nullptr;
    SPX_REQUIRE(workspace_bytes >= spx_radial_workspace_bytes(hm, wm, smooth), "workspace too small");
    for (const spx_method_out* o : {halfmax, gradient})
        if (o) SPX_REQUIRE(o->centers && o->status && o->metrics && o->center_local && o->edge_px && o->n_metrics >= 8,
                           "null pointer or too few metric columns");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // radii = np.arange(0, hypot(hm, wm) + step, step)
    const double stop = hypot((double)hm, (double)wm) + radial_step;
    const int n_radii = (int)ceil(stop / radial_step);
    const int rays = tuning().radial_rays;
    auto go = [&](auto smooth_c, auto rays_c) {
        return launch_radial<decltype(smooth_c)::value, decltype(rays_c)::value>(
            cleaned, voronoi, boxes, which, n, hm, wm, width, n_angles, radial_step, n_radii,
            smooth ? smooth_weights : nullptr, smooth ? smooth_radius : 0, halfmax, gradient, workspace, s);
    };
    using T = std::true_type;
    using F = std::false_type;
    using R0 = std::integral_constant<int, 0>;
    using R2 = std::integral_constant<int, 2>;
    if (smooth) return rays == 2 ? go(T{}, R2{}) : go(T{}, R0{});
    return rays == 2 ? go(F{}, R2{}) : go(F{}, R0{});
}

}  // extern "C"
