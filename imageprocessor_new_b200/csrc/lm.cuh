// One warp fits one 2-D Gaussian to one cell by Levenberg-Marquardt.
//
// Model (subpx/_cpu/deblend.py:9-12, 48-71): params [A, x0, y0, u1, u2, u3], precision L L^T with
// L = [[e^u1, 0], [u2, e^u3]]; value A exp(-(a^2 + b^2) / 2), a = e^u1 dx + u2 dy, b = e^u3 dy.
// Iteration (fit_gaussians_batch, subpx/_cpu/deblend.py:174-254): normal equations J^T J and J^T r
// over the cell's mask pixels, damping lam * diag + 1e-12, trial clipped to A in [0, 3 max|d|] and
// u1, u3 in [-log(cap), -log(0.5)], accepted when the cost does not rise (lam / 3, else lam * 4);
// stop when the relative cost drop is <= 1e-12, max |step| < 1e-7, lam > 1e12 or after max_iter.
//
// Layout: the cell's mask pixels are compacted into (value, packed local x | y << 16) arrays; lanes
// stride over them, the 27 sums are all-reduced so every lane holds identical totals, and
// every lane solves the damped 6x6 system (Cholesky, fully unrolled in registers) and takes the
// same decisions, so the warp never diverges on control flow.
//
// Two arithmetics, chosen by the type of the staged values. double: every sum in FP64 (the
// reference's arithmetic). float: the residuals, the model, the Jacobian and the per-lane sums run
// in FP32 -- J^T J by plain FMA (it only shapes the step), J^T r and the cost by Kahan-compensated
// summation (they set the fixed point and the acceptance test) -- and the lane totals are added in
// FP64; the damped solve, the clipping, the acceptance test and the stop rule stay FP64.
#pragma once

#include "common.cuh"

namespace spx {

constexpr double kSigmaMin = 0.5;  // _SIGMA_MIN

struct GaussEval {
    double shape, a, b;
};

__device__ __forceinline__ GaussEval gauss_eval(const double* p, double e1, double e3, double dx, double dy) {
    GaussEval g;
    g.a = e1 * dx + p[4] * dy;
    g.b = e3 * dy;
    g.shape = exp(-0.5 * (g.a * g.a + g.b * g.b));
    return g;
}

// Solves (N + diag(lam * N_ii + 1e-12)) s = g for the symmetric 6x6 N given by its upper triangle
// (21 values, row-major) by Cholesky; NaN propagates into s when the matrix is not positive. The
// factor keeps the reciprocals of its diagonal (one rsqrt per pivot, multiplications instead of
// the square roots and divisions, which sit on the fit's critical path).
__device__ __forceinline__ void damped_solve(const double* nu, const double* g, double lam, double* s) {
    // Dense 6x6 storage with compile-time indices only, so the factor stays in registers.
    double U[6][6];
    int q = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j)
            if (j >= i) {
                double v = nu[q++];
                if (i == j) v = v + (lam * v + 1e-12);
                U[i][j] = v;
            }
    // In-place Cholesky of the upper triangle, U^T U = M, with 1 / U_ii kept on the diagonal.
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double d = U[i][i];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (k < i) d -= U[k][i] * U[k][i];
        const double inv = rsqrt(d);  // NaN when not positive definite
        U[i][i] = inv;
#pragma unroll
        for (int j = 0; j < 6; ++j)
            if (j > i) {
                double v = U[i][j];
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    if (k < i) v -= U[k][i] * U[k][j];
                U[i][j] = v * inv;
            }
    }
    // U^T y = g, then U s = y.
    double y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double v = g[i];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (k < i) v -= U[k][i] * y[k];
        y[i] = v * U[i][i];
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double v = y[i];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (k > i) v -= U[i][k] * s[k];
        s[i] = v * U[i][i];
    }
}

// Warp totals of the 27 sums on every lane with the additions of a butterfly all-reduce (the same
// partial sums meet at every level, so the totals are identical to 27 separate butterflies) but as a
// reduce-scatter: at each level a lane keeps half of its slots, adding its partner's copy of them,
// so 31 additions and shuffles replace 135; lane i then holds total i and broadcasts it.
// With `slot` (shared memory, 27 doubles) the totals go there instead (lane i writes total i) and s is
// left as it was; without it every lane's s receives them.
__device__ __forceinline__ void warp_allreduce27(double* s, int lane, double* slot = nullptr) {
    double a[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) a[i] = i < 27 ? s[i] : 0.0;
#pragma unroll
    for (int half = 16; half >= 1; half >>= 1) {
        const bool upper = (lane & half) != 0;
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const double send = upper ? a[j] : a[j + half];
            const double keep = upper ? a[j + half] : a[j];
            a[j] = keep + __shfl_xor_sync(0xffffffffu, send, half);
        }
    }
    if (slot) {
        // The totals stay in the shared-memory slot (lane i writes total i), where the solve reads
        // them, instead of 27 registers on every lane.
        if (lane < 27) slot[lane] = a[0];
        __syncwarp();
        return;
    }
#pragma unroll
    for (int i = 0; i < 27; ++i) s[i] = __shfl_sync(0xffffffffu, a[0], i);
}

// One pass over the pixels at params q: the 21 upper-triangle entries of J^T J and the 6 of J^T r
// as warp totals into slot[0..26] (shared memory) and the cost sum of r^2 with r = v - A shape
// (numpy's model-then-residual order), returned on all lanes.
__device__ __forceinline__ double warp_normal_pass(const double* q, const double* v, const int* xy, int n, int lane,
                                                   double* slot) {
    double s[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) s[i] = 0.0;
    double acc = 0.0;
    const double e1 = exp(q[3]), e3 = exp(q[5]);
    for (int k = lane; k < n; k += 32) {
        const int c = xy[k];
        const double dx = (double)(c & 0xffff) - q[1], dy = (double)(c >> 16) - q[2];
        const GaussEval g = gauss_eval(q, e1, e3, dx, dy);
        const double model = q[0] * g.shape;
        const double r = v[k] - model;
        acc += r * r;
        double J[6];
        J[0] = g.shape;
        J[1] = model * (g.a * e1);
        J[2] = model * (g.a * q[4] + g.b * e3);
        J[3] = -model * (g.a * e1 * dx);
        J[4] = -model * (g.a * dy);
        J[5] = -model * (g.b * e3 * dy);
        int t = 0;
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j) s[t++] += J[i] * J[j];
#pragma unroll
        for (int i = 0; i < 6; ++i) s[21 + i] += J[i] * r;
    }
    warp_allreduce27(s, lane, slot);
    return warp_sum(acc);
}

// Kahan-compensated FP32 running sum; s - c is the total to about twice FP32 precision.
struct KahanF {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float x) {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double total() const { return (double)s - (double)c; }
};

// Exact float of a 16-bit unsigned field: the field as the mantissa of 2^23, minus 2^23.
__device__ __forceinline__ float u16_to_float(int u) { return __int_as_float(0x4b000000 | u) - 8388608.0f; }

// The FP32 pass: as warp_normal_pass above with the per-pixel arithmetic and lane sums in FP32
// (ROI-local coordinates keep dx, dy within a few ulp of 64) and FP64 warp totals.
__device__ __forceinline__ double warp_normal_pass(const double* q, const float* v, const int* xy, int n, int lane,
                                                   double* slot) {
    double s[27];
    float jj[21];
#pragma unroll
    for (int i = 0; i < 21; ++i) jj[i] = 0.0f;
    KahanF jr[6], cost;
    const float e1 = (float)exp(q[3]), e3 = (float)exp(q[5]);
    const float A = (float)q[0], x0 = (float)q[1], y0 = (float)q[2], u2 = (float)q[4];
    for (int k = lane; k < n; k += 32) {
        const int c = xy[k];
        const float dx = u16_to_float(c & 0xffff) - x0, dy = u16_to_float(c >> 16) - y0;
        const float a = fmaf(e1, dx, u2 * dy), b = e3 * dy;
        const float shape = __expf(-0.5f * fmaf(a, a, b * b));
        const float model = A * shape;
        const float r = v[k] - model;
        cost.add(r * r);
        float J[6];
        J[0] = shape;
        J[1] = model * (a * e1);
        J[2] = model * fmaf(a, u2, b * e3);
        J[3] = -model * (a * e1 * dx);
        J[4] = -model * (a * dy);
        J[5] = -model * (b * e3 * dy);
        int t = 0;
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j, ++t) jj[t] = fmaf(J[i], J[j], jj[t]);
#pragma unroll
        for (int i = 0; i < 6; ++i) jr[i].add(J[i] * r);
    }
#pragma unroll
    for (int i = 0; i < 21; ++i) s[i] = (double)jj[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) s[21 + i] = jr[i].total();
    warp_allreduce27(s, lane, slot);
    return warp_sum(cost.total());
}

// Fits p (ROI-local, identical on all lanes) to the n compacted pixels. Returns the number of
// iterations run. `cap` is the cell's sigma cap, `amp_cap` 3 * max(max|v|, 1e-12).
//
// Each trial's cost is evaluated in the same pass as its normal equations. Every pass leaves its
// sums in one of the warp's two shared-memory slots (`slots`, 54 doubles): the pass at the kept
// params wrote slot `kept`, which the solve reads; a trial writes the other one, which becomes the
// kept slot when the trial is accepted (the usual case) and is overwritten by the next trial when
// it is not. The sums never occupy registers during the solve. The arithmetic of every sum is that
// of separate Jacobian and cost passes.
// `cost_tol` is the relative cost drop at or below which an accepted step ends the fit (1e-12, the
// reference's rule, by default).
// `final_cost` (optional) receives the cost at the returned params (the same on every lane).
template <typename T>
__device__ inline int warp_lm_fit(double* p, const T* v, const int* xy, int n, double cap, double amp_cap,
                                  int max_iter, int lane, double* slots, double cost_tol = 1e-12,
                                  double* final_cost = nullptr) {
    int kept = 0;
    double cost = warp_normal_pass(p, v, xy, n, lane, slots);
    if (final_cost) *final_cost = cost;
    if (!isfinite(cost)) return 0;
    double lam = 1e-3;
    const double lo = -log(cap), hi = -log(kSigmaMin);
    int it = 0;
    for (; it < max_iter; ++it) {
        double step[6];
        damped_solve(slots + 27 * kept, slots + 27 * kept + 21, lam, step);
        double trial[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) trial[i] = p[i] + step[i];
        // np.clip semantics: NaN passes through.
        trial[0] = trial[0] < 0.0 ? 0.0 : (trial[0] > amp_cap ? amp_cap : trial[0]);
        trial[3] = trial[3] < lo ? lo : (trial[3] > hi ? hi : trial[3]);
        trial[5] = trial[5] < lo ? lo : (trial[5] > hi ? hi : trial[5]);
        double smax = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) smax = fmax(smax, fabs(step[i]));
        // fmax ignores NaN; a NaN step is not "small" (np.abs(nan) < 1e-7 is False).
        bool small = smax < 1e-7;
#pragma unroll
        for (int i = 0; i < 6; ++i) small = small && !isnan(step[i]);
        // The trial's sums go to the other slot; a rejected trial leaves the kept slot as it was.
        const double new_cost = warp_normal_pass(trial, v, xy, n, lane, slots + 27 * (kept ^ 1));
        const bool better = isfinite(new_cost) && new_cost <= cost;
        const bool done = (better && (cost - new_cost <= cost_tol * fmax(cost, 1e-300))) || small;
        if (better) {
#pragma unroll
            for (int i = 0; i < 6; ++i) p[i] = trial[i];
            lam /= 3.0;
            cost = new_cost;
            kept ^= 1;
        } else {
            lam *= 4.0;
        }
        if (done || lam > 1e12) { ++it; break; }
    }
    __syncwarp();
    if (final_cost) *final_cost = cost;
    return it;
}

// sigma_major of the Cholesky parameters in closed form: the precision L L^T has determinant
// (e1 e3)^2, so its smaller eigenvalue is that over the larger one.
__device__ __forceinline__ double sigma_major(const double* p) {
    const double e1 = exp(p[3]), u2 = p[4], e3 = exp(p[5]);
    const double a = e1 * e1, b = e1 * u2, c = u2 * u2 + e3 * e3;
    const double half = (a - c) / 2;
    const double larger = (a + c) / 2 + sqrt(half * half + b * b);
    const double smaller = larger > 0 ? (e1 * e3) * (e1 * e3) / larger : 0.0;
    return 1.0 / sqrt(fmax(smaller, 1e-300));
}

}  // namespace spx
