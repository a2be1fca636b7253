// Joint deblending on the device: background map + one 2-D Gaussian per hole.
//
// Reference: subpx/_cpu/deblend.py (deblend 421-522, fit_gaussians_batch 174-254, initial_params
// 152-171, fit_status 262-277, clean_cells 136-149, render_models 87-107, _tile_medians 280-291,
// _upsample_rows / _upsample_tiles / _tile_centers 294-320) and subpx/_gpu/cells.py:11-38 (cell
// boxes and masks). Host code (Python) drives the outer iteration and the tile interpolation; every
// per-pixel and per-cell step is a kernel here.
//
// Cells are implicit: cell j is box j (origin, size) intersected with Voronoi label j, so no mask
// stack is stored. A fit kernel stages each cell's cleaned pixels (image - background - (model -
// own model)) once into the warp's shared-memory slice and runs the whole LM loop there; a work
// queue hands cells to persistent warps. The model image is gathered, not scattered: each 16x16
// tile sums the truncated Gaussians that reach it in increasing cell order (NumPy's bincount order),
// so it is deterministic without atomics.

#include "bins.cuh"
#include "image.cuh"
#include "lm.cuh"
#include "select.cuh"

namespace spx {
namespace {

constexpr int kFitWarpsMax = 8;  // largest tuning().fit_warps (sizes the global staging fallback)
// Static shared memory of the fit kernels: two 27-double LM sum slots per warp.
constexpr int kLmSlotBytes = kFitWarpsMax * 54 * (int)sizeof(double);

__device__ __forceinline__ int render_radius(const double* p, int cap) {
    double r = ceil(4.0 * sigma_major(p));
    if (!(r >= 2.0)) r = 2.0;  // NaN -> 2, as np.clip(nan) would not, but NaN params are never rendered
    if (r > (double)cap) r = (double)cap;
    return (int)r;
}

// ------------------------------------------------------------------------------- cell geometry

__global__ void k_cells_setup(const double* rows, int n, int pad, int H, int W, const int* vor,
                              int4* boxes, int* counts, double* caps) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int j = blockIdx.x * warps + (threadIdx.x >> 5); j < n; j += gridDim.x * warps) {
        const double* r = rows + 6LL * j;
        // int() truncates toward zero, as astype(np.int32).
        const int x0 = max(0, (int)r[0] - pad), y0 = max(0, (int)r[1] - pad);
        const int x1 = min(W, (int)(r[0] + r[2]) + pad), y1 = min(H, (int)(r[1] + r[3]) + pad);
        const int bw = max(0, x1 - x0), bh = max(0, y1 - y0);
        int c = 0;
        for (int k = lane; k < bw * bh; k += 32) {
            const int yy = y0 + k / bw, xx = x0 + k % bw;
            c += vor[(long long)yy * W + xx] == j;
        }
        c = warp_sum_i(c);
        if (lane == 0) {
            boxes[j] = make_int4(x0, y0, bw, bh);
            counts[j] = c;
            caps[j] = fmax(1.0, sqrt((double)c / 3.141592653589793));
        }
    }
}

// --------------------------------------------------------------------------------- fit status

// fit_status (subpx/_cpu/deblend.py:262-277) of ROI-local params p of cell j.
__device__ __forceinline__ int fit_status_of(const double* p, double cap, int j, int4 box, int hm, int wm, const int* vor, int W) {
    for (int i = 0; i < 6; ++i)
        if (!isfinite(p[i])) return SPX_ST_FIT_DIVERGED;
    int st = SPX_ST_OK;
    const double sig = sigma_major(p);
    if (p[0] <= 0.0 || sig >= 0.999 * cap) st = SPX_ST_NON_GAUSSIAN_FIT;
    // np.round (half to even) of the centre, clipped to the stack.
    int cy = (int)rint(p[2]), cx = (int)rint(p[1]);
    cy = min(max(cy, 0), hm - 1);
    cx = min(max(cx, 0), wm - 1);
    bool inside = p[1] >= -0.5 && p[1] <= wm - 0.5 && p[2] >= -0.5 && p[2] <= hm - 0.5;
    inside = inside && cx < box.z && cy < box.w && vor[(long long)(box.y + cy) * W + (box.x + cx)] == j;
    if (st == SPX_ST_OK && !inside) st = SPX_ST_CENTER_OUTSIDE_CELL;
    return st;
}

// ---------------------------------------------------------------------------------- staging

// Compacts cell j's mask pixels: v[slot] = value(yy, xx) (box-local coords), xy[slot] packed.
// Returns the pixel count (same on all lanes).
template <typename T, typename F>
__device__ int stage_cell(int4 box, int j, const int* vor, int W, T* v, int* xy, int lane, F value) {
    int base = 0;
    const int P = box.z * box.w;
    for (int k0 = 0; k0 < P; k0 += 32) {
        const int k = k0 + lane;
        bool in = false;
        int yy = 0, xx = 0;
        if (k < P) {
            yy = k / box.z;
            xx = k - yy * box.z;
            in = vor[(long long)(box.y + yy) * W + (box.x + xx)] == j;
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
            const int slot = base + __popc(m & ((1u << lane) - 1u));
            v[slot] = (T)value(yy, xx);
            xy[slot] = xx | (yy << 16);
        }
        base += __popc(m);
    }
    __syncwarp();
    return base;
}

// ------------------------------------------------------------------- narrow boxes (<= 32 columns)

// A box at most 32 columns wide and kMaskRowsMax rows high keeps one 32-bit in-cell mask per box
// row (bit xx of row yy: vor(box.y + yy, box.x + xx) == j) in the warp's LM slots, which are free
// before its fit. The border test and the staging then read the Voronoi labels once, lane xx
// handling column xx, with four rows' loads in flight together and the pixel loads typed (no dtype
// branch per load). Border values and staged pixels come out in the same row-major order as the
// general path's, so the staged cell, and with it the fit, is the same.
constexpr int kMaskRowsMax = 2 * 54;

__device__ __forceinline__ void cell_row_masks(const int* vor, int W, int4 box, int j, uint32_t* rowm, int lane) {
    for (int y0 = 0; y0 < box.w; y0 += 4) {
        int lab[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int yy = y0 + u;
            lab[u] = (yy < box.w && lane < box.z) ? vor[(long long)(box.y + yy) * W + (box.x + lane)] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t m = __ballot_sync(0xffffffffu, lab[u] == j);
            if (lane == 0 && y0 + u < box.w) rowm[y0 + u] = m;
        }
    }
    __syncwarp();
}

// Image::at for a known pixel type.
template <typename Px>
__device__ __forceinline__ double px_at(const Image& img, int y, int x) {
    const double v = (double)static_cast<const Px*>(img.data)[(long long)y * img.W + x];
    return img.sign < 0 ? -v : v;
}

// Values of the cell's border pixels (mask pixels with an 8-neighbour outside the mask or the box)
// into out[0, count), row-major; returns count.
template <typename Px>
__device__ int gather_border(const Image& img, int4 box, const uint32_t* rowm, double* out, int lane) {
    // All three of columns lane - 1, lane, lane + 1 of a row in the mask (column -1 and 32 are outside).
    auto full3 = [&](uint32_t m) { return lane >= 1 && lane <= 30 && ((m >> (lane - 1)) & 7u) == 7u; };
    int base = 0;
    for (int y0 = 0; y0 < box.w; y0 += 4) {
        bool border[4];
        double val[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int yy = y0 + u;
            border[u] = false;
            if (yy < box.w) {
                const uint32_t cur = rowm[yy];
                const uint32_t up = yy > 0 ? rowm[yy - 1] : 0u, dn = yy + 1 < box.w ? rowm[yy + 1] : 0u;
                border[u] = ((cur >> lane) & 1u) && !(full3(up) && full3(cur) && full3(dn));
            }
            val[u] = border[u] ? px_at<Px>(img, box.y + yy, box.x + lane) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t m = __ballot_sync(0xffffffffu, border[u]);
            if (border[u]) out[base + __popc(m & ((1u << lane) - 1u))] = val[u];
            base += __popc(m);
        }
    }
    __syncwarp();
    return base;
}

// stage_cell from the row masks: v[slot] = value - bg0 (rounded to T), xy[slot] packed.
template <typename Px, typename T>
__device__ int stage_cell_masked(const Image& img, int4 box, const uint32_t* rowm, double bg0, T* v, int* xy,
                                 int lane) {
    int base = 0;
    for (int y0 = 0; y0 < box.w; y0 += 4) {
        bool in[4];
        double val[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int yy = y0 + u;
            in[u] = yy < box.w && ((rowm[yy] >> lane) & 1u);
            val[u] = in[u] ? px_at<Px>(img, box.y + yy, box.x + lane) - bg0 : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t m = __ballot_sync(0xffffffffu, in[u]);
            if (in[u]) {
                const int slot = base + __popc(m & ((1u << lane) - 1u));
                v[slot] = (T)val[u];
                xy[slot] = lane | ((y0 + u) << 16);
            }
            base += __popc(m);
        }
    }
    __syncwarp();
    return base;
}

// Order statistics k1 and k2 (0-based) of n <= 128 values s[0, n), none NaN, by counting ranks
// (ties ordered by position, so the ranks are a permutation of 0..n-1): each lane ranks its up to
// four values against all n.
__device__ __forceinline__ void warp_rank_select2(const double* s, int n, int k1, int k2, int lane, double* r1,
                                                  double* r2) {
    double mine[4];
    int rank[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        mine[u] = lane + 32 * u < n ? s[lane + 32 * u] : 0.0;
        rank[u] = 0;
    }
    for (int k = 0; k < n; ++k) {
        const double x = s[k];
#pragma unroll
        for (int u = 0; u < 4; ++u) rank[u] += (x < mine[u] || (x == mine[u] && k < lane + 32 * u)) ? 1 : 0;
    }
    double c1 = 0.0, c2 = 0.0;
    bool h1 = false, h2 = false;
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if (lane + 32 * u < n) {
            if (rank[u] == k1) { c1 = mine[u]; h1 = true; }
            if (rank[u] == k2) { c2 = mine[u]; h2 = true; }
        }
    const unsigned b1 = __ballot_sync(0xffffffffu, h1), b2 = __ballot_sync(0xffffffffu, h2);
    *r1 = __shfl_sync(0xffffffffu, c1, __ffs(b1) - 1);
    *r2 = __shfl_sync(0xffffffffu, c2, __ffs(b2) - 1);
}

// Narrow-box front end of the initial fit: the 10th-percentile border background (unless a level
// is given) and the staged cell; returns the cell's pixel count.
template <typename Px, typename T>
__device__ __forceinline__ int narrow_front(const Image& img, int4 box, const uint32_t* rowm, bool level, double* vbuf, T* v,
                            int* xy, int lane, double* bg0);

// NumPy's 'linear' q-th percentile of the n values s[0, n) (any order; n >= 1), which the warp may
// reorder: rank selection of the two order statistics for n <= 128 without NaN, else a bitonic sort
// of s padded with +inf to a power of two (s holds room for it).
__device__ double warp_percentile(double* s, int n, double q, int lane) {
    bool nan = false;
    for (int i = lane; i < n; i += 32) nan = nan || isnan(s[i]);
    if (n <= 128 && !__any_sync(0xffffffffu, nan)) {
        // The index arithmetic of sorted_percentile.
        const double virt = __dmul_rn((double)(n - 1), q);
        const double below = floor(virt);
        int lo = (int)below;
        if (lo < 0) lo = 0;
        if (lo > n - 1) lo = n - 1;
        int hi = lo + 1 < n ? lo + 1 : n - 1;
        const bool last = virt >= (double)(n - 1);
        if (last) lo = hi = n - 1;
        double a, b;
        warp_rank_select2(s, n, lo, hi, lane, &a, &b);
        __syncwarp();
        if (last) return a;
        const double gamma = __dsub_rn(virt, below);
        const double diff = __dsub_rn(b, a);
        if (gamma >= 0.5) return __dsub_rn(b, __dmul_rn(diff, __dsub_rn(1.0, gamma)));
        return __dadd_rn(a, __dmul_rn(diff, gamma));
    }
    int m2 = 1;
    while (m2 < n) m2 <<= 1;
    for (int i = n + lane; i < m2; i += 32) s[i] = dinf();
    __syncwarp();
    warp_bitonic_sort(s, m2, lane);
    const double r = sorted_percentile(s, n, q);
    __syncwarp();
    return r;
}

template <typename Px, typename T>
__device__ __forceinline__ int narrow_front(const Image& img, int4 box, const uint32_t* rowm, bool level, double* vbuf, T* v,
                            int* xy, int lane, double* bg0) {
    if (!level) {
        const int nb = gather_border<Px>(img, box, rowm, vbuf, lane);
        *bg0 = nb > 0 ? warp_percentile(vbuf, nb, 0.1, lane) : 0.0;
    }
    return stage_cell_masked<Px, T>(img, box, rowm, *bg0, v, xy, lane);
}

// --------------------------------------------------------------------------------- kernels

struct FitArgs {
    Image img;
    const int* vor;
    const int4* boxes;
    const double* caps;
    int n, hm, wm;
    int cap_px;       // per-warp pixel capacity of the staging buffers
    int max_iter;
    double cost_tol;  // relative cost drop that ends a plain-start fit (1e-12: the reference's rule)
    int* queue;       // work counter (reset by the host before the launch)
    double* gbuf_v;   // global staging when shared memory is too small (else null)
    int* gbuf_xy;
    int rows_per_image;  // > 0: the image is a stack of such images; seeds are in their own image's rows
};

// Initial fit: 10th-percentile cell-border background, initial_params, LM, status.
// Optional warm start of the initial fits: per-cell starting params (ROI-local) with a validity
// flag; the border background and whether the plain start had to be used are reported.
struct WarmStart {
    const double* params;
    const uint8_t* ok;
    double* background;
    uint8_t* fallback;
    double cost_tol;  // relative cost drop that ends a warm-started fit
    double* cost;     // optional: the LM cost (sum of squared residuals) at each cell's returned params
};

// T: type of the staged cell values and of the LM's per-pixel arithmetic (double or float).
// Launch bounds: at most 8 warps, two such blocks per SM, which caps registers at 128 (a few spilled
// in the solve) so that 16 warps of 4-warp blocks fit per SM.
template <typename T, typename Px>
__global__ void __launch_bounds__(kFitWarpsMax * 32, 2) k_fit_initial(FitArgs a, const double* seeds, double background_level, int has_level,
                              double* params, uint8_t* status, int* iters, WarmStart warm) {
    extern __shared__ unsigned char smem[];
    __shared__ double lm_slots[kFitWarpsMax][54];  // kept / trial normal-equation sums per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* vbuf;  // the warp's staging buffer: border values (double), then the cell's values (T)
    int* xy;
    if (a.gbuf_v) {
        const long long w = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
        vbuf = a.gbuf_v + w * a.cap_px;
        xy = a.gbuf_xy + w * a.cap_px;
    } else {
        vbuf = reinterpret_cast<double*>(smem) + (long long)warp * a.cap_px;
        xy = reinterpret_cast<int*>(reinterpret_cast<double*>(smem) + (long long)(blockDim.x >> 5) * a.cap_px) +
             (long long)warp * a.cap_px;
    }
    T* v = reinterpret_cast<T*>(vbuf);
    while (true) {
        int j = 0;
        if (lane == 0) j = atomicAdd(a.queue, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= a.n) break;
        const int4 box = a.boxes[j];
        // Border pixels: mask pixels with an 8-neighbour outside the mask or the box. Narrow boxes
        // take the row-mask path; wider ones test the labels per pixel.
        auto in_cell = [&](int yy, int xx) {
            return yy >= 0 && xx >= 0 && yy < box.w && xx < box.z &&
                   a.vor[(long long)(box.y + yy) * a.img.W + (box.x + xx)] == j;
        };
        double bg0 = background_level;
        int n;
        if (box.z <= 32 && box.w <= kMaskRowsMax) {
            uint32_t* rowm = reinterpret_cast<uint32_t*>(lm_slots[warp]);
            cell_row_masks(a.vor, a.img.W, box, j, rowm, lane);
            n = narrow_front<Px>(a.img, box, rowm, has_level, vbuf, v, xy, lane, &bg0);
        } else {
            if (!has_level) {
                // Stage border values into v, then take the 10th percentile.
                int base = 0;
                const int P = box.z * box.w;
                for (int k0 = 0; k0 < P; k0 += 32) {
                    const int k = k0 + lane;
                    bool border = false;
                    int yy = 0, xx = 0;
                    if (k < P) {
                        yy = k / box.z;
                        xx = k - yy * box.z;
                        if (in_cell(yy, xx)) {
                            for (int dy = -1; dy <= 1 && !border; ++dy)
                                for (int dx = -1; dx <= 1; ++dx)
                                    if (!in_cell(yy + dy, xx + dx)) { border = true; break; }
                        }
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, border);
                    if (border) vbuf[base + __popc(m & ((1u << lane) - 1u))] = a.img.at(box.y + yy, box.x + xx);
                    base += __popc(m);
                }
                __syncwarp();
                bg0 = base > 0 ? warp_percentile(vbuf, base, 0.1, lane) : 0.0;
            }
            n = stage_cell(box, j, a.vor, a.img.W, v, xy, lane, [&](int yy, int xx) {
                return a.img.at(box.y + yy, box.x + xx) - bg0;
            });
        }
        // initial_params: amplitude = peak, centre = seed, sigma from the core's second moment.
        double peak = -dinf();
        for (int k = lane; k < n; k += 32) peak = fmax(peak, (double)v[k]);
        peak = warp_max(peak);
        // Box origin in the seed's own image (a stack's boxes are in stack rows).
        const int box_y = a.rows_per_image > 0 ? box.y % a.rows_per_image : box.y;
        const double sx = seeds[2LL * j] - box.x, sy = seeds[2LL * j + 1] - box_y;
        double tot = 0.0, mom = 0.0, amax = 0.0;
        for (int k = lane; k < n; k += 32) {
            const double d = (double)v[k];
            amax = fmax(amax, fabs(d));
            if (d > 0.2 * peak) {
                const double dx = (double)(xy[k] & 0xffff) - sx, dy = (double)(xy[k] >> 16) - sy;
                tot += d;
                mom += d * (dx * dx + dy * dy);
            }
        }
        tot = warp_sum(tot);
        mom = warp_sum(mom);
        amax = warp_max(amax);
        const double var = (mom / fmax(tot, 1e-300)) / 2.0;
        const double sigma = sqrt(fmax(var, 0.25));
        double p[6] = {fmax(peak, 1e-12), sx, sy, -log(sigma), 0.0, -log(sigma)};
        const double cap = a.caps[j];
        const double amp_cap = 3.0 * fmax(amax, 1e-12);
        int it = 0, st = 0;
        double final_cost = dnan();
        bool fell_back = false, done = false;
        if (warm.params && (!warm.ok || warm.ok[j])) {
            // Warm start: LM from the predicted params; kept when it meets the stop rule within
            // max_iter and ends "ok", else the plain start below runs as well.
            double q[6];
            bool finite = true;
            for (int i = 0; i < 6; ++i) {
                q[i] = warm.params[6LL * j + i];
                finite = finite && isfinite(q[i]);
            }
            if (finite && q[0] > 0.0) {
                it = warp_lm_fit(q, v, xy, n, cap, amp_cap, a.max_iter, lane, lm_slots[warp], warm.cost_tol,
                                 &final_cost);
                st = fit_status_of(q, cap, j, box, a.hm, a.wm, a.vor, a.img.W);
                if (it < a.max_iter && st == SPX_ST_OK) {
                    for (int i = 0; i < 6; ++i) p[i] = q[i];
                    done = true;
                }
            }
            fell_back = !done;
        }
        if (!done) {
            it += warp_lm_fit(p, v, xy, n, cap, amp_cap, a.max_iter, lane, lm_slots[warp], a.cost_tol, &final_cost);
            st = fit_status_of(p, cap, j, box, a.hm, a.wm, a.vor, a.img.W);
        }
        if (lane == 0) {
            for (int i = 0; i < 6; ++i) params[6LL * j + i] = p[i];
            status[j] = (uint8_t)st;
            if (iters) iters[j] = it;
            if (warm.background) warm.background[j] = bg0;
            if (warm.fallback) warm.fallback[j] = fell_back;
            if (warm.cost) warm.cost[j] = final_cost;
        }
        __syncwarp();
    }
}

// One deblending iteration for every cell: clean (image - background - (model - own)), LM from the
// current params, relaxation p + relax * (fitted - p) (non-finite components step 0), status of
// the relaxed params, and max |step[1:]| (NaN unless the cell is "ok" with a finite fit).
template <typename T>
__global__ void __launch_bounds__(kFitWarpsMax * 32, 2) k_fit_iteration(FitArgs a, spx_bgmap bg, const double* model, int radius_cap,
                                const double* params, double relaxation, double* params_out,
                                uint8_t* status_out, double* maxstep, int* iters) {
    extern __shared__ unsigned char smem[];
    __shared__ double lm_slots[kFitWarpsMax][54];  // kept / trial normal-equation sums per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T* v;
    int* xy;
    if (a.gbuf_v) {
        const long long w = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
        v = reinterpret_cast<T*>(a.gbuf_v + w * a.cap_px);
        xy = a.gbuf_xy + w * a.cap_px;
    } else {
        v = reinterpret_cast<T*>(reinterpret_cast<double*>(smem) + (long long)warp * a.cap_px);
        xy = reinterpret_cast<int*>(reinterpret_cast<double*>(smem) + (long long)(blockDim.x >> 5) * a.cap_px) +
             (long long)warp * a.cap_px;
    }
    while (true) {
        int j = 0;
        if (lane == 0) j = atomicAdd(a.queue, 1);
        j = __shfl_sync(0xffffffffu, j, 0);
        if (j >= a.n) break;
        const int4 box = a.boxes[j];
        double p0[6];
        for (int i = 0; i < 6; ++i) p0[i] = params[6LL * j + i];
        const double gx0 = p0[1] + box.x, gy0 = p0[2] + box.y;
        const int r = render_radius(p0, radius_cap);
        const double e1 = exp(p0[3]), e3 = exp(p0[5]);
        const int n = stage_cell(box, j, a.vor, a.img.W, v, xy, lane, [&](int yy, int xx) {
            const int y = box.y + yy, x = box.x + xx;
            const double dx = (double)x - gx0, dy = (double)y - gy0;
            double own = 0.0;
            if (fabs(dx) <= r && fabs(dy) <= r) {
                const double aa = e1 * dx + p0[4] * dy, bb = e3 * dy;
                own = p0[0] * exp(-0.5 * (aa * aa + bb * bb));
            }
            const double raw = a.img.at(y, x);
            return (raw - bg_at(bg, y, x)) - (model[(long long)y * a.img.W + x] - own);
        });
        double amax = 0.0;
        for (int k = lane; k < n; k += 32) amax = fmax(amax, fabs((double)v[k]));
        amax = warp_max(amax);
        double p[6];
        for (int i = 0; i < 6; ++i) p[i] = p0[i];
        const double cap = a.caps[j];
        const int it =
            warp_lm_fit(p, v, xy, n, cap, 3.0 * fmax(amax, 1e-12), a.max_iter, lane, lm_slots[warp], a.cost_tol);
        if (lane == 0) {
            double q[6];
            bool finite = true;
            double ms = 0.0;
            for (int i = 0; i < 6; ++i) {
                finite = finite && isfinite(p[i]);
                const double step = isfinite(p[i]) ? p[i] - p0[i] : 0.0;
                q[i] = p0[i] + relaxation * step;
                if (i >= 1) ms = fmax(ms, fabs(step));
            }
            const int st = fit_status_of(q, cap, j, box, a.hm, a.wm, a.vor, a.img.W);
            for (int i = 0; i < 6; ++i) params_out[6LL * j + i] = q[i];
            status_out[j] = (uint8_t)st;
            maxstep[j] = (st == SPX_ST_OK && finite) ? ms : dnan();
            if (iters) iters[j] = it;
        }
        __syncwarp();
    }
}

// Global centres and render radii of all cells (for the render's bin grid).
__global__ void k_render_prep(const double* params, const int4* boxes, int n, int radius_cap,
                              double* centres, int* radius, uint8_t* valid, int* rmax) {
    int local = 0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double* p = params + 6LL * j;
        bool ok = true;
        for (int i = 0; i < 6; ++i) ok = ok && isfinite(p[i]);
        const int4 b = boxes[j];
        centres[2LL * j] = p[1] + b.x;
        centres[2LL * j + 1] = p[2] + b.y;
        const int r = ok ? render_radius(p, radius_cap) : 0;
        radius[j] = r;
        valid[j] = ok;
        local = max(local, r);
    }
    for (int o = 16; o > 0; o >>= 1) local = max(local, __shfl_xor_sync(0xffffffffu, local, o));
    if ((threadIdx.x & 31) == 0) atomicMax(rmax, local);
}

// Render tiles: Tile x Tile pixels per 256-thread block (16: one pixel per thread, 32: four rows
// per thread, 64: sixteen rows per thread, fewer tiles to gather candidates for), chosen by
// tuning().render_tile.
constexpr int kRenderCap = 2048;

// model(y, x) = sum over cells (increasing index) whose truncated square covers the pixel, each
// term A exp(-(a^2 + b^2) / 2) for |x - X0| <= r and |y - Y0| <= r (render_models).
template <int kRenderTile>
__global__ void __launch_bounds__(256) k_render(int H, int W, BinGrid g, const double* params,
                                               const double* centres, const int* radius,
                                               const int* rmax_dev, double* model, int* overflow) {
    __shared__ int cand[kRenderCap];
    __shared__ int s_n;
    const int tx0 = blockIdx.x * kRenderTile, ty0 = blockIdx.y * kRenderTile;
    const int tx1 = min(tx0 + kRenderTile, W) - 1, ty1 = min(ty0 + kRenderTile, H) - 1;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const int rmax = *rmax_dev;
    const int gx0 = bin_index((double)(tx0 - rmax - 1), g.cell, g.gw);
    const int gx1 = bin_index((double)(tx1 + rmax + 1), g.cell, g.gw);
    const int gy0 = bin_index((double)(ty0 - rmax - 1), g.cell, g.gh);
    const int gy1 = bin_index((double)(ty1 + rmax + 1), g.cell, g.gh);
    for (int gy = gy0; gy <= gy1; ++gy) {
        const int j0 = g.start[gy * g.gw + gx0], j1 = g.start[gy * g.gw + gx1 + 1];
        for (int k = j0 + threadIdx.x; k < j1; k += blockDim.x) {
            const int id = g.id[k];
            const double2 c = g.xy[k];
            const double r = (double)radius[id];
            if (c.x + r >= tx0 && c.x - r <= tx1 && c.y + r >= ty0 && c.y - r <= ty1) {
                const int slot = atomicAdd(&s_n, 1);
                if (slot < kRenderCap) cand[slot] = id;
            }
        }
    }
    __syncthreads();
    const int m = s_n;
    if (m > kRenderCap) {
        if (threadIdx.x == 0) atomicExch(overflow, 1);
        return;
    }
    // Increasing cell order by rank: ids are distinct, so each candidate's slot is the number of
    // smaller ids (one barrier instead of a bitonic network's log^2 m).
    __shared__ int sorted[kRenderCap];
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        const int id = cand[t];
        int rank = 0;
        for (int q = 0; q < m; ++q) rank += cand[q] < id;
        sorted[rank] = id;
    }
    __syncthreads();
    // Each candidate's centre, amplitude, precision factors and the integer bounds of its truncated
    // square are staged once per tile (chunks of 256), so a pixel tests a candidate with integer
    // compares and a term costs one exp. |x - cx| <= r <=> ceil(cx - r) <= x <= floor(cx + r) for
    // integer x and r: x - cx and cx -+ r are exact in FP64 for coordinates below 2^16.
    __shared__ double s_cx[256], s_cy[256], s_a[256], s_e1[256], s_u2[256], s_e3[256];
    __shared__ int4 s_box[256];  // x lo, x hi, y lo, y hi
    constexpr int kRows = kRenderTile * kRenderTile / 256;
    const int x = tx0 + (threadIdx.x % kRenderTile), yb = ty0 + (threadIdx.x / kRenderTile);
    double acc[kRows];
#pragma unroll
    for (int q = 0; q < kRows; ++q) acc[q] = 0.0;
    for (int c0 = 0; c0 < m; c0 += 256) {
        const int cn = min(256, m - c0);
        if ((int)threadIdx.x < cn) {
            const int id = sorted[c0 + threadIdx.x];
            const double* p = params + 6LL * id;
            const double cxv = centres[2LL * id], cyv = centres[2LL * id + 1], rv = (double)radius[id];
            s_cx[threadIdx.x] = cxv;
            s_cy[threadIdx.x] = cyv;
            s_box[threadIdx.x] = make_int4((int)ceil(cxv - rv), (int)floor(cxv + rv), (int)ceil(cyv - rv),
                                           (int)floor(cyv + rv));
            s_a[threadIdx.x] = p[0];
            s_e1[threadIdx.x] = exp(p[3]);
            s_u2[threadIdx.x] = p[4];
            s_e3[threadIdx.x] = exp(p[5]);
        }
        __syncthreads();
        for (int k = 0; k < cn; ++k) {
            const int4 bx = s_box[k];
            if (x < bx.x || x > bx.y) continue;
            const double dx = (double)x - s_cx[k];
#pragma unroll
            for (int q = 0; q < kRows; ++q) {
                const int yq = yb + q * (256 / kRenderTile);
                if (yq < bx.z || yq > bx.w) continue;
                const double dy = (double)yq - s_cy[k];
                const double aa = s_e1[k] * dx + s_u2[k] * dy, bb = s_e3[k] * dy;
                const double val = s_a[k] * exp(-0.5 * (aa * aa + bb * bb));
                if (val != 0.0) acc[q] += val;
            }
        }
        __syncthreads();
    }
    if (x < W)
#pragma unroll
        for (int q = 0; q < kRows; ++q) {
            const int y = yb + q * (256 / kRenderTile);
            if (y < H) model[(long long)y * W + x] = acc[q];
        }
}

// Cleaned cells (image - background - (model - own)) of the cells in `which` (all when null) as
// an (n_out, hm, wm) stack, zero outside each cell (DeblendState.cleaned).
__global__ void k_clean_stack(Image img, const int* vor, const int4* boxes, const double* params,
                              int radius_cap, spx_bgmap bg, const double* model, const int* which,
                              int n_out, int hm, int wm, double* out) {
    const long long total = (long long)n_out * hm * wm;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int c, k;
        divmod_idx(t, hm * wm, &c, &k);
        const int yy = k / wm, xx = k % wm;
        const int j = which ? which[c] : c;
        const int4 b = boxes[j];
        double v = 0.0;
        if (yy < b.w && xx < b.z) {
            const int y = b.y + yy, x = b.x + xx;
            if (vor[(long long)y * img.W + x] == j) {
                const double* p = params + 6LL * j;
                const double dx = (double)x - (p[1] + b.x), dy = (double)y - (p[2] + b.y);
                const int r = render_radius(p, radius_cap);
                double own = 0.0;
                if (fabs(dx) <= r && fabs(dy) <= r) {
                    const double aa = exp(p[3]) * dx + p[4] * dy, bb = exp(p[5]) * dy;
                    own = p[0] * exp(-0.5 * (aa * aa + bb * bb));
                }
                v = (img.at(y, x) - bg_at(bg, y, x)) - (model[(long long)y * img.W + x] - own);
            }
        }
        out[t] = v;
    }
}

// The measured cells from their stored masks (the compact result files' rebuild): out = image -
// background - (model - own Gaussian) on the mask, 0 elsewhere, with global params, the same
// arithmetic as k_clean_stack.
__global__ void k_clean_masked(Image img, const uint8_t* masks, const int* origins, const double* params_global,
                               int radius_cap, spx_bgmap bg, const double* model, int n, int hm, int wm,
                               double* out) {
    const long long total = (long long)n * hm * wm;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int c, k;
        divmod_idx(t, hm * wm, &c, &k);
        double v = 0.0;
        if (masks[t]) {
            const int y = origins[2LL * c + 1] + k / wm, x = origins[2LL * c] + k % wm;
            const double* p = params_global + 6LL * c;
            const double dx = (double)x - p[1], dy = (double)y - p[2];
            const int r = render_radius(p, radius_cap);
            double own = 0.0;
            if (fabs(dx) <= r && fabs(dy) <= r) {
                const double aa = exp(p[3]) * dx + p[4] * dy, bb = exp(p[5]) * dy;
                own = p[0] * exp(-0.5 * (aa * aa + bb * bb));
            }
            v = (img.at(y, x) - bg_at(bg, y, x)) - (model[(long long)y * img.W + x] - own);
        }
        out[t] = v;
    }
}

// Support labels of deblended cells for re-refining their centres (detect_centers with
// background="model", subpx/centers.py:258-268): cell j's window of the (n x hm x wm) cleaned stack,
// laid out as rows j*hm .. j*hm + hm - 1 of a tall image, gets label j + 1 where the cell's mask
// holds and the cleaned value exceeds 0.2 x the peak (the fitted amplitude when finite and
// positive, else the largest cleaned value on the mask); rows_out[j] = the window as a refine row
// [0, j*hm, wm, hm, j + 1]. One warp per cell.
__global__ void k_support_labels(const double* cleaned, const int* vor, const int4* boxes, const double* params, int n,
                                 int hm, int wm, int W, int* labels, int* rows_out) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    const int area = hm * wm;
    for (int j = blockIdx.x * warps + (threadIdx.x >> 5); j < n; j += gridDim.x * warps) {
        const int4 b = boxes[j];
        const double* c = cleaned + (long long)j * area;
        auto inside = [&](int k) {
            const int yy = k / wm, xx = k % wm;
            return yy < b.w && xx < b.z && vor[(long long)(b.y + yy) * W + b.x + xx] == j;
        };
        double peak = params[6LL * j];
        if (!(isfinite(peak) && peak > 0.0)) {
            double m = -dinf();
            for (int k = lane; k < area; k += 32)
                if (inside(k)) m = fmax(m, c[k]);
            peak = warp_max(m);
        }
        const double level = __dmul_rn(0.2, peak);
        for (int k = lane; k < area; k += 32)
            labels[(long long)j * area + k] = (inside(k) && c[k] > level) ? j + 1 : 0;
        if (lane < 5) {
            const int v[5] = {0, j * hm, wm, hm, j + 1};
            rows_out[5LL * j + lane] = v[lane];
        }
    }
}

// ------------------------------------------------------------------------------ tile medians

constexpr int kTileThreads = 512;
constexpr int kTileSmemKeys = 24576;  // keys held in shared memory (192 KiB)

struct TileSel {
    Image img;
    const double* model;      // null: residual = image
    const unsigned int* d2;   // distance map (free mode)
    const uint8_t* usable;    // null: all usable
    int mode;                 // SPX_TILE_FREE: model < thr_model & dist >= thr_dist; SPX_TILE_USABLE; SPX_TILE_ALL
    double thr_model;
    unsigned long long d2_min;  // sqrt((double)d2) >= thr_dist  <=>  d2 >= d2_min (set by the host)
    // A pixel's loads (pixel of type Px, model, distance, usable flag), none of them conditional on
    // another's value, so that a thread's loads of several pixels are in flight together.
    struct Loaded {
        double raw, m;
        unsigned int dd;
        uint8_t use;
    };
    template <typename Px>
    __device__ __forceinline__ Loaded load(long long i) const {
        Loaded q;
        q.raw = (double)static_cast<const Px*>(img.data)[i];
        q.m = model ? model[i] : 0.0;
        q.dd = mode == SPX_TILE_FREE ? d2[i] : 0u;
        q.use = (mode != SPX_TILE_ALL && usable) ? usable[i] : (uint8_t)1;
        return q;
    }
    // The pixel's residual and whether the tile's median takes it.
    __device__ __forceinline__ bool decide(const Loaded& q, double* value) const {
        bool ok = true;
        if (mode != SPX_TILE_ALL) {
            ok = q.use != 0;
            if (mode == SPX_TILE_FREE) ok = ok && q.m < thr_model && (unsigned long long)q.dd >= d2_min;
        }
        *value = (img.sign < 0 ? -q.raw : q.raw) - q.m;
        return ok;
    }
    template <typename Px>
    __device__ __forceinline__ bool select(int y, int x, double* value) const {
        return decide(load<Px>((long long)y * img.W + x), value);
    }
};

// Median (mean of the two middle values, NaN when empty) and count of the selected residuals of
// each tile: the selected pixels' order-preserving 64-bit keys are staged in shared memory (each
// warp reserves its slots with one atomic), with their smallest and largest key, and cta_select
// finds the middle one(s).
template <typename Px>
__global__ void __launch_bounds__(kTileThreads, 2) k_tile_median(TileSel sel, int tile, int nx, int smem_keys,
                                                              double* medians, long long* counts) {
    extern __shared__ unsigned long long keys[];
    __shared__ int hist[2048];
    __shared__ int warp_tot[32], s_pick[3];
    __shared__ int s_count;
    __shared__ unsigned long long s_keys[2], s_kmin, s_kmax;
    const int ty = blockIdx.x / nx, tx = blockIdx.x % nx;
    const int y0 = ty * tile, x0 = tx * tile;
    const int th = min(tile, sel.img.H - y0), tw = min(tile, sel.img.W - x0);
    const long long P = (long long)th * tw;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_count = 0;
        s_kmin = ~0ull;
        s_kmax = 0;
    }
    __syncthreads();
    // Pass 0: count and (when they fit) stage the keys, kPass0 pixels per thread at a time so
    // that their loads are in flight together. The loop bounds are the same for every thread, so
    // the warp votes are over full warps.
    constexpr int kPass0 = 8;
    unsigned long long kmin = ~0ull, kmax = 0;
    for (int k0 = 0; k0 < (int)P; k0 += kPass0 * blockDim.x) {
        double v[kPass0];
        bool take[kPass0];
        TileSel::Loaded q[kPass0];
#pragma unroll
        for (int u = 0; u < kPass0; ++u) {
            const int k = min(k0 + u * (int)blockDim.x + (int)threadIdx.x, (int)P - 1);
            const int yy = k / tw, xx = k - yy * tw;
            q[u] = sel.load<Px>((long long)(y0 + yy) * sel.img.W + (x0 + xx));
        }
#pragma unroll
        for (int u = 0; u < kPass0; ++u) {
            take[u] = sel.decide(q[u], &v[u]) && k0 + u * (int)blockDim.x + (int)threadIdx.x < (int)P;
        }
#pragma unroll
        for (int u = 0; u < kPass0; ++u) {
            const unsigned ballot = __ballot_sync(0xffffffffu, take[u]);
            if (ballot == 0u) continue;
            int base = 0;
            if (lane == 0) base = atomicAdd(&s_count, __popc(ballot));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (take[u]) {
                const int slot = base + __popc(ballot & ((1u << lane) - 1u));
                const unsigned long long key = order_key(v[u]);
                if (slot < smem_keys) keys[slot] = key;
                kmin = min(kmin, key);
                kmax = max(kmax, key);
            }
        }
    }
    kmin = warp_min_u64(kmin);
    kmax = warp_max_u64(kmax);
    if (lane == 0) {
        atomicMin(&s_kmin, kmin);
        atomicMax(&s_kmax, kmax);
    }
    __syncthreads();
    const int c = s_count;
    if (c == 0) {
        if (threadIdx.x == 0) {
            medians[blockIdx.x] = dnan();
            counts[blockIdx.x] = 0;
        }
        return;
    }
    const bool in_smem = c <= smem_keys;
    auto for_keys = [&](auto&& fn) {
        if (in_smem) {
            for (int i = threadIdx.x; i < c; i += blockDim.x) fn(keys[i]);
        } else {
            for (int k = threadIdx.x; k < (int)P; k += blockDim.x) {
                const int yy = k / tw, xx = k - yy * tw;
                double v;
                if (sel.select<Px>(y0 + yy, x0 + xx, &v)) fn(order_key(v));
            }
        }
    };
    unsigned long long k1, k2;
    cta_select<kTileThreads>(for_keys, (c - 1) / 2, (c & 1) == 0, s_kmin, s_kmax, hist, warp_tot, s_pick, s_keys,
                             &k1, &k2);
    if (threadIdx.x == 0) {
        medians[blockIdx.x] = __ddiv_rn(__dadd_rn(key_value(k1), key_value(k2)), 2.0);
        counts[blockIdx.x] = c;
    }
}

// rows[j][x] = np.interp(x, xc, medians[j]) with xc the tile-centre columns.
__global__ void k_bg_rows(const double* medians, int ny, int nx, int tile, int W, double* rows) {
    const long long total = (long long)ny * W;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int j, x;
        divmod_idx(t, W, &j, &x);
        const double* fp = medians + (long long)j * nx;
        auto xc = [&](int i) { return (double)(i * tile + min((i + 1) * tile, W) - 1) / 2.0; };
        const double xv = (double)x;
        double res;
        if (nx == 1) {
            res = fp[0];
        } else if (xv < xc(0)) {
            res = fp[0];
        } else if (xv > xc(nx - 1)) {
            res = fp[nx - 1];
        } else {
            // xc(i) <= x < xc(i+1); tiles are `tile` wide so the interval is x / tile or one below.
            int i = min(max(x / tile, 0), nx - 1);
            while (i > 0 && xc(i) > xv) --i;
            while (i < nx - 1 && xc(i + 1) <= xv) ++i;
            if (i == nx - 1 || xc(i) == xv) {
                res = fp[i];
            } else {
                const double slope = __ddiv_rn(__dsub_rn(fp[i + 1], fp[i]), __dsub_rn(xc(i + 1), xc(i)));
                res = __dadd_rn(__dmul_rn(slope, __dsub_rn(xv, xc(i))), fp[i]);
                if (isnan(res)) {
                    res = __dadd_rn(__dmul_rn(slope, __dsub_rn(xv, xc(i + 1))), fp[i + 1]);
                    if (isnan(res) && fp[i] == fp[i + 1]) res = fp[i];
                }
            }
        }
        rows[t] = res;
    }
}

// residual = image - background - model at every pixel (revise_seeds' input).
__global__ void k_residual(Image img, spx_bgmap bg, const double* model, double* out) {
    const long long total = (long long)img.H * img.W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int y, x;
        divmod_idx(i, img.W, &y, &x);
        out[i] = (img.at(y, x) - bg_at(bg, y, x)) - model[i];
    }
}

// ------------------------------------------------------------------------ order statistics

// Selected values of one request: values[i * stride] where the selection holds (mask[i] != 0 when
// mask is given; finite values only when finite_only).
struct QuantileReq {
    const double* values;
    int stride;
    const uint8_t* mask;
    int finite_only;
    int n;
    int mode;     // 0: np.median; 1: np.percentile(q) with linear interpolation
    double q;
};

__device__ __forceinline__ bool q_select(const QuantileReq& r, int i, double* v) {
    // Both loads are issued whatever the mask says, so a thread's loads of several values overlap.
    const bool in = !r.mask || r.mask[i];
    const double x = r.values[(long long)i * r.stride];
    *v = x;
    return in && !(r.finite_only && !isfinite(x));
}

constexpr int kQuantThreads = 1024;
constexpr int kQuantAhead = 4;

// One CTA per request: out[2 * b] = result (NaN when nothing is selected), out[2 * b + 1] = count.
// A counting pass finds the count, whether a NaN is selected and the smallest and largest key;
// cta_select then finds the order statistics, kQuantAhead values per thread loaded before their
// histogram updates so that the loads overlap.
__global__ void __launch_bounds__(kQuantThreads) k_quantiles(const QuantileReq* reqs, double* out) {
    __shared__ int hist[2048];
    __shared__ int warp_tot[32];
    __shared__ int s_pick[3];
    __shared__ int s_count, s_nan;
    __shared__ unsigned long long s_keys[2], s_kmin, s_kmax;
    const QuantileReq r = reqs[blockIdx.x];
    if (threadIdx.x == 0) {
        s_count = s_nan = 0;
        s_kmin = ~0ull;
        s_kmax = 0;
    }
    __syncthreads();
    int c = 0, nan = 0;
    unsigned long long kmin = ~0ull, kmax = 0;
    for (int i = threadIdx.x; i < r.n; i += kQuantThreads) {
        double v;
        if (q_select(r, i, &v)) {
            ++c;
            nan += isnan(v);
            const unsigned long long key = order_key(v);
            kmin = min(kmin, key);
            kmax = max(kmax, key);
        }
    }
    kmin = warp_min_u64(kmin);
    kmax = warp_max_u64(kmax);
    atomicAdd(&s_count, c);
    atomicAdd(&s_nan, nan);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&s_kmin, kmin);
        atomicMax(&s_kmax, kmax);
    }
    __syncthreads();
    const int n = s_count;
    const bool any_nan = s_nan != 0;
    auto for_keys = [&](auto&& fn) {
        for (int i0 = threadIdx.x; i0 < r.n; i0 += kQuantAhead * kQuantThreads) {
            double v[kQuantAhead];
            bool ok[kQuantAhead];
#pragma unroll
            for (int u = 0; u < kQuantAhead; ++u) {
                const int i = i0 + u * kQuantThreads;
                ok[u] = i < r.n && q_select(r, i, &v[u]);
            }
#pragma unroll
            for (int u = 0; u < kQuantAhead; ++u)
                if (ok[u]) fn(order_key(v[u]));
        }
    };
    double res = dnan();
    if (n > 0 && !any_nan) {  // numpy: a NaN among the values makes the median / percentile NaN
        unsigned long long ka, kb;
        if (r.mode == 0) {
            cta_select<kQuantThreads>(for_keys, (n - 1) / 2, (n & 1) == 0, s_kmin, s_kmax, hist, warp_tot, s_pick,
                                      s_keys, &ka, &kb);
            res = __ddiv_rn(__dadd_rn(key_value(ka), key_value(kb)), 2.0);
        } else {
            // numpy 'linear': virtual index (n - 1) q, _lerp of the neighbours.
            const double virt = __dmul_rn((double)(n - 1), r.q);
            const double below = floor(virt);
            const int lo = min(max((int)below, 0), n - 1), hi = min(lo + 1, n - 1);
            cta_select<kQuantThreads>(for_keys, lo, hi != lo, s_kmin, s_kmax, hist, warp_tot, s_pick, s_keys, &ka,
                                      &kb);
            const double a = key_value(ka);
            const double b = key_value(kb);
            if (virt >= (double)(n - 1)) {
                res = b;
            } else {
                const double g = __dsub_rn(virt, below), diff = __dsub_rn(b, a);
                res = g >= 0.5 ? __dsub_rn(b, __dmul_rn(diff, __dsub_rn(1.0, g))) : __dadd_rn(a, __dmul_rn(diff, g));
            }
        }
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = res;
        out[2 * blockIdx.x + 1] = (double)n;
    }
}

// Per-cell amplitude, 2 sqrt(2 ln 2) sigma_major and the "good" flag (status ok and A > 0).
__global__ void k_cell_stats(const double* params, const uint8_t* status, int n, double* fwhm, uint8_t* good) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double* p = params + 6LL * j;
        good[j] = status[j] == SPX_ST_OK && p[0] > 0.0;
        fwhm[j] = 2.0 * 1.1774100225154747 * sigma_major(p);
    }
}

// map_coordinates(background map, [y, x], order=1, mode="nearest") at points [x, y].
__global__ void k_background_at(spx_bgmap bg, int H, int W, const double* pts, int n, double sign, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = pts[2 * i], y = pts[2 * i + 1];
        const double fy = floor(y), fx = floor(x);
        const double ty = y - fy, tx = x - fx;
        const int y0 = min(max((int)fy, 0), H - 1), y1 = min(max((int)fy + 1, 0), H - 1);
        const int x0 = min(max((int)fx, 0), W - 1), x1 = min(max((int)fx + 1, 0), W - 1);
        double acc = 0.0;
        acc += bg_at(bg, y0, x0) * (1.0 - ty) * (1.0 - tx);
        acc += bg_at(bg, y0, x1) * (1.0 - ty) * tx;
        acc += bg_at(bg, y1, x0) * ty * (1.0 - tx);
        acc += bg_at(bg, y1, x1) * ty * tx;
        out[i] = sign * acc;
    }
}

struct FitLayout {
    int* queue;
    double* gbuf_v;
    int* gbuf_xy;
};

int fit_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

int fit_blocks() { return fit_sms() * tuning().fit_blocks_per_sm; }

// Shared memory per block for cap_px pixels per warp; 0 when it does not fit (global staging).
size_t fit_smem(int cap_px, int warps) {
    const size_t bytes = (size_t)warps * cap_px * (sizeof(double) + sizeof(int));
    return bytes <= 200 * 1024 ? bytes : 0;
}

// Workspace layout: the staging fallback (cells too large for shared memory) always runs 4 blocks
// of 8 warps per SM, so a workspace stays valid whatever the autotuner picks later.
FitLayout fit_layout(void* ws, int cap_px, size_t* bytes) {
    Arena a(ws);
    FitLayout L;
    L.queue = a.take<int>(4);
    const bool global = fit_smem(cap_px, kFitWarpsMax) == 0;
    const long long warps = global ? (long long)fit_sms() * 4 * kFitWarpsMax : 0;
    L.gbuf_v = global ? a.take<double>(warps * cap_px) : nullptr;
    L.gbuf_xy = global ? a.take<int>(warps * cap_px) : nullptr;
    if (!global) { a.take<double>(1); a.take<int>(1); }
    if (bytes) *bytes = a.used;
    return L;
}

}  // namespace
}  // namespace spx

using namespace spx;

namespace {

int pow2_at_least(int n) {
    int m = 1;
    while (m < n) m <<= 1;
    return m;
}

template <typename Launch>
int launch_fit(const FitArgs& a0, FitLayout L, cudaStream_t s, Launch&& launch) {
    FitArgs a = a0;
    a.queue = L.queue;
    a.gbuf_v = L.gbuf_v;
    a.gbuf_xy = L.gbuf_xy;
    SPX_CUDA(cudaMemsetAsync(L.queue, 0, sizeof(int), s));
    const int warps = a.gbuf_v ? kFitWarpsMax : tuning().fit_warps;
    const size_t smem = a.gbuf_v ? 0 : fit_smem(a.cap_px, warps);
    return launch(a, smem, warps, a.gbuf_v ? fit_sms() * 4 : fit_blocks());
}

struct RenderLayout {
    BinStorage bins;
    double* centres;
    int* radius;
    uint8_t* valid;
    int* rmax;
    int* overflow;
};

RenderLayout render_layout(void* ws, int n, int H, int W, size_t* bytes) {
    Arena a(ws);
    RenderLayout L;
    L.bins = bin_layout(a, n, H, W, bin_cell_size(n, H, W, 1.0, 8.0));
    L.centres = a.take<double>(2 * (size_t)(n > 0 ? n : 1));
    L.radius = a.take<int>(n > 0 ? n : 1);
    L.valid = a.take<uint8_t>(n > 0 ? n : 1);
    L.rmax = a.take<int>(1);
    L.overflow = a.take<int>(1);
    if (bytes) *bytes = a.used;
    return L;
}

}  // namespace

extern "C" {

int spx_cells_setup(const double* rows, int n, int pad, int height, int width, const int* voronoi,
                    int* boxes, int* counts, double* caps, void* stream) {
    SPX_REQUIRE(n >= 0 && pad >= 0 && height > 0 && width > 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(rows && voronoi && boxes && counts && caps, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_cells_setup<<<grid_for(n, 8, 148 * 16), 256, 0, s>>>(rows, n, pad, height, width, voronoi,
                                                           reinterpret_cast<int4*>(boxes), counts, caps);
    return check_launch("k_cells_setup");
}

size_t spx_fit_workspace_bytes(int max_cell_pixels) {
    size_t b = 0;
    fit_layout(nullptr, pow2_at_least(max_cell_pixels > 0 ? max_cell_pixels : 1), &b);
    return b;
}

int spx_deblend_initial(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                        const int* boxes, const double* caps, const double* seeds, int n, int hm, int wm,
                        int max_cell_pixels, double background_level, int has_level, int max_iter,
                        double* params, uint8_t* status, int* iterations, void* workspace,
                        size_t workspace_bytes, void* stream) {
    return spx_deblend_initial_warm(img, dtype, sign, height, width, voronoi, boxes, caps, seeds, n, hm, wm,
                                    max_cell_pixels, background_level, has_level, max_iter, nullptr, nullptr, 1e-12,
                                    params, status, iterations, nullptr, nullptr, nullptr, nullptr, workspace,
                                    workspace_bytes, stream);
}

}  // extern "C"

namespace {

// The fit options with their defaults (FP64, the reference's 1e-12 stop rule) and checks.
int read_fit_options(const spx_fit_options* o, bool* f32, double* cost_tol, int* rows_per_image, int height) {
    *f32 = o && o->precision == SPX_FIT_F32;
    *cost_tol = o ? o->cost_tol : 1e-12;
    *rows_per_image = o ? o->rows_per_image : 0;
    SPX_REQUIRE(!o || o->precision == SPX_FIT_F64 || o->precision == SPX_FIT_F32, "bad fit precision");
    SPX_REQUIRE(*cost_tol > 0.0 && *cost_tol < 1.0, "fit cost_tol must be in (0, 1)");
    SPX_REQUIRE(*rows_per_image == 0 || (*rows_per_image > 0 && height % *rows_per_image == 0),
                "rows_per_image must be 0 or divide the image height");
    return SPX_OK;
}

template <typename T, typename Px>
int launch_fit_initial_px(const FitArgs& a0, FitLayout L, cudaStream_t s, const double* seeds,
                          double background_level, int has_level, double* params, uint8_t* status, int* iterations,
                          WarmStart warm) {
    return launch_fit(a0, L, s, [&](const FitArgs& fa, size_t smem, int warps, int blocks) -> int {
        if (smem + kLmSlotBytes > 48 * 1024)
            SPX_CUDA(cudaFuncSetAttribute(k_fit_initial<T, Px>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_fit_initial<T, Px><<<blocks, warps * 32, smem, s>>>(fa, seeds, background_level, has_level, params,
                                                               status, iterations, warm);
        return check_launch("k_fit_initial");
    });
}

// The pixel type is a template parameter of the initial fit (its narrow-box front end loads pixels
// without a dtype branch per load).
template <typename T>
int launch_fit_initial(const FitArgs& a0, FitLayout L, cudaStream_t s, const double* seeds, double background_level,
                       int has_level, double* params, uint8_t* status, int* iterations, WarmStart warm) {
    switch (a0.img.dtype) {
        case SPX_U8:
            return launch_fit_initial_px<T, uint8_t>(a0, L, s, seeds, background_level, has_level, params, status,
                                                     iterations, warm);
        case SPX_U16:
            return launch_fit_initial_px<T, uint16_t>(a0, L, s, seeds, background_level, has_level, params, status,
                                                      iterations, warm);
        case SPX_F32:
            return launch_fit_initial_px<T, float>(a0, L, s, seeds, background_level, has_level, params, status,
                                                   iterations, warm);
        default:
            return launch_fit_initial_px<T, double>(a0, L, s, seeds, background_level, has_level, params, status,
                                                    iterations, warm);
    }
}

template <typename T>
int launch_fit_iteration(const FitArgs& a0, FitLayout L, cudaStream_t s, const spx_bgmap& bg, const double* model,
                         int radius_cap, const double* params, double relaxation, double* params_out,
                         uint8_t* status_out, double* maxstep, int* iterations) {
    return launch_fit(a0, L, s, [&](const FitArgs& fa, size_t smem, int warps, int blocks) -> int {
        if (smem + kLmSlotBytes > 48 * 1024)
            SPX_CUDA(cudaFuncSetAttribute(k_fit_iteration<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_fit_iteration<T><<<blocks, warps * 32, smem, s>>>(fa, bg, model, radius_cap, params, relaxation,
                                                             params_out, status_out, maxstep, iterations);
        return check_launch("k_fit_iteration");
    });
}

}  // namespace

extern "C" {

int spx_deblend_initial_warm(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                             const int* boxes, const double* caps, const double* seeds, int n, int hm, int wm,
                             int max_cell_pixels, double background_level, int has_level, int max_iter,
                             const double* init_params, const uint8_t* init_ok, double warm_cost_tol,
                             double* params, uint8_t* status, int* iterations, double* background_out,
                             uint8_t* fallback_out, double* cost_out, const spx_fit_options* options,
                             void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(warm_cost_tol > 0.0, "warm_cost_tol must be positive");
    SPX_REQUIRE(n >= 0 && height > 0 && width > 0 && max_iter >= 1, "bad arguments");
    bool f32 = false;
    double cost_tol = 1e-12;
    int rows_per_image = 0;
    if (int e = read_fit_options(options, &f32, &cost_tol, &rows_per_image, height)) return e;
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(img && voronoi && boxes && caps && seeds && params && status && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_fit_workspace_bytes(max_cell_pixels), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int cap_px = pow2_at_least(max_cell_pixels > 0 ? max_cell_pixels : 1);
    FitLayout L = fit_layout(workspace, cap_px, nullptr);
    FitArgs a{Image{img, dtype, sign, height, width}, voronoi, reinterpret_cast<const int4*>(boxes), caps, n,
              hm, wm, cap_px, max_iter, cost_tol, nullptr, nullptr, nullptr, rows_per_image};
    const WarmStart warm{init_params, init_ok, background_out, fallback_out, warm_cost_tol, cost_out};
    return f32 ? launch_fit_initial<float>(a, L, s, seeds, background_level, has_level, params, status, iterations,
                                           warm)
               : launch_fit_initial<double>(a, L, s, seeds, background_level, has_level, params, status,
                                            iterations, warm);
}

int spx_deblend_iteration(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                          const int* boxes, const double* caps, int n, int hm, int wm, int max_cell_pixels,
                          const spx_bgmap* background, const double* model, int radius_cap,
                          const double* params, double relaxation, int max_iter, double* params_out,
                          uint8_t* status_out, double* maxstep, int* iterations, const spx_fit_options* options,
                          void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && height > 0 && width > 0 && max_iter >= 1, "bad arguments");
    bool f32 = false;
    double cost_tol = 1e-12;
    int rows_per_image = 0;
    if (int e = read_fit_options(options, &f32, &cost_tol, &rows_per_image, height)) return e;
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(img && voronoi && boxes && caps && background && model && params && params_out && status_out &&
                    maxstep && workspace,
                "null pointer");
    SPX_REQUIRE(params != params_out, "params_out must not alias params");
    SPX_REQUIRE(workspace_bytes >= spx_fit_workspace_bytes(max_cell_pixels), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int cap_px = pow2_at_least(max_cell_pixels > 0 ? max_cell_pixels : 1);
    FitLayout L = fit_layout(workspace, cap_px, nullptr);
    FitArgs a{Image{img, dtype, sign, height, width}, voronoi, reinterpret_cast<const int4*>(boxes), caps, n,
              hm, wm, cap_px, max_iter, cost_tol, nullptr, nullptr, nullptr};
    return f32 ? launch_fit_iteration<float>(a, L, s, *background, model, radius_cap, params, relaxation, params_out,
                                             status_out, maxstep, iterations)
               : launch_fit_iteration<double>(a, L, s, *background, model, radius_cap, params, relaxation,
                                              params_out, status_out, maxstep, iterations);
}

int spx_render_overflow(void* workspace, int n, int height, int width, int* flag_out, int reset, void* stream) {
    SPX_REQUIRE(workspace && flag_out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RenderLayout L = render_layout(workspace, n, height, width, nullptr);
    if (reset) {
        SPX_CUDA(cudaMemsetAsync(L.overflow, 0, sizeof(int), s));
        return SPX_OK;
    }
    SPX_CUDA(cudaMemcpyAsync(flag_out, L.overflow, sizeof(int), cudaMemcpyDeviceToHost, s));
    SPX_CUDA(cudaStreamSynchronize(s));
    return SPX_OK;
}

size_t spx_render_workspace_bytes(int n, int height, int width) {
    size_t b = 0;
    render_layout(nullptr, n, height, width, &b);
    return b;
}

int spx_render_model(const double* params, const int* boxes, int n, int height, int width, int radius_cap,
                     double* model, void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && height > 0 && width > 0 && radius_cap >= 2, "bad arguments");
    SPX_REQUIRE(model && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_render_workspace_bytes(n, height, width), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RenderLayout L = render_layout(workspace, n, height, width, nullptr);
    SPX_CUDA(cudaMemsetAsync(L.rmax, 0, sizeof(int), s));
    if (n > 0) {
        SPX_REQUIRE(params && boxes, "null pointer");
        k_render_prep<<<grid_for(n, 256), 256, 0, s>>>(params, reinterpret_cast<const int4*>(boxes), n, radius_cap,
                                                       L.centres, L.radius, L.valid, L.rmax);
        if (int e = check_launch("k_render_prep")) return e;
    }
    if (int e = bin_build(L.bins, L.centres, 2, nullptr, L.valid, n, s)) return e;
    const int tile = tuning().render_tile;
    const dim3 grid((width + tile - 1) / tile, (height + tile - 1) / tile);
    if (tile == 16)
        k_render<16><<<grid, 256, 0, s>>>(height, width, bin_view(L.bins), params, L.centres, L.radius, L.rmax, model,
                                          L.overflow);
    else if (tile == 64)
        k_render<64><<<grid, 256, 0, s>>>(height, width, bin_view(L.bins), params, L.centres, L.radius, L.rmax, model,
                                          L.overflow);
    else
        k_render<32><<<grid, 256, 0, s>>>(height, width, bin_view(L.bins), params, L.centres, L.radius, L.rmax, model,
                                          L.overflow);
    return check_launch("k_render");
}

int spx_clean_cells(const void* img, int dtype, double sign, int height, int width, const int* voronoi,
                    const int* boxes, const double* params, int radius_cap, const spx_bgmap* background,
                    const double* model, const int* which, int n_out, int hm, int wm, double* out, void* stream) {
    SPX_REQUIRE(n_out >= 0 && hm >= 0 && wm >= 0, "bad arguments");
    if (n_out == 0 || hm == 0 || wm == 0) return SPX_OK;
    SPX_REQUIRE(img && voronoi && boxes && params && background && model && out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long total = (long long)n_out * hm * wm;
    k_clean_stack<<<grid_for(total, 256), 256, 0, s>>>(Image{img, dtype, sign, height, width}, voronoi,
                                                       reinterpret_cast<const int4*>(boxes), params, radius_cap,
                                                       *background, model, which, n_out, hm, wm, out);
    return check_launch("k_clean_stack");
}

int spx_clean_masked(const void* img, int dtype, double sign, int height, int width, const uint8_t* masks,
                     const int* origins, const double* params_global, int radius_cap, const spx_bgmap* background,
                     const double* model, int n, int hm, int wm, double* out, void* stream) {
    SPX_REQUIRE(n >= 0 && hm >= 0 && wm >= 0 && height > 0 && width > 0, "bad arguments");
    if (n == 0 || hm == 0 || wm == 0) return SPX_OK;
    SPX_REQUIRE(img && masks && origins && params_global && background && model && out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long total = (long long)n * hm * wm;
    k_clean_masked<<<grid_for(total, 256), 256, 0, s>>>(Image{img, dtype, sign, height, width}, masks, origins,
                                                        params_global, radius_cap, *background, model, n, hm, wm,
                                                        out);
    return check_launch("k_clean_masked");
}

int spx_support_labels(const double* cleaned, const int* voronoi, const int* boxes, const double* params, int n,
                       int hm, int wm, int width, int* labels, int* rows_out, void* stream) {
    SPX_REQUIRE(n >= 0 && hm >= 0 && wm >= 0 && width > 0, "bad arguments");
    if (n == 0 || hm == 0 || wm == 0) return SPX_OK;
    SPX_REQUIRE(cleaned && voronoi && boxes && params && labels && rows_out, "null pointer");
    SPX_REQUIRE((long long)n * hm < (1LL << 31), "cell stack too tall");
    k_support_labels<<<grid_for(n, 8, 148 * 16), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        cleaned, voronoi, reinterpret_cast<const int4*>(boxes), params, n, hm, wm, width, labels, rows_out);
    return check_launch("k_support_labels");
}

int spx_tile_medians(const void* img, int dtype, double sign, int height, int width, const double* model,
                     const unsigned int* dist2, const uint8_t* usable, int mode, double thr_model, double thr_dist,
                     int tile, double* medians, long long* counts, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && tile >= 1, "bad arguments");
    SPX_REQUIRE(mode == SPX_TILE_FREE || mode == SPX_TILE_USABLE || mode == SPX_TILE_ALL, "bad mode");
    SPX_REQUIRE(img && medians && counts && (mode != SPX_TILE_FREE || dist2), "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int ny = (height + tile - 1) / tile, nx = (width + tile - 1) / tile;
    const long long t2 = (long long)tile * tile;
    const int smem_keys = (int)(t2 < kTileSmemKeys ? t2 : kTileSmemKeys);
    const size_t smem = (size_t)smem_keys * sizeof(unsigned long long);
    auto kernel = dtype == SPX_U8 ? k_tile_median<uint8_t>
                  : dtype == SPX_U16 ? k_tile_median<uint16_t>
                  : dtype == SPX_F32 ? k_tile_median<float> : k_tile_median<double>;
    SPX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // Smallest integer squared distance whose square root reaches thr_dist (sqrt is correctly
    // rounded here and on the device, and monotonic), so the kernel compares integers.
    unsigned long long d2_min = 0;
    if (thr_dist != thr_dist) {
        d2_min = 1ull << 33;  // NaN: no distance passes
    } else if (thr_dist > 0.0) {
        const double t2 = ceil(thr_dist * thr_dist);
        unsigned long long d = t2 > 8.0e9 ? (1ull << 33) : (unsigned long long)t2;
        while (d > 0 && sqrt((double)(d - 1)) >= thr_dist) --d;
        while (d < (1ull << 33) && !(sqrt((double)d) >= thr_dist)) ++d;
        d2_min = d;
    }
    TileSel sel{Image{img, dtype, sign, height, width}, model, dist2, usable, mode, thr_model, d2_min};
    kernel<<<ny * nx, kTileThreads, smem, s>>>(sel, tile, nx, smem_keys, medians, counts);
    return check_launch("k_tile_median");
}

int spx_background_rows(const double* medians, int ny, int nx, int tile, int width, double* rows, void* stream) {
    SPX_REQUIRE(ny >= 1 && nx >= 1 && tile >= 1 && width > 0, "bad arguments");
    SPX_REQUIRE(medians && rows, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long total = (long long)ny * width;
    k_bg_rows<<<grid_for(total, 256), 256, 0, s>>>(medians, ny, nx, tile, width, rows);
    return check_launch("k_bg_rows");
}

int spx_quantiles(const void* requests, int n_requests, double* out, void* stream) {
    SPX_REQUIRE(n_requests >= 1 && n_requests <= 64, "between 1 and 64 requests");
    SPX_REQUIRE(requests && out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_quantiles<<<n_requests, kQuantThreads, 0, s>>>(static_cast<const QuantileReq*>(requests), out);
    return check_launch("k_quantiles");
}

int spx_cell_stats(const double* params, const uint8_t* status, int n, double* fwhm, uint8_t* good, void* stream) {
    SPX_REQUIRE(n >= 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(params && status && fwhm && good, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_cell_stats<<<grid_for(n, 256), 256, 0, s>>>(params, status, n, fwhm, good);
    return check_launch("k_cell_stats");
}

int spx_background_at(const spx_bgmap* background, int height, int width, const double* points, int n,
                      double sign, double* out, void* stream) {
    SPX_REQUIRE(n >= 0 && height > 0 && width > 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(background && points && out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_background_at<<<grid_for(n, 256), 256, 0, s>>>(*background, height, width, points, n, sign, out);
    return check_launch("k_background_at");
}

int spx_residual(const void* img, int dtype, double sign, int height, int width, const spx_bgmap* background,
                 const double* model, double* out, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0, "bad arguments");
    SPX_REQUIRE(img && background && model && out, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_residual<<<grid_for((long long)height * width, 256), 256, 0, s>>>(Image{img, dtype, sign, height, width},
                                                                        *background, model, out);
    return check_launch("k_residual");
}

}  // extern "C"
