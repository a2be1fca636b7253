// Windows of the tail CD family (subpx/_cpu/invariant_cd.py:878-964, _wide_cells): each reported
// hole on a square window of (2 radius + 1) pixels around its rounded fitted centre, holding its own
// share of the light -- (image - background map) x own model / (model image + floor) -- with three
// byte masks: inside the image, the hole's own territory (closer to it than to its 8 nearest modelled
// holes) and the level pixels (the farthest tenth, at least 4, of the territory).
//
// The 8 nearest holes come from a grid of buckets (one counting sort of the fitted centres) searched
// ring by ring until no unvisited bucket can hold a nearer hole; ties in distance go to the lower
// index. One CTA builds one window: pixel values and distances in parallel, the level cut by the CTA
// radix select over the territory's distances.

#include "image.cuh"
#include "lm.cuh"
#include "scan.cuh"
#include "select.cuh"

namespace spx {
namespace {

constexpr int kWideThreads = 256;
constexpr int kWideMaxSide = 64;  // window side limit (its distances stay in shared memory)
constexpr int kKnn = 8;           // neighbours besides the hole itself

// Global fitted centre of hole j: params (ROI-local) plus the box origin, or the box centre when the
// centre is not finite.
__global__ void k_wide_centers(const double* params, const int4* boxes, int n, int hm, int wm, double* centers) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int4 b = boxes[j];
        const double px = params[6LL * j + 1], py = params[6LL * j + 2];
        const double fx = __dadd_rn((double)b.x, (double)(wm - 1) / 2.0);
        const double fy = __dadd_rn((double)b.y, (double)(hm - 1) / 2.0);
        const double cx = __dadd_rn(px, (double)b.x), cy = __dadd_rn(py, (double)b.y);
        centers[2LL * j] = isfinite(cx) ? cx : fx;
        centers[2LL * j + 1] = isfinite(cy) ? cy : fy;
    }
}

__device__ __forceinline__ int grid_cell(double v, double inv_g, int n) {
    const double c = floor(v * inv_g);
    return c < 0.0 ? 0 : (c >= (double)n ? n - 1 : (int)c);
}

__global__ void k_grid_count(const double* centers, int n, double inv_g, int gx, int gy, int* cell_of, int* counts) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int c = grid_cell(centers[2LL * j + 1], inv_g, gy) * gx + grid_cell(centers[2LL * j], inv_g, gx);
        cell_of[j] = c;
        atomicAdd(&counts[c], 1);
    }
}

__global__ void k_grid_fill(int n, const int* cell_of, const int* offsets, int* cursor, int* items) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int c = cell_of[j];
        items[offsets[c] + atomicAdd(&cursor[c], 1)] = j;
    }
}

// Row `i` of `neighbours`: the reported hole itself, then its k nearest other holes by distance (ties:
// lower index first); -1 where there are fewer. After rings 0..r of buckets around the hole's bucket,
// every unvisited hole is at least r bucket sides away, so the search stops once the k-th distance is
// below that.
__global__ void k_knn(const double* centers, const int* rows, int n_rep, int k, double g, double inv_g, int gx,
                      int gy, const int* offsets, const int* counts, const int* items, int* neighbours) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_rep; i += gridDim.x * blockDim.x) {
        const int self = rows[i];
        const double qx = centers[2LL * self], qy = centers[2LL * self + 1];
        const int cx = grid_cell(qx, inv_g, gx), cy = grid_cell(qy, inv_g, gy);
        double bd[kKnn];
        int bi[kKnn];
        int have = 0;
        const int rmax = k > 0 ? max(gx, gy) : -1;
        for (int r = 0; r <= rmax; ++r) {
            for (int yy = cy - r; yy <= cy + r; ++yy) {
                if (yy < 0 || yy >= gy) continue;
                const bool edge_row = yy == cy - r || yy == cy + r;
                for (int xx = cx - r; xx <= cx + r; xx += edge_row ? 1 : 2 * r) {
                    if (xx >= 0 && xx < gx) {
                        const int c = yy * gx + xx;
                        for (int q = offsets[c], e = offsets[c] + counts[c]; q < e; ++q) {
                            const int j = items[q];
                            if (j == self) continue;
                            const double dx = __dsub_rn(centers[2LL * j], qx), dy = __dsub_rn(centers[2LL * j + 1], qy);
                            const double d = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                            if (have == k && !(d < bd[k - 1] || (d == bd[k - 1] && j < bi[k - 1]))) continue;
                            int p = have < k ? have++ : k - 1;
                            while (p > 0 && (d < bd[p - 1] || (d == bd[p - 1] && j < bi[p - 1]))) {
                                bd[p] = bd[p - 1];
                                bi[p] = bi[p - 1];
                                --p;
                            }
                            bd[p] = d;
                            bi[p] = j;
                        }
                    }
                    if (r == 0) break;
                }
            }
            const double reach = (double)r * g;
            if (have == k && bd[k - 1] < reach * reach) break;
        }
        int* out = neighbours + (long long)i * (kKnn + 1);
        out[0] = self;
        for (int q = 0; q < kKnn; ++q) out[q + 1] = q < have ? bi[q] : -1;
    }
}

// Render radius of a hole's model, the deblend's rule (subpx/_cpu/deblend.py:83-84): ceil(4 sigma_major)
// clipped to [2, cap].
__device__ __forceinline__ int render_radius_of(const double* p, int cap) {
    double r = ceil(4.0 * sigma_major(p));
    if (!(r >= 2.0)) r = 2.0;
    if (r > (double)cap) r = (double)cap;
    return (int)r;
}

struct WideArgs {
    Image img;
    spx_bgmap bg;
    const double* model;    // (H, W) model image
    const double* params;   // (n_all, 6) ROI-local
    const int4* boxes;      // (n_all) cell boxes (origin x, y)
    const double* centers;  // (n_all, 2) global fitted centres (k_wide_centers)
    const int* rows;        // (n) reported holes
    const int* neighbours;  // (n, 9)
    int n, radius, side, cap;
    double floor;
    float* cells;           // (n, side, side)
    uint8_t* inside;        // (n, side, side)
    uint8_t* level;
    uint8_t* territory;
    int* origins;           // (n, 2) window origins x, y
};

__global__ void __launch_bounds__(kWideThreads) k_wide_cells(WideArgs a) {
    __shared__ double dist0[kWideMaxSide * kWideMaxSide];  // distance to the hole, -inf off its territory
    __shared__ double nbr[2 * (kKnn + 1)];
    __shared__ int hist[2048];
    __shared__ int warp_tot[32], s_pick[3], s_count;
    __shared__ unsigned long long s_keys[2], s_kmin, s_kmax;
    const int tid = threadIdx.x, lane = tid & 31;
    const int S = a.side, area = S * S;
    for (int i = blockIdx.x; i < a.n; i += gridDim.x) {
        const int self = a.rows[i];
        __syncthreads();  // the previous window's shared reads are done
        if (tid < kKnn + 1) {
            const int j = a.neighbours[(long long)i * (kKnn + 1) + tid];
            nbr[2 * tid] = j >= 0 ? a.centers[2LL * j] : INFINITY;
            nbr[2 * tid + 1] = j >= 0 ? a.centers[2LL * j + 1] : INFINITY;
        }
        if (tid == 0) {
            s_count = 0;
            s_kmin = ~0ull;
            s_kmax = 0ull;
        }
        // Window origin: rint of the fitted centre (round half to even) minus the radius.
        const double ccx = a.centers[2LL * self], ccy = a.centers[2LL * self + 1];
        const int ox = (int)rint(ccx) - a.radius, oy = (int)rint(ccy) - a.radius;
        if (tid == 0) {
            a.origins[2LL * i] = ox;
            a.origins[2LL * i + 1] = oy;
        }
        // The hole's own model: its global parameters (zero where not all finite) within the render box.
        const int4 box = a.boxes[self];
        double p[6];
        bool good = true;
        for (int q = 0; q < 6; ++q) {
            p[q] = a.params[6LL * self + q];
            good = good && isfinite(p[q]);
        }
        double pr[6];
        for (int q = 0; q < 6; ++q) pr[q] = isfinite(p[q]) ? p[q] : 0.0;
        const double render = good ? (double)render_radius_of(pr, a.cap) : 0.0;
        const double gx0 = good ? __dadd_rn(p[1], (double)box.x) : 0.0, gy0 = good ? __dadd_rn(p[2], (double)box.y) : 0.0;
        const double amp = good ? p[0] : 0.0, e1 = exp(good ? p[3] : 0.0), u2 = good ? p[4] : 0.0;
        const double e3 = exp(good ? p[5] : 0.0);
        __syncthreads();
        int cnt = 0;
        unsigned long long kmin = ~0ull, kmax = 0ull;
        for (int t = tid; t < area; t += kWideThreads) {
            const int y = oy + t / S, x = ox + t % S;
            const bool in = y >= 0 && y < a.img.H && x >= 0 && x < a.img.W;
            const int yc = min(max(y, 0), a.img.H - 1), xc = min(max(x, 0), a.img.W - 1);
            const double gx = (double)x, gy = (double)y;
            const double dx = __dsub_rn(gx, gx0), dy = __dsub_rn(gy, gy0);
            double own = 0.0;
            if (good && fabs(dx) <= render && fabs(dy) <= render) {
                const double aa = __dadd_rn(__dmul_rn(e1, dx), __dmul_rn(u2, dy)), bb = __dmul_rn(e3, dy);
                own = __dmul_rn(amp, exp(__dmul_rn(-0.5, __dadd_rn(__dmul_rn(aa, aa), __dmul_rn(bb, bb)))));
            }
            // Distances to the hole and its neighbours; the territory is where the hole is nearest.
            double d[kKnn + 1];
#pragma unroll
            for (int q = 0; q <= kKnn; ++q) {
                const double ex = __dsub_rn(gx, nbr[2 * q]), ey = __dsub_rn(gy, nbr[2 * q + 1]);
                d[q] = sqrt(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)));
            }
            double nearest = INFINITY;
#pragma unroll
            for (int q = 1; q <= kKnn; ++q) nearest = fmin(nearest, d[q]);
            const bool mine = d[0] <= nearest;
            const bool terr = in && mine;
            const double win = __dsub_rn(a.img.at(yc, xc), bg_at(a.bg, yc, xc));
            const double total = a.model[(long long)yc * a.img.W + xc];
            const double v = in ? __ddiv_rn(__dmul_rn(win, own), __dadd_rn(total, a.floor)) : 0.0;
            const long long o = (long long)i * area + t;
            a.cells[o] = (float)v;
            a.inside[o] = in;
            a.territory[o] = terr;
            const double key_v = terr ? d[0] : -INFINITY;
            dist0[t] = key_v;
            cnt += terr;
            const unsigned long long key = order_key(key_v);
            kmin = min(kmin, key);
            kmax = max(kmax, key);
        }
        cnt = warp_sum_i(cnt);
        kmin = warp_min_u64(kmin);
        kmax = warp_max_u64(kmax);
        if (lane == 0) {
            atomicAdd(&s_count, cnt);
            atomicMin(&s_kmin, kmin);
            atomicMax(&s_kmax, kmax);
        }
        __syncthreads();
        // Level pixels: territory distances at or above the keep-th largest (descending, -inf outside
        // the territory), keep = clip(max(count // 10, 4), 1, area) - 1.
        const int count = s_count;
        const int keep = min(max(max(count / 10, 4), 1), area) - 1;
        auto for_keys = [&](auto&& fn) {
            for (int t = tid; t < area; t += kWideThreads) fn(order_key(dist0[t]));
        };
        unsigned long long kth, kth2;
        cta_select<kWideThreads>(for_keys, area - 1 - keep, false, s_kmin, s_kmax, hist, warp_tot, s_pick, s_keys,
                                 &kth, &kth2);
        const double cut = key_value(kth);
        for (int t = tid; t < area; t += kWideThreads) {
            const long long o = (long long)i * area + t;
            a.level[o] = a.territory[o] && dist0[t] >= cut;
        }
    }
}

// Workspace pieces of spx_wide_cells: centres, bucket counts / offsets / cursors, the sorted holes,
// the scan's scratch and the neighbour table. Sized with a null base, then carved from the real one.
struct WideWorkspace {
    double* centers;
    int *counts, *offsets, *cursor, *cell_of, *items, *total, *scratch, *neighbours;
    size_t bytes;
    WideWorkspace(void* base, int n_all, int n_rep, long long n_cells) {
        Arena ar(base);
        centers = ar.take<double>(2LL * std::max(n_all, 1));
        counts = ar.take<int>(n_cells);
        offsets = ar.take<int>(n_cells);
        cursor = ar.take<int>(n_cells);
        cell_of = ar.take<int>(std::max(n_all, 1));
        items = ar.take<int>(std::max(n_all, 1));
        total = ar.take<int>(1);
        scratch = ar.take<int>(scan_scratch_ints(n_cells));
        neighbours = ar.take<int>((long long)std::max(n_rep, 1) * (kKnn + 1));
        bytes = ar.used + 256;
    }
};

void grid_dims(int height, int width, double bucket, int* gx, int* gy) {
    *gx = (int)std::min<double>(std::max(1.0, ceil(width / bucket)), 1 << 20);
    *gy = (int)std::min<double>(std::max(1.0, ceil(height / bucket)), 1 << 20);
}

}  // namespace

extern "C" {

size_t spx_wide_cells_workspace_bytes(int n_all, int n_rep, int height, int width, double bucket) {
    if (!(bucket > 0.0) || n_all < 0 || n_rep < 0 || height < 1 || width < 1) return 0;
    int gx, gy;
    grid_dims(height, width, bucket, &gx, &gy);
    return WideWorkspace(nullptr, n_all, n_rep, (long long)gx * gy).bytes;
}

int spx_wide_cells(const void* img, int dtype, double sign, int height, int width, const spx_bgmap* background,
                   const double* model, const double* params, const int* boxes, int n_all, int hm, int wm,
                   const int* rows, int n_rep, int radius, double bucket, double floor, float* cells, uint8_t* inside,
                   uint8_t* level, uint8_t* territory, int* origins, int* neighbours_out, void* workspace,
                   size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n_all >= 0 && n_rep >= 0 && height >= 1 && width >= 1 && radius >= 0 && hm >= 1 && wm >= 1,
                "bad arguments");
    SPX_REQUIRE(bucket > 0.0 && isfinite(bucket), "bucket must be positive");
    SPX_REQUIRE(2 * radius + 1 <= kWideMaxSide, "tail window wider than 64 pixels");
    if (n_rep == 0) return SPX_OK;
    SPX_REQUIRE(n_all >= 1, "reported holes without modelled holes");
    SPX_REQUIRE(img && background && model && params && boxes && rows && cells && inside && level && territory &&
                    origins && workspace,
                "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_wide_cells_workspace_bytes(n_all, n_rep, height, width, bucket),
                "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int gx, gy;
    grid_dims(height, width, bucket, &gx, &gy);
    const long long n_cells = (long long)gx * gy;
    WideWorkspace w(workspace, n_all, n_rep, n_cells);
    int* neighbours = neighbours_out ? neighbours_out : w.neighbours;
    const int4* b4 = reinterpret_cast<const int4*>(boxes);
    SPX_CUDA(cudaMemsetAsync(w.counts, 0, sizeof(int) * n_cells, s));
    SPX_CUDA(cudaMemsetAsync(w.cursor, 0, sizeof(int) * n_cells, s));
    k_wide_centers<<<grid_for(n_all, 256), 256, 0, s>>>(params, b4, n_all, hm, wm, w.centers);
    k_grid_count<<<grid_for(n_all, 256), 256, 0, s>>>(w.centers, n_all, 1.0 / bucket, gx, gy, w.cell_of, w.counts);
    if (int e = exclusive_scan(w.counts, n_cells, w.offsets, w.total, w.scratch, s)) return e;
    k_grid_fill<<<grid_for(n_all, 256), 256, 0, s>>>(n_all, w.cell_of, w.offsets, w.cursor, w.items);
    const int k = std::min(kKnn, n_all - 1);
    k_knn<<<grid_for(n_rep, 128), 128, 0, s>>>(w.centers, rows, n_rep, k, bucket, 1.0 / bucket, gx, gy, w.offsets,
                                               w.counts, w.items, neighbours);
    WideArgs a{Image{img, dtype, sign, height, width}, *background, model, params, b4, w.centers, rows, neighbours,
               n_rep, radius, 2 * radius + 1, std::max(hm, wm), floor, cells, inside, level, territory, origins};
    k_wide_cells<<<std::min(n_rep, 148 * 8), kWideThreads, 0, s>>>(a);
    return check_launch("k_wide_cells");
}

}  // extern "C"

}  // namespace spx
