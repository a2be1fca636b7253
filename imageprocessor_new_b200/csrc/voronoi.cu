// Voronoi partition: label of the nearest seed for every pixel.
//
// Reference: subpx/_cpu/cells.py:8-33 (cKDTree k=2 query, exact ties resolved by the lowest seed
// index on recomputed squared distances) and subpx/_gpu/voronoi.py (same rule). The rule is
// argmin over seeds of (d2, index) with d2 = (px-sx)*(px-sx) + (py-sy)*(py-sy) rounded without FMA.
//
// B200 layout: seeds are counting-sorted into a grid of square bins (about one seed per bin). One
// CTA labels a 16x16 pixel tile: warp 0 bounds the distance from the tile centre to its nearest
// seed, which bounds the search square every pixel of the tile needs; the seeds of that square
// (contiguous runs of the bin-sorted array, one run per bin row) are staged through shared memory
// in chunks and each thread keeps its own (d2, index) minimum. Writes are 4 B/px, coalesced.

#include "common.cuh"
#include "scan.cuh"

namespace spx {
namespace {

constexpr int kTile = 16;
constexpr int kThreads = kTile * kTile;

struct Grid {
    int gw, gh;
    double cell;
};

__device__ __forceinline__ int bin_of(double v, double cell, int n) {
    long long b = (long long)floor(v / cell);
    if (b < 0) b = 0;
    if (b > n - 1) b = n - 1;
    return (int)b;
}

__global__ void k_bin_count(const double* seeds, int n, Grid g, int* counts) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int bx = bin_of(seeds[2 * i], g.cell, g.gw), by = bin_of(seeds[2 * i + 1], g.cell, g.gh);
        atomicAdd(&counts[by * g.gw + bx], 1);
    }
}

// Scatter seeds into bin order; within a bin the order is arbitrary (ties compare indices).
__global__ void k_bin_fill(const double* seeds, int n, Grid g, const int* start, int* fill,
                           double2* sorted_xy, int* sorted_id) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int bx = bin_of(seeds[2 * i], g.cell, g.gw), by = bin_of(seeds[2 * i + 1], g.cell, g.gh);
        const int b = by * g.gw + bx;
        const int slot = start[b] + atomicAdd(&fill[b], 1);
        sorted_xy[slot] = make_double2(seeds[2 * i], seeds[2 * i + 1]);
        sorted_id[slot] = i;
    }
}

__device__ __forceinline__ double dist2(double px, double py, double sx, double sy) {
    const double dx = __dsub_rn(px, sx), dy = __dsub_rn(py, sy);
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

__global__ void __launch_bounds__(kThreads) k_voronoi(int H, int W, Grid g, const int* start,
                                                       const double2* sxy, const int* sid, int n,
                                                       int* labels) {
    __shared__ double2 c_xy[kThreads];
    __shared__ int c_id[kThreads];
    __shared__ double s_bound;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
    const int lane = threadIdx.x & 31;
    // Tile centre, clipped to the image part of the tile.
    const double cx = 0.5 * (tx0 + min(tx0 + kTile, W) - 1), cy = 0.5 * (ty0 + min(ty0 + kTile, H) - 1);
    const double half_diag = 0.5 * sqrt((double)(min(kTile, W - tx0) - 1) * (min(kTile, W - tx0) - 1) +
                                        (double)(min(kTile, H - ty0) - 1) * (min(kTile, H - ty0) - 1));
    if (threadIdx.x < 32) {
        // Nearest-seed distance bound of the centre: rings of bins until one holds a seed, plus
        // one more ring.
        const int bx = bin_of(cx, g.cell, g.gw), by = bin_of(cy, g.cell, g.gh);
        double best = dinf();
        int found_ring = -1;
        const int max_ring = max(g.gw, g.gh);
        for (int R = 0; R <= max_ring; ++R) {
            const int side = 2 * R + 1;
            const int count = R == 0 ? 1 : 4 * (side - 1);
            for (int k = lane; k < count; k += 32) {
                int gx, gy;
                if (R == 0) { gx = bx; gy = by; }
                else if (k < side) { gx = bx - R + k; gy = by - R; }
                else if (k < 2 * side) { gx = bx - R + (k - side); gy = by + R; }
                else if (k < 2 * side + (side - 2)) { gx = bx - R; gy = by - R + 1 + (k - 2 * side); }
                else { gx = bx + R; gy = by - R + 1 + (k - 2 * side - (side - 2)); }
                if (gx < 0 || gy < 0 || gx >= g.gw || gy >= g.gh) continue;
                const int b = gy * g.gw + gx;
                for (int j = start[b]; j < start[b + 1]; ++j) {
                    const double2 s = sxy[j];
                    best = fmin(best, dist2(cx, cy, s.x, s.y));
                }
            }
            best = warp_min(best);
            if (best < dinf() && found_ring < 0) found_ring = R;
            if (found_ring >= 0 && R >= found_ring + 1) break;
        }
        if (lane == 0) s_bound = sqrt(best) + 2.0 * half_diag + 1.0;
    }
    __syncthreads();
    const double R = s_bound;
    const int gx0 = bin_of(cx - R, g.cell, g.gw), gx1 = bin_of(cx + R, g.cell, g.gw);
    const int gy0 = bin_of(cy - R, g.cell, g.gh), gy1 = bin_of(cy + R, g.cell, g.gh);
    const int x = tx0 + (threadIdx.x % kTile), y = ty0 + (threadIdx.x / kTile);
    const double px = (double)x, py = (double)y;
    double best = dinf();
    int label = 0x7fffffff;
    for (int gy = gy0; gy <= gy1; ++gy) {
        const int j0 = start[gy * g.gw + gx0], j1 = start[gy * g.gw + gx1 + 1];
        for (int base = j0; base < j1; base += kThreads) {
            const int m = min(kThreads, j1 - base);
            __syncthreads();
            if ((int)threadIdx.x < m) {
                c_xy[threadIdx.x] = sxy[base + threadIdx.x];
                c_id[threadIdx.x] = sid[base + threadIdx.x];
            }
            __syncthreads();
            for (int k = 0; k < m; ++k) {
                const double2 s = c_xy[k];
                const double d2 = dist2(px, py, s.x, s.y);
                const int id = c_id[k];
                if (d2 < best || (d2 == best && id < label)) { best = d2; label = id; }
            }
        }
    }
    if (x < W && y < H) labels[(long long)y * W + x] = label;
}

__global__ void k_fill(int* labels, long long n, int v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        labels[i] = v;
}

Grid make_grid(int n, int H, int W) {
    Grid g;
    double cell = floor(sqrt((double)H * (double)W / (double)(n > 0 ? n : 1)));
    if (cell < 1.0) cell = 1.0;
    g.cell = cell;
    g.gw = (int)ceil(W / cell);
    g.gh = (int)ceil(H / cell);
    if (g.gw < 1) g.gw = 1;
    if (g.gh < 1) g.gh = 1;
    return g;
}

struct VorLayout {
    int* counts;
    int* start;
    int* fill;
    double2* sorted_xy;
    int* sorted_id;
    int* scratch;
};

VorLayout vor_layout(void* ws, int n, int H, int W, size_t* bytes) {
    const Grid g = make_grid(n, H, W);
    const long long bins = (long long)g.gw * g.gh;
    Arena a(ws);
    VorLayout L;
    L.counts = a.take<int>(bins + 1);
    L.start = a.take<int>(bins + 1);
    L.fill = a.take<int>(bins + 1);
    L.sorted_xy = a.take<double2>(n > 0 ? n : 1);
    L.sorted_id = a.take<int>(n > 0 ? n : 1);
    L.scratch = a.take<int>(scan_scratch_ints(bins + 1));
    if (bytes) *bytes = a.used;
    return L;
}

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

size_t spx_voronoi_workspace_bytes(int n, int height, int width) {
    size_t b = 0;
    vor_layout(nullptr, n, height, width, &b);
    return b;
}

int spx_voronoi_labels(const double* seeds, int n, int height, int width, int* labels,
                       void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && n >= 0, "bad arguments");
    SPX_REQUIRE(labels, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long hw = (long long)height * width;
    if (n <= 1) {
        k_fill<<<grid_for(hw, 256), 256, 0, s>>>(labels, hw, n == 0 ? -1 : 0);
        return check_launch("k_fill");
    }
    SPX_REQUIRE(seeds && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_voronoi_workspace_bytes(n, height, width), "workspace too small");
    const Grid g = make_grid(n, height, width);
    const long long bins = (long long)g.gw * g.gh;
    VorLayout L = vor_layout(workspace, n, height, width, nullptr);
    SPX_CUDA(cudaMemsetAsync(L.counts, 0, (bins + 1) * sizeof(int), s));
    SPX_CUDA(cudaMemsetAsync(L.fill, 0, (bins + 1) * sizeof(int), s));
    k_bin_count<<<grid_for(n, 256), 256, 0, s>>>(seeds, n, g, L.counts);
    if (int e = check_launch("k_bin_count")) return e;
    // start[b] = seeds in bins before b; start[bins] = n (the extra zero count).
    if (int e = exclusive_scan(L.counts, bins + 1, L.start, nullptr, L.scratch, s)) return e;
    k_bin_fill<<<grid_for(n, 256), 256, 0, s>>>(seeds, n, g, L.start, L.fill, L.sorted_xy, L.sorted_id);
    if (int e = check_launch("k_bin_fill")) return e;
    const dim3 grid((width + kTile - 1) / kTile, (height + kTile - 1) / kTile);
    k_voronoi<<<grid, kThreads, 0, s>>>(height, width, g, L.start, L.sorted_xy, L.sorted_id, n, labels);
    return check_launch("k_voronoi");
}

}  // extern "C"
