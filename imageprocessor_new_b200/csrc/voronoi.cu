// Voronoi partition, distance-to-nearest-seed-pixel map and nearest-point queries.
//
// Reference: subpx/_cpu/cells.py:8-33 (cKDTree k=2 query, exact ties resolved by the lowest seed
// index on recomputed squared distances) and subpx/_gpu/voronoi.py (same rule). The rule is
// argmin over seeds of (d2, index) with d2 = (px-sx)*(px-sx) + (py-sy)*(py-sy) rounded without FMA.
// The distance map replaces scipy.ndimage.distance_transform_edt of the seed-pixel mask
// (subpx/_cpu/deblend.py:452-457): squared distance to the nearest rint()-ed seed pixel.
//
// B200 layout: seeds are counting-sorted into a grid of square bins (about one seed per bin). One
// CTA labels a 16x16 pixel tile: warp 0 bounds the distance from the tile centre to its nearest
// seed, which bounds the search square every pixel of the tile needs; the seeds of that square
// (contiguous runs of the bin-sorted array, one run per bin row) are staged through shared memory
// in chunks and each thread keeps its own (d2, index) minimum. Writes are 4 B/px, coalesced.

#include "bins.cuh"

namespace spx {

__global__ void k_bin_count(const double* pts, int stride, const int* origin, const uint8_t* valid,
                            long long n, int gw, int gh, double cell, int* counts) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (valid && !valid[i]) continue;
        double x = pts[i * stride], y = pts[i * stride + 1];
        if (origin) { x += origin[2 * i]; y += origin[2 * i + 1]; }
        atomicAdd(&counts[bin_index(y, cell, gh) * gw + bin_index(x, cell, gw)], 1);
    }
}

__global__ void k_bin_fill(const double* pts, int stride, const int* origin, const uint8_t* valid,
                           long long n, int gw, int gh, double cell, const int* start, int* fill,
                           double2* xy, int* id) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (valid && !valid[i]) continue;
        double x = pts[i * stride], y = pts[i * stride + 1];
        if (origin) { x += origin[2 * i]; y += origin[2 * i + 1]; }
        const int b = bin_index(y, cell, gh) * gw + bin_index(x, cell, gw);
        const int slot = start[b] + atomicAdd(&fill[b], 1);
        xy[slot] = make_double2(x, y);
        id[slot] = (int)i;
    }
}

int bin_build(BinStorage& b, const double* pts, int stride, const int* origin, const uint8_t* valid,
              long long n, cudaStream_t s) {
    const long long bins = (long long)b.gw * b.gh;
    SPX_CUDA(cudaMemsetAsync(b.counts, 0, (bins + 1) * sizeof(int), s));
    SPX_CUDA(cudaMemsetAsync(b.fill, 0, (bins + 1) * sizeof(int), s));
    if (n > 0) {
        k_bin_count<<<grid_for(n, 256), 256, 0, s>>>(pts, stride, origin, valid, n, b.gw, b.gh, b.cell, b.counts);
        if (int e = check_launch("k_bin_count")) return e;
    }
    if (int e = exclusive_scan(b.counts, bins + 1, b.start, nullptr, b.scratch, s)) return e;
    if (n > 0) {
        k_bin_fill<<<grid_for(n, 256), 256, 0, s>>>(pts, stride, origin, valid, n, b.gw, b.gh, b.cell, b.start,
                                                    b.fill, b.xy, b.id);
        if (int e = check_launch("k_bin_fill")) return e;
    }
    return SPX_OK;
}

namespace {

constexpr int kTile = 16;
constexpr int kThreads = kTile * kTile;
constexpr int kRowsMax = 64;  // bin rows of a search square that the one-pass candidate staging takes

__device__ __forceinline__ double dist2(double px, double py, double sx, double sy) {
    const double dx = __dsub_rn(px, sx), dy = __dsub_rn(py, sy);
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

// Smallest squared distance from (cx, cy) to any point, by rings of bins until one holds a point,
// plus one more ring (called by one full warp; the result is the same on every lane).
__device__ double warp_nearest_bound(const BinGrid& g, double cx, double cy, int lane) {
    const int bx = bin_index(cx, g.cell, g.gw), by = bin_index(cy, g.cell, g.gh);
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
            for (int j = g.start[b]; j < g.start[b + 1]; ++j) {
                const double2 s = g.xy[j];
                best = fmin(best, dist2(cx, cy, s.x, s.y));
            }
        }
        best = warp_min(best);
        if (best < dinf() && found_ring < 0) found_ring = R;
        if (found_ring >= 0 && R >= found_ring + 1) break;
    }
    return best;
}

// labels != null: nearest-seed index; d2 != null: squared distance to the nearest seed.
// The tile at (tx0, ty0): its centre and the half of its diagonal (pixel centres).
__device__ __forceinline__ void tile_geometry(int H, int W, int tx0, int ty0, double* cx, double* cy,
                                              double* half_diag) {
    const int ex = min(kTile, W - tx0), ey = min(kTile, H - ty0);
    *cx = 0.5 * (tx0 + tx0 + ex - 1);
    *cy = 0.5 * (ty0 + ty0 + ey - 1);
    *half_diag = 0.5 * sqrt((double)(ex - 1) * (ex - 1) + (double)(ey - 1) * (ey - 1));
}

// Per 16 x 16 tile, the radius around its centre that holds every seed that can be the nearest of
// one of its pixels: the centre's nearest-seed distance plus the tile's diagonal, plus 1 px of
// slack for rounding (infinite without seeds). One warp per tile, so that the ring searches'
// dependent loads of many tiles overlap.
__global__ void k_tile_bounds(int H, int W, BinGrid g, int tiles_x, int tiles, double* bound) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int t = blockIdx.x * warps + (threadIdx.x >> 5); t < tiles; t += gridDim.x * warps) {
        double cx, cy, half_diag;
        tile_geometry(H, W, (t % tiles_x) * kTile, (t / tiles_x) * kTile, &cx, &cy, &half_diag);
        const double best = warp_nearest_bound(g, cx, cy, lane);
        if (lane == 0) bound[t] = sqrt(best) + 2.0 * half_diag + 1.0;
    }
}

__global__ void __launch_bounds__(kThreads) k_voronoi(int H, int W, BinGrid g, const double* bound, int* labels,
                                                       unsigned int* d2out) {
    __shared__ double2 c_xy[kThreads];
    __shared__ int c_id[kThreads];
    __shared__ int row_j0[kRowsMax], row_pre[kRowsMax + 1];
    __shared__ int s_kept;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
    const int lane = threadIdx.x & 31;
    double cx, cy, half_diag;
    tile_geometry(H, W, tx0, ty0, &cx, &cy, &half_diag);
    const double R = bound[blockIdx.y * gridDim.x + blockIdx.x];
    int gx0, gx1, gy0, gy1;
    if (isfinite(R)) {
        gx0 = bin_index(cx - R, g.cell, g.gw);
        gx1 = bin_index(cx + R, g.cell, g.gw);
        gy0 = bin_index(cy - R, g.cell, g.gh);
        gy1 = bin_index(cy + R, g.cell, g.gh);
    } else {
        gx0 = gy0 = 0;
        gx1 = g.gw - 1;
        gy1 = g.gh - 1;
    }
    const int x = tx0 + (threadIdx.x % kTile), y = ty0 + (threadIdx.x / kTile);
    const double px = (double)x, py = (double)y;
    double best = dinf();
    int label = 0x7fffffff;
    auto scan = [&](int m) {
        for (int k = 0; k < m; ++k) {
            const double2 s = c_xy[k];
            const double d2 = dist2(px, py, s.x, s.y);
            const int id = c_id[k];
            if (d2 < best || (d2 == best && id < label)) { best = d2; label = id; }
        }
    };
    // The search square's seeds as runs of the bin-sorted array, one per bin row, with their
    // prefix; warp 0 builds it (lane r takes rows r and r + 32).
    const int n_rows = gy1 - gy0 + 1;
    int total = kThreads + 1;
    if (isfinite(R) && n_rows <= kRowsMax) {
        if (threadIdx.x < 32) {
            int len[2] = {0, 0};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = lane + 32 * h;
                if (r < n_rows) {
                    const int b = (gy0 + r) * g.gw;
                    row_j0[r] = g.start[b + gx0];
                    len[h] = g.start[b + gx1 + 1] - row_j0[r];
                }
            }
            // Inclusive scans of the two halves, the second offset by the first's total.
            int a = len[0], c = len[1];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int ua = __shfl_up_sync(0xffffffffu, a, o), uc = __shfl_up_sync(0xffffffffu, c, o);
                if (lane >= o) { a += ua; c += uc; }
            }
            const int first = __shfl_sync(0xffffffffu, a, 31);
            row_pre[lane + 1] = a;
            row_pre[lane + 33] = first + c;
            if (lane == 0) {
                row_pre[0] = 0;
                s_kept = 0;
            }
        }
        __syncthreads();
        total = row_pre[n_rows];
    }
    if (total <= kThreads) {
        // Seeds farther than R from the tile centre are no pixel's nearest (nor tied): a pixel p of
        // the tile has a seed within |p - c| + sqrt(best) <= half_diag + sqrt(best), and a seed s
        // with |s - c| > sqrt(best) + 2 half_diag is farther from p than that. R keeps 1 px of
        // slack for rounding. The rest are compacted (in no particular order: the (d2, index) rule
        // does not depend on it).
        const int t = threadIdx.x;
        bool keep = false;
        double2 sxy = make_double2(0.0, 0.0);
        int sid = 0;
        if (t < total) {
            int r = 0;
            while (row_pre[r + 1] <= t) ++r;
            const int j = row_j0[r] + (t - row_pre[r]);
            sxy = g.xy[j];
            sid = g.id[j];
            keep = dist2(cx, cy, sxy.x, sxy.y) <= R * R;
        }
        const unsigned vote = __ballot_sync(0xffffffffu, keep);
        int base = 0;
        if (lane == 0 && vote) base = atomicAdd(&s_kept, __popc(vote));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (keep) {
            const int slot = base + __popc(vote & ((1u << lane) - 1u));
            c_xy[slot] = sxy;
            c_id[slot] = sid;
        }
        __syncthreads();
        scan(s_kept);
    } else {
        for (int gy = gy0; gy <= gy1; ++gy) {
            const int j0 = g.start[gy * g.gw + gx0], j1 = g.start[gy * g.gw + gx1 + 1];
            for (int base = j0; base < j1; base += kThreads) {
                const int m = min(kThreads, j1 - base);
                __syncthreads();
                if ((int)threadIdx.x < m) {
                    c_xy[threadIdx.x] = g.xy[base + threadIdx.x];
                    c_id[threadIdx.x] = g.id[base + threadIdx.x];
                }
                __syncthreads();
                scan(m);
            }
        }
    }
    if (x < W && y < H) {
        if (labels) labels[(long long)y * W + x] = label;
        if (d2out) d2out[(long long)y * W + x] = best < 4294967295.0 ? (unsigned int)best : 0xffffffffu;
    }
}

// Nearest point of the grid to each query point (excluding the point with the same index when
// exclude_self): distance (not squared) to out_dist.
__global__ void k_nearest_query(BinGrid g, const double* q, int nq, int exclude_self, double* out_dist) {
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int i = blockIdx.x * warps + (threadIdx.x >> 5); i < nq; i += gridDim.x * warps) {
        const double qx = q[2 * i], qy = q[2 * i + 1];
        const int bx = bin_index(qx, g.cell, g.gw), by = bin_index(qy, g.cell, g.gh);
        double best = dinf();
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
                for (int j = g.start[b]; j < g.start[b + 1]; ++j) {
                    if (exclude_self && g.id[j] == i) continue;
                    const double2 s = g.xy[j];
                    best = fmin(best, dist2(qx, qy, s.x, s.y));
                }
            }
            best = warp_min(best);
            // Points beyond ring R are at least R * cell away (from inside the query's bin); stop
            // once that exceeds the best distance found.
            const double reach = (double)R * g.cell;
            if (best < dinf() && reach * reach > best) break;
        }
        if (lane == 0) out_dist[i] = sqrt(best);
    }
}

__global__ void k_fill(int* labels, long long n, int v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        labels[i] = v;
}

__global__ void k_seed_pixels(const double* seeds, int n, int H, int W, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = fmin(fmax(rint(seeds[2 * i]), 0.0), (double)(W - 1));
        const double y = fmin(fmax(rint(seeds[2 * i + 1]), 0.0), (double)(H - 1));
        out[2 * i] = x;
        out[2 * i + 1] = y;
    }
}

}  // namespace
}  // namespace spx

using namespace spx;

namespace {

struct VorWs {
    BinStorage bins;
    double* seed_px;
    double* tile_bound;  // one per 16 x 16 tile
};

VorWs vor_layout(void* ws, int n, int H, int W, size_t* bytes) {
    Arena a(ws);
    VorWs v;
    v.bins = bin_layout(a, n, H, W, bin_cell_size(n, H, W));
    v.seed_px = a.take<double>(2 * (size_t)(n > 0 ? n : 1));
    v.tile_bound = a.take<double>((size_t)((W + kTile - 1) / kTile) * ((H + kTile - 1) / kTile));
    if (bytes) *bytes = a.used;
    return v;
}

int launch_voronoi(const VorWs& L, int H, int W, int* labels, unsigned int* d2, cudaStream_t s) {
    const dim3 grid((W + kTile - 1) / kTile, (H + kTile - 1) / kTile);
    const int tiles = (int)(grid.x * grid.y);
    k_tile_bounds<<<grid_for(tiles, 8, 148 * 16), 256, 0, s>>>(H, W, bin_view(L.bins), (int)grid.x, tiles,
                                                               L.tile_bound);
    if (int e = check_launch("k_tile_bounds")) return e;
    k_voronoi<<<grid, kThreads, 0, s>>>(H, W, bin_view(L.bins), L.tile_bound, labels, d2);
    return check_launch("k_voronoi");
}

}  // namespace

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
    VorWs L = vor_layout(workspace, n, height, width, nullptr);
    if (int e = bin_build(L.bins, seeds, 2, nullptr, nullptr, n, s)) return e;
    if (int e = launch_voronoi(L, height, width, labels, nullptr, s)) return e;
    return SPX_OK;
}

int spx_seed_distance_map(const double* seeds, int n, int height, int width, unsigned int* d2,
                          void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(height > 0 && width > 0 && n >= 1, "bad arguments");
    SPX_REQUIRE(seeds && d2 && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_voronoi_workspace_bytes(n, height, width), "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    VorWs L = vor_layout(workspace, n, height, width, nullptr);
    k_seed_pixels<<<grid_for(n, 256), 256, 0, s>>>(seeds, n, height, width, L.seed_px);
    if (int e = check_launch("k_seed_pixels")) return e;
    if (int e = bin_build(L.bins, L.seed_px, 2, nullptr, nullptr, n, s)) return e;
    if (int e = launch_voronoi(L, height, width, nullptr, d2, s)) return e;
    return SPX_OK;
}

int spx_nearest_distances(const double* points, int n, const double* queries, int nq, int exclude_self,
                          int height, int width, double* out, void* workspace, size_t workspace_bytes,
                          void* stream) {
    SPX_REQUIRE(n >= 1 && nq >= 0, "bad arguments");
    SPX_REQUIRE(points && out && workspace && (queries || nq == 0), "null pointer");
    SPX_REQUIRE(workspace_bytes >= spx_voronoi_workspace_bytes(n, height, width), "workspace too small");
    if (nq == 0) return SPX_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    VorWs L = vor_layout(workspace, n, height, width, nullptr);
    if (int e = bin_build(L.bins, points, 2, nullptr, nullptr, n, s)) return e;
    k_nearest_query<<<grid_for(nq, 8, 148 * 32), 256, 0, s>>>(bin_view(L.bins), queries, nq, exclude_self, out);
    return check_launch("k_nearest_query");
}

}  // extern "C"
