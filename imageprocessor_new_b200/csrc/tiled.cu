// Tiled centre detection helpers: band keep rule and the merge of near-duplicate centres.
//
// Reference: subpx/_gpu/centers.py:1811-1843 (bands of tile_h rows stepping tile_h - overlap, keep
// y in [y0 + overlap/2, y1 - overlap/2) except at the image edges) and dedupe_centers
// (subpx/centers.py:335-378): union-find over every pair of centres with squared distance <= eps^2,
// each cluster replaced by the mean of its members (summed in index order). The reference visits
// all O(N^2) pairs in Python; here a bin grid of cell >= eps restricts candidate pairs to the 3x3
// neighbouring bins, unions link the larger root under the smaller (so a cluster's root is its
// smallest member) and clusters are emitted in order of that smallest member.

#include "bins.cuh"

namespace spx {
namespace {

__global__ void k_keep_flags(const double* c, int n, double y_off, double lo, double hi, int* flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = c[2 * i], y = c[2 * i + 1];
        const double gy = y + y_off;
        flags[i] = isfinite(x) && isfinite(y) && gy >= lo && gy < hi;
    }
}

__global__ void k_keep_scatter(const double* c, int n, double y_off, const int* flags, const int* offs,
                               const int* base, double* out, int capacity) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!flags[i]) continue;
        const int o = *base + offs[i];
        if (o < capacity) {
            out[2LL * o] = c[2 * i];
            out[2LL * o + 1] = c[2 * i + 1] + y_off;
        }
    }
}

__global__ void k_add_count(int* base, const int* total) { *base += *total; }

__device__ __forceinline__ int uf_find(int* p, int a) {
    while (true) {
        const int b = p[a];
        if (b == a) return a;
        const int c = p[b];
        if (c == b) return b;
        p[a] = c;
        a = c;
    }
}

__device__ void uf_unite(int* p, int a, int b) {
    while (true) {
        a = uf_find(p, a);
        b = uf_find(p, b);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }
        const int old = atomicMin(&p[a], b);
        if (old == a) return;
        a = old;
    }
}

__global__ void k_shift(const double* pts, int n, double x0, double y0, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[2 * i] = pts[2 * i] - x0;
        out[2 * i + 1] = pts[2 * i + 1] - y0;
    }
}

__global__ void k_iota(int* p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = i;
}

// Pairs within eps: bins from the shifted coordinates, distances from the original ones (the
// reference's pts[j] - pts[i]).
__global__ void k_pairs(BinGrid g, const double* shifted, const double* pts, int n, double eps2, int* parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = pts[2 * i], y = pts[2 * i + 1];
        const int bx = bin_index(shifted[2 * i], g.cell, g.gw), by = bin_index(shifted[2 * i + 1], g.cell, g.gh);
        for (int gy = max(by - 1, 0); gy <= min(by + 1, g.gh - 1); ++gy)
            for (int gx = max(bx - 1, 0); gx <= min(bx + 1, g.gw - 1); ++gx) {
                const int b = gy * g.gw + gx;
                for (int k = g.start[b]; k < g.start[b + 1]; ++k) {
                    const int j = g.id[k];
                    if (j <= i) continue;
                    const double dx = __dsub_rn(pts[2LL * j], x), dy = __dsub_rn(pts[2LL * j + 1], y);
                    if (__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= eps2) uf_unite(parent, i, j);
                }
            }
    }
}

__global__ void k_roots(int* parent, int n, int* is_root) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = uf_find(parent, i);
        parent[i] = r;
        is_root[i] = r == i;
    }
}

__global__ void k_cluster_count(const int* parent, const int* slot_of, int n, int* counts) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&counts[slot_of[parent[i]]], 1);
}

__global__ void k_cluster_fill(const int* parent, const int* slot_of, int n, const int* offs, int* fill,
                               int* members) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = slot_of[parent[i]];
        members[offs[c] + atomicAdd(&fill[c], 1)] = i;
    }
}

// Mean of each cluster, members added in increasing index order (np.add.at order).
__global__ void k_cluster_mean(const double* pts, const int* offs, int* members, int nc, double* out) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        int* m = members + offs[c];
        const int k = offs[c + 1] - offs[c];
        for (int a = 1; a < k; ++a) {  // insertion sort of the (few) member indices
            const int v = m[a];
            int b = a - 1;
            while (b >= 0 && m[b] > v) { m[b + 1] = m[b]; --b; }
            m[b + 1] = v;
        }
        double sx = 0.0, sy = 0.0;
        for (int a = 0; a < k; ++a) {
            sx = __dadd_rn(sx, pts[2LL * m[a]]);
            sy = __dadd_rn(sy, pts[2LL * m[a] + 1]);
        }
        out[2LL * c] = __ddiv_rn(sx, (double)max(k, 1));
        out[2LL * c + 1] = __ddiv_rn(sy, (double)max(k, 1));
    }
}

}  // namespace
}  // namespace spx

using namespace spx;

namespace {

// The grid covers the points' bounding box (given by the caller) with square cells >= eps.
struct Frame {
    double x0, y0, cell;
    int gw, gh;
};

Frame make_frame(double xmin, double ymin, double xmax, double ymax, double eps, long long n) {
    Frame f;
    const double w = fmax(xmax - xmin, 1.0), h = fmax(ymax - ymin, 1.0);
    double cell = sqrt(w * h * 2.0 / (double)(n > 0 ? n : 1));
    if (cell < eps) cell = eps;
    if (cell <= 0) cell = 1.0;
    // Keep the grid below 2^26 bins.
    while ((w / cell + 1) * (h / cell + 1) > 67108864.0) cell *= 2.0;
    f.x0 = xmin;
    f.y0 = ymin;
    f.cell = cell;
    f.gw = (int)floor(w / cell) + 1;
    f.gh = (int)floor(h / cell) + 1;
    return f;
}

struct DedupeWs {
    BinStorage bins;
    double* shifted;
    int* parent;
    int* slot;
    int* counts;
    int* offs;
    int* fill;
    int* members;
    int* scratch;
    int* total;
};

DedupeWs dedupe_ws(void* ws, int n, const Frame& f, size_t* bytes) {
    Arena a(ws);
    DedupeWs L;
    const int m = n > 0 ? n : 1;
    // bin_layout sizes the grid from an image of gw*cell x gh*cell pixels.
    L.bins = bin_layout(a, m, (int)(f.gh * f.cell), (int)(f.gw * f.cell), f.cell);
    L.shifted = a.take<double>(2 * (size_t)m);
    L.parent = a.take<int>(m);
    L.slot = a.take<int>(m);
    L.counts = a.take<int>(m + 1);
    L.offs = a.take<int>(m + 1);
    L.fill = a.take<int>(m + 1);
    L.members = a.take<int>(m);
    L.scratch = a.take<int>(scan_scratch_ints(m + 1));
    L.total = a.take<int>(2);
    if (bytes) *bytes = a.used;
    return L;
}

}  // namespace

extern "C" {

int spx_keep_band(const double* centers, int n, double y_offset, double keep_lo, double keep_hi, double* out,
                  int* count, int capacity, void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && capacity >= 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(centers && out && count && workspace, "null pointer");
    SPX_REQUIRE(workspace_bytes >= (size_t)(2 * n + scan_scratch_ints(n) + 8) * sizeof(int) + 1024, "workspace too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena a(workspace);
    int* flags = a.take<int>(n);
    int* offs = a.take<int>(n);
    int* scratch = a.take<int>(scan_scratch_ints(n));
    int* total = a.take<int>(2);
    k_keep_flags<<<grid_for(n, 256), 256, 0, s>>>(centers, n, y_offset, keep_lo, keep_hi, flags);
    if (int e = check_launch("k_keep_flags")) return e;
    if (int e = exclusive_scan(flags, n, offs, total, scratch, s)) return e;
    k_keep_scatter<<<grid_for(n, 256), 256, 0, s>>>(centers, n, y_offset, flags, offs, count, out, capacity);
    if (int e = check_launch("k_keep_scatter")) return e;
    k_add_count<<<1, 1, 0, s>>>(count, total);
    return check_launch("k_add_count");
}

size_t spx_keep_band_workspace_bytes(int n) {
    return (size_t)(2 * (size_t)(n > 0 ? n : 1) + scan_scratch_ints(n > 0 ? n : 1) + 8) * sizeof(int) + 1024 +
           4 * 256;
}

size_t spx_dedupe_workspace_bytes(int n, double xmin, double ymin, double xmax, double ymax, double eps) {
    size_t b = 0;
    dedupe_ws(nullptr, n, make_frame(xmin, ymin, xmax, ymax, eps, n), &b);
    return b;
}

int spx_dedupe_centers(const double* centers, int n, double xmin, double ymin, double xmax, double ymax, double eps,
                       double* out, int* count, void* workspace, size_t workspace_bytes, void* stream) {
    SPX_REQUIRE(n >= 0 && eps >= 0, "bad arguments");
    SPX_REQUIRE(count && (n == 0 || (centers && out && workspace)), "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        SPX_CUDA(cudaMemsetAsync(count, 0, sizeof(int), s));
        return SPX_OK;
    }
    const Frame f = make_frame(xmin, ymin, xmax, ymax, eps, n);
    SPX_REQUIRE(workspace_bytes >= spx_dedupe_workspace_bytes(n, xmin, ymin, xmax, ymax, eps), "workspace too small");
    DedupeWs L = dedupe_ws(workspace, n, f, nullptr);
    k_shift<<<grid_for(n, 256), 256, 0, s>>>(centers, n, f.x0, f.y0, L.shifted);
    if (int e = check_launch("k_shift")) return e;
    if (int e = bin_build(L.bins, L.shifted, 2, nullptr, nullptr, n, s)) return e;
    k_iota<<<grid_for(n, 256), 256, 0, s>>>(L.parent, n);
    if (int e = check_launch("k_iota")) return e;
    k_pairs<<<grid_for(n, 256), 256, 0, s>>>(bin_view(L.bins), L.shifted, centers, n, eps * eps, L.parent);
    if (int e = check_launch("k_pairs")) return e;
    k_roots<<<grid_for(n, 256), 256, 0, s>>>(L.parent, n, L.slot);
    if (int e = check_launch("k_roots")) return e;
    // slot[i] = number of roots before i (cluster index of root i), count = number of clusters.
    if (int e = exclusive_scan(L.slot, n, L.slot, count, L.scratch, s)) return e;
    SPX_CUDA(cudaMemsetAsync(L.counts, 0, (n + 1) * sizeof(int), s));
    SPX_CUDA(cudaMemsetAsync(L.fill, 0, (n + 1) * sizeof(int), s));
    k_cluster_count<<<grid_for(n, 256), 256, 0, s>>>(L.parent, L.slot, n, L.counts);
    if (int e = check_launch("k_cluster_count")) return e;
    if (int e = exclusive_scan(L.counts, n + 1, L.offs, nullptr, L.scratch, s)) return e;
    k_cluster_fill<<<grid_for(n, 256), 256, 0, s>>>(L.parent, L.slot, n, L.offs, L.fill, L.members);
    if (int e = check_launch("k_cluster_fill")) return e;
    // Clusters: count of them is at most n; the mean kernel reads offs[c + 1] for c < clusters.
    k_cluster_mean<<<grid_for(n, 256), 256, 0, s>>>(centers, L.offs, L.members, n, out);
    return check_launch("k_cluster_mean");
}

}  // extern "C"
