// Square-bin grid of 2-D points (counting sort by bin), shared by the Voronoi partition, the model
// render and nearest-point queries. Points outside the image fall into the clamped edge bins, and a
// query of a rectangle clamps its bin range the same way, so every point inside the rectangle is
// found.
#pragma once

#include "common.cuh"
#include "scan.cuh"

namespace spx {

struct BinGrid {
    int gw, gh;
    double cell;
    const int* start;    // (gw*gh + 1) offsets into xy/id
    const double2* xy;   // points in bin order
    const int* id;       // original index of each point
};

__device__ __forceinline__ int bin_index(double v, double cell, int n) {
    double f = floor(v / cell);
    if (!(f >= 0.0)) f = 0.0;  // also maps NaN to 0
    if (f > (double)(n - 1)) f = (double)(n - 1);
    return (int)f;
}

struct BinStorage {
    int gw, gh;
    double cell;
    int* counts;
    int* start;
    int* fill;
    double2* xy;
    int* id;
    int* scratch;
};

// Cell size for about `per_bin` points per bin over an H x W image (at least min_cell).
inline double bin_cell_size(long long n, int H, int W, double per_bin = 1.0, double min_cell = 1.0) {
    double cell = floor(sqrt((double)H * (double)W * per_bin / (double)(n > 0 ? n : 1)));
    if (cell < min_cell) cell = min_cell;
    return cell;
}

// Lays out (or sizes, with a null arena base) the storage of a grid of n points.
inline BinStorage bin_layout(Arena& a, long long n, int H, int W, double cell) {
    BinStorage b;
    b.cell = cell;
    b.gw = (int)ceil(W / cell);
    b.gh = (int)ceil(H / cell);
    if (b.gw < 1) b.gw = 1;
    if (b.gh < 1) b.gh = 1;
    const long long bins = (long long)b.gw * b.gh;
    b.counts = a.take<int>(bins + 1);
    b.start = a.take<int>(bins + 1);
    b.fill = a.take<int>(bins + 1);
    b.xy = a.take<double2>(n > 0 ? n : 1);
    b.id = a.take<int>(n > 0 ? n : 1);
    b.scratch = a.take<int>(scan_scratch_ints(bins + 1));
    return b;
}

// Sorts n points (x at pts[i*stride], y at pts[i*stride+1], optionally offset per point by
// origin[2i], origin[2i+1]) into bins. Points whose `valid` flag is 0 are left out.
int bin_build(BinStorage& b, const double* pts, int stride, const int* origin, const uint8_t* valid,
              long long n, cudaStream_t s);

inline BinGrid bin_view(const BinStorage& b) {
    return BinGrid{b.gw, b.gh, b.cell, b.start, b.xy, b.id};
}

}  // namespace spx
