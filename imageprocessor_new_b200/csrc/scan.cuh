// Exclusive prefix sum of int32 counts in three launches (block sums, one-block scan of the block
// sums, per-block scan plus offset). Used for order-preserving compaction and counting sorts.
#pragma once

#include "common.cuh"

namespace spx {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void k_scan_tile_sums(const int* in, long long n, int* tile_sums);
__global__ void k_scan_tile_sums_exclusive(int* tile_sums, int tiles, int* total);
__global__ void k_scan_apply(const int* in, long long n, const int* tile_offsets, int* out);

inline int scan_tiles(long long n) { return (int)((n + kScanTile - 1) / kScanTile); }

// Workspace ints needed by exclusive_scan for n items.
inline long long scan_scratch_ints(long long n) { return scan_tiles(n) + 1; }

// out[i] = sum(in[0..i)); *total (device) = sum(in). `in` and `out` may alias.
int exclusive_scan(const int* in, long long n, int* out, int* total, int* scratch, cudaStream_t s);

}  // namespace spx
