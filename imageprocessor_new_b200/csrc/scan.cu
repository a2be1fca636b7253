#include "scan.cuh"

namespace spx {

__global__ void k_scan_tile_sums(const int* in, long long n, int* tile_sums) {
    __shared__ int s[32];
    const long long base = (long long)blockIdx.x * kScanTile;
    int acc = 0;
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
        const long long k = base + i;
        if (k < n) acc += in[k];
    }
    acc = warp_sum_i(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0;
        v = warp_sum_i(v);
        if (threadIdx.x == 0) tile_sums[blockIdx.x] = v;
    }
}

__global__ void k_scan_tile_sums_exclusive(int* tile_sums, int tiles, int* total) {
    __shared__ int s[kScanThreads];
    const int per = (tiles + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    int acc = 0;
    for (int i = 0; i < per; ++i)
        if (b0 + i < tiles) acc += tile_sums[b0 + i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const int v = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int run = s[threadIdx.x] - acc;
    for (int i = 0; i < per; ++i)
        if (b0 + i < tiles) {
            const int v = tile_sums[b0 + i];
            tile_sums[b0 + i] = run;
            run += v;
        }
    if (threadIdx.x == blockDim.x - 1 && total) *total = s[threadIdx.x];
}

__global__ void k_scan_apply(const int* in, long long n, const int* tile_offsets, int* out) {
    __shared__ int s[kScanThreads];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int acc = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        acc += v[i];
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const int t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    int run = tile_offsets[blockIdx.x] + s[threadIdx.x] - acc;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) {
            out[base + i] = run;
            run += v[i];
        }
}

int exclusive_scan(const int* in, long long n, int* out, int* total, int* scratch, cudaStream_t s) {
    const int tiles = scan_tiles(n);
    if (n <= 0) {
        if (total) SPX_CUDA(cudaMemsetAsync(total, 0, sizeof(int), s));
        return SPX_OK;
    }
    SPX_REQUIRE(tiles <= kScanThreads * 64, "scan too large");
    k_scan_tile_sums<<<tiles, kScanThreads, 0, s>>>(in, n, scratch);
    if (int e = check_launch("k_scan_tile_sums")) return e;
    k_scan_tile_sums_exclusive<<<1, kScanThreads, 0, s>>>(scratch, tiles, total);
    if (int e = check_launch("k_scan_tile_sums_exclusive")) return e;
    k_scan_apply<<<tiles, kScanThreads, 0, s>>>(in, n, scratch, out);
    return check_launch("k_scan_apply");
}

}  // namespace spx
