// Order statistics over a CTA: order-preserving 64-bit keys of doubles and the radix select that
// the tile medians, the quantiles and the averaged peaks of the area methods use.
#pragma once

#include "common.cuh"

namespace spx {
namespace {

__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_value(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)u);
}

// Inclusive scan of one int per thread over a CTA of NT threads (NT / 32 <= 32 warps).
template <int NT>
__device__ __forceinline__ int cta_incl_scan(int v, int* warp_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int w = lane < NT / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        if (lane < NT / 32) warp_tot[lane] = w;
    }
    __syncthreads();
    const int r = v + (warp ? warp_tot[warp - 1] : 0);
    __syncthreads();
    return r;
}

// One radix pass of a CTA-wide select: hist[2048] holds the counts of the current digit (at most 11
// bits) among the keys that match the prefix so far; finds the digit holding the kk-th key, the
// rank inside it and the digit's count (s_pick[0..2]). NT threads, each owning 2048 / NT
// consecutive bins.
template <int NT>
__device__ __forceinline__ void cta_pick_digit(const int* hist, int nb, int kk, int* warp_tot, int* s_pick) {
    constexpr int per = 2048 / NT;
    const int b0 = per * threadIdx.x;
    int c[per];
    int mine = 0;
#pragma unroll
    for (int j = 0; j < per; ++j) {
        c[j] = b0 + j < nb ? hist[b0 + j] : 0;
        mine += c[j];
    }
    const int incl = cta_incl_scan<NT>(mine, warp_tot);
    int excl = incl - mine;
    if (excl <= kk && kk < incl) {
#pragma unroll
        for (int j = 0; j < per; ++j) {
            if (kk < excl + c[j]) {
                s_pick[0] = b0 + j;
                s_pick[1] = kk - excl;
                s_pick[2] = c[j];
                break;
            }
            excl += c[j];
        }
    }
    __syncthreads();
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The k-th smallest (0-based) of the 64-bit keys that for_keys visits and, when want_next, the
// (k+1)-th, by a CTA-wide radix select. kmin and kmax are the smallest and largest key: the bits
// above the highest one where they differ are common to all keys, so the 11-bit digits start
// below it; the passes stop as soon as the digit holding the k-th key holds no other key, and one
// last pass fetches that key and the smallest key above it. The keys' order statistics are
// exact, so the result does not depend on how many passes ran.
// for_keys(fn) calls fn(key) on every key once, spread over the CTA's threads; all NT threads
// call this function. s_pick: 3 ints, s_keys: 2 keys of shared memory.
template <int NT, class ForKeys>
__device__ void cta_select(ForKeys&& for_keys, int k, bool want_next, unsigned long long kmin,
                           unsigned long long kmax, int* hist, int* warp_tot, int* s_pick,
                           unsigned long long* s_keys, unsigned long long* key_k, unsigned long long* key_next) {
    if (kmin == kmax) {
        *key_k = *key_next = kmin;
        return;
    }
    const int top = 63 - __clzll((long long)(kmin ^ kmax));
    // Bits top+1..63 are common to every key (the shift of 2 by 63 is 0, so top = 63 leaves none).
    unsigned long long pmask = ~((2ull << top) - 1ull);
    unsigned long long prefix = kmin & pmask;
    int shift = top + 1, kk = k, cnt = 0;
    while (shift > 0) {
        const int bits = shift < 11 ? shift : 11, nb = 1 << bits;
        shift -= bits;
        for (int i = threadIdx.x; i < nb; i += NT) hist[i] = 0;
        __syncthreads();
        for_keys([&](unsigned long long key) {
            if ((key & pmask) == prefix) atomicAdd(&hist[(key >> shift) & (nb - 1)], 1);
        });
        __syncthreads();
        cta_pick_digit<NT>(hist, nb, kk, warp_tot, s_pick);
        prefix |= (unsigned long long)s_pick[0] << shift;
        pmask |= (unsigned long long)(nb - 1) << shift;
        kk = s_pick[1];
        cnt = s_pick[2];
        __syncthreads();
        if (cnt == 1) break;
    }
    // Fully resolved (shift 0): every key with the prefix equals it, and the (k+1)-th is the same
    // key when the digit holds it too. Otherwise the k-th is the digit's only key.
    const bool resolved = shift == 0;
    if (resolved && (!want_next || kk + 1 < cnt)) {
        *key_k = *key_next = prefix;
        return;
    }
    if (threadIdx.x == 0) {
        s_keys[0] = prefix;
        s_keys[1] = ~0ull;
    }
    __syncthreads();
    unsigned long long mn = ~0ull;
    for_keys([&](unsigned long long key) {
        const unsigned long long m = key & pmask;
        if (m == prefix) {
            if (!resolved) s_keys[0] = key;
        } else if (m > prefix && key < mn) {
            mn = key;
        }
    });
    mn = warp_min_u64(mn);
    if ((threadIdx.x & 31) == 0 && mn != ~0ull) atomicMin(&s_keys[1], mn);
    __syncthreads();
    *key_k = s_keys[0];
    *key_next = want_next ? s_keys[1] : s_keys[0];
    __syncthreads();
}

}  // namespace
}  // namespace spx
