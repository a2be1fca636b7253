// The learned warm start of the LM fits: a 1024 -> 256 -> 256 -> 7 MLP on 32x32 cell patches.
//
// GEMMs run on the 5th-generation tensor cores: one CTA of 128 threads computes a 128 x BN tile of
// C = A B^T (A: M x K, B: N x K, both bf16 and K-contiguous) with the accumulator in TMEM. Operand
// tiles of 64 K are copied with cp.async into a two-stage ring of 128-byte-swizzled shared-memory
// tiles, one K-block ahead, two CTAs per SM; thread 0 issues four tcgen05.mma (K = 16 each) per stage and commits
// them to the stage's mbarrier, which gates the reuse of that stage. The epilogue reads TMEM with
// tcgen05.ld (warp w owns rows 32w..32w+31) and applies scale, bias, ReLU or the ReLU derivative of a forward
// activation, and writes f32 and/or bf16 outputs, row-major or transposed (the transposed copies
// feed the weight-gradient GEMMs, whose reduction runs over the batch).
//
// Every wait on an mbarrier is bounded; a wait that runs out sets the error flag and the kernel
// still frees its TMEM.

#include <cuda_bf16.h>

#include "umma.cuh"

namespace spx {
namespace {

constexpr int kGemmThreads = 128;
constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
// Shared-memory ring of K-blocks. Two stages (97 KB with BN = 256) let two CTAs share an SM, so one
// CTA's copies overlap the other's MMAs: 1.4-1.6x faster MLP forward passes than four stages at
// one CTA per SM, same bits.
constexpr int kGemmStages = 2;
constexpr long long kWaitLimit = 1ll << 24;

struct GemmEpi {
    float scale;
    const float* bias;
    int relu;
    const __nv_bfloat16* mask_act;
    int ld_mask;
    float* out_f32;
    int ld_f32;
    int accumulate;
    __nv_bfloat16* out_bf16;
    int ld_bf16;
    __nv_bfloat16* out_bf16_t;
    int ld_t;
};

// Copies rows [r0, r0 + rows) x K-block kb of a K-contiguous bf16 matrix into a swizzled tile,
// zero past `valid_rows` and past K.
__device__ __forceinline__ void load_tile(uint8_t* tile, const __nv_bfloat16* src, int ld, int r0, int rows,
                                          int valid_rows, int kb, int K) {
    const int chunks = rows * 8;
    for (int c = threadIdx.x; c < chunks; c += kGemmThreads) {
        const int r = c >> 3, ch = c & 7;
        const int k = kb * kGemmBK + ch * 8;
        const int row = r0 + r;
        int bytes = 0;
        const __nv_bfloat16* p = src;
        if (row < valid_rows && k < K) {
            bytes = min(16, (K - k) * 2);
            p = src + (long long)row * ld + k;
        }
        cp_async16(tile + r * 128 + ((ch ^ (r & 7)) << 4), p, bytes);
    }
}

__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B,
                                                            int ldb, int M, int N, int K, int BN, uint32_t tmem_cols,
                                                            GemmEpi ep, int* err) {
    extern __shared__ uint8_t smem_raw[];
    // kGemmStages 1024-byte aligned stages [A | B], then one mbarrier per stage and the TMEM address.
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int a_bytes = kGemmBM * 128, b_bytes = BN * 128, stage_bytes = a_bytes + b_bytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(base + kGemmStages * stage_bytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + kGemmStages);
    const int warp = threadIdx.x >> 5;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
    auto stage_a = [&](int s) { return base + s * stage_bytes; };
    auto stage_b = [&](int s) { return base + s * stage_bytes + a_bytes; };

    if (warp == 0) tmem_alloc(tmem_slot, tmem_cols);
    if (threadIdx.x == 0)
        for (int s = 0; s < kGemmStages; ++s) mbar_init(&mbar[s], 1);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc_bf16(kGemmBM, BN);
    const int nk = (K + kGemmBK - 1) / kGemmBK;
    bool ok = true;

    // Prologue: the first kGemmStages - 1 K-blocks in flight (one cp.async group each, empty
    // groups past the end keep the group count uniform).
    for (int kb = 0; kb < kGemmStages - 1; ++kb) {
        if (kb < nk) {
            load_tile(stage_a(kb), A, lda, m0, kGemmBM, M, kb, K);
            load_tile(stage_b(kb), B, ldb, n0, BN, N, kb, K);
        }
        cp_async_commit();
    }
    for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % kGemmStages;
        const int kn = kb + kGemmStages - 1;  // block to fetch now, into the stage block kb - 1 used
        if (kn < nk) {
            const int sn = kn % kGemmStages;
            // Every thread polls with its own bounded wait; the outcome is made block-uniform so that
            // either all threads refill the stage or none does (a stage the MMA may still read is
            // never overwritten), and the loop is left by all threads together.
            if (kb >= 1) ok = __syncthreads_and(mbar_wait(&mbar[sn], ((kb - 1) / kGemmStages) & 1, kWaitLimit)) != 0;
            if (!ok) break;
            load_tile(stage_a(sn), A, lda, m0, kGemmBM, M, kn, K);
            load_tile(stage_b(sn), B, ldb, n0, BN, N, kn, K);
        }
        cp_async_commit();
        asm volatile("cp.async.wait_group %0;\n" : : "n"(kGemmStages - 1) : "memory");
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint64_t ad = umma_desc_sw128(smem_u32(stage_a(s)));
            const uint64_t bd = umma_desc_sw128(smem_u32(stage_b(s)));
#pragma unroll
            for (int k = 0; k < kGemmBK / 16; ++k)
                umma_bf16(tmem, ad + (uint64_t)((k * 32) >> 4), bd + (uint64_t)((k * 32) >> 4), idesc,
                          (kb > 0 || k > 0) ? 1u : 0u);
            umma_commit(&mbar[s]);
        }
    }
    // The last commit covers every MMA of the tile. `ok` is block-uniform here and after the wait, so
    // the warp-collective tcgen05.ld of the epilogue runs with whole warps or not at all.
    if (ok) ok = __syncthreads_and(mbar_wait(&mbar[(nk - 1) % kGemmStages], ((nk - 1) / kGemmStages) & 1,
                                             kWaitLimit)) != 0;
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // no copy into shared memory outlives the block
    tc_fence_after();
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);

    if (ok) {
        const int m = m0 + warp * 32 + (threadIdx.x & 31);
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_ld16(lane_addr + (uint32_t)c0, v);
            if (m >= M) continue;
            const int nb = n0 + c0;
            const int cnt = min(16, N - nb);
            if (cnt <= 0) continue;
            float x[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int n = nb + i;
                float t = v[i] * ep.scale;
                if (i < cnt) {
                    if (ep.bias) t += ep.bias[n];
                    if (ep.mask_act && !(__bfloat162float(ep.mask_act[(long long)m * ep.ld_mask + n]) > 0.0f)) t = 0.0f;
                }
                if (ep.relu) t = fmaxf(t, 0.0f);
                x[i] = t;
            }
            // Row-major outputs: 16-byte vector stores for a full, aligned chunk of 16 columns.
            if (ep.out_f32) {
                float* o = ep.out_f32 + (long long)m * ep.ld_f32 + nb;
                if (cnt == 16 && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
                    float4* o4 = reinterpret_cast<float4*>(o);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        float4 w = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
                        if (ep.accumulate) {
                            const float4 u = o4[q];
                            w.x += u.x; w.y += u.y; w.z += u.z; w.w += u.w;
                        }
                        o4[q] = w;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (i < cnt) o[i] = ep.accumulate ? o[i] + x[i] : x[i];
                }
            }
            if (ep.out_bf16) {
                __nv_bfloat16* o = ep.out_bf16 + (long long)m * ep.ld_bf16 + nb;
                if (cnt == 16 && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
                    uint4 pk[2];
                    uint32_t* w = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
                        w[q] = *reinterpret_cast<const uint32_t*>(&h);
                    }
                    reinterpret_cast<uint4*>(o)[0] = pk[0];
                    reinterpret_cast<uint4*>(o)[1] = pk[1];
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (i < cnt) o[i] = __float2bfloat16_rn(x[i]);
                }
            }
            if (ep.out_bf16_t)  // consecutive rows on consecutive lanes: coalesced per column
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (i < cnt) ep.out_bf16_t[(long long)(nb + i) * ep.ld_t + m] = __float2bfloat16_rn(x[i]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols);
}

// Weighted MSE gradient: dy = 2 w_j (y - t) / B as bf16, row-major (B x ldd, zero in the padding
// columns) and transposed (ldd x B); loss += sum w_j (y - t)^2 / B (f64 atomics per block).
__global__ void k_mse_grad(const float* y, const float* t, const float* w, int B, int nout, int ldd,
                           __nv_bfloat16* dy, __nv_bfloat16* dy_t, double* loss) {
    __shared__ double s_part[32];
    double part = 0.0;
    const long long total = (long long)B * ldd;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int b, j;
        divmod_idx(i, ldd, &b, &j);
        float g = 0.0f;
        if (j < nout) {
            const float d = y[(long long)b * nout + j] - t[(long long)b * nout + j];
            part += (double)w[j] * d * d;
            g = 2.0f * w[j] * d / (float)B;
        }
        const __nv_bfloat16 gb = __float2bfloat16_rn(g);
        dy[i] = gb;
        dy_t[(long long)j * B + b] = gb;
    }
    part = warp_sum(part);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) acc += s_part[i];
        atomicAdd(loss, acc / (double)B);
    }
}

// out[r] = sum over the row r of a bf16 matrix (R x C), f32 accumulation, one warp per row.
__global__ void k_rowsum_bf16(const __nv_bfloat16* src, int R, int C, float* out) {
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < R; r += gridDim.x * (blockDim.x >> 5)) {
        float acc = 0.0f;
        for (int c = lane; c < C; c += 32) acc += __bfloat162float(src[(long long)r * C + c]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[r] = acc;
    }
}

// AdamW on f32 parameters (rows x cols): m, v moments, bias-corrected step, decoupled decay; then
// the bf16 copy (row-major, padded to out_rows rows of zeros) and/or its transpose (cols x ld_t).
__global__ void k_adamw(float* p, const float* g, float* m, float* v, int rows, int cols, float lr, float beta1,
                        float beta2, float eps, float wd, float c1, float c2, __nv_bfloat16* out, int out_rows,
                        __nv_bfloat16* out_t, int ld_t) {
    const long long total = (long long)max(rows, out_rows) * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int r, c;
        divmod_idx(i, cols, &r, &c);
        float w = 0.0f;
        if (r < rows) {
            const float gi = g[i];
            const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
            const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            const float mh = mi / c1, vh = vi / c2;
            w = p[i] - lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
            p[i] = w;
        }
        if (out && r < out_rows) out[i] = __float2bfloat16_rn(w);
        if (out_t && r < rows) out_t[(long long)c * ld_t + r] = __float2bfloat16_rn(w);
    }
}

// dst (C x R) = src (R x C)^T for bf16, through 32 x 32 shared-memory tiles.
__global__ void k_transpose_bf16(const __nv_bfloat16* src, int R, int C, __nv_bfloat16* dst) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < R && c < C) tile[i][threadIdx.x] = src[(long long)r * C + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < R && c < C) dst[(long long)c * R + r] = tile[threadIdx.x][i];
    }
}

// Standardised MLP outputs -> ROI-local LM starting params: A = t0 amp, x0 = ox + 16 + t1 - box.x,
// y0 = oy + 16 + t2 - box.y, u = t3..t5 (t = y * std + mean); ok = finite and A > 0.
__global__ void k_outputs_to_params(const float* y, const double* mean, const double* stdv, const double* norm,
                                    const int4* boxes, int n, double* params, uint8_t* ok) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double t[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) t[j] = (double)y[7LL * i + j] * stdv[j] + mean[j];
        const double* nm = norm + 4LL * i;
        const int4 b = boxes[i];
        // Patch origin relative to the box first (exact integers), so the result does not depend on
        // where the box sits (a stack's rows).
        const double p[6] = {t[0] * nm[3], (nm[0] - b.x) + 16.0 + t[1], (nm[1] - b.y) + 16.0 + t[2], t[3], t[4],
                             t[5]};
        bool good = p[0] > 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            good = good && isfinite(p[j]);
            params[6LL * i + j] = p[j];
        }
        ok[i] = good;
    }
}

size_t gemm_smem(int BN) { return kGemmStages * (size_t)(kGemmBM * 128 + BN * 128) + 8 * kGemmStages + 16 + 1024; }

}  // namespace
}  // namespace spx

using namespace spx;

extern "C" {

int spx_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K, const spx_gemm_epilogue* epi,
                  int* error_flag, void* stream) {
    SPX_REQUIRE(M > 0 && N > 0 && K > 0 && lda >= K && ldb >= K, "bad GEMM shape");
    SPX_REQUIRE(lda % 8 == 0 && ldb % 8 == 0, "lda and ldb must be multiples of 8 (16-byte rows)");
    SPX_REQUIRE(A && B && epi && error_flag, "null pointer");
    SPX_REQUIRE(reinterpret_cast<uintptr_t>(A) % 16 == 0 && reinterpret_cast<uintptr_t>(B) % 16 == 0,
                "operands must be 16-byte aligned");
    SPX_REQUIRE(epi->out_f32 || epi->out_bf16 || epi->out_bf16_t, "no output");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Column tile: all of N up to 256 (a multiple of 16), else 256-wide tiles.
    const int BN = N >= 256 ? 256 : ((N + 15) / 16) * 16;
    uint32_t cols = 32;
    while ((int)cols < BN) cols <<= 1;
    const size_t smem = gemm_smem(BN);
    SPX_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    GemmEpi ep{epi->scale,
               epi->bias,
               epi->relu,
               static_cast<const __nv_bfloat16*>(epi->mask_act),
               epi->ld_mask,
               epi->out_f32,
               epi->ld_f32,
               epi->accumulate,
               static_cast<__nv_bfloat16*>(epi->out_bf16),
               epi->ld_bf16,
               static_cast<__nv_bfloat16*>(epi->out_bf16_t),
               epi->ld_t};
    const dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + BN - 1) / BN);
    k_gemm_bf16<<<grid, kGemmThreads, smem, s>>>(static_cast<const __nv_bfloat16*>(A), lda,
                                                 static_cast<const __nv_bfloat16*>(B), ldb, M, N, K, BN, cols, ep,
                                                 error_flag);
    return check_launch("k_gemm_bf16");
}

int spx_mlp_loss_grad(const float* y, const float* t, const float* weights, int batch, int n_out, int ld_grad,
                      void* dy, void* dy_t, double* loss, void* stream) {
    SPX_REQUIRE(batch > 0 && n_out > 0 && ld_grad >= n_out, "bad arguments");
    SPX_REQUIRE(y && t && weights && dy && dy_t && loss, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_mse_grad<<<grid_for((long long)batch * ld_grad, 256, 148 * 4), 256, 0, s>>>(
        y, t, weights, batch, n_out, ld_grad, static_cast<__nv_bfloat16*>(dy), static_cast<__nv_bfloat16*>(dy_t), loss);
    return check_launch("k_mse_grad");
}

int spx_rowsum_bf16(const void* src, int rows, int cols, float* out, void* stream) {
    SPX_REQUIRE(rows > 0 && cols > 0 && src && out, "bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_rowsum_bf16<<<grid_for(rows, 8, 148 * 8), 256, 0, s>>>(static_cast<const __nv_bfloat16*>(src), rows, cols, out);
    return check_launch("k_rowsum_bf16");
}

int spx_adamw(float* param, const float* grad, float* m, float* v, int rows, int cols, int step, float lr, float beta1,
              float beta2, float eps, float weight_decay, void* out_bf16, int out_rows, void* out_bf16_t, int ld_t,
              void* stream) {
    SPX_REQUIRE(rows > 0 && cols > 0 && step >= 1 && out_rows >= 0 && (!out_bf16_t || ld_t >= rows),
                "bad arguments");
    SPX_REQUIRE(param && grad && m && v, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_adamw<<<grid_for((long long)max(rows, out_rows) * cols, 256), 256, 0, s>>>(
        param, grad, m, v, rows, cols, lr, beta1, beta2, eps, weight_decay, c1, c2,
        static_cast<__nv_bfloat16*>(out_bf16), out_rows, static_cast<__nv_bfloat16*>(out_bf16_t), ld_t);
    return check_launch("k_adamw");
}

int spx_transpose_bf16(const void* src, int rows, int cols, void* dst, void* stream) {
    SPX_REQUIRE(rows > 0 && cols > 0 && src && dst && src != dst, "bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    k_transpose_bf16<<<grid, dim3(32, 8), 0, s>>>(static_cast<const __nv_bfloat16*>(src), rows, cols,
                                                 static_cast<__nv_bfloat16*>(dst));
    return check_launch("k_transpose_bf16");
}

int spx_mlp_outputs_to_params(const float* y, const double* out_mean, const double* out_std, const double* norm,
                              const int* boxes, int n, double* params, uint8_t* ok, void* stream) {
    SPX_REQUIRE(n >= 0, "bad arguments");
    if (n == 0) return SPX_OK;
    SPX_REQUIRE(y && out_mean && out_std && norm && boxes && params && ok, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_outputs_to_params<<<grid_for(n, 256), 256, 0, s>>>(y, out_mean, out_std, norm,
                                                        reinterpret_cast<const int4*>(boxes), n, params, ok);
    return check_launch("k_outputs_to_params");
}

}  // extern "C"
