// fno_kernels.cuh -- kernels of the learned initial guess (Fourier neural
// operator): a batched strided GEMM with FP32 accumulation (the weight
// operand may be stored in BF16), bias + GELU, their backward passes, channel
// sums, the MSE loss and Adam with BF16 weight copies.  Every dense piece of
// the network (pointwise channel mixing, the truncated DFT onto the retained
// modes, the per-mode channel mixing) is expressed as this GEMM.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace fno {

__device__ __forceinline__ float ldf(const float* p) { return *p; }
__device__ __forceinline__ float ldf(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// C[b](i,j) = alpha * sum_k A[b](i,k) B[b](k,j) + beta * C[b](i,j)
// element (i,k) of A[b] at A + b*sAb + i*sAi + k*sAk, likewise B and C.
// 64x64 output tile per block, 16-wide K slices, 256 threads x (4x4).
template <typename TA>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, float alpha, const TA* __restrict__ A,
                                              long long sAb, long long sAi, long long sAk, const float* __restrict__ B,
                                              long long sBb, long long sBk, long long sBj, float beta, float* C,
                                              long long sCb, long long sCi, long long sCj) {
    __shared__ float As[16][68];
    __shared__ float Bs[16][68];
    const long long b = blockIdx.z;
    const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    A += b * sAb;
    B += b * sBb;
    C += b * sCb;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[r][q] = 0.f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int e = threadIdx.x; e < 1024; e += 256) {
            // A tile: 64 rows x 16 k; choose the walk that keeps the
            // contiguous index fastest across threads
            int ii, kk;
            if (sAk == 1) { kk = e % 16; ii = e / 16; } else { ii = e % 64; kk = e / 64; }
            const int i = i0 + ii, k = k0 + kk;
            As[kk][ii] = (i < M && k < K) ? ldf(A + i * sAi + k * sAk) : 0.f;
            int jj, kb;
            if (sBj == 1) { jj = e % 64; kb = e / 64; } else { kb = e % 16; jj = e / 16; }
            const int j = j0 + jj, kq = k0 + kb;
            Bs[kb][jj] = (j < N && kq < K) ? B[kq * sBk + j * sBj] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], bb[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = As[kk][ty * 4 + r];
#pragma unroll
            for (int q = 0; q < 4; ++q) bb[q] = Bs[kk][tx * 4 + q];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[r][q] = fmaf(a[r], bb[q], acc[r][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = i0 + ty * 4 + r, j = j0 + tx * 4 + q;
            if (i < M && j < N) {
                float* c = C + i * sCi + j * sCj;
                *c = beta == 0.f ? alpha * acc[r][q] : alpha * acc[r][q] + beta * *c;
            }
        }
}

__device__ __forceinline__ float gelu_f(float x) {
    const float c = 0.7978845608028654f;  // sqrt(2/pi)
    return 0.5f * x * (1.f + tanhf(c * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_g(float x) {
    const float c = 0.7978845608028654f;
    const float u = c * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c * (1.f + 3.f * 0.044715f * x * x);
}

// z[b,c,s] += bias[c]; h = act(z) (act 1: GELU, 0: identity)
__global__ void k_bias_act(float* z, float* h, const float* bias, long long C, long long S, long long n, int act) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long c = (t / S) % C;
        const float v = z[t] + (bias ? bias[c] : 0.f);
        z[t] = v;
        if (h) h[t] = act ? gelu_f(v) : v;
    }
}

__global__ void k_act_bwd(float* dz, const float* dh, const float* z, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        dz[t] = dh[t] * gelu_g(z[t]);
}

// out[c] = beta*out[c] + sum_{b,s} x[b,c,s] in a fixed order.  S == 1 (the
// per-chunk weight-gradient partials): one thread per channel walks b, the
// reads coalesced across channels.  Otherwise one block per channel, each
// thread with eight independent accumulators over its strided elements.
__global__ void k_channel_sum_rows(float* out, const float* x, long long B, long long C, float beta) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    double acc = 0.0;
    for (long long b = 0; b < B; ++b) acc += x[b * C + c];
    out[c] = beta * out[c] + (float)acc;
}

__global__ void k_channel_sum(float* out, const float* x, long long B, long long C, long long S, float beta) {
    const long long c = blockIdx.x;
    const long long bd = blockDim.x;
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = 0.0;
    for (long long b = 0; b < B; ++b) {
        const float* row = x + (b * C + c) * S;
        long long s = threadIdx.x;
        for (; s + 7 * bd < S; s += 8 * bd) {
#pragma unroll
            for (int q = 0; q < 8; ++q) a[q] += row[s + q * bd];
        }
        for (; s < S; s += bd) a[0] += row[s];
    }
    const double acc = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = beta * out[c] + (float)red[0];
}

__global__ void k_axpy(float* y, const float* x, float a, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] += a * x[t];
}

// per-block partial sums of (out-target)^2; dout = 2 (out-target)/n
__global__ void k_mse(const float* out, const float* tgt, float* dout, double* part, long long n) {
    double acc = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const float d = out[t] - tgt[t];
        acc += (double)d * d;
        if (dout) dout[t] = 2.f * d / (float)n;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_sum_parts(const double* part, int n, double scale, double* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += part[i];
        *out = s * scale;
    }
}

// Adam on the FP32 master weights; wb receives the BF16 copy the GEMMs read.
__global__ void k_adam(float* w, __nv_bfloat16* wb, const float* g, float* m, float* v, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const float gg = g[t];
        const float mm = b1 * m[t] + (1.f - b1) * gg;
        const float vv = b2 * v[t] + (1.f - b2) * gg * gg;
        m[t] = mm;
        v[t] = vv;
        const float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        w[t] -= upd;
        if (wb) wb[t] = __float2bfloat16(w[t]);
    }
}

__global__ void k_to_bf16(const float* x, __nv_bfloat16* y, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] = __float2bfloat16(x[t]);
}

// Real block form of the per-mode complex channel mixing G = R H:
//   Rbig[mode] = [[Rr, -Ri], [Ri, Rr]]   (2O x 2C), R stored [mode][O][C]
__global__ void k_rbig_build(const float* rr, const float* ri, __nv_bfloat16* rb, long long nmodes, int O, int C) {
    const long long n = nmodes * 4LL * O * C;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long mode = t / (4LL * O * C);
        const int e = (int)(t % (4LL * O * C));
        const int row = e / (2 * C), col = e % (2 * C);
        const int po = row / O, o = row % O, pc = col / C, c = col % C;
        const long long src = (mode * O + o) * C + c;
        float v;
        if (po == pc) v = rr[src];
        else v = (po == 0) ? -ri[src] : ri[src];
        rb[t] = __float2bfloat16(v);
    }
}

// Gradient of the block form folded back: dRr = d00 + d11, dRi = d10 - d01.
__global__ void k_rbig_fold(const float* drb, float* drr, float* dri, long long nmodes, int O, int C) {
    const long long n = nmodes * (long long)O * C;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long mode = t / ((long long)O * C);
        const int o = (int)((t / C) % O), c = (int)(t % C);
        const float* d = drb + mode * 4LL * O * C;
        const float d00 = d[(long long)o * 2 * C + c], d01 = d[(long long)o * 2 * C + C + c];
        const float d10 = d[(long long)(O + o) * 2 * C + c], d11 = d[(long long)(O + o) * 2 * C + C + c];
        drr[t] = d00 + d11;
        dri[t] = d10 - d01;
    }
}

// ------------------------------------------------- tensor-core dense layer
// z[m][n] = sum_k A(m,k) x[k][n] + bias[m],  h = GELU(z) or z,  for the
// pointwise channel mixes (M, K <= 128 channels, n over all B*N*N points).
// A(m,k) = W[m*K+k] (or W[k*M+m] when transposed), BF16; x is FP32 and is
// rounded to BF16 on its way into shared memory; accumulation is FP32 in
// tensor memory.  One CTA (4 warps) per 256 columns of n:
//   - warp 0 allocates 256 TMEM columns (the 128 x 256 FP32 accumulator);
//   - all threads stage A (K-major) and the x tile (N-major) in shared memory
//     in the 8x8 core-matrix layout without swizzle;
//   - thread 0 issues one tcgen05.mma (kind::f16, M=128, N=256, K=16) per 16
//     channels and commits to an mbarrier;
//   - each warp reads its 32 accumulator lanes with tcgen05.ld, adds the
//     bias, applies GELU and stores rows of z and h.
// The mbarrier wait is bounded; on expiry the CTA sets *err and skips its
// stores (the accumulator is freed either way).
namespace tc {
// columns of n per CTA (accumulator width); the TMEM it takes (TN columns
// of 512) bounds the CTAs resident per SM
#ifndef FNO_DENSE_TN
#define FNO_DENSE_TN 128
#endif
constexpr int TN = FNO_DENSE_TN;
constexpr int TM = 128;      // accumulator rows (M padded)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle): start, leading and stride
// byte offsets in 16-byte units, version 1 at bits 46-47.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: F32 accumulator, BF16 A and B, A K-major, B N-major,
// N = TN, M = TM.
__host__ __device__ constexpr uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (0u << 15) | (1u << 16) | ((uint32_t)(TN >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
}
}  // namespace tc

__global__ void __launch_bounds__(128, 1)
k_dense_tc(const __nv_bfloat16* __restrict__ W, int transw, const float* __restrict__ x, const float* __restrict__ bias,
           float* __restrict__ z, float* __restrict__ h, int M, int K, long long BS, int act, int* err) {
    using namespace tc;
    extern __shared__ __align__(1024) unsigned char smraw[];
    const int KP = (K + 15) / 16 * 16;
    // 1024-byte aligned operand tiles
    const uint32_t base = smem_u32(smraw);
    const uint32_t pad = (1024u - (base & 1023u)) & 1023u;
    unsigned char* sA = smraw + pad;                          // TM x KP bf16, K-major cores
    unsigned char* sB = sA + (size_t)TM * KP * 2;              // KP x TN bf16, N-major cores
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long n0 = (long long)blockIdx.x * TN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // A: element (m, k) -> core (k/8, m/8), row m%8, column k%8
    for (int e = tid; e < TM * KP; e += 128) {
        const int m = e / KP, k = e - (e / KP) * KP;
        __nv_bfloat16 v = __float2bfloat16(0.f);
        if (m < M && k < K) v = transw ? W[(size_t)k * M + m] : W[(size_t)m * K + k];
        const int off = (((k >> 3) * (TM / 8) + (m >> 3)) << 7) + ((m & 7) << 4) + ((k & 7) << 1);
        *(__nv_bfloat16*)(sA + off) = v;
    }
    // B: eight consecutive n of one k -> 16 bytes of core (k/8, n/8), row k%8
    for (int e = tid; e < KP * (TN / 8); e += 128) {
        const int k = e / (TN / 8), g = e - (e / (TN / 8)) * (TN / 8);
        const long long n = n0 + g * 8;
        float f[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) f[j] = 0.f;
        if (k < K) {
            const float* src = x + (size_t)k * BS + n;
            if (n + 8 <= BS && ((((size_t)k * BS + n) & 3) == 0)) {
                const float4 a = *(const float4*)src, b = *(const float4*)(src + 4);
                f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w; f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) f[j] = (n + j < BS) ? src[j] : 0.f;
            }
        }
        __nv_bfloat162 p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) p[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
        const int off = (((k >> 3) * (TN / 8) + g) << 7) + ((k & 7) << 4);
        *(uint4*)(sB + off) = *(uint4*)p;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (tid == 0) {
        const uint32_t idesc = idesc_bf16();
        for (int s = 0; s < KP / 16; ++s) {
            // K-major A: K chunks TM/8 cores apart, 8-row groups 128 B apart
            const uint64_t da = sdesc(smem_u32(sA) + s * 2 * (TM / 8) * 128, (TM / 8) * 128, 128);
            // N-major B: k groups TN/8 cores apart, 8-column groups 128 B apart
            const uint64_t db = sdesc(smem_u32(sB) + s * 2 * (TN / 8) * 128, (TN / 8) * 128, 128);
            const uint32_t acc = s > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(&mbar)));
    }
    // bounded wait for the accumulator (phase 0)
    uint32_t done = 0;
    for (long long it = 0; it < (1LL << 22) && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(&mbar)), "r"(0));
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done) {
        if (lane == 0) atomicExch(err, 1);
    } else {
        const int m = warp * 32 + lane;
        const float bm = (bias && m < M) ? bias[m] : 0.f;
        for (int cb = 0; cb < TN / 16; ++cb) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < M) {
                float v[16], g[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    v[j] = __uint_as_float(r[j]) + bm;
                    g[j] = act ? gelu_f(v[j]) : v[j];
                }
                const long long nb = n0 + cb * 16;
                const size_t row = (size_t)m * BS + nb;
                if (nb + 16 <= BS && (row & 3) == 0) {
                    // each thread owns 64 contiguous bytes of its row
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (z) *(float4*)(z + row + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                        if (h) *(float4*)(h + row + 4 * q) = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
                    }
                } else {
                    for (int j = 0; j < 16; ++j) {
                        if (nb + j < BS) {
                            if (z) z[row + j] = v[j];
                            if (h) h[row + j] = g[j];
                        }
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
}

}  // namespace fno
