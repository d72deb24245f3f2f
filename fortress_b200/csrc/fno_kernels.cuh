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

// out[c] = beta*out[c] + sum_{b,s} x[b,c,s]; one block per channel, fixed order.
__global__ void k_channel_sum(float* out, const float* x, long long B, long long C, long long S, float beta) {
    const long long c = blockIdx.x;
    double acc = 0.0;
    for (long long b = 0; b < B; ++b)
        for (long long s = threadIdx.x; s < S; s += blockDim.x) acc += x[(b * C + c) * S + s];
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

}  // namespace fno
