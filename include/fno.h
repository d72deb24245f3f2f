/*
 * fno.h -- C ABI of the kernels that train and evaluate the learned initial
 * guess (a Fourier neural operator mapping physical parameters to a spinor).
 * No counterpart in the reference (FORTRESS starts from fixed analytic
 * guesses, cgpe1d.f90:707-790); the guess it produces feeds fgpe_set_state.
 *
 * All pointers are device pointers; all calls are asynchronous on `stream`
 * (cudaStream_t, NULL = legacy default stream) and return 0 or an FGPE_E_*
 * code.  Tensors are float32 unless stated; weight operands may be bfloat16.
 */
#ifndef FNO_H
#define FNO_H
#ifdef __cplusplus
extern "C" {
#endif

/* Batched strided GEMM with FP32 accumulation:
 *   C[b](i,j) = alpha * sum_k A[b](i,k) B[b](k,j) + beta * C[b](i,j)
 * with A[b](i,k) at A + b*sAb + i*sAi + k*sAk (elements; likewise B, C).
 * a_bf16 != 0: A holds bfloat16 values. */
int fno_gemm(int batch, int M, int N, int K, float alpha, const void *A, int a_bf16, long long sAb,
             long long sAi, long long sAk, const float *B, long long sBb, long long sBk, long long sBj,
             float beta, float *C, long long sCb, long long sCi, long long sCj, void *stream);
/* fno_gemm on the tensor cores (tcgen05.mma, FP32 accumulation in tensor
 * memory): each FP32 operand is split into a bfloat16 head and tail and the
 * product keeps hi*hi + hi*lo + lo*hi (about 16 significant bits per
 * operand; a bfloat16 A is exact).  Strides must be >= 0.  When B is shared
 * by all batch entries (sBb == 0), or A is (sAb == 0, taken transposed), the
 * entries' rows form one tall GEMM.  *err_dev (device int) is set to 1 if a
 * CTA's wait for its accumulator ran out. */
int fno_gemm_tc(int batch, int M, int N, int K, float alpha, const void *A, int a_bf16, long long sAb,
                long long sAi, long long sAk, const float *B, long long sBb, long long sBk, long long sBj,
                float beta, float *C, long long sCb, long long sCi, long long sCj, int *err_dev, void *stream);
/* z[b,c,s] += bias[c] (bias may be NULL); h = GELU(z) if act else z (h may be NULL). */
int fno_bias_act(float *z, float *h, const float *bias, long long C, long long S, long long n, int act, void *stream);
/* dz = dh * GELU'(z) */
int fno_act_bwd(float *dz, const float *dh, const float *z, long long n, void *stream);
/* out[c] = beta*out[c] + sum over b and s of x[b,c,s] */
int fno_channel_sum(float *out, const float *x, long long B, long long C, long long S, float beta, void *stream);
/* y += a*x */
int fno_axpy(float *y, const float *x, float a, long long n, void *stream);
/* loss = mean((out-target)^2) into *loss_dev (double, device); dout = d loss/d out (may be NULL);
 * scratch: >= 256 doubles of device memory. */
int fno_mse(const float *out, const float *target, float *dout, double *loss_dev, double *scratch, long long n, void *stream);
/* One Adam step (bias-corrected, step t >= 1) on FP32 master weights w;
 * w_bf16 (may be NULL) receives the bfloat16 copy. */
int fno_adam(float *w, void *w_bf16, const float *g, float *m, float *v, long long n, float lr, float beta1,
             float beta2, float eps, int t, void *stream);
int fno_to_bf16(const float *x, void *y, long long n, void *stream);
/* Dense (pointwise channel-mixing) layer on the tensor cores (tcgen05):
 *   z[m][j] = sum_k A(m,k) x[k][j] + bias[m],  h[m][j] = GELU(z) if act else z,
 * A(m,k) = W[m*K+k] (W[k*M+m] if transpose_w), W bfloat16, x float32 (rounded
 * to bfloat16 for the products), FP32 accumulation; 1 <= M, K <= 128,
 * j < n.  z or h may be NULL (not both); bias may be NULL.  *err_dev (device
 * int) is set to 1 if a CTA's wait for its accumulator ran out. */
int fno_dense_tc(const void *w_bf16, int transpose_w, const float *x, const float *bias, float *z, float *h, int M,
                 int K, long long n, int act, int *err_dev, void *stream);
/* Per-mode complex channel mixing in real block form: from Rr, Ri [mode][O][C]
 * (float) build rbig [mode][2O][2C] = [[Rr,-Ri],[Ri,Rr]] in bfloat16, and fold
 * a gradient of that block form back to dRr = d00 + d11, dRi = d10 - d01. */
int fno_rbig_build(const float *rr, const float *ri, void *rbig_bf16, long long nmodes, int O, int C, void *stream);
int fno_rbig_fold(const float *drbig, float *drr, float *dri, long long nmodes, int O, int C, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FNO_H */
