// fno_gemm_tc.cuh -- the learned guess's strided batched GEMM on the tensor
// cores (tcgen05), for the spectral layers: the truncated DFTs onto and off
// the retained modes, the per-mode channel mixing, and their backward and
// weight-gradient products.
//
//   C[b](i,j) = alpha * sum_k A[b](i,k) B[b](k,j) + beta * C[b](i,j)
//
// The same contract as k_gemm (element (i,k) of A[b] at A + b*sAb + i*sAi +
// k*sAk, likewise B and C), with FP32 operands carried at about 16
// significant bits: each FP32 operand is split into a BF16 head and a BF16
// tail (v = hi + lo, lo = bf16(v - hi)), and a tile accumulates
// hi*hi + hi*lo + lo*hi in FP32 in tensor memory (the lo*lo term, about
// 2^-16 of the product, is dropped).  A BF16 operand (the channel-mixing
// weights) has no tail, so those tiles take two products per K step.
//
// Tiles are 128 rows (the accumulator's TMEM lanes) by GN columns (16 to 256,
// chosen from N).  With B shared by every batch entry (sBb == 0) the rows of
// all entries form one M dimension ("fold"), so a stage of many small
// products, such as one DFT matrix applied to thousands of channel planes,
// becomes one tall GEMM.  A CTA (4 warps) is persistent over tiles:
//   - all threads stage a 64-deep K slice of A (K-major 8x8 core matrices)
//     and of B (N-major core matrices), head and tail, in shared memory;
//   - thread 0 issues the tcgen05.mma (kind::f16, M = 128, N = GN, K = 16)
//     of the slice and commits to an mbarrier, which every thread waits on
//     (bounded) before the slice's buffers are refilled;
//   - each warp reads its 32 accumulator lanes (tcgen05.ld) and writes its
//     rows of C.
// If a wait runs out, the CTA sets *err, stops issuing, and frees its TMEM.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fno {

struct GemmTc {
    int M, N, K;        // per batch entry
    int batch, fold;    // fold: the rows of all entries form one M dimension
    float alpha, beta;
    const void* A;
    long long sAb, sAi, sAk;
    const float* B;
    long long sBb, sBk, sBj;
    float* C;
    long long sCb, sCi, sCj;
    int* err;
    int avec;           // 1: FP32 A read as float4 along K (contiguous, 16-byte aligned rows)
    int bvec;           // 1: B read as float4 along N; 2: along K (likewise)
    int cvec;           // 1: C rows contiguous along N on 16-byte boundaries (float4 epilogue)
};

namespace gtc {
constexpr int TM = 128;   // tile rows = accumulator lanes
constexpr int KC = 64;    // K slice staged per round (four K = 16 products)
constexpr int LB = 16;    // loads in flight per thread while staging

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor without swizzle: start address, leading
// and stride byte offsets in 16-byte units, descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: F32 accumulator (bit 4), BF16 A and B (bits 7, 10),
// A K-major (bit 15 clear), B N-major (bit 16), N / 8 at bit 17, M / 16 at 24.
template <int GN> __host__ __device__ constexpr uint32_t idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(GN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

template <int GN> constexpr int tmem_cols() { return GN < 32 ? 32 : GN; }

// bytes of one operand copy (head or tail) of a K slice
constexpr int a_bytes() { return TM * KC * 2; }
template <int GN> constexpr int b_bytes() { return KC * GN * 2; }
template <int GN> constexpr size_t smem_bytes() { return 1024 + 2 * (size_t)a_bytes() + 2 * (size_t)b_bytes<GN>(); }

// element (m, k) of a K-major A slice: core matrix (k/8, m/8), row m%8, column k%8
__device__ __forceinline__ int a_off(int m, int k) { return (((k >> 3) * (TM / 8) + (m >> 3)) << 7) + ((m & 7) << 4) + ((k & 7) << 1); }
// element (k, n) of an N-major B slice: core matrix (k/8, n/8), row k%8, column n%8
template <int GN> __device__ __forceinline__ int b_off(int k, int n) {
    return (((k >> 3) * (GN / 8) + (n >> 3)) << 7) + ((k & 7) << 4) + ((n & 7) << 1);
}

__device__ __forceinline__ float ld_any(const float* p) { return *p; }
__device__ __forceinline__ float ld_any(const __nv_bfloat16* p) { return __bfloat162float(*p); }

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// four consecutive elements of one core-matrix row (8 bytes): head and tail
__device__ __forceinline__ void put4(unsigned char* h, unsigned char* l, int off, float4 v) {
    __nv_bfloat16 hi[4], lo[4];
    split_bf16(v.x, hi[0], lo[0]);
    split_bf16(v.y, hi[1], lo[1]);
    split_bf16(v.z, hi[2], lo[2]);
    split_bf16(v.w, hi[3], lo[3]);
    *(uint2*)(h + off) = *(const uint2*)hi;
    *(uint2*)(l + off) = *(const uint2*)lo;
}

__device__ __forceinline__ void mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(id), "r"(acc));
}

// bounded wait on an mbarrier phase; 1 if it completed
__device__ __forceinline__ int wait_phase(uint32_t bar, uint32_t parity) {
    uint32_t done = 0;
    for (long long it = 0; it < (1LL << 22) && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity));
    }
    return (int)done;
}
}  // namespace gtc

template <typename TA, int GN>
__global__ void __launch_bounds__(128, 1) k_gemm_tc(GemmTc g) {
    using namespace gtc;
    using bf16 = __nv_bfloat16;
    constexpr bool A_SPLIT = sizeof(TA) == 4;
    extern __shared__ __align__(1024) unsigned char smraw[];
    const uint32_t base = smem_u32(smraw);
    const uint32_t pad = (1024u - (base & 1023u)) & 1023u;   // 1024-byte aligned operand slices
    unsigned char* sAh = smraw + pad;
    unsigned char* sAl = sAh + a_bytes();
    unsigned char* sBh = sAl + a_bytes();
    unsigned char* sBl = sBh + b_bytes<GN>();
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ long long rowA[TM], rowC[TM];   // element offsets of the tile's rows (-1: past the end)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TA* A = (const TA*)g.A;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(tmem_cols<GN>()));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    const long long rows = g.fold ? (long long)g.batch * g.M : (long long)g.M;
    const long long mt = (rows + TM - 1) / TM;
    const long long nt = (g.N + GN - 1) / GN;
    const long long ntiles = mt * nt * (g.fold ? 1 : g.batch);
    uint32_t phase = 0;
    bool ok = true;
    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long bq = tile / (mt * nt);          // batch entry (0 when folded)
        const long long rem = tile - bq * (mt * nt);
        const long long m0 = (rem / nt) * TM;
        const int n0 = (int)(rem % nt) * GN;
        {
            const long long r = m0 + tid;
            long long oa = -1, oc = -1;
            if (r < rows) {
                const long long eb = g.fold ? r / g.M : bq;
                const long long ei = g.fold ? r - eb * g.M : r;
                oa = eb * g.sAb + ei * g.sAi;
                oc = eb * g.sCb + ei * g.sCi;
            }
            rowA[tid] = oa;
            rowC[tid] = oc;
        }
        const long long bofs = g.fold ? 0 : bq * g.sBb;
        __syncthreads();
        for (int k0 = 0; k0 < g.K && ok; k0 += KC) {
            // K extent staged this round, a multiple of 16 (the products read
            // no further): short K (the retained modes) stages only its columns
            const int kx = min(KC, (g.K - k0 + 15) / 16 * 16);
            const int kx4 = kx / 4;
            if (A_SPLIT && g.avec) {
                // A rows as float4 along K: 16 consecutive threads read one
                // row's 256-byte slice; 8 vectors in flight per thread
#pragma unroll 1
                for (int e0 = 0; e0 < TM * kx4; e0 += 128 * 8) {
                    float4 v[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int e = min(e0 + tid + j * 128, TM * kx4 - 1);
                        const int m = e / kx4, kq = (e % kx4) * 4;
                        const long long oa = rowA[m];
                        const float* src = (const float*)A + oa + k0 + kq;
                        if (oa >= 0 && k0 + kq + 3 < g.K) {
                            v[j] = *(const float4*)src;
                        } else {
                            v[j].x = (oa >= 0 && k0 + kq < g.K) ? src[0] : 0.f;
                            v[j].y = (oa >= 0 && k0 + kq + 1 < g.K) ? src[1] : 0.f;
                            v[j].z = (oa >= 0 && k0 + kq + 2 < g.K) ? src[2] : 0.f;
                            v[j].w = 0.f;
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int e = e0 + tid + j * 128;
                        if (e < TM * kx4) {
                            const int m = e / kx4, kq = (e % kx4) * 4;
                            put4(sAh, sAl, a_off(m, kq), v[j]);
                        }
                    }
                }
            } else {
                // A slice, walking the contiguous index fastest across threads;
                // each thread issues LB independent loads before it converts and
                // stores them (the loads' latency overlaps)
                const bool akf = g.sAk == 1;
#pragma unroll 1
                for (int e0 = 0; e0 < TM * kx; e0 += 128 * LB) {
                    float v[LB];
#pragma unroll
                    for (int j = 0; j < LB; ++j) {
                        const int e = min(e0 + tid + j * 128, TM * kx - 1);   // TM*kx is a multiple of 128*LB
                        const int m = akf ? e / kx : e % TM, k = akf ? e % kx : e / TM;
                        const long long oa = rowA[m];
                        v[j] = (oa >= 0 && k0 + k < g.K) ? ld_any(A + oa + (long long)(k0 + k) * g.sAk) : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < LB; ++j) {
                        const int e = e0 + tid + j * 128;
                        if (e >= TM * kx) continue;
                        const int m = akf ? e / kx : e % TM, k = akf ? e % kx : e / TM;
                        const int off = a_off(m, k);
                        if (A_SPLIT) {
                            bf16 hi, lo;
                            split_bf16(v[j], hi, lo);
                            *(bf16*)(sAh + off) = hi;
                            *(bf16*)(sAl + off) = lo;
                        } else {
                            *(bf16*)(sAh + off) = __float2bfloat16_rn(v[j]);   // exact: v came from BF16
                        }
                    }
                }
            }
            if (g.bvec) {
                // B as float4 along N (bvec 1) or along K (bvec 2)
                const bool nvec = g.bvec == 1;
                const int NV = kx * GN / 4;
#pragma unroll 1
                for (int e0 = 0; e0 < NV; e0 += 128 * 8) {
                    float4 v[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int e = e0 + tid + j * 128;
                        v[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (e < NV) {
                            const int k = nvec ? e / (GN / 4) : (e % kx4) * 4;
                            const int n = nvec ? (e % (GN / 4)) * 4 : e / kx4;
                            const float* src = g.B + bofs + (long long)(k0 + k) * g.sBk + (long long)(n0 + n) * g.sBj;
                            const int lim = nvec ? (k0 + k < g.K ? g.N - (n0 + n) : 0) : (n0 + n < g.N ? g.K - (k0 + k) : 0);
                            // the vector runs along the unit-stride index
                            if (lim >= 4) {
                                v[j] = *(const float4*)src;
                            } else {
                                if (lim > 0) v[j].x = src[0];
                                if (lim > 1) v[j].y = src[1];
                                if (lim > 2) v[j].z = src[2];
                            }
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int e = e0 + tid + j * 128;
                        if (e < NV) {
                            if (nvec) {
                                const int k = e / (GN / 4), nq = (e % (GN / 4)) * 4;
                                put4(sBh, sBl, b_off<GN>(k, nq), v[j]);
                            } else {
                                const int kq = (e % kx4) * 4, n = e / kx4;
                                const float f[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    bf16 hi, lo;
                                    split_bf16(f[q], hi, lo);
                                    const int off = b_off<GN>(kq + q, n);
                                    *(bf16*)(sBh + off) = hi;
                                    *(bf16*)(sBl + off) = lo;
                                }
                            }
                        }
                    }
                }
            } else {
                // B slice
                const bool bnf = g.sBj == 1;
#pragma unroll 1
                for (int e0 = 0; e0 < kx * GN; e0 += 128 * LB) {
                    float v[LB];
#pragma unroll
                    for (int j = 0; j < LB; ++j) {
                        const int e = e0 + tid + j * 128;
                        const int n = bnf ? e % GN : e / kx, k = bnf ? e / GN : e % kx;
                        v[j] = (e < kx * GN && k0 + k < g.K && n0 + n < g.N)
                                   ? g.B[bofs + (long long)(k0 + k) * g.sBk + (long long)(n0 + n) * g.sBj]
                                   : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < LB; ++j) {
                        const int e = e0 + tid + j * 128;
                        if (e < kx * GN) {
                            const int n = bnf ? e % GN : e / kx, k = bnf ? e / GN : e % kx;
                            bf16 hi, lo;
                            split_bf16(v[j], hi, lo);
                            const int off = b_off<GN>(k, n);
                            *(bf16*)(sBh + off) = hi;
                            *(bf16*)(sBl + off) = lo;
                        }
                    }
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (tid == 0) {
                const uint32_t id = idesc<GN>();
                const int ks = min(KC / 16, (g.K - k0 + 15) / 16);
                for (int s = 0; s < ks; ++s) {
                    // K-major A: the two K halves of a step TM/8 cores apart, row groups 128 B apart;
                    // N-major B: the two K halves GN/8 cores apart, column groups 128 B apart
                    const uint32_t ao = (uint32_t)s * 2 * (TM / 8) * 128, bo = (uint32_t)s * 2 * (GN / 8) * 128;
                    const uint64_t dah = sdesc(smem_u32(sAh) + ao, (TM / 8) * 128, 128);
                    const uint64_t dbh = sdesc(smem_u32(sBh) + bo, (GN / 8) * 128, 128);
                    const uint64_t dbl = sdesc(smem_u32(sBl) + bo, (GN / 8) * 128, 128);
                    mma(tmem, dah, dbh, id, (k0 > 0 || s > 0) ? 1u : 0u);
                    mma(tmem, dah, dbl, id, 1u);
                    if (A_SPLIT) mma(tmem, sdesc(smem_u32(sAl) + ao, (TM / 8) * 128, 128), dbh, id, 1u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&mbar)));
            }
            const int done = wait_phase(smem_u32(&mbar), phase);
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            ok = __syncthreads_and(done) != 0;
        }
        if (!ok) break;
        // epilogue: warp w holds rows 32w..32w+31 of the tile in TMEM lanes
        const long long oc = rowC[warp * 32 + lane];
        for (int cb = 0; cb < GN / 16; ++cb) {
            if (n0 + cb * 16 >= g.N) break;   // uniform across the block
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (oc >= 0) {
                const int nb = n0 + cb * 16;
                float* crow = g.C + oc + (long long)nb * g.sCj;
                float out[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) out[j] = g.alpha * __uint_as_float(r[j]);
                if (g.cvec && nb + 16 <= g.N) {
                    // 64 contiguous bytes of the row: float4 reads and writes
                    float4* c4 = (float4*)crow;
                    if (g.beta != 0.f) {
                        float4 o[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) o[q] = c4[q];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            out[4 * q] += g.beta * o[q].x;
                            out[4 * q + 1] += g.beta * o[q].y;
                            out[4 * q + 2] += g.beta * o[q].z;
                            out[4 * q + 3] += g.beta * o[q].w;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) c4[q] = make_float4(out[4 * q], out[4 * q + 1], out[4 * q + 2], out[4 * q + 3]);
                } else {
                    // all reads of C before any write, so they overlap
                    if (g.beta != 0.f) {
                        float o[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) o[j] = nb + j < g.N ? crow[(long long)j * g.sCj] : 0.f;
#pragma unroll
                        for (int j = 0; j < 16; ++j) out[j] += g.beta * o[j];
                    }
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (nb + j < g.N) crow[(long long)j * g.sCj] = out[j];
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (!ok && tid == 0) atomicExch(g.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols<GN>()));
}

}  // namespace fno
