// fgpe_persist.cuh -- the persistent batch kernel: one launch advances every
// q2D instance of a batch (all grid sizes with size-specialised transforms,
// one spin and precision) by K whole split steps.
//
// Work items.  Per step the items are the column tiles of every instance
// (F_y, pending scale + KE + SOC, F_y^-1 over TX adjacent x positions) and
// then the row chunks of every instance (each a few tiles of R x lines:
// F_x^-1, SE, SP, NORMC partials, F_x).  Blocks take item tickets from one
// atomic counter, in that order, step after step, until all K steps are
// handed out.  Per instance, device counters order the work:
//   col_done[i]  column tiles finished (over the whole launch),
//   row_done[i]  row chunks finished,
//   fin[i]       steps whose NORMC, scales and info are published.
// A column tile of step s waits for fin[i] >= s; a row chunk of step s waits
// for col_done[i] >= (s+1) * column tiles.  The block that finishes the last
// row chunk of an instance's step reduces its chunk partials in a fixed
// order, publishes NORMC and the next scales (as the last block of the
// single-instance row pass does), then advances fin[i].
//
// Why this cannot deadlock: a block waits only on items with smaller tickets
// and holds no other unfinished item while it waits, and tickets are taken by
// running blocks in increasing order; so the unfinished item with the
// smallest ticket never waits on anything unfinished.  Blocks need not be
// co-resident.  Every wait is still bounded (wait_ns of device time): on
// expiry the block records an error code and the item it waited on and
// leaves; every other block sees the code at its next ticket or wait and
// leaves too, so a launch always ends and the host reports the error.
//
// Coherence.  Data that one block writes and another reads in the same
// launch (tiles of S, the scales and SIG in info, NORMC partials) is read
// through L2 only (cp.async.cg, ld.global.cg): an SM's L1 is not coherent
// with other SMs' writes inside a launch.  Producers fence before they
// count; consumers poll with ld.acquire.
#pragma once
#include <algorithm>

#include "fgpe_kernels.cuh"
#include "fgpe_group.cuh"

namespace fgpe {

// One instance of a persistent batch.
struct PInst {
    InstDesc d;          // constants, state buffers, info, NORMC partial slots
    const int* fy;       // y position -> frequency map of the kernel's y plan
    int col_tiles;       // x positions / TX
    int row_tiles;       // y rows / R
    int chunk;           // row tiles per row item (divides row_tiles)
};

enum { PCTL_TICKET = 0, PCTL_ERR = 1, PCTL_WHERE = 2, PCTL_STEP = 3, PCTL_LEN = 4 };
enum { PERR_NONE = 0, PERR_WAIT_COL = 1, PERR_WAIT_ROW = 2 };

struct PersistArgs {
    const PInst* inst;
    const unsigned* items;   // per step: ncol column items, then nrow row items: (instance << 16) | index
    int ncol, nrow;          // items per step
    int nsteps;
    unsigned* sync;          // [3][ninst]: col_done, row_done, fin (zero at launch)
    unsigned* ctl;           // PCTL_*: ticket, error code, item waited on, its step (zero at launch)
    long long wait_ns;       // bound on one wait, in ns of %globaltimer
    int ninst;
    int stall;               // tests: this instance's first row wait targets a count never reached (-1: none)
};

// Tile shape of a kernel variant for line length N.
__host__ __device__ constexpr int pow2_floor(int v) {
    int p = 1;
    while (2 * p <= v) p *= 2;
    return p;
}
// Rows per row tile: R*N about RN values, R a power of two.
__host__ __device__ constexpr int prow_r(int rn, int n) { return rn / n >= 1 ? pow2_floor(rn / n) : 1; }
// x positions per column tile: TXB bytes of each line element.
template <typename T> __host__ __device__ constexpr int pcol_tx(int txb) { return txb / (int)sizeof(cx<T>); }

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Thread 0: wait until *p >= target, at most wait_ns; false on expiry (error
// recorded) or when another block has recorded an error.
static __device__ bool pwait(const unsigned* p, unsigned target, const PersistArgs& a, unsigned code, unsigned item,
                      unsigned step) {
    if (ld_acquire_u32(p) >= target) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        __nanosleep(128);
        if (ld_acquire_u32(p) >= target) return true;
        if (*(volatile unsigned*)&a.ctl[PCTL_ERR] != 0u) return false;
        if ((long long)(global_ns() - t0) > a.wait_ns) {
            if (atomicCAS(&a.ctl[PCTL_ERR], 0u, code) == 0u) {
                a.ctl[PCTL_WHERE] = item;
                a.ctl[PCTL_STEP] = step;
            }
            __threadfence();
            return false;
        }
    }
}

// After a block's global writes: make them visible, then count the item.
__device__ __forceinline__ void psignal(unsigned* ctr) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(ctr, 1u);
}

// Radix passes of more than this many tasks per thread stay rolled: one
// kernel holds the transforms of every line length, under one register cap.
#ifndef FGPE_PERSIST_UNROLL
#define FGPE_PERSIST_UNROLL 1
#endif
constexpr int kPUnroll = FGPE_PERSIST_UNROLL;

// ------------------------------------------------------------ column tile
// F_y, pending scale + KE + SOC, F_y^-1 on TX adjacent x positions of one
// instance (the arithmetic of k_col_group, with the y plan PV).
template <typename T, int MS, int N, int TX, int TH, int PV>
__device__ __forceinline__ void pcol_tile(const PInst& P, const StepConst& c, int x0, cx<T>* cur) {
    using CT = ColTile<N, TX>;
    constexpr int LPN = CT::LPN;
    constexpr int EPC = 16 / (int)sizeof(cx<T>);
    static_assert(TX % EPC == 0, "column tile narrower than a 16-byte chunk");
    constexpr int CPL = TX / EPC;
    constexpr int NCH = MS * N * CPL;
    const long long np = c.npts;
    const long long stride = c.nx;
    cx<T>* S = (cx<T>*)P.d.S;
    #pragma unroll 1
    for (int ch = threadIdx.x; ch < NCH; ch += TH) {
        const int tc = (ch % CPL) * EPC;
        const int q = ch / CPL;
        const int e = q % N, m = q / N;
        cp16(cur + (m * LPN + e + (e >> 3)) * TX + tc, S + (size_t)m * np + x0 + (size_t)e * stride + tc);
    }
    cp_commit();
    // this step's pending scales, published by another block: read through L2
    const double cfac = 1.0 / (double)c.npts;
    T fac[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) fac[m] = (T)(__ldcg(P.d.info + INFO_SC + m) * cfac);
    cp_wait<0>();
    __syncthreads();
    const cx<T>* tw = (const cx<T>*)c.twy;
    ct_fft<T, false, N, MS * TX, TH, CT, 0, 0, PV, kPUnroll>(cur, tw);
    #pragma unroll 1
    for (int p = threadIdx.x; p < N * TX; p += TH) {
        const int tt = p % TX, e = p / TX;
        const int ix = c.fx[x0 + tt], iy = P.fy[e];
        cx<T> v[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) v[m] = cscale(cur[(m * LPN + e + (e >> 3)) * TX + tt], fac[m]);
        apply_ke<T, MS>(c, ix, iy, 0, v);
        apply_soc<T, MS>(c, c.kx[ix], c.ky[iy], v);
#pragma unroll
        for (int m = 0; m < MS; ++m) cur[(m * LPN + e + (e >> 3)) * TX + tt] = v[m];
    }
    __syncthreads();
    ct_fft<T, true, N, MS * TX, TH, CT, 0, 0, PV, kPUnroll>(cur, tw);
    #pragma unroll 1
    for (int idx = threadIdx.x; idx < MS * N * TX; idx += TH) {
        const int tt = idx % TX, q = idx / TX, e = q % N, m = q / N;
        S[(size_t)m * np + x0 + (size_t)e * stride + tt] = cur[(m * LPN + e + (e >> 3)) * TX + tt];
    }
    __syncthreads();
}

// --------------------------------------------------------------- row tile
// F_x^-1, SE, SP, NORMC partials (into acc), snapshot, F_x on R x lines of
// one instance (the arithmetic of k_row_group).
template <typename T, int MS, int N, int R, int TH>
__device__ __forceinline__ void prow_tile(const PInst& P, const StepConst& c, int lt, int snap, cx<T>* cur,
                                          double (&acc)[MS]) {
    using RT = RowTile<N, MS * R>;
    constexpr int LP = RT::LP;
    constexpr int NCH = MS * R * N;
    const long long np = c.npts;
    cx<T>* S = (cx<T>*)P.d.S;
    const int row0 = lt * R;
    if constexpr (sizeof(cx<T>) == 16) {
        #pragma unroll 1
        for (int ch = threadIdx.x; ch < NCH; ch += TH) {
            const int x = ch % N, q = ch / N, r = q % R, m = q / R;
            cp16(cur + (m * R + r) * LP + x + (x >> 3), S + (size_t)m * np + (size_t)(row0 + r) * N + x);
        }
        cp_commit();
        cp_wait<0>();
    } else {
        // complex64: two elements per 16-byte L2 load (x even, so x and x + 1
        // share one padding group; the padded layout leaves no 16-byte
        // aligned destination for cp.async)
        #pragma unroll 1
        for (int ch = threadIdx.x; ch < NCH / 2; ch += TH) {
            const int x = (ch % (N / 2)) * 2, q = ch / (N / 2), r = q % R, m = q / R;
            const float4 v = __ldcg((const float4*)(S + (size_t)m * np + (size_t)(row0 + r) * N + x));
            cx<T>* d = cur + (m * R + r) * LP + x + (x >> 3);
            d[0] = mk<T>(v.x, v.y);
            d[1] = mk<T>(v.z, v.w);
        }
    }
    __syncthreads();
    const cx<T>* twx = (const cx<T>*)c.twx;
    cx<T>* sn = snap == 1 ? (cx<T>*)P.d.psi : snap == 2 ? (cx<T>*)P.d.prev : nullptr;
    ct_fft<T, true, N, MS * R, TH, RT, 0, 0, 0, kPUnroll>(cur, twx);
    #pragma unroll 1
    for (int p = threadIdx.x; p < R * N; p += TH) {
        const int x = p % N, r = p / N;
        const int row = row0 + r;
        const int j = row % c.ny, kk = row / c.ny;
        cx<T> v[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) v[m] = cur[(m * R + r) * LP + x + (x >> 3)];
        const cx<T> eV = pot_phase<T>(c, x, j, kk);
        apply_se<T, MS>(c, v);
        apply_sp<T, MS>(c, eV, v);
        const double w = c.wx[x] * c.wy[j];
#pragma unroll
        for (int m = 0; m < MS; ++m) {
            acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
            cur[(m * R + r) * LP + x + (x >> 3)] = v[m];
        }
        if (sn) {
#pragma unroll
            for (int m = 0; m < MS; ++m) sn[(size_t)m * np + (size_t)row * N + x] = v[m];
        }
    }
    __syncthreads();
    ct_fft<T, false, N, MS * R, TH, RT, 0, 0, 0, kPUnroll>(cur, twx);
    #pragma unroll 1
    for (int idx = threadIdx.x; idx < MS * R * N; idx += TH) {
        const int x = idx % N, q = idx / N, r = q % R, m = q / R;
        S[(size_t)m * np + (size_t)(row0 + r) * N + x] = cur[(m * R + r) * LP + x + (x >> 3)];
    }
    __syncthreads();
}

// ------------------------------------------------------------- row item
// A chunk of row tiles of one instance, then its NORMC partial; the block
// that completes the instance's step reduces the partials in chunk order,
// publishes norms, scales and SIG (and, before the last step, the info copy
// of the CONV snapshot), then advances fin[inst].
template <typename T, int MS, int N, int R, int TH>
__device__ void prow_item(const PersistArgs& a, const PInst& P, const StepConst& c, int inst, int chunk, int step,
                          int snap, cx<T>* cur, double* red, double* bsum) {
    __shared__ int is_last;
    double acc[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) acc[m] = 0.0;
    for (int k = 0; k < P.chunk; ++k) prow_tile<T, MS, N, R, TH>(P, c, chunk * P.chunk + k, snap, cur, acc);
    block_sum<MS>(acc, red, bsum);
    if (threadIdx.x < MS) P.d.part[(size_t)chunk * MS + threadIdx.x] = bsum[threadIdx.x];
    const unsigned nchunks = (unsigned)(P.row_tiles / P.chunk);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        is_last = atomicAdd(&a.sync[a.ninst + inst], 1u) == (unsigned)(step + 1) * nchunks - 1u;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
#pragma unroll
    for (int m = 0; m < MS; ++m) acc[m] = 0.0;
    for (unsigned b = threadIdx.x; b < nchunks; b += TH) {
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] += __ldcg(P.d.part + (size_t)b * MS + m);
    }
    block_sum<MS>(acc, red, red + 32 * MS);
    if (threadIdx.x == 0) {
        double* info = P.d.info;
        double tot = 0, n[MS], sc[MS], sig[2];
        for (int m = 0; m < MS; ++m) { n[m] = red[32 * MS + m]; tot += n[m]; info[INFO_NORM + m] = n[m]; }
        info[INFO_TOTAL] = tot;
        if (c.sink) {
            volatile unsigned* ctr = c.sink_ctr;
            const unsigned k = *ctr;
            *ctr = k + 1u;
            double* d = c.sink + (size_t)(k % (unsigned)c.sink_n) * MS;
            for (int m = 0; m < MS; ++m) d[m] = n[m];
        }
        sig[0] = __ldcg(info + INFO_SIG);
        sig[1] = __ldcg(info + INFO_SIG + 1);
        const int rc = compute_scales<MS>(c, n, sig, sc);
        info[INFO_SIG] = sig[0];
        info[INFO_SIG + 1] = sig[1];
        bool bad = !(tot == tot) || !(tot < 1e300);
        for (int m = 0; m < MS; ++m) { info[INFO_SC + m] = sc[m]; bad = bad || !(sc[m] == sc[m]); }
        if (bad) info[INFO_ERR] = 1.0;
        if (rc) info[INFO_ERR] = (double)rc;
        if (snap == 2)
            for (int i = 0; i < INFO_LEN; ++i) P.d.info_prev[i] = __ldcg(info + i);
        __threadfence();
        atomicExch(&a.sync[2 * a.ninst + inst], (unsigned)(step + 1));
    }
    __syncthreads();
}

// ---------------------------------------------------------------- kernel
// Variant <TH threads, RN values per row tile, TXB bytes per column tile
// row, PV y plan>: the shape the autotuner picks per batch.
#define FGPE_PSIZES(CALL) CALL(128) CALL(192) CALL(256) CALL(384) CALL(512)

template <typename T, int MS, int TH, int RN, int TXB, int PV>
__global__ void __launch_bounds__(TH, 2) k_persist(PersistArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* cur = (cx<T>*)smraw;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    __shared__ StepConst c;
    __shared__ unsigned s_ticket;
    __shared__ int s_ok;
    const unsigned per = (unsigned)(a.ncol + a.nrow);
    const unsigned total = per * (unsigned)a.nsteps;
    int cur_inst = -1;
    for (;;) {
        if (threadIdx.x == 0)
            s_ticket = *(volatile unsigned*)&a.ctl[PCTL_ERR] ? total : atomicAdd(&a.ctl[PCTL_TICKET], 1u);
        __syncthreads();
        const unsigned t = s_ticket;
        if (t >= total) break;
        const int step = (int)(t / per);
        const unsigned r = t - (unsigned)step * per;
        const bool col = r < (unsigned)a.ncol;
        const unsigned e = a.items[r];
        const int inst = (int)(e >> 16), idx = (int)(e & 0xffffu);
        const PInst& P = a.inst[inst];
        if (threadIdx.x == 0) {
            bool ok;
            if (col) {
                ok = pwait(&a.sync[2 * a.ninst + inst], (unsigned)step, a, PERR_WAIT_COL, t, (unsigned)step);
            } else {
                unsigned target = (unsigned)(step + 1) * (unsigned)P.col_tiles;
                if (inst == a.stall && step == 0) target = 0xffffffffu;
                ok = pwait(&a.sync[inst], target, a, PERR_WAIT_ROW, t, (unsigned)step);
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) break;
        if (inst != cur_inst) {
            load_const(c, P.d.c);
            cur_inst = inst;
            __syncthreads();
        }
        if (col) {
            switch (c.ny) {
#define PCOL(NN) \
                case NN: pcol_tile<T, MS, NN, pcol_tx<T>(TXB), TH, PV>(P, c, idx * pcol_tx<T>(TXB), cur); break;
                FGPE_PSIZES(PCOL)
#undef PCOL
                default: break;
            }
            psignal(&a.sync[inst]);
        } else {
            const int snap = step == a.nsteps - 1 ? 1 : (step == a.nsteps - 2 ? 2 : 0);
            switch (c.nx) {
#define PROW(NN) \
                case NN: prow_item<T, MS, NN, prow_r(RN, NN), TH>(a, P, c, inst, idx, step, snap, cur, red, bsum); break;
                FGPE_PSIZES(PROW)
#undef PROW
                default: break;
            }
        }
    }
}

// Shared memory of variant <RN, TXB> for the sizes present (bit i of mask:
// size i of 128, 192, 256, 384, 512 on either axis).
template <typename T, int MS>
inline size_t persist_smem(int rn, int txb, int nmask) {
    const int ns[5] = {128, 192, 256, 384, 512};
    size_t s = 0;
    for (int i = 0; i < 5; ++i) {
        if (!(nmask >> i & 1)) continue;
        const size_t row = (size_t)MS * prow_r(rn, ns[i]) * cpad(ns[i]) * sizeof(cx<T>);
        const size_t col = (size_t)MS * cpad(ns[i]) * pcol_tx<T>(txb) * sizeof(cx<T>);
        s = std::max(s, std::max(row, col));
    }
    return s;
}

}  // namespace fgpe
