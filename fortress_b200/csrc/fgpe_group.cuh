// fgpe_group.cuh -- grouped passes: one launch advances every instance of a
// batch that shares a grid shape (q2D, both axes of a size the size-
// specialised kernels cover), instead of one launch per instance.
//
// A group's instances differ in their physics (TAU, GAMMA, ALPHA, DT) and
// state buffers, described per instance by an InstDesc in device memory.  A
// launch walks the tiles of all of them: column tiles are independent; row
// tiles are taken in chunks of consecutive tiles of one instance, each chunk
// adds its NORMC partial to the instance's slot for that chunk, and the
// block that completes an instance's last chunk reduces the slots in a
// fixed order and publishes the norms and next scales (as the last block of
// the single-instance row pass does), so results do not depend on timing.
// The per-tile arithmetic is that of k_row_fast / k_col_fast.
#pragma once
#include "fgpe_fast.cuh"

namespace fgpe {

struct InstDesc {
    StepConst c;
    void* S;            // x-spectral state (in/out)
    void* psi;          // real-space snapshot target of mode 1
    void* prev;         // real-space snapshot target of mode 2
    double* info;       // INFO_* vector
    double* info_prev;  // receives info after a mode-2 step
    double* part;       // NORMC partials, [chunks][MS]
    unsigned* counter;  // chunks finished in the current launch (0 between)
};

struct GroupArgs {
    const InstDesc* d;
    int ninst;
    int tiles;          // tiles per instance
    int chunk;          // row pass: tiles per chunk (divides tiles)
    int snap;           // row pass: 0 none, 1 real-space state to psi, 2 to prev (+ info to info_prev)
};

// The StepConst of the tile's instance, copied into shared memory when the
// instance changes (device functions read it there rather than from global
// memory).  Callers synchronise before using it.
__device__ __forceinline__ void load_const(StepConst& dst, const StepConst& src) {
    const int nw = (int)(sizeof(StepConst) / 4);
    const unsigned* s = (const unsigned*)&src;
    unsigned* d = (unsigned*)&dst;
    for (int i = threadIdx.x; i < nw; i += blockDim.x) d[i] = s[i];
}

// Completion of one instance's NORMC after a chunk has written its slot.
template <int MS>
__device__ void finish_group_norms(const InstDesc& D, const StepConst& c, int nchunk, bool keep_prev,
                                   double* red) {
    __shared__ int is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(D.counter, 1u) == (unsigned)nchunk - 1u);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double acc[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) acc[m] = 0.0;
    for (int b = threadIdx.x; b < nchunk; b += blockDim.x) {
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] += __ldcg(D.part + (size_t)b * MS + m);
    }
    block_sum<MS>(acc, red, red + 32 * MS);
    if (threadIdx.x == 0) {
        double tot = 0, n[MS], sc[MS];
        double* info = D.info;
        for (int m = 0; m < MS; ++m) { n[m] = red[32 * MS + m]; tot += n[m]; info[INFO_NORM + m] = n[m]; }
        info[INFO_TOTAL] = tot;
        sink_norms<MS>(c, n);
        const int rc = compute_scales<MS>(c, n, info + INFO_SIG, sc);
        bool bad = !(tot == tot) || !(tot < 1e300);
        for (int m = 0; m < MS; ++m) { info[INFO_SC + m] = sc[m]; bad = bad || !(sc[m] == sc[m]); }
        if (bad) info[INFO_ERR] = 1.0;
        if (rc) info[INFO_ERR] = (double)rc;
        if (keep_prev)
            for (int i = 0; i < INFO_LEN; ++i) D.info_prev[i] = info[i];
        *D.counter = 0u;
    }
    __syncthreads();
}

// ------------------------------------------------------------ row pass
// ROW_FULL of every instance: tiles of R x-lines, chunks of g.chunk tiles.
template <typename T, int MS, int N, int R, int TH, int NBUF = FGPE_ROW_NBUF>
__global__ void __launch_bounds__(TH, row_minb(TH)) k_row_group(GroupArgs g) {
    using RT = RowTile<N, MS * R>;
    constexpr int LP = RT::LP;
    constexpr int TILE = MS * R * LP;
    constexpr int NCH = MS * R * N;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* bufs = (cx<T>*)smraw;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    __shared__ StepConst c;
    const int nci = g.tiles / g.chunk;            // chunks per instance
    const int nchunks = g.ninst * nci;
    // k-th tile of this block: chunk blockIdx.x + (k / chunk) * gridDim.x
    auto tile_of = [&](int k, int& inst, int& lt) -> bool {
        const int q = k / g.chunk;
        const int chunk = blockIdx.x + q * gridDim.x;
        if (chunk >= nchunks) return false;
        inst = chunk / nci;
        lt = (chunk - inst * nci) * g.chunk + (k - q * g.chunk);
        return true;
    };
    auto issue = [&](int inst, int lt, cx<T>* dst) {
        const InstDesc& D = g.d[inst];
        const cx<T>* src = (const cx<T>*)D.S;
        const long long np = D.c.npts;
        const int row0 = lt * R;
        for (int ch = threadIdx.x; ch < NCH; ch += TH) {
            const int x = ch % N;
            const int q = ch / N;
            const int r = q % R, m = q / R;
            cp_elem<T>(dst + (m * R + r) * LP + x + (x >> 3), src + (size_t)m * np + (size_t)(row0 + r) * N + x);
        }
    };
    double acc[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) acc[m] = 0.0;
    int inst = 0, lt = 0, cur_inst = -1;
    bool have = tile_of(0, inst, lt);
    if (NBUF == 2) {
        if (have) issue(inst, lt, bufs);
        cp_commit();
    }
    for (int k = 0; have; ++k) {
        cx<T>* cur = bufs + (NBUF == 2 ? (k & 1) * TILE : 0);
        int ninst = 0, nlt = 0;
        const bool nxt = tile_of(k + 1, ninst, nlt);
        if (inst != cur_inst) {
            __syncthreads();                       // nobody still reads the old constants
            load_const(c, g.d[inst].c);
            cur_inst = inst;
        }
        if (NBUF == 2) {
            if (nxt) issue(ninst, nlt, bufs + ((k + 1) & 1) * TILE);
            cp_commit();
            cp_wait<1>();
        } else {
            issue(inst, lt, cur);
            cp_commit();
            cp_wait<0>();
        }
        __syncthreads();
        const InstDesc& D = g.d[inst];
        const long long np = c.npts;
        const cx<T>* twx = (const cx<T>*)c.twx;
        const int row0 = lt * R;
        cx<T>* snap = g.snap == 1 ? (cx<T>*)D.psi : g.snap == 2 ? (cx<T>*)D.prev : nullptr;
        ct_fft<T, true, N, MS * R, TH, RT>(cur, twx);
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
            double w = c.wx[x] * c.wy[j];
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
                cur[(m * R + r) * LP + x + (x >> 3)] = v[m];
            }
            if (snap) {
#pragma unroll
                for (int m = 0; m < MS; ++m) snap[(size_t)m * np + (size_t)row * N + x] = v[m];
            }
        }
        __syncthreads();
        ct_fft<T, false, N, MS * R, TH, RT>(cur, twx);
        cx<T>* S = (cx<T>*)D.S;
        for (int idx = threadIdx.x; idx < MS * R * N; idx += TH) {
            const int x = idx % N, q = idx / N, r = q % R, m = q / R;
            S[(size_t)m * np + (size_t)(row0 + r) * N + x] = cur[(m * R + r) * LP + x + (x >> 3)];
        }
        __syncthreads();
        if ((k + 1) % g.chunk == 0) {
            // this block's chunk of the instance is done: publish its partial
            block_sum<MS>(acc, red, bsum);
            const int chunk = blockIdx.x + (k / g.chunk) * gridDim.x;
            if (threadIdx.x < MS) D.part[(size_t)(chunk - inst * nci) * MS + threadIdx.x] = bsum[threadIdx.x];
#pragma unroll
            for (int m = 0; m < MS; ++m) acc[m] = 0.0;
            finish_group_norms<MS>(D, c, nci, g.snap == 2, red);
        }
        inst = ninst; lt = nlt; have = nxt;
    }
    cp_wait<0>();
}

// --------------------------------------------------------- column pass
// The 2D column pass (F_y, scale + KE + SOC, F_y^-1) of every instance:
// tiles of TX adjacent x positions, full y lines.
template <typename T, int MS, int N, int TX, int TH>
__global__ void __launch_bounds__(TH, FGPE_COL_MINB) k_col_group(GroupArgs g) {
    using CT = ColTile<N, TX>;
    constexpr int LPN = CT::LPN;
    constexpr int EPC = 16 / (int)sizeof(cx<T>);
    static_assert(TX % EPC == 0, "column tile narrower than a 16-byte chunk");
    constexpr int CPL = TX / EPC;
    constexpr int NCH = MS * N * CPL;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* cur = (cx<T>*)smraw;
    __shared__ StepConst c;
    const int ntiles = g.ninst * g.tiles;
    int cur_inst = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int inst = t / g.tiles;
        const int x0 = (t - inst * g.tiles) * TX;
        const InstDesc& D = g.d[inst];
        if (inst != cur_inst) {
            load_const(c, D.c);
            cur_inst = inst;
        }
        const long long np = D.c.npts;
        const long long stride = D.c.nx;
        cx<T>* S = (cx<T>*)D.S;
        for (int ch = threadIdx.x; ch < NCH; ch += TH) {
            const int tc = (ch % CPL) * EPC;
            const int q = ch / CPL;
            const int e = q % N, m = q / N;
            cp16(cur + (m * LPN + e + (e >> 3)) * TX + tc, S + (size_t)m * np + x0 + (size_t)e * stride + tc);
        }
        cp_commit();
        cp_wait<0>();
        __syncthreads();
        const double cfac = 1.0 / (double)c.npts;
        T fac[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) fac[m] = (T)(D.info[INFO_SC + m] * cfac);
        const cx<T>* tw = (const cx<T>*)c.twy;
        ct_fft<T, false, N, MS * TX, TH, CT>(cur, tw);
        for (int p = threadIdx.x; p < N * TX; p += TH) {
            const int tt = p % TX, e = p / TX;
            const int ix = c.fx[x0 + tt], iy = c.fy[e];
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = cscale(cur[(m * LPN + e + (e >> 3)) * TX + tt], fac[m]);
            apply_ke<T, MS>(c, ix, iy, 0, v);
            apply_soc<T, MS>(c, c.kx[ix], c.ky[iy], v);
#pragma unroll
            for (int m = 0; m < MS; ++m) cur[(m * LPN + e + (e >> 3)) * TX + tt] = v[m];
        }
        __syncthreads();
        ct_fft<T, true, N, MS * TX, TH, CT>(cur, tw);
        for (int idx = threadIdx.x; idx < MS * N * TX; idx += TH) {
            const int tt = idx % TX, q = idx / TX, e = q % N, m = q / N;
            S[(size_t)m * np + x0 + (size_t)e * stride + tt] = cur[(m * LPN + e + (e >> 3)) * TX + tt];
        }
        __syncthreads();
    }
}

}  // namespace fgpe
