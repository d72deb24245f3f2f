// fgpe_fast.cuh -- compile-time specialised, persistent row/column kernels.
//
// Same algorithm and data layout as the generic kernels (in-place DIF
// forward / DIT inverse transforms, digit-reversed spectra, padded shared
// tiles), but the line length N, the tile shape and the block size are
// template constants, so all index arithmetic folds to shifts and the
// butterfly loops unroll.  Each block is persistent over tiles and
// double-buffers them: while tile i is transformed, tile i+1 streams into the
// other shared buffer with cp.async (16-byte chunks, padded destination), so
// HBM traffic overlaps the FP64/FP32 work.
#pragma once
#include "fgpe_device.cuh"
#include "fgpe_kernels.h"

namespace fgpe {

struct CPlan {
    int nf;
    int r[12];
};
// Radix plans.  pv = 0: radix 8 while it divides, then one 4 or 2, then
// 3s and 5s (the plan of every kernel and of the handle's spectral layout).
// pv = 1: as 0, but a trailing 8*2 pair becomes 4*4 (no radix-2 pass).
// pv = 2: the radices of plan 0 in reverse order (small radices on the
// longest stride).  Only transforms whose spectra stay inside one kernel
// (the y lines of the persistent batch kernel) use pv != 0.
// pv = 3: a radix-16 pass first where it saves a pass: 2^7 -> 16*8,
// 2^8 -> 16*16 (128, 256, 384 = 16*8*3); other lengths as plan 0.  Used by
// the column passes that transform forward and back in one launch (the q2D
// y pass, the 3D z pass), whose spectra never leave the kernel.
constexpr CPlan cplan(int n, int pv = 0) {
    CPlan p{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
    if (pv == 3) {
        int e = 0, m = n;
        while (m % 2 == 0) { m /= 2; ++e; }
        if (e == 7 || e == 8) {
            p.r[p.nf++] = 16;
            p.r[p.nf++] = e == 7 ? 8 : 16;
            n = m;
        }
    }
    while (n % 8 == 0) { p.r[p.nf++] = 8; n /= 8; }
    if (n % 4 == 0) { p.r[p.nf++] = 4; n /= 4; }
    if (n % 2 == 0) {
        if (pv == 1 && p.nf > 0 && p.r[p.nf - 1] == 8) { p.r[p.nf - 1] = 4; p.r[p.nf++] = 4; }
        else p.r[p.nf++] = 2;
        n /= 2;
    }
    while (n % 3 == 0) { p.r[p.nf++] = 3; n /= 3; }
    while (n % 5 == 0) { p.r[p.nf++] = 5; n /= 5; }
    if (pv == 2)
        for (int i = 0, j = p.nf - 1; i < j; ++i, --j) { const int t = p.r[i]; p.r[i] = p.r[j]; p.r[j] = t; }
    return p;
}
constexpr int cplan_block(int n, int pass, int pv = 0) {
    CPlan pl = cplan(n, pv);
    int b = n;
    for (int i = 0; i < pass; ++i) b /= pl.r[i];
    return b;
}
constexpr int cpad(int n) { return n + (n + 7) / 8; }

// ------------------------------------------------------------ line maps
// A line map also names the groups of tasks that touch disjoint sets of
// lines: GROUP(nb) consecutive tasks form one group when a pass has nb
// butterflies per line.  With one task per thread, each group is a
// contiguous run of threads that only reads and writes its own lines.
template <int N, int NL> struct RowTile {
    static constexpr int LP = cpad(N);
    static __device__ __forceinline__ void split(int b, int nb, int& l, int& q) { l = b / nb; q = b - l * nb; }
    static __device__ __forceinline__ int at(int l, int e) { return l * LP + e + (e >> 3); }
    static constexpr int GROUP(int nb) { return nb; }
};
template <int N, int TX> struct ColTile {
    static constexpr int LPN = cpad(N);
    static constexpr int GROUP(int nb) { return nb * TX; }
    static __device__ __forceinline__ void split(int b, int nb, int& l, int& q) {
        const int t = b % TX; const int w = b / TX; q = w % nb; const int m = w / nb; l = m * TX + t;
    }
    static __device__ __forceinline__ int at(int l, int e) { return ((l / TX) * LPN + e + (e >> 3)) * TX + (l % TX); }
};

// One radix-R pass over NL lines.  Between two passes only the threads that
// share lines need to wait for each other: when every thread has exactly one
// task in this pass and in the next (same radix, so the same task -> line
// assignment) and the task groups are whole warps, the pass ends on the named
// barrier of its group (ids 1..15) instead of the block barrier.  NEXT_R is
// the radix of the next pass of the same transform, 0 after the last.
// WARP = 1: the lines belong to one warp (TH = 32, tasks by lane) and every
// pass ends on __syncwarp.
template <typename T, bool INV, int N, int NL, int TH, int P, class Map, int NEXT_R = 0, int WARP = 0, int PV = 0,
          int UMAX = 0>
__device__ __forceinline__ void ct_pass(cx<T>* s, const cx<T>* __restrict__ tw) {
    constexpr CPlan pl = cplan(N, PV);
    constexpr int R = pl.r[P];
    constexpr int BP = cplan_block(N, P, PV);
    constexpr int SI = BP / R, NB = N / R, TOT = NL * NB, ITER = (TOT + TH - 1) / TH, TSTEP = N / BP;
    constexpr int GT = Map::GROUP(NB);
    constexpr bool GROUPED = NEXT_R == R && TOT == TH && GT % 32 == 0 && TOT % GT == 0 && TOT / GT <= 15;
    static_assert(!WARP || TH == 32, "warp-scope passes run on 32 lanes");
    const int tid = WARP ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
    // UMAX > 0: passes of more than UMAX tasks per thread stay rolled (the
    // register budget of kernels that hold several line lengths)
    constexpr int UNR = (UMAX == 0 || ITER <= UMAX) ? ITER : 1;
#pragma unroll UNR
    for (int it = 0; it < ITER; ++it) {
        const int b = tid + it * TH;
        if ((TOT % TH) == 0 || b < TOT) {
            int l, q; Map::split(b, NB, l, q);
            const int blk = q / SI, n2 = q - blk * SI;
            const int e0 = blk * BP + n2;
            cx<T> v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = s[Map::at(l, e0 + r * SI)];
            if (!INV) {
                Dft<T, false, R>::run(v);
                if (SI > 1 && n2) {
                    cx<T> w[R];
                    tw_powers<T, R>(tw, n2, TSTEP, w);
#pragma unroll
                    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
                }
            } else {
                if (SI > 1 && n2) {
                    cx<T> w[R];
                    tw_powers<T, R>(tw, n2, TSTEP, w);
#pragma unroll
                    for (int r = 1; r < R; ++r) v[r] = cmulc(v[r], w[r]);
                }
                Dft<T, true, R>::run(v);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) s[Map::at(l, e0 + r * SI)] = v[r];
        }
    }
    if constexpr (WARP) {
        __syncwarp();
    } else if constexpr (GROUPED) {
        const int g = (int)threadIdx.x / GT;
        asm volatile("bar.sync %0, %1;\n" ::"r"(1 + g), "r"(GT) : "memory");
    } else {
        __syncthreads();
    }
}

template <typename T, bool INV, int N, int NL, int TH, class Map, int WARP = 0, int P = 0, int PV = 0, int UMAX = 0>
__device__ __forceinline__ void ct_fft(cx<T>* s, const cx<T>* __restrict__ tw) {
    constexpr CPlan pl = cplan(N, PV);
    if constexpr (P < pl.nf) {
        constexpr int PP = INV ? pl.nf - 1 - P : P;
        constexpr int NEXT_R = P + 1 < pl.nf ? pl.r[INV ? PP - 1 : PP + 1] : 0;
        ct_pass<T, INV, N, NL, TH, PP, Map, NEXT_R, WARP, PV, UMAX>(s, tw);
        ct_fft<T, INV, N, NL, TH, Map, WARP, P + 1, PV, UMAX>(s, tw);
    }
}

// ------------------------------------------------------------- cp.async
#ifdef FGPE_CHECK_ALIGN
// Diagnostic build only: record the first misaligned copy and skip it.
static __device__ unsigned long long g_align_fault[4];
__device__ __forceinline__ bool align_bad(const void* s, const void* g, unsigned bytes, int site) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(s);
    if ((d % bytes) == 0 && ((unsigned long long)g % bytes) == 0) return false;
    if (atomicCAS(&g_align_fault[0], 0ull, 1ull) == 0ull) {
        g_align_fault[1] = (unsigned long long)site;
        g_align_fault[2] = d;
        g_align_fault[3] = (unsigned long long)g;
    }
    return true;
}
#define FGPE_ALIGN_GUARD(s, g, b, site) if (align_bad(s, g, b, site)) return
#else
#define FGPE_ALIGN_GUARD(s, g, b, site)
#endif

__device__ __forceinline__ void cp16(void* smem_dst, const void* gsrc) {
    FGPE_ALIGN_GUARD(smem_dst, gsrc, 16, 16);
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp8(void* smem_dst, const void* gsrc) {
    FGPE_ALIGN_GUARD(smem_dst, gsrc, 8, 8);
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
// One complex element: 16-byte copy for complex128, 8-byte for complex64 (the
// padded row layout puts complex64 elements on 8-byte boundaries only).
template <typename T> __device__ __forceinline__ void cp_elem(cx<T>* smem_dst, const cx<T>* gsrc) {
    if constexpr (sizeof(cx<T>) == 16) cp16(smem_dst, gsrc);
    else cp8(smem_dst, gsrc);
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Blocks per SM the launch bounds target and shared buffers per block
// (2 = double-buffered prefetch).
// Resident blocks per SM the row kernel is compiled for: small blocks (up to
// 192 threads: the spin-1 rows) run 4 per SM, the others 2, unless
// FGPE_ROW_MINB fixes it at build time.
#ifndef FGPE_ROW_MINB
#define FGPE_ROW_MINB 0
#endif
constexpr int row_minb(int th) { return FGPE_ROW_MINB ? FGPE_ROW_MINB : (th <= 192 ? 4 : 2); }
#ifndef FGPE_ROW_NBUF
#define FGPE_ROW_NBUF 2
#endif
#ifndef FGPE_COL_MINB
#define FGPE_COL_MINB 2
#endif
#ifndef FGPE_COL_NBUF
#define FGPE_COL_NBUF 1
#endif
#ifndef FGPE_TW_SMEM
#define FGPE_TW_SMEM 0
#endif

// ------------------------------------------------------------ row kernel
// Tiles of R x-lines (all MS components); see k_row for the three modes.
template <typename T, int MS, int N, int R, int TH, int NBUF = FGPE_ROW_NBUF>
__global__ void __launch_bounds__(TH, row_minb(TH)) k_row_fast(StepConst c, RowArgs a) {
    // a programmatic dependent launch starts before the previous pass ends:
    // wait for it (and its memory) before touching the state
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    using RT = RowTile<N, MS * R>;
    constexpr int LP = RT::LP;
    constexpr int TILE = MS * R * LP;
    constexpr int NCH = MS * R * N;                    // one async copy per element
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* bufs = (cx<T>*)smraw;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    const long long np = c.npts;
    const int ntiles = (c.ny * c.nz) / R;
    const cx<T>* twx = (const cx<T>*)c.twx;
    if (FGPE_TW_SMEM) {
        // the twiddle table sits after the tile buffers
        cx<T>* tws = bufs + NBUF * TILE;
        for (int i = threadIdx.x; i < N; i += TH) tws[i] = twx[i];
        twx = tws;   // made visible by the first barrier of the tile loop
    }
    const cx<T>* src = (a.mode == ROW_FWD) ? (const cx<T>*)a.psi : (const cx<T>*)a.S;
    cx<T>* S = (cx<T>*)a.S;
    cx<T>* snap = (cx<T>*)a.snap;

    auto issue = [&](int tile, cx<T>* dst) {
        const int row0 = tile * R;
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
    int tile = blockIdx.x;
    if (NBUF == 2) {
        if (tile < ntiles) issue(tile, bufs);
        cp_commit();
    }
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        cx<T>* cur = bufs + (NBUF == 2 ? (it & 1) * TILE : 0);
        if (NBUF == 2) {
            const int nt = tile + gridDim.x;
            if (nt < ntiles) issue(nt, bufs + ((it + 1) & 1) * TILE);
            cp_commit();
            cp_wait<1>();
        } else {
            issue(tile, cur);
            cp_commit();
            cp_wait<0>();
        }
        __syncthreads();
        const int row0 = tile * R;
        if (a.mode == ROW_FWD) {
            ct_fft<T, false, N, MS * R, TH, RT>(cur, twx);
        } else {
            ct_fft<T, true, N, MS * R, TH, RT>(cur, twx);
            if (a.mode == ROW_INV) {
                const T inv = (T)(1.0 / N);
                cx<T>* dst = (cx<T>*)a.psi;
                for (int idx = threadIdx.x; idx < MS * R * N; idx += TH) {
                    const int x = idx % N, q = idx / N, r = q % R, m = q / R;
                    dst[(size_t)m * np + (size_t)(row0 + r) * N + x] = cscale(cur[(m * R + r) * LP + x + (x >> 3)], inv);
                }
                __syncthreads();
                continue;
            }
            for (int p = threadIdx.x; p < R * N; p += TH) {
                const int x = p % N, r = p / N;
                const int row = row0 + r;
                const int j = row % c.ny, k = row / c.ny;
                cx<T> v[MS];
#pragma unroll
                for (int m = 0; m < MS; ++m) v[m] = cur[(m * R + r) * LP + x + (x >> 3)];
                const cx<T> eV = pot_phase<T>(c, x, j, k);
                apply_se<T, MS>(c, v);
                apply_sp<T, MS>(c, eV, v);
                double w = c.wx[x];
                if (c.dim >= 2) w *= c.wy[j];
                if (c.dim >= 3) w *= c.wz[k];
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
        }
        for (int idx = threadIdx.x; idx < MS * R * N; idx += TH) {
            const int x = idx % N, q = idx / N, r = q % R, m = q / R;
            S[(size_t)m * np + (size_t)(row0 + r) * N + x] = cur[(m * R + r) * LP + x + (x >> 3)];
        }
        __syncthreads();
    }
    cp_wait<0>();
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    if (a.mode != ROW_FULL) return;
    block_sum<MS>(acc, red, bsum);
    if (threadIdx.x < MS) a.part[(size_t)blockIdx.x * MS + threadIdx.x] = bsum[threadIdx.x];
    finish_norms<MS>(c, a.part, a.counter, a.info, red);
}

// ------------------------------------------------------- warp-row kernel
// The row pass (ROW_FULL) with one warp per x row: the MS component lines of
// one (y, z) position sit in the warp's private shared memory, so the inverse
// transform, SE, SP, the NORMC partials and the forward transform need only
// __syncwarp; the block meets once at the end, for its NORMC partial and the
// last-block reduction.  Rows are dealt to the warps of the grid in turn;
// with NBUF = 2 a warp prefetches its next row with cp.async while it works
// on the current one.  Per element the arithmetic is that of k_row_fast.
#ifndef FGPE_WROW_NBUF
#define FGPE_WROW_NBUF 1
#endif
template <typename T, int MS, int N, int WPB, int NBUF>
__global__ void __launch_bounds__(WPB * 32, 2) k_row_warp(StepConst c, RowArgs a) {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    using RT = RowTile<N, MS>;
    constexpr int LP = RT::LP;
    constexpr int TILE = MS * LP;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    cx<T>* mine = (cx<T>*)smraw + (size_t)warp * NBUF * TILE;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    const long long np = c.npts;
    const int nrows = c.ny * c.nz;
    const int nw = (int)gridDim.x * WPB;
    const cx<T>* twx = (const cx<T>*)c.twx;
    cx<T>* S = (cx<T>*)a.S;
    cx<T>* snap = (cx<T>*)a.snap;
    auto issue = [&](int row, cx<T>* dst) {
        for (int ch = lane; ch < MS * N; ch += 32) {
            const int x = ch % N, m = ch / N;
            cp_elem<T>(dst + m * LP + x + (x >> 3), S + (size_t)m * np + (size_t)row * N + x);
        }
    };
    double acc[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) acc[m] = 0.0;
    int row = (int)blockIdx.x * WPB + warp;
    if (NBUF == 2) {
        if (row < nrows) issue(row, mine);
        cp_commit();
    }
    for (int it = 0; row < nrows; ++it, row += nw) {
        cx<T>* cur = mine + (NBUF == 2 ? (it & 1) * TILE : 0);
        if (NBUF == 2) {
            const int nr = row + nw;
            if (nr < nrows) issue(nr, mine + ((it + 1) & 1) * TILE);
            cp_commit();
            cp_wait<1>();
        } else {
            issue(row, cur);
            cp_commit();
            cp_wait<0>();
        }
        __syncwarp();
        ct_fft<T, true, N, MS, 32, RT, 1>(cur, twx);
        const int j = row % c.ny, k = row / c.ny;
        for (int x = lane; x < N; x += 32) {
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = cur[m * LP + x + (x >> 3)];
            const cx<T> eV = pot_phase<T>(c, x, j, k);
            apply_se<T, MS>(c, v);
            apply_sp<T, MS>(c, eV, v);
            double w = c.wx[x];
            if (c.dim >= 2) w *= c.wy[j];
            if (c.dim >= 3) w *= c.wz[k];
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
                cur[m * LP + x + (x >> 3)] = v[m];
            }
            if (snap) {
#pragma unroll
                for (int m = 0; m < MS; ++m) snap[(size_t)m * np + (size_t)row * N + x] = v[m];
            }
        }
        __syncwarp();
        ct_fft<T, false, N, MS, 32, RT, 1>(cur, twx);
        for (int idx = lane; idx < MS * N; idx += 32) {
            const int x = idx % N, m = idx / N;
            S[(size_t)m * np + (size_t)row * N + x] = cur[m * LP + x + (x >> 3)];
        }
        __syncwarp();
    }
    cp_wait<0>();
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    block_sum<MS>(acc, red, bsum);
    if (threadIdx.x < MS) a.part[(size_t)blockIdx.x * MS + threadIdx.x] = bsum[threadIdx.x];
    finish_norms<MS>(c, a.part, a.counter, a.info, red);
}

// --------------------------------------------------------- column kernel
// Tiles of TX adjacent x positions, full lines of N along the transformed
// axis; persistent over (x-tile, other) pairs.
// PV: radix plan of the lines (cplan); a plan other than the handle's needs
// a pass that transforms forward and back, with a.fline its position map.
template <typename T, int MS, int N, int TX, int TH, int NBUF = FGPE_COL_NBUF, int PV = 0>
__global__ void __launch_bounds__(TH, FGPE_COL_MINB) k_col_fast(StepConst c, ColArgs a) {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    using CT = ColTile<N, TX>;
    constexpr int LPN = CT::LPN;
    constexpr int TILE = MS * LPN * TX;
    constexpr int EPC = 16 / (int)sizeof(cx<T>);
    // every 16-byte chunk starts at a multiple of EPC elements of a tile row
    // of TX elements: destinations stay 16-byte aligned
    static_assert(TX % EPC == 0, "column tile narrower than a 16-byte chunk");
    constexpr int CPL = TX / EPC;                      // chunks per (m, e)
    constexpr int NCH = MS * N * CPL;
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* bufs = (cx<T>*)smraw;
    __shared__ cx<T> usoc[TX * MS * MS];     // per-column SO-coupling matrices (z pass)
    const long long np = c.npts;
    const int nxt = c.nx / TX;
    const int nother = (int)a.n_other;
    const int ntiles = nxt * nother;
    const cx<T>* tw = (const cx<T>*)a.tw;
    if (FGPE_TW_SMEM) {
        cx<T>* tws = bufs + NBUF * TILE;
        for (int i = threadIdx.x; i < N; i += TH) tws[i] = tw[i];
        tw = tws;
    }
    cx<T>* S = (cx<T>*)a.S;
    T fac[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) fac[m] = (a.flags & COL_SCALE) ? (T)(a.info[INFO_SC + m] * a.cfac) : (T)1;

    auto issue = [&](int tile, cx<T>* dst) {
        const int x0 = (tile % nxt) * TX;
        const long long off = (long long)(tile / nxt) * a.other_stride + x0;
        for (int ch = threadIdx.x; ch < NCH; ch += TH) {
            const int tc = (ch % CPL) * EPC;
            const int q = ch / CPL;
            const int e = q % N, m = q / N;
            cp16(dst + (m * LPN + e + (e >> 3)) * TX + tc, S + (size_t)m * np + off + (size_t)e * a.axis_stride + tc);
        }
    };

    int tile = blockIdx.x;
    if (NBUF == 2) {
        if (tile < ntiles) issue(tile, bufs);
        cp_commit();
    }
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        cx<T>* cur = bufs + (NBUF == 2 ? (it & 1) * TILE : 0);
        if (NBUF == 2) {
            const int nt = tile + gridDim.x;
            if (nt < ntiles) issue(nt, bufs + ((it + 1) & 1) * TILE);
            cp_commit();
            cp_wait<1>();
        } else {
            issue(tile, cur);
            cp_commit();
            cp_wait<0>();
        }
        __syncthreads();
        const int x0 = (tile % nxt) * TX;
        const int oth = tile / nxt;
        const long long off = (long long)oth * a.other_stride + x0;
        // with KE/SOC in this pass the scale rides on the pointwise step
        // (the transform is linear); otherwise it takes its own sweep
        const bool fold = (a.flags & COL_SCALE) && (a.flags & COL_KOP);
        if ((a.flags & COL_SCALE) && !fold) {
            // component loop outermost and unrolled: fac[] stays in registers
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                for (int idx = threadIdx.x; idx < N * TX; idx += TH) {
                    const int t = idx % TX, e = idx / TX;
                    cx<T>& v = cur[(m * LPN + e + (e >> 3)) * TX + t];
                    v = cscale(v, fac[m]);
                }
            }
            __syncthreads();
        }
        if (a.flags & COL_FWD) ct_fft<T, false, N, MS * TX, TH, CT, 0, 0, PV>(cur, tw);
        if (a.flags & COL_KOP) {
            // z lines: (kx, ky) is fixed along each line of the tile, so the
            // SO-coupling exponential is one MS x MS matrix per tile column,
            // built here by applying apply_soc to the unit vectors and then
            // applied to every point as one matrix-vector product
            const bool zmat = a.axis == 2 && (a.flags & COL_SOC);
            if (zmat) {
                if (threadIdx.x < TX * MS) {
                    const int t = threadIdx.x / MS, j = threadIdx.x - (threadIdx.x / MS) * MS;
                    cx<T> u[MS];
#pragma unroll
                    for (int m = 0; m < MS; ++m) u[m] = mk<T>(m == j ? (T)1 : (T)0, (T)0);
                    const int ixt = c.fx[x0 + t], iyt = a.fother[oth];
                    apply_soc<T, MS>(c, c.kx[ixt], c.ky[iyt], u);
                    // the kx, ky part of KE, exp(-i CDT (kx^2 + ky^2)), is a
                    // scalar along the line: folded into the matrix
                    const cx<T> f = (a.flags & COL_KE) ? fmul(c.imag, ((const cx<T>*)c.kex)[ixt], ((const cx<T>*)c.key)[iyt])
                                                        : mk<T>((T)1, (T)0);
#pragma unroll
                    for (int r = 0; r < MS; ++r) usoc[(t * MS + r) * MS + j] = cmul(u[r], f);
                }
                __syncthreads();
            }
            for (int p = threadIdx.x; p < N * TX; p += TH) {
                const int t = p % TX, e = p / TX;
                const int ix = c.fx[x0 + t];
                // y lines: ky at the line position; z lines: ky at the tile's y
                int iy, iz;
                if (a.axis == 1) { iy = a.fline[e]; iz = 0; } else { iy = a.fother[oth]; iz = a.fline[e]; }
                cx<T> v[MS];
#pragma unroll
                for (int m = 0; m < MS; ++m) v[m] = cur[(m * LPN + e + (e >> 3)) * TX + t];
                if (fold) {
#pragma unroll
                    for (int m = 0; m < MS; ++m) v[m] = cscale(v[m], fac[m]);
                }
                if (zmat) {
                    if (a.flags & COL_KE) {
                        // the kz part, exp(-i CDT (kz^2 - 2 L GAMMAZ kz)) per component
                        const cx<T>* kez = (const cx<T>*)c.kez;
#pragma unroll
                        for (int m = 0; m < MS; ++m) v[m] = fmul(c.imag, kez[m * c.nz + iz], v[m]);
                    }
                } else if (a.flags & COL_KE) {
                    apply_ke<T, MS>(c, ix, iy, iz, v);
                }
                if (zmat) {
                    const cx<T>* U = usoc + t * MS * MS;
                    cx<T> w[MS];
#pragma unroll
                    for (int r = 0; r < MS; ++r) {
                        cx<T> acc = cmul(U[r * MS], v[0]);
#pragma unroll
                        for (int q = 1; q < MS; ++q) acc = cmac(acc, U[r * MS + q], v[q]);
                        w[r] = acc;
                    }
#pragma unroll
                    for (int m = 0; m < MS; ++m) v[m] = w[m];
                } else if (a.flags & COL_SOC) {
                    apply_soc<T, MS>(c, c.kx[ix], c.ky[iy], v);
                }
#pragma unroll
                for (int m = 0; m < MS; ++m) cur[(m * LPN + e + (e >> 3)) * TX + t] = v[m];
            }
            __syncthreads();
        }
        if (a.flags & COL_INV) ct_fft<T, true, N, MS * TX, TH, CT, 0, 0, PV>(cur, tw);
        for (int idx = threadIdx.x; idx < MS * N * TX; idx += TH) {
            const int t = idx % TX, q = idx / TX, e = q % N, m = q / N;
            S[(size_t)m * np + off + (size_t)e * a.axis_stride + t] = cur[(m * LPN + e + (e >> 3)) * TX + t];
        }
        __syncthreads();
    }
    cp_wait<0>();
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

}  // namespace fgpe
