// fgpe_kernels.cu -- the propagator kernels.
//
// State between steps (2D/3D): S = F_x[psi], the x-transformed real-space
// spinor psi, plus a pending scalar `scale` (imaginary-time renormalisation,
// 1/sqrt(total norm)); the physical state is phi = scale * psi.  One split
// step (cgpe1d.f90:434-441, 470-472) is then
//   2D: col pass   (y)  : load S * scale/N, F_y, KE, SOC, F_y^-1, store
//       row pass   (x)  : load, F_x^-1, SE, SP, NORMC partials, F_x, store
//   3D: col pass y (F_y, with scale/N), col pass z (F_z, KE, SOC, F_z^-1),
//       col pass y (F_y^-1), row pass x as above
// so a 2D step streams the spinor through HBM twice and a 3D step four times.
// The row pass's last block finishes the NORMC reduction in a fixed order and
// publishes norms and the next scale (no host round trip).
//   1D: the whole spinor lives in one block's shared memory and the block
//       loops over steps; long lines take the four-step split, either as
//       two passes per step or on one thread-block cluster for a whole call.
#pragma once
#include <cooperative_groups.h>
#include "fgpe_device.cuh"
#include "fgpe_kernels.h"

namespace fgpe {

// ------------------------------------------------------------ reductions
// Deterministic block sum of NV doubles per thread into out[NV] (thread 0).
template <int NV>
__device__ __forceinline__ void block_sum(double (&acc)[NV], double* red, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double v = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[q * 32 + warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0;
        for (int w = 0; w < nw; ++w) s += red[threadIdx.x * 32 + w];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0) { for (int w = 0; w < nw; ++w) r = fmax(r, red[w]); }
    __syncthreads();
    return r;
}

// Last-block completion of the NORMC reduction: the partials
// partial[b*MS+m] of every block are summed by the whole last block in a
// fixed order (thread t takes blocks t, t+T, ..., then the block tree), so
// the result does not depend on which block finishes last; info[] receives
// scale, total and norms.  red holds at least 32*(MS+1) doubles.
template <int MS>
__device__ __forceinline__ void finish_norms(const StepConst& c, const double* part, unsigned* counter,
                                             double* info, double* red) {
    __shared__ int is_last;
    __threadfence();
    if (threadIdx.x == 0) is_last = (atomicAdd(counter, 1u) == gridDim.x * gridDim.y - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const int nb = gridDim.x * gridDim.y;
    double acc[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) acc[m] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] += __ldcg(part + (size_t)b * MS + m);
    }
    block_sum<MS>(acc, red, red + 32 * MS);
    if (threadIdx.x < MS) red[threadIdx.x] = red[32 * MS + threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0, n[MS], sc[MS];
        for (int m = 0; m < MS; ++m) { n[m] = red[m]; tot += red[m]; info[INFO_NORM + m] = red[m]; }
        info[INFO_TOTAL] = tot;
        sink_norms<MS>(c, n);
        const int rc = compute_scales<MS>(c, n, info + INFO_SIG, sc);
        bool bad = !(tot == tot) || !(tot < 1e300);
        for (int m = 0; m < MS; ++m) { info[INFO_SC + m] = sc[m]; bad = bad || !(sc[m] == sc[m]); }
        if (bad) info[INFO_ERR] = 1.0;
        if (rc) info[INFO_ERR] = (double)rc;
        *counter = 0u;
    }
}

// -------------------------------------------------------------- row pass
// mode ROW_FULL: one split step's real-space part (S -> S).
// mode ROW_FWD : prologue psi -> S (forward x transform only).
// mode ROW_INV : psi <- F_x^-1[S] / NX (rebuild the real-space copy).
template <typename T, int MS>
__global__ void __launch_bounds__(256)
k_row(StepConst c, RowArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = (cx<T>*)smraw;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    const int nx = c.nx, R = a.rows;
    const int lp = padded_len(nx);
    const RowMap mp{lp};
    const int row0 = blockIdx.x * R;
    const long long np = c.npts;
    const cx<T>* twx = (const cx<T>*)c.twx;
    const int nel = MS * R * nx;
    const cx<T>* src = (a.mode == ROW_FWD) ? (const cx<T>*)a.psi : (const cx<T>*)a.S;
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int x = idx % nx, q = idx / nx, r = q % R, m = q / R;
        sm[(m * R + r) * lp + pad_idx(x)] = src[(size_t)m * np + (size_t)(row0 + r) * nx + x];
    }
    __syncthreads();
    if (a.mode == ROW_FWD) {
        block_fft<T, false>(sm, mp, MS * R, c.px, twx);
    } else {
        block_fft<T, true>(sm, mp, MS * R, c.px, twx);
        if (a.mode == ROW_INV) {
            const T inv = (T)(1.0 / nx);
            cx<T>* dst = (cx<T>*)a.psi;
            for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
                const int x = idx % nx, q = idx / nx, r = q % R, m = q / R;
                dst[(size_t)m * np + (size_t)(row0 + r) * nx + x] = cscale(sm[(m * R + r) * lp + pad_idx(x)], inv);
            }
            return;
        }
        // SE + SP + NORMC partials
        double acc[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] = 0.0;
        cx<T>* snap = (cx<T>*)a.snap;
        for (int p = threadIdx.x; p < R * nx; p += blockDim.x) {
            const int x = p % nx, r = p / nx;
            const int row = row0 + r;
            const int j = row % c.ny, k = row / c.ny;
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = sm[(m * R + r) * lp + pad_idx(x)];
            const cx<T> eV = pot_phase<T>(c, x, j, k);
            apply_se<T, MS>(c, v);
            apply_sp<T, MS>(c, eV, v);
            double w = c.wx[x];
            if (c.dim >= 2) w *= c.wy[j];
            if (c.dim >= 3) w *= c.wz[k];
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
                sm[(m * R + r) * lp + pad_idx(x)] = v[m];
            }
            if (snap) {
#pragma unroll
                for (int m = 0; m < MS; ++m) snap[(size_t)m * np + (size_t)row * nx + x] = v[m];
            }
        }
        block_sum<MS>(acc, red, bsum);
        if (threadIdx.x < MS) a.part[(size_t)blockIdx.x * MS + threadIdx.x] = bsum[threadIdx.x];
        finish_norms<MS>(c, a.part, a.counter, a.info, red);
        __syncthreads();
        // F_x of the new real-space state
        block_fft<T, false>(sm, mp, MS * R, c.px, twx);
    }
    cx<T>* dst = (cx<T>*)a.S;
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int x = idx % nx, q = idx / nx, r = q % R, m = q / R;
        dst[(size_t)m * np + (size_t)(row0 + r) * nx + x] = sm[(m * R + r) * lp + pad_idx(x)];
    }
}

// ----------------------------------------------------------- column pass
// A tile of TX adjacent x positions, full lines of length n along the
// transformed axis (stride a.axis_stride), all MS components.
template <typename T, int MS>
__global__ void __launch_bounds__(256)
k_col(StepConst c, ColArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = (cx<T>*)smraw;
    const int TX = a.tx, n = a.n;
    const int lpn = padded_len(n);
    const ColMap mp{TX, lpn};
    const int x0 = blockIdx.x * TX;
    const long long off = (long long)blockIdx.y * a.other_stride + x0;
    const long long np = c.npts;
    const cx<T>* tw = (const cx<T>*)a.tw;
    const int nel = MS * n * TX;
    cx<T>* S = (cx<T>*)a.S;
    T fac[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) fac[m] = (a.flags & COL_SCALE) ? (T)(a.info[INFO_SC + m] * a.cfac) : (T)1;
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int t = idx % TX, q = idx / TX, e = q % n, m = q / n;
        cx<T> v = S[(size_t)m * np + off + (size_t)e * a.axis_stride + t];
        if (a.flags & COL_SCALE) v = cscale(v, fac[m]);
        sm[(m * lpn + pad_idx(e)) * TX + t] = v;
    }
    __syncthreads();
    if (a.flags & COL_FWD) block_fft<T, false>(sm, mp, MS * TX, a.plan, tw);
    if (a.flags & COL_KOP) {
        // spectral positions -> frequency indices (digit-reversed order)
        for (int p = threadIdx.x; p < n * TX; p += blockDim.x) {
            const int t = p % TX, e = p / TX;
            const int ix = c.fx[x0 + t];
            // y lines: ky at the line position; z lines: ky at the block's y
            int iy, iz;
            if (a.axis == 1) { iy = c.fy[e]; iz = 0; } else { iy = c.fy[blockIdx.y]; iz = c.fz[e]; }
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = sm[(m * lpn + pad_idx(e)) * TX + t];
            if (a.flags & COL_KE) apply_ke<T, MS>(c, ix, iy, iz, v);
            if (a.flags & COL_SOC) apply_soc<T, MS>(c, c.kx[ix], c.ky[iy], v);
#pragma unroll
            for (int m = 0; m < MS; ++m) sm[(m * lpn + pad_idx(e)) * TX + t] = v[m];
        }
        __syncthreads();
    }
    if (a.flags & COL_INV) block_fft<T, true>(sm, mp, MS * TX, a.plan, tw);
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int t = idx % TX, q = idx / TX, e = q % n, m = q / n;
        S[(size_t)m * np + off + (size_t)e * a.axis_stride + t] = sm[(m * lpn + pad_idx(e)) * TX + t];
    }
}

// ---------------------------------------------------- long 1D lines
// Row pass of a step (rows p2 of Q, N1 points each): scale by sc_m/N, F_N1,
// KE and SOC at the 1D frequency k = k2 + N2*k1, F_N1^-1.  c.px/c.fx are the
// N1 transform's plan and position map, c.py/c.fy the N2 ones.
template <typename T, int MS>
__global__ void __launch_bounds__(256)
k_r1d(StepConst c, Split1dArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = (cx<T>*)smraw;
    const int n1 = a.n1, R = a.tile;
    const int lp = padded_len(n1);
    const RowMap mp{lp};
    const int row0 = blockIdx.x * R;
    const long long np = c.npts;
    cx<T>* S = (cx<T>*)a.S;
    T fac[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) fac[m] = (T)(a.info[INFO_SC + m] / (double)np);
    const int nel = MS * R * n1;
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int x = idx % n1, q = idx / n1, r = q % R, m = q / R;
        sm[(m * R + r) * lp + pad_idx(x)] = cscale(S[(size_t)m * np + (size_t)(row0 + r) * n1 + x], fac[m]);
    }
    __syncthreads();
    block_fft<T, false>(sm, mp, MS * R, c.px, (const cx<T>*)a.tw1);
    for (int p = threadIdx.x; p < R * n1; p += blockDim.x) {
        const int x = p % n1, r = p / n1;
        const int k = c.fy[row0 + r] + a.n2 * c.fx[x];
        cx<T> v[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) v[m] = sm[(m * R + r) * lp + pad_idx(x)];
        apply_ke<T, MS>(c, k, 0, 0, v);
        apply_soc<T, MS>(c, c.kx[k], 0.0, v);
#pragma unroll
        for (int m = 0; m < MS; ++m) sm[(m * R + r) * lp + pad_idx(x)] = v[m];
    }
    __syncthreads();
    block_fft<T, true>(sm, mp, MS * R, c.px, (const cx<T>*)a.tw1);
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int x = idx % n1, q = idx / n1, r = q % R, m = q / R;
        S[(size_t)m * np + (size_t)(row0 + r) * n1 + x] = sm[(m * R + r) * lp + pad_idx(x)];
    }
}

// Column pass (columns n1, N2 points each, TX adjacent columns per block).
//  C1D_FULL: conj twiddle, F_N2^-1 (real space), SE, SP, NORMC partials
//            (+ snapshot), F_N2, twiddle; the last block finishes NORMC and
//            the next scales.
//  C1D_FWD : psi (real space) -> Q (prologue).
//  C1D_INV : Q -> psi = x (export; the pending scales stay in info).
template <typename T, int MS>
__global__ void __launch_bounds__(256)
k_c1d(StepConst c, Split1dArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = (cx<T>*)smraw;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    const int n1 = a.n1, n2 = a.n2, TX = a.tile;
    const int lpn = padded_len(n2);
    const ColMap mp{TX, lpn};
    const int x0 = blockIdx.x * TX;
    const long long np = c.npts;
    const cx<T>* twn = (const cx<T>*)a.twn;
    const cx<T>* tw2 = (const cx<T>*)a.tw2;
    cx<T>* S = (cx<T>*)a.S;
    const int nel = MS * n2 * TX;
    const cx<T>* src = a.mode == C1D_FWD ? (const cx<T>*)a.psi : S;
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int t = idx % TX, q = idx / TX, e = q % n2, m = q / n2;
        cx<T> v = src[(size_t)m * np + (size_t)e * n1 + x0 + t];
        if (a.mode != C1D_FWD) v = cmulc(v, twn[(size_t)(x0 + t) * c.fy[e]]);   // conj twiddle
        sm[(m * lpn + pad_idx(e)) * TX + t] = v;
    }
    __syncthreads();
    if (a.mode != C1D_FWD) block_fft<T, true>(sm, mp, MS * TX, c.py, tw2);
    if (a.mode == C1D_INV) {
        const T inv = (T)(1.0 / n2);
        cx<T>* dst = (cx<T>*)a.psi;
        for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
            const int t = idx % TX, q = idx / TX, e = q % n2, m = q / n2;
            dst[(size_t)m * np + (size_t)e * n1 + x0 + t] = cscale(sm[(m * lpn + pad_idx(e)) * TX + t], inv);
        }
        return;
    }
    if (a.mode == C1D_FULL) {
        double acc[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] = 0.0;
        cx<T>* snap = (cx<T>*)a.snap;
        for (int p = threadIdx.x; p < n2 * TX; p += blockDim.x) {
            const int t = p % TX, e = p / TX;
            const int x = x0 + t + n1 * e;             // 1D grid index
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = sm[(m * lpn + pad_idx(e)) * TX + t];
            const cx<T> eV = pot_phase<T>(c, x, 0, 0);
            apply_se<T, MS>(c, v);
            apply_sp<T, MS>(c, eV, v);
            const double w = c.wx[x];
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
                sm[(m * lpn + pad_idx(e)) * TX + t] = v[m];
            }
            if (snap) {
#pragma unroll
                for (int m = 0; m < MS; ++m) snap[(size_t)m * np + x] = v[m];
            }
        }
        block_sum<MS>(acc, red, bsum);
        if (threadIdx.x < MS) a.part[(size_t)blockIdx.x * MS + threadIdx.x] = bsum[threadIdx.x];
        finish_norms<MS>(c, a.part, a.counter, a.info, red);
        __syncthreads();
    }
    block_fft<T, false>(sm, mp, MS * TX, c.py, tw2);
    for (int idx = threadIdx.x; idx < nel; idx += blockDim.x) {
        const int t = idx % TX, q = idx / TX, e = q % n2, m = q / n2;
        S[(size_t)m * np + (size_t)e * n1 + x0 + t] = cmul(sm[(m * lpn + pad_idx(e)) * TX + t], twn[(size_t)(x0 + t) * c.fy[e]]);
    }
}

// --------------------------------------- long 1D lines on one cluster
// The row and column passes of k_r1d/k_c1d on one thread-block cluster of
// CL1D CTAs that stays resident for all nsteps steps of a call.  Q (n2 rows
// of n1 points per component) lives in the CTAs' shared memory: CTA r keeps
// rows [r*RR, (r+1)*RR), RR = n2/CL1D, for the row phase, and transforms
// columns [r*CC, (r+1)*CC), CC = n1/CL1D, in the column phase.  It gathers
// those columns from the other CTAs' row tiles and scatters them back through
// distributed shared memory, so a step touches no global memory except the
// snapshots.  The row tiles alternate between two buffers: step s reads
// buffer s&1 and scatters into buffer (s+1)&1, which nobody reads in step s,
// so one cluster barrier after the row phase and one after the scatter are
// all a step needs.  NORMC: each CTA's block sum goes to its slot in every
// CTA; after the second barrier every CTA adds the CL1D sums in the same order
// and derives the same scales (compute_scales is deterministic), and scales
// its own rows for the next step.  Per element the arithmetic is that of
// k_r1d/k_c1d; only the order of the NORMC sum differs.  Every thread of every
// CTA takes both barriers on every step (no early exit).
constexpr int CL1D = 8;

template <typename T, int MS>
__global__ void __cluster_dims__(CL1D, 1, 1) __launch_bounds__(256)
k_cl1d(StepConst c, Cluster1dArgs a) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    __shared__ double part[CL1D * MS];
    __shared__ double s_sc[MS];
    __shared__ double s_sig[2];
    const int n1 = a.n1, n2 = a.n2;
    const int RR = n2 / CL1D, CC = n1 / CL1D;
    const int lp1 = padded_len(n1), lpn = padded_len(n2);
    const int nrow = MS * RR * n1;
    const int rtile = MS * RR * lp1;               // one row buffer, [m][r][pad(x)]
    cx<T>* rowbuf = (cx<T>*)smraw;                 // two row buffers
    cx<T>* cols = rowbuf + 2 * rtile;              // [m][pad(e)][t], t < CC
    const RowMap rmp{lp1};
    const ColMap cmp{CC, lpn};
    const int rank = (int)cl.block_rank();
    const int row0 = rank * RR, x0 = rank * CC;
    const long long np = c.npts;
    const cx<T>* twn = (const cx<T>*)a.twn;
    const cx<T>* tw1 = (const cx<T>*)a.tw1;
    const cx<T>* tw2 = (const cx<T>*)a.tw2;
    cx<T>* S = (cx<T>*)a.S;
    if (threadIdx.x < MS) s_sc[threadIdx.x] = a.info[INFO_SC + threadIdx.x];
    if (threadIdx.x < 2) s_sig[threadIdx.x] = a.info[INFO_SIG + threadIdx.x];
    __syncthreads();
    // this CTA's rows, scaled by sc_m/N as the row pass loads them
    for (int idx = threadIdx.x; idx < nrow; idx += blockDim.x) {
        const int x = idx % n1, q = idx / n1, r = q % RR, m = q / RR;
        rowbuf[(m * RR + r) * lp1 + pad_idx(x)] =
            cscale(S[(size_t)m * np + (size_t)(row0 + r) * n1 + x], (T)(s_sc[m] / (double)np));
    }
    __syncthreads();
    const int ncol = MS * n2 * CC;
    for (int step = 0; step < a.nsteps; ++step) {
        cx<T>* rows = rowbuf + (step & 1) * rtile;        // this step's rows
        cx<T>* next = rowbuf + ((step + 1) & 1) * rtile;  // scatter target
        // ---- row phase: F_N1, KE and SOC at k = k2 + N2*k1, F_N1^-1
        block_fft<T, false>(rows, rmp, MS * RR, c.px, tw1);
        for (int p = threadIdx.x; p < RR * n1; p += blockDim.x) {
            const int x = p % n1, r = p / n1;
            const int k = c.fy[row0 + r] + n2 * c.fx[x];
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = rows[(m * RR + r) * lp1 + pad_idx(x)];
            apply_ke<T, MS>(c, k, 0, 0, v);
            apply_soc<T, MS>(c, c.kx[k], 0.0, v);
#pragma unroll
            for (int m = 0; m < MS; ++m) rows[(m * RR + r) * lp1 + pad_idx(x)] = v[m];
        }
        __syncthreads();
        block_fft<T, true>(rows, rmp, MS * RR, c.px, tw1);
        cl.sync();                               // (1) every row tile of this step is complete
        // ---- column phase: gather with the conjugate twiddle, F_N2^-1,
        // SE, SP, NORMC (+ snapshot), F_N2
        for (int idx = threadIdx.x; idx < ncol; idx += blockDim.x) {
            const int t = idx % CC, q = idx / CC, e = q % n2, m = q / n2;
            const cx<T>* src = cl.map_shared_rank(rows, e / RR);
            const cx<T> v = src[(m * RR + e % RR) * lp1 + pad_idx(x0 + t)];
            cols[(m * lpn + pad_idx(e)) * CC + t] = cmulc(v, twn[(size_t)(x0 + t) * c.fy[e]]);
        }
        __syncthreads();
        block_fft<T, true>(cols, cmp, MS * CC, c.py, tw2);
        cx<T>* snap = step == a.nsteps - 1 ? (cx<T>*)a.snap_last
                    : (step == a.nsteps - 2 ? (cx<T>*)a.snap_prev : nullptr);
        double acc[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] = 0.0;
        for (int p = threadIdx.x; p < n2 * CC; p += blockDim.x) {
            const int t = p % CC, e = p / CC;
            const int x = x0 + t + n1 * e;             // 1D grid index
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = cols[(m * lpn + pad_idx(e)) * CC + t];
            const cx<T> eV = pot_phase<T>(c, x, 0, 0);
            apply_se<T, MS>(c, v);
            apply_sp<T, MS>(c, eV, v);
            const double w = c.wx[x];
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
                cols[(m * lpn + pad_idx(e)) * CC + t] = v[m];
            }
            if (snap) {
#pragma unroll
                for (int m = 0; m < MS; ++m) snap[(size_t)m * np + x] = v[m];
            }
        }
        block_sum<MS>(acc, red, bsum);
        if (threadIdx.x < MS) {
            for (int q = 0; q < CL1D; ++q) cl.map_shared_rank(part, q)[rank * MS + threadIdx.x] = bsum[threadIdx.x];
        }
        block_fft<T, false>(cols, cmp, MS * CC, c.py, tw2);
        // ---- scatter with the twiddle into the owners' next rows
        for (int idx = threadIdx.x; idx < ncol; idx += blockDim.x) {
            const int t = idx % CC, q = idx / CC, e = q % n2, m = q / n2;
            cx<T>* dst = cl.map_shared_rank(next, e / RR);
            dst[(m * RR + e % RR) * lp1 + pad_idx(x0 + t)] =
                cmul(cols[(m * lpn + pad_idx(e)) * CC + t], twn[(size_t)(x0 + t) * c.fy[e]]);
        }
        cl.sync();                               // (2) next rows complete, block sums in place
        if (threadIdx.x == 0) {
            double n[MS], sc[MS], tot = 0;
            for (int m = 0; m < MS; ++m) {
                double s = 0;
                for (int q = 0; q < CL1D; ++q) s += part[q * MS + m];
                n[m] = s;
                tot += s;
            }
            const int rc = compute_scales<MS>(c, n, s_sig, sc);
            bool bad = !(tot == tot) || !(tot < 1e300);
            for (int m = 0; m < MS; ++m) { s_sc[m] = sc[m]; bad = bad || !(sc[m] == sc[m]); }
            if (rank == 0) {
                double* info = a.info;
                for (int m = 0; m < MS; ++m) { info[INFO_NORM + m] = n[m]; info[INFO_SC + m] = sc[m]; }
                info[INFO_TOTAL] = tot;
                sink_norms<MS>(c, n);
                info[INFO_SIG] = s_sig[0];
                info[INFO_SIG + 1] = s_sig[1];
                if (bad) info[INFO_ERR] = 1.0;
                if (rc) info[INFO_ERR] = (double)rc;
                if (step == a.nsteps - 2 && a.info_prev) {
                    for (int i = 0; i < INFO_LEN; ++i) a.info_prev[i] = info[i];
                }
            }
        }
        __syncthreads();
        // the next row phase loads its rows scaled by sc_m/N (the last step
        // leaves the scales pending in info)
        if (step + 1 < a.nsteps) {
            for (int idx = threadIdx.x; idx < nrow; idx += blockDim.x) {
                const int x = idx % n1, q = idx / n1, r = q % RR, m = q / RR;
                cx<T>& v = next[(m * RR + r) * lp1 + pad_idx(x)];
                v = cscale(v, (T)(s_sc[m] / (double)np));
            }
            __syncthreads();
        }
    }
    // Q back to global memory; the scales stay pending in info
    const cx<T>* fin = rowbuf + (a.nsteps & 1) * rtile;
    for (int idx = threadIdx.x; idx < nrow; idx += blockDim.x) {
        const int x = idx % n1, q = idx / n1, r = q % RR, m = q / RR;
        S[(size_t)m * np + (size_t)(row0 + r) * n1 + x] = fin[(m * RR + r) * lp1 + pad_idx(x)];
    }
}

// ------------------------------------------------------------- 1D steps
// One block holds PHI(NX, MS) and runs nsteps full split steps
// (cgpe1d.f90:434-472); psi is normalised in place every imaginary step so
// scale stays 1.  snap_prev receives the state after step nsteps-1.
template <typename T, int MS>
__global__ void __launch_bounds__(512, 1)
k_1d(StepConst c, OneDArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    cx<T>* sm = (cx<T>*)smraw;
    __shared__ double red[32 * (MS + 1)];
    __shared__ double bsum[MS];
    __shared__ double s_sc[MS];
    const int nx = c.nx;
    const int lp = padded_len(nx);
    const RowMap mp{lp};
    const cx<T>* tw = (const cx<T>*)c.twx;
    cx<T>* psi = (cx<T>*)a.psi;
    for (int idx = threadIdx.x; idx < MS * nx; idx += blockDim.x) {
        const int x = idx % nx, m = idx / nx;
        sm[m * lp + pad_idx(x)] = cscale(psi[(size_t)m * nx + x], (T)a.info[INFO_SC + m]);
    }
    __syncthreads();
    const T invn = (T)(1.0 / nx);
    for (int step = 0; step < a.nsteps; ++step) {
        block_fft<T, false>(sm, mp, MS, c.px, tw);
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = sm[m * lp + pad_idx(x)];
            const int ix = c.fx[x];
            apply_ke<T, MS>(c, ix, 0, 0, v);
            apply_soc<T, MS>(c, c.kx[ix], 0.0, v);
#pragma unroll
            for (int m = 0; m < MS; ++m) sm[m * lp + pad_idx(x)] = v[m];
        }
        __syncthreads();
        block_fft<T, true>(sm, mp, MS, c.px, tw);
        double acc[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) acc[m] = 0.0;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            cx<T> v[MS];
#pragma unroll
            for (int m = 0; m < MS; ++m) v[m] = cscale(sm[m * lp + pad_idx(x)], invn);
            apply_se<T, MS>(c, v);
            apply_sp<T, MS>(c, pot_phase<T>(c, x, 0, 0), v);
            const double w = c.wx[x];
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                acc[m] += w * ((double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y);
                sm[m * lp + pad_idx(x)] = v[m];
            }
        }
        block_sum<MS>(acc, red, bsum);
        if (threadIdx.x == 0) {
            double tot = 0, n[MS], sc[MS];
            for (int m = 0; m < MS; ++m) { n[m] = bsum[m]; tot += bsum[m]; }
            sink_norms<MS>(c, n);
            const int rc = compute_scales<MS>(c, n, a.info + INFO_SIG, sc);
            for (int m = 0; m < MS; ++m) s_sc[m] = sc[m];
            if (rc) a.info[INFO_ERR] = (double)rc;
            if (step == a.nsteps - 1) {
                for (int m = 0; m < MS; ++m) a.info[INFO_NORM + m] = bsum[m];
                a.info[INFO_TOTAL] = tot;
                if (!(tot == tot) || !(tot < 1e300)) a.info[INFO_ERR] = 1.0;
            }
        }
        __syncthreads();
        if (c.imag) {
            for (int idx = threadIdx.x; idx < MS * nx; idx += blockDim.x) {
                const int x = idx % nx, m = idx / nx;
                sm[m * lp + pad_idx(x)] = cscale(sm[m * lp + pad_idx(x)], (T)s_sc[m]);
            }
            __syncthreads();
        }
        if (a.snap_prev && step == a.nsteps - 2) {
            if (threadIdx.x < MS) a.info_prev[INFO_SC + threadIdx.x] = 1.0;
            cx<T>* sp = (cx<T>*)a.snap_prev;
            for (int idx = threadIdx.x; idx < MS * nx; idx += blockDim.x) {
                const int x = idx % nx, m = idx / nx;
                sp[(size_t)m * nx + x] = sm[m * lp + pad_idx(x)];
            }
        }
    }
    for (int idx = threadIdx.x; idx < MS * nx; idx += blockDim.x) {
        const int x = idx % nx, m = idx / nx;
        psi[(size_t)m * nx + x] = sm[m * lp + pad_idx(x)];
    }
    if (threadIdx.x < MS) a.info[INFO_SC + threadIdx.x] = 1.0;
}

// ------------------------------------------------------------ observables
// Energy, chemical potentials, magnetisation, rms sizes and norms of
// phi = scale*psi (ENERGY cgpe1d.f90:1077-1240 with DIFF diff.f90:4-33,
// RAD cgpe1d.f90:1036-1072, NORMC), and max |phi - phi_prev| (CONV,
// cgpe1d.f90:482).  Per-point densities are weighted by the separable Simpson
// weights wx(i) wy(j) wz(k) and reduced per block; the last block adds the
// block partials in order.
//
// The spin-orbit energy terms of the reference's six ENERGY variants are all
// Re sum_m phi_m^* [-2i (gx Fx Dx + gy Fy Dy + gz Fz Dz) phi]_m with the
// standard spin matrices (Fy = (F+ - F-)/2i); the chemical potential of
// component m takes the m-th row of the same sum.

// DIFF at index i of a periodic line of length n: 5-point centred formula at
// i < 4 and i >= n-4 (indices wrapped, diff.f90:16-24, 31-32), 9-point
// Richardson in between (diff.f90:26-29).
template <typename T, class LD>
__device__ __forceinline__ double2 dline(const LD& ld, int i, int n, double h) {
    auto P = [&](int q) { q = q < 0 ? q + n : (q >= n ? q - n : q); return ld(q); };
    double2 d;
    if (i >= 4 && i <= n - 5) {
        double2 a = P(i - 4), b = P(i - 3), cc = P(i - 2), e = P(i - 1), f = P(i + 1), g = P(i + 2), hh = P(i + 3), k = P(i + 4);
        d.x = (3.0 * a.x - 32.0 * b.x + 168.0 * cc.x - 672.0 * e.x + 672.0 * f.x - 168.0 * g.x + 32.0 * hh.x - 3.0 * k.x) / (840.0 * h);
        d.y = (3.0 * a.y - 32.0 * b.y + 168.0 * cc.y - 672.0 * e.y + 672.0 * f.y - 168.0 * g.y + 32.0 * hh.y - 3.0 * k.y) / (840.0 * h);
    } else {
        double2 a = P(i - 2), b = P(i - 1), e = P(i + 1), f = P(i + 2);
        d.x = (a.x - 8.0 * b.x + 8.0 * e.x - f.x) / (12.0 * h);
        d.y = (a.y - 8.0 * b.y + 8.0 * e.y - f.y) / (12.0 * h);
    }
    return d;
}

// (F_axis u)_m for the standard spin matrices; axis 0 = x, 1 = y, 2 = z.
template <int MS>
__device__ __forceinline__ double2 fmat_row(int axis, int m, const double2* u) {
    constexpr int S = MS / 2;
    double2 r = make_double2(0, 0);
    if (axis == 2) { r.x = (S - m) * u[m].x; r.y = (S - m) * u[m].y; return r; }
    // ladder coefficients c_m = <m|F|m+1> (m 0-based, spin projection S-m)
    auto cf = [&](int q) {  // between q and q+1
        const double mq = S - q;  // projection of q
        return 0.5 * sqrt((double)(S * (S + 1)) - mq * (mq - 1.0));
    };
    if (m > 0) {
        const double cc = cf(m - 1);  // element (m, m-1)
        if (axis == 0) { r.x += cc * u[m - 1].x; r.y += cc * u[m - 1].y; }
        else { r.x += -cc * u[m - 1].y; r.y += cc * u[m - 1].x; }         // +i c
    }
    if (m < MS - 1) {
        const double cc = cf(m);      // element (m, m+1)
        if (axis == 0) { r.x += cc * u[m + 1].x; r.y += cc * u[m + 1].y; }
        else { r.x += cc * u[m + 1].y; r.y += -cc * u[m + 1].x; }         // -i c
    }
    return r;
}

template <typename T, int MS>
__global__ void __launch_bounds__(256)
k_obs(StepConst c, ObsArgs a) {
    constexpr int NQ = 3 * MS + 2;  // norm[MS], e, mz, mu[MS], rms2[MS]
    __shared__ double red[32 * (NQ + 1)];
    __shared__ double bsum[NQ];
    __shared__ int is_last;
    const long long np = c.npts;
    const cx<T>* psi = (const cx<T>*)a.psi;
    const cx<T>* prev = (const cx<T>*)a.prev;
    double s_m[MS], sp_m[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) { s_m[m] = a.info[INFO_SC + m]; sp_m[m] = prev ? a.info_prev[INFO_SC + m] : 0.0; }
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
    double cmax = 0.0;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < np) {
        const int i = (int)(t % c.nx);
        const long long rr = t / c.nx;
        const int j = (int)(rr % c.ny), k = (int)(rr / c.ny);
        double2 P[MS], X[MS], Y[MS], Z[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) {
            const cx<T> v = psi[(size_t)m * np + t];
            P[m] = make_double2(s_m[m] * (double)v.x, s_m[m] * (double)v.y);
            if (prev) {
                const cx<T> u = prev[(size_t)m * np + t];
                const double dx = P[m].x - sp_m[m] * (double)u.x, dy = P[m].y - sp_m[m] * (double)u.y;
                cmax = fmax(cmax, sqrt(dx * dx + dy * dy));
            }
        }
        double w = c.wx[i];
        if (c.dim >= 2) w *= c.wy[j];
        if (c.dim >= 3) w *= c.wz[k];
        double a2[MS], rho = 0;
#pragma unroll
        for (int m = 0; m < MS; ++m) { a2[m] = P[m].x * P[m].x + P[m].y * P[m].y; rho += a2[m]; }
        double r2 = c.xg[i] * c.xg[i];
        if (c.dim >= 2) r2 += c.yg[j] * c.yg[j];
        if (c.dim >= 3) r2 += c.zg[k] * c.zg[k];
#pragma unroll
        for (int m = 0; m < MS; ++m) { acc[m] = w * a2[m]; acc[2 * MS + 2 + m] = w * r2 * a2[m]; }
        if (a.mode == OBS_FULL) {
            const size_t base = (size_t)j * c.nx + (size_t)k * c.nx * c.ny;
#pragma unroll
            for (int m = 0; m < MS; ++m) {
                const cx<T>* pm = psi + (size_t)m * np;
                const double s = s_m[m];
                auto lx = [&](int q) { cx<T> v = pm[base + q]; return make_double2(s * (double)v.x, s * (double)v.y); };
                X[m] = dline<T>(lx, i, c.nx, a.dx);
                Y[m] = make_double2(0, 0); Z[m] = make_double2(0, 0);
                if (c.dim >= 2) {
                    const size_t b2 = (size_t)i + (size_t)k * c.nx * c.ny;
                    auto ly = [&](int q) { cx<T> v = pm[b2 + (size_t)q * c.nx]; return make_double2(s * (double)v.x, s * (double)v.y); };
                    Y[m] = dline<T>(ly, j, c.ny, a.dy);
                }
                if (c.dim >= 3) {
                    const size_t b3 = (size_t)i + (size_t)j * c.nx;
                    const size_t st = (size_t)c.nx * c.ny;
                    auto lz = [&](int q) { cx<T> v = pm[b3 + (size_t)q * st]; return make_double2(s * (double)v.x, s * (double)v.y); };
                    Z[m] = dline<T>(lz, k, c.nz, a.dz);
                }
            }
            double V = c.vx[i];
            if (c.dim >= 2) V += c.vy[j];
            if (c.dim >= 3) V += c.vz[k];
            const double t0 = c.tau0, t1 = c.tau1, t2 = c.tau2;
            // spin densities (reference SX/SY conventions; FY enters squared
            // for spin-1 and through FX - i FY for spin-2)
            double fx = 0, fy = 0, fz = 0;
            constexpr int S = MS / 2;
            for (int m = 0; m < MS; ++m) fz += (S - m) * a2[m];
            for (int m = 0; m < MS - 1; ++m) {
                const double mq = S - m;
                const double cc = sqrt((double)(S * (S + 1)) - mq * (mq - 1.0));  // 2 <m|Fx|m+1>
                const double zr = P[m].x * P[m + 1].x + P[m].y * P[m + 1].y;       // Re conj(p_m) p_{m+1}
                const double zi = P[m].x * P[m + 1].y - P[m].y * P[m + 1].x;       // Im
                fx += cc * zr;
                fy += (MS == 3 ? -cc : cc) * zi;
            }
            // gradient energy and spin-orbit term
            double kin[MS], so[MS];
            for (int m = 0; m < MS; ++m) {
                kin[m] = X[m].x * X[m].x + X[m].y * X[m].y + Y[m].x * Y[m].x + Y[m].y * Y[m].y + Z[m].x * Z[m].x + Z[m].y * Z[m].y;
                double2 gx = fmat_row<MS>(0, m, X);
                double2 gy = fmat_row<MS>(1, m, Y);
                double2 gz = fmat_row<MS>(2, m, Z);
                double2 g;
                g.x = c.gx * gx.x + (c.dim >= 2 ? c.gy * gy.x : 0.0) + (c.dim >= 3 ? c.gz * gz.x : 0.0);
                g.y = c.gx * gx.y + (c.dim >= 2 ? c.gy * gy.y : 0.0) + (c.dim >= 3 ? c.gz * gz.y : 0.0);
                // Re conj(P_m) (-2i g) = 2 Re(-i conj(P) g) = 2 (P.x g.y - P.y g.x)
                so[m] = 2.0 * (P[m].x * g.y - P[m].y * g.x);
            }
            double e = V * rho + t0 * rho * rho / 2.0 + t1 * (fx * fx + fy * fy + fz * fz) / 2.0;
            double mu[MS];
            if constexpr (MS == 3) {
                // Re(conj(p3) p2^2 conj(p1)) and Re(p1 p3 conj(p2)^2)
                const double2 p22 = make_double2(P[1].x * P[1].x - P[1].y * P[1].y, 2 * P[1].x * P[1].y);
                const double2 p13 = make_double2(P[0].x * P[2].x - P[0].y * P[2].y, P[0].x * P[2].y + P[0].y * P[2].x);
                const double re_x = p22.x * p13.x + p22.y * p13.y;  // Re(p2^2 conj(p1 p3))
                mu[0] = V * a2[0] + t0 * rho * a2[0] + t1 * (a2[0] + a2[1] - a2[2]) * a2[0] + t1 * re_x;
                mu[1] = V * a2[1] + t0 * rho * a2[1] + t1 * (a2[0] + a2[2]) * a2[1] + 2.0 * t1 * re_x;
                mu[2] = V * a2[2] + t0 * rho * a2[2] + t1 * (a2[1] + a2[2] - a2[0]) * a2[2] + t1 * re_x;
            } else {
                double2 v5[5];
                for (int m = 0; m < 5; ++m) v5[m] = P[m];
                double2 cc6[6];
                couplings2<double>(v5, t1, t2, cc6);
                // theta = (2 p1 p5 - 2 p2 p4 + p3^2)/sqrt5
                double2 th;
                th.x = (2 * (v5[0].x * v5[4].x - v5[0].y * v5[4].y) - 2 * (v5[1].x * v5[3].x - v5[1].y * v5[3].y)
                        + (v5[2].x * v5[2].x - v5[2].y * v5[2].y)) / sqrt(5.0);
                th.y = (2 * (v5[0].x * v5[4].y + v5[0].y * v5[4].x) - 2 * (v5[1].x * v5[3].y + v5[1].y * v5[3].x)
                        + 2 * v5[2].x * v5[2].y) / sqrt(5.0);
                e += t2 * (th.x * th.x + th.y * th.y) / 2.0;
                double2 hv[5];
                hmul<double>(cc6, v5, hv);
                const double fz2 = fz;
                const double d0[5] = {V + t0 * rho + 2.0 * t1 * fz2 + 0.4 * t2 * a2[4],
                                      V + t0 * rho + t1 * fz2 + 0.4 * t2 * a2[3],
                                      V + t0 * rho + 0.2 * t2 * a2[2],
                                      V + t0 * rho - t1 * fz2 + 0.4 * t2 * a2[1],
                                      V + t0 * rho - 2.0 * t1 * fz2 + 0.4 * t2 * a2[0]};
                for (int m = 0; m < MS; ++m)
                    mu[m] = d0[m] * a2[m] + (hv[m].x * v5[m].x + hv[m].y * v5[m].y);  // Re((H p)_m conj(p_m))
            }
            for (int m = 0; m < MS; ++m) { e += kin[m] + so[m]; mu[m] += so[m] + kin[m]; }
            acc[MS] = w * e;
            double mz = 0;
            for (int m = 0; m < MS; ++m) mz += (S - m) * a2[m];
            acc[MS + 1] = w * mz;
            for (int m = 0; m < MS; ++m) acc[MS + 2 + m] = w * mu[m];
        }
    }
    block_sum<NQ>(acc, red, bsum);
    const double bm = block_max(cmax, red);
    if (threadIdx.x < NQ) a.part[(size_t)blockIdx.x * (NQ + 1) + threadIdx.x] = bsum[threadIdx.x];
    if (threadIdx.x == 0) a.part[(size_t)blockIdx.x * (NQ + 1) + NQ] = bm;
    __threadfence();
    if (threadIdx.x == 0) is_last = (atomicAdd(a.counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    // the whole last block adds the block partials in a fixed order (thread t
    // takes blocks t, t+256, ..., then the block tree) and takes their max
    __threadfence();
    const int nb = gridDim.x;
    double r[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) r[q] = 0.0;
    double mx = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const double* pb = a.part + (size_t)b * (NQ + 1);
#pragma unroll
        for (int q = 0; q < NQ; ++q) r[q] += __ldcg(pb + q);
        mx = fmax(mx, __ldcg(pb + NQ));
    }
    block_sum<NQ>(r, red, bsum);
    const double gmax = block_max(mx, red);
    if (threadIdx.x == 0) {
        for (int q = 0; q < NQ; ++q) red[q] = bsum[q];
        red[NQ] = gmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double* o = a.out;
        double tot = 0;
        for (int m = 0; m < MS; ++m) { o[OBS_NORM + m] = red[m]; tot += red[m]; }
        o[OBS_EN] = red[MS] / tot;
        o[OBS_MZ] = red[MS + 1];
        for (int m = 0; m < MS; ++m) o[OBS_MU + m] = red[MS + 2 + m] / (red[m] + 1.0e-40);
        for (int m = 0; m < MS; ++m) o[OBS_RMS + m] = sqrt(red[2 * MS + 2 + m]);
        o[OBS_CONV] = red[NQ];
        o[OBS_TOTAL] = tot;
        if (a.mode == OBS_NORMALIZE) {
            // NORMT: the pending scales absorb 1/sqrt(total)
            for (int m = 0; m < MS; ++m) a.info[INFO_SC + m] = a.info[INFO_SC + m] / sqrt(tot);
        }
        *a.counter = 0u;
    }
}

// psi_m <- sc_m psi_m (folds the pending scales into the state); n2 counts
// reals, per2 = 2*NPTS reals per component.
template <typename T>
__global__ void k_apply_scale(T* psi, long long n2, long long per2, double* info) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
        psi[t] = (T)(info[INFO_SC + t / per2] * (double)psi[t]);
}

// Per-step read-back of NORMC: copies the MS component norms to dst, which is
// device memory or pinned host memory that the device addresses directly.  As
// a programmatic dependent launch it waits for the step's last pass and keeps
// the step chain on the SMs instead of a copy-engine transfer between steps.
static __global__ void k_norms_out(const double* __restrict__ info, double* __restrict__ dst, int ms) {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    if ((int)threadIdx.x < ms) dst[threadIdx.x] = info[INFO_NORM + threadIdx.x];
}

// Unfused single operators on a full real/Fourier-space buffer (parity
// checks of individual reference subroutines).
template <typename T, int MS>
__global__ void k_pointwise_op(StepConst c, PointArgs a) {
    const long long np = c.npts;
    cx<T>* psi = (cx<T>*)a.psi;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % c.nx);
        const long long rr = t / c.nx;
        const int j = (int)(rr % c.ny), k = (int)(rr / c.ny);
        cx<T> v[MS];
#pragma unroll
        for (int m = 0; m < MS; ++m) v[m] = psi[(size_t)m * np + t];
        switch (a.op) {
            case OP_KE: apply_ke<T, MS>(c, i, j, k, v); break;
            case OP_SOC: apply_soc<T, MS>(c, c.kx[i], c.dim >= 2 ? c.ky[j] : 0.0, v); break;
            case OP_SE: apply_se<T, MS>(c, v); break;
            case OP_SP: apply_sp<T, MS>(c, pot_phase<T>(c, i, j, k), v); break;
            case OP_SCALE: {
#pragma unroll
                for (int m = 0; m < MS; ++m) v[m] = cscale(v[m], (T)a.factor);
            } break;
        }
#pragma unroll
        for (int m = 0; m < MS; ++m) psi[(size_t)m * np + t] = v[m];
    }
}

}  // namespace fgpe
