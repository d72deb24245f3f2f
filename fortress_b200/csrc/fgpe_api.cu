// fgpe_api.cu -- host side of the C ABI declared in include/fgpe.h.
//
// A handle owns every device buffer of one propagator instance:
//   S     x-spectral spinor (2D/3D), complex T, PHI layout (NX,NY,NZ,M)
//   psi   real-space spinor (the current state is info[SCALE] * psi)
//   prev  real-space spinor one step older (for CONV)
//   tables: k grids, x grids, Simpson weights, trap parts, twiddles, KE factors
// Launch shapes (rows per block, column tile widths, threads) are chosen once
// at creation from the grid size and the shared-memory budget.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fgpe.h"
#include "fgpe_kernels.cuh"
#include "fgpe_fast.cuh"
#include "fgpe_group.cuh"
#include "fgpe_persist.h"
#include "fno_kernels.cuh"
#include "fno_gemm_tc.cuh"
#include "../../include/fno.h"

using namespace fgpe;

namespace {

const double kPi = 3.14159265358979323846264338327950288;
thread_local std::string g_last_error;

struct Launch {
    int T = 0;
    size_t smem = 0;
    int tile = 0;          // rows (row pass) or TX (column pass)
    dim3 grid;
};

}  // namespace

struct fgpe_s {
    fgpe_params p;
    int ms = 0;
    long long npts = 0;
    int fp32 = 0;
    size_t cs = 16;        // bytes per complex element in device buffers
    cudaStream_t st = nullptr;
    bool own_stream = false;
    StepConst sc;
    void *S = nullptr, *psi = nullptr, *prev = nullptr, *stage = nullptr;
    double *info = nullptr, *info_prev = nullptr, *obs = nullptr, *part = nullptr;
    unsigned* counters = nullptr;
    int* pmap = nullptr;         // position->frequency maps of the three axes
    double* dtab = nullptr;
    void* ctab = nullptr;
    double* h_small = nullptr;   // pinned, 64 doubles
    Launch row, col[3], k1, obsl;
    // 1D lines too long for one block: N = n1*n2 split (k_r1d / k_c1d)
    bool split1d = false;
    int n1 = 0, n2 = 0;
    Launch r1d, c1d;
    const void *twn = nullptr, *tw1 = nullptr, *tw2 = nullptr;
    // the same split on one thread-block cluster for a whole call (k_cl1d)
    bool cl1d = false;
    size_t cl1d_smem = 0;
    // CUDA graph of kBulkSteps whole steps without snapshots, replayed for
    // the bulk of multi-step calls (built on first use, dropped when the
    // kernel choice changes)
    cudaGraphExec_t bulk = nullptr;
    bool bulk_off = false;
    bool fast_row = false, fast_col[3] = {false, false, false};
    bool has_fast_row = false, has_fast_col[3] = {false, false, false};
    int fast_row_grid = 0, fast_col_grid[3] = {0, 0, 0};
    bool col_wide[3] = {false, false, false};   // column pass uses the wide tiles
    // column passes that transform forward and back in one launch (q2D y,
    // 3D z) on the radix-16 plan (cplan pv 3) with its own position map
    bool col_r16[3] = {false, false, false};
    int col_r16_grid[3] = {0, 0, 0};
    int* pmap16 = nullptr;
    const int* fline16[3] = {nullptr, nullptr, nullptr};
    // row pass with one warp per x row (k_row_warp), where a row fits 16 KB
    bool has_warp_row = false, warp_row = false;
    int warp_row_grid = 0;
    bool psi_valid = false, S_valid = false, prev_valid = false, norms_valid = false, has_state = false;
    long long launches = 0;
    std::string msg;
    // kernel timing (fgpe_profile_enable)
    int device = 0;              // ordinal of the device the handle was created on
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> ev_rec;   // (class, pool index of start)
    double prof_ms[4] = {0, 0, 0, 0};
    long long prof_n[4] = {0, 0, 0, 0};
};

namespace {

int fail(fgpe_t* h, int code, const std::string& m) {
    if (h) h->msg = m;
    g_last_error = m;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(h, FGPE_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool plan_fft(int n, FftPlan* pl) {
    pl->n = n; pl->nf = 0;
    int m = n;
    std::vector<int> f;
    while (m % 8 == 0) { f.push_back(8); m /= 8; }
    if (m % 4 == 0) { f.push_back(4); m /= 4; }
    if (m % 2 == 0) { f.push_back(2); m /= 2; }
    while (m % 3 == 0) { f.push_back(3); m /= 3; }
    while (m % 5 == 0) { f.push_back(5); m /= 5; }
    if (m != 1 || f.size() > 16) return false;
    for (size_t i = 0; i < f.size(); ++i) pl->r[i] = f[i];
    pl->nf = (int)f.size();
    return true;
}

// simpson.f90:4-21 applied to unit vectors: the weight of every node.
std::vector<double> simpson_weights(int n, double dx) {
    std::vector<double> w(n, 0.0);
    if (n == 1) { w[0] = 1.0; return w; }
    std::vector<double> f(n, 0.0);
    for (int t = 0; t < n; ++t) {
        std::fill(f.begin(), f.end(), 0.0);
        f[t] = 1.0;
        double f1 = f[1] + f[n - 5], f2 = f[2];
        for (int i = 4; i <= n - 6; i += 2) { f1 += f[i - 1]; f2 += f[i]; }
        w[t] = dx * (f[0] + 4.0 * f1 + 2.0 * f2 + f[n - 4]) / 3.0 + 3.0 * dx * (f[n - 4] + 3.0 * (f[n - 3] + f[n - 2]) + f[n - 1]) / 8.0;
    }
    return w;
}

// Allow each kernel the opt-in shared-memory maximum minus its static part.
template <class K> cudaError_t allow_smem(K kern) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

template <class K> cudaError_t allow_smem_exact(K kern, size_t bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T, int MS> cudaError_t set_smem_attrs() {
    cudaError_t e = allow_smem(k_row<T, MS>);
    if (e == cudaSuccess) e = allow_smem(k_col<T, MS>);
    if (e == cudaSuccess) e = allow_smem(k_1d<T, MS>);
    if (e == cudaSuccess) e = allow_smem(k_r1d<T, MS>);
    if (e == cudaSuccess) e = allow_smem(k_c1d<T, MS>);
    if (e == cudaSuccess) e = allow_smem(k_cl1d<T, MS>);
    return e;
}

// ------------------------------------------------ specialised fast kernels
// Line lengths with compiled persistent kernels; other sizes use the generic
// kernels (same layout and results).
constexpr int kFastN[] = {128, 192, 256, 384, 512};

#ifndef FGPE_COL_TX32
#define FGPE_COL_TX32 2
#endif
template <typename T> constexpr int col_tx() { return sizeof(T) == 8 ? 2 : FGPE_COL_TX32; }
// Rows per row-kernel tile (FGPE_ROW_R256 fixes it for 256-point rows at
// build time).
#ifndef FGPE_ROW_R256
#define FGPE_ROW_R256 0
#endif
constexpr int row_r(int n) { return n >= 384 ? 1 : (n == 256 && FGPE_ROW_R256 ? FGPE_ROW_R256 : 512 / n); }
constexpr int fast_threads(int tot) {
    const int iter = (tot + 511) / 512;
    const int per = (tot + iter - 1) / iter;
    return (per + 31) / 32 * 32;
}
// Thread counts of the size-specialised kernels: one radix-8 butterfly per
// thread and pass unless FGPE_ROW_TH / FGPE_COL_TH fix them at build time.
#ifndef FGPE_ROW_TH
#define FGPE_ROW_TH 0
#endif
#ifndef FGPE_COL_TH
#define FGPE_COL_TH 0
#endif
template <typename T, int MS, int N> constexpr int row_th() {
    return FGPE_ROW_TH ? FGPE_ROW_TH : fast_threads(MS * row_r(N) * N / 8);
}
template <typename T, int MS, int N> constexpr int col_th() {
    return FGPE_COL_TH ? FGPE_COL_TH : fast_threads(MS * col_tx<T>() * N / 8);
}
// Wide column tiles: FGPE_COL_WIDE_BYTES (default 128) contiguous bytes of x
// per line element (8 complex doubles, 16 complex floats), for grids with
// enough tiles (3D) where the 32-byte segments of the narrow tiles waste DRAM
// bursts; FGPE_COL_NBUF_W shared buffers per block (default FGPE_COL_NBUF).
#ifndef FGPE_COL_WIDE_BYTES
#define FGPE_COL_WIDE_BYTES 128
#endif
#ifndef FGPE_COL_NBUF_W
#define FGPE_COL_NBUF_W FGPE_COL_NBUF
#endif
template <typename T> constexpr int col_txw() { return FGPE_COL_WIDE_BYTES / (int)sizeof(cx<T>); }
template <typename T, int MS, int N> constexpr size_t col_smem_w() {
    return (size_t)FGPE_COL_NBUF_W * MS * cpad(N) * col_txw<T>() * sizeof(cx<T>);
}
template <typename T, int MS, int N> constexpr bool wide_ok() { return col_smem_w<T, MS, N>() <= 113 * 1024; }
template <typename T, int MS, int N> constexpr int col_th_w() { return fast_threads(MS * col_txw<T>() * N / 8); }
template <typename T, int MS, int N> constexpr size_t row_smem() {
    return ((size_t)FGPE_ROW_NBUF * MS * row_r(N) * cpad(N) + (FGPE_TW_SMEM ? N : 0)) * sizeof(cx<T>);
}
template <typename T, int MS, int N> constexpr size_t col_smem() {
    return ((size_t)FGPE_COL_NBUF * MS * cpad(N) * col_tx<T>() + (FGPE_TW_SMEM ? N : 0)) * sizeof(cx<T>);
}

template <class K> int grid_for(K kern, int th, size_t smem, int ntiles) {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (allow_smem_exact(kern, smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, th, smem) != cudaSuccess || per < 1) return 0;
    return std::min(ntiles, per * nsm);
}

template <typename T, int MS, int N> int setup_fast_row(fgpe_t* h) {
    const int rows = h->p.ny * h->p.nz;
    if (rows % row_r(N)) return 0;
    return grid_for(k_row_fast<T, MS, N, row_r(N), row_th<T, MS, N>()>, row_th<T, MS, N>(), row_smem<T, MS, N>(),
                    rows / row_r(N));
}
// Grid of the column kernel for one axis (0: none); *wide tells whether the
// wide tiles were chosen: they need 128-byte rows of x and at least four
// waves of tiles, so that their fewer, larger tiles still fill the GPU.
template <typename T, int MS, int N> int setup_fast_col(fgpe_t* h, int n_other, bool* wide) {
    *wide = false;
    if constexpr (wide_ok<T, MS, N>()) {
        if (h->p.nx % col_txw<T>() == 0) {
            const int ntw = (h->p.nx / col_txw<T>()) * n_other;
            const int g = grid_for(k_col_fast<T, MS, N, col_txw<T>(), col_th_w<T, MS, N>(), FGPE_COL_NBUF_W>, col_th_w<T, MS, N>(),
                                   col_smem_w<T, MS, N>(), ntw);
            if (g > 0 && ntw >= 4 * g) { *wide = true; return g; }
        }
    }
    if (h->p.nx % col_tx<T>()) return 0;
    return grid_for(k_col_fast<T, MS, N, col_tx<T>(), col_th<T, MS, N>()>, col_th<T, MS, N>(), col_smem<T, MS, N>(),
                    (h->p.nx / col_tx<T>()) * n_other);
}
// Radix-16 plan for the column passes that transform forward and back in one
// launch, on lengths where it saves a radix pass (128, 256, 384); build knob
// FGPE_COL_R16 (0: every column pass on the handle's plan).
#ifndef FGPE_COL_R16
#define FGPE_COL_R16 1
#endif
constexpr bool r16_len(int n) { return FGPE_COL_R16 && cplan(n, 3).r[0] == 16; }
// Grid of the radix-16 form of the column kernel with the same tiles as
// setup_fast_col chose (0: not available).
template <typename T, int MS, int N> int setup_fast_col_r16(fgpe_t* h, int n_other, bool wide) {
    if constexpr (r16_len(N)) {
        if constexpr (wide_ok<T, MS, N>()) {
            if (wide)
                return grid_for(k_col_fast<T, MS, N, col_txw<T>(), col_th_w<T, MS, N>(), FGPE_COL_NBUF_W, 3>,
                                col_th_w<T, MS, N>(), col_smem_w<T, MS, N>(), (h->p.nx / col_txw<T>()) * n_other);
        }
        if (!wide)
            return grid_for(k_col_fast<T, MS, N, col_tx<T>(), col_th<T, MS, N>(), FGPE_COL_NBUF, 3>, col_th<T, MS, N>(),
                            col_smem<T, MS, N>(), (h->p.nx / col_tx<T>()) * n_other);
    }
    return 0;
}
// Warp-row kernel: rows of MS lines up to 16 KB (FP64 spin-1 to 256 points,
// spin-2 to 128; FP32 spin-1 to 512, spin-2 to 256); warps per block so that
// two blocks of NBUF rows per warp fit the shared memory.
template <typename T, int MS, int N> constexpr size_t wrow_tile() { return (size_t)MS * cpad(N) * sizeof(cx<T>); }
template <typename T, int MS, int N> constexpr bool wrow_ok() { return wrow_tile<T, MS, N>() <= 16 * 1024; }
template <typename T, int MS, int N> constexpr int wrow_wpb() {
    const int w = (int)((110 * 1024) / (wrow_tile<T, MS, N>() * FGPE_WROW_NBUF));
    return w < 1 ? 1 : (w > 8 ? 8 : w);
}
template <typename T, int MS, int N> int setup_warp_row(fgpe_t* h) {
    if constexpr (!wrow_ok<T, MS, N>()) {
        return 0;
    } else {
        constexpr int W = wrow_wpb<T, MS, N>();
        const int rows = h->p.ny * h->p.nz;
        return grid_for(k_row_warp<T, MS, N, W, FGPE_WROW_NBUF>, W * 32,
                        (size_t)W * FGPE_WROW_NBUF * wrow_tile<T, MS, N>(), (rows + W - 1) / W);
    }
}

// The size-specialised kernels go out as programmatic dependent launches
// (outside stream capture): the next pass is launched while the previous one
// drains and waits on griddepcontrol.wait before it touches the state.  Their
// grids are one wave of resident blocks, so a waiting block never keeps the
// previous pass from finishing.
template <class K, class A>
void launch_pdl(fgpe_t* h, K kern, int grid, int threads, size_t smem, const A& a) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(h->st, &cs);
    if (cs != cudaStreamCaptureStatusNone) {
        kern<<<grid, threads, smem, h->st>>>(h->sc, a);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, h->sc, a);
}
template <typename T, int MS, int N> void run_fast_row(fgpe_t* h, const RowArgs& a) {
    launch_pdl(h, k_row_fast<T, MS, N, row_r(N), row_th<T, MS, N>()>, h->fast_row_grid, row_th<T, MS, N>(),
               row_smem<T, MS, N>(), a);
}
template <typename T, int MS, int N> void run_warp_row(fgpe_t* h, const RowArgs& a) {
    if constexpr (wrow_ok<T, MS, N>()) {
        constexpr int W = wrow_wpb<T, MS, N>();
        launch_pdl(h, k_row_warp<T, MS, N, W, FGPE_WROW_NBUF>, h->warp_row_grid, W * 32,
                   (size_t)W * FGPE_WROW_NBUF * wrow_tile<T, MS, N>(), a);
    }
}
template <typename T, int MS, int N> void run_fast_col(fgpe_t* h, int axis, const ColArgs& a0, bool r16) {
    ColArgs a = a0;
    if constexpr (r16_len(N)) {
        if (r16) {
            a.fline = h->fline16[axis];
            if constexpr (wide_ok<T, MS, N>()) {
                if (h->col_wide[axis]) {
                    launch_pdl(h, k_col_fast<T, MS, N, col_txw<T>(), col_th_w<T, MS, N>(), FGPE_COL_NBUF_W, 3>,
                               h->col_r16_grid[axis], col_th_w<T, MS, N>(), col_smem_w<T, MS, N>(), a);
                    return;
                }
            }
            launch_pdl(h, k_col_fast<T, MS, N, col_tx<T>(), col_th<T, MS, N>(), FGPE_COL_NBUF, 3>, h->col_r16_grid[axis],
                       col_th<T, MS, N>(), col_smem<T, MS, N>(), a);
            return;
        }
    }
    if constexpr (wide_ok<T, MS, N>()) {
        if (h->col_wide[axis]) {
            launch_pdl(h, k_col_fast<T, MS, N, col_txw<T>(), col_th_w<T, MS, N>(), FGPE_COL_NBUF_W>, h->fast_col_grid[axis],
                       col_th_w<T, MS, N>(), col_smem_w<T, MS, N>(), a);
            return;
        }
    }
    launch_pdl(h, k_col_fast<T, MS, N, col_tx<T>(), col_th<T, MS, N>()>, h->fast_col_grid[axis], col_th<T, MS, N>(),
               col_smem<T, MS, N>(), a);
}

#define FAST_SWITCH(n, CALL)            \
    switch (n) {                         \
        case 128: CALL(128); break;      \
        case 192: CALL(192); break;      \
        case 256: CALL(256); break;      \
        case 384: CALL(384); break;      \
        case 512: CALL(512); break;      \
        default: break;                  \
    }

bool fast_size(int n) {
    for (int v : kFastN) if (v == n) return true;
    return false;
}

// Event pair around one launch when profiling is on.
struct ProfScope {
    fgpe_t* h; int cls; int idx = -1;
    ProfScope(fgpe_t* hh, int c) : h(hh), cls(c) {
        if (!h->prof) return;
        idx = (int)h->ev_rec.size() * 2;
        while ((int)h->ev_pool.size() < idx + 2) {
            cudaEvent_t e; cudaEventCreate(&e); h->ev_pool.push_back(e);
        }
        cudaEventRecord(h->ev_pool[idx], h->st);
    }
    ~ProfScope() {
        if (idx < 0) return;
        cudaEventRecord(h->ev_pool[idx + 1], h->st);
        h->ev_rec.push_back({cls, idx});
    }
};

// ---------------------------------------------------------------- launches
template <typename T, int MS>
void launch_row(fgpe_t* h, int mode, void* snap) {
    RowArgs a;
    a.S = h->S; a.psi = h->psi; a.snap = snap; a.part = h->part; a.counter = h->counters;
    a.info = h->info; a.rows = h->row.tile; a.mode = mode;
    ProfScope ps(h, 0);
    if (h->warp_row && mode == ROW_FULL) {
#define RUNW(NN) run_warp_row<T, MS, NN>(h, a)
        FAST_SWITCH(h->p.nx, RUNW)
#undef RUNW
        h->launches++;
        return;
    }
    if (h->fast_row) {
#define RUNR(NN) run_fast_row<T, MS, NN>(h, a)
        FAST_SWITCH(h->p.nx, RUNR)
#undef RUNR
        h->launches++;
        return;
    }
    k_row<T, MS><<<h->row.grid, h->row.T, h->row.smem, h->st>>>(h->sc, a);
    h->launches++;
}

template <typename T, int MS>
void launch_col(fgpe_t* h, int axis, int flags) {
    ColArgs a;
    a.S = h->S;
    a.tw = axis == 1 ? h->sc.twy : h->sc.twz;
    a.plan = axis == 1 ? h->sc.py : h->sc.pz;
    a.info = h->info;
    a.cfac = 1.0 / (double)h->npts;
    a.n = axis == 1 ? h->p.ny : h->p.nz;
    a.axis_stride = axis == 1 ? h->p.nx : (long long)h->p.nx * h->p.ny;
    a.other_stride = h->p.dim == 2 ? 0 : (axis == 1 ? (long long)h->p.nx * h->p.ny : h->p.nx);
    a.tx = h->col[axis].tile;
    a.flags = flags;
    a.n_other = h->p.dim == 2 ? 1 : (axis == 1 ? h->p.nz : h->p.ny);
    a.axis = axis;
    a.fline = axis == 1 ? h->sc.fy : h->sc.fz;
    // radix-16 lines: a pass that transforms forward and back (q2D y, 3D z),
    // or the y passes of a 3D step when all its column passes run the
    // size-specialised kernels (the y spectra then use that plan throughout
    // the step: the z pass reads ky through fother)
    const bool y16 = h->p.dim == 3 && (flags & COL_STEP) && h->col_r16[1] && h->fast_col[1] && h->fast_col[2];
    a.fother = y16 ? h->fline16[1] : h->sc.fy;
    const bool r16 = h->col_r16[axis] && ((axis == 1 && y16) || ((flags & COL_FWD) && (flags & COL_INV)));
    ProfScope ps(h, axis);
    if (h->fast_col[axis]) {
#define RUNC(NN) run_fast_col<T, MS, NN>(h, axis, a, r16)
        FAST_SWITCH(a.n, RUNC)
#undef RUNC
        h->launches++;
        return;
    }
    k_col<T, MS><<<h->col[axis].grid, h->col[axis].T, h->col[axis].smem, h->st>>>(h->sc, a);
    h->launches++;
}

template <typename T, int MS>
void launch_obs(fgpe_t* h, int mode, bool with_prev) {
    ObsArgs a;
    a.psi = h->psi; a.prev = with_prev ? h->prev : nullptr;
    a.info = h->info; a.info_prev = h->info_prev;
    a.part = h->part; a.counter = h->counters + 1; a.out = h->obs;
    a.dx = h->p.dx; a.dy = h->p.dy; a.dz = h->p.dz; a.mode = mode;
    k_obs<T, MS><<<h->obsl.grid, 256, 0, h->st>>>(h->sc, a);
    h->launches++;
}

template <typename T, int MS>
void launch_point(fgpe_t* h, int op, double factor) {
    PointArgs a; a.psi = h->psi; a.op = op; a.factor = factor;
    const long long blocks = std::min<long long>((h->npts + 255) / 256, 148LL * 16);
    k_pointwise_op<T, MS><<<(unsigned)blocks, 256, 0, h->st>>>(h->sc, a);
    h->launches++;
}

template <typename T, int MS>
void launch_1d(fgpe_t* h, int nsteps, void* snap_prev) {
    OneDArgs a;
    a.psi = h->psi; a.snap_prev = snap_prev; a.info = h->info; a.info_prev = h->info_prev;
    a.nsteps = nsteps;
    ProfScope ps(h, 3);
    k_1d<T, MS><<<1, h->k1.T, h->k1.smem, h->st>>>(h->sc, a);
    h->launches++;
}

template <typename T, int MS>
Split1dArgs split_args(fgpe_t* h, int mode, void* snap) {
    Split1dArgs a;
    a.S = h->S; a.psi = h->psi; a.snap = snap;
    a.twn = h->twn; a.tw1 = h->tw1; a.tw2 = h->tw2;
    a.part = h->part; a.counter = h->counters; a.info = h->info;
    a.n1 = h->n1; a.n2 = h->n2; a.mode = mode; a.tile = 0;
    return a;
}

template <typename T, int MS>
void launch_r1d(fgpe_t* h) {
    Split1dArgs a = split_args<T, MS>(h, C1D_FULL, nullptr);
    a.tile = h->r1d.tile;
    ProfScope ps(h, 0);
    k_r1d<T, MS><<<h->r1d.grid, h->r1d.T, h->r1d.smem, h->st>>>(h->sc, a);
    h->launches++;
}

template <typename T, int MS>
void launch_c1d(fgpe_t* h, int mode, void* snap) {
    Split1dArgs a = split_args<T, MS>(h, mode, snap);
    a.tile = h->c1d.tile;
    ProfScope ps(h, 1);
    k_c1d<T, MS><<<h->c1d.grid, h->c1d.T, h->c1d.smem, h->st>>>(h->sc, a);
    h->launches++;
}

// The cluster form of the 1D split when n1 and n2 divide over the cluster,
// both halves of Q fit the CTAs' shared memory and the cluster can be
// resident; otherwise h->cl1d stays false and the two passes run.
template <typename T, int MS>
void setup_cl1d(fgpe_t* h) {
    h->cl1d = false;
    if (h->n1 % CL1D || h->n2 % CL1D) return;
    const size_t smem = (size_t)MS * (2 * (size_t)(h->n2 / CL1D) * padded_len(h->n1) +
                                      (size_t)padded_len(h->n2) * (h->n1 / CL1D)) * sizeof(cx<T>);
    if (smem > 200 * 1024) return;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL1D);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, k_cl1d<T, MS>, &cfg) != cudaSuccess || nc < 1) {
        cudaGetLastError();
        return;
    }
    h->cl1d = true;
    h->cl1d_smem = smem;
}

// All nsteps of a call in one launch of the cluster kernel.
template <typename T, int MS>
void launch_cl1d(fgpe_t* h, int nsteps, void* snap_last, void* snap_prev) {
    Cluster1dArgs a;
    a.S = h->S; a.snap_last = snap_last; a.snap_prev = snap_prev;
    a.twn = h->twn; a.tw1 = h->tw1; a.tw2 = h->tw2;
    a.info = h->info; a.info_prev = h->info_prev;
    a.n1 = h->n1; a.n2 = h->n2; a.nsteps = nsteps;
    ProfScope ps(h, 3);
    k_cl1d<T, MS><<<CL1D, 256, h->cl1d_smem, h->st>>>(h->sc, a);
    h->launches++;
}

// Kernel launches of one step call of k whole steps on h.
static long long step_launches(const fgpe_t* h, int k) {
    if (h->cl1d) return 1;
    return (long long)k * (h->p.dim == 1 ? (h->split1d ? 2 : 1) : (h->p.dim == 2 ? 2 : 4));
}

// dispatch on (precision, spin)
#define DISPATCH(h, FN, ...)                                                  \
    do {                                                                      \
        if ((h)->fp32) {                                                      \
            if ((h)->ms == 3) FN<float, 3>(__VA_ARGS__); else FN<float, 5>(__VA_ARGS__);   \
        } else {                                                              \
            if ((h)->ms == 3) FN<double, 3>(__VA_ARGS__); else FN<double, 5>(__VA_ARGS__); \
        }                                                                     \
    } while (0)

template <typename T>
__global__ void k_export(const T* psi, double* out, long long n2, long long per2, const double* info) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
        out[t] = info[INFO_SC + t / per2] * (double)psi[t];
}
template <typename T>
__global__ void k_import(const double* in, T* psi, long long n2) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
        psi[t] = (T)in[t];
}

int check_err(fgpe_t* h) {
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return FGPE_OK;
}

// Digit-reversed position -> frequency index of the in-place DIF transform
// with radices r[0..nf-1] (r[0] acts on the longest stride).
std::vector<int> position_map(const FftPlan& pl) {
    const int n = pl.n;
    std::vector<int> f(n);
    for (int k = 0; k < n; ++k) {
        int rem = k, pos = 0, block = n;
        for (int p = 0; p < pl.nf; ++p) {
            const int d = rem % pl.r[p];
            rem /= pl.r[p];
            block /= pl.r[p];
            pos += d * block;
        }
        f[pos] = k;
    }
    return f;
}

// dst[natural] = src[position] (to_natural) or dst[position] = src[natural].
template <typename T, int MS>
__global__ void k_permute(StepConst c, const cx<T>* src, cx<T>* dst, int to_natural) {
    const long long np = c.npts;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % c.nx);
        const long long rr = t / c.nx;
        const int j = (int)(rr % c.ny), k = (int)(rr / c.ny);
        const long long nat = c.fx[i] + (long long)c.nx * (c.fy[j] + (long long)c.ny * c.fz[k]);
#pragma unroll
        for (int m = 0; m < MS; ++m) {
            if (to_natural) dst[(size_t)m * np + nat] = src[(size_t)m * np + t];
            else dst[(size_t)m * np + t] = src[(size_t)m * np + nat];
        }
    }
}

template <typename T, int MS>
void launch_permute(fgpe_t* h, int to_natural) {
    k_permute<T, MS><<<148 * 8, 256, 0, h->st>>>(h->sc, (const cx<T>*)h->psi, (cx<T>*)h->S, to_natural);
    h->launches++;
    std::swap(h->psi, h->S);
}

int materialize(fgpe_t* h) {
    if (h->psi_valid) return FGPE_OK;
    if (!h->S_valid) return fail(h, FGPE_E_STATE, "no state set");
    if (h->split1d) DISPATCH(h, launch_c1d, h, C1D_INV, nullptr);
    else DISPATCH(h, launch_row, h, ROW_INV, nullptr);
    CK(cudaGetLastError());
    h->psi_valid = true;
    return FGPE_OK;
}

int sync_info_err(fgpe_t* h, const double* dinfo) {
    CK(cudaMemcpyAsync(h->h_small, dinfo, sizeof(double) * INFO_LEN, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return FGPE_OK;
}

}  // namespace

// =================================================================== API
extern "C" {

int fgpe_version(void) { return 10000; }

int fgpe_device_ok(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return 0;
    int dev = 0; cudaGetDevice(&dev);
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, dev) != cudaSuccess) return 0;
    return pr.major == 10 ? 1 : 0;
}

const char* fgpe_last_error(const fgpe_t* h) { return h ? h->msg.c_str() : g_last_error.c_str(); }

int fgpe_create(const fgpe_params* pin, fgpe_t** out) {
    fgpe_t* h = nullptr;
    if (!pin || !out) return fail(h, FGPE_E_ARG, "null argument");
    fgpe_params p = *pin;
    if (p.dim < 1 || p.dim > 3) return fail(h, FGPE_E_ARG, "dim must be 1, 2 or 3");
    if (p.spin != 1 && p.spin != 2) return fail(h, FGPE_E_ARG, "spin must be 1 or 2");
    if (p.dim < 2) { p.ny = 1; p.dy = 1.0; }
    if (p.dim < 3) { p.nz = 1; p.dz = 1.0; }
    const int ns[3] = {p.nx, p.ny, p.nz};
    for (int a = 0; a < p.dim; ++a)
        if (ns[a] < 8 || ns[a] % 2) return fail(h, FGPE_E_ARG, "grid sizes must be even and >= 8 (Simpson rule)");
    if (!(p.dt > 0)) return fail(h, FGPE_E_ARG, "dt must be positive");
    if (p.precision != FGPE_FP64 && p.precision != FGPE_FP32) return fail(h, FGPE_E_ARG, "unknown precision");
    if (!fgpe_device_ok()) return fail(h, FGPE_E_CUDA, "no sm_100 CUDA device available");

    h = new fgpe_s();
    h->p = p;
    cudaGetDevice(&h->device);
    h->ms = 2 * p.spin + 1;
    h->npts = (long long)p.nx * p.ny * p.nz;
    h->fp32 = p.precision == FGPE_FP32;
    h->cs = h->fp32 ? 8 : 16;
    StepConst& c = h->sc;
    memset(&c, 0, sizeof(c));
    c.dim = p.dim; c.spin = p.spin; c.ms = h->ms;
    c.nx = p.nx; c.ny = p.ny; c.nz = p.nz; c.npts = h->npts;
    c.dt = p.dt; c.imag = p.imag_time ? 1 : 0;
    c.tau0 = p.tau[0]; c.tau1 = p.tau[1]; c.tau2 = p.tau[2];
    c.gx = p.gamma[0]; c.gy = p.dim >= 2 ? p.gamma[1] : 0.0; c.gz = p.dim >= 3 ? p.gamma[2] : 0.0;
    c.se_half = (p.dim == 1 && p.spin == 2);
    c.se_ge = (p.dim == 1);
    {
        // cgpe1d.f90:250, 443-444: projection in imaginary time when no SOC
        bool soc = fabs(p.gamma[0]) > 1e-40 || (p.dim >= 2 && fabs(p.gamma[1]) > 1e-40) || (p.dim >= 3 && fabs(p.gamma[2]) > 1e-40);
        c.project = (p.imag_time && !soc) ? 1 : 0;
        c.mag = p.mag;
    }
    for (int a = 0; a < 3; ++a) {
        FftPlan* pl = a == 0 ? &c.px : a == 1 ? &c.py : &c.pz;
        if (!plan_fft(ns[a], pl)) {
            delete h;
            return fail(nullptr, FGPE_E_ARG, "grid size " + std::to_string(ns[a]) + " is not of the form 2^a 3^b 5^c");
        }
    }

    // ---- host tables
    const double L[3] = {p.nx * p.dx, p.ny * p.dy, p.nz * p.dz};
    const double dd[3] = {p.dx, p.dy, p.dz};
    const double al[3] = {p.alpha[0], p.alpha[1], p.alpha[2]};
    std::vector<double> dt_all;
    size_t off_k[3], off_x[3], off_w[3], off_v[3];
    for (int a = 0; a < 3; ++a) {
        const int n = ns[a];
        std::vector<double> k(n), x(n), w, v(n);
        // cgpe1d.f90:692-704
        if (a < p.dim) {
            for (int i = 1; i <= 1 + n / 2; ++i) k[i - 1] = (i - 1.0) * 2.0 * kPi / L[a];
            for (int i = 1; i <= n / 2 - 1; ++i) k[i + n / 2] = -k[n / 2 - i];
            for (int i = 1; i <= n; ++i) x[i - 1] = (-1.0 + 2.0 * (i - 1.0) / n) * L[a] / 2.0;
            w = simpson_weights(n, dd[a]);
            for (int i = 0; i < n; ++i) v[i] = al[a] * al[a] * (x[i] * x[i]);
        } else {
            k[0] = 0; x[0] = 0; w.assign(1, 1.0); v[0] = 0;
        }
        off_k[a] = dt_all.size(); dt_all.insert(dt_all.end(), k.begin(), k.end());
        off_x[a] = dt_all.size(); dt_all.insert(dt_all.end(), x.begin(), x.end());
        off_w[a] = dt_all.size(); dt_all.insert(dt_all.end(), w.begin(), w.end());
        off_v[a] = dt_all.size(); dt_all.insert(dt_all.end(), v.begin(), v.end());
    }
    // complex tables (as doubles; converted to T below)
    std::vector<double> ct;
    size_t off_tw[3], off_ke[3], off_pv[3];
    auto phase = [&](double xx, double* re, double* im) {  // exp(-i CDT xx)
        if (p.imag_time) { *re = exp(-p.dt * xx); *im = 0.0; }
        else { *re = cos(p.dt * xx); *im = -sin(p.dt * xx); }
    };
    for (int a = 0; a < 3; ++a) {
        const int n = ns[a];
        off_tw[a] = ct.size() / 2;
        for (int t = 0; t < n; ++t) {
            const double ang = -2.0 * kPi * (double)t / (double)n;
            ct.push_back(cos(ang)); ct.push_back(sin(ang));
        }
    }
    for (int a = 0; a < 3; ++a) {
        const int n = ns[a];
        const double* k = &dt_all[off_k[a]];
        off_ke[a] = ct.size() / 2;
        if (a < 2 || p.dim < 3) {
            for (int i = 0; i < n; ++i) {
                double re, im;
                phase(a < p.dim ? k[i] * k[i] : 0.0, &re, &im);
                ct.push_back(re); ct.push_back(im);
            }
        } else {
            // 3D: exp(-i CDT (kz^2 - 2 L gz kz)), L = m - SPIN (cgpe3d.f90:892)
            for (int m = 0; m < h->ms; ++m) {
                const int Lm = m - p.spin;
                for (int i = 0; i < n; ++i) {
                    double re, im;
                    phase(k[i] * k[i] - 2.0 * Lm * p.gamma[2] * k[i], &re, &im);
                    ct.push_back(re); ct.push_back(im);
                }
            }
        }
    }

    for (int a = 0; a < 3; ++a) {
        // exp(-i CDT ALPHA^2 X^2) per axis (1 on unused axes)
        const double* v = &dt_all[off_v[a]];
        off_pv[a] = ct.size() / 2;
        for (int i = 0; i < ns[a]; ++i) {
            double re, im;
            phase(a < p.dim ? v[i] : 0.0, &re, &im);
            ct.push_back(re); ct.push_back(im);
        }
    }

    // 1D lines of N*M >= 3072 complex values (or too long for one block's
    // shared memory) are split N = n1*n2 (n1 the divisor nearest sqrt(N)) for
    // the four-step transform: from there on the two passes over many SMs beat
    // the single-block kernel (FP64 step: spin-1 1024 points 16 vs 18 us,
    // spin-2 2048 points 18 vs 53 us; at 512 points the single block wins).
    size_t off_tw1 = 0, off_tw2 = 0;
    const size_t line1d = (size_t)h->ms * padded_len(p.nx) * h->cs;
    const bool must_split = p.dim == 1 && line1d > 200 * 1024;
    const bool prefer_split = p.dim == 1 &&
                              ((long long)p.nx * h->ms >= 3072 || p.kernels == FGPE_KERNELS_SPLIT_1D ||
                               p.kernels == FGPE_KERNELS_CLUSTER_1D) &&
                              p.kernels != FGPE_KERNELS_SINGLE_1D;
    if (must_split || prefer_split) {
        int best = 0;
        const double half = 0.5 * log((double)p.nx);
        for (int d = 8; d <= p.nx / 8; ++d)
            if (p.nx % d == 0 && (!best || fabs(log((double)d) - half) < fabs(log((double)best) - half))) best = d;
        if (!best) { fgpe_destroy(h); return fail(nullptr, FGPE_E_ARG, "1D grid has no factorisation into two lines of >= 8"); }
        h->split1d = true;
        h->n1 = best;
        h->n2 = p.nx / best;
        plan_fft(h->n1, &c.px);
        plan_fft(h->n2, &c.py);
        off_tw1 = ct.size() / 2;
        for (int t = 0; t < h->n1; ++t) { const double ang = -2.0 * kPi * t / h->n1; ct.push_back(cos(ang)); ct.push_back(sin(ang)); }
        off_tw2 = ct.size() / 2;
        for (int t = 0; t < h->n2; ++t) { const double ang = -2.0 * kPi * t / h->n2; ct.push_back(cos(ang)); ct.push_back(sin(ang)); }
    }

    CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    h->own_stream = true;
    {
        std::vector<int> pm;
        size_t offp[3];
        for (int a = 0; a < 3; ++a) {
            const FftPlan& pl = a == 0 ? c.px : a == 1 ? c.py : c.pz;
            std::vector<int> f = position_map(pl);
            offp[a] = pm.size();
            pm.insert(pm.end(), f.begin(), f.end());
        }
        CK(cudaMalloc(&h->pmap, pm.size() * sizeof(int)));
        CK(cudaMemcpy(h->pmap, pm.data(), pm.size() * sizeof(int), cudaMemcpyHostToDevice));
        c.fx = h->pmap + offp[0]; c.fy = h->pmap + offp[1]; c.fz = h->pmap + offp[2];
    }
    const size_t bytes = (size_t)h->npts * h->ms * h->cs;
    CK(cudaMalloc(&h->S, bytes));
    CK(cudaMalloc(&h->psi, bytes));
    CK(cudaMalloc(&h->prev, bytes));
    CK(cudaMalloc(&h->dtab, dt_all.size() * sizeof(double)));
    CK(cudaMemcpy(h->dtab, dt_all.data(), dt_all.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (h->fp32) {
        std::vector<float> f(ct.begin(), ct.end());
        CK(cudaMalloc(&h->ctab, f.size() * sizeof(float)));
        CK(cudaMemcpy(h->ctab, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    } else {
        CK(cudaMalloc(&h->ctab, ct.size() * sizeof(double)));
        CK(cudaMemcpy(h->ctab, ct.data(), ct.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    const size_t ces = h->cs;  // bytes per complex table entry
    c.kx = h->dtab + off_k[0]; c.ky = h->dtab + off_k[1]; c.kz = h->dtab + off_k[2];
    c.xg = h->dtab + off_x[0]; c.yg = h->dtab + off_x[1]; c.zg = h->dtab + off_x[2];
    c.wx = h->dtab + off_w[0]; c.wy = h->dtab + off_w[1]; c.wz = h->dtab + off_w[2];
    c.vx = h->dtab + off_v[0]; c.vy = h->dtab + off_v[1]; c.vz = h->dtab + off_v[2];
    c.twx = (char*)h->ctab + off_tw[0] * ces; c.twy = (char*)h->ctab + off_tw[1] * ces; c.twz = (char*)h->ctab + off_tw[2] * ces;
    c.kex = (char*)h->ctab + off_ke[0] * ces; c.key = (char*)h->ctab + off_ke[1] * ces; c.kez = (char*)h->ctab + off_ke[2] * ces;
    c.pvx = (char*)h->ctab + off_pv[0] * ces; c.pvy = (char*)h->ctab + off_pv[1] * ces; c.pvz = (char*)h->ctab + off_pv[2] * ces;
    if (h->split1d) {
        h->twn = c.twx;   // W_N^j of the whole line
        h->tw1 = (char*)h->ctab + off_tw1 * ces;
        h->tw2 = (char*)h->ctab + off_tw2 * ces;
    }

    // ---- launch shapes
    const size_t budget = 100 * 1024;   // two blocks per SM
    const size_t hard = 200 * 1024;     // one block per SM
    const int ms = h->ms;
    if (p.dim == 1) {
        const int lp = padded_len(p.nx);
        h->k1.smem = (size_t)ms * lp * h->cs;
        h->k1.T = 512;
    }
    if (h->split1d) {
        // row pass: R rows of n1 per block; column pass: TX columns of n2.
        // These lines are short and the passes latency-bound, so the tiles
        // stay small enough for at least 128 blocks where the line allows.
        int R = 1;
        for (int r = 2; r <= 64; r *= 2) {
            if (h->n2 % r || h->n2 / r < 128 || (size_t)ms * r * padded_len(h->n1) * h->cs > budget) break;
            R = r;
            if ((size_t)ms * r * h->n1 >= 2048) break;
        }
        int TX = 1;
        for (int tx = 2; tx <= 16; tx *= 2) {
            if (h->n1 % tx || h->n1 / tx < 128 || (size_t)ms * tx * padded_len(h->n2) * h->cs > budget) break;
            TX = tx;
            if ((size_t)tx * h->cs >= 32) break;
        }
        h->r1d.tile = R; h->r1d.T = 256; h->r1d.smem = (size_t)ms * R * padded_len(h->n1) * h->cs;
        h->r1d.grid = dim3(h->n2 / R);
        h->c1d.tile = TX; h->c1d.T = 256; h->c1d.smem = (size_t)ms * TX * padded_len(h->n2) * h->cs;
        h->c1d.grid = dim3(h->n1 / TX);
        if (h->r1d.smem > hard || h->c1d.smem > hard) {
            fgpe_destroy(h);
            return fail(nullptr, FGPE_E_ARG, "1D grid too large for the split transform");
        }
    } else {
        // row pass: R rows per block, R | NY*NZ
        const int rows = p.ny * p.nz;
        const int lp = padded_len(p.nx);
        int best = 0;
        for (int R = 1; R <= rows && R <= 64; ++R) {
            if (rows % R) continue;
            const size_t sm = (size_t)ms * R * lp * h->cs;
            if (sm > (R == 1 ? hard : budget)) break;
            best = R;
            if ((size_t)ms * R * p.nx >= 2048) break;   // enough work per block
        }
        if (!best) { fgpe_destroy(h); return fail(nullptr, FGPE_E_ARG, "x lines too long for the row kernel"); }
        h->row.tile = best;
        h->row.smem = (size_t)ms * best * lp * h->cs;
        h->row.T = 256;
        h->row.grid = dim3(rows / best);
    }
    for (int a = 1; a < p.dim; ++a) {
        const int n = ns[a];
        const int lpn = padded_len(n);
        int best = 0;
        for (int TX = 1; TX <= 16 && TX <= p.nx; TX *= 2) {
            if (p.nx % TX) break;
            const size_t sm = (size_t)ms * lpn * TX * h->cs;
            if (sm > (TX == 1 ? hard : budget)) break;
            best = TX;
            if ((size_t)TX * h->cs >= 32) break;          // whole 32-byte sectors per line
        }
        if (!best) { fgpe_destroy(h); return fail(nullptr, FGPE_E_ARG, "lines too long for the column kernel"); }
        h->col[a].tile = best;
        h->col[a].smem = (size_t)ms * lpn * best * h->cs;
        h->col[a].T = 256;
        const int other = p.dim == 2 ? 1 : (a == 1 ? p.nz : p.ny);
        h->col[a].grid = dim3(p.nx / best, other);
    }
    // specialised persistent kernels where compiled for this size
    const bool allow_fast = p.kernels != FGPE_KERNELS_GENERIC;
    const bool allow_fast_row = allow_fast && p.kernels != FGPE_KERNELS_FAST_COL_ONLY;
    const bool allow_fast_col = allow_fast && p.kernels != FGPE_KERNELS_FAST_ROW_ONLY;
    if (allow_fast_row && p.dim >= 2 && fast_size(p.nx)) {
        int g = 0;
#define SETR(NN) g = h->fp32 ? (ms == 3 ? setup_fast_row<float, 3, NN>(h) : setup_fast_row<float, 5, NN>(h)) \
                             : (ms == 3 ? setup_fast_row<double, 3, NN>(h) : setup_fast_row<double, 5, NN>(h))
        FAST_SWITCH(p.nx, SETR)
#undef SETR
        if (g > 0) { h->fast_row = h->has_fast_row = true; h->fast_row_grid = g; }
        int gw = 0;
#define SETW(NN) gw = h->fp32 ? (ms == 3 ? setup_warp_row<float, 3, NN>(h) : setup_warp_row<float, 5, NN>(h)) \
                              : (ms == 3 ? setup_warp_row<double, 3, NN>(h) : setup_warp_row<double, 5, NN>(h))
        FAST_SWITCH(p.nx, SETW)
#undef SETW
        if (gw > 0) {
            h->has_warp_row = true;
            h->warp_row_grid = gw;
            h->warp_row = p.kernels == FGPE_KERNELS_WARP_ROW || (p.kernels == FGPE_KERNELS_AUTO && !h->fp32);
        }
    }
    for (int a = 1; a < p.dim; ++a) {
        if (!allow_fast_col || !fast_size(ns[a])) continue;
        const int nob = p.dim == 2 ? 1 : (a == 1 ? p.nz : p.ny);
        int g = 0;
        bool wide = false;
#define SETC(NN) g = h->fp32 ? (ms == 3 ? setup_fast_col<float, 3, NN>(h, nob, &wide) : setup_fast_col<float, 5, NN>(h, nob, &wide)) \
                             : (ms == 3 ? setup_fast_col<double, 3, NN>(h, nob, &wide) : setup_fast_col<double, 5, NN>(h, nob, &wide))
        FAST_SWITCH(ns[a], SETC)
#undef SETC
        if (g > 0) { h->fast_col[a] = h->has_fast_col[a] = true; h->fast_col_grid[a] = g; h->col_wide[a] = wide; }
        // the pass that carries KE and SOC (q2D y, 3D z) transforms forward
        // and back in one launch, and the 3D y spectra live only between the
        // step's two y passes: these lines may take the radix-16 plan
        const bool fused = (p.dim == 2 && a == 1) || p.dim == 3;
        if (g > 0 && fused && r16_len(ns[a])) {
            int g16 = 0;
#define SETC16(NN) g16 = h->fp32 ? (ms == 3 ? setup_fast_col_r16<float, 3, NN>(h, nob, wide) : setup_fast_col_r16<float, 5, NN>(h, nob, wide)) \
                                 : (ms == 3 ? setup_fast_col_r16<double, 3, NN>(h, nob, wide) : setup_fast_col_r16<double, 5, NN>(h, nob, wide))
            FAST_SWITCH(ns[a], SETC16)
#undef SETC16
            if (g16 > 0) {
                const CPlan cp = cplan(ns[a], 3);
                FftPlan pl;
                pl.n = ns[a]; pl.nf = cp.nf;
                for (int f = 0; f < cp.nf; ++f) pl.r[f] = cp.r[f];
                const std::vector<int> f = position_map(pl);
                if (!h->pmap16) CK(cudaMalloc(&h->pmap16, 2 * 512 * sizeof(int)));
                CK(cudaMemcpy(h->pmap16 + (a - 1) * 512, f.data(), f.size() * sizeof(int), cudaMemcpyHostToDevice));
                h->fline16[a] = h->pmap16 + (a - 1) * 512;
                h->col_r16[a] = true;
                h->col_r16_grid[a] = g16;
            }
        }
    }
    cudaGetLastError();   // clear any attribute/occupancy probe error
    h->obsl.grid = dim3((unsigned)((h->npts + 255) / 256));
    const size_t nq = 3 * ms + 3;
    const size_t npart = std::max<size_t>(std::max<size_t>((size_t)h->obsl.grid.x * nq,
                                                           (size_t)std::max<int>(std::max<int>(h->row.grid.x, h->fast_row_grid),
                                                                                 h->warp_row_grid) * ms),
                                          (size_t)h->c1d.grid.x * ms) + 64;
    CK(cudaMalloc(&h->part, npart * sizeof(double)));
    CK(cudaMalloc(&h->info, 4 * INFO_LEN * sizeof(double)));
    h->info_prev = h->info + INFO_LEN;
    h->obs = h->info + 2 * INFO_LEN;
    CK(cudaMalloc(&h->counters, 4 * sizeof(unsigned)));
    CK(cudaMemset(h->counters, 0, 4 * sizeof(unsigned)));
    CK(cudaMallocHost(&h->h_small, 64 * sizeof(double)));
    std::vector<double> info0(4 * INFO_LEN, 0.0);
    for (int m = 0; m < 5; ++m) { info0[INFO_SC + m] = 1.0; info0[INFO_LEN + INFO_SC + m] = 1.0; }
    info0[INFO_SIG] = info0[INFO_SIG + 1] = 20.0;   // cgpe1d.f90:425-426
    CK(cudaMemcpy(h->info, info0.data(), info0.size() * sizeof(double), cudaMemcpyHostToDevice));
    {
        cudaError_t e1 = h->fp32 ? set_smem_attrs<float, 3>() : set_smem_attrs<double, 3>();
        cudaError_t e2 = h->fp32 ? set_smem_attrs<float, 5>() : set_smem_attrs<double, 5>();
        CK(e1);
        CK(e2);
    }
    // The cluster keeps a step on 8 SMs: it wins while the line is short
    // (FP64 step, cluster vs two passes: spin-1 1024 points 11.0 vs 15.4 us,
    // spin-2 2048 points 16.7 vs 18.2 us) and loses beyond (spin-2 4096
    // points 28 vs 19 us), so by default it takes lines of N*M <= 10240.
    const bool want_cl1d = p.kernels == FGPE_KERNELS_CLUSTER_1D ||
                           (p.kernels != FGPE_KERNELS_SPLIT_1D && (long long)p.nx * h->ms <= 10240);
    if (h->split1d && want_cl1d) {
        DISPATCH(h, setup_cl1d, h);
        if (!h->cl1d && p.kernels == FGPE_KERNELS_CLUSTER_1D) {
            fgpe_destroy(h);
            return fail(nullptr, FGPE_E_ARG, "1D split does not fit one 8-CTA cluster (N1, N2 multiples of 8, 200 KB)");
        }
    }
    CK(cudaGetLastError());
    *out = h;
    return FGPE_OK;
}

int fgpe_destroy(fgpe_t* h) {
    if (!h) return FGPE_OK;
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->bulk) cudaGraphExecDestroy(h->bulk);
    cudaFree(h->S); cudaFree(h->psi); cudaFree(h->prev); cudaFree(h->stage);
    cudaFree(h->dtab); cudaFree(h->ctab); cudaFree(h->part); cudaFree(h->info);
    cudaFree(h->counters); cudaFree(h->pmap); cudaFree(h->pmap16);
    if (h->h_small) cudaFreeHost(h->h_small);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    if (h->own_stream && h->st) cudaStreamDestroy(h->st);
    delete h;
    return FGPE_OK;
}

int fgpe_set_stream(fgpe_t* h, void* stream) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    CK(cudaStreamSynchronize(h->st));
    if (h->own_stream) cudaStreamDestroy(h->st);
    if (stream) { h->st = (cudaStream_t)stream; h->own_stream = false; }
    else { CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking)); h->own_stream = true; }
    return FGPE_OK;
}

static int ensure_stage(fgpe_t* h) {
    if (h->stage) return FGPE_OK;
    CK(cudaMalloc(&h->stage, (size_t)h->npts * h->ms * 16));
    return FGPE_OK;
}

static int import_dev(fgpe_t* h, const void* src_dev) {
    const long long n2 = h->npts * h->ms * 2;
    if (h->fp32) {
        k_import<float><<<148 * 8, 256, 0, h->st>>>((const double*)src_dev, (float*)h->psi, n2);
        h->launches++;
    } else {
        CK(cudaMemcpyAsync(h->psi, src_dev, (size_t)n2 * 8, cudaMemcpyDeviceToDevice, h->st));
    }
    double one[INFO_LEN] = {0};   // pageable source: staged before the call returns
    for (int m = 0; m < 5; ++m) one[INFO_SC + m] = 1.0;
    one[INFO_SIG] = one[INFO_SIG + 1] = 20.0;
    CK(cudaMemcpyAsync(h->info, one, sizeof(one), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->info_prev, one, sizeof(one), cudaMemcpyHostToDevice, h->st));
    CK(cudaGetLastError());
    h->psi_valid = true; h->S_valid = false; h->prev_valid = false; h->norms_valid = false; h->has_state = true;
    return FGPE_OK;
}

int fgpe_set_state(fgpe_t* h, const double* phi) {
    if (!h || !phi) return fail(h, FGPE_E_ARG, "null argument");
    const size_t bytes = (size_t)h->npts * h->ms * 16;
    if (h->fp32) {
        int r = ensure_stage(h); if (r) return r;
        CK(cudaMemcpyAsync(h->stage, phi, bytes, cudaMemcpyHostToDevice, h->st));
        return import_dev(h, h->stage);
    }
    CK(cudaMemcpyAsync(h->psi, phi, bytes, cudaMemcpyHostToDevice, h->st));
    double one[INFO_LEN] = {0};
    for (int m = 0; m < 5; ++m) one[INFO_SC + m] = 1.0;
    one[INFO_SIG] = one[INFO_SIG + 1] = 20.0;
    CK(cudaMemcpyAsync(h->info, one, sizeof(one), cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->info_prev, one, sizeof(one), cudaMemcpyHostToDevice, h->st));
    h->psi_valid = true; h->S_valid = false; h->prev_valid = false; h->norms_valid = false; h->has_state = true;
    return FGPE_OK;
}

int fgpe_set_state_device(fgpe_t* h, const void* phi_dev) {
    if (!h || !phi_dev) return fail(h, FGPE_E_ARG, "null argument");
    return import_dev(h, phi_dev);
}

static int export_to(fgpe_t* h, void* dst, cudaMemcpyKind kind) {
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    int r = materialize(h); if (r) return r;
    r = ensure_stage(h); if (r) return r;
    const long long n2 = h->npts * h->ms * 2;
    if (h->fp32) k_export<float><<<148 * 8, 256, 0, h->st>>>((const float*)h->psi, (double*)h->stage, n2, 2 * h->npts, h->info);
    else k_export<double><<<148 * 8, 256, 0, h->st>>>((const double*)h->psi, (double*)h->stage, n2, 2 * h->npts, h->info);
    h->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, h->stage, (size_t)n2 * 8, kind, h->st));
    CK(cudaStreamSynchronize(h->st));
    return check_err(h);
}

int fgpe_get_state(fgpe_t* h, double* phi) {
    if (!h || !phi) return fail(h, FGPE_E_ARG, "null argument");
    return export_to(h, phi, cudaMemcpyDeviceToHost);
}

int fgpe_get_state_device(fgpe_t* h, void* phi_dev) {
    if (!h || !phi_dev) return fail(h, FGPE_E_ARG, "null argument");
    return export_to(h, phi_dev, cudaMemcpyDeviceToDevice);
}

constexpr int kBulkSteps = 16;

int fgpe_step_ex(fgpe_t* h, int nsteps, int flags) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    if (nsteps <= 0) return FGPE_OK;
    const bool snap = !(flags & FGPE_STEP_NO_SNAPSHOT);
    if (h->p.dim == 1 && !h->split1d) {
        // the state of a 1D handle always lives in psi
        int done = 0;
        while (done < nsteps) {
            const int chunk = std::min(4096, nsteps - done);
            const bool last = done + chunk == nsteps;
            void* sp = nullptr;
            if (last) {
                if (chunk == 1) {
                    CK(cudaMemcpyAsync(h->prev, h->psi, (size_t)h->npts * h->ms * h->cs, cudaMemcpyDeviceToDevice, h->st));
                    CK(cudaMemcpyAsync(h->info_prev, h->info, INFO_LEN * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
                } else {
                    sp = h->prev;
                }
            }
            DISPATCH(h, launch_1d, h, chunk, sp);
            CK(cudaGetLastError());
            done += chunk;
        }
        h->prev_valid = true; h->psi_valid = true; h->norms_valid = true;
        return FGPE_OK;
    }
    if (!h->S_valid) {
        if (!h->psi_valid) return fail(h, FGPE_E_STATE, "no state set");
        if (h->split1d) DISPATCH(h, launch_c1d, h, C1D_FWD, nullptr);
        else DISPATCH(h, launch_row, h, ROW_FWD, nullptr);
        CK(cudaGetLastError());
        h->S_valid = true;
    }
    h->prev_valid = false;
    // one step: the state before the call becomes the CONV reference; with
    // two or more steps the row pass of step n-1 writes it anyway (and the
    // buffers keep their roles, which CUDA-graph replays rely on)
    if (snap && h->psi_valid && nsteps == 1) {
        std::swap(h->psi, h->prev);
        CK(cudaMemcpyAsync(h->info_prev, h->info, INFO_LEN * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
        h->prev_valid = true;
    }
    h->psi_valid = false;
    if (h->cl1d) {
        // the whole call on one cluster: one launch, no graph
        void* sl = snap ? h->psi : nullptr;
        void* sp = (snap && nsteps >= 2) ? h->prev : nullptr;
        DISPATCH(h, launch_cl1d, h, nsteps, sl, sp);
        CK(cudaGetLastError());
        if (sp) h->prev_valid = true;
        h->psi_valid = snap;
        h->norms_valid = true;
        return FGPE_OK;
    }
    // the passes of one step; sn: real-space snapshot target of the step
    auto launch_step = [&](void* sn) {
        if (h->split1d) {
            DISPATCH(h, launch_r1d, h);
            DISPATCH(h, launch_c1d, h, C1D_FULL, sn);
            return;
        }
        if (h->p.dim == 2) {
            DISPATCH(h, launch_col, h, 1, COL_SCALE | COL_FWD | COL_KOP | COL_INV | COL_STEP);
        } else {
            DISPATCH(h, launch_col, h, 1, COL_SCALE | COL_FWD | COL_STEP);
            DISPATCH(h, launch_col, h, 2, COL_FWD | COL_KOP | COL_INV | COL_STEP);
            DISPATCH(h, launch_col, h, 1, COL_INV | COL_STEP);
        }
        DISPATCH(h, launch_row, h, ROW_FULL, sn);
    };
    // bulk steps (no snapshot: all but the last two of a snapshotting call)
    // as replays of a captured graph, unless profiling or already capturing
    int s = 0;
    const int tail = snap ? 2 : 0;
    if (!h->prof && !h->bulk_off && nsteps - tail >= 2 * kBulkSteps) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(h->st, &cs));
        if (cs == cudaStreamCaptureStatusNone) {
            if (!h->bulk) {
                const long long l0 = h->launches;
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    for (int k = 0; k < kBulkSteps; ++k) launch_step(nullptr);
                    e = cudaStreamEndCapture(h->st, &g);
                }
                if (e == cudaSuccess) e = cudaGraphInstantiate(&h->bulk, g, 0);
                if (g) cudaGraphDestroy(g);
                h->launches = l0;
                if (e != cudaSuccess) {      // no graph on this stream: stay eager
                    cudaGetLastError();
                    h->bulk = nullptr;
                    h->bulk_off = true;
                }
            }
            if (h->bulk) {
                const int per = h->split1d ? 2 : (h->p.dim == 2 ? 2 : 4);
                while (nsteps - tail - s >= kBulkSteps) {
                    CK(cudaGraphLaunch(h->bulk, h->st));
                    h->launches += (long long)per * kBulkSteps;
                    s += kBulkSteps;
                }
            }
        }
    }
    for (; s < nsteps; ++s) {
        void* sn = nullptr;
        if (snap && s == nsteps - 1) sn = h->psi;
        if (snap && s == nsteps - 2) sn = h->prev;
        launch_step(sn);
        if (snap && s == nsteps - 2) {
            CK(cudaMemcpyAsync(h->info_prev, h->info, INFO_LEN * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
            h->prev_valid = true;
        }
    }
    CK(cudaGetLastError());
    h->psi_valid = snap;
    h->norms_valid = true;
    return FGPE_OK;
}

int fgpe_step(fgpe_t* h, int nsteps) { return fgpe_step_ex(h, nsteps, FGPE_STEP_DEFAULT); }

int fgpe_normalize(fgpe_t* h, double* tnorm) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    int r = materialize(h); if (r) return r;
    DISPATCH(h, launch_obs, h, OBS_NORMALIZE, false);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_small, h->obs, OBS_LEN * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    const double tot = h->h_small[OBS_TOTAL];
    if (!(tot == tot) || !(tot > 0) || !(tot < 1e300)) return fail(h, FGPE_E_NONFINITE, "non-finite or zero total norm");
    if (tnorm) *tnorm = sqrt(tot);
    return check_err(h);
}

int fgpe_norms(fgpe_t* h, double* norm) {
    if (!h || !norm) return fail(h, FGPE_E_ARG, "null argument");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    if (h->norms_valid) {
        int r = sync_info_err(h, h->info); if (r) return r;
        for (int m = 0; m < h->ms; ++m) norm[m] = h->h_small[INFO_NORM + m];
        if (h->h_small[INFO_ERR] == 2.0)
            return fail(h, FGPE_E_NEWTON, "Newton-Raphson subroutine could not calculate the roots within 1e-6 tolerance");
        if (h->h_small[INFO_ERR] != 0.0) return fail(h, FGPE_E_NONFINITE, "non-finite norm in a step");
        return check_err(h);
    }
    int r = materialize(h); if (r) return r;
    DISPATCH(h, launch_obs, h, OBS_NORMS, false);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_small, h->obs, OBS_LEN * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int m = 0; m < h->ms; ++m) norm[m] = h->h_small[OBS_NORM + m];
    return check_err(h);
}

int fgpe_observables(fgpe_t* h, double* en, double* mu, double* mz, double* rms) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    int r = materialize(h); if (r) return r;
    DISPATCH(h, launch_obs, h, OBS_FULL, false);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_small, h->obs, OBS_LEN * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    const double* o = h->h_small;
    if (en) *en = o[OBS_EN];
    if (mz) *mz = o[OBS_MZ];
    for (int m = 0; m < h->ms; ++m) {
        if (mu) mu[m] = o[OBS_MU + m];
        if (rms) rms[m] = o[OBS_RMS + m];
    }
    if (!(o[OBS_EN] == o[OBS_EN])) return fail(h, FGPE_E_NONFINITE, "non-finite energy");
    return check_err(h);
}

int fgpe_conv(fgpe_t* h, double* max_dphi) {
    if (!h || !max_dphi) return fail(h, FGPE_E_ARG, "null argument");
    if (!h->prev_valid) return fail(h, FGPE_E_STATE, "no previous-step snapshot (step with snapshots first)");
    int r = materialize(h); if (r) return r;
    DISPATCH(h, launch_obs, h, OBS_NORMS, true);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_small, h->obs, OBS_LEN * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    *max_dphi = h->h_small[OBS_CONV];
    return check_err(h);
}

int fgpe_center(fgpe_t* h, double* out) {
    if (!h || !out) return fail(h, FGPE_E_ARG, "null argument");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    int r = materialize(h); if (r) return r;
    const long long idx = (long long)(h->p.nx / 2) + (long long)h->p.nx * ((h->p.ny > 1 ? h->p.ny / 2 : 0) + (long long)h->p.ny * (h->p.nz > 1 ? h->p.nz / 2 : 0));
    for (int m = 0; m < h->ms; ++m)
        CK(cudaMemcpyAsync((char*)h->h_small + m * 16, (char*)h->psi + ((size_t)m * h->npts + idx) * h->cs, h->cs, cudaMemcpyDeviceToHost, h->st));
    CK(cudaMemcpyAsync(h->h_small + 32, h->info, INFO_LEN * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int m = 0; m < h->ms; ++m) {
        const double s = h->h_small[32 + INFO_SC + m];
        double re, im;
        if (h->fp32) { float f[2]; memcpy(f, (char*)h->h_small + m * 16, 8); re = f[0]; im = f[1]; }
        else { memcpy(&re, (char*)h->h_small + m * 16, 8); memcpy(&im, (char*)h->h_small + m * 16 + 8, 8); }
        out[2 * m] = s * re; out[2 * m + 1] = s * im;
    }
    return FGPE_OK;
}

int fgpe_apply_op(fgpe_t* h, int op) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    int r = materialize(h); if (r) return r;
    // fold the pending scale into psi
    if (h->fp32) k_apply_scale<float><<<148 * 8, 256, 0, h->st>>>((float*)h->psi, h->npts * h->ms * 2, 2 * h->npts, h->info);
    else k_apply_scale<double><<<148 * 8, 256, 0, h->st>>>((double*)h->psi, h->npts * h->ms * 2, 2 * h->npts, h->info);
    h->launches++;
    const double ones[5] = {1.0, 1.0, 1.0, 1.0, 1.0};   // pageable source: staged before the call returns
    CK(cudaMemcpyAsync(h->info + INFO_SC, ones, sizeof(ones), cudaMemcpyHostToDevice, h->st));
    if (h->split1d && (op == FGPE_OP_FFT || op == FGPE_OP_BFT))
        return fail(h, FGPE_E_ARG, "the unfused FFT/BFT need the whole 1D line in one block (this line is split)");
    switch (op) {
        case FGPE_OP_FFT: {
            void* keep = h->S;
            h->S = h->psi;                                    // in place
            DISPATCH(h, launch_row, h, ROW_FWD, nullptr);
            if (h->p.dim >= 2) DISPATCH(h, launch_col, h, 1, COL_FWD);
            if (h->p.dim >= 3) DISPATCH(h, launch_col, h, 2, COL_FWD);
            h->S = keep;
            DISPATCH(h, launch_permute, h, 1);                // digit-reversed -> natural
        } break;
        case FGPE_OP_BFT: {
            DISPATCH(h, launch_permute, h, 0);                // natural -> digit-reversed
            void* keep = h->S;
            h->S = h->psi;
            if (h->p.dim >= 3) DISPATCH(h, launch_col, h, 2, COL_INV);
            if (h->p.dim >= 2) DISPATCH(h, launch_col, h, 1, COL_INV);
            DISPATCH(h, launch_row, h, ROW_INV, nullptr);     // psi <- F_x^-1[psi]/NX
            h->S = keep;
            if (h->p.dim >= 2) DISPATCH(h, launch_point, h, OP_SCALE, 1.0 / ((double)h->p.ny * h->p.nz));
        } break;
        case FGPE_OP_KE: DISPATCH(h, launch_point, h, OP_KE, 0.0); break;
        case FGPE_OP_SOC: DISPATCH(h, launch_point, h, OP_SOC, 0.0); break;
        case FGPE_OP_SE: DISPATCH(h, launch_point, h, OP_SE, 0.0); break;
        case FGPE_OP_SP: DISPATCH(h, launch_point, h, OP_SP, 0.0); break;
        default: return fail(h, FGPE_E_ARG, "unknown operator");
    }
    CK(cudaGetLastError());
    h->psi_valid = true; h->S_valid = false; h->prev_valid = false; h->norms_valid = false;
    return FGPE_OK;
}

int fgpe_set_kernels(fgpe_t* h, int kernels) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    if (h->bulk) { CK(cudaStreamSynchronize(h->st)); cudaGraphExecDestroy(h->bulk); h->bulk = nullptr; }
    const bool fast = kernels != FGPE_KERNELS_GENERIC;
    h->fast_row = fast && h->has_fast_row && kernels != FGPE_KERNELS_FAST_COL_ONLY;
    h->warp_row = h->has_warp_row && (kernels == FGPE_KERNELS_WARP_ROW || (kernels == FGPE_KERNELS_AUTO && !h->fp32));
    for (int a = 0; a < 3; ++a) h->fast_col[a] = fast && h->has_fast_col[a] && kernels != FGPE_KERNELS_FAST_ROW_ONLY;
    return FGPE_OK;
}

int fgpe_norms_async(fgpe_t* h, double* dst) {
    if (!h || !dst) return fail(h, FGPE_E_ARG, "null argument");
    if (!h->norms_valid) return fail(h, FGPE_E_STATE, "no step taken since the state was set");
    // Device memory of this device and pinned host memory the device can
    // address take a one-warp kernel in the step chain; anything else
    // (pageable memory, another device) a copy.
    cudaPointerAttributes at = {};
    double* ddst = nullptr;
    if (cudaPointerGetAttributes(&at, dst) == cudaSuccess &&
        ((at.type == cudaMemoryTypeHost && at.devicePointer) ||
         (at.type == cudaMemoryTypeDevice && at.device == h->device)))
        ddst = (double*)at.devicePointer;
    else
        cudaGetLastError();
    if (!ddst) {
        CK(cudaMemcpyAsync(dst, h->info + INFO_NORM, h->ms * sizeof(double), cudaMemcpyDefault, h->st));
        return FGPE_OK;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(h->st, &cs));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(32);
    cfg.stream = h->st;
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    la[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = la;
    cfg.numAttrs = cs == cudaStreamCaptureStatusNone ? 1 : 0;
    CK(cudaLaunchKernelEx(&cfg, k_norms_out, (const double*)h->info, ddst, h->ms));
    h->launches++;
    return FGPE_OK;
}

int fgpe_norms_sink(fgpe_t* h, double* dst, int count) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    double* ddst = nullptr;
    if (dst) {
        if (count < 1) return fail(h, FGPE_E_ARG, "sink needs at least one record");
        cudaPointerAttributes at = {};
        if (cudaPointerGetAttributes(&at, dst) == cudaSuccess &&
            ((at.type == cudaMemoryTypeHost && at.devicePointer) ||
             (at.type == cudaMemoryTypeDevice && at.device == h->device)))
            ddst = (double*)at.devicePointer;
        cudaGetLastError();
        if (!ddst) return fail(h, FGPE_E_ARG, "sink must be pinned host memory or memory of the handle's device");
    }
    // no step in flight may still write the previous ring
    CK(cudaStreamSynchronize(h->st));
    h->sc.sink = ddst;
    h->sc.sink_n = ddst ? count : 0;
    h->sc.sink_ctr = h->counters + 2;
    CK(cudaMemsetAsync(h->counters + 2, 0, sizeof(unsigned), h->st));
    // the bulk-step graph holds the kernel arguments it was captured with
    if (h->bulk) { cudaGraphExecDestroy(h->bulk); h->bulk = nullptr; }
    return FGPE_OK;
}

int fgpe_profile_enable(fgpe_t* h, int on) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    h->prof = on != 0;
    return FGPE_OK;
}

int fgpe_profile_read(fgpe_t* h, double* ms, long long* n, int reset) {
    if (!h) return fail(h, FGPE_E_ARG, "null handle");
    CK(cudaStreamSynchronize(h->st));
    for (auto& r : h->ev_rec) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, h->ev_pool[r.second], h->ev_pool[r.second + 1]));
        h->prof_ms[r.first] += t;
        h->prof_n[r.first] += 1;
    }
    h->ev_rec.clear();
    for (int i = 0; i < 4; ++i) {
        if (ms) ms[i] = h->prof_ms[i];
        if (n) n[i] = h->prof_n[i];
        if (reset) { h->prof_ms[i] = 0; h->prof_n[i] = 0; }
    }
    return FGPE_OK;
}

#ifdef FGPE_CHECK_ALIGN
// Diagnostic builds only (not part of the ABI).
int fgpe_debug_align_fault(unsigned long long* out4) {
    fgpe_t* h = nullptr;
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpyFromSymbol(out4, g_align_fault, 4 * sizeof(unsigned long long)));
    return FGPE_OK;
}
#endif

// ================================================================ batches
}  // extern "C"

// One group of the grouped batch mode: instances of one q2D grid shape,
// spin and precision whose passes run as shared launches (fgpe_group.cuh).
struct BatchGroup {
    int nx = 0, ny = 0, ms = 0, fp32 = 0;
    std::vector<int> members;
    InstDesc* d_desc = nullptr;      // per-instance descriptors (device)
    InstDesc* h_desc = nullptr;      // pinned staging of the descriptors
    double* part = nullptr;          // NORMC chunk partials [members][chunks][MS]
    unsigned* counter = nullptr;     // per-instance chunk counters
    int row_tiles = 0, chunk = 0, col_tiles = 0, row_grid = 0, col_grid = 0;
};

// Persistent mode: the instances of one spin and precision that the
// persistent kernel covers (fgpe_persist.cuh), advanced by one launch per
// captured graph.
struct PersistSet {
    int ms = 0, fp32 = 0;
    std::vector<int> members;
    PInst* d_inst = nullptr;         // per-instance table (device)
    PInst* h_inst = nullptr;         // pinned staging of the table
    unsigned* d_items = nullptr;     // one step's items: column tiles, then row chunks
    int ncol = 0, nrow = 0;
    double* part = nullptr;          // NORMC chunk partials
    std::vector<size_t> part_off;    // per member, in doubles
    unsigned* sync = nullptr;        // 3 counters per member, then PCTL_LEN control words
    int* ymaps = nullptr;            // y position maps of the variant's plan
    std::vector<std::pair<int, size_t>> ymap_off;   // (ny, offset)
    std::vector<int> col_tiles, row_tiles, chunk;
    size_t smem = 0;
    int grid = 0;
};

struct fgpe_batch_s {
    std::vector<fgpe_t*> inst;
    int mode = FGPE_BATCH_BRANCHES;
    std::vector<BatchGroup> groups;         // grouped mode: instances sharing launches
    std::vector<PersistSet> psets;          // persistent mode: one kernel per set
    int pvariant = 0;                       // persistent mode: kernel variant (kPersistShapes)
    double wait_ms = 2000.0;                // persistent mode: bound on one device-side wait
    int stall = -1;                         // persistent mode, tests: instance whose first wait cannot end
    std::vector<int> loose;                 // grouped/persistent mode: instances on their own branches
    cudaStream_t origin = nullptr;
    std::vector<cudaStream_t> lanes;
    std::vector<cudaEvent_t> ev;            // fork/join events, one per lane + 1
    int width = 0;                          // concurrent branches
    int ksteps = 0;                         // steps per captured graph
    cudaGraphExec_t exec = nullptr;
    int exec_steps = 0;
    std::string msg;
};

namespace {
int bfail(fgpe_batch_t* b, int code, const std::string& m) {
    if (b) b->msg = m;
    g_last_error = m;
    return code;
}
#define BCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return bfail(b, FGPE_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void drop_graph(fgpe_batch_t* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->exec_steps = 0;
}

int set_width(fgpe_batch_t* b, int w) {
    w = std::max(1, std::min<int>(w, (int)b->inst.size()));
    if (w == b->width) return FGPE_OK;
    drop_graph(b);
    for (cudaStream_t s : b->lanes) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    b->lanes.assign(w, nullptr);
    b->ev.assign(2 * w + 1, nullptr);
    for (int i = 0; i < w; ++i) BCK(cudaStreamCreateWithFlags(&b->lanes[i], cudaStreamNonBlocking));
    for (auto& e : b->ev) BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->width = w;
    return FGPE_OK;
}

// Capture nsteps of every instance as parallel branches (instance i runs on
// lane i % width) of one graph.
int capture(fgpe_batch_t* b, int nsteps) {
    drop_graph(b);
    // states must be in the spectral work buffer before capture (prologue)
    for (fgpe_t* h : b->inst) {
        if (!h->has_state) return bfail(b, FGPE_E_STATE, "batch instance without a state");
        if (h->p.dim >= 2 && !h->S_valid) {
            DISPATCH(h, launch_row, h, ROW_FWD, nullptr);
            BCK(cudaGetLastError());
            h->S_valid = true;
        }
        BCK(cudaStreamSynchronize(h->st));
    }
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    BCK(cudaEventRecord(b->ev[0], b->origin));
    for (int l = 0; l < b->width; ++l) BCK(cudaStreamWaitEvent(b->lanes[l], b->ev[0], 0));
    for (size_t i = 0; i < b->inst.size(); ++i) {
        fgpe_t* h = b->inst[i];
        cudaStream_t keep = h->st;
        const bool prof = h->prof;
        h->st = b->lanes[i % b->width];
        h->prof = false;
        const int rc = fgpe_step_ex(h, nsteps, FGPE_STEP_DEFAULT);
        h->st = keep;
        h->prof = prof;
        if (rc) { cudaGraph_t junk; cudaStreamEndCapture(b->origin, &junk); if (junk) cudaGraphDestroy(junk); return rc; }
    }
    for (int l = 0; l < b->width; ++l) {
        BCK(cudaEventRecord(b->ev[1 + l], b->lanes[l]));
        BCK(cudaStreamWaitEvent(b->origin, b->ev[1 + l], 0));
    }
    BCK(cudaStreamEndCapture(b->origin, &g));
    cudaError_t e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    BCK(e);
    b->exec_steps = nsteps;
    return FGPE_OK;
}
// ----------------------------------------------------------- grouped mode
constexpr int group_chunk(int tiles) {
    int c = 1;
    for (int d = 1; d <= 16; ++d) if (tiles % d == 0) c = d;
    return c;
}
template <typename T, int MS, int NX> int setup_group_row(BatchGroup& g) {
    constexpr int R = row_r(NX), TH = row_th<T, MS, NX>();
    if (g.ny % R) return FGPE_E_ARG;
    g.row_tiles = g.ny / R;
    g.chunk = group_chunk(g.row_tiles);
    const size_t smem = (size_t)FGPE_ROW_NBUF * MS * R * cpad(NX) * sizeof(cx<T>);
    g.row_grid = grid_for(k_row_group<T, MS, NX, R, TH>, TH, smem, (int)g.members.size() * (g.row_tiles / g.chunk));
    return g.row_grid > 0 ? FGPE_OK : FGPE_E_CUDA;
}
template <typename T, int MS, int NY> int setup_group_col(BatchGroup& g) {
    constexpr int TX = col_tx<T>(), TH = col_th<T, MS, NY>();
    if (g.nx % TX) return FGPE_E_ARG;
    g.col_tiles = g.nx / TX;
    const size_t smem = (size_t)MS * cpad(NY) * TX * sizeof(cx<T>);
    g.col_grid = grid_for(k_col_group<T, MS, NY, TX, TH>, TH, smem, (int)g.members.size() * g.col_tiles);
    return g.col_grid > 0 ? FGPE_OK : FGPE_E_CUDA;
}
template <typename T, int MS, int NX> void launch_group_row(const BatchGroup& g, int snap, cudaStream_t st) {
    constexpr int R = row_r(NX), TH = row_th<T, MS, NX>();
    const size_t smem = (size_t)FGPE_ROW_NBUF * MS * R * cpad(NX) * sizeof(cx<T>);
    GroupArgs a{g.d_desc, (int)g.members.size(), g.row_tiles, g.chunk, snap};
    k_row_group<T, MS, NX, R, TH><<<g.row_grid, TH, smem, st>>>(a);
}
template <typename T, int MS, int NY> void launch_group_col(const BatchGroup& g, cudaStream_t st) {
    constexpr int TX = col_tx<T>(), TH = col_th<T, MS, NY>();
    const size_t smem = (size_t)MS * cpad(NY) * TX * sizeof(cx<T>);
    GroupArgs a{g.d_desc, (int)g.members.size(), g.col_tiles, 1, 0};
    k_col_group<T, MS, NY, TX, TH><<<g.col_grid, TH, smem, st>>>(a);
}
template <typename T, int MS> int group_setup_tm(BatchGroup& g) {
    int r = FGPE_E_ARG;
#define GR(NN) r = setup_group_row<T, MS, NN>(g)
    FAST_SWITCH(g.nx, GR)
#undef GR
    if (r) return r;
    r = FGPE_E_ARG;
#define GC(NN) r = setup_group_col<T, MS, NN>(g)
    FAST_SWITCH(g.ny, GC)
#undef GC
    return r;
}
template <typename T, int MS> void group_launch_tm(const BatchGroup& g, int snap, cudaStream_t st) {
#define GC(NN) launch_group_col<T, MS, NN>(g, st)
    FAST_SWITCH(g.ny, GC)
#undef GC
#define GR(NN) launch_group_row<T, MS, NN>(g, snap, st)
    FAST_SWITCH(g.nx, GR)
#undef GR
}
int group_setup(BatchGroup& g) {
    if (g.fp32) return g.ms == 3 ? group_setup_tm<float, 3>(g) : group_setup_tm<float, 5>(g);
    return g.ms == 3 ? group_setup_tm<double, 3>(g) : group_setup_tm<double, 5>(g);
}
// One whole step of every instance of g: the column pass, then the row pass.
void group_step(const BatchGroup& g, int snap, cudaStream_t st) {
    if (g.fp32) { if (g.ms == 3) group_launch_tm<float, 3>(g, snap, st); else group_launch_tm<float, 5>(g, snap, st); }
    else { if (g.ms == 3) group_launch_tm<double, 3>(g, snap, st); else group_launch_tm<double, 5>(g, snap, st); }
}

void free_groups(fgpe_batch_t* b) {
    for (BatchGroup& g : b->groups) {
        if (g.d_desc) cudaFree(g.d_desc);
        if (g.h_desc) cudaFreeHost(g.h_desc);
        if (g.part) cudaFree(g.part);
        if (g.counter) cudaFree(g.counter);
    }
    b->groups.clear();
    b->loose.clear();
}

// Sort the instances into groups (q2D, size-specialised kernels on both
// axes, same grid, spin and precision) and instances that keep their own
// graph branches; allocate descriptors, NORMC slots and counters.
int build_groups(fgpe_batch_t* b) {
    free_groups(b);
    for (int i = 0; i < (int)b->inst.size(); ++i) {
        fgpe_t* h = b->inst[i];
        const bool ok = h->p.dim == 2 && h->fast_row && h->fast_col[1] && fast_size(h->p.nx) && fast_size(h->p.ny);
        if (!ok) { b->loose.push_back(i); continue; }
        BatchGroup* g = nullptr;
        for (BatchGroup& q : b->groups)
            if (q.nx == h->p.nx && q.ny == h->p.ny && q.ms == h->ms && q.fp32 == h->fp32) g = &q;
        if (!g) {
            b->groups.emplace_back();
            g = &b->groups.back();
            g->nx = h->p.nx; g->ny = h->p.ny; g->ms = h->ms; g->fp32 = h->fp32;
        }
        g->members.push_back(i);
    }
    for (BatchGroup& g : b->groups) {
        int r = group_setup(g);
        if (r) { free_groups(b); return bfail(b, r, "grouped batch: no launch shape for a group"); }
        const size_t n = g.members.size();
        const size_t slots = n * (size_t)(g.row_tiles / g.chunk) * g.ms;
        BCK(cudaMalloc(&g.d_desc, n * sizeof(InstDesc)));
        BCK(cudaMallocHost(&g.h_desc, n * sizeof(InstDesc)));
        BCK(cudaMalloc(&g.part, slots * sizeof(double)));
        BCK(cudaMalloc(&g.counter, n * sizeof(unsigned)));
        BCK(cudaMemset(g.counter, 0, n * sizeof(unsigned)));
    }
    return FGPE_OK;
}

// Descriptors from the handles' current buffers and constants (a handle's
// psi/prev roles and its NORMC sink can change between calls), copied ahead
// of the graph launch on the batch's launch stream.
int refresh_descs(fgpe_batch_t* b) {
    for (BatchGroup& g : b->groups) {
        const int nci = g.row_tiles / g.chunk;
        for (size_t k = 0; k < g.members.size(); ++k) {
            fgpe_t* h = b->inst[g.members[k]];
            InstDesc& d = g.h_desc[k];
            d.c = h->sc;
            d.S = h->S; d.psi = h->psi; d.prev = h->prev;
            d.info = h->info; d.info_prev = h->info_prev;
            d.part = g.part + k * (size_t)nci * g.ms;
            d.counter = g.counter + k;
        }
        BCK(cudaMemcpyAsync(g.d_desc, g.h_desc, g.members.size() * sizeof(InstDesc), cudaMemcpyHostToDevice,
                            b->origin));
    }
    return FGPE_OK;
}

// Grouped mode capture: each group's nsteps as a branch of shared launches
// (the last two steps write the real-space snapshots of CONV, as a
// multi-step fgpe_step does), the remaining instances as their own branches.
int capture_grouped(fgpe_batch_t* b, int nsteps) {
    drop_graph(b);
    int r = build_groups(b);
    if (r) return r;
    for (fgpe_t* h : b->inst) {
        if (!h->has_state) return bfail(b, FGPE_E_STATE, "batch instance without a state");
        if (h->p.dim >= 2 && !h->S_valid) {
            DISPATCH(h, launch_row, h, ROW_FWD, nullptr);
            BCK(cudaGetLastError());
            h->S_valid = true;
        }
        BCK(cudaStreamSynchronize(h->st));
    }
    const int nbr = (int)b->groups.size() + (int)b->loose.size();
    r = set_width(b, std::max(b->width, std::min(nbr, 64)));
    if (r) return r;
    r = refresh_descs(b);
    if (r) return r;
    BCK(cudaStreamSynchronize(b->origin));
    cudaGraph_t gr;
    BCK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    BCK(cudaEventRecord(b->ev[0], b->origin));
    for (int l = 0; l < b->width; ++l) BCK(cudaStreamWaitEvent(b->lanes[l], b->ev[0], 0));
    int lane = 0;
    for (const BatchGroup& g : b->groups) {
        cudaStream_t st = b->lanes[lane++ % b->width];
        for (int s = 0; s < nsteps; ++s) group_step(g, s == nsteps - 1 ? 1 : (s == nsteps - 2 ? 2 : 0), st);
        for (int i : g.members) {
            fgpe_t* h = b->inst[i];
            h->S_valid = true; h->psi_valid = true; h->prev_valid = true; h->norms_valid = true;
        }
    }
    for (int i : b->loose) {
        fgpe_t* h = b->inst[i];
        cudaStream_t keep = h->st;
        const bool prof = h->prof;
        h->st = b->lanes[lane++ % b->width];
        h->prof = false;
        const int rc = fgpe_step_ex(h, nsteps, FGPE_STEP_DEFAULT);
        h->st = keep;
        h->prof = prof;
        if (rc) { cudaGraph_t junk; cudaStreamEndCapture(b->origin, &junk); if (junk) cudaGraphDestroy(junk); return rc; }
    }
    for (int l = 0; l < b->width; ++l) {
        BCK(cudaEventRecord(b->ev[1 + l], b->lanes[l]));
        BCK(cudaStreamWaitEvent(b->origin, b->ev[1 + l], 0));
    }
    BCK(cudaStreamEndCapture(b->origin, &gr));
    cudaError_t e = cudaGraphInstantiate(&b->exec, gr, 0);
    cudaGraphDestroy(gr);
    BCK(e);
    BCK(cudaGetLastError());
    b->exec_steps = nsteps;
    return FGPE_OK;
}

// ------------------------------------------------------- persistent mode
void free_psets(fgpe_batch_t* b) {
    for (PersistSet& p : b->psets) {
        if (p.d_inst) cudaFree(p.d_inst);
        if (p.h_inst) cudaFreeHost(p.h_inst);
        if (p.d_items) cudaFree(p.d_items);
        if (p.part) cudaFree(p.part);
        if (p.sync) cudaFree(p.sync);
        if (p.ymaps) cudaFree(p.ymaps);
    }
    b->psets.clear();
    b->loose.clear();
}

template <typename T, int MS> int pset_prepare(PersistSet& p, int variant, int nmask) {
    const PersistShape& sh = kPersistShapes[variant];
    p.smem = persist_smem<T, MS>(sh.rn, sh.txb, nmask);
    int bps = 0;
    cudaError_t e = persist_prepare<T, MS>(variant, p.smem, &bps);
    if (e != cudaSuccess) return FGPE_E_CUDA;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    p.grid = bps * sms;
    return p.grid > 0 ? FGPE_OK : FGPE_E_ARG;
}

// Sort the instances into persistent sets (q2D, size-specialised kernels on
// both axes; one set per spin and precision) and instances that keep their
// own graph branches; build each set's item list, y maps and counters.
int build_psets(fgpe_batch_t* b) {
    free_groups(b);
    free_psets(b);
    const PersistShape& sh = kPersistShapes[b->pvariant];
    const int fast_ns[5] = {128, 192, 256, 384, 512};
    for (int i = 0; i < (int)b->inst.size(); ++i) {
        fgpe_t* h = b->inst[i];
        const bool ok = h->p.dim == 2 && h->fast_row && h->fast_col[1] && fast_size(h->p.nx) && fast_size(h->p.ny);
        if (!ok) { b->loose.push_back(i); continue; }
        PersistSet* p = nullptr;
        for (PersistSet& q : b->psets)
            if (q.ms == h->ms && q.fp32 == h->fp32) p = &q;
        if (!p) {
            b->psets.emplace_back();
            p = &b->psets.back();
            p->ms = h->ms; p->fp32 = h->fp32;
        }
        p->members.push_back(i);
    }
    for (PersistSet& p : b->psets) {
        const int n = (int)p.members.size();
        if (n > 65535) { free_psets(b); return bfail(b, FGPE_E_ARG, "persistent batch: more than 65535 instances in one set"); }
        const int cs = p.fp32 ? 8 : 16;
        const int tx = sh.txb / cs;
        int nmask = 0;
        std::vector<unsigned> col_items, row_items;
        size_t nparts = 0;
        for (int k = 0; k < n; ++k) {
            const fgpe_t* h = b->inst[p.members[k]];
            const int r = prow_r(sh.rn, h->p.nx);
            if (tx < 1 || h->p.nx % tx || h->p.ny % r) {
                free_psets(b);
                return bfail(b, FGPE_E_ARG, "persistent batch: grid not divisible by the variant's tiles");
            }
            for (int z = 0; z < 5; ++z) if (h->p.nx == fast_ns[z] || h->p.ny == fast_ns[z]) nmask |= 1 << z;
            const int ct = h->p.nx / tx, rt = h->p.ny / r;
            int ch = 1;
            for (int d = 1; d <= 4; ++d) if (rt % d == 0) ch = d;
            p.col_tiles.push_back(ct);
            p.row_tiles.push_back(rt);
            p.chunk.push_back(ch);
            for (int t = 0; t < ct; ++t) col_items.push_back(((unsigned)k << 16) | (unsigned)t);
            for (int c = 0; c < rt / ch; ++c) row_items.push_back(((unsigned)k << 16) | (unsigned)c);
            p.part_off.push_back(nparts);
            nparts += (size_t)(rt / ch) * p.ms;
            bool have = false;
            for (auto& yo : p.ymap_off) have = have || yo.first == h->p.ny;
            if (!have) p.ymap_off.push_back({h->p.ny, 0});
        }
        p.ncol = (int)col_items.size();
        p.nrow = (int)row_items.size();
        std::vector<unsigned> items(col_items);
        items.insert(items.end(), row_items.begin(), row_items.end());
        // y maps of the variant's radix plan (the x layout stays the handle's)
        std::vector<int> ym;
        for (auto& yo : p.ymap_off) {
            const CPlan cp = cplan(yo.first, sh.pv);
            FftPlan pl;
            pl.n = yo.first; pl.nf = cp.nf;
            for (int f = 0; f < cp.nf; ++f) pl.r[f] = cp.r[f];
            yo.second = ym.size();
            std::vector<int> f = position_map(pl);
            ym.insert(ym.end(), f.begin(), f.end());
        }
        int r = p.fp32 ? (p.ms == 3 ? pset_prepare<float, 3>(p, b->pvariant, nmask) : pset_prepare<float, 5>(p, b->pvariant, nmask))
                       : (p.ms == 3 ? pset_prepare<double, 3>(p, b->pvariant, nmask) : pset_prepare<double, 5>(p, b->pvariant, nmask));
        if (r) { free_psets(b); return bfail(b, r, "persistent batch: the kernel variant does not fit the device"); }
        BCK(cudaMalloc(&p.d_inst, n * sizeof(PInst)));
        BCK(cudaMallocHost(&p.h_inst, n * sizeof(PInst)));
        BCK(cudaMalloc(&p.d_items, items.size() * sizeof(unsigned)));
        BCK(cudaMemcpy(p.d_items, items.data(), items.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
        BCK(cudaMalloc(&p.part, nparts * sizeof(double)));
        BCK(cudaMalloc(&p.sync, (3 * (size_t)n + PCTL_LEN) * sizeof(unsigned)));
        BCK(cudaMemset(p.sync, 0, (3 * (size_t)n + PCTL_LEN) * sizeof(unsigned)));
        BCK(cudaMalloc(&p.ymaps, ym.size() * sizeof(int)));
        BCK(cudaMemcpy(p.ymaps, ym.data(), ym.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    return FGPE_OK;
}

// Instance tables from the handles' current buffers and constants, copied
// ahead of the graph launch on the batch's launch stream.
int refresh_pinst(fgpe_batch_t* b) {
    for (PersistSet& p : b->psets) {
        for (size_t k = 0; k < p.members.size(); ++k) {
            fgpe_t* h = b->inst[p.members[k]];
            PInst& q = p.h_inst[k];
            q.d.c = h->sc;
            q.d.S = h->S; q.d.psi = h->psi; q.d.prev = h->prev;
            q.d.info = h->info; q.d.info_prev = h->info_prev;
            q.d.part = p.part + p.part_off[k];
            q.d.counter = nullptr;
            q.fy = nullptr;
            for (auto& yo : p.ymap_off) if (yo.first == h->p.ny) q.fy = p.ymaps + yo.second;
            q.col_tiles = p.col_tiles[k];
            q.row_tiles = p.row_tiles[k];
            q.chunk = p.chunk[k];
        }
        BCK(cudaMemcpyAsync(p.d_inst, p.h_inst, p.members.size() * sizeof(PInst), cudaMemcpyHostToDevice, b->origin));
    }
    return FGPE_OK;
}

// Persistent mode capture: per set, the counters cleared and one kernel
// launch for all nsteps; the remaining instances as their own branches.
int capture_persistent(fgpe_batch_t* b, int nsteps) {
    drop_graph(b);
    int r = build_psets(b);
    if (r) return r;
    for (const PersistSet& p : b->psets)   // tickets are 32-bit: items per launch stay below 2^31
        if ((long long)(p.ncol + p.nrow) * nsteps >= (1LL << 31))
            return bfail(b, FGPE_E_ARG, "persistent batch: too many work items per launch (lower steps_per_graph)");
    for (fgpe_t* h : b->inst) {
        if (!h->has_state) return bfail(b, FGPE_E_STATE, "batch instance without a state");
        if (h->p.dim >= 2 && !h->S_valid) {
            DISPATCH(h, launch_row, h, ROW_FWD, nullptr);
            BCK(cudaGetLastError());
            h->S_valid = true;
        }
        BCK(cudaStreamSynchronize(h->st));
    }
    const int nbr = (int)b->psets.size() + (int)b->loose.size();
    r = set_width(b, std::max(b->width, std::min(nbr, 64)));
    if (r) return r;
    r = refresh_pinst(b);
    if (r) return r;
    BCK(cudaStreamSynchronize(b->origin));
    cudaGraph_t gr;
    BCK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    BCK(cudaEventRecord(b->ev[0], b->origin));
    for (int l = 0; l < b->width; ++l) BCK(cudaStreamWaitEvent(b->lanes[l], b->ev[0], 0));
    int lane = 0;
    cudaError_t le = cudaSuccess;
    for (const PersistSet& p : b->psets) {
        cudaStream_t st = b->lanes[lane++ % b->width];
        const int n = (int)p.members.size();
        if (le == cudaSuccess) le = cudaMemsetAsync(p.sync, 0, (3 * (size_t)n + PCTL_LEN) * sizeof(unsigned), st);
        PersistArgs a;
        a.inst = p.d_inst;
        a.items = p.d_items;
        a.ncol = p.ncol;
        a.nrow = p.nrow;
        a.nsteps = nsteps;
        a.sync = p.sync;
        a.ctl = p.sync + 3 * (size_t)n;
        a.wait_ns = (long long)(b->wait_ms * 1e6);
        a.ninst = n;
        a.stall = -1;
        for (int k = 0; k < n; ++k) if (p.members[k] == b->stall) a.stall = k;
        if (le == cudaSuccess)
            le = p.fp32 ? (p.ms == 3 ? persist_launch<float, 3>(b->pvariant, a, p.grid, p.smem, st)
                                     : persist_launch<float, 5>(b->pvariant, a, p.grid, p.smem, st))
                        : (p.ms == 3 ? persist_launch<double, 3>(b->pvariant, a, p.grid, p.smem, st)
                                     : persist_launch<double, 5>(b->pvariant, a, p.grid, p.smem, st));
        for (int i : p.members) {
            fgpe_t* h = b->inst[i];
            h->S_valid = true; h->psi_valid = true; h->prev_valid = true; h->norms_valid = true;
        }
    }
    for (int i : b->loose) {
        fgpe_t* h = b->inst[i];
        cudaStream_t keep = h->st;
        const bool prof = h->prof;
        h->st = b->lanes[lane++ % b->width];
        h->prof = false;
        const int rc = fgpe_step_ex(h, nsteps, FGPE_STEP_DEFAULT);
        h->st = keep;
        h->prof = prof;
        if (rc) { cudaGraph_t junk; cudaStreamEndCapture(b->origin, &junk); if (junk) cudaGraphDestroy(junk); return rc; }
    }
    for (int l = 0; l < b->width; ++l) {
        BCK(cudaEventRecord(b->ev[1 + l], b->lanes[l]));
        BCK(cudaStreamWaitEvent(b->origin, b->ev[1 + l], 0));
    }
    cudaGraph_t junk = nullptr;
    if (le != cudaSuccess) {
        cudaStreamEndCapture(b->origin, &junk);
        if (junk) cudaGraphDestroy(junk);
        return bfail(b, FGPE_E_CUDA, std::string("persistent batch launch: ") + cudaGetErrorString(le));
    }
    BCK(cudaStreamEndCapture(b->origin, &gr));
    cudaError_t e = cudaGraphInstantiate(&b->exec, gr, 0);
    cudaGraphDestroy(gr);
    BCK(e);
    BCK(cudaGetLastError());
    b->exec_steps = nsteps;
    return FGPE_OK;
}

// After a synchronised persistent launch: a device-side wait that ran out
// leaves its code in the set's control words.
int check_psets(fgpe_batch_t* b) {
    for (const PersistSet& p : b->psets) {
        unsigned ctl[PCTL_LEN];
        BCK(cudaMemcpy(ctl, p.sync + 3 * p.members.size(), sizeof(ctl), cudaMemcpyDeviceToHost));
        if (ctl[PCTL_ERR] == PERR_NONE) continue;
        const unsigned per = (unsigned)(p.ncol + p.nrow);
        const unsigned r = per ? ctl[PCTL_WHERE] % per : 0;
        unsigned e = 0;
        BCK(cudaMemcpy(&e, p.d_items + r, sizeof(e), cudaMemcpyDeviceToHost));
        const int k = (int)(e >> 16);
        const int inst = k < (int)p.members.size() ? p.members[k] : -1;
        b->exec_steps = 0;   // the states are not those of whole steps: capture afresh
        drop_graph(b);
        return bfail(b, FGPE_E_TIMEOUT,
                     std::string("persistent batch: a device-side wait ran out (") +
                         (ctl[PCTL_ERR] == PERR_WAIT_COL ? "column tile" : "row chunk") + " of instance " +
                         std::to_string(inst) + ", step " + std::to_string(ctl[PCTL_STEP]) + " of the launch)");
    }
    return FGPE_OK;
}

}  // namespace

extern "C" {

int fgpe_batch_create(const fgpe_params* p, int count, fgpe_batch_t** out) {
    fgpe_batch_t* b = nullptr;
    if (!p || count < 1 || !out) return bfail(b, FGPE_E_ARG, "bad batch arguments");
    b = new fgpe_batch_s();
    for (int i = 0; i < count; ++i) {
        fgpe_t* h = nullptr;
        const int rc = fgpe_create(&p[i], &h);
        if (rc) { fgpe_batch_destroy(b); return bfail(nullptr, rc, "instance " + std::to_string(i) + ": " + g_last_error); }
        b->inst.push_back(h);
    }
    BCK(cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking));
    int r = set_width(b, std::min(count, 64));
    if (r) return r;
    b->ksteps = 16;
    *out = b;
    return FGPE_OK;
}

int fgpe_batch_destroy(fgpe_batch_t* b) {
    if (!b) return FGPE_OK;
    if (b->origin) cudaStreamSynchronize(b->origin);
    drop_graph(b);
    free_groups(b);
    free_psets(b);
    for (cudaStream_t s : b->lanes) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->origin) cudaStreamDestroy(b->origin);
    for (fgpe_t* h : b->inst) fgpe_destroy(h);
    delete b;
    return FGPE_OK;
}

int fgpe_batch_size(const fgpe_batch_t* b) { return b ? (int)b->inst.size() : 0; }

int fgpe_batch_instance(fgpe_batch_t* b, int i, fgpe_t** h) {
    if (!b || !h || i < 0 || i >= (int)b->inst.size()) return bfail(b, FGPE_E_ARG, "bad instance index");
    *h = b->inst[i];
    return FGPE_OK;
}

const char* fgpe_batch_last_error(const fgpe_batch_t* b) { return b ? b->msg.c_str() : g_last_error.c_str(); }

int fgpe_batch_config(fgpe_batch_t* b, int width, int steps_per_graph) {
    if (!b) return bfail(b, FGPE_E_ARG, "null batch");
    if (width > 0) { int r = set_width(b, width); if (r) return r; }
    if (steps_per_graph > 0 && steps_per_graph != b->ksteps) { b->ksteps = steps_per_graph; drop_graph(b); }
    return FGPE_OK;
}

int fgpe_batch_step(fgpe_batch_t* b, int nsteps) {
    if (!b) return bfail(b, FGPE_E_ARG, "null batch");
    // wait for work queued on the instances' own streams (set_state etc.)
    for (fgpe_t* h : b->inst) BCK(cudaStreamSynchronize(h->st));
    int left = nsteps;
    while (left > 0) {
        int k = std::min(left, b->ksteps);
        if (k == 1 && left > 1) k = 2;
        if (k == 1) {
            // a single step keeps the one-step CONV semantics: run eagerly
            for (size_t i = 0; i < b->inst.size(); ++i) {
                fgpe_t* h = b->inst[i];
                cudaStream_t keep = h->st;
                h->st = b->lanes[i % b->width];
                const int rc = fgpe_step_ex(h, 1, FGPE_STEP_DEFAULT);
                h->st = keep;
                if (rc) return rc;
            }
            for (int l = 0; l < b->width; ++l) BCK(cudaStreamSynchronize(b->lanes[l]));
            left -= 1;
            continue;
        }
        if (!b->exec || b->exec_steps != k) {
            int r = b->mode == FGPE_BATCH_GROUPED      ? capture_grouped(b, k)
                    : b->mode == FGPE_BATCH_PERSISTENT ? capture_persistent(b, k)
                                                       : capture(b, k);
            if (r) return r;
        } else if (b->mode == FGPE_BATCH_GROUPED) {
            int r = refresh_descs(b);
            if (r) return r;
        } else if (b->mode == FGPE_BATCH_PERSISTENT) {
            int r = refresh_pinst(b);
            if (r) return r;
        }
        BCK(cudaGraphLaunch(b->exec, b->origin));
        for (fgpe_t* h : b->inst) h->launches += step_launches(h, k);
        left -= k;
        if (b->mode == FGPE_BATCH_PERSISTENT) {
            BCK(cudaStreamSynchronize(b->origin));
            int r = check_psets(b);
            if (r) return r;
        }
    }
    BCK(cudaStreamSynchronize(b->origin));
    return FGPE_OK;
}

// fgpe_batch_step with device timing: CUDA events on the launch stream
// before the first and after the last graph launch.  Only whole graphs are
// timed, so nsteps must not leave a single-step remainder.
int fgpe_batch_step_timed(fgpe_batch_t* b, int nsteps, double* device_ms) {
    if (!b || !device_ms) return bfail(b, FGPE_E_ARG, "null argument");
    if (nsteps < 2 || (nsteps % b->ksteps) == 1)
        return bfail(b, FGPE_E_ARG, "timed batch steps need nsteps >= 2 and no single-step remainder");
    for (fgpe_t* h : b->inst) BCK(cudaStreamSynchronize(h->st));
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    int rc = FGPE_OK;
    int left = nsteps;
    cudaError_t err = cudaEventRecord(e0, b->origin);
    while (err == cudaSuccess && rc == FGPE_OK && left > 0) {
        int k = std::min(left, b->ksteps);
        if (k == 1) k = 2;   // cannot happen: remainder 1 rejected above
        if (!b->exec || b->exec_steps != k)
            rc = b->mode == FGPE_BATCH_GROUPED      ? capture_grouped(b, k)
                 : b->mode == FGPE_BATCH_PERSISTENT ? capture_persistent(b, k)
                                                    : capture(b, k);
        else if (b->mode == FGPE_BATCH_GROUPED) rc = refresh_descs(b);
        else if (b->mode == FGPE_BATCH_PERSISTENT) rc = refresh_pinst(b);
        if (rc) break;
        err = cudaGraphLaunch(b->exec, b->origin);
        for (fgpe_t* h : b->inst) h->launches += step_launches(h, k);
        left -= k;
    }
    if (err == cudaSuccess && rc == FGPE_OK) err = cudaEventRecord(e1, b->origin);
    if (err == cudaSuccess && rc == FGPE_OK) err = cudaStreamSynchronize(b->origin);
    float ms = 0.f;
    if (err == cudaSuccess && rc == FGPE_OK) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    BCK(err);
    if (b->mode == FGPE_BATCH_PERSISTENT) {
        rc = check_psets(b);
        if (rc) return rc;
    }
    *device_ms = ms;
    return FGPE_OK;
}

// Observables of every instance: out[i*OBS] = en, mz, conv (if requested and
// available, else -1), then mu[M], rms[M], norm[M] (stride 3+3*M).
int fgpe_batch_observables(fgpe_batch_t* b, double* out, int with_conv) {
    if (!b || !out) return bfail(b, FGPE_E_ARG, "null argument");
    const int n = (int)b->inst.size();
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        fgpe_t* h = b->inst[i];
        const int ms = h->ms;
        double* o = out + off;
        off += 3 + 3 * ms;
        int r = fgpe_observables(h, &o[0], o + 3, &o[1], o + 3 + ms);
        if (r) return r;
        r = fgpe_norms(h, o + 3 + 2 * ms);
        if (r) return r;
        o[2] = -1.0;
        if (with_conv && h->prev_valid) { r = fgpe_conv(h, &o[2]); if (r) return r; }
    }
    return FGPE_OK;
}

// Autotuner: times candidate (kernel family per grid-size class, branch
// width, steps per graph) settings on the batch itself and keeps the fastest.
// The instances' states are saved before and restored after the trials, so
// tuning does not advance the physics.  The result is remembered in a small
// text cache (one line per batch signature) when cache_path is given.
int fgpe_batch_autotune(fgpe_batch_t* b, int trial_steps, const char* cache_path) {
    if (!b) return bfail(b, FGPE_E_ARG, "null batch");
    const int n = (int)b->inst.size();
    if (trial_steps < 2) trial_steps = 8;
    // signature: device, precision, spin and the sorted grid sizes
    cudaDeviceProp prop;
    int dev = 0; cudaGetDevice(&dev); cudaGetDeviceProperties(&prop, dev);
    std::vector<std::string> sizes;
    for (fgpe_t* h : b->inst)
        sizes.push_back(std::to_string(h->p.nx) + "x" + std::to_string(h->p.ny) + "x" + std::to_string(h->p.nz) + "s" +
                        std::to_string(h->p.spin) + (h->fp32 ? "f" : "d"));
    std::vector<std::string> classes = sizes;
    std::sort(classes.begin(), classes.end());
    classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
    std::string sig = std::string(prop.name) + "|" + std::to_string(n);
    for (auto& c : classes) sig += "|" + c + ":" + std::to_string(std::count(sizes.begin(), sizes.end(), c));
    for (char& ch : sig) if (ch == ' ') ch = '_';
    // cached?
    if (cache_path) {
        FILE* f = fopen(cache_path, "r");
        if (f) {
            char line[8192];
            while (fgets(line, sizeof line, f)) {
                std::string l(line);
                if (l.compare(0, sig.size() + 1, sig + " ") != 0) continue;
                int w = 0, k = 0, md = FGPE_BATCH_BRANCHES, pv = 0;
                double tms = 0;
                char fam[4096] = {0};
                const int got = sscanf(l.c_str() + sig.size() + 1, "%d %d %4095s %lf %d %d", &w, &k, fam, &tms, &md, &pv);
                if (got >= 3) {
                    fclose(f);
                    std::string fs(fam);
                    for (size_t ci = 0; ci < classes.size() && ci < fs.size(); ++ci)
                        for (int i = 0; i < n; ++i)
                            if (sizes[i] == classes[ci]) fgpe_set_kernels(b->inst[i], fs[ci] == 'g' ? FGPE_KERNELS_GENERIC : FGPE_KERNELS_AUTO);
                    int rm = fgpe_batch_variant(b, got >= 6 ? pv : 0, nullptr);
                    if (rm) return rm;
                    rm = fgpe_batch_mode(b, got >= 5 ? md : FGPE_BATCH_BRANCHES);
                    if (rm) return rm;
                    return fgpe_batch_config(b, w, k);
                }
            }
            fclose(f);
        }
    }
    // save states (spectral buffer or real-space copy, plus the info vector);
    // every path out of the search below restores them and frees the copies
    std::vector<void*> save(n, nullptr), save_info(n, nullptr);
    std::vector<char> flags(3 * n);
    int saved = 0;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    auto finish = [&](int rc) -> int {
        for (int i = 0; i < saved; ++i) {
            fgpe_t* h = b->inst[i];
            const size_t bytes = (size_t)h->npts * h->ms * h->cs;
            cudaError_t e = cudaStreamSynchronize(h->st);
            if (e == cudaSuccess) e = cudaMemcpy(h->S, save[i], bytes, cudaMemcpyDeviceToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(h->psi, (char*)save[i] + bytes, bytes, cudaMemcpyDeviceToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(h->info, save_info[i], 2 * INFO_LEN * sizeof(double), cudaMemcpyDeviceToDevice);
            if (e == cudaSuccess) {
                h->S_valid = flags[3 * i]; h->psi_valid = flags[3 * i + 1]; h->prev_valid = flags[3 * i + 2];
            } else if (rc == FGPE_OK) {
                rc = bfail(b, FGPE_E_CUDA, std::string("autotune: restoring instance states: ") + cudaGetErrorString(e));
            }
        }
        for (int i = 0; i < n; ++i) {
            if (save[i]) cudaFree(save[i]);
            if (save_info[i]) cudaFree(save_info[i]);
        }
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        return rc;
    };
#define ACK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return finish(bfail(b, FGPE_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_))); \
    } while (0)
    for (int i = 0; i < n; ++i) {
        fgpe_t* h = b->inst[i];
        ACK(cudaStreamSynchronize(h->st));
        const size_t bytes = (size_t)h->npts * h->ms * h->cs;
        ACK(cudaMalloc(&save[i], 2 * bytes));
        ACK(cudaMalloc(&save_info[i], 2 * INFO_LEN * sizeof(double)));
        ACK(cudaMemcpy(save[i], h->S, bytes, cudaMemcpyDeviceToDevice));
        ACK(cudaMemcpy((char*)save[i] + bytes, h->psi, bytes, cudaMemcpyDeviceToDevice));
        ACK(cudaMemcpy(save_info[i], h->info, 2 * INFO_LEN * sizeof(double), cudaMemcpyDeviceToDevice));
        flags[3 * i] = h->S_valid; flags[3 * i + 1] = h->psi_valid; flags[3 * i + 2] = h->prev_valid;
        saved = i + 1;
    }
    ACK(cudaEventCreate(&t0));
    ACK(cudaEventCreate(&t1));
    auto timed = [&](int w, int k, double* ms) -> int {
        int r = fgpe_batch_config(b, w, k);
        if (r) return r;
        r = fgpe_batch_step(b, k);          // warm-up, includes capture
        if (r) return r;
        BCK(cudaEventRecord(t0, b->origin));
        r = fgpe_batch_step(b, trial_steps);
        if (r) return r;
        BCK(cudaEventRecord(t1, b->origin));
        BCK(cudaEventSynchronize(t1));
        float f = 0;
        BCK(cudaEventElapsedTime(&f, t0, t1));
        *ms = f / trial_steps;
        return FGPE_OK;
    };
    // 1) kernel family per size class (fast where available), at a default shape
    std::string fam(classes.size(), 'f');
    double best_ms = 1e30;
    for (size_t ci = 0; ci < classes.size(); ++ci) {
        double tms[2] = {1e30, 1e30};
        for (int opt = 0; opt < 2; ++opt) {
            for (int i = 0; i < n; ++i)
                if (sizes[i] == classes[ci]) fgpe_set_kernels(b->inst[i], opt ? FGPE_KERNELS_GENERIC : FGPE_KERNELS_AUTO);
            int r = timed(std::min(n, 64), 8, &tms[opt]);
            if (r) return finish(r);
        }
        const int pick = tms[1] < tms[0] ? 1 : 0;
        fam[ci] = pick ? 'g' : 'f';
        for (int i = 0; i < n; ++i)
            if (sizes[i] == classes[ci]) fgpe_set_kernels(b->inst[i], pick ? FGPE_KERNELS_GENERIC : FGPE_KERNELS_AUTO);
        best_ms = std::min(tms[0], tms[1]);
    }
    // 2) branch width and steps per graph, one branch per instance
    int bw = std::min(n, 64), bk = 8, bmode = FGPE_BATCH_BRANCHES;
    const int widths[] = {4, 16, 32, 64, 128, 256, 512};
    const int ks[] = {4, 8, 32};
    for (int w : widths) {
        if (w > n) continue;
        for (int k : ks) {
            double ms = 0;
            int r = timed(w, k, &ms);
            if (r) return finish(r);
            if (ms < best_ms) { best_ms = ms; bw = w; bk = k; }
        }
    }
    // 3) grouped launches (instances of one q2D grid shape share each pass)
    {
        int r = fgpe_batch_mode(b, FGPE_BATCH_GROUPED);
        if (r) return finish(r);
        for (int k : ks) {
            double ms = 0;
            r = timed(std::min(n, 64), k, &ms);
            if (r) return finish(r);
            if (ms < best_ms) { best_ms = ms; bw = std::min(n, 64); bk = k; bmode = FGPE_BATCH_GROUPED; }
        }
    }
    // 4) one persistent launch per graph for all covered instances, for every
    //    kernel variant (threads per block, rows per row tile, bytes per
    //    column tile row, radix plan of the y lines)
    int bvar = b->pvariant;
    {
        int r = fgpe_batch_mode(b, FGPE_BATCH_PERSISTENT);
        if (r) return finish(r);
        for (int v = 0; v < kPersistVariants; ++v) {
            r = fgpe_batch_variant(b, v, nullptr);
            if (r) return finish(r);
            for (int k : ks) {
                double ms = 0;
                r = timed(std::min(n, 64), k, &ms);
                if (r == FGPE_E_ARG) break;   // this variant's tiles do not fit the batch
                if (r) return finish(r);
                if (ms < best_ms) { best_ms = ms; bw = std::min(n, 64); bk = k; bmode = FGPE_BATCH_PERSISTENT; bvar = v; }
            }
        }
        r = fgpe_batch_variant(b, bvar, nullptr);
        if (r) return finish(r);
        r = fgpe_batch_mode(b, bmode);
        if (r) return finish(r);
    }
#undef ACK
    int r = finish(FGPE_OK);
    if (r) return r;
    r = fgpe_batch_config(b, bw, bk);
    if (r) return r;
    if (cache_path) {
        FILE* f = fopen(cache_path, "a");
        if (f) {
            fprintf(f, "%s %d %d %s %.6f %d %d\n", sig.c_str(), bw, bk, fam.c_str(), best_ms, bmode, bvar);
            fclose(f);
        }
    }
    return FGPE_OK;
}

int fgpe_batch_mode(fgpe_batch_t* b, int mode) {
    if (!b) return bfail(b, FGPE_E_ARG, "null batch");
    if (mode != FGPE_BATCH_BRANCHES && mode != FGPE_BATCH_GROUPED && mode != FGPE_BATCH_PERSISTENT)
        return bfail(b, FGPE_E_ARG, "unknown batch mode");
    if (mode != b->mode) {
        drop_graph(b);
        free_groups(b);
        free_psets(b);
        b->mode = mode;
    }
    return FGPE_OK;
}

int fgpe_batch_variant(fgpe_batch_t* b, int variant, int* current) {
    if (!b) return bfail(b, FGPE_E_ARG, "null batch");
    if (variant >= kPersistVariants) return bfail(b, FGPE_E_ARG, "unknown persistent kernel variant");
    if (variant >= 0 && variant != b->pvariant) {
        drop_graph(b);
        free_psets(b);
        b->pvariant = variant;
    }
    if (current) *current = b->pvariant;
    return FGPE_OK;
}

int fgpe_batch_variants(void) { return kPersistVariants; }

int fgpe_batch_variant_shape(int variant, int* shape) {
    if (variant < 0 || variant >= kPersistVariants || !shape) return FGPE_E_ARG;
    const PersistShape& s = kPersistShapes[variant];
    shape[0] = s.th;
    shape[1] = s.rn;
    shape[2] = s.txb;
    shape[3] = s.pv;
    return FGPE_OK;
}

int fgpe_batch_wait_bound(fgpe_batch_t* b, double wait_ms, int stall_instance) {
    if (!b) return bfail(b, FGPE_E_ARG, "null batch");
    if (!(wait_ms > 0.0) || wait_ms > 600000.0) return bfail(b, FGPE_E_ARG, "wait bound must be in (0, 600000] ms");
    if (stall_instance < -1 || stall_instance >= (int)b->inst.size()) return bfail(b, FGPE_E_ARG, "bad instance index");
    b->wait_ms = wait_ms;
    b->stall = stall_instance;
    drop_graph(b);
    return FGPE_OK;
}

int fgpe_batch_tuning(const fgpe_batch_t* b, int* width, int* steps_per_graph) {
    if (!b) return FGPE_E_ARG;
    if (width) *width = b->width;
    if (steps_per_graph) *steps_per_graph = b->ksteps;
    return FGPE_OK;
}

int fgpe_kernel_launches(fgpe_t* h, long long* count) {
    if (!h || !count) return fail(h, FGPE_E_ARG, "null argument");
    *count = h->launches;
    return FGPE_OK;
}

}  // extern "C"

// ================================================================ FNO ABI
extern "C" {

static int fno_ck(cudaError_t e) {
    if (e != cudaSuccess) { g_last_error = cudaGetErrorString(e); return FGPE_E_CUDA; }
    return FGPE_OK;
}
static unsigned fno_grid(long long n) { long long g = (n + 255) / 256; return (unsigned)std::min<long long>(g, 148LL * 32); }

int fno_gemm(int batch, int M, int N, int K, float alpha, const void* A, int a_bf16, long long sAb, long long sAi,
             long long sAk, const float* B, long long sBb, long long sBk, long long sBj, float beta, float* C,
             long long sCb, long long sCi, long long sCj, void* stream) {
    if (batch <= 0 || M <= 0 || N <= 0 || K <= 0) return FGPE_E_ARG;
    if (batch > 65535) return FGPE_E_ARG;
    dim3 grid((N + 63) / 64, (M + 63) / 64, batch);
    cudaStream_t st = (cudaStream_t)stream;
    if (a_bf16)
        fno::k_gemm<__nv_bfloat16><<<grid, 256, 0, st>>>(M, N, K, alpha, (const __nv_bfloat16*)A, sAb, sAi, sAk, B, sBb,
                                                         sBk, sBj, beta, C, sCb, sCi, sCj);
    else
        fno::k_gemm<float><<<grid, 256, 0, st>>>(M, N, K, alpha, (const float*)A, sAb, sAi, sAk, B, sBb, sBk, sBj, beta, C,
                                                 sCb, sCi, sCj);
    return fno_ck(cudaGetLastError());
}

}  // extern "C"

// Tensor-core variant of fno_gemm (fno_gemm_tc.cuh).  When A is shared by
// every batch entry and B is not, the product is taken transposed (C^T =
// B^T A^T) so that the shared operand becomes B and the entries fold into one
// tall GEMM; the tile width GN is the smallest of 16..256 that covers N.
// CTAs per SM: as many as the shared memory (about 227 KB) and the 512 TMEM
// columns hold, at most four; CTAs beyond those resident wait their turn.
template <int GN> constexpr int gemm_tc_per_sm() {
    const int by_smem = (int)((227 * 1024) / (fno::gtc::smem_bytes<GN>() + 3 * 1024));
    const int by_tmem = 512 / fno::gtc::tmem_cols<GN>();
    return std::min(4, std::min(by_smem, by_tmem));
}

template <typename TA, int GN> static int gemm_tc_launch(const fno::GemmTc& g, cudaStream_t st) {
    static bool attr_set[64] = {false};
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return FGPE_E_ARG;
    const size_t smem = fno::gtc::smem_bytes<GN>();
    if (!attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fno::k_gemm_tc<TA, GN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return fno_ck(e);
        attr_set[dev] = true;
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long rows = g.fold ? (long long)g.batch * g.M : (long long)g.M;
    const long long tiles = (rows + fno::gtc::TM - 1) / fno::gtc::TM * ((g.N + GN - 1) / GN) * (g.fold ? 1 : g.batch);
    const long long grid = std::min<long long>(tiles, (long long)gemm_tc_per_sm<GN>() * nsm);
    fno::k_gemm_tc<TA, GN><<<(unsigned)grid, 128, smem, st>>>(g);
    return fno_ck(cudaGetLastError());
}

template <typename TA> static int gemm_tc_width(const fno::GemmTc& g, cudaStream_t st) {
    if (g.N <= 16) return gemm_tc_launch<TA, 16>(g, st);
    if (g.N <= 32) return gemm_tc_launch<TA, 32>(g, st);
    if (g.N <= 64) return gemm_tc_launch<TA, 64>(g, st);
    if (g.N <= 128) return gemm_tc_launch<TA, 128>(g, st);
    return gemm_tc_launch<TA, 256>(g, st);
}

extern "C" {

int fno_gemm_tc(int batch, int M, int N, int K, float alpha, const void* A, int a_bf16, long long sAb, long long sAi,
                long long sAk, const float* B, long long sBb, long long sBk, long long sBj, float beta, float* C,
                long long sCb, long long sCi, long long sCj, int* err_dev, void* stream) {
    if (!A || !B || !C || !err_dev) { g_last_error = "null argument"; return FGPE_E_ARG; }
    if (batch <= 0 || M <= 0 || N <= 0 || K <= 0) { g_last_error = "empty GEMM"; return FGPE_E_ARG; }
    if (sAb < 0 || sAi < 0 || sAk < 0 || sBb < 0 || sBk < 0 || sBj < 0 || sCb < 0 || sCi < 0 || sCj < 0) {
        g_last_error = "negative stride";
        return FGPE_E_ARG;
    }
    fno::GemmTc g{M, N, K, batch, 0, alpha, beta, A, sAb, sAi, sAk, B, sBb, sBk, sBj, C, sCb, sCi, sCj, err_dev, 0, 0, 0};
    if (batch > 1 && sAb == 0 && sBb != 0 && !a_bf16) {
        // C^T = B^T A^T: the shared A becomes the B operand
        g = fno::GemmTc{N, M, K, batch, 0, alpha, beta, B, sBb, sBj, sBk, (const float*)A, 0, sAk, sAi,
                        C, sCb, sCj, sCi, err_dev, 0, 0, 0};
    }
    g.fold = batch > 1 && g.sBb == 0;
    // float4 operand reads where the unit-stride runs start on 16-byte boundaries
    const bool a16 = ((uintptr_t)g.A & 15) == 0, b16 = ((uintptr_t)g.B & 15) == 0;
    g.avec = !a_bf16 && a16 && g.sAk == 1 && g.sAi % 4 == 0 && g.sAb % 4 == 0;
    if (b16 && g.sBb % 4 == 0) {
        if (g.sBj == 1 && g.sBk % 4 == 0) g.bvec = 1;
        else if (g.sBk == 1 && g.sBj % 4 == 0) g.bvec = 2;
    }
    g.cvec = ((uintptr_t)g.C & 15) == 0 && g.sCj == 1 && g.sCi % 4 == 0 && g.sCb % 4 == 0;
    const cudaStream_t st = (cudaStream_t)stream;
    return a_bf16 ? gemm_tc_width<__nv_bfloat16>(g, st) : gemm_tc_width<float>(g, st);
}

int fno_bias_act(float* z, float* h, const float* bias, long long C, long long S, long long n, int act, void* stream) {
    fno::k_bias_act<<<fno_grid(n), 256, 0, (cudaStream_t)stream>>>(z, h, bias, C, S, n, act);
    return fno_ck(cudaGetLastError());
}

int fno_act_bwd(float* dz, const float* dh, const float* z, long long n, void* stream) {
    fno::k_act_bwd<<<fno_grid(n), 256, 0, (cudaStream_t)stream>>>(dz, dh, z, n);
    return fno_ck(cudaGetLastError());
}

int fno_channel_sum(float* out, const float* x, long long B, long long C, long long S, float beta, void* stream) {
    if (S == 1)
        fno::k_channel_sum_rows<<<(unsigned)((C + 255) / 256), 256, 0, (cudaStream_t)stream>>>(out, x, B, C, beta);
    else
        fno::k_channel_sum<<<(unsigned)C, 256, 0, (cudaStream_t)stream>>>(out, x, B, C, S, beta);
    return fno_ck(cudaGetLastError());
}

int fno_axpy(float* y, const float* x, float a, long long n, void* stream) {
    fno::k_axpy<<<fno_grid(n), 256, 0, (cudaStream_t)stream>>>(y, x, a, n);
    return fno_ck(cudaGetLastError());
}

int fno_mse(const float* out, const float* target, float* dout, double* loss_dev, double* scratch, long long n,
            void* stream) {
    fno::k_mse<<<256, 256, 0, (cudaStream_t)stream>>>(out, target, dout, scratch, n);
    fno::k_sum_parts<<<1, 32, 0, (cudaStream_t)stream>>>(scratch, 256, 1.0 / (double)n, loss_dev);
    return fno_ck(cudaGetLastError());
}

int fno_adam(float* w, void* w_bf16, const float* g, float* m, float* v, long long n, float lr, float beta1,
             float beta2, float eps, int t, void* stream) {
    const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
    fno::k_adam<<<fno_grid(n), 256, 0, (cudaStream_t)stream>>>(w, (__nv_bfloat16*)w_bf16, g, m, v, n, lr, beta1, beta2,
                                                              eps, c1, c2);
    return fno_ck(cudaGetLastError());
}

int fno_to_bf16(const float* x, void* y, long long n, void* stream) {
    fno::k_to_bf16<<<fno_grid(n), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16*)y, n);
    return fno_ck(cudaGetLastError());
}

#ifndef FNO_DENSE_GUARD
#define FNO_DENSE_GUARD 0
#endif
static const size_t kDenseGuard = FNO_DENSE_GUARD;

int fno_dense_tc(const void* w_bf16, int transpose_w, const float* x, const float* bias, float* z, float* h, int M,
                 int K, long long n, int act, int* err_dev, void* stream) {
    if (!w_bf16 || !x || !err_dev || (!z && !h)) { g_last_error = "null argument"; return FGPE_E_ARG; }
    if (M < 1 || M > fno::tc::TM || K < 1 || K > 128 || n < 1) {
        g_last_error = "dense layer needs 1 <= M <= 128 output and 1 <= K <= 128 input channels";
        return FGPE_E_ARG;
    }
    const int KP = (K + 15) / 16 * 16;
    // operand tiles plus alignment slack and a guard region behind them
    const size_t smem = 1024 + (size_t)fno::tc::TM * KP * 2 + (size_t)KP * fno::tc::TN * 2 + kDenseGuard;
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fno::k_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(1024 + (size_t)fno::tc::TM * 128 * 2 + (size_t)128 * fno::tc::TN * 2 +
                                                   kDenseGuard));
        if (e != cudaSuccess) return fno_ck(e);
        attr_set[dev] = true;
    }
    const long long blocks = (n + fno::tc::TN - 1) / fno::tc::TN;
    if (blocks > 0x7fffffffLL) { g_last_error = "too many columns"; return FGPE_E_ARG; }
    fno::k_dense_tc<<<(unsigned)blocks, 128, smem, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)w_bf16, transpose_w, x, bias, z, h, M, K, n, act, err_dev);
    return fno_ck(cudaGetLastError());
}

int fno_rbig_build(const float* rr, const float* ri, void* rbig, long long nmodes, int O, int C, void* stream) {
    if (nmodes <= 0 || O <= 0 || C <= 0) return FGPE_E_ARG;
    fno::k_rbig_build<<<fno_grid(nmodes * 4LL * O * C), 256, 0, (cudaStream_t)stream>>>(rr, ri, (__nv_bfloat16*)rbig,
                                                                                        nmodes, O, C);
    return fno_ck(cudaGetLastError());
}

int fno_rbig_fold(const float* drbig, float* drr, float* dri, long long nmodes, int O, int C, void* stream) {
    if (nmodes <= 0 || O <= 0 || C <= 0) return FGPE_E_ARG;
    fno::k_rbig_fold<<<fno_grid(nmodes * (long long)O * C), 256, 0, (cudaStream_t)stream>>>(drbig, drr, dri, nmodes, O, C);
    return fno_ck(cudaGetLastError());
}

}  // extern "C"

// ================================================================ checkpoints
// Full-precision checkpoint of a handle's state, bit-exact on resume: the
// raw device buffers that hold the state (real-space psi and/or the
// x-spectral S, whichever are current) with the per-component pending scales,
// the last NORMC and the projection's Newton start values (info[]).  The
// reference has no checkpoint; a long imaginary-time run can stop at an STP
// boundary and continue in another process.
//
// File layout (native byte order): "FGPECKP1", u32 version = 1, the
// fgpe_params of the handle, i64 step, 8 caller doubles, u32 flags
// (1 psi, 2 S, 4 norms), info[INFO_LEN], then psi and/or S (npts*M complex
// of the handle's precision), then u64 FNV-1a of everything before it.
namespace {
const char kCkpMagic[8] = {'F', 'G', 'P', 'E', 'C', 'K', 'P', '1'};

struct Fnv {
    unsigned long long h = 1469598103934665603ULL;
    void add(const void* p, size_t n) {
        const unsigned char* b = (const unsigned char*)p;
        for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ULL; }
    }
};
}  // namespace

extern "C" int fgpe_checkpoint_save(fgpe_t* h, const char* path, long long step, const double* user) {
    if (!h || !path) return fail(h, FGPE_E_ARG, "null argument");
    if (!h->has_state) return fail(h, FGPE_E_STATE, "no state set");
    const size_t bytes = (size_t)h->npts * h->ms * h->cs;
    std::vector<unsigned char> psi, S;
    if (h->psi_valid) { psi.resize(bytes); CK(cudaMemcpyAsync(psi.data(), h->psi, bytes, cudaMemcpyDeviceToHost, h->st)); }
    if (h->S_valid) { S.resize(bytes); CK(cudaMemcpyAsync(S.data(), h->S, bytes, cudaMemcpyDeviceToHost, h->st)); }
    double info[INFO_LEN];
    CK(cudaMemcpyAsync(info, h->info, sizeof(info), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    const unsigned version = 1;
    const unsigned flags = (h->psi_valid ? 1u : 0u) | (h->S_valid ? 2u : 0u) | (h->norms_valid ? 4u : 0u);
    double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (user) memcpy(u, user, sizeof(u));
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return fail(h, FGPE_E_ARG, std::string("cannot open ") + tmp + " for writing");
    Fnv fnv;
    bool ok = true;
    auto put = [&](const void* p, size_t n) {
        if (!n) return;
        fnv.add(p, n);
        ok = ok && fwrite(p, 1, n, f) == n;
    };
    put(kCkpMagic, 8); put(&version, 4); put(&h->p, sizeof(fgpe_params)); put(&step, 8); put(u, sizeof(u));
    put(&flags, 4); put(info, sizeof(info)); put(psi.data(), psi.size()); put(S.data(), S.size());
    ok = ok && fwrite(&fnv.h, 1, 8, f) == 8;
    ok = (fclose(f) == 0) && ok;
    if (!ok || rename(tmp.c_str(), path) != 0) { remove(tmp.c_str()); return fail(h, FGPE_E_ARG, std::string("cannot write ") + path); }
    return FGPE_OK;
}

extern "C" int fgpe_checkpoint_load(fgpe_t* h, const char* path, long long* step, double* user) {
    if (!h || !path) return fail(h, FGPE_E_ARG, "null argument");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(h, FGPE_E_ARG, std::string("cannot open ") + path);
    std::vector<unsigned char> all;
    {
        unsigned char buf[1 << 16];
        size_t n;
        while ((n = fread(buf, 1, sizeof(buf), f)) > 0) all.insert(all.end(), buf, buf + n);
        fclose(f);
    }
    const size_t bytes = (size_t)h->npts * h->ms * h->cs;
    const size_t head = 8 + 4 + sizeof(fgpe_params) + 8 + 64 + 4 + sizeof(double) * INFO_LEN;
    if (all.size() < head + 8 || memcmp(all.data(), kCkpMagic, 8) != 0)
        return fail(h, FGPE_E_ARG, std::string(path) + " is not a checkpoint");
    Fnv fnv;
    fnv.add(all.data(), all.size() - 8);
    unsigned long long sum;
    memcpy(&sum, all.data() + all.size() - 8, 8);
    if (sum != fnv.h) return fail(h, FGPE_E_ARG, std::string(path) + ": checksum mismatch");
    size_t o = 8;
    unsigned version, flags;
    fgpe_params p;
    long long st;
    double u[8], info[INFO_LEN];
    memcpy(&version, &all[o], 4); o += 4;
    memcpy(&p, &all[o], sizeof(p)); o += sizeof(p);
    memcpy(&st, &all[o], 8); o += 8;
    memcpy(u, &all[o], 64); o += 64;
    memcpy(&flags, &all[o], 4); o += 4;
    memcpy(info, &all[o], sizeof(info)); o += sizeof(info);
    if (version != 1) return fail(h, FGPE_E_ARG, "unsupported checkpoint version");
    if (p.dim != h->p.dim || p.spin != h->p.spin || p.nx != h->p.nx || p.ny != h->p.ny || p.nz != h->p.nz ||
        p.precision != h->p.precision)
        return fail(h, FGPE_E_ARG, "checkpoint grid, spin or precision differs from the handle's");
    // a resume continues bit-identically only under the same physics: the
    // spacings, time step, time mode, couplings, trap and MAG must match too
    {
        bool same = p.dx == h->p.dx && p.dy == h->p.dy && p.dz == h->p.dz && p.dt == h->p.dt &&
                    p.imag_time == h->p.imag_time && p.mag == h->p.mag;
        for (int i = 0; i < 3; ++i)
            same = same && p.tau[i] == h->p.tau[i] && p.gamma[i] == h->p.gamma[i] && p.alpha[i] == h->p.alpha[i];
        if (!same)
            return fail(h, FGPE_E_ARG,
                        "checkpoint parameters (spacings, DT, time mode, TAU, GAMMA, ALPHA or MAG) differ from the handle's");
    }
    const size_t want = head + ((flags & 1) ? bytes : 0) + ((flags & 2) ? bytes : 0) + 8;
    if (all.size() != want || !(flags & 3)) return fail(h, FGPE_E_ARG, std::string(path) + ": truncated or malformed");
    if (flags & 1) { CK(cudaMemcpyAsync(h->psi, &all[o], bytes, cudaMemcpyHostToDevice, h->st)); o += bytes; }
    if (flags & 2) { CK(cudaMemcpyAsync(h->S, &all[o], bytes, cudaMemcpyHostToDevice, h->st)); o += bytes; }
    CK(cudaMemcpyAsync(h->info, info, sizeof(info), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));   // host buffers go out of scope
    h->psi_valid = (flags & 1) != 0;
    h->S_valid = (flags & 2) != 0;
    h->norms_valid = (flags & 4) != 0;
    h->prev_valid = false;
    h->has_state = true;
    if (step) *step = st;
    if (user) memcpy(user, u, sizeof(u));
    return FGPE_OK;
}

// ===================================================== NORMC without allocation
// fgpe_normc_noalloc: NORMC of a caller's device-resident spinor with no
// handle and no allocation of any kind.  Its only scratch is the file-scope
// array below (per-line Simpson integrals plus the last-block counter).  Its
// device address is looked up on every call, in the context current at the
// call: the first call in a context loads the module there (the set-up
// step), later lookups only read the runtime's symbol table and synchronise
// nothing.  So a context created after cudaDeviceReset, or a caller's own
// non-primary context, gets its own scratch rather than a stale address.
// The counter must be zero when a call starts: it is zero when the module is
// loaded and the last block of every call sets it back to zero.  The line
// values need no initial contents (every call writes all it reads).  Two calls
// in flight at once on one device share the scratch and race.
namespace {

constexpr long long kNoAllocMaxValues = 262144;  // lines x components (2 MiB)

struct NoAllocScratch {
    double line[kNoAllocMaxValues];
    unsigned int counter;
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Weight of node i (0-based) of the reference's SIMPSON (simpson.f90:4-21) on
// an even number n >= 8 of nodes: Simpson 1/3 over nodes 1..n-3 and 3/8 over
// the last four (1-based f): f=1 -> h/3; even f <= n-4 -> 4h/3; odd 3 <= f <=
// n-5 -> 2h/3; f=n-3 -> h/3 + 3h/8; f=n-2, n-1 -> 9h/8; f=n -> 3h/8.
__device__ __forceinline__ double noalloc_simpson_w(int i, int n, double h) {
    if (n == 1) return 1.0;
    const int f = i + 1;
    if (f == 1) return h / 3.0;
    if (f == n) return 3.0 * h / 8.0;
    if (f == n - 1 || f == n - 2) return 9.0 * h / 8.0;
    if (f == n - 3) return h / 3.0 + 3.0 * h / 8.0;
    return (f % 2 == 0) ? 4.0 * h / 3.0 : 2.0 * h / 3.0;
}

// One warp per x line: Simpson integral of |phi_m|^2 along x into the
// scratch; the last block to finish integrates the lines over y and z with
// the same weights in a fixed order and restores the counter.
template <int MS>
__global__ void __launch_bounds__(256)
k_normc_noalloc(const double2* __restrict__ phi, int nx, int ny, long long nlines, long long npts, double dx,
                double dy, double dz, int nz, NoAllocScratch* s, double* __restrict__ norm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long l = (long long)blockIdx.x * 8 + warp; l < nlines; l += (long long)gridDim.x * 8) {
        const double2* row = phi + l * nx;
#pragma unroll
        for (int m = 0; m < MS; ++m) {
            double acc = 0.0;
            for (int i = lane; i < nx; i += 32) {
                const double2 v = row[(size_t)m * npts + i];
                acc += noalloc_simpson_w(i, nx, dx) * (v.x * v.x + v.y * v.y);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) s->line[l * MS + m] = acc;
        }
    }
    __threadfence();
    __syncthreads();
    __shared__ unsigned int last;
    if (threadIdx.x == 0) last = (atomicAdd(&s->counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double red[256];
    for (int m = 0; m < MS; ++m) {
        double acc = 0.0;
        for (long long l = threadIdx.x; l < nlines; l += 256) {
            const int j = (int)(l % ny), k = (int)(l / ny);
            acc += noalloc_simpson_w(j, ny, dy) * noalloc_simpson_w(k, nz, dz) * __ldcg(&s->line[l * MS + m]);
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) norm[m] = red[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) s->counter = 0u;
}

}  // namespace

extern "C" int fgpe_normc_noalloc(int dim, int spin, int nx, int ny, int nz, double dx, double dy, double dz,
                                  const void* phi_dev, double* norm_dev, void* stream) {
    if (!phi_dev || !norm_dev) return fail(nullptr, FGPE_E_ARG, "null argument");
    if (dim < 1 || dim > 3) return fail(nullptr, FGPE_E_ARG, "dim must be 1, 2 or 3");
    if (spin != 1 && spin != 2) return fail(nullptr, FGPE_E_ARG, "spin must be 1 or 2");
    if (dim < 2) ny = 1;
    if (dim < 3) nz = 1;
    const int n[3] = {nx, ny, nz};
    const double d[3] = {dx, dy, dz};
    for (int a = 0; a < dim; ++a) {
        if (n[a] < 8 || n[a] % 2) return fail(nullptr, FGPE_E_ARG, "every grid axis needs an even number >= 8 of points");
        if (!(d[a] > 0.0)) return fail(nullptr, FGPE_E_ARG, "grid spacings must be positive");
    }
    const int ms = 2 * spin + 1;
    const long long nlines = (long long)ny * nz;
    if (nlines * ms > kNoAllocMaxValues)
        return fail(nullptr, FGPE_E_ARG,
                    "grid too large for the static scratch: (ny*nz lines) x components = " +
                        std::to_string(nlines * ms) + " exceeds " + std::to_string(kNoAllocMaxValues));
    NoAllocScratch* s = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&s, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(nullptr, FGPE_E_CUDA, std::string("scratch lookup: ") + cudaGetErrorString(e));
    const long long npts = nlines * nx;
    const unsigned grid = (unsigned)std::min<long long>((nlines + 7) / 8, 148LL * 8);
    cudaStream_t st = (cudaStream_t)stream;
    if (ms == 3)
        k_normc_noalloc<3><<<grid, 256, 0, st>>>((const double2*)phi_dev, nx, ny, nlines, npts, dx, dy, dz, nz, s, norm_dev);
    else
        k_normc_noalloc<5><<<grid, 256, 0, st>>>((const double2*)phi_dev, nx, ny, nlines, npts, dx, dy, dz, nz, s, norm_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(nullptr, FGPE_E_CUDA, cudaGetErrorString(e));
    return FGPE_OK;
}
