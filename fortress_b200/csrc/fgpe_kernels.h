// fgpe_kernels.h -- argument blocks shared by the kernels and the host API.
#pragma once
#include "fgpe_device.cuh"

namespace fgpe {

// Layout of the per-handle device "info" vector (doubles).
enum {
    INFO_TOTAL = 1,   // sum of the norms of the last step (before NORMT)
    INFO_ERR = 2,     // 1: non-finite reduction, 2: Newton projection failed
    INFO_NORM = 3,    // NORMC of the last step, MS values (3..7)
    INFO_SC = 8,      // pending per-component scale: phi_m = sc_m * psi_m (8..12)
    INFO_SIG = 13,    // SIG(1:2) of the spin-2 magnetisation projection (13, 14)
    INFO_LEN = 16
};

// Layout of the observables result vector.
enum {
    OBS_EN = 0, OBS_MZ = 1, OBS_CONV = 2, OBS_TOTAL = 3,
    OBS_NORM = 4, OBS_MU = 9, OBS_RMS = 14, OBS_LEN = 20
};

enum { ROW_FULL = 0, ROW_FWD = 1, ROW_INV = 2 };
// Column-pass work: COL_KE and COL_SOC act in k-space between the forward
// and inverse transforms of the pass (KE before SOC, cgpe3d.f90:452-454).
// Every step applies both in one pass (2D: the y pass; 3D: the z pass).
// COL_STEP marks the passes of a split step: between the forward and inverse y
// passes of a 3D step the y spectra never leave the step, so those passes may
// use a radix plan of their own (with ColArgs::fline / fother its maps).
enum { COL_SCALE = 1, COL_FWD = 2, COL_KE = 4, COL_INV = 8, COL_SOC = 16, COL_KOP = COL_KE | COL_SOC, COL_STEP = 32 };
enum { OBS_FULL = 0, OBS_NORMS = 1, OBS_NORMALIZE = 2 };
enum { OP_KE = 1, OP_SOC = 2, OP_SE = 3, OP_SP = 4, OP_SCALE = 5 };

struct RowArgs {
    void* S;           // x-spectral spinor (in/out)
    void* psi;         // real-space spinor (ROW_FWD source / ROW_INV target)
    void* snap;        // ROW_FULL: optional real-space snapshot target
    double* part;      // per-block NORMC partials
    unsigned* counter; // last-block counter (zero between launches)
    double* info;      // INFO_* vector
    int rows;          // rows (x lines) per block
    int mode;
};

struct ColArgs {
    void* S;
    const void* tw;    // twiddles of the transformed axis
    FftPlan plan;
    double* info;
    double cfac;       // 1/(NX*NY*NZ) folded into the scale on load
    long long axis_stride, other_stride;
    int n, tx, flags;
    int n_other;       // number of positions along the third axis (1 in 2D)
    int axis;          // transformed axis: 1 (y) or 2 (z)
    const int* fline;  // position -> frequency map of the transformed axis in the pass's radix plan
    const int* fother; // z lines: position -> frequency map of y, in the plan of the step's y passes
};

// Long 1D lines, N = N1*N2 points, handled as an N2 x N1 array (x = n1 + N1*n2)
// in two passes per step (four-step transform): the state between passes is
// Q[p2][n1] = W_N^(n1*k2) * sum_n2 x[n1 + N1*n2] W_N2^(n2*k2), row p2 holding
// the column frequency k2 = fy[p2].
enum { C1D_FULL = 0, C1D_FWD = 1, C1D_INV = 2 };
struct Split1dArgs {
    void* S;           // Q (in/out)
    void* psi;         // real space (C1D_FWD source, C1D_INV target)
    void* snap;        // C1D_FULL: optional real-space snapshot target
    const void* twn;   // W_N^j, j < N
    const void* tw1;   // twiddles of the N1 transform
    const void* tw2;   // twiddles of the N2 transform
    double* part;
    unsigned* counter;
    double* info;
    int n1, n2;
    int tile;          // rows (row pass) or columns (column pass) per block
    int mode;
};

// Long 1D lines on one thread-block cluster, resident for a whole call.
struct Cluster1dArgs {
    void* S;           // Q: loaded at entry, stored at exit (scales pending in info)
    void* snap_last;   // real-space state after the last step, or null
    void* snap_prev;   // real-space state after step nsteps-2, or null
    const void* twn;   // W_N^j, j < N
    const void* tw1;   // twiddles of the N1 transform
    const void* tw2;   // twiddles of the N2 transform
    double* info;      // INFO_* vector: scales and SIG in; norms, scales, SIG, error out
    double* info_prev; // receives the INFO_* vector after step nsteps-2 (with snap_prev)
    int n1, n2;
    int nsteps;
};

struct OneDArgs {
    void* psi;
    void* snap_prev;
    double* info;
    double* info_prev;
    int nsteps;
};

struct ObsArgs {
    const void* psi;
    const void* prev;
    double* info;
    const double* info_prev;
    double* part;
    unsigned* counter;
    double* out;
    double dx, dy, dz;
    int mode;
};

struct PointArgs {
    void* psi;
    int op;
    double factor;
};

}  // namespace fgpe
