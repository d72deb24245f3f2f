// fgpe_device.cuh -- device building blocks of the split-step propagator:
// complex helpers, the shared-memory Stockham FFT over many lines, and the
// per-point physics (KE+SOC in Fourier space, SE+SP in real space).
//
// Precision: T = double (plain FP64 path) or float (FP32 bulk path). Every
// reduction (norms, energies) is accumulated in double regardless of T.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fgpe {

// ---------------------------------------------------------------- complex
template <typename T> struct cx_t;
template <> struct cx_t<double> { typedef double2 type; };
template <> struct cx_t<float> { typedef float2 type; };
template <typename T> using cx = typename cx_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ cx<T> mk(T r, T i) { cx<T> z; z.x = r; z.y = i; return z; }
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
// acc + a * b and acc + a * conj(b), each part one chain of two FMAs onto acc
template <typename C> __host__ __device__ __forceinline__ C cmac(C acc, C a, C b) {
    C r; r.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x)); r.y = fma(a.x, b.y, fma(a.y, b.x, acc.y)); return r;
}
template <typename C> __host__ __device__ __forceinline__ C cmacc(C acc, C a, C b) {
    C r; r.x = fma(a.x, b.x, fma(a.y, b.y, acc.x)); r.y = fma(a.y, b.x, fma(-a.x, b.y, acc.y)); return r;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename S> __host__ __device__ __forceinline__ C cscale(C a, S s) { a.x *= s; a.y *= s; return a; }
// multiply by i (sign = +1) or -i (sign = -1)
template <typename C> __host__ __device__ __forceinline__ C cmuli(C a, int sign) {
    C r; if (sign > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; } return r;
}
template <typename C> __host__ __device__ __forceinline__ auto cabs2(C a) -> decltype(a.x) { return a.x * a.x + a.y * a.y; }

__device__ __forceinline__ void sincos_t(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ void sincos_t(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ double exp_t(double a) { return exp(a); }
__device__ __forceinline__ float exp_t(float a) { return expf(a); }
__device__ __forceinline__ double sqrt_t(double a) { return sqrt(a); }
__device__ __forceinline__ float sqrt_t(float a) { return sqrtf(a); }
__device__ __forceinline__ double sinh_t(double a) { return sinh(a); }
__device__ __forceinline__ float sinh_t(float a) { return sinhf(a); }
__device__ __forceinline__ double sin_t(double a) { return sin(a); }
__device__ __forceinline__ float sin_t(float a) { return sinf(a); }

// exp(-i CDT x) for real x: CDT = DT (real time) or -i DT (imaginary time).
template <typename T> __device__ __forceinline__ cx<T> cdt_phase(int imag, T dt, T x) {
    if (imag) return mk<T>(exp_t(-dt * x), (T)0);
    T s, c; sincos_t(dt * x, &s, &c);
    return mk<T>(c, -s);
}

// a * b where a is an exp(-i CDT x) factor: in imaginary time (CDT = -i DT)
// a is real, so the product is a scale (2 multiplies instead of 4 and 2 adds)
template <typename C> __device__ __forceinline__ C fmul(int imag, C a, C b) {
    if (imag) { b.x *= a.x; b.y *= a.x; return b; }
    return cmul(a, b);
}

// ------------------------------------------------------------------- FFT
// A transform length n = prod(r[0..nf-1]), radices from {2,3,4,5,8}.
//
// Forward transforms are in-place decimation in frequency: pass p works on
// blocks of Bp = n / (r0...r_{p-1}) elements, applies DFT_r to the r
// elements at stride Bp/r and then the twiddles W_Bp^{n2 k1}.  The spectrum
// comes out in mixed-radix digit-reversed order; a position->frequency map
// (per axis) tells the k-space operators which k sits where.  The inverse is
// the exact adjoint (conjugate twiddles, then DFT_r with +i, passes in reverse
// order) and takes digit-reversed input back to natural order, so no
// reordering pass is ever needed.  Every butterfly reads and writes only its
// own r slots: a thread holds r values, and passes are separated by one
// barrier.
struct FftPlan {
    int n, nf;
    int r[16];
};

__host__ __device__ __forceinline__ int padded_len(int n) { return n + (n + 7) / 8; }
__device__ __forceinline__ int pad_idx(int e) { return e + (e >> 3); }

// Lines of a row tile: line l starts at l*lp, element e at pad_idx(e) (one
// spare slot every 8 elements keeps strided butterflies off shared bank
// conflicts).
struct RowMap {
    int lp;
    __device__ __forceinline__ void split(int b, int nb, int& l, int& q) const { l = b / nb; q = b - l * nb; }
    __device__ __forceinline__ int base(int l) const { return l * lp; }
    __device__ __forceinline__ int at(int base, int e) const { return base + pad_idx(e); }
};

// Column tile [m][e][t], t < tx fastest (consecutive threads walk t first).
struct ColMap {
    int tx, lpn;  // tile width, padded line length
    __device__ __forceinline__ void split(int b, int nb, int& l, int& q) const {
        const int t = b % tx; const int w = b / tx; q = w % nb; const int m = w / nb; l = m * tx + t;
    }
    __device__ __forceinline__ int base(int l) const { return (l / tx) * lpn * tx + (l % tx); }
    __device__ __forceinline__ int at(int base, int e) const { return base + pad_idx(e) * tx; }
};

template <typename T, bool INV, int R> struct Dft;

template <typename T, bool INV> struct Dft<T, INV, 2> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        cx<T> a = v[0]; v[0] = cadd(a, v[1]); v[1] = csub(a, v[1]);
    }
};
template <typename T, bool INV> struct Dft<T, INV, 4> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        const int sg = INV ? 1 : -1;
        cx<T> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        cx<T> b0 = cadd(v[1], v[3]), b1 = cmuli(csub(v[1], v[3]), sg);
        v[0] = cadd(a0, b0); v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1); v[3] = csub(a1, b1);
    }
};
template <typename T, bool INV> struct Dft<T, INV, 8> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        const int sg = INV ? 1 : -1;
        const T h = (T)0.70710678118654752440084436210484903928;
        cx<T> a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { a[k] = cadd(v[k], v[k + 4]); b[k] = csub(v[k], v[k + 4]); }
        // b_k *= W8^k (forward W8 = e^{-i pi/4}; inverse its conjugate)
        b[1] = mk<T>(h * (b[1].x - sg * b[1].y), h * (b[1].y + sg * b[1].x));
        b[2] = cmuli(b[2], sg);
        b[3] = mk<T>(-h * (b[3].x + sg * b[3].y), h * (sg * b[3].x - b[3].y));
        Dft<T, INV, 4>::run(a);
        Dft<T, INV, 4>::run(b);
#pragma unroll
        for (int k = 0; k < 4; ++k) { v[2 * k] = a[k]; v[2 * k + 1] = b[k]; }
    }
};
// 16 points as 4 x 4: x[n1 + 4 n2] -> 4-point DFTs over n2, twiddles
// W16^(n1 k2), 4-point DFTs over n1 -> X[4 k1 + k2] (natural order out).
template <typename T, bool INV> struct Dft<T, INV, 16> {
    static __device__ __forceinline__ cx<T> rot(cx<T> a, T c, T s) {   // a * (c + i s)
        return mk<T>(a.x * c - a.y * s, a.x * s + a.y * c);
    }
    static __device__ __forceinline__ void run(cx<T>* v) {
        const T sg = INV ? (T)1 : (T)-1;
        const T c1 = (T)0.92387953251128675612818318939678828682;   // cos(pi/8)
        const T s1 = (T)0.38268343236508977172845998403039886676;   // sin(pi/8)
        const T h = (T)0.70710678118654752440084436210484903928;    // cos(pi/4)
        cx<T> y[4][4];
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) {
#pragma unroll
            for (int n2 = 0; n2 < 4; ++n2) y[n1][n2] = v[n1 + 4 * n2];
            Dft<T, INV, 4>::run(y[n1]);
        }
        // W16^m = cos(m pi/8) + i sg sin(m pi/8) for m = n1 k2
        y[1][1] = rot(y[1][1], c1, sg * s1);
        y[1][2] = rot(y[1][2], h, sg * h);
        y[1][3] = rot(y[1][3], s1, sg * c1);
        y[2][1] = rot(y[2][1], h, sg * h);
        y[2][2] = cmuli(y[2][2], INV ? 1 : -1);
        y[2][3] = rot(y[2][3], -h, sg * h);
        y[3][1] = rot(y[3][1], s1, sg * c1);
        y[3][2] = rot(y[3][2], -h, sg * h);
        y[3][3] = rot(y[3][3], -c1, -sg * s1);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) {
            cx<T> z[4] = {y[0][k2], y[1][k2], y[2][k2], y[3][k2]};
            Dft<T, INV, 4>::run(z);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) v[4 * k1 + k2] = z[k1];
        }
    }
};
template <typename T, bool INV> struct Dft<T, INV, 3> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        const T s = (T)0.86602540378443864676372317075293618347 * (INV ? 1 : -1);
        cx<T> t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        cx<T> y0 = cadd(v[0], t1);
        cx<T> m = mk<T>(v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y);
        cx<T> r = mk<T>(-s * t2.y, s * t2.x);  // i*s*t2
        v[0] = y0; v[1] = cadd(m, r); v[2] = csub(m, r);
    }
};
template <typename T, bool INV> struct Dft<T, INV, 5> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        const T c1 = (T)0.30901699437494742410229341718281905886;   // cos(2pi/5)
        const T c2 = (T)-0.80901699437494742410229341718281905886;  // cos(4pi/5)
        const T s1 = (T)0.95105651629515357211643933337938214340 * (INV ? 1 : -1);
        const T s2 = (T)0.58778525229247312916870595463907276860 * (INV ? 1 : -1);
        cx<T> a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        cx<T> a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        cx<T> y0 = cadd(v[0], cadd(a1, a2));
        cx<T> m1 = mk<T>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
        cx<T> m2 = mk<T>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
        // i*(s1 b1 + s2 b2) and i*(s2 b1 - s1 b2)
        cx<T> n1 = mk<T>(-(s1 * b1.y + s2 * b2.y), s1 * b1.x + s2 * b2.x);
        cx<T> n2 = mk<T>(-(s2 * b1.y - s1 * b2.y), s2 * b1.x - s1 * b2.x);
        v[0] = y0; v[1] = cadd(m1, n1); v[4] = csub(m1, n1); v[2] = cadd(m2, n2); v[3] = csub(m2, n2);
    }
};

// Twiddle powers w^1..w^(R-1) of w = tw[j]: in FP64 one table load and R-2
// complex products (w^2k = (w^k)^2, w^(2k+1) = w^2k * w) instead of R-1 loads
// that compete with the butterflies for the shared-memory/L1 bandwidth (the
// row pass of the 512^2 spin-2 step: 50.6 -> 43.6 us); the products add a few
// ulp.  In FP32 those ulp would be visible after a few steps, so FP32 loads
// every power.  FGPE_TW_POW 0 loads them in FP64 too.
#ifndef FGPE_TW_POW
#define FGPE_TW_POW 1
#endif
template <typename T, int R>
__device__ __forceinline__ void tw_powers(const cx<T>* __restrict__ tw, int j, int tstep, cx<T> (&w)[R]) {
    if (!FGPE_TW_POW || sizeof(T) == 4) {
#pragma unroll
        for (int r = 1; r < R; ++r) w[r] = tw[j * r * tstep];
        return;
    }
    w[1] = tw[j * tstep];
#pragma unroll
    for (int r = 2; r < R; ++r) w[r] = (r % 2 == 0) ? cmul(w[r / 2], w[r / 2]) : cmul(w[r - 1], w[1]);
}

template <typename T, bool INV, int R, class Map>
__device__ __forceinline__ void fft_pass(cx<T>* s, const Map& mp, int nlines, int n, int Bp,
                                         const cx<T>* __restrict__ tw) {
    const int si = Bp / R;
    const int nb = n / R;
    const int total = nlines * nb;
    const int tstep = n / Bp;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int l, q; mp.split(b, nb, l, q);
        const int blk = q / si, n2 = q - blk * si;
        const int e0 = blk * Bp + n2;
        const int bs = mp.base(l);
        cx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s[mp.at(bs, e0 + r * si)];
        if (!INV) {
            Dft<T, false, R>::run(v);
            if (n2) {
                cx<T> w[R];
                tw_powers<T, R>(tw, n2, tstep, w);
#pragma unroll
                for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
            }
        } else {
            if (n2) {
                cx<T> w[R];
                tw_powers<T, R>(tw, n2, tstep, w);
#pragma unroll
                for (int r = 1; r < R; ++r) v[r] = cmulc(v[r], w[r]);
            }
            Dft<T, true, R>::run(v);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) s[mp.at(bs, e0 + r * si)] = v[r];
    }
    __syncthreads();
}

template <typename T, bool INV, class Map>
__device__ __forceinline__ void fft_dispatch(int R, cx<T>* s, const Map& mp, int nlines, int n, int Bp,
                                             const cx<T>* __restrict__ tw) {
    switch (R) {
        case 8: fft_pass<T, INV, 8>(s, mp, nlines, n, Bp, tw); break;
        case 4: fft_pass<T, INV, 4>(s, mp, nlines, n, Bp, tw); break;
        case 2: fft_pass<T, INV, 2>(s, mp, nlines, n, Bp, tw); break;
        case 3: fft_pass<T, INV, 3>(s, mp, nlines, n, Bp, tw); break;
        default: fft_pass<T, INV, 5>(s, mp, nlines, n, Bp, tw); break;
    }
}

// Transform all nlines lines held in shared memory (caller has synchronised).
template <typename T, bool INV, class Map>
__device__ void block_fft(cx<T>* s, const Map& mp, int nlines, const FftPlan& pl, const cx<T>* __restrict__ tw) {
    if (!INV) {
        int Bp = pl.n;
        for (int p = 0; p < pl.nf; ++p) { fft_dispatch<T, false>(pl.r[p], s, mp, nlines, pl.n, Bp, tw); Bp /= pl.r[p]; }
    } else if (pl.nf > 0) {
        int Bp = pl.r[pl.nf - 1];
        for (int p = pl.nf - 1; p >= 0; --p) {
            fft_dispatch<T, true>(pl.r[p], s, mp, nlines, pl.n, Bp, tw);
            if (p > 0) Bp *= pl.r[p - 1];
        }
    }
}

// -------------------------------------------------------------- constants
struct StepConst {
    int dim, spin, ms;
    int nx, ny, nz;
    long long npts;
    double dt;
    int imag;
    double tau0, tau1, tau2;
    double gx, gy, gz;
    int se_half;              // 1D spin-2 predictor uses CDT/2 (cgpe1d.f90:1443)
    int se_ge;                // 1D spin-1 uses |OMEGA| >= EPS (cgpe1d.f90:1413)
    int project;              // imaginary time without SOC: magnetisation projection
    double mag;               // MAG of the projection
    const double *kx, *ky, *kz;
    const double *xg, *yg, *zg;
    const double *wx, *wy, *wz;     // Simpson weight vectors
    const double *vx, *vy, *vz;     // ALPHA^2 X^2 etc. (V is their sum)
    const void *twx, *twy, *twz;    // twiddle tables, complex T
    const void *kex, *key, *kez;    // kinetic factors: kex[nx], key[ny], kez[ms*nz]
    const void *pvx, *pvy, *pvz;    // potential factors exp(-i CDT ALPHA^2 X^2) per axis
    const int *fx, *fy, *fz;        // spectral position -> frequency index
    FftPlan px, py, pz;
    double* sink;                   // per-step NORMC ring (pinned host or device), or null
    unsigned* sink_ctr;             // steps appended since the ring was set
    int sink_n;                     // records of MS doubles in the ring
};

// Append one step's NORMC to the sink ring (called by one thread).
template <int MS>
__device__ __forceinline__ void sink_norms(const StepConst& c, const double* n) {
    if (!c.sink) return;
    const unsigned k = *c.sink_ctr;
    *c.sink_ctr = k + 1u;
    double* d = c.sink + (size_t)(k % (unsigned)c.sink_n) * MS;
    for (int m = 0; m < MS; ++m) d[m] = n[m];
}

// --------------------------------------------------------- SOC + KE at k
// Spin-orbit eigenbasis at beta = 0 (cgpe1d.f90:627-675; the beta-dependent
// matrices of cgpe2d.f90:1578-1638 are P(beta) A0 with
// P = diag(exp(-i (S-m) beta))).
template <int MS> struct A0;
template <> struct A0<3> {
    static __device__ __forceinline__ double at(int r, int c) {
        const double h = 0.70710678118654752440;
        const double a[3][3] = {{0.5, -h, 0.5}, {-h, 0.0, h}, {0.5, h, 0.5}};
        return a[r][c];
    }
};
template <> struct A0<5> {
    static __device__ __forceinline__ double at(int r, int c) {
        const double q = 0.61237243569579452455;  // sqrt(0.375)
        const double a[5][5] = {{0.25, -0.5, q, -0.5, 0.25},
                                {-0.5, 0.5, 0.0, -0.5, 0.5},
                                {q, 0.0, -0.5, 0.0, q},
                                {-0.5, -0.5, 0.0, 0.5, 0.5},
                                {0.25, 0.5, q, 0.5, 0.25}};
        return a[r][c];
    }
};

// exp(-i CDT x) for |dt x| <= 1/16 by the Taylor series of sin/cos (real
// time) or exp (imaginary time) truncated after the x^10 term: the first
// omitted term is below (1/16)^11/11! ~ 8e-22, under FP64 rounding.
template <typename T> __device__ __forceinline__ cx<T> small_phase(int imag, T th) {
    const T t2 = th * th;
    if constexpr (sizeof(T) == 4) {
        // FP32: terms to th^5; the first omitted one is below
        // (1/16)^6/6! ~ 8e-11, under FP32 rounding (6e-8)
        if (imag) {
            const T e = (T)1 - th * ((T)1 - th * ((T)(1.0 / 2) - th * ((T)(1.0 / 6) - th * ((T)(1.0 / 24)
                        - th * (T)(1.0 / 120)))));
            return mk<T>(e, (T)0);
        }
        const T cs = (T)1 - t2 * ((T)(1.0 / 2) - t2 * (T)(1.0 / 24));
        const T sn = th * ((T)1 - t2 * ((T)(1.0 / 6) - t2 * (T)(1.0 / 120)));
        return mk<T>(cs, -sn);
    }
    if (imag) {
        // exp(-th) = sum (-th)^k/k!
        const T e = (T)1 - th * ((T)1 - th * ((T)(1.0 / 2) - th * ((T)(1.0 / 6) - th * ((T)(1.0 / 24) - th * ((T)(1.0 / 120)
                    - th * ((T)(1.0 / 720) - th * ((T)(1.0 / 5040) - th * ((T)(1.0 / 40320) - th * ((T)(1.0 / 362880)
                    - th * (T)(1.0 / 3628800))))))))));
        return mk<T>(e, (T)0);
    }
    const T cs = (T)1 - t2 * ((T)(1.0 / 2) - t2 * ((T)(1.0 / 24) - t2 * ((T)(1.0 / 720) - t2 * ((T)(1.0 / 40320)
                 - t2 * (T)(1.0 / 3628800)))));
    const T sn = th * ((T)1 - t2 * ((T)(1.0 / 6) - t2 * ((T)(1.0 / 120) - t2 * ((T)(1.0 / 5040) - t2 * (T)(1.0 / 362880)))));
    return mk<T>(cs, -sn);
}

// v <- exp(-i CDT H_SO(k)) v with H_SO = A(beta) diag(L alpha) A(beta)^H,
// alpha = 2 sqrt(gx^2 kx^2 + gy^2 ky^2) in 2D/3D (cgpe2d.f90:1571-1594) and
// alpha = 2 gx kx, beta = 0 in 1D (cgpe1d.f90:1516-1520).
template <typename T, int MS>
__device__ __forceinline__ void apply_soc(const StepConst& c, double kx, double ky, cx<T>* v) {
    constexpr int S = MS / 2;
    double alpha, cb = 1.0, sb = 0.0;
    if (c.dim == 1) {
        alpha = 2.0 * c.gx * kx;
    } else {
        const double ax = c.gx * kx, ay = c.gy * ky;
        const double r2 = ax * ax + ay * ay;
        if (r2 > 0.0) {
            // one reciprocal square root for |.|, cos beta and sin beta
            const double ir = rsqrt(r2);
            alpha = 2.0 * r2 * ir;
            if (alpha > 1.0e-40) { cb = ax * ir; sb = ay * ir; }
        } else {
            alpha = 0.0;
        }
    }
    if (alpha == 0.0) return;  // exp(0) = 1
    // phases e^{i c beta}, c = S-m: w_m = conj(P_m) v_m = e^{+i (S-m) beta} v_m
    cx<T> e1 = mk<T>((T)cb, (T)sb);
    cx<T> e2 = cmul(e1, e1);
    cx<T> w[MS];
#pragma unroll
    for (int m = 0; m < MS; ++m) {
        const int cc = S - m;
        cx<T> ph = cc == 0 ? mk<T>(1, 0) : cc == 1 ? e1 : cc == -1 ? cconj(e1) : cc == 2 ? e2 : cconj(e2);
        w[m] = cmul(v[m], ph);
    }
    // u = A0^T w
    cx<T> u[MS];
#pragma unroll
    for (int r = 0; r < MS; ++r) {
        cx<T> s = mk<T>(0, 0);
#pragma unroll
        for (int q = 0; q < MS; ++q) {
            const T a = (T)A0<MS>::at(q, r);
            if (a != (T)0) { s.x += a * w[q].x; s.y += a * w[q].y; }
        }
        u[r] = s;
    }
    // u_L *= exp(-i CDT L alpha); the angle dt*alpha is small for resolved
    // grids, where the series of small_phase replaces sincos / exp
    const T th = (T)(c.dt * alpha);
    const bool small = fabs(th) <= (T)0.0625;
    const cx<T> l1 = small ? small_phase<T>(c.imag, th) : cdt_phase<T>(c.imag, (T)c.dt, (T)alpha);
    // real time: exp(+i dt alpha) = conj; imaginary time: exp(+dt alpha)
    const cx<T> lm1 = c.imag ? (small ? small_phase<T>(1, -th) : mk<T>(exp_t(th), (T)0)) : cconj(l1);
#pragma unroll
    for (int m = 0; m < MS; ++m) {
        const int L = m - S;
        if (L == 1) u[m] = cmul(u[m], l1);
        else if (L == -1) u[m] = cmul(u[m], lm1);
        else if (L == 2) u[m] = cmul(u[m], cmul(l1, l1));
        else if (L == -2) u[m] = cmul(u[m], cmul(lm1, lm1));
    }
    // w = A0 u ; v = P w
#pragma unroll
    for (int r = 0; r < MS; ++r) {
        cx<T> s = mk<T>(0, 0);
#pragma unroll
        for (int q = 0; q < MS; ++q) {
            const T a = (T)A0<MS>::at(r, q);
            if (a != (T)0) { s.x += a * u[q].x; s.y += a * u[q].y; }
        }
        const int cc = S - r;
        cx<T> ph = cc == 0 ? mk<T>(1, 0) : cc == 1 ? e1 : cc == -1 ? cconj(e1) : cc == 2 ? e2 : cconj(e2);
        v[r] = cmulc(s, ph);
    }
}

// KE (cgpe1d.f90:838, cgpe2d.f90:824, cgpe3d.f90:892): the factor
// exp(-i CDT |k|^2) is separable, precomputed per axis; 3D carries the
// per-component -2 L GAMMAZ KZ term in kez[m*nz + iz].
template <typename T, int MS>
__device__ __forceinline__ void apply_ke(const StepConst& c, int ix, int iy, int iz, cx<T>* v) {
    const cx<T>* kex = (const cx<T>*)c.kex;
    cx<T> f = kex[ix];
    if (c.dim >= 2) f = fmul(c.imag, f, ((const cx<T>*)c.key)[iy]);
    if (c.dim == 3) {
        const cx<T>* kez = (const cx<T>*)c.kez;
#pragma unroll
        for (int m = 0; m < MS; ++m) v[m] = fmul(c.imag, fmul(c.imag, f, kez[m * c.nz + iz]), v[m]);
    } else {
#pragma unroll
        for (int m = 0; m < MS; ++m) v[m] = fmul(c.imag, f, v[m]);
    }
}

// ------------------------------------------------------------- SE and SP
// Spin-2 couplings C12, C13, C23, C34, C35, C45 (MAT_C, cgpe1d.f90:928-952)
// from FX, FY (FXYZ with the reference's SX/SY, cgpe1d.f90:677-687).
template <typename T>
__device__ __forceinline__ void couplings2(const cx<T>* v, T t1, T t2, cx<T>* c) {
    const T s15 = (T)1.22474487139158904909864203735294569598;  // sqrt(1.5)
    cx<T> z01 = cmulc(v[1], v[0]);   // conj(v0) v1
    cx<T> z12 = cmulc(v[2], v[1]);
    cx<T> z23 = cmulc(v[3], v[2]);
    cx<T> z34 = cmulc(v[4], v[3]);
    const T fx = (T)2 * (z01.x + s15 * z12.x + s15 * z23.x + z34.x);
    const T fy = (T)2 * (z01.y + s15 * z12.y + s15 * z23.y + z34.y);
    const cx<T> fm = mk<T>(fx, -fy);  // FX - i FY
    const T a = (T)0.4 * t2, b = (T)0.2 * t2;
    cx<T> p;
    p = cmulc(v[3], v[4]); c[0] = mk<T>(t1 * fm.x - a * p.x, t1 * fm.y - a * p.y);
    p = cmulc(v[2], v[4]); c[1] = mk<T>(b * p.x, b * p.y);
    p = cmulc(v[2], v[3]); c[2] = mk<T>(s15 * t1 * fm.x - b * p.x, s15 * t1 * fm.y - b * p.y);
    p = cmulc(v[1], v[2]); c[3] = mk<T>(s15 * t1 * fm.x - b * p.x, s15 * t1 * fm.y - b * p.y);
    p = cmulc(v[0], v[2]); c[4] = mk<T>(b * p.x, b * p.y);
    p = cmulc(v[0], v[1]); c[5] = mk<T>(t1 * fm.x - a * p.x, t1 * fm.y - a * p.y);
}

// y = H v for the zero-diagonal Hermitian H with upper entries c; every
// further product of a row accumulates by FMA onto the first one.
template <typename T>
__device__ __forceinline__ void hmul(const cx<T>* c, const cx<T>* v, cx<T>* y) {
    y[0] = cmac(cmul(c[0], v[1]), c[1], v[2]);
    y[1] = cmac(cmulc(v[0], c[0]), c[2], v[2]);
    y[2] = cmac(cmac(cmacc(cmulc(v[0], c[1]), v[1], c[2]), c[3], v[3]), c[4], v[4]);
    y[3] = cmac(cmulc(v[2], c[3]), c[5], v[4]);
    y[4] = cmacc(cmulc(v[2], c[4]), v[3], c[5]);
}

// 1/k for k <= 41 (k = 0 unused), so that the Taylor loops of the spin-2 SE
// multiply instead of dividing (an FP64 division costs tens of instructions).
static __constant__ double kInvK[42] = {0.0, 1.0 / 1, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8, 1.0 / 9, 1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20, 1.0 / 21, 1.0 / 22, 1.0 / 23, 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30, 1.0 / 31, 1.0 / 32, 1.0 / 33, 1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39, 1.0 / 40, 1.0 / 41};
template <typename T> __device__ __forceinline__ T inv_k(int k) { return (T)kInvK[k]; }

template <typename T> struct Eps;
template <> struct Eps<double> { static __device__ __forceinline__ double v() { return 1.1e-16; } };
template <> struct Eps<float> { static __device__ __forceinline__ float v() { return 6.0e-8f; } };

// Spin-2 SE (cgpe2d.f90:1480-1547): predictor phi1 = phi - i cdp C(phi) phi,
// corrector C = (C(phi) + C(phi1))/2, then phi <- exp(-i CDT H(C)) phi.  The
// reference diagonalises H with ZHEEV; the exponential's action is computed
// here by a scaled Taylor series (terms until below rounding), which yields
// the same unique matrix function.
template <typename T>
__device__ __forceinline__ void se_spin2(const StepConst& c, cx<T>* v) {
    const T t1 = (T)c.tau1, t2 = (T)c.tau2;
    cx<T> ca[6], cb[6], p1[5], hv[5];
    couplings2<T>(v, t1, t2, ca);
    // -i*cdp: real time -i dt (/2 in 1D), imaginary time -dt (/2)
    const T dtp = (T)(c.se_half ? 0.5 * c.dt : c.dt);
    hmul<T>(ca, v, hv);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        if (c.imag) p1[m] = mk<T>(v[m].x - dtp * hv[m].x, v[m].y - dtp * hv[m].y);
        else p1[m] = mk<T>(v[m].x + dtp * hv[m].y, v[m].y - dtp * hv[m].x);
    }
    couplings2<T>(p1, t1, t2, cb);
#pragma unroll
    for (int q = 0; q < 6; ++q) ca[q] = mk<T>((ca[q].x + cb[q].x) * (T)0.5, (ca[q].y + cb[q].y) * (T)0.5);
    // bound ||H||_1 with |re|+|im| per entry
    T a[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) a[q] = fabs(ca[q].x) + fabs(ca[q].y);
    T col = fmax(fmax(a[0] + a[1], a[0] + a[2]), fmax(a[1] + a[2] + a[3] + a[4], fmax(a[3] + a[5], a[4] + a[5])));
    const T dt = (T)c.dt;
    const T nrm = dt * col;
    if (nrm == (T)0) return;
    int nsub = 1;
    T h = dt, hn = nrm;        // z = -i h (real) or -h (imag)
    if (nrm > (T)0.5) {
        nsub = (int)ceil(nrm / (T)0.5);
        if (nsub > 4096) nsub = 4096;
        h = dt / (T)nsub;
        hn = nrm / (T)nsub;
    }
    // Number of Taylor terms fixed beforehand: the remainder after K terms is
    // below hn^(K+1)/(K+1)! * e^hn relative to |v|, and |y| >= e^-hn |v|
    // (e^{-h H} can contract by at most e^-hn), so stop once
    // hn^(K+1)/(K+1)! * e^(2 hn) <= eps.  On 0 <= hn <= 1/2, e^(2 hn) lies
    // below its chord 1 + 2 (e - 1) hn < 1 + 4 hn, which stands in for it.
    // hn <= 1/2 keeps K <= 18 in FP64.
    int K = 1;
    {
        const T e2 = (T)1 + (T)4 * hn;
        T bnd = hn * hn * (T)0.5;
        while (bnd * e2 > Eps<T>::v() * (T)0.5 && K < 40) { ++K; bnd *= hn * inv_k<T>(K + 1); }
    }
    for (int sidx = 0; sidx < nsub; ++sidx) {
        cx<T> term[5], y[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) { term[m] = v[m]; y[m] = v[m]; }
        for (int k = 1; k <= K; ++k) {
            hmul<T>(ca, term, hv);
            const T f = h * inv_k<T>(k);
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                if (c.imag) term[m] = mk<T>(-f * hv[m].x, -f * hv[m].y);
                else term[m] = mk<T>(f * hv[m].y, -f * hv[m].x);
                y[m] = cadd(y[m], term[m]);
            }
        }
#pragma unroll
        for (int m = 0; m < 5; ++m) v[m] = y[m];
    }
}

// Spin-1 SE closed form (cgpe2d.f90:1449-1479): A1 = tau1 phi2 phi3*,
// B1 = tau1 phi2 phi1*, OMEGA = CDT sqrt(|A1|^2+|B1|^2); the products
// DELTA*CDT^2 and KAPPA*CDT are real / purely imaginary and are formed
// directly (cos x - 1 = -2 sin^2(x/2) avoids the cancellation).
template <typename T>
__device__ __forceinline__ void se_spin1(const StepConst& c, cx<T>* v) {
    const T t1 = (T)c.tau1;
    cx<T> A1 = cscale(cmulc(v[1], v[2]), t1);
    cx<T> B1 = cscale(cmulc(v[1], v[0]), t1);
    const T aa = cabs2(A1), bb = cabs2(B1);
    const T r2 = aa + bb;
    const T dt = (T)c.dt;
    T dc;                 // DELTA*CDT^2 (real)
    T kf;                 // KAPPA*CDT = kf (imaginary time) or i kf (real time)
    const T z = dt * dt * r2;   // |OMEGA|^2
    if (z <= (T)(1.0 / 256)) {
        // |OMEGA| <= 1/16: 2 sinh^2(x/2)/x^2 = sum x^2n/(2n+2)!, sinh(x)/x =
        // sum x^2n/(2n+1)! (sin: x^2 -> -x^2), to x^10 (next term < 1e-20
        // relative): no square root, division or transcendental call, and the
        // |OMEGA| -> 0 limits (DELTA*CDT^2 = CDT^2/2, KAPPA*CDT = -i CDT) are
        // the leading terms
        const T zz = c.imag ? z : -z;
        T g, f;
        if constexpr (sizeof(T) == 4) {
            // FP32: to x^4; the next terms are below (1/256)^3/8! ~ 1.5e-12
            g = (T)(1.0 / 2) + zz * ((T)(1.0 / 24) + zz * (T)(1.0 / 720));
            f = (T)1 + zz * ((T)(1.0 / 6) + zz * (T)(1.0 / 120));
        } else {
            g = (T)(1.0 / 2) + zz * ((T)(1.0 / 24) + zz * ((T)(1.0 / 720) + zz * ((T)(1.0 / 40320) +
                zz * ((T)(1.0 / 3628800) + zz * (T)(1.0 / 479001600)))));
            f = (T)1 + zz * ((T)(1.0 / 6) + zz * ((T)(1.0 / 120) + zz * ((T)(1.0 / 5040) +
                zz * ((T)(1.0 / 362880) + zz * (T)(1.0 / 39916800)))));
        }
        dc = (c.imag ? (T)1 : (T)-1) * dt * dt * g;
        kf = -dt * f;
    } else {
    const T r = sqrt_t(r2);
    const T x = dt * r;   // |OMEGA|
    const bool big = c.se_ge ? (x >= (T)1e-40) : (x > (T)1e-40);
    if (c.imag) {
        if (big) { T sh = sinh_t((T)0.5 * x); dc = (T)2 * sh * sh / r2; kf = -sinh_t(x) / r; }
        else { dc = (T)0.5 * dt * dt; kf = -dt; }
    } else {
        if (big) { T sn = sin_t((T)0.5 * x); dc = (T)-2 * sn * sn / r2; kf = -sin_t(x) / r; }
        else { dc = (T)-0.5 * dt * dt; kf = -dt; }
    }
    }
    const cx<T> p1 = v[0], p2 = v[1], p3 = v[2];
    // TMP(1) = dc (|A1|^2 p1 + A1 B1* p3) + KAPPA*CDT A1 p2
    cx<T> u1 = cadd(cscale(p1, aa), cmul(cmulc(A1, B1), p3));
    cx<T> u3 = cadd(cmul(cmulc(B1, A1), p1), cscale(p3, bb));
    // KAPPA*CDT is real or purely imaginary: its products are two multiplies
    auto kmul = [&](cx<T> q) { return c.imag ? mk<T>(kf * q.x, kf * q.y) : mk<T>(-kf * q.y, kf * q.x); };
    cx<T> w1 = kmul(cmul(A1, p2));
    cx<T> w2 = kmul(cadd(cmulc(p1, A1), cmulc(p3, B1)));
    cx<T> w3 = kmul(cmul(B1, p2));
    v[0] = cadd(p1, cadd(cscale(u1, dc), w1));
    v[1] = cadd(p2, cadd(cscale(p2, dc * r2), w2));
    v[2] = cadd(p3, cadd(cscale(u3, dc), w3));
}


// exp(-i CDT V) at grid point (i, j, k): V = vx + vy + vz is separable, so
// the factor is the product of the per-axis tables.
template <typename T>
__device__ __forceinline__ cx<T> pot_phase(const StepConst& c, int i, int j, int k) {
    cx<T> e = ((const cx<T>*)c.pvx)[i];
    if (c.dim >= 2) e = fmul(c.imag, e, ((const cx<T>*)c.pvy)[j]);
    if (c.dim >= 3) e = fmul(c.imag, e, ((const cx<T>*)c.pvz)[k]);
    return e;
}

// SP (cgpe1d.f90:847-896): phi_m <- phi_m exp(-i CDT T_m), densities after SE.
// T_m = V + tau0 rho + B_m.  exp(-i CDT V) = eV comes from the per-axis
// tables (pot_phase); the density parts tau0 rho and B_m (tau1/tau2 terms)
// are small for physical states and use small_phase when |dt x| <= 1/16.
template <typename T, int MS>
__device__ __forceinline__ void apply_sp(const StepConst& c, cx<T> eV, cx<T>* v) {
    const T t0 = (T)c.tau0, t1 = (T)c.tau1, t2 = (T)c.tau2;
    T a[MS], rho = 0;
#pragma unroll
    for (int m = 0; m < MS; ++m) { a[m] = cabs2(v[m]); rho += a[m]; }
    T B[MS];
    if constexpr (MS == 3) {
        B[0] = t1 * (a[0] + a[1] - a[2]);
        B[1] = t1 * (a[0] + a[2]);
        B[2] = t1 * (a[2] + a[1] - a[0]);
    } else {
        const T fz = (T)2 * a[0] + a[1] - a[MS - 2] - (T)2 * a[MS - 1];
        B[0] = (T)2 * t1 * fz + (T)0.4 * t2 * a[MS - 1];
        B[1] = t1 * fz + (T)0.4 * t2 * a[MS - 2];
        B[2] = (T)0.2 * t2 * a[2];
        B[MS - 2] = -t1 * fz + (T)0.4 * t2 * a[1];
        B[MS - 1] = (T)-2 * t1 * fz + (T)0.4 * t2 * a[0];
    }
    // one phase per component for the density parts, exp(-i CDT (tau0 rho +
    // B_m)), as the reference takes one exponential of T_m (cgpe1d.f90:
    // 871-873, 890-892); in imaginary time every factor is real
    const T dt = (T)c.dt;
    const T d0 = t0 * rho;
#pragma unroll
    for (int m = 0; m < MS; ++m) {
        const T x = d0 + B[m];
        const T th = dt * x;
        const cx<T> eB = fabs(th) <= (T)0.0625 ? small_phase<T>(c.imag, th) : cdt_phase<T>(c.imag, dt, x);
        v[m] = fmul(c.imag, fmul(c.imag, eV, eB), v[m]);
    }
}

template <typename T, int MS>
__device__ __forceinline__ void apply_se(const StepConst& c, cx<T>* v) {
    if constexpr (MS == 3) se_spin1<T>(c, v);
    else se_spin2<T>(c, v);
}

// --------------------------------------------- renormalisation scales
// After a step's NORMC (norms n[m]): the scales that bring phi to the next
// step, phi_m <- sc_m phi_m.
//  real time: 1.
//  imaginary time with SOC: NORMT, sc_m = 1/sqrt(sum n) (cgpe1d.f90:472).
//  imaginary time without SOC: projection PHI_m <- SIGMA_m PHI_m, then NORMT
//  (cgpe1d.f90:443-470): spin-1 closed form (cgpe1d.f90:447-450; the 3D
//  program places EPS inside the square root, cgpe3d.f90:464-465), spin-2
//  SIGMA_m = exp((SIG1 + c_m SIG2) DT) with SIG from the Newton-Raphson solve
//  of NEWTON/USRFUN (cgpe1d.f90:1245-1319), started from the previous step's
//  SIG (20, 20 initially), NTRIAL = 1000, TOL_NR = 1e-6.
// Returns 0, or 2 when the Newton iteration did not converge.
template <int MS>
__device__ int compute_scales(const StepConst& c, const double* n, double* sig, double* sc) {
    double tot = 0;
    for (int m = 0; m < MS; ++m) tot += n[m];
    if (!c.imag) { for (int m = 0; m < MS; ++m) sc[m] = 1.0; return 0; }
    if (!c.project) { const double s = 1.0 / sqrt(tot); for (int m = 0; m < MS; ++m) sc[m] = s; return 0; }
    const double EPSV = 1.0e-40, mag = c.mag;
    double sg[MS];
    int rc = 0;
    if constexpr (MS == 3) {
        const double inner = sqrt(4.0 * (1.0 - mag * mag) * n[0] * n[2] + mag * mag * n[1] * n[1]);
        if (c.dim == 3) sg[1] = sqrt(1.0 - mag * mag) / sqrt(n[1] + inner + EPSV);
        else sg[1] = sqrt(1.0 - mag * mag) / (sqrt(n[1] + inner) + EPSV);
        sg[0] = sqrt(1.0 + mag - sg[1] * sg[1] * n[1]) / (sqrt(2.0 * n[0]) + EPSV);
        sg[2] = sqrt(1.0 - mag - sg[1] * sg[1] * n[1]) / (sqrt(2.0 * n[2]) + EPSV);
    } else {
        const double dt = c.dt;
        double x1 = sig[0], x2 = sig[1], p1 = 0, p2 = 0;
        for (int k = 0; k < 1000; ++k) {
            const double e1 = exp(2.0 * (x1 + 2.0 * x2) * dt), e2 = exp(2.0 * (x1 + x2) * dt), e3 = exp(2.0 * x1 * dt),
                         e4 = exp(2.0 * (x1 - x2) * dt), e5 = exp(2.0 * (x1 - 2.0 * x2) * dt);
            const double f1 = e1 * n[0] + e2 * n[1] + e3 * n[2] + e4 * n[3] + e5 * n[4] - 1.0;
            const double f2 = 2.0 * e1 * n[0] + e2 * n[1] - e4 * n[3] - 2.0 * e5 * n[4] - mag;
            const double j11 = (e1 * n[0] + e2 * n[1] + e3 * n[2] + e4 * n[3] + e5 * n[4]) * 2.0 * dt;
            const double j12 = e1 * n[0] * 4.0 * dt + e2 * n[1] * 2.0 * dt + e4 * n[3] * (-2.0 * dt) + e5 * n[4] * (-4.0 * dt);
            const double j21 = (2.0 * e1 * n[0] + e2 * n[1] - e4 * n[3] - 2.0 * e5 * n[4]) * 2.0 * dt;
            const double j22 = 2.0 * e1 * n[0] * 4.0 * dt + e2 * n[1] * 2.0 * dt - e4 * n[3] * (-2.0 * dt)
                               - 2.0 * e5 * n[4] * (-4.0 * dt);
            p2 = (f2 * j11 - f1 * j21) / (j21 * j12 - j11 * j22);
            p1 = (-f1 - j12 * p2) / j11;
            x1 += p1; x2 += p2;
            if (fmax(fabs(p1), fabs(p2)) <= 1.0e-6) break;
        }
        if (fmax(fabs(p1), fabs(p2)) > 1.0e-6) rc = 2;
        sig[0] = x1; sig[1] = x2;
        for (int m = 0; m < MS; ++m) sg[m] = exp((x1 + (2 - m) * x2) * dt);
    }
    double t2 = 0;
    for (int m = 0; m < MS; ++m) t2 += sg[m] * sg[m] * n[m];
    const double inv = 1.0 / sqrt(t2);
    for (int m = 0; m < MS; ++m) sc[m] = sg[m] * inv;
    return rc;
}

}  // namespace fgpe
