/*
 * cgpe_oracle.c -- CPU restatement (FP64, OpenMP) of the FORTRESS split-step
 * Fourier propagator for spin-orbit-coupled spin-1 / spin-2 condensates.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: only tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline legs of bench.py load it,
 * and only to compare results against.  The product library (fortress_b200)
 * never links, loads or calls it.
 *
 * Every routine names the reference routine it restates (file:line in the
 * FORTRESS sources SRC/cgpe1d.f90, SRC/cgpe2d.f90, SRC/cgpe3d.f90,
 * SRC/diff.f90, SRC/simpson.f90).  Two third-party pieces of the reference are
 * not part of its sources and are restated from their published algorithms:
 *   - FFTW3 c2c transforms (version unpinned by the reference Makefile):
 *     here a mixed-radix Stockham FFT, forward sign -1, unnormalised.
 *   - LAPACK ZHEEV (unpinned): here a cyclic complex Jacobi eigensolver; the
 *     matrix exponential V diag(exp(-i CDT w)) V^H it feeds is unique, so the
 *     eigenvector phase convention does not matter.
 *
 * Parity pin: the oracle is checked against the reference's only known-answer
 * output (OUTPUT/ of the 1D spin-2 run of INPUT/input1D.dat), see
 * tests/test_oracle_golden.py.
 *
 * Layout: the state is Fortran column-major PHI(NX,NY,NZ,M), complex128,
 * x fastest, one contiguous block per spin component.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cd;

/* cgpe1d.f90:33-37 */
static const double PI = 3.14159265358979323846264338327950288;
static const double AMU = 1.66e-27, HBAR = 1.054560653e-34, AU = 0.529177208e-10;
static const double EPS = 1.0e-40;

typedef struct {
    int dim, spin;             /* 1..3, 1..2 */
    int nx, ny, nz;            /* ny = nz = 1 in 1D, nz = 1 in 2D */
    double dx, dy, dz, dt;
    int imag;                  /* SWITCH_IM */
    double tau[3];
    double gx, gy, gz;         /* GAMMAX, GAMMAY, GAMMAZ */
    double ax, ay, az;         /* ALPHAX, ALPHAY, ALPHAZ */
} orc_params;

/* ------------------------------------------------------------------ FFT */
typedef struct {
    int n, nf;
    int fac[40];
    cd *w;      /* w[t] = exp(-2 pi i t / n) */
} fftplan;

static void plan_init(fftplan *p, int n) {
    p->n = n; p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2)
        while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
    p->w = (cd *)malloc(sizeof(cd) * (size_t)n);
    for (int t = 0; t < n; ++t) {
        double a = -2.0 * PI * (double)t / (double)n;
        p->w[t] = cos(a) + I * sin(a);
    }
}

static void plan_free(fftplan *p) { free(p->w); p->w = NULL; }

/* One Stockham autosort transform of x (length n); y is scratch.  sign = -1
 * forward (FFTW_FORWARD), +1 backward; unnormalised like FFTW.  The result
 * ends up in x. */
static void fft1(const fftplan *p, cd *x, cd *y, int sign) {
    const int n = p->n;
    if (n == 1) return;
    cd *src = x, *dst = y;
    int ns = 1;
    cd v[64], o[64];
    for (int f = 0; f < p->nf; ++f) {
        const int r = p->fac[f];
        const int nr = n / r;
        const int tstep = n / (ns * r);
        for (int j = 0; j < nr; ++j) {
            const int k = j % ns;
            for (int q = 0; q < r; ++q) {
                cd tw = p->w[(size_t)((long)q * k * tstep % n)];
                if (sign > 0) tw = conj(tw);
                v[q] = src[j + q * nr] * tw;
            }
            if (r == 2) {
                o[0] = v[0] + v[1]; o[1] = v[0] - v[1];
            } else if (r == 4) {
                cd a0 = v[0] + v[2], a1 = v[0] - v[2];
                cd b0 = v[1] + v[3], b1 = (v[1] - v[3]) * (sign < 0 ? -I : I);
                o[0] = a0 + b0; o[2] = a0 - b0;
                o[1] = a1 + b1; o[3] = a1 - b1;
            } else {
                /* generic odd factor: naive DFT of length r */
                for (int a = 0; a < r; ++a) {
                    cd s = 0;
                    for (int b = 0; b < r; ++b) {
                        cd tw = p->w[(size_t)((long)a * b % r) * (n / r)];
                        if (sign > 0) tw = conj(tw);
                        s += v[b] * tw;
                    }
                    o[a] = s;
                }
            }
            const int base = (j / ns) * ns * r + k;
            for (int q = 0; q < r; ++q) dst[base + q * ns] = o[q];
        }
        cd *t = src; src = dst; dst = t;
        ns *= r;
    }
    if (src != x) memcpy(x, src, sizeof(cd) * (size_t)n);
}

/* ------------------------------------------------------------- handle */
typedef struct {
    orc_params p;
    int ms;                    /* 2*SPIN+1 */
    long npts;                 /* NX*NY*NZ */
    cd cdt;                    /* CDT: -i DT (imaginary) or DT (real) */
    double *x, *y, *z, *kx, *ky, *kz;
    cd *phi;                   /* PHI(NX,NY,NZ,MS) */
    fftplan px, py, pz;
    int switch_soc;            /* cgpe1d.f90:250 */
    double mag;                /* MAG */
    double sig[2];             /* SIG(1:2), cgpe1d.f90:425-426 */
} orc_t;

static inline long IDX(const orc_t *h, int i, int j, int k) {
    return i + (long)h->p.nx * (j + (long)h->p.ny * k);
}

/* Grids, cgpe1d.f90:692-704 (KX in FFT order, Nyquist positive; X centred). */
static void make_k(double *k, int n, double l) {
    for (int i = 1; i <= 1 + n / 2; ++i) k[i - 1] = (i - 1.0) * 2.0 * PI / l;
    for (int i = 1; i <= n / 2 - 1; ++i) k[i + n / 2] = -k[n / 2 - i];
}
static void make_x(double *x, int n, double l) {
    for (int i = 1; i <= n; ++i) x[i - 1] = (-1.0 + 2.0 * (i - 1.0) / n) * l / 2.0;
}

orc_t *orc_create(const orc_params *p) {
    orc_t *h = (orc_t *)calloc(1, sizeof(orc_t));
    h->p = *p;
    if (h->p.dim < 2) { h->p.ny = 1; h->p.dy = 1.0; }
    if (h->p.dim < 3) { h->p.nz = 1; h->p.dz = 1.0; }
    h->ms = 2 * p->spin + 1;
    h->npts = (long)h->p.nx * h->p.ny * h->p.nz;
    h->cdt = p->imag ? -I * p->dt : p->dt + 0.0 * I;   /* cgpe1d.f90:292, 306 */
    h->x = calloc(h->p.nx, sizeof(double)); h->kx = calloc(h->p.nx, sizeof(double));
    h->y = calloc(h->p.ny, sizeof(double)); h->ky = calloc(h->p.ny, sizeof(double));
    h->z = calloc(h->p.nz, sizeof(double)); h->kz = calloc(h->p.nz, sizeof(double));
    make_k(h->kx, h->p.nx, h->p.nx * h->p.dx); make_x(h->x, h->p.nx, h->p.nx * h->p.dx);
    if (h->p.dim >= 2) { make_k(h->ky, h->p.ny, h->p.ny * h->p.dy); make_x(h->y, h->p.ny, h->p.ny * h->p.dy); }
    if (h->p.dim >= 3) { make_k(h->kz, h->p.nz, h->p.nz * h->p.dz); make_x(h->z, h->p.nz, h->p.nz * h->p.dz); }
    h->phi = (cd *)calloc((size_t)h->npts * h->ms, sizeof(cd));
    plan_init(&h->px, h->p.nx); plan_init(&h->py, h->p.ny); plan_init(&h->pz, h->p.nz);
    /* cgpe1d.f90:250, cgpe2d.f90:251, cgpe3d.f90:256 */
    h->switch_soc = fabs(p->gx) > EPS || (p->dim >= 2 && fabs(p->gy) > EPS) || (p->dim >= 3 && fabs(p->gz) > EPS);
    h->mag = 0.0;
    h->sig[0] = h->sig[1] = 20.0;
    return h;
}

void orc_destroy(orc_t *h) {
    if (!h) return;
    free(h->x); free(h->y); free(h->z); free(h->kx); free(h->ky); free(h->kz);
    free(h->phi);
    plan_free(&h->px); plan_free(&h->py); plan_free(&h->pz);
    free(h);
}

void orc_set_state(orc_t *h, const double *re_im) {
    memcpy(h->phi, re_im, sizeof(cd) * (size_t)h->npts * h->ms);
}
void orc_get_state(const orc_t *h, double *re_im) {
    memcpy(re_im, h->phi, sizeof(cd) * (size_t)h->npts * h->ms);
}
void orc_grids(const orc_t *h, double *x, double *y, double *z, double *kx, double *ky, double *kz) {
    memcpy(x, h->x, sizeof(double) * h->p.nx); memcpy(kx, h->kx, sizeof(double) * h->p.nx);
    memcpy(y, h->y, sizeof(double) * h->p.ny); memcpy(ky, h->ky, sizeof(double) * h->p.ny);
    memcpy(z, h->z, sizeof(double) * h->p.nz); memcpy(kz, h->kz, sizeof(double) * h->p.nz);
}

static double V_at(const orc_t *h, int i, int j, int k) {
    /* V = ALPHAX^2 X^2 (+ ALPHAY^2 Y^2 (+ ALPHAZ^2 Z^2)), cgpe1d.f90:710,
     * cgpe2d.f90:693, cgpe3d.f90:752 */
    double v = h->p.ax * h->p.ax * h->x[i] * h->x[i];
    if (h->p.dim >= 2) v += h->p.ay * h->p.ay * h->y[j] * h->y[j];
    if (h->p.dim >= 3) v += h->p.az * h->p.az * h->z[k] * h->z[k];
    return v;
}

/* ------------------------------------------------------- FFT / BFT (C4) */
/* FFT: cgpe1d.f90:1324-1338, cgpe2d.f90:1364-1378, cgpe3d.f90:1748-1763.
 * BFT: cgpe1d.f90:1343-1358 etc., divides by NX*NY*NZ. Full d-dimensional
 * c2c transform of each component (PLAN_DFT_2D(NY,NX) on column-major data is
 * the ordinary 2D DFT with x fastest). */
static void fft_axis(orc_t *h, cd *a, int axis, int sign) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    const fftplan *pl = axis == 0 ? &h->px : axis == 1 ? &h->py : &h->pz;
    const int n = pl->n;
    if (n == 1) return;
    const long nlines = h->npts / n;
#pragma omp parallel
    {
        cd *line = (cd *)malloc(sizeof(cd) * n), *scr = (cd *)malloc(sizeof(cd) * n);
#pragma omp for schedule(static)
        for (long L = 0; L < nlines; ++L) {
            long base, stride;
            if (axis == 0) { base = L * nx; stride = 1; }
            else if (axis == 1) { long i = L % nx, k = L / nx; base = i + (long)nx * ny * k; stride = nx; }
            else { base = L; stride = (long)nx * ny; }
            for (int t = 0; t < n; ++t) line[t] = a[base + t * stride];
            fft1(pl, line, scr, sign);
            for (int t = 0; t < n; ++t) a[base + t * stride] = line[t];
        }
        free(line); free(scr);
    }
    (void)nz;
}

void orc_fft(orc_t *h) {
    for (int m = 0; m < h->ms; ++m) {
        cd *a = h->phi + (size_t)m * h->npts;
        for (int ax = 0; ax < h->p.dim; ++ax) fft_axis(h, a, ax, -1);
    }
}

void orc_bft(orc_t *h) {
    for (int m = 0; m < h->ms; ++m) {
        cd *a = h->phi + (size_t)m * h->npts;
        for (int ax = 0; ax < h->p.dim; ++ax) fft_axis(h, a, ax, +1);
    }
    const long tot = h->npts * h->ms;
#pragma omp parallel for
    for (long t = 0; t < tot; ++t) h->phi[t] = h->phi[t] / (double)h->npts;
}

/* Plain 1D transforms exposed for the FFT cross-check against numpy. */
void orc_fft1d(int n, double *re_im, int sign) {
    fftplan p; plan_init(&p, n);
    cd *scr = malloc(sizeof(cd) * n);
    fft1(&p, (cd *)re_im, scr, sign);
    free(scr); plan_free(&p);
}

/* ------------------------------------------------------------- KE (C5) */
/* cgpe1d.f90:826-842, cgpe2d.f90:812-829, cgpe3d.f90:875-899 (3D adds the
 * per-component -2 L GAMMAZ KZ term, L = -SPIN..SPIN -> component L+SPIN+1). */
void orc_ke(orc_t *h) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz, S = h->p.spin;
    const cd cdt = h->cdt;
    for (int m = 0; m < h->ms; ++m) {
        const int L = m - S;
        cd *a = h->phi + (size_t)m * h->npts;
#pragma omp parallel for collapse(2)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    double e = h->kx[i] * h->kx[i];
                    if (h->p.dim >= 2) e = h->kx[i] * h->kx[i] + h->ky[j] * h->ky[j];
                    if (h->p.dim >= 3) e = h->kx[i] * h->kx[i] + h->ky[j] * h->ky[j] + h->kz[k] * h->kz[k]
                                           - 2.0 * L * h->p.gz * h->kz[k];
                    a[IDX(h, i, j, k)] *= cexp(-I * cdt * e);
                }
    }
}

/* ------------------------------------------------------------ SOC (C6) */
/* Spin-orbit eigenbasis A.
 * 1D: constant real A, cgpe1d.f90:627-675, phase 2*J*GAMMAX*KX for J=-S..S.
 * 2D/3D: A(beta), cgpe2d.f90:1578-1588 (spin-1), 1610-1638 (spin-2) and
 * cgpe3d.f90:930-991; phase L*ALPHA with ALPHA = 2 sqrt(gx^2 kx^2 + gy^2 ky^2),
 * BETA = atan2(gy ky, gx kx) (0 when ALPHA <= EPS). */
static void soc_matrix(int spin, double beta, cd A[5][5]) {
    /* A[row][col], rows/cols 0-based */
    cd e1 = cexp(-I * beta), e2 = cexp(-2.0 * I * beta);
    if (spin == 1) {
        A[0][0] = 0.5 * e2;            A[1][0] = -sqrt(0.5) * e1; A[2][0] = 0.5;
        A[0][1] = -sqrt(0.5) * e2;     A[1][1] = 0.0;             A[2][1] = sqrt(0.5);
        A[0][2] = A[0][0];             A[1][2] = -A[1][0];        A[2][2] = A[2][0];
    } else {
        A[0][0] = 0.25 * e2;  A[1][0] = -0.5 * e1; A[2][0] = sqrt(0.375);
        A[3][0] = conj(A[1][0]); A[4][0] = conj(A[0][0]);
        A[0][1] = -0.5 * e2;  A[1][1] = 0.5 * e1;  A[2][1] = 0.0;
        A[3][1] = -conj(A[1][1]); A[4][1] = -conj(A[0][1]);
        A[0][2] = sqrt(0.375) * e2; A[1][2] = A[2][1]; A[2][2] = -0.5;
        A[3][2] = A[2][1]; A[4][2] = conj(A[0][2]);
        A[0][3] = -0.5 * e2;  A[1][3] = -0.5 * e1; A[2][3] = A[2][1];
        A[3][3] = -conj(A[1][3]); A[4][3] = -conj(A[0][3]);
        A[0][4] = 0.25 * e2;  A[1][4] = 0.5 * e1;  A[2][4] = sqrt(0.375);
        A[3][4] = conj(A[1][4]); A[4][4] = conj(A[0][4]);
    }
}

static void soc_matrix_1d(int spin, cd A[5][5]) {
    /* cgpe1d.f90:627-675: real matrices */
    if (spin == 1) {
        A[0][0] = 0.5; A[1][0] = -sqrt(0.5); A[2][0] = A[0][0];
        A[0][1] = A[1][0]; A[1][1] = 0.0; A[2][1] = -A[1][0];
        A[0][2] = A[0][0]; A[1][2] = -A[1][0]; A[2][2] = A[0][0];
    } else {
        A[0][0] = 0.25; A[1][0] = -0.5; A[2][0] = sqrt(0.375); A[3][0] = A[1][0]; A[4][0] = A[0][0];
        A[0][1] = A[1][0]; A[1][1] = -A[1][0]; A[2][1] = 0.0; A[3][1] = A[1][0]; A[4][1] = -A[1][0];
        A[0][2] = A[2][0]; A[1][2] = A[2][1]; A[2][2] = A[1][0]; A[3][2] = A[2][1]; A[4][2] = A[2][0];
        A[0][3] = A[1][0]; A[1][3] = A[1][0]; A[2][3] = A[2][1]; A[3][3] = -A[1][0]; A[4][3] = -A[1][0];
        A[0][4] = A[0][0]; A[1][4] = -A[1][0]; A[2][4] = A[2][0]; A[3][4] = -A[1][0]; A[4][4] = A[0][0];
    }
}

void orc_soc(orc_t *h) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz, S = h->p.spin, ms = h->ms;
    const cd cdt = h->cdt;
    const long np = h->npts;
    cd *phi = h->phi;
    cd A1d[5][5];
    if (h->p.dim == 1) soc_matrix_1d(S, A1d);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                cd A[5][5], v[5], u[5];
                double ph[5];
                if (h->p.dim == 1) {
                    memcpy(A, A1d, sizeof(A));
                    for (int L = -S; L <= S; ++L) ph[L + S] = 2.0 * L * h->p.gx * h->kx[i];
                } else {
                    double alpha = 2.0 * sqrt(h->p.gx * h->p.gx * h->kx[i] * h->kx[i]
                                            + h->p.gy * h->p.gy * h->ky[j] * h->ky[j]);
                    double beta = alpha <= EPS ? 0.0 : atan2(h->p.gy * h->ky[j], h->p.gx * h->kx[i]);
                    soc_matrix(S, beta, A);
                    for (int L = -S; L <= S; ++L) ph[L + S] = L * alpha;
                }
                const long p0 = IDX(h, i, j, k);
                for (int m = 0; m < ms; ++m) v[m] = phi[p0 + m * np];
                /* u = A^H v (1D: A^T v with real A) */
                for (int r = 0; r < ms; ++r) {
                    cd s = 0;
                    for (int c = 0; c < ms; ++c) s += conj(A[c][r]) * v[c];
                    u[r] = s * cexp(-I * cdt * ph[r]);
                }
                for (int r = 0; r < ms; ++r) {
                    cd s = 0;
                    for (int c = 0; c < ms; ++c) s += A[r][c] * u[c];
                    phi[p0 + r * np] = s;
                }
            }
}

/* -------------------------------------------------- FXYZ / MAT_C (C9) */
/* FXYZ: cgpe1d.f90:901-922 with SX, SY, SZ of cgpe1d.f90:639-687.
 * Spin-1: SY(1,2) = +i/sqrt2 (as built by the RESHAPE at cgpe1d.f90:642).
 * Spin-2: SY(m,m+1) = -i c_m, c = (1, sqrt1.5, sqrt1.5, 1) (cgpe1d.f90:682). */
static void fxyz_point(int spin, const cd *v, double *fx, double *fy, double *fz) {
    if (spin == 1) {
        const double r = sqrt(0.5);
        /* SX = sqrt(.5)*[[0,1,0],[1,0,1],[0,1,0]] */
        cd sx1 = r * v[1], sx2 = r * (v[0] + v[2]), sx3 = r * v[1];
        *fx = creal(conj(v[0]) * sx1 + conj(v[1]) * sx2 + conj(v[2]) * sx3);
        /* SY = (i/sqrt2) * columns (0,-1,0),(1,0,-1),(0,1,0) */
        cd c = I / sqrt(2.0);
        cd sy1 = c * v[1], sy2 = c * (-v[0] + v[2]), sy3 = c * (-v[1]);
        *fy = creal(conj(v[0]) * sy1 + conj(v[1]) * sy2 + conj(v[2]) * sy3);
        *fz = cabs(v[0]) * cabs(v[0]) - cabs(v[2]) * cabs(v[2]);
    } else {
        const double s = sqrt(1.5);
        cd sx[5], sy[5];
        sx[0] = v[1]; sx[1] = v[0] + s * v[2]; sx[2] = s * v[1] + s * v[3];
        sx[3] = s * v[2] + v[4]; sx[4] = v[3];
        sy[0] = -I * v[1]; sy[1] = I * v[0] - I * s * v[2]; sy[2] = I * s * v[1] - I * s * v[3];
        sy[3] = I * s * v[2] - I * v[4]; sy[4] = I * v[3];
        cd ax = 0, ay = 0;
        for (int m = 0; m < 5; ++m) { ax += conj(v[m]) * sx[m]; ay += conj(v[m]) * sy[m]; }
        *fx = creal(ax); *fy = creal(ay);
        double a[5];
        for (int m = 0; m < 5; ++m) a[m] = cabs(v[m]) * cabs(v[m]);
        *fz = 2.0 * a[0] + a[1] + 0.0 * a[2] - a[3] - 2.0 * a[4];
    }
}

/* MAT_C: cgpe1d.f90:928-952.  c[0..5] = C12, C13, C23, C34, C35, C45. */
static void matc_point(const double *tau, const cd *v, cd fminus, cd *c) {
    c[0] = tau[1] * fminus - 0.4 * tau[2] * v[3] * conj(v[4]);
    c[1] = 0.2 * tau[2] * v[2] * conj(v[4]);
    c[2] = sqrt(1.5) * tau[1] * fminus - 0.2 * tau[2] * v[2] * conj(v[3]);
    c[3] = sqrt(1.5) * tau[1] * fminus - 0.2 * tau[2] * v[1] * conj(v[2]);
    c[4] = 0.2 * tau[2] * v[0] * conj(v[2]);
    c[5] = tau[1] * fminus - 0.4 * tau[2] * v[0] * conj(v[1]);
}

static void couplings(const double *tau, const cd *v, cd *c) {
    double fx, fy, fz;
    fxyz_point(2, v, &fx, &fy, &fz);
    matc_point(tau, v, fx - I * fy, c);
}

/* ------------------------------------------------- 5x5 Hermitian eigen */
/* Cyclic complex Jacobi (stands in for LAPACK ZHEEV).  a is overwritten;
 * on return w holds eigenvalues and v the eigenvectors in columns. */
static void jacobi_herm(int n, cd a[5][5], double *w, cd v[5][5]) {
    for (int r = 0; r < n; ++r) for (int c = 0; c < n; ++c) v[r][c] = (r == c);
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0, dia = 0;
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                double m2 = creal(a[r][c]) * creal(a[r][c]) + cimag(a[r][c]) * cimag(a[r][c]);
                if (r != c) off += m2; else dia += m2;
            }
        if (off == 0.0 || off <= 1e-34 * (dia + off)) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double mag = cabs(a[p][q]);
                if (mag == 0.0) continue;
                cd ph = a[p][q] / mag;                    /* e^{i phi} */
                double app = creal(a[p][p]), aqq = creal(a[q][q]);
                double theta = (aqq - app) / (2.0 * mag);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                /* J = D R with D = diag(1, conj(ph)) on (p,q), R = [[c,s],[-s,c]] */
                cd jpp = cs, jpq = sn, jqp = -sn * conj(ph), jqq = cs * conj(ph);
                for (int k = 0; k < n; ++k) {            /* columns: A <- A J */
                    cd akp = a[k][p], akq = a[k][q];
                    a[k][p] = akp * jpp + akq * jqp;
                    a[k][q] = akp * jpq + akq * jqq;
                    cd vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = vkp * jpp + vkq * jqp;
                    v[k][q] = vkp * jpq + vkq * jqq;
                }
                for (int k = 0; k < n; ++k) {            /* rows: A <- J^H A */
                    cd apk = a[p][k], aqk = a[q][k];
                    a[p][k] = conj(jpp) * apk + conj(jqp) * aqk;
                    a[q][k] = conj(jpq) * apk + conj(jqq) * aqk;
                }
                a[p][q] = 0; a[q][p] = 0;
                a[p][p] = creal(a[p][p]); a[q][q] = creal(a[q][q]);
            }
    }
    for (int r = 0; r < n; ++r) w[r] = creal(a[r][r]);
}

/* Exposed for the cross-check against scipy's zheev: exp(-i cdt H) v for the
 * zero-diagonal Hermitian 5x5 built from c[6] (upper entries). */
void orc_expm_se2(const double *c_reim, double cdt_re, double cdt_im, double *v_reim) {
    const cd *c = (const cd *)c_reim;
    cd *v = (cd *)v_reim;
    cd cdt = cdt_re + I * cdt_im;
    cd a[5][5] = {{0}}, vec[5][5];
    double w[5];
    a[0][1] = c[0]; a[0][2] = c[1]; a[1][2] = c[2]; a[2][3] = c[3]; a[2][4] = c[4]; a[3][4] = c[5];
    a[1][0] = conj(c[0]); a[2][0] = conj(c[1]); a[2][1] = conj(c[2]);
    a[3][2] = conj(c[3]); a[4][2] = conj(c[4]); a[4][3] = conj(c[5]);
    jacobi_herm(5, a, w, vec);
    cd u[5];
    for (int r = 0; r < 5; ++r) {
        cd s = 0;
        for (int k = 0; k < 5; ++k) s += conj(vec[k][r]) * v[k];
        u[r] = cexp(-I * cdt * w[r]) * s;
    }
    for (int r = 0; r < 5; ++r) {
        cd s = 0;
        for (int k = 0; k < 5; ++k) s += vec[r][k] * u[k];
        v[r] = s;
    }
}

/* -------------------------------------------------------------- SE (C7) */
/* Spin-1: cgpe1d.f90:1407-1435 (.GE. EPS), cgpe2d.f90:1449-1479 and
 * cgpe3d.f90:1637-1672 (.GT. EPS).
 * Spin-2: cgpe1d.f90:1436-1497 (predictor with CDT/2), cgpe2d.f90:1480-1547
 * and cgpe3d.f90:1673-1741 (predictor with CDT). */
void orc_se(orc_t *h) {
    const long np = h->npts;
    const cd cdt = h->cdt;
    cd *phi = h->phi;
    const double *tau = h->p.tau;
    if (h->p.spin == 1) {
        const int ge = (h->p.dim == 1);
#pragma omp parallel for
        for (long t = 0; t < np; ++t) {
            cd p1 = phi[t], p2 = phi[t + np], p3 = phi[t + 2 * np];
            cd A1 = tau[1] * p2 * conj(p3);
            cd B1 = tau[1] * p2 * conj(p1);
            cd om = cdt * sqrt(cabs(A1) * cabs(A1) + cabs(B1) * cabs(B1));
            cd del, kap;
            int big = ge ? (cabs(om) >= EPS) : (cabs(om) > EPS);
            if (big) { del = (ccos(om) - 1.0) / (om * om); kap = -I * csin(om) / om; }
            else { del = -0.5; kap = -I; }
            cd t1 = (del * cdt * cdt) * (A1 * conj(A1) * p1 + A1 * conj(B1) * p3) + kap * cdt * A1 * p2;
            cd t2 = (del * cdt * cdt) * (A1 * conj(A1) + B1 * conj(B1)) * p2 + kap * cdt * (conj(A1) * p1 + conj(B1) * p3);
            cd t3 = (del * cdt * cdt) * (conj(A1) * B1 * p1 + B1 * conj(B1) * p3) + kap * cdt * B1 * p2;
            phi[t] = p1 + t1; phi[t + np] = p2 + t2; phi[t + 2 * np] = p3 + t3;
        }
    } else {
        const cd cdp = (h->p.dim == 1) ? cdt / 2.0 : cdt;
#pragma omp parallel for
        for (long t = 0; t < np; ++t) {
            cd v[5], v1[5], c[6], c1[6];
            for (int m = 0; m < 5; ++m) v[m] = phi[t + m * np];
            couplings(tau, v, c);
            v1[0] = v[0] - (I * cdp) * (c[0] * v[1] + c[1] * v[2]);
            v1[1] = v[1] - (I * cdp) * (conj(c[0]) * v[0] + c[2] * v[2]);
            v1[2] = v[2] - (I * cdp) * (conj(c[1]) * v[0] + conj(c[2]) * v[1] + c[3] * v[3] + c[4] * v[4]);
            v1[3] = v[3] - (I * cdp) * (conj(c[3]) * v[2] + c[5] * v[4]);
            v1[4] = v[4] - (I * cdp) * (conj(c[4]) * v[2] + conj(c[5]) * v[3]);
            couplings(tau, v1, c1);
            for (int q = 0; q < 6; ++q) c[q] = (c[q] + c1[q]) / 2.0;
            orc_expm_se2((const double *)c, creal(cdt), cimag(cdt), (double *)v);
            for (int m = 0; m < 5; ++m) phi[t + m * np] = v[m];
        }
    }
}

/* -------------------------------------------------------------- SP (C8) */
/* cgpe1d.f90:847-896, cgpe2d.f90:834-886, cgpe3d.f90:1009-1065 */
void orc_sp(orc_t *h) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    const long np = h->npts;
    const cd cdt = h->cdt;
    const double *tau = h->p.tau;
    cd *phi = h->phi;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const long t = IDX(h, i, j, k);
                const double v = V_at(h, i, j, k);
                double a[5], T[5], rho = 0;
                for (int m = 0; m < h->ms; ++m) { a[m] = cabs(phi[t + m * np]); a[m] *= a[m]; rho += a[m]; }
                if (h->p.spin == 1) {
                    T[0] = v + tau[0] * rho + tau[1] * (a[0] + a[1] - a[2]);
                    T[1] = v + tau[0] * rho + tau[1] * (a[0] + a[2]);
                    T[2] = v + tau[0] * rho + tau[1] * (a[2] + a[1] - a[0]);
                } else {
                    double fz = 2.0 * a[0] + a[1] - a[3] - 2.0 * a[4];
                    T[0] = v + tau[0] * rho + 2.0 * tau[1] * fz + 0.4 * tau[2] * a[4];
                    T[1] = v + tau[0] * rho + tau[1] * fz + 0.4 * tau[2] * a[3];
                    T[2] = v + tau[0] * rho + 0.2 * tau[2] * a[2];
                    T[3] = v + tau[0] * rho - tau[1] * fz + 0.4 * tau[2] * a[1];
                    T[4] = v + tau[0] * rho - 2.0 * tau[1] * fz + 0.4 * tau[2] * a[0];
                }
                for (int m = 0; m < h->ms; ++m) phi[t + m * np] *= cexp(-I * cdt * T[m]);
            }
}

/* ------------------------------------------------- SIMPSON / DIFF (C12-13) */
/* simpson.f90:4-21, literally. */
double orc_simpson(const double *f, int n, double dx) {
    double f1 = f[1] + f[n - 5], f2 = f[2];
    for (int i = 4; i <= n - 6; i += 2) { f1 += f[i - 1]; f2 += f[i]; }
    return dx * (f[0] + 4.0 * f1 + 2.0 * f2 + f[n - 4]) / 3.0
         + 3.0 * dx * (f[n - 4] + 3.0 * (f[n - 3] + f[n - 2]) + f[n - 1]) / 8.0;
}

/* diff.f90:4-33, literally (1-based indices shifted to 0-based). */
void orc_diff(const double *p, int n, double dx, double *d) {
#define P(i) p[(i) - 1]
    d[0] = (P(n - 1) - 8.0 * P(n) + 8.0 * P(2) - P(3)) / (12.0 * dx);
    d[1] = (P(n) - 8.0 * P(1) + 8.0 * P(3) - P(4)) / (12.0 * dx);
    for (int i = 3; i <= 4; ++i) d[i - 1] = (P(i - 2) - 8.0 * P(i - 1) + 8.0 * P(i + 1) - P(i + 2)) / (12.0 * dx);
    for (int i = n - 3; i <= n - 2; ++i) d[i - 1] = (P(i - 2) - 8.0 * P(i - 1) + 8.0 * P(i + 1) - P(i + 2)) / (12.0 * dx);
    for (int i = 5; i <= n - 4; ++i)
        d[i - 1] = (3.0 * P(i - 4) - 32.0 * P(i - 3) + 168.0 * P(i - 2) - 672.0 * P(i - 1)
                    + 672.0 * P(i + 1) - 168.0 * P(i + 2) + 32.0 * P(i + 3) - 3.0 * P(i + 4)) / (840.0 * dx);
    d[n - 2] = (P(n - 3) - 8.0 * P(n - 2) + 8.0 * P(n) - P(1)) / (12.0 * dx);
    d[n - 1] = (P(n - 2) - 8.0 * P(n - 1) + 8.0 * P(1) - P(2)) / (12.0 * dx);
#undef P
}

/* Nested Simpson over a field f(NX,NY,NZ): x first, then y, then z
 * (cgpe2d.f90:972-985, cgpe3d.f90:1156-1172). */
static double nested_simpson(const orc_t *h, const double *f) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    if (h->p.dim == 1) return orc_simpson(f, nx, h->p.dx);
    double *tz = malloc(sizeof(double) * nz);
#pragma omp parallel for
    for (int k = 0; k < nz; ++k) {
        double *ty = malloc(sizeof(double) * ny);
        for (int j = 0; j < ny; ++j) ty[j] = orc_simpson(f + (size_t)nx * (j + (size_t)ny * k), nx, h->p.dx);
        tz[k] = orc_simpson(ty, ny, h->p.dy);
        free(ty);
    }
    double r = h->p.dim == 2 ? tz[0] : orc_simpson(tz, nz, h->p.dz);
    free(tz);
    return r;
}

/* ---------------------------------------------------------- NORMC (C10) */
/* cgpe1d.f90:957-993, cgpe2d.f90:947-986, cgpe3d.f90:1129-1173 */
void orc_normc(const orc_t *h, double *norm) {
    double *f = malloc(sizeof(double) * h->npts);
    for (int m = 0; m < h->ms; ++m) {
        const cd *a = h->phi + (size_t)m * h->npts;
#pragma omp parallel for
        for (long t = 0; t < h->npts; ++t) { double v = cabs(a[t]); f[t] = v * v; }
        norm[m] = nested_simpson(h, f);
    }
    free(f);
}

/* NORMT: cgpe1d.f90:998-1031 etc.  Returns TNORM and divides PHI by it. */
double orc_normt(orc_t *h) {
    double *f = malloc(sizeof(double) * h->npts);
    const long np = h->npts;
#pragma omp parallel for
    for (long t = 0; t < np; ++t) {
        double s = 0;
        for (int m = 0; m < h->ms; ++m) { double v = cabs(h->phi[t + m * np]); s += v * v; }
        f[t] = s;
    }
    double tn = sqrt(nested_simpson(h, f));
    free(f);
    const long tot = np * h->ms;
#pragma omp parallel for
    for (long t = 0; t < tot; ++t) h->phi[t] = h->phi[t] / tn;
    return tn;
}

/* ------------------------------------------------------------ RAD (C11) */
/* cgpe1d.f90:1036-1072 (X2), cgpe2d.f90:1032-1071 (X2+Y2),
 * cgpe3d.f90:1224-1268 (R2).  Not divided by the component norm. */
void orc_rad(const orc_t *h, double *rms) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    double *f = malloc(sizeof(double) * h->npts);
    for (int m = 0; m < h->ms; ++m) {
        const cd *a = h->phi + (size_t)m * h->npts;
#pragma omp parallel for collapse(2)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    double r2 = h->x[i] * h->x[i];
                    if (h->p.dim >= 2) r2 += h->y[j] * h->y[j];
                    if (h->p.dim >= 3) r2 += h->z[k] * h->z[k];
                    long t = IDX(h, i, j, k);
                    f[t] = r2 * cabs(a[t]) * cabs(a[t]);
                }
        rms[m] = sqrt(nested_simpson(h, f));
    }
    free(f);
}

/* --------------------------------------------------------- ENERGY (C11) */
/* Derivatives of every component along every axis with DIFF applied to the
 * real and imaginary parts separately (cgpe1d.f90:1144-1148,
 * cgpe2d.f90:1143-1166, cgpe3d.f90:1342-1379). */
static void grad_axis(const orc_t *h, const cd *a, int axis, cd *out) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    const int n = axis == 0 ? nx : axis == 1 ? ny : nz;
    const double d = axis == 0 ? h->p.dx : axis == 1 ? h->p.dy : h->p.dz;
    const long nlines = h->npts / n;
#pragma omp parallel
    {
        double *re = malloc(sizeof(double) * n), *im = malloc(sizeof(double) * n);
        double *dre = malloc(sizeof(double) * n), *dim_ = malloc(sizeof(double) * n);
#pragma omp for
        for (long L = 0; L < nlines; ++L) {
            long base, stride;
            if (axis == 0) { base = L * nx; stride = 1; }
            else if (axis == 1) { long i = L % nx, k = L / nx; base = i + (long)nx * ny * k; stride = nx; }
            else { base = L; stride = (long)nx * ny; }
            for (int t = 0; t < n; ++t) { re[t] = creal(a[base + t * stride]); im[t] = cimag(a[base + t * stride]); }
            orc_diff(re, n, d, dre); orc_diff(im, n, d, dim_);
            for (int t = 0; t < n; ++t) out[base + t * stride] = dre[t] + I * dim_[t];
        }
        free(re); free(im); free(dre); free(dim_);
    }
}

/* Energy / chemical potential / magnetisation densities, literally per case:
 *  1D spin-1 cgpe1d.f90:1153-1181, 1D spin-2 cgpe1d.f90:1185-1232,
 *  2D spin-1 cgpe2d.f90:1170-1203, 2D spin-2 cgpe2d.f90:1212-1268,
 *  3D spin-1 cgpe3d.f90:1383-1420, 3D spin-2 cgpe3d.f90:1434-1493.
 * out[0] = energy density, out[1] = mz density, out[2+m] = mu_m density. */
static void energy_point(const orc_t *h, double V, const cd *P, const cd *X, const cd *Y, const cd *Z, double *out) {
    const double *tau = h->p.tau;
    const double gx = h->p.gx, gy = h->p.gy, gz = h->p.gz;
    const int S = h->p.spin, dim = h->p.dim, ms = h->ms;
    double a[5], rho = 0, dp2[5];
    for (int m = 0; m < ms; ++m) {
        a[m] = cabs(P[m]) * cabs(P[m]); rho += a[m];
        dp2[m] = cabs(X[m]) * cabs(X[m]);
        if (dim >= 2) dp2[m] += cabs(Y[m]) * cabs(Y[m]);
        if (dim >= 3) dp2[m] += cabs(Z[m]) * cabs(Z[m]);
    }
    double fx, fy, fz;
    fxyz_point(S, P, &fx, &fy, &fz);
#define CJ(q) conj(P[q])
    if (S == 1) {
        cd so_e, so1, so2, so3;
        if (dim == 1) {
            so_e = sqrt(2.0) * gx * (-I * CJ(0) * X[1] - I * CJ(2) * X[1] - I * CJ(1) * (X[0] + X[2]));
            so1 = sqrt(2.0) * gx * (-I * CJ(0) * X[1]);
            so2 = sqrt(2.0) * gx * (-I * CJ(1) * (X[0] + X[2]));
            so3 = sqrt(2.0) * gx * (-I * CJ(2) * X[1]);
        } else {
            so_e = sqrt(2.0) * (CJ(0) * (-I * gx * X[1] - gy * Y[1]) + CJ(1) * (-I * gx * X[2] - gy * Y[2])
                              + CJ(1) * (-I * gx * X[0] + gy * Y[0]) + CJ(2) * (-I * gx * X[1] + gy * Y[1]));
            so1 = sqrt(2.0) * (CJ(0) * (-I * gx * X[1] - gy * Y[1]));
            so2 = sqrt(2.0) * (CJ(1) * (-I * gx * X[2] - gy * Y[2]) + CJ(1) * (-I * gx * X[0] + gy * Y[0]));
            so3 = sqrt(2.0) * (CJ(2) * (-I * gx * X[1] + gy * Y[1]));
            if (dim == 3) {
                /* cgpe3d.f90:1391-1396: 2*sqrt(.5) prefactor on the xy part
                 * (equal to sqrt2) plus the gamma_z terms; 1404-1419 */
                so_e = 2.0 * sqrt(0.5) * (CJ(0) * (-I * gx * X[1] - gy * Y[1]) + CJ(1) * (-I * gx * X[2] - gy * Y[2])
                              + CJ(1) * (-I * gx * X[0] + gy * Y[0]) + CJ(2) * (-I * gx * X[1] + gy * Y[1]))
                     + 2.0 * (CJ(0) * (-I * gz * Z[0]) + CJ(2) * (I * gz * Z[2]));
                so1 = sqrt(2.0) * (CJ(0) * (-I * gx * X[1] - gy * Y[1] - I * sqrt(2.0) * gz * Z[0]));
                so3 = sqrt(2.0) * (CJ(2) * (-I * gx * X[1] + gy * Y[1] + I * gz * sqrt(2.0) * Z[2]));
            }
        }
        out[0] = creal(V * rho + tau[0] * rho * rho / 2.0 + tau[1] * (fx * fx + fy * fy + fz * fz) / 2.0
                       + dp2[0] + dp2[1] + dp2[2] + so_e);
        out[1] = a[0] - a[2];
        out[2] = creal(V * a[0] + dp2[0] + tau[0] * (a[0] + a[1] + a[2]) * a[0]
                       + tau[1] * (a[0] + a[1] - a[2]) * a[0] + tau[1] * CJ(2) * P[1] * P[1] * CJ(0) + so1);
        out[3] = creal(V * a[1] + dp2[1] + tau[0] * (a[0] + a[1] + a[2]) * a[1]
                       + tau[1] * (a[0] + a[2]) * a[1] + 2.0 * tau[1] * P[0] * P[2] * CJ(1) * CJ(1) + so2);
        out[4] = creal(V * a[2] + dp2[2] + tau[0] * (a[0] + a[1] + a[2]) * a[2]
                       + tau[1] * (a[1] + a[2] - a[0]) * a[2] + tau[1] * CJ(0) * P[1] * P[1] * CJ(2) + so3);
    } else {
        cd c[6];
        matc_point(tau, P, fx - I * fy, c);
        cd th = (2.0 * P[0] * P[4] - 2.0 * P[1] * P[3] + P[2] * P[2]) / sqrt(5.0);
        cd so_e, so[5];
        const double s6 = sqrt(6.0), s15 = sqrt(1.5);
        if (dim == 1) {
            so_e = gx * (-I * 2.0 * (CJ(0) * X[1]) - I * 2.0 * (CJ(1) * X[0])
                         - I * s6 * (CJ(1) * X[2] + CJ(2) * X[1] + CJ(2) * X[3] + CJ(3) * X[2])
                         - I * 2.0 * (CJ(3) * X[4] + CJ(4) * X[3]));
            so[0] = -I * 2.0 * gx * (CJ(0) * X[1]);
            so[1] = gx * (-I * 2.0 * (CJ(1) * X[0]) - I * s6 * CJ(1) * X[2]);
            so[2] = -I * gx * s6 * (CJ(2) * X[1] + CJ(2) * X[3]);
            so[3] = gx * (-I * s6 * CJ(3) * X[2] - I * 2.0 * CJ(3) * X[4]);
            so[4] = -I * 2.0 * gx * CJ(4) * X[3];
        } else if (dim == 2) {
            so_e = -I * 2.0 * (CJ(0) * gx * X[1] - I * CJ(0) * gy * Y[1]
                   + CJ(1) * gx * X[0] + I * CJ(1) * gy * Y[0]
                   + sqrt(3.0 / 2.0) * (CJ(1) * gx * X[2] - I * CJ(1) * gy * Y[2]
                        + CJ(2) * gx * X[1] + I * CJ(2) * gy * Y[1] + CJ(2) * gx * X[3]
                        - I * CJ(2) * gy * Y[3] + CJ(3) * gx * X[2] + I * CJ(3) * gy * Y[2])
                   + CJ(3) * gx * X[4] - I * CJ(3) * gy * Y[4] + CJ(4) * gx * X[3] + I * CJ(4) * gy * Y[3]);
            so[0] = -I * 2.0 * (CJ(0) * gx * X[1] - I * CJ(0) * gy * Y[1]);
            so[1] = -I * 2.0 * (CJ(1) * gx * X[0] + I * CJ(1) * gy * Y[0]
                                + s15 * (CJ(1) * gx * X[2] - I * CJ(1) * gy * Y[2]));
            so[2] = -I * 2.0 * (s15 * (CJ(2) * gx * X[1] + I * CJ(2) * gy * Y[1]
                                       + CJ(2) * gx * X[3] - I * CJ(2) * gy * Y[3]));
            so[3] = -I * 2.0 * (CJ(3) * gx * X[4] - I * CJ(3) * gy * Y[4]
                                + s15 * (CJ(3) * gx * X[2] + I * CJ(3) * gy * Y[2]));
            so[4] = -I * 2.0 * (CJ(4) * gx * X[3] + I * CJ(4) * gy * Y[3]);
        } else {
            so_e = -I * CJ(0) * (2.0 * gx * X[1] - I * 2.0 * gy * Y[1] + 4.0 * gz * Z[0])
                 - I * CJ(1) * (gx * (2.0 * X[0] + s6 * X[2]) + I * gy * (2.0 * Y[0] - s6 * Y[2]) + 2.0 * gz * Z[1])
                 - I * CJ(2) * (gx * s6 * (X[1] + X[3]) + I * gy * s6 * (Y[1] - Y[3]))
                 - I * CJ(3) * (gx * (s6 * X[2] + 2.0 * X[4]) + I * gy * (s6 * Y[2] - 2.0 * Y[4]) - 2.0 * gz * Z[3])
                 - I * CJ(4) * (2.0 * gx * X[3] + I * 2.0 * gy * Y[3] - 4.0 * gz * Z[4]);
            so[0] = -I * 2.0 * (CJ(0) * gx * X[1] - I * CJ(0) * gy * Y[1] + 2.0 * CJ(0) * gz * Z[0]);
            so[1] = -I * 2.0 * (CJ(1) * gx * X[0] + I * CJ(1) * gy * Y[0]
                                + s15 * (CJ(1) * gx * X[2] - I * CJ(1) * gy * Y[2]) + CJ(1) * gz * Z[1]);
            so[2] = -I * 2.0 * (s15 * (CJ(2) * gx * X[1] + I * CJ(2) * gy * Y[1]
                                       + CJ(2) * gx * X[3] - I * CJ(2) * gy * Y[3]));
            so[3] = -I * 2.0 * (CJ(3) * gx * X[4] - I * CJ(3) * gy * Y[4]
                                + s15 * (CJ(3) * gx * X[2] + I * CJ(3) * gy * Y[2]) - CJ(3) * gz * Z[3]);
            so[4] = -I * 2.0 * (CJ(4) * gx * X[3] + I * CJ(4) * gy * Y[3] - 2.0 * CJ(4) * gz * Z[4]);
        }
        out[0] = creal(V * rho + tau[0] * rho * rho / 2.0 + tau[1] * (fx * fx + fy * fy + fz * fz) / 2.0
                       + tau[2] * (th * conj(th)) / 2.0 + dp2[0] + dp2[1] + dp2[2] + dp2[3] + dp2[4] + so_e);
        out[1] = 2.0 * a[0] + a[1] - a[3] - 2.0 * a[4];
        out[2] = creal((V + tau[0] * rho + 2.0 * tau[1] * fz + 0.4 * tau[2] * a[4]) * a[0]
                       + (c[0] * P[1] + c[1] * P[2]) * CJ(0) + so[0] + dp2[0]);
        out[3] = creal((V + tau[0] * rho + tau[1] * fz + 0.4 * tau[2] * a[3]) * a[1]
                       + (conj(c[0]) * P[0] + c[2] * P[2]) * CJ(1) + so[1] + dp2[1]);
        out[4] = creal((V + tau[0] * rho + 0.2 * tau[2] * a[2]) * a[2]
                       + (conj(c[1]) * P[0] + conj(c[2]) * P[1] + c[3] * P[3] + c[4] * P[4]) * CJ(2) + so[2] + dp2[2]);
        out[5] = creal((V + tau[0] * rho - tau[1] * fz + 0.4 * tau[2] * a[1]) * a[3]
                       + (conj(c[3]) * P[2] + c[5] * P[4]) * CJ(3) + so[3] + dp2[3]);
        out[6] = creal((V + tau[0] * rho - 2.0 * tau[1] * fz + 0.4 * tau[2] * a[0]) * a[4]
                       + (conj(c[4]) * P[2] + conj(c[5]) * P[3]) * CJ(4) + so[4] + dp2[4]);
    }
#undef CJ
}

/* ENERGY: EN = int(e)/sum(NORM), MZ = int(mz), MU_m = int(mu_m)/(NORM_m+EPS)
 * (cgpe1d.f90:1235-1239, cgpe2d.f90:1276-1280, cgpe3d.f90:1506-1510). */
void orc_energy(const orc_t *h, double *mu, double *en, double *mz) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz, ms = h->ms, dim = h->p.dim;
    const long np = h->npts;
    double norm[5];
    orc_normc(h, norm);
    cd *gx = malloc(sizeof(cd) * np * ms), *gy = NULL, *gz = NULL;
    for (int m = 0; m < ms; ++m) grad_axis(h, h->phi + m * np, 0, gx + m * np);
    if (dim >= 2) { gy = malloc(sizeof(cd) * np * ms); for (int m = 0; m < ms; ++m) grad_axis(h, h->phi + m * np, 1, gy + m * np); }
    if (dim >= 3) { gz = malloc(sizeof(cd) * np * ms); for (int m = 0; m < ms; ++m) grad_axis(h, h->phi + m * np, 2, gz + m * np); }
    const int nq = ms + 2;
    double *f = malloc(sizeof(double) * np * nq);
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long t = IDX(h, i, j, k);
                cd P[5], X[5], Y[5] = {0}, Z[5] = {0};
                for (int m = 0; m < ms; ++m) {
                    P[m] = h->phi[t + m * np]; X[m] = gx[t + m * np];
                    if (gy) Y[m] = gy[t + m * np];
                    if (gz) Z[m] = gz[t + m * np];
                }
                double out[7];
                energy_point(h, V_at(h, i, j, k), P, X, Y, Z, out);
                for (int q = 0; q < nq; ++q) f[t + q * np] = out[q];
            }
    double sn = 0;
    for (int m = 0; m < ms; ++m) sn += norm[m];
    *en = nested_simpson(h, f) / sn;
    *mz = nested_simpson(h, f + np);
    for (int m = 0; m < ms; ++m) mu[m] = nested_simpson(h, f + (2 + m) * np) / (norm[m] + EPS);
    free(f); free(gx); free(gy); free(gz);
}

void orc_set_mag(orc_t *h, double mag) { h->mag = mag; }
void orc_get_sig(const orc_t *h, double *sig) { sig[0] = h->sig[0]; sig[1] = h->sig[1]; }

/* USRFUN, cgpe1d.f90:1292-1319 */
static void usrfun(const double *x, double *fvec, double fjac[2][2], const double *n, double mag, double dt) {
    double e1 = exp(2.0 * (x[0] + 2.0 * x[1]) * dt), e2 = exp(2.0 * (x[0] + x[1]) * dt), e3 = exp(2.0 * x[0] * dt);
    double e4 = exp(2.0 * (x[0] - x[1]) * dt), e5 = exp(2.0 * (x[0] - 2.0 * x[1]) * dt);
    fvec[0] = e1 * n[0] + e2 * n[1] + e3 * n[2] + e4 * n[3] + e5 * n[4] - 1.0;
    fvec[1] = 2.0 * e1 * n[0] + e2 * n[1] - e4 * n[3] - 2.0 * e5 * n[4] - mag;
    fjac[0][0] = (e1 * n[0] + e2 * n[1] + e3 * n[2] + e4 * n[3] + e5 * n[4]) * 2.0 * dt;
    fjac[0][1] = e1 * n[0] * 4.0 * dt + e2 * n[1] * 2.0 * dt + e4 * n[3] * (-2.0 * dt) + e5 * n[4] * (-4.0 * dt);
    fjac[1][0] = (2.0 * e1 * n[0] + e2 * n[1] - e4 * n[3] - 2.0 * e5 * n[4]) * 2.0 * dt;
    fjac[1][1] = 2.0 * e1 * n[0] * 4.0 * dt + e2 * n[1] * 2.0 * dt - e4 * n[3] * (-2.0 * dt) - 2.0 * e5 * n[4] * (-4.0 * dt);
}

/* NEWTON, cgpe1d.f90:1245-1291 (NTRIAL = 1000, TOL_NR = 1e-6).  Returns 1
 * when the root was not found within tolerance (ERR_MSG). */
static int newton(double *x, const double *n, double mag, double dt) {
    double p[2] = {0, 0}, fvec[2], fjac[2][2];
    for (int k = 0; k < 1000; ++k) {
        usrfun(x, fvec, fjac, n, mag, dt);
        p[1] = (fvec[1] * fjac[0][0] - fvec[0] * fjac[1][0]) / (fjac[1][0] * fjac[0][1] - fjac[0][0] * fjac[1][1]);
        p[0] = (-fvec[0] - fjac[0][1] * p[1]) / fjac[0][0];
        x[0] += p[0]; x[1] += p[1];
        if (fmax(fabs(p[0]), fabs(p[1])) <= 1.0e-6) break;
    }
    return fmax(fabs(p[0]), fabs(p[1])) > 1.0e-6;
}

/* Projection of the imaginary-time no-SOC branch, cgpe1d.f90:444-469
 * (3D spin-1 EPS placement cgpe3d.f90:464-465). */
static int project(orc_t *h, const double *norm) {
    double sg[5];
    const double mag = h->mag;
    if (h->p.spin == 1) {
        double inner = sqrt(4.0 * (1.0 - mag * mag) * norm[0] * norm[2] + mag * mag * norm[1] * norm[1]);
        if (h->p.dim == 3) sg[1] = sqrt(1.0 - mag * mag) / sqrt(norm[1] + inner + EPS);
        else sg[1] = sqrt(1.0 - mag * mag) / (sqrt(norm[1] + inner) + EPS);
        sg[0] = sqrt(1.0 + mag - sg[1] * sg[1] * norm[1]) / (sqrt(2.0 * norm[0]) + EPS);
        sg[2] = sqrt(1.0 - mag - sg[1] * sg[1] * norm[1]) / (sqrt(2.0 * norm[2]) + EPS);
    } else {
        if (newton(h->sig, norm, mag, h->p.dt)) return 1;
        sg[0] = exp((h->sig[0] + 2.0 * h->sig[1]) * h->p.dt);
        sg[1] = exp((h->sig[0] + h->sig[1]) * h->p.dt);
        sg[2] = exp(h->sig[0] * h->p.dt);
        sg[3] = exp((h->sig[0] - h->sig[1]) * h->p.dt);
        sg[4] = exp((h->sig[0] - 2.0 * h->sig[1]) * h->p.dt);
    }
    const long np = h->npts;
    for (int m = 0; m < h->ms; ++m)
        for (long t = 0; t < np; ++t) h->phi[t + m * np] *= sg[m];
    return 0;
}

/* ----------------------------------------------------- one split step */
/* cgpe1d.f90:434-441 then 443-474 (imaginary time with SOC: NORMT only).
 * norm_out receives NORMC before the renormalisation (what file3 reports). */
int orc_step(orc_t *h, int nsteps, double *norm_out) {
    double nbuf[5];
    for (int s = 0; s < nsteps; ++s) {
        orc_fft(h); orc_ke(h); orc_soc(h); orc_bft(h); orc_se(h); orc_sp(h);
        double *n = norm_out ? norm_out : nbuf;
        orc_normc(h, n);
        if (h->p.imag) {
            if (!h->switch_soc && project(h, n)) return 1;   /* ERR_MSG -> STOP */
            orc_normt(h);
        }
    }
    return 0;
}

/* max |phi - other| over all points and components (CONV numerator,
 * cgpe1d.f90:482). */
double orc_maxdiff(const orc_t *h, const double *other) {
    const cd *o = (const cd *)other;
    const long tot = h->npts * h->ms;
    double mx = 0;
#pragma omp parallel for reduction(max : mx)
    for (long t = 0; t < tot; ++t) { double d = cabs(h->phi[t] - o[t]); if (d > mx) mx = d; }
    return mx;
}

/* -------------------------------------------------- initial guesses (C3) */
/* INITIALIZE, cgpe1d.f90:707-790, cgpe2d.f90:689-776, cgpe3d.f90:747-837,
 * including the reference's TF-branch typos (cgpe1d.f90:753, cgpe2d.f90:699,
 * cgpe3d.f90:798). */
void orc_initialize(orc_t *h, int option_fpc, double mag) {
    const int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz, S = h->p.spin, dim = h->p.dim;
    const long np = h->npts;
    const double *tau = h->p.tau;
    const double ax = h->p.ax, ay = h->p.ay, az = h->p.az;
    double nrm = dim == 1 ? sqrt(sqrt(PI)) : dim == 2 ? sqrt(PI) : pow(PI, 0.75);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long t = IDX(h, i, j, k);
                double x2 = h->x[i] * h->x[i], y2 = h->y[j] * h->y[j], z2 = h->z[k] * h->z[k];
                double tmp = ax * x2, vv = ax * ax * x2;
                if (dim >= 2) { tmp += ay * y2; vv += ay * ay * y2; }
                if (dim >= 3) { tmp += az * z2; vv += az * az * z2; }
                double g = exp(-tmp / 2.0) / nrm;
                double v[5] = {0, 0, 0, 0, 0};
                if (S == 1) {
                    if (option_fpc == 1) {
                        double base, ex1, ex2, thr_pow, tf;
                        if (dim == 1) { base = 3.0 * (tau[0] + tau[2]) / 4.0; ex1 = 0.67; ex2 = 0.33; thr_pow = 0;
                                        /* cgpe1d.f90:717-723 uses TAU(2), zero for spin-1 */
                                        double r = pow(base, ex1) - vv;
                                        tf = r >= 0 ? r / (tau[0] + tau[2]) : 0.0;
                                        int tfb = pow(base, ex2) >= 10.0;
                                        double f = tfb ? sqrt(tf) : g;
                                        v[0] = ((1.0 + mag) / 2.0) * f; v[1] = sqrt((1.0 - mag * mag) / 2.0) * f; v[2] = ((1.0 - mag) / 2.0) * f;
                                        (void)thr_pow;
                        } else if (dim == 2) {
                            base = 4.0 * (tau[0] + tau[1]) / (2.0 * PI);
                            double r = pow(base, 8.0) - vv;        /* cgpe2d.f90:699 typo kept */
                            tf = r >= 0 ? (pow(base, 0.5) - vv) / (tau[0] + tau[1]) : 0.0;
                            int tfb = pow(base, 0.25) >= 10.0;
                            double f = tfb ? sqrt(tf) : g;
                            v[0] = ((1.0 + mag) / 2.0) * f; v[1] = sqrt((1.0 - mag * mag) / 2.0) * f; v[2] = ((1.0 - mag) / 2.0) * f;
                        } else {
                            base = 15.0 * (tau[0] + tau[1]) / (8.0 * PI);
                            double r = pow(base, 0.4) - vv;
                            tf = r >= 0 ? r / (tau[0] + tau[1]) : 0.0;
                            int tfb = pow(base, 0.2) >= 10.0;
                            double f = tfb ? sqrt(tf) : g;
                            v[0] = ((1.0 + mag) / 2.0) * f; v[1] = sqrt((1.0 - mag * mag) / 2.0) * f; v[2] = ((1.0 - mag) / 2.0) * f;
                        }
                    } else if (option_fpc == 2) {
                        v[0] = sqrt((1.0 + mag) / 2.0) * g; v[1] = 0.0; v[2] = sqrt((1.0 - mag) / 2.0) * g;
                    } else {
                        /* Gaussian; the 3D spin-1 default uses the unweighted
                         * X2+Y2+Z2 (cgpe3d.f90:783-785) */
                        double gg = dim == 3 ? exp(-(x2 + y2 + z2) / 2.0) / pow(PI, 0.75) : g;
                        v[0] = v[1] = v[2] = gg;
                    }
                } else {
                    if (option_fpc == 1) {
                        double f;
                        if (dim == 1) {
                            double base = 3.0 * (tau[0] + 4.0 * tau[1]) / 4.0;
                            double r = pow(base, 0.67) - vv;
                            double tf = r >= 0 ? r / (tau[0] + 4.0 * tau[1]) : 0.0;
                            /* cgpe1d.f90:753 misplaced parenthesis kept */
                            int tfb = (3.0 * pow(tau[0] + 4.0 * tau[1] / 4.0, 0.33)) >= 10.0;
                            f = tfb ? sqrt(tf) : g;
                        } else if (dim == 2) {
                            double base = 4.0 * (tau[0] + 4.0 * tau[1]) / (2.0 * PI);
                            double r = pow(base, 0.5) - vv;
                            double tf = r >= 0 ? r / (tau[0] + 4.0 * tau[1]) : 0.0;
                            int tfb = pow(base, 0.25) >= 10.0;
                            f = tfb ? sqrt(tf) : g;
                        } else {
                            double base = 15.0 * (tau[0] + 4.0 * tau[1]) / (8.0 * PI);
                            double r = pow(base, 0.4) - vv;
                            double tf = r >= 0 ? r / (tau[0] + 4.0 * tau[1]) : 0.0;
                            /* cgpe3d.f90:798 uses the 2D guard, kept */
                            int tfb = pow(4.0 * (tau[0] + 4.0 * tau[1]) / (2.0 * PI), 0.25) >= 10.0;
                            f = tfb ? sqrt(tf) : g;
                        }
                        v[0] = ((2.0 + mag) * (2.0 + mag) / 16.0) * f;
                        v[1] = ((sqrt(4.0 - mag * mag) * (2.0 + mag)) / 8.0) * f;
                        v[2] = ((sqrt(1.5) * (4.0 - mag * mag)) / 8.0) * f;
                        v[3] = ((sqrt(4.0 - mag * mag) * (2.0 - mag)) / 8.0) * f;
                        v[4] = ((2.0 - mag) * (2.0 - mag) / 16.0) * f;
                    } else if (option_fpc == 2) {
                        v[0] = (sqrt(2.0 + mag) / 2.0) * g; v[4] = (sqrt(2.0 - mag) / 2.0) * g;
                    } else if (option_fpc == 3) {
                        v[0] = sqrt((1.0 + mag) / 3.0) * g; v[3] = sqrt((2.0 - mag) / 3.0) * g;
                    } else {
                        double a = dim == 3 ? 1.0 : sqrt(0.2);     /* cgpe3d.f90:827-831 has no sqrt(0.2) */
                        for (int m = 0; m < 5; ++m) v[m] = a * g;
                    }
                }
                for (int m = 0; m < h->ms; ++m) h->phi[t + m * np] = v[m];
            }
}

/* ---------------------------------------------------- TAU and AOSC (C2) */
/* cgpe1d.f90:321-332 (q1D factor sqrt(ALPHAY*ALPHAZ)/(2 pi)),
 * cgpe2d.f90:325-336 (q2D factor sqrt(ALPHAZ/(2 pi))), cgpe3d.f90:334-345. */
void orc_tau(int dim, int spin, int natoms, double mass, double a0, double a2, double a4,
             double nux, double nuy, double nuz, double *tau, double *aosc_out) {
    double alphay = nuy / nux, alphaz = nuz / nux;
    double omegam = 2.0 * PI * nux;
    double aosc = sqrt(HBAR / (mass * AMU * omegam));
    double geo = dim == 1 ? sqrt(alphay * alphaz) / (2.0 * PI) : dim == 2 ? sqrt(alphaz / (2.0 * PI)) : 1.0;
    /* The spin-1 formulas use REAL(NATOMS) (single precision conversion of an
     * integer, exact for realistic atom numbers). */
    double na = (double)(float)natoms;
    tau[2] = 0.0;
    if (spin == 1) {
        tau[0] = 2.0 * geo * (4.0 * PI * na * (a0 * AU + 2.0 * a2 * AU) / (3.0 * aosc));
        tau[1] = 2.0 * geo * (4.0 * PI * na * (a2 * AU - a0 * AU) / (3.0 * aosc));
    } else {
        double nd = (double)natoms;
        tau[0] = 2.0 * (geo * 4.0 * PI * nd * (4.0 * a2 * AU + 3.0 * a4 * AU) / (7.0 * aosc));
        tau[1] = 2.0 * (geo * 4.0 * PI * nd * (a4 * AU - a2 * AU) / (7.0 * aosc));
        tau[2] = 2.0 * (geo * 4.0 * PI * nd * (7.0 * a0 * AU - 10.0 * a2 * AU + 3.0 * a4 * AU) / (7.0 * aosc));
    }
    *aosc_out = aosc;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
