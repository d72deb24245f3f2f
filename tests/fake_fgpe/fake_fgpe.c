/* fake_fgpe.c -- a host-only stand-in for libfgpe.so, used by the CPU test of
 * the drop-in driver's output files (tests/test_driver_formats_cpu.py).
 *
 * It implements the entry points of include/fgpe.h that the driver calls,
 * with deterministic values the test can recompute, so that the driver's
 * file layout (every WRITE of the reference's programs) is checked without a
 * GPU.  No arithmetic of the propagator is involved:
 *   state        kept as set (fgpe_get_state returns it unchanged)
 *   fgpe_step    advances a step counter c
 *   NORMC        norm[m] = 0.1 + 0.05 m + 1e-7 c
 *   observables  en = 3 + 1/(1 + c), mu[m] = en + 0.1 m, mz = 1e-5 c,
 *                rms[m] = 1.5 + 0.01 m + 1e-6 c
 *   CONV         max|dphi| = 1e-3 / (1 + c)
 *   centre       the state at (nx/2, ny/2, nz/2) (0-based)
 */
#include <stdlib.h>
#include <string.h>

#include "../../include/fgpe.h"

struct fgpe_s {
    fgpe_params p;
    int ms;
    long long npts, c;
    double* phi;
};

int fgpe_create(const fgpe_params* p, fgpe_t** out) {
    fgpe_t* h = (fgpe_t*)calloc(1, sizeof(fgpe_t));
    h->p = *p;
    h->ms = 2 * p->spin + 1;
    h->npts = (long long)p->nx * (p->dim >= 2 ? p->ny : 1) * (p->dim >= 3 ? p->nz : 1);
    h->phi = (double*)calloc((size_t)h->npts * h->ms * 2, sizeof(double));
    *out = h;
    return FGPE_OK;
}
int fgpe_destroy(fgpe_t* h) {
    if (h) { free(h->phi); free(h); }
    return FGPE_OK;
}
const char* fgpe_last_error(const fgpe_t* h) { (void)h; return "fake"; }
int fgpe_set_state(fgpe_t* h, const double* phi) {
    memcpy(h->phi, phi, sizeof(double) * 2 * h->npts * h->ms);
    return FGPE_OK;
}
int fgpe_get_state(fgpe_t* h, double* phi) {
    memcpy(phi, h->phi, sizeof(double) * 2 * h->npts * h->ms);
    return FGPE_OK;
}
int fgpe_normalize(fgpe_t* h, double* tnorm) {
    (void)h;
    if (tnorm) *tnorm = 1.0;
    return FGPE_OK;
}
int fgpe_step(fgpe_t* h, int nsteps) {
    h->c += nsteps;
    return FGPE_OK;
}
int fgpe_norms(fgpe_t* h, double* norm) {
    for (int m = 0; m < h->ms; ++m) norm[m] = 0.1 + 0.05 * m + 1e-7 * (double)h->c;
    return FGPE_OK;
}
int fgpe_observables(fgpe_t* h, double* en, double* mu, double* mz, double* rms) {
    *en = 3.0 + 1.0 / (1.0 + (double)h->c);
    for (int m = 0; m < h->ms; ++m) {
        mu[m] = *en + 0.1 * m;
        rms[m] = 1.5 + 0.01 * m + 1e-6 * (double)h->c;
    }
    *mz = 1e-5 * (double)h->c;
    return FGPE_OK;
}
int fgpe_conv(fgpe_t* h, double* max_dphi) {
    *max_dphi = 1e-3 / (1.0 + (double)h->c);
    return FGPE_OK;
}
int fgpe_center(fgpe_t* h, double* out) {
    const int ny = h->p.dim >= 2 ? h->p.ny : 1, nz = h->p.dim >= 3 ? h->p.nz : 1;
    const long long t = h->p.nx / 2 + (long long)h->p.nx * (ny / 2 + (long long)ny * (nz / 2));
    for (int m = 0; m < h->ms; ++m) {
        out[2 * m] = h->phi[2 * (t + m * h->npts)];
        out[2 * m + 1] = h->phi[2 * (t + m * h->npts) + 1];
    }
    return FGPE_OK;
}
