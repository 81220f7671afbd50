// fftw_shim.cpp -- test infrastructure: implementation of the FFTW-API subset
// declared in shims/fftw3.h on top of oracle/fft.h.  FFTW semantics kept:
// r2c / c2r over an n0 x n1 x n2 real array (last index fastest); in place
// (in == out) the real rows have a pitch of 2(n2/2+1) doubles, out of place the
// real array is dense; c2r is unnormalised.  Also answers the one OpenMP
// runtime query that file makes.
#include "fftw3.h"

#include "../fft.h"

struct dmd_fftw_plan_s {
    int n0, n1, n2;
    bool r2c;
    double* real;
    double* cplx;
};

extern "C" {

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned) {
    return new dmd_fftw_plan_s{n0, n1, n2, true, in, reinterpret_cast<double*>(out)};
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned) {
    return new dmd_fftw_plan_s{n0, n1, n2, false, out, reinterpret_cast<double*>(in)};
}

void fftw_execute(const fftw_plan p) {
    const bool inplace = p->real == p->cplx;
    const size_t pitch = inplace ? static_cast<size_t>(2 * (p->n2 / 2 + 1)) : static_cast<size_t>(p->n2);
    if (p->r2c) dmd_fft::r2c3d(p->real, pitch, p->cplx, p->n0, p->n1, p->n2);
    else dmd_fft::c2r3d(p->cplx, p->real, pitch, p->n0, p->n1, p->n2);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

// The reference's PME sizes FFTW's thread pool with omp_get_max_threads()
// (coulomb_pme.cpp:17); the OpenMP runtime is not installed here and the
// transforms are single-threaded, so the query answers 1.
int omp_get_max_threads(void) { return 1; }

}  // extern "C"
