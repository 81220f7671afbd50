/* fftw3.h -- test infrastructure: a stand-in for the FFTW3 API subset that the
 * reference's PME (src/force/coulomb_pme.cpp) calls, so that file compiles
 * unmodified into the CPU checker (FFTW3 is not installed here and cannot be).
 * Declarations follow FFTW's public API (names, argument order, types); the
 * transforms are this repo's own (oracle/fft.h), FFTW's in-place layout kept.
 * Planning flags are accepted and ignored; threads are ignored (single thread). */
#ifndef DMD_FFTW3_SHIM_H
#define DMD_FFTW3_SHIM_H

typedef double fftw_complex[2];
typedef struct dmd_fftw_plan_s* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

#ifdef __cplusplus
extern "C" {
#endif

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
