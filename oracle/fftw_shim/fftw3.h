/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Minimal FFTW-3 API declarations, written for this project, so that the
 * reference's PowerGrid/fftCPU.cpp (fftCPU.cpp:35-176) compiles and links
 * here although FFTW is not installed.  Only the entry points that file
 * calls are declared.  The implementation (fftw_shim.cpp) is a project FFT
 * (fft_engine.hpp), not FFTW: every number measured through it says so.
 */
#ifndef PG_ORACLE_FFTW3_SHIM_H
#define PG_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct pg_fftwf_plan_s* fftwf_plan;
typedef struct pg_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
