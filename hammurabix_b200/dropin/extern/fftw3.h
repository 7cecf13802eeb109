/* Declarations of the FFTW 3 entry points the hammurabiX objects linked
 * into the drop-in call, for builds where FFTW is not installed.  They
 * follow FFTW 3's public API (C linkage, fftw_complex = double[2]).  With
 * FFTW installed, build against its own header and library instead
 * (EXTERN_INC / EXTERN_LIBS in ../Makefile).  extern_stubs.cc defines the
 * allocation and plan calls Grid_brnd / Grid_ternd::build_grid make; a
 * transform throws, because no generator left on FFTW is replaced here. */
#ifndef HXG_DROPIN_FFTW3_H
#define HXG_DROPIN_FFTW3_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct hxg_dropin_fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
fftw_complex *fftw_alloc_complex(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
void fftw_destroy_plan(fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);
#ifdef __cplusplus
}
#endif
#endif
