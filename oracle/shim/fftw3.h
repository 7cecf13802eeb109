/* Stand-in for FFTW 3.3's fftw3.h.  On the integration path FFTW only
 * allocates buffers and creates plans (Grid_brnd/Grid_ternd::build_grid);
 * the random-field generators run the transforms, here an unnormalised
 * direct-sum DFT for the small grids of the tests (shim.cc). */
#ifndef HXO_SHIM_FFTW3_H
#define HXO_SHIM_FFTW3_H
#include <cstddef>
typedef double fftw_complex[2];
typedef struct hxo_fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
fftw_complex *fftw_alloc_complex(std::size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
void fftw_destroy_plan(fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);
#endif
