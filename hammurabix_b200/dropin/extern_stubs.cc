// extern_stubs.cc -- FFTW and GSL entry points for drop-in builds where
// neither library is installed.
//
// On the line-of-sight path FFTW only allocates the random-field grids and
// creates plans (Grid_brnd::build_grid, source/grid/grid_brnd.cc:25-55;
// Grid_ternd::build_grid, source/grid/grid_ternd.cc:26-40; their
// destructors, include/grid.h:75-87, 129-134).  Those calls are served
// here: fftw_alloc_complex is an aligned allocation, a plan is a token that
// records its shape.  The B200 build replaces the generators Brnd_es and
// TErnd_dft with device code (generators_b200.cc); the ones it does not
// replace (Brnd_jf12, Brnd_mhd) draw from GSL's RNG and run FFTW
// transforms, and here they fail loudly: gsl_rng_alloc and
// fftw_execute_dft throw std::runtime_error.  Where GSL and FFTW are
// installed, link them instead of this file (EXTERN_LIBS in the Makefile)
// and those generators run on the CPU as in the reference.
#include <cstdlib>
#include <new>
#include <string>
#include <stdexcept>

#include <fftw3.h>
#include <gsl/gsl_randist.h>
#include <gsl/gsl_rng.h>

namespace {
[[noreturn]] void unsupported(const char *what) {
  throw std::runtime_error(std::string(what) +
                           ": this random-field generator is not replaced on the B200 "
                           "build and needs GSL and FFTW, which this build does not link "
                           "(supported generators: Brnd_es, TErnd_dft)");
}
}  // namespace

struct hxg_dropin_fftw_plan_s {
  int n0, n1, n2, sign;
};
struct hxg_dropin_gsl_rng_type_s {
  int id;
};

extern "C" {

fftw_complex *fftw_alloc_complex(size_t n) {
  void *p = nullptr;
  // FFTW aligns to at least 16 bytes; 64 keeps whole cache lines
  if (posix_memalign(&p, 64, (n > 0 ? n : 1) * sizeof(fftw_complex)) != 0) throw std::bad_alloc();
  return static_cast<fftw_complex *>(p);
}

void fftw_free(void *p) { std::free(p); }

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *, fftw_complex *, int sign,
                           unsigned) {
  return new hxg_dropin_fftw_plan_s{n0, n1, n2, sign};
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute_dft(const fftw_plan, fftw_complex *, fftw_complex *) {
  unsupported("fftw_execute_dft");
}

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}

static const hxg_dropin_gsl_rng_type_s kTaus{0};
const gsl_rng_type *gsl_rng_taus = &kTaus;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *) { unsupported("gsl_rng_alloc"); }
void gsl_rng_set(const gsl_rng *, unsigned long int) { unsupported("gsl_rng_set"); }
void gsl_rng_free(gsl_rng *) {}
double gsl_rng_uniform(const gsl_rng *) { unsupported("gsl_rng_uniform"); }
double gsl_ran_ugaussian(const gsl_rng *) { unsupported("gsl_ran_ugaussian"); }

}  // extern "C"
