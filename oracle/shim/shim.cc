/*
 * shim.cc -- bodies for the stand-in GSL / FFTW headers in this directory.
 * Test infrastructure for the oracle build of the reference (oracle/Makefile).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include <fftw3.h>
#include <gsl/gsl_randist.h>
#include <gsl/gsl_rng.h>
#include <gsl/gsl_sf_synchrotron.h>

// ---- synchrotron functions, from their integral definitions -------------
// F(x) = x * Int_x^inf K_{5/3}(t) dt.  With t = x*exp(u) the integrand
// K_{5/3}(t)*t is smooth in u; composite 10-point Gauss-Legendre panels.
static const double kGLx[10] = {
    -0.9739065285171717, -0.8650633666889845, -0.6794095682990244,
    -0.4333953941292472, -0.1488743389816312, 0.1488743389816312,
    0.4333953941292472,  0.6794095682990244,  0.8650633666889845,
    0.9739065285171717};
static const double kGLw[10] = {
    0.0666713443086881, 0.1494513491505806, 0.2190863625159820,
    0.2692667193099963, 0.2955242247147529, 0.2955242247147529,
    0.2692667193099963, 0.2190863625159820, 0.1494513491505806,
    0.0666713443086881};

double gsl_sf_synchrotron_1(const double x) {
  if (!(x > 0)) return 0.;
  const double umax = std::log((x + 80.) / x);
  const int panels = 64 + static_cast<int>(16. * umax);
  const double h = umax / panels;
  double acc = 0.;
  for (int p = 0; p < panels; ++p) {
    const double a = p * h;
    for (int k = 0; k < 10; ++k) {
      const double u = a + 0.5 * h * (kGLx[k] + 1.);
      const double t = x * std::exp(u);
      acc += kGLw[k] * std::cyl_bessel_k(5. / 3., t) * t;
    }
  }
  return x * acc * 0.5 * h;
}

double gsl_sf_synchrotron_2(const double x) {
  if (!(x > 0)) return 0.;
  return x * std::cyl_bessel_k(2. / 3., x);
}

// ---- GSL RNG stand-in (generators only; never on the integration path) --
static const gsl_rng_type kTaus = {1};
const gsl_rng_type *gsl_rng_taus = &kTaus;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *) {
  gsl_rng *r = static_cast<gsl_rng *>(std::malloc(sizeof(gsl_rng)));
  r->state = 0x9E3779B97F4A7C15ULL;
  return r;
}
void gsl_rng_set(const gsl_rng *r, unsigned long int seed) {
  const_cast<gsl_rng *>(r)->state = seed * 0x9E3779B97F4A7C15ULL + 1;
}
void gsl_rng_free(gsl_rng *r) { std::free(r); }
double gsl_rng_uniform(const gsl_rng *r) {
  gsl_rng *s = const_cast<gsl_rng *>(r);
  unsigned long long z = (s->state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (z >> 11) * (1.0 / 9007199254740992.0);
}
double gsl_ran_ugaussian(const gsl_rng *r) {
  double u1 = gsl_rng_uniform(r), u2 = gsl_rng_uniform(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2. * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// ---- FFTW stand-in: allocation and plan bookkeeping only ----------------
struct hxo_fftw_plan_s {
  int dummy;
};
fftw_complex *fftw_alloc_complex(std::size_t n) {
  return static_cast<fftw_complex *>(std::malloc(n * sizeof(fftw_complex)));
}
void fftw_free(void *p) { std::free(p); }
fftw_plan fftw_plan_dft_3d(int, int, int, fftw_complex *, fftw_complex *, int,
                           unsigned) {
  return new hxo_fftw_plan_s{0};
}
void fftw_destroy_plan(fftw_plan p) { delete p; }
void fftw_execute_dft(const fftw_plan, fftw_complex *, fftw_complex *) {
  std::fprintf(stderr, "oracle build: FFTs (random-field generators) are not "
                       "available; read field grids from files instead\n");
  std::abort();
}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}
