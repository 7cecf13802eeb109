/*
 * shim.cc -- bodies for the stand-in GSL / FFTW headers in this directory.
 * Test infrastructure for the oracle build of the reference (oracle/Makefile).
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

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

// ---- GSL RNG stand-in ----------------------------------------------------
// Default: splitmix64 uniforms, Box-Muller normals.  Cell-stream mode
// (hxo_shim_cell_stream(k), k > 0): draw t of a generator seeded with s is
// deviate t % k of k-space cell 1 + t / k (the generators skip cell 0), from
// Philox4x32-10 (Salmon et al., SC 2011) keyed by s with counter
// {cell, cell >> 32, block, 0x52464721} and Box-Muller on 53-bit uniforms:
// the same deviates the device generators draw for that cell.
// The reference CLI (oracle/_ref/hamx) takes the mode from the environment:
// HXO_SHIM_CELL_STREAM = "k" or "k0,k1,..." per gsl_rng_set call in order
// (the Pipeline runs TErnd_dft before Brnd_es, main_std.cc:35-36).
static int g_cell_stream = 0;
extern "C" void hxo_shim_cell_stream(int k) { g_cell_stream = k; }
static int cells_for_next_seed() {
  static int calls = 0;
  const int call = calls++;
  if (g_cell_stream > 0) return g_cell_stream;
  const char *e = std::getenv("HXO_SHIM_CELL_STREAM");
  if (!e) return 0;
  int k = 0;
  for (int i = 0; i <= call && *e; ++i) {
    k = std::atoi(e);
    while (*e && *e != ',') ++e;
    if (*e == ',') ++e;
  }
  return k;
}

static void philox4x32_10(unsigned c[4], unsigned k0, unsigned k1) {
  for (int r = 0; r < 10; ++r) {
    const unsigned long long p0 = 0xD2511F53ull * c[0], p1 = 0xCD9E8D57ull * c[2];
    const unsigned n0 = (unsigned)(p1 >> 32) ^ c[1] ^ k0;
    const unsigned n2 = (unsigned)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (unsigned)p1;
    c[3] = (unsigned)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

static double cell_deviate(unsigned long long seed, unsigned long long cell, int q) {
  const int b = q / 2, pair = q % 2;
  unsigned c[4] = {(unsigned)cell, (unsigned)(cell >> 32), (unsigned)b, 0x52464721u};
  philox4x32_10(c, (unsigned)seed, (unsigned)(seed >> 32));
  double u[2];
  for (int i = 0; i < 2; ++i) {
    const unsigned long long w = ((unsigned long long)c[2 * i] << 21) ^ (c[2 * i + 1] >> 11);
    u[i] = ((double)(w & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
  }
  const double r = std::sqrt(-2. * std::log(u[0]));
  const double a = 6.283185307179586476925 * u[1];
  return pair == 0 ? r * std::cos(a) : r * std::sin(a);
}

static const gsl_rng_type kTaus = {1};
const gsl_rng_type *gsl_rng_taus = &kTaus;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *) {
  gsl_rng *r = static_cast<gsl_rng *>(std::malloc(sizeof(gsl_rng)));
  r->state = 0x9E3779B97F4A7C15ULL;
  r->seed = 0;
  r->draws = 0;
  r->cells = 0;
  return r;
}
void gsl_rng_set(const gsl_rng *r, unsigned long int seed) {
  gsl_rng *s = const_cast<gsl_rng *>(r);
  s->state = seed * 0x9E3779B97F4A7C15ULL + 1;
  s->seed = seed;
  s->draws = 0;
  s->cells = cells_for_next_seed();
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
  const int k = r->cells;
  if (k > 0) {
    gsl_rng *s = const_cast<gsl_rng *>(r);
    const unsigned long long t = s->draws++;
    return cell_deviate(s->seed, 1 + t / k, (int)(t % k));
  }
  double u1 = gsl_rng_uniform(r), u2 = gsl_rng_uniform(r);
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2. * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// ---- FFTW stand-in: unnormalised 3-D DFT by separable direct sums --------
// FFTW's definition: out[k] = sum_j in[j] exp(sign 2 pi i j k / n) along
// each axis, row-major (n2 fastest).  O(n) per output, for the small grids
// the tests run.
struct hxo_fftw_plan_s {
  int n[3];
  int sign;
};
fftw_complex *fftw_alloc_complex(std::size_t n) {
  return static_cast<fftw_complex *>(std::malloc(n * sizeof(fftw_complex)));
}
void fftw_free(void *p) { std::free(p); }
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *, fftw_complex *, int sign,
                           unsigned) {
  return new hxo_fftw_plan_s{{n0, n1, n2}, sign};
}
void fftw_destroy_plan(fftw_plan p) { delete p; }
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
  const std::size_t n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
  const std::size_t total = n0 * n1 * n2;
  if (out != in)
    for (std::size_t i = 0; i < total; ++i) out[i][0] = in[i][0], out[i][1] = in[i][1];
  const std::size_t stride[3] = {n1 * n2, n2, 1};
  for (int ax = 0; ax < 3; ++ax) {
    const std::size_t n = p->n[ax];
    std::vector<double> wr(n), wi(n), lr(n), li(n);
    for (std::size_t m = 0; m < n; ++m) {
      const double a = 6.283185307179586476925 * (double)m / (double)n;
      wr[m] = std::cos(a);
      wi[m] = p->sign * std::sin(a);
    }
    const std::size_t st = stride[ax];
    for (std::size_t base = 0; base < total; ++base) {
      if ((base / st) % n != 0) continue;  // first element of each line
      for (std::size_t k = 0; k < n; ++k) {
        double sr = 0., si = 0.;
        for (std::size_t j = 0; j < n; ++j) {
          const std::size_t m = (j * k) % n;
          const double xr = out[base + j * st][0], xi = out[base + j * st][1];
          sr += xr * wr[m] - xi * wi[m];
          si += xr * wi[m] + xi * wr[m];
        }
        lr[k] = sr;
        li[k] = si;
      }
      for (std::size_t k = 0; k < n; ++k) out[base + k * st][0] = lr[k], out[base + k * st][1] = li[k];
    }
  }
}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}
