/* Second CPU oracle for the fixed-particle Cahn-Hilliard time loop (FP64, C99).
 *
 * TEST INFRASTRUCTURE ONLY.  The tests, the smoke check and the CPU-baseline leg
 * of the benchmark may call it; the product library never does.
 *
 * It restates core_shell.jl:17-103 of saswataiith/embedded-spinodal-core-shell-julia
 * a second time, independently of the NumPy oracle (core_shell_oracle.py), and
 * with its own FFT: a recursive decimation-in-time transform over the prime
 * factors of n (radix 2, radix 3, and a plain DFT for any other prime), with
 * twiddle factors from long-double cos/sin.  It shares no code with pocketfft
 * (the NumPy oracle's FFT) or FFTW (the reference's), so the two oracles
 * agreeing pins both.
 *
 * Layout: element (i, j) of a field -- x = i (contiguous, the direction kx
 * varies along, core_shell.jl:21), y = j -- sits at j*n + i: the bytes of the
 * Julia matrix c[i, j] and of a C-ordered NumPy array a[j, i].  The history is
 * the Julia matrix zeros(steps+1, 6) (core_shell.jl:89), column-major.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

static const double kPi = 3.14159265358979323846;

/* ---- FFT ------------------------------------------------------------------ */

typedef struct {
  int n;       /* transform length */
  cplx* tw;    /* e^{-2 pi i e / n}, e < n */
  cplx* buf;   /* scratch, n */
  cplx* line;  /* gathered column, n */
} Plan;

static int smallest_factor(int n) {
  if (n % 2 == 0) return 2;
  if (n % 3 == 0) return 3;
  for (int f = 5; f * f <= n; f += 2)
    if (n % f == 0) return f;
  return n;
}

/* out[k] = sum_x in[x * stride] e^{-2 pi i k x / m}, for a sub-length m of the
 * plan's n (m divides n); out is contiguous and must not alias in. */
static void fft_rec(const Plan* P, cplx* out, const cplx* in, int m, int stride, cplx* scratch) {
  if (m == 1) {
    out[0] = in[0];
    return;
  }
  const int r = smallest_factor(m), q = m / r, step = P->n / m;
  /* sub-transforms of the r decimated sequences, into out[t*q .. t*q+q) */
  for (int t = 0; t < r; ++t) fft_rec(P, out + t * q, in + t * stride, q, stride * r, scratch);
  /* butterflies: X[k + q u] = sum_t W_m^{t (k + q u)} Y_t[k] */
  for (int k = 0; k < q; ++k) {
    for (int u = 0; u < r; ++u) {
      cplx acc = 0.0;
      for (int t = 0; t < r; ++t) {
        const long e = ((long)t * (k + (long)q * u)) % m;
        acc += P->tw[e * step] * out[t * q + k];
      }
      scratch[k + q * u] = acc;
    }
  }
  memcpy(out, scratch, sizeof(cplx) * (size_t)m);
}

static int plan_init(Plan* P, int n) {
  P->n = n;
  P->tw = malloc(sizeof(cplx) * (size_t)n);
  P->buf = malloc(sizeof(cplx) * (size_t)n);
  P->line = malloc(sizeof(cplx) * (size_t)n * 2);
  if (!P->tw || !P->buf || !P->line) return -1;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int e = 0; e < n; ++e) {
    const long double a = two_pi * (long double)e / (long double)n;
    P->tw[e] = (double)cosl(a) - I * (double)sinl(a);
  }
  return 0;
}

static void plan_free(Plan* P) {
  free(P->tw);
  free(P->buf);
  free(P->line);
}

/* 1-D transform of n values at stride s in place; inverse = conj(F(conj x)) / n */
static void fft_line(const Plan* P, cplx* a, int s, int inverse) {
  const int n = P->n;
  cplx* in = P->line;
  cplx* out = P->line + n;
  for (int x = 0; x < n; ++x) in[x] = inverse ? conj(a[(size_t)x * s]) : a[(size_t)x * s];
  fft_rec(P, out, in, n, 1, P->buf);
  for (int x = 0; x < n; ++x) a[(size_t)x * s] = inverse ? conj(out[x]) / n : out[x];
}

/* 2-D transform of an n x n field (rows along x, then columns along y) */
static void fft2(const Plan* P, cplx* a, int inverse) {
  const int n = P->n;
  for (int j = 0; j < n; ++j) fft_line(P, a + (size_t)j * n, 1, inverse);
  for (int i = 0; i < n; ++i) fft_line(P, a + i, n, inverse);
}

/* ---- the model (core_shell.jl) ---------------------------------------------- */

typedef struct {
  double A, B, chi, P, ca, cb, cc, kappa, mobility, Q;
} Params; /* core_shell.jl:4-15, field order of Parameters */

typedef struct {
  int n;
  double dx;
  double* kd;  /* first-derivative wavenumber, Nyquist zeroed (core_shell.jl:20) */
  double* k2;  /* |k|^2 with the Nyquist kept (core_shell.jl:23), n*n */
  double *h, *g, *M;
  Plan plan;
  cplx *w1, *w2, *w3;  /* complex work fields */
  double *mu, *gx, *gy;
} Model;

/* core_shell.jl:17-25 */
static void make_grid(Model* m) {
  const int n = m->n;
  for (int i = 0; i < n; ++i) {
    const int f = i < (n + 1) / 2 ? i : i - n; /* fftfreq ordering */
    const double k = 2.0 * kPi * (double)f / ((double)n * m->dx);
    m->kd[i] = (n % 2 == 0 && i == n / 2) ? 0.0 : k;
  }
  for (int j = 0; j < n; ++j) {
    const int fj = j < (n + 1) / 2 ? j : j - n;
    const double kj = 2.0 * kPi * (double)fj / ((double)n * m->dx);
    for (int i = 0; i < n; ++i) {
      const int fi = i < (n + 1) / 2 ? i : i - n;
      const double ki = 2.0 * kPi * (double)fi / ((double)n * m->dx);
      m->k2[(size_t)j * n + i] = ki * ki + kj * kj;
    }
  }
}

/* core_shell.jl:39-43 */
static void geometry(Model* m, const double* phi, const Params* p) {
  const size_t N = (size_t)m->n * m->n;
  for (size_t k = 0; k < N; ++k) {
    const double f = phi[k];
    m->h[k] = f * f * f * (10.0 - 15.0 * f + 6.0 * f * f);
    m->g[k] = f * f * (1.0 - f) * (1.0 - f);
    m->M[k] = p->mobility * m->h[k];
  }
}

/* core_shell.jl:45-49 */
static double bulk_energy(double c, double h, double g, const Params* p) {
  return p->A * (1.0 - h) * (c - p->ca) * (c - p->ca) + p->B * h * (c - p->cb) * (c - p->cb) * (c - p->cc) * (c - p->cc) +
         p->P * (1.0 - p->chi * c) * g;
}

/* core_shell.jl:51-55 */
static double bulk_derivative(double c, double h, double g, const Params* p) {
  return 2.0 * p->A * (1.0 - h) * (c - p->ca) + 2.0 * p->B * h * (c - p->cb) * (c - p->cc) * (2.0 * c - p->cb - p->cc) -
         p->chi * p->P * g;
}

/* core_shell.jl:57-60: mu = f'(c) + Re IFFT(2 kappa k^2 FFT(c)) */
static void chemical_potential(Model* m, const double* c, const Params* p) {
  const size_t N = (size_t)m->n * m->n;
  for (size_t k = 0; k < N; ++k) m->w1[k] = c[k];
  fft2(&m->plan, m->w1, 0);
  for (size_t k = 0; k < N; ++k) m->w1[k] *= 2.0 * p->kappa * m->k2[k];
  fft2(&m->plan, m->w1, 1);
  for (size_t k = 0; k < N; ++k) m->mu[k] = bulk_derivative(c[k], m->h[k], m->g[k], p) + creal(m->w1[k]);
}

/* core_shell.jl:62-70: divergence^ into w3, returns the dissipation */
static double transport_rate(Model* m, const double* c, const Params* p) {
  const int n = m->n;
  const size_t N = (size_t)n * n;
  chemical_potential(m, c, p);
  for (size_t k = 0; k < N; ++k) m->w1[k] = m->mu[k];
  fft2(&m->plan, m->w1, 0); /* mu^ */
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const size_t k = (size_t)j * n + i;
      m->w2[k] = I * m->kd[i] * m->w1[k];
      m->w3[k] = I * m->kd[j] * m->w1[k];
    }
  fft2(&m->plan, m->w2, 1);
  fft2(&m->plan, m->w3, 1);
  double diss = 0.0;
  for (size_t k = 0; k < N; ++k) {
    m->gx[k] = creal(m->w2[k]);
    m->gy[k] = creal(m->w3[k]);
    diss += m->M[k] * (m->gx[k] * m->gx[k] + m->gy[k] * m->gy[k]);
  }
  for (size_t k = 0; k < N; ++k) {
    m->w2[k] = m->M[k] * m->gx[k];
    m->w3[k] = m->M[k] * m->gy[k];
  }
  fft2(&m->plan, m->w2, 0);
  fft2(&m->plan, m->w3, 0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const size_t k = (size_t)j * n + i;
      m->w3[k] = I * m->kd[i] * m->w2[k] + I * m->kd[j] * m->w3[k];
    }
  return diss * m->dx * m->dx;
}

/* core_shell.jl:72-76 */
static void step(Model* m, double* c, const Params* p, double dt) {
  const size_t N = (size_t)m->n * m->n;
  transport_rate(m, c, p); /* divergence^ in w3 */
  for (size_t k = 0; k < N; ++k) m->w1[k] = c[k];
  fft2(&m->plan, m->w1, 0);
  for (size_t k = 0; k < N; ++k) {
    const double den = 1.0 + 2.0 * p->Q * p->kappa * m->k2[k] * m->k2[k] * dt;
    m->w1[k] += dt * m->w3[k] / den;
  }
  fft2(&m->plan, m->w1, 1);
  for (size_t k = 0; k < N; ++k) c[k] = creal(m->w1[k]);
}

/* core_shell.jl:78-82 (Parseval; the Nyquist mode included) */
static double energy(Model* m, const double* c, const Params* p) {
  const size_t N = (size_t)m->n * m->n;
  for (size_t k = 0; k < N; ++k) m->w1[k] = c[k];
  fft2(&m->plan, m->w1, 0);
  double grad = 0.0, bulk = 0.0;
  for (size_t k = 0; k < N; ++k) {
    const double a = cabs(m->w1[k]);
    grad += m->k2[k] * a * a;
    bulk += bulk_energy(c[k], m->h[k], m->g[k], p);
  }
  return (bulk + p->kappa * grad / (double)N) * m->dx * m->dx;
}

static void model_free(Model* m) {
  free(m->kd);
  free(m->k2);
  free(m->h);
  free(m->g);
  free(m->M);
  free(m->w1);
  free(m->w2);
  free(m->w3);
  free(m->mu);
  free(m->gx);
  free(m->gy);
  plan_free(&m->plan);
}

/* core_shell.jl:84-103 without the CSV output.  Returns 0, 1 (bad argument),
 * 3 (non-finite composition: *bad_step = s, after its history row) or 5 (out of
 * memory).  c_out receives the final field (unchanged from c0 on status 3). */
int cso_run_simulation(int n, double dx, const double* phi, const double* params, const double* c0, int steps,
                       double dt, double* c_out, double* history, int64_t* bad_step) {
  if (n < 2 || !(dx > 0.0) || !phi || !params || !c0 || !c_out || steps < 0) return 1;
  Params p;
  memcpy(&p, params, sizeof p);
  Model m;
  memset(&m, 0, sizeof m);
  m.n = n;
  m.dx = dx;
  const size_t N = (size_t)n * n;
  m.kd = malloc(sizeof(double) * (size_t)n);
  m.k2 = malloc(sizeof(double) * N);
  m.h = malloc(sizeof(double) * N);
  m.g = malloc(sizeof(double) * N);
  m.M = malloc(sizeof(double) * N);
  m.w1 = malloc(sizeof(cplx) * N);
  m.w2 = malloc(sizeof(cplx) * N);
  m.w3 = malloc(sizeof(cplx) * N);
  m.mu = malloc(sizeof(double) * N);
  m.gx = malloc(sizeof(double) * N);
  m.gy = malloc(sizeof(double) * N);
  double* c = malloc(sizeof(double) * N);
  if (plan_init(&m.plan, n) || !m.kd || !m.k2 || !m.h || !m.g || !m.M || !m.w1 || !m.w2 || !m.w3 || !m.mu || !m.gx ||
      !m.gy || !c) {
    free(c);
    model_free(&m);
    return 5;
  }
  make_grid(&m);
  geometry(&m, phi, &p);
  memcpy(c, c0, sizeof(double) * N);
  if (bad_step) *bad_step = -1;
  const size_t ld = (size_t)steps + 1;
  int status = 0;
  for (int s = 0; s <= steps; ++s) {
    const double diss = transport_rate(&m, c, &p);
    double sum = 0.0, mn = INFINITY, mx = -INFINITY;
    int finite = 1;
    for (size_t k = 0; k < N; ++k) {
      sum += c[k];
      mn = fmin(mn, c[k]);
      mx = fmax(mx, c[k]);
      if (!isfinite(c[k])) finite = 0;
    }
    if (history) {
      history[s] = (double)s * dt;
      history[s + ld] = sum / (double)N;
      history[s + 2 * ld] = energy(&m, c, &p);
      history[s + 3 * ld] = mn;
      history[s + 4 * ld] = mx;
      history[s + 5 * ld] = diss;
    }
    if (!finite) {
      if (bad_step) *bad_step = s;
      status = 3;
      break;
    }
    if (s < steps) step(&m, c, &p, dt);
  }
  memcpy(c_out, status ? c0 : c, sizeof(double) * N);
  free(c);
  model_free(&m);
  return status;
}

/* One 2-D forward (inverse = 0) or inverse transform of an n x n complex field
 * given as interleaved (re, im) doubles, in place: exposed so the tests can
 * check the FFT on its own against a direct DFT. */
int cso_fft2(int n, double* data, int inverse) {
  if (n < 1 || !data) return 1;
  Plan P;
  if (plan_init(&P, n)) {
    plan_free(&P);
    return 5;
  }
  fft2(&P, (cplx*)data, inverse);
  plan_free(&P);
  return 0;
}
