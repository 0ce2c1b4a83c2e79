// Kernel sets for grid sizes without a tuned, compile-time plan: any n from 2 to
// 4096, odd or even, whose largest prime factor is at most 127 (or any n up to
// 512).  The reference's make_grid / fft accept every n (core_shell.jl:17-25,
// FFTW); the tuned sets cover the even 2^a 3^b sizes the benchmarks use, and
// these kernels give every other size the same step, bit-for-bit semantics and
// history, at lower speed.
//
// Layout (per instance, runtime n, K = n/2 + 1 half-spectrum modes):
//   S, F : K x n complex, element (y, kx) at y*K + kx -- the x-transform of the
//          real rows (kx = 0 .. n/2).  No packing: the self-conjugate modes
//          (kx = 0, and kx = n/2 for even n) are stored as complex numbers whose
//          imaginary parts are kept at zero, which is the real.(ifft(...))
//          projection of core_shell.jl:59,64-65,75 for those modes.
//   G    : pair array, (y, kx) -> (x-transform of d mu/dx, of d mu/dy), then the
//          same for the fluxes M grad mu.
// The derivative wavenumber of the even-n Nyquist is zero (core_shell.jl:20),
// k^2 keeps it (:23); odd n has no Nyquist.
//
// Transforms: one length-n DFT per block at a time, in shared memory, as a
// Stockham sequence of radix passes with runtime radices (4, 2, 3, 5, 7, then
// any prime factor).  A pass of radix r computes every output as the r-term sum
// sum_s x_s w^(s e) with the twiddle folded into the exponent e, reading the
// plain table e^{-2 pi i j / n}: O(n r) work per pass, exact-table accuracy.
// Blocks stride over the row pairs / columns of their instance (grid = fixed
// blocks x instances), so the launch needs no size; partial sums and the
// last-arriver fold follow the tuned kernels (esc_kernels.cuh).
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "esc_dispatch.cuh"

namespace esc {
namespace gen {

constexpr int kThreads = 256;
constexpr int kBlocks = 128;  // blocks per instance in every kernel
constexpr int kMaxPass = 16;
constexpr int kMaxPrime = 127;

struct GPlan {
  int n, np;
  int r[kMaxPass];
};

// radices of n: fours first, then a two, then the odd primes in increasing order
__device__ void make_plan(int n, GPlan& p) {
  p.n = n;
  p.np = 0;
  int m = n;
  while (m % 4 == 0 && p.np < kMaxPass) {
    p.r[p.np++] = 4;
    m /= 4;
  }
  if (m % 2 == 0 && p.np < kMaxPass) {
    p.r[p.np++] = 2;
    m /= 2;
  }
  for (int f = 3; f * f <= m && p.np < kMaxPass; f += 2)
    while (m % f == 0 && p.np < kMaxPass) {
      p.r[p.np++] = f;
      m /= f;
    }
  if (m > 1 && p.np < kMaxPass) p.r[p.np++] = m;
}

__device__ __forceinline__ bool selfconj(int k, int n) { return k == 0 || 2 * k == n; }

// Length-n DFT of a[0..n) (shared memory), b[0..n) the ping-pong partner;
// returns the buffer holding the result.  Every thread of the block calls it.
template <bool INV, typename R>
__device__ cpx<R>* gfft(cpx<R>* a, cpx<R>* b, const GPlan& pl, const cpx<R>* __restrict__ tw) {
  const int n = pl.n;
  int ns = 1;
  for (int p = 0; p < pl.np; ++p) {
    const int r = pl.r[p];
    const int m = n / r;            // butterflies of this pass
    const int L = n / (ns * r);     // twiddle stride of butterfly k
    for (int o = threadIdx.x; o < n; o += blockDim.x) {
      const int q = o / m, j = o - q * m;
      const int k = j % ns;
      const int e = k * L + q * m;  // exponent of input s is s*e (mod n), e < n
      cpx<R> acc = a[j];
      int idx = e;
      for (int s = 1; s < r; ++s) {
        const cpx<R> x = a[j + s * m];
        const cpx<R> w = ldc(tw + idx);
        acc = acc + (INV ? cmulconj(x, w) : cmul(x, w));
        idx += e;
        if (idx >= n) idx -= n;
      }
      b[(j / ns) * ns * r + k + q * ns] = acc;
    }
    __syncthreads();
    cpx<R>* t = a;
    a = b;
    b = t;
    ns *= r;
  }
  return a;
}

// shared plan + status of the block's instance
struct Head {
  GPlan pl;
  int status;
};

__device__ __forceinline__ void setup(Head& h, const InstDev& I) {
  if (threadIdx.x == 0) {
    make_plan(I.n, h.pl);
    h.status = *(volatile const int*)I.status;
  }
  __syncthreads();
}

// Full spectrum Z(k) = Xa(k) + i Xb(k) of two real rows from their half spectra.
template <typename R, typename LD>
__device__ __forceinline__ cpx<R> merge_pair(int k, int n, int K, LD&& ld) {
  cpx<R> a, b;
  if (k < K) {
    ld(k, a, b);
    if (selfconj(k, n)) {
      a.y = 0;
      b.y = 0;
    }
  } else {
    ld(n - k, a, b);
    a = cconj(a);
    b = cconj(b);
  }
  return mkc<R>(a.x - b.y, a.y + b.x);
}

// Half spectra of the two real rows a, b from Y = DFT(a + i b): for k < K,
// Xa(k) = (Y(k) + conj Y(n-k)) / 2 and Xb(k) = -i (Y(k) - conj Y(n-k)) / 2.
template <typename R>
__device__ __forceinline__ void split_at(const cpx<R>* y, int k, int n, cpx<R>& xa, cpx<R>& xb) {
  const cpx<R> y1 = y[k], y2 = cconj(y[(n - k) % n]);
  xa = cscale(y1 + y2, (R)0.5);
  xb = cscale(times_negi(y1 - y2), (R)0.5);
}

template <typename R>
__device__ __forceinline__ R wn(int i, int n, double kunit) {  // 2 pi fftfreq(n, dx)[i]
  return (R)(kunit * (double)(2 * i < n ? i : i - n));
}

// ---- init: c (FP64 real) -> S ------------------------------------------------------
template <typename SR>
__global__ void __launch_bounds__(kThreads) kg_init(const InstDev* __restrict__ insts) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Head h;
  const InstDev& I = insts[blockIdx.y];
  setup(h, I);
  const int n = h.pl.n, K = n / 2 + 1, npairs = (n + 1) / 2;
  cpx<SR>* A = reinterpret_cast<cpx<SR>*>(smraw);
  cpx<SR>* B = A + n;
  cpx<SR>* S = reinterpret_cast<cpx<SR>*>(I.S);
  const cpx<SR>* tw = reinterpret_cast<const cpx<SR>*>(I.tw_s);
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    const int ya = 2 * p, yb = ya + 1;
    const bool hasb = yb < n;
    for (int x = threadIdx.x; x < n; x += blockDim.x)
      A[x] = mkc<SR>((SR)I.cio[(size_t)ya * n + x], hasb ? (SR)I.cio[(size_t)yb * n + x] : (SR)0);
    __syncthreads();
    const cpx<SR>* Y = gfft<false>(A, B, h.pl, tw);
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      cpx<SR> xa, xb;
      split_at(Y, k, n, xa, xb);
      S[(size_t)ya * K + k] = xa;
      if (hasb) S[(size_t)yb * K + k] = xb;
    }
    __syncthreads();
  }
}

// ---- final: S -> c (FP64 real) -------------------------------------------------------
template <typename SR>
__global__ void __launch_bounds__(kThreads) kg_final(const InstDev* __restrict__ insts) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Head h;
  const InstDev& I = insts[blockIdx.y];
  setup(h, I);
  if (h.status) return;  // a stopped instance keeps its input c
  const int n = h.pl.n, K = n / 2 + 1, npairs = (n + 1) / 2;
  cpx<SR>* A = reinterpret_cast<cpx<SR>*>(smraw);
  cpx<SR>* B = A + n;
  const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
  const cpx<SR>* tw = reinterpret_cast<const cpx<SR>*>(I.tw_s);
  const double inv = 1.0 / n;
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    const int ya = 2 * p, yb = ya + 1;
    const bool hasb = yb < n;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      A[k] = merge_pair<SR>(k, n, K, [&](int i, cpx<SR>& a, cpx<SR>& b) {
        a = S[(size_t)ya * K + i];
        b = hasb ? S[(size_t)yb * K + i] : mkc<SR>(0, 0);
      });
    __syncthreads();
    const cpx<SR>* Z = gfft<true>(A, B, h.pl, tw);
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
      I.cio[(size_t)ya * n + x] = (double)Z[x].x * inv;
      if (hasb) I.cio[(size_t)yb * n + x] = (double)Z[x].y * inv;
    }
    __syncthreads();
  }
}

// ---- row A: c, bulk terms, history partials, F = x-transform of f' ------------------
template <typename SR, typename WR>
__global__ void __launch_bounds__(kThreads) kg_row_a(const InstDev* __restrict__ insts, const int* __restrict__ base,
                                                     int s_local) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Head h;
  __shared__ double red[32];
  __shared__ int lastflag;
  const InstDev& I = insts[blockIdx.y];
  setup(h, I);
  if (h.status) return;
  const int n = h.pl.n, K = n / 2 + 1, npairs = (n + 1) / 2;
  cpx<SR>* A = reinterpret_cast<cpx<SR>*>(smraw);
  cpx<SR>* B = A + n;
  const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
  cpx<WR>* F = reinterpret_cast<cpx<WR>*>(I.F);
  const WR* phi = reinterpret_cast<const WR*>(I.phi);
  const ModelParams mp = I.p;
  const double inv = 1.0 / n;
  double sum_c = 0.0, sum_f = 0.0, mn = INFINITY, mx = -INFINITY, bad = 0.0;
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    const int ya = 2 * p, yb = ya + 1;
    const bool hasb = yb < n;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      A[k] = merge_pair<SR>(k, n, K, [&](int i, cpx<SR>& a, cpx<SR>& b) {
        a = S[(size_t)ya * K + i];
        b = hasb ? S[(size_t)yb * K + i] : mkc<SR>(0, 0);
      });
    __syncthreads();
    const cpx<SR>* Z = gfft<true>(A, B, h.pl, reinterpret_cast<const cpx<SR>*>(I.tw_s));
    // f' of both rows into the other buffer (work precision), then its forward transform
    cpx<WR>* W0 = reinterpret_cast<cpx<WR>*>(Z == A ? B : A);
    cpx<WR>* W1 = reinterpret_cast<cpx<WR>*>(const_cast<cpx<SR>*>(Z));
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
      const double ca = (double)Z[x].x * inv, cb = hasb ? (double)Z[x].y * inv : 0.0;
      const WR pa = __ldg(phi + (size_t)ya * n + x), pb = hasb ? __ldg(phi + (size_t)yb * n + x) : (WR)0;
      double fa, fb = 0.0, ea, eb = 0.0;
      if constexpr (kSplitMixed<SR, WR>) {
        f2 fp, fv;
        bulk_pair_split(ca, cb, (float)pa, (float)pb, mp, fp, fv);
        fa = fp.v.x;
        ea = fv.v.x;
        if (hasb) {
          fb = fp.v.y;
          eb = fv.v.y;
        }
      } else {
        SR f1, e1;
        bulk<SR>((SR)ca, (SR)pa, mp, f1, e1);
        fa = f1;
        ea = e1;
        if (hasb) {
          bulk<SR>((SR)cb, (SR)pb, mp, f1, e1);
          fb = f1;
          eb = e1;
        }
      }
      sum_c += hasb ? ca + cb : ca;
      sum_f += hasb ? ea + eb : ea;
      mn = fmin(mn, hasb ? fmin(ca, cb) : ca);
      mx = fmax(mx, hasb ? fmax(ca, cb) : ca);
      bad += (nonfinite_bits(ca) || (hasb && nonfinite_bits(cb))) ? 1.0 : 0.0;
      W0[x] = mkc<WR>((WR)fa, (WR)fb);
    }
    __syncthreads();
    const cpx<WR>* Y = gfft<false>(W0, W1, h.pl, reinterpret_cast<const cpx<WR>*>(I.tw_w));
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      cpx<WR> xa, xb;
      split_at(Y, k, n, xa, xb);
      F[(size_t)ya * K + k] = xa;
      if (hasb) F[(size_t)yb * K + k] = xb;
    }
    __syncthreads();
  }
  const double r_sum = block_reduce<OpSum>(sum_c, red);
  const double r_min = block_reduce<OpMin>(mn, red);
  const double r_max = block_reduce<OpMax>(mx, red);
  const double r_f = block_reduce<OpSum>(sum_f, red);
  const double r_bad = block_reduce<OpSum>(bad, red);
  if (threadIdx.x == 0) {
    double* pp = I.part + (size_t)blockIdx.x * 5;
    pp[0] = r_sum;
    pp[1] = r_min;
    pp[2] = r_max;
    pp[3] = r_f;
    pp[4] = r_bad;
  }
  const int tiles = gridDim.x;
  if (!arrive_last(&I.cnt[0], tiles, &lastflag)) return;
  const double a_sum = reduce_partials<OpSum>(I.part + 0, tiles, 5, 0.0, red);
  const double a_min = reduce_partials<OpMin>(I.part + 1, tiles, 5, INFINITY, red);
  const double a_max = reduce_partials<OpMax>(I.part + 2, tiles, 5, -INFINITY, red);
  const double a_f = reduce_partials<OpSum>(I.part + 3, tiles, 5, 0.0, red);
  const double a_bad = reduce_partials<OpSum>(I.part + 4, tiles, 5, 0.0, red);
  if (threadIdx.x == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) {
      const size_t ld = (size_t)I.hist_ld;
      I.hist[s] = (double)s * I.dt;
      I.hist[s + 1 * ld] = a_sum / ((double)n * n);
      I.hist[s + 3 * ld] = a_min;
      I.hist[s + 4 * ld] = a_max;
    }
    I.scal[0] = a_f;
    if (a_bad > 0.0) {
      *I.bad_step = s;
      *I.status = kStatusNonFinite;
    }
    I.cnt[0] = 0;
  }
}

// ---- column A: c^, gradient energy, mu^, inverse y-transforms of i k mu^ -> G --------
template <typename SR, typename WR>
__global__ void __launch_bounds__(kThreads) kg_col_a(const InstDev* __restrict__ insts, const int* __restrict__ base,
                                                     int s_local) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Head h;
  __shared__ double red[32];
  __shared__ int lastflag;
  const InstDev& I = insts[blockIdx.y];
  setup(h, I);
  if (h.status) return;
  const int n = h.pl.n, K = n / 2 + 1;
  // three buffers of n complex SR; the WR transforms use the same slots
  cpx<SR>* P0 = reinterpret_cast<cpx<SR>*>(smraw);
  cpx<SR>* P1 = P0 + n;
  cpx<SR>* P2 = P1 + n;
  const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
  const cpx<WR>* F = reinterpret_cast<const cpx<WR>*>(I.F);
  cpx2<WR>* Gp = reinterpret_cast<cpx2<WR>*>(I.G);
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)n * I.dx);
  const double kappa = I.p.kappa;
  const WR scale = (WR)(1.0 / ((double)n * (double)n));
  double gsum = 0.0;
  for (int kx = blockIdx.x; kx < K; kx += gridDim.x) {
    const bool sc = selfconj(kx, n);
    const double kxf = kunit * (double)kx;                  // kx <= n/2: the non-negative branch
    const WR kxd = (2 * kx == n) ? (WR)0 : (WR)kxf;         // derivative Nyquist zeroed
    const double wgt = sc ? 1.0 : 2.0;                      // modes kx and -kx of the full spectrum
    for (int y = threadIdx.x; y < n; y += blockDim.x) P0[y] = S[(size_t)y * K + kx];
    __syncthreads();
    cpx<SR>* C = gfft<false>(P0, P1, h.pl, reinterpret_cast<const cpx<SR>*>(I.tw_s));  // c^ (kx, .)
    cpx<SR>* freeS = (C == P0) ? P1 : P0;
    cpx<WR>* Fa = reinterpret_cast<cpx<WR>*>(freeS);
    cpx<WR>* Fb = reinterpret_cast<cpx<WR>*>(P2);
    for (int y = threadIdx.x; y < n; y += blockDim.x) Fa[y] = F[(size_t)y * K + kx];
    __syncthreads();
    cpx<WR>* Fh = gfft<false>(Fa, Fb, h.pl, reinterpret_cast<const cpx<WR>*>(I.tw_w));  // f'^ (kx, .)
    // mu^ and the two derivative spectra: the x-derivative into the free work slot, the
    // y-derivative in place over f'^ (same element type, same index: no other thread's data)
    cpx<WR>* Dx = (Fh == Fa) ? Fb : Fa;
    cpx<WR>* Dy = Fh;
    for (int ky = threadIdx.x; ky < n; ky += blockDim.x) {
      const double kyf = kunit * (double)(2 * ky < n ? ky : ky - n);
      const double k2 = kxf * kxf + kyf * kyf;
      const cpx<SR> c = C[ky];
      gsum += wgt * k2 * ((double)c.x * c.x + (double)c.y * c.y);
      const cpx<WR> mu = cscale(Fh[ky] + ccast<WR>(cscale(c, (SR)(2.0 * kappa * k2))), scale);
      const WR kyd = (2 * ky == n) ? (WR)0 : (WR)kyf;
      Dx[ky] = times_i(cscale(mu, kxd));
      Dy[ky] = times_i(cscale(mu, kyd));
    }
    __syncthreads();
    // inverse transforms; c^'s slot is free now and serves as the partner buffer
    cpx<WR>* Cw = reinterpret_cast<cpx<WR>*>(C);
    cpx<WR>* gx = gfft<true>(Dx, Cw, h.pl, reinterpret_cast<const cpx<WR>*>(I.tw_w));
    cpx<WR>* spare2 = (gx == Dx) ? Cw : Dx;
    cpx<WR>* gy = gfft<true>(Dy, spare2, h.pl, reinterpret_cast<const cpx<WR>*>(I.tw_w));
    for (int y = threadIdx.x; y < n; y += blockDim.x) {
      cpx2<WR> o;
      o.a = gx[y];
      o.b = gy[y];
      if (sc) {  // self-conjugate column: the real.() projection
        o.a.y = 0;
        o.b.y = 0;
      }
      Gp[(size_t)y * K + kx] = o;
    }
    __syncthreads();
  }
  const double r = block_reduce<OpSum>(gsum, red);
  double* part = I.part + (size_t)5 * gridDim.x;
  if (threadIdx.x == 0) part[blockIdx.x] = r;
  const int tiles = gridDim.x;
  if (!arrive_last(&I.cnt[1], tiles, &lastflag)) return;
  const double gr = reduce_partials<OpSum>(part, tiles, 1, 0.0, red);
  if (threadIdx.x == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) I.hist[s + 2 * (size_t)I.hist_ld] = (I.scal[0] + kappa * gr / ((double)n * n)) * I.dx * I.dx;
    I.cnt[1] = 0;
  }
}

// ---- row B: grad mu, dissipation, M grad mu, forward x-transform back into G ----------
template <typename SR, typename WR>
__global__ void __launch_bounds__(kThreads) kg_row_b(const InstDev* __restrict__ insts, const int* __restrict__ base,
                                                     int s_local) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Head h;
  __shared__ double red[32];
  __shared__ int lastflag;
  const InstDev& I = insts[blockIdx.y];
  setup(h, I);
  if (h.status) return;
  const int n = h.pl.n, K = n / 2 + 1;
  cpx<WR>* A = reinterpret_cast<cpx<WR>*>(smraw);
  cpx<WR>* B = A + n;
  cpx2<WR>* Gp = reinterpret_cast<cpx2<WR>*>(I.G);
  const WR* phi = reinterpret_cast<const WR*>(I.phi);
  const cpx<WR>* tw = reinterpret_cast<const cpx<WR>*>(I.tw_w);
  const WR M0 = (WR)I.p.mobility;
  double dsum = 0.0;
  for (int y = blockIdx.x; y < n; y += gridDim.x) {
    cpx2<WR>* row = Gp + (size_t)y * K;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      A[k] = merge_pair<WR>(k, n, K, [&](int i, cpx<WR>& a, cpx<WR>& b) {
        const cpx2<WR> q = row[i];
        a = q.a;
        b = q.b;
      });
    __syncthreads();
    cpx<WR>* Z = gfft<true>(A, B, h.pl, tw);  // (d mu/dx, d mu/dy) in (re, im)
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
      const WR M = mobility_of<WR>(__ldg(phi + (size_t)y * n + x), M0);
      const cpx<WR> g = Z[x];
      dsum += (double)M * ((double)g.x * g.x + (double)g.y * g.y);
      Z[x] = cscale(g, M);
    }
    __syncthreads();
    const cpx<WR>* Y = gfft<false>(Z, Z == A ? B : A, h.pl, tw);
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      cpx2<WR> o;
      split_at(Y, k, n, o.a, o.b);
      row[k] = o;
    }
    __syncthreads();
  }
  const double r = block_reduce<OpSum>(dsum, red);
  double* part = I.part + (size_t)6 * gridDim.x;
  if (threadIdx.x == 0) part[blockIdx.x] = r;
  const int tiles = gridDim.x;
  if (!arrive_last(&I.cnt[2], tiles, &lastflag)) return;
  const double d = reduce_partials<OpSum>(part, tiles, 1, 0.0, red);
  if (threadIdx.x == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) I.hist[s + 5 * (size_t)I.hist_ld] = d * I.dx * I.dx;
    I.cnt[2] = 0;
  }
}

// ---- column B: divergence, stabilised increment, S += increment ----------------------
template <typename SR, typename WR>
__global__ void __launch_bounds__(kThreads) kg_col_b(const InstDev* __restrict__ insts) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Head h;
  __shared__ double red[32];
  const InstDev& I = insts[blockIdx.y];
  setup(h, I);
  if (h.status) return;
  const int n = h.pl.n, K = n / 2 + 1;
  cpx<WR>* P0 = reinterpret_cast<cpx<WR>*>(smraw);
  cpx<WR>* P1 = P0 + n;
  cpx<WR>* P2 = P1 + n;
  const cpx2<WR>* Gp = reinterpret_cast<const cpx2<WR>*>(I.G);
  cpx<SR>* S = reinterpret_cast<cpx<SR>*>(I.S);
  const cpx<WR>* tw = reinterpret_cast<const cpx<WR>*>(I.tw_w);
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)n * I.dx);
  const double c1 = 2.0 * I.p.Q * I.p.kappa * I.dt;  // den = 1 + c1 k2^2
  const WR dtn = (WR)(I.dt / (double)n);
  for (int kx = blockIdx.x; kx < K; kx += gridDim.x) {
    const bool sc = selfconj(kx, n);
    const double kxf = kunit * (double)kx;
    const WR kxd = (2 * kx == n) ? (WR)0 : (WR)kxf;
    for (int y = threadIdx.x; y < n; y += blockDim.x) P0[y] = Gp[(size_t)y * K + kx].a;
    __syncthreads();
    cpx<WR>* Fx = gfft<false>(P0, P1, h.pl, tw);
    cpx<WR>* f1 = (Fx == P0) ? P1 : P0;
    for (int y = threadIdx.x; y < n; y += blockDim.x) f1[y] = Gp[(size_t)y * K + kx].b;
    __syncthreads();
    cpx<WR>* Fy = gfft<false>(f1, P2, h.pl, tw);
    for (int ky = threadIdx.x; ky < n; ky += blockDim.x) {
      const double kyf = kunit * (double)(2 * ky < n ? ky : ky - n);
      const double k2 = kxf * kxf + kyf * kyf;
      const WR iden = (WR)(1.0 / (1.0 + c1 * k2 * k2));
      const WR kyd = (2 * ky == n) ? (WR)0 : (WR)kyf;
      const cpx<WR> div = times_i(cscale(Fx[ky], kxd) + cscale(Fy[ky], kyd));
      Fx[ky] = cscale(div, iden * dtn);
    }
    __syncthreads();
    cpx<WR>* spare = (Fy == f1) ? P2 : f1;
    const cpx<WR>* inc = gfft<true>(Fx, spare, h.pl, tw);
    // exact mass conservation: the kx = 0 increments must sum to zero over y
    double corr = 0.0;
    if (kx == 0) {
      double colsum = 0.0;
      for (int y = threadIdx.x; y < n; y += blockDim.x) colsum += (double)inc[y].x;
      corr = block_reduce<OpSum>(colsum, red) / (double)n;
    }
    for (int y = threadIdx.x; y < n; y += blockDim.x) {
      cpx<SR>* sp = S + (size_t)y * K + kx;
      const cpx<SR> s0 = *sp;
      const cpx<WR> d = inc[y];
      *sp = mkc<SR>(s0.x + (SR)((double)d.x - corr), sc ? (SR)0 : s0.y + (SR)d.y);
    }
    __syncthreads();
  }
}

// ---- kernel sets ---------------------------------------------------------------------
// dynamic shared memory: three buffers of n complex state values
constexpr size_t smem_for(int nmax) { return (size_t)3 * nmax * 16; }

template <int NMAX, typename SR, typename WR>
struct GKS {
  static constexpr size_t SM = smem_for(NMAX);
  static cudaError_t prepare() {
    const int big = (int)smem_for(4096);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(kg_init<SR>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(kg_final<SR>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(kg_row_a<SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(kg_col_a<SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(kg_row_b<SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    return cudaFuncSetAttribute(kg_col_b<SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  }
  static cudaError_t no_prep() { return cudaSuccess; }
  static void no_tables(const void*, const void*, cudaStream_t) {}
  static void init(const InstDev* d, int count, cudaStream_t st) {
    kg_init<SR><<<dim3(kBlocks, count), kThreads, SM, st>>>(d);
  }
  static void fin(const InstDev* d, int count, cudaStream_t st) {
    kg_final<SR><<<dim3(kBlocks, count), kThreads, SM, st>>>(d);
  }
  static void row_a(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    kg_row_a<SR, WR><<<dim3(kBlocks, count), kThreads, SM, st>>>(d, base, s);
  }
  static void col_a(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    kg_col_a<SR, WR><<<dim3(kBlocks, count), kThreads, SM, st>>>(d, base, s);
  }
  static void row_b(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    kg_row_b<SR, WR><<<dim3(kBlocks, count), kThreads, SM, st>>>(d, base, s);
  }
  static void col_b(const InstDev* d, int count, cudaStream_t st) {
    kg_col_b<SR, WR><<<dim3(kBlocks, count), kThreads, SM, st>>>(d);
  }
  static KernelSet make(int n, int prec) {
    KernelSet k{};
    k.n = n;
    k.prec = prec;
    k.T = kThreads;
    k.E = 0;
    k.tiles_pairs = kBlocks;
    k.tiles_rows = kBlocks;
    k.tiles_cols = kBlocks;
    k.part_len = 7 * kBlocks;
    k.smem = SM;
    k.sr_bytes = sizeof(SR);
    k.wr_bytes = sizeof(WR);
    k.cplx_per_field = (size_t)(n / 2 + 1) * n;
    k.generic = true;
    k.prepare = &prepare;
    k.prepare_pipe = &no_prep;
    k.prepare_warp = &no_prep;
    k.fill_tables = &no_tables;
    k.init = &init;
    k.fin = &fin;
    k.row_a = &row_a;
    k.col_a = &col_a;
    k.row_b = &row_b;
    k.col_b = &col_b;
    k.E_alt = 0;  // no alternative column plan
    return k;
  }
};

}  // namespace gen
}  // namespace esc

namespace {

int largest_prime_factor(int n) {
  int p = 1, m = n;
  for (int f = 2; f * f <= m; ++f)
    while (m % f == 0) {
      p = f;
      m /= f;
    }
  return m > 1 ? (m > p ? m : p) : p;
}

}  // namespace

// Sizes the runtime-n kernels accept: 2 <= n <= 4096 with every prime factor at
// most 127, or any n up to 512 (a pass of radix r costs n r per transform).
int esc_generic_supported(int n) {
  if (n < 2 || n > 4096) return 0;
  return (largest_prime_factor(n) <= esc::gen::kMaxPrime || n <= 512) ? 1 : 0;
}

const esc::KernelSet* esc_generic_kernels(int n, int prec) {
  if (!esc_generic_supported(n)) return nullptr;
  static std::mutex mu;
  static std::map<std::pair<int, int>, esc::KernelSet> sets;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(n, prec);
  auto it = sets.find(key);
  if (it != sets.end()) return &it->second;
  esc::KernelSet k;
  const bool mixed = prec == esc::kMixed;
  if (n <= 64)
    k = mixed ? esc::gen::GKS<64, double, float>::make(n, prec) : esc::gen::GKS<64, double, double>::make(n, prec);
  else if (n <= 256)
    k = mixed ? esc::gen::GKS<256, double, float>::make(n, prec) : esc::gen::GKS<256, double, double>::make(n, prec);
  else if (n <= 1024)
    k = mixed ? esc::gen::GKS<1024, double, float>::make(n, prec)
              : esc::gen::GKS<1024, double, double>::make(n, prec);
  else
    k = mixed ? esc::gen::GKS<4096, double, float>::make(n, prec)
              : esc::gen::GKS<4096, double, double>::make(n, prec);
  return &sets.emplace(key, k).first->second;
}
