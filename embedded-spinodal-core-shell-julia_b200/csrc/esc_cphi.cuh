// Coupled c-phi model in 3-D: conserved composition c (Cahn-Hilliard) and an
// evolving order parameter phi (Allen-Cahn), FP64.  The step is that of the
// reference's 2023 3-D program (original/2023-3d/evolve.cu:86-186 with the
// kernels of original/2023-3d/EvoKernels.h):
//   local terms df/dc, df/dphi and M = mobility h(phi)        (EvoKernels.h:1-37)
//   mu^ = FFT(df/dc) + 2 kappa_c k^2 c^, mu = Re IFFT(mu^)/N   (EvoKernels.h:38-72)
//   div = sum_a D_a(M D_a mu), D_a the fourth-order periodic difference (EvoKernels.h:74-419)
//   c^' = (dt div^ + lhs c^)/lhs, lhs = 1 + 2 Q kappa_c k^4 dt;
//   phi^' = (phi^ - L dt FFT(df/dphi)) / (1 + 2 L kappa_phi k^2 dt)   (EvoKernels.h:432-470)
//   mass check on c^'(0), bounds -0.4 <= c <= 1.4, convergence max|dc| <= tol
//                                                              (evolve.cu:145-181)
// The z-gradient of mu uses dz (the reference passes dy, evolve.cu:124).
//
// Layout (the reference's): real fields a[k + nz (j + ny i)], z contiguous.
// Spectra are half spectra along z: K = nz/2 + 1 modes per (i, j) line, element
// (i, j, kz) at kz + K (j + ny i); the self-conjugate modes kz = 0 and nz/2 are
// kept real (the Re IFFT projection).  A 3-D transform is a z pass (two real
// lines packed into one complex FFT and split), a y pass and an x pass over
// strided lines (W adjacent kz lines per block, so every row of a tile is a
// contiguous segment).  Per step, twelve stages (the x passes launch one kernel per
// chain of transforms, so fourteen launches):
//   zf(local)  c, phi lines -> df/dc + i df/dphi -> z-FFT -> D1, D2 half spectra
//   y fwd      D1, D2
//   x spec 1   x-FFT D1 -> mu^ = D1 + 2 kappa_c k^2 C^ -> inverse x-FFT -> D1;
//              then x-FFT D2 -> Ph = (Ph - L dt D2)/(1 + 2 L kappa_phi k^2 dt)
//   y inv      D1
//   zi(mu)     D1 -> mu (two lines per complex inverse FFT) -> mu; fourth-order
//              z derivative, M, again -> div (the z part)
//   fd y, fd x div += D_a(M D_a mu) along y, then x (runtime-size line stencils)
//   zf(div)    div lines in pairs -> z-FFT -> D1
//   y fwd      D1
//   x spec 2   x-FFT D1 -> C^ = (dt div^ + lhs C^)/lhs (mass check at k = 0) ->
//              inverse x-FFT -> D1;  then Ph -> inverse x-FFT -> D2
//   y inv      D1, D2
//   zi(final)  c + i phi from D1, D2 -> c, phi; history row, bounds,
//              convergence and non-finite checks (last-arriver fold)
#pragma once
#include "esc_dispatch.cuh"

namespace esc {
namespace cphi {

// device status word: 0 running, else the stop reason
constexpr int kRunning = 0, kConverged = 1, kOutOfBounds = 2, kMassError = 3, kNonFinite = 4;
constexpr double kCLow = -0.4, kCHigh = 1.4;  // EvoKernels.h:499

struct Params {
  double A, B, chi, P, ca, cb1, cb2, A0, kappa_c, kappa_phi, mobility, relax, Q;
};

struct Dev {
  int nx, ny, nz, K;
  double dx, dy, dz, dt, tol, comperr;
  double invN;
  Params p;
  double *c, *phi, *mu, *div;      // real fields, nx*ny*nz
  double2 *Ch, *Ph, *D1, *D2;      // half spectra, nx*ny*K
  double* hist;                    // column-major (hist_ld x 6), rows after 0..steps steps
  int hist_ld;
  double* part;                    // block partials (6 per block)
  unsigned* cnt;                   // arrival counters [0] final fold, [1] stats fold
  double* scal;                    // [0] mean composition of the input (mass reference)
  int* status;
  long long* stop_step;
  const int* base;                 // steps completed before the current captured chunk
};

__device__ __forceinline__ double wavenumber3(int i, int n, double dk) {
  return dk * (double)(2 * i <= n ? i : i - n);  // the Nyquist kept positive (main.cu:146-158)
}

// df/dc and df/dphi of kernel_cphi_der (EvoKernels.h:19-33)
__device__ __forceinline__ void local_terms(double c, double ph, const Params& p, double& dfdc, double& dfdphi) {
  const double h = ph * ph * ph * (10.0 - 15.0 * ph + 6.0 * ph * ph);
  const double g = (ph * ph) * (1.0 - ph) * (1.0 - ph);
  const double hp = 30.0 * (ph * ph - 2.0 * ph * ph * ph + ph * ph * ph * ph);
  const double gp = 2.0 * ph - 6.0 * ph * ph + 4.0 * ph * ph * ph;
  dfdc = 2.0 * p.A * (1.0 - h) * (c - p.ca) + 2.0 * p.B * h * (c - p.cb1) * (c - p.cb2) * (2.0 * c - p.cb1 - p.cb2) -
         p.chi * p.P * g;
  dfdphi = -1.0 * hp * (p.A * (c - p.ca) * (c - p.ca) + p.A0) +
           hp * p.B * (c - p.cb1) * (c - p.cb1) * (c - p.cb2) * (c - p.cb2) + (1.0 - p.chi * c) * p.P * gp;
}
__device__ __forceinline__ double mobility3(double ph, double M0) {
  return ph * ph * ph * (10.0 - 15.0 * ph + 6.0 * ph * ph) * M0;
}

// fourth-order central difference (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2]) / (12 h)
template <typename V>
__device__ __forceinline__ V fd4(V p2, V p1, V m1, V m2, double inv12h) {
  return (-1.0 * p2 + 8.0 * p1 - 8.0 * m1 + m2) * inv12h;
}

// Hermitian completion of half spectra a, b (K = n/2 + 1 modes) at full index k,
// packed as a + i b; the self-conjugate modes are projected to their real parts
template <int N>
__device__ __forceinline__ cpx<double> merge_half(const double2* __restrict__ a, const double2* __restrict__ b, int k) {
  const bool up = 2 * k > N;
  const int idx = up ? N - k : k;
  double2 va = a[idx];
  double2 vb = b ? b[idx] : make_double2(0.0, 0.0);
  if (idx == 0 || 2 * idx == N) {
    va.y = 0.0;
    vb.y = 0.0;
  }
  if (up) {
    va.y = -va.y;
    vb.y = -vb.y;
  }
  return mkc<double>(va.x - vb.y, va.y + vb.x);
}

// ---- z passes: lines along the contiguous axis, one group of T threads per unit --------
enum ZMode { kZInit = 0, kZLocal = 1, kZDiv = 2 };

// A line of at most 32 threads lives inside one warp: its exchanges use the
// swizzled layout of the warp-independent 2-D row kernels and only __syncwarp;
// larger groups use the padded row layout and block barriers.
template <class P>
struct ZGeom {
  static constexpr int N = P::N, E = P::E, T = P::T, G = kBlock / T, K = N / 2 + 1;
  static constexpr bool kInWarp = T <= 32;
  using Sync = typename std::conditional<kInWarp, WarpSync, BlockSync>::type;
  using Lay = typename std::conditional<kInWarp, SwizzleLayout<N, sizeof(cpx<double>)>, RowLayout<N>>::type;
  static constexpr size_t smem() {
    return (size_t)G * (kInWarp ? N : RowLayout<N>::stride) * sizeof(cpx<double>);
  }
  // layout of group g of the block (its index inside the warp when lines share a warp)
  static __device__ __forceinline__ Lay layout(int g) {
    if constexpr (kInWarp) {
      return Lay{g * N, (int)((threadIdx.x & 31) / T)};
    } else {
      return Lay{g * RowLayout<N>::stride};
    }
  }
};

// resident 256-thread blocks per SM the coupled kernels are compiled for
template <class P>
constexpr int cphi_minb() {
  return P::E <= 8 ? 2 : 1;
}
// the kernels that hold one transform's values at a time (z forward, strided
// lines, final z inverse) fit 80 registers without spills at E <= 8: three blocks
template <class P>
constexpr int cphi_minb_light() {
  return P::E <= 8 ? 3 : 1;
}
// the z forward kernel fits 64 registers without spills at E <= 8: four blocks
template <class P>
constexpr int cphi_minb_zf() {
  return P::E <= 8 ? 4 : 1;
}

// forward z transforms.  kZInit: (c + i phi) of line q -> D1 = c^, D2 = phi^;
// kZLocal: (df/dc + i df/dphi) of line q -> D1, D2; kZDiv: div of lines 2q, 2q+1 -> D1.
template <class P>
__global__ void __launch_bounds__(kBlock, cphi_minb_zf<P>()) k3_zf(const Dev* __restrict__ dp, int mode) {
  using ZG = ZGeom<P>;
  constexpr int N = ZG::N, E = ZG::E, T = ZG::T, G = ZG::G, K = ZG::K;
  extern __shared__ __align__(16) unsigned char smraw[];
  const Dev& d = *dp;
  if (*(volatile const int*)d.status) return;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const long L = (long)d.nx * d.ny;
  const long units = mode == kZDiv ? (L + 1) / 2 : L;
  const long q = (long)blockIdx.x * G + g;
  const bool active = q < units;
  const long la = mode == kZDiv ? 2 * q : q;
  const bool hasb = mode != kZDiv || la + 1 < L;
  cpx<double> v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    double a = 0.0, b = 0.0;
    if (active) {
      if (mode == kZDiv) {
        a = d.div[la * N + x];
        b = hasb ? d.div[(la + 1) * N + x] : 0.0;
      } else {
        const double cv = d.c[la * N + x], pv = d.phi[la * N + x];
        if (mode == kZInit) {
          a = cv;
          b = pv;
        } else {
          local_terms(cv, pv, d.p, a, b);
        }
      }
    }
    v[m] = mkc<double>(a, b);
  }
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const auto lay = ZG::layout(g);
  fft<false, P, typename ZG::Sync>(v, t, sm, lay, PassTable<P, double>{});
#pragma unroll
  for (int m = 0; m < E; ++m) sm[lay(t + T * m)] = v[m];
  ZG::Sync::sync();
  double2* oa = d.D1 + la * K;
  double2* ob = mode == kZDiv ? d.D1 + (la + 1) * K : d.D2 + la * K;
  if (active) {
    for (int k = t; k < K; k += T) {
      const cpx<double> y1 = sm[lay(k)], y2 = cconj(sm[lay(k == 0 ? 0 : N - k)]);
      const cpx<double> xa = cscale(y1 + y2, 0.5), xb = cscale(times_negi(y1 - y2), 0.5);
      oa[k] = make_double2(xa.x, xa.y);
      if (hasb) ob[k] = make_double2(xb.x, xb.y);
    }
  }
}

// inverse z transform of mu^ (lines 2q, 2q+1 of D1 in one complex FFT), then the
// z part of div: D_z(M D_z mu) along the line; writes mu and div
template <class P>
__global__ void __launch_bounds__(kBlock, cphi_minb_light<P>()) k3_zi_mu(const Dev* __restrict__ dp) {
  using ZG = ZGeom<P>;
  constexpr int N = ZG::N, E = ZG::E, T = ZG::T, G = ZG::G, K = ZG::K;
  extern __shared__ __align__(16) unsigned char smraw[];
  const Dev& d = *dp;
  if (*(volatile const int*)d.status) return;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const long L = (long)d.nx * d.ny;
  const long q = (long)blockIdx.x * G + g;
  const bool active = q < (L + 1) / 2;
  const long la = 2 * q;
  const bool hasb = la + 1 < L;
  cpx<double> v[E];
#pragma unroll
  for (int m = 0; m < E; ++m)
    v[m] = active ? merge_half<N>(d.D1 + la * K, hasb ? d.D1 + (la + 1) * K : nullptr, t + T * m)
                  : mkc<double>(0.0, 0.0);
  if (active) {
    // phi is read after the transform: pull the pair's lines into L2 now (one
    // prefetch per 128-byte line, 16 doubles)
    const int count = (hasb ? 2 : 1) * N;
    for (int i = 16 * t; i < count; i += 16 * T) prefetch_l2(d.phi + la * N + i);
  }
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const auto lay = ZG::layout(g);
  fft<true, P, typename ZG::Sync>(v, t, sm, lay, PassTable<P, double>{});
  const double inv12 = 1.0 / (12.0 * d.dz);
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    v[m] = cscale(v[m], d.invN);
    sm[lay(x)] = v[m];
    if (active) {
      d.mu[la * N + x] = v[m].x;
      if (hasb) d.mu[(la + 1) * N + x] = v[m].y;
    }
  }
  ZG::Sync::sync();
  // q = M D_z mu at this thread's points (lane x: line a, lane y: line b)
  cpx<double> qv[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    const cpx<double> p2 = sm[lay((x + 2) % N)], p1 = sm[lay((x + 1) % N)];
    const cpx<double> m1 = sm[lay((x + N - 1) % N)], m2 = sm[lay((x + N - 2) % N)];
    const double dmx = fd4(p2.x, p1.x, m1.x, m2.x, inv12), dmy = fd4(p2.y, p1.y, m1.y, m2.y, inv12);
    double Ma = 0.0, Mb = 0.0;
    if (active) {
      Ma = mobility3(d.phi[la * N + x], d.p.mobility);
      Mb = hasb ? mobility3(d.phi[(la + 1) * N + x], d.p.mobility) : 0.0;
    }
    qv[m] = mkc<double>(Ma * dmx, Mb * dmy);
  }
  ZG::Sync::sync();
#pragma unroll
  for (int m = 0; m < E; ++m) sm[lay(t + T * m)] = qv[m];
  ZG::Sync::sync();
  if (!active) return;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    const cpx<double> p2 = sm[lay((x + 2) % N)], p1 = sm[lay((x + 1) % N)];
    const cpx<double> m1 = sm[lay((x + N - 1) % N)], m2 = sm[lay((x + N - 2) % N)];
    d.div[la * N + x] = fd4(p2.x, p1.x, m1.x, m2.x, inv12);
    if (hasb) d.div[(la + 1) * N + x] = fd4(p2.y, p1.y, m1.y, m2.y, inv12);
  }
}

// six partial values per block: sum c, sum phi, min c, max c, max |dc|, #non-finite
struct Six {
  double v[6];
};
__device__ __forceinline__ void six_warp(Six& s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s.v[0] += __shfl_xor_sync(0xffffffffu, s.v[0], o);
    s.v[1] += __shfl_xor_sync(0xffffffffu, s.v[1], o);
    s.v[2] = fmin(s.v[2], __shfl_xor_sync(0xffffffffu, s.v[2], o));
    s.v[3] = fmax(s.v[3], __shfl_xor_sync(0xffffffffu, s.v[3], o));
    s.v[4] = fmax(s.v[4], __shfl_xor_sync(0xffffffffu, s.v[4], o));
    s.v[5] += __shfl_xor_sync(0xffffffffu, s.v[5], o);
  }
}
__device__ __forceinline__ void six_join(Six& a, const Six& b) {
  a.v[0] += b.v[0];
  a.v[1] += b.v[1];
  a.v[2] = fmin(a.v[2], b.v[2]);
  a.v[3] = fmax(a.v[3], b.v[3]);
  a.v[4] = fmax(a.v[4], b.v[4]);
  a.v[5] += b.v[5];
}
__device__ __forceinline__ Six six_identity() {
  Six s;
  s.v[0] = 0.0;
  s.v[1] = 0.0;
  s.v[2] = INFINITY;
  s.v[3] = -INFINITY;
  s.v[4] = 0.0;
  s.v[5] = 0.0;
  return s;
}
// block reduction in a fixed order; the result is valid in thread 0
__device__ __forceinline__ Six six_block(Six s, Six* red) {
  six_warp(s);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = s;
  __syncthreads();
  Six r = six_identity();
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) six_join(r, red[w]);
  __syncthreads();
  return r;
}

// Folds the partials of every block once all have arrived; the last block's
// thread 0 gets the totals.  Returns true in that thread.
__device__ __forceinline__ bool six_fold(const Six& mine, double* part, unsigned* counter, Six* red, int* flag,
                                         Six& total) {
  if (threadIdx.x == 0)
    for (int i = 0; i < 6; ++i) part[(size_t)blockIdx.x * 6 + i] = mine.v[i];
  if (!arrive_last(counter, gridDim.x, flag)) return false;
  Six s = six_identity();
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    Six o;
#pragma unroll
    for (int i = 0; i < 6; ++i) o.v[i] = __ldcg(part + (size_t)b * 6 + i);
    six_join(s, o);
  }
  total = six_block(s, red);
  if (threadIdx.x == 0) *counter = 0;
  return threadIdx.x == 0;
}

// inverse z transform of (c^' + i phi^') per line -> c, phi; history row and stop checks
template <class P>
__global__ void __launch_bounds__(kBlock, cphi_minb_light<P>()) k3_zi_final(const Dev* __restrict__ dp, int s_local) {
  using ZG = ZGeom<P>;
  constexpr int N = ZG::N, E = ZG::E, T = ZG::T, G = ZG::G, K = ZG::K;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Six red[kBlock / 32];
  __shared__ int lastflag;
  const Dev& d = *dp;
  if (*(volatile const int*)d.status) return;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const long L = (long)d.nx * d.ny;
  const long l = (long)blockIdx.x * G + g;
  const bool active = l < L;
  // the previous c is loaded beside the spectra, before the transform: the stores
  // below go to the same addresses, and loads issued after them would each wait
  // for a full memory round trip in turn
  double* __restrict__ cp = d.c + l * N;
  double* __restrict__ pp = d.phi + l * N;
  cpx<double> v[E];
  double co[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    v[m] = active ? merge_half<N>(d.D1 + l * K, d.D2 + l * K, t + T * m) : mkc<double>(0.0, 0.0);
    co[m] = active ? cp[t + T * m] : 0.0;
  }
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const auto lay = ZG::layout(g);
  fft<true, P, typename ZG::Sync>(v, t, sm, lay, PassTable<P, double>{});
  Six s = six_identity();
  if (active) {
    int nbad = 0;
    const double invN = d.invN;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int o = t + T * m;
      const double cn = v[m].x * invN, pn = v[m].y * invN;
      const double co_ = co[m];
      cp[o] = cn;
      pp[o] = pn;
      s.v[0] += cn;
      s.v[1] += pn;
      s.v[2] = fmin(s.v[2], cn);
      s.v[3] = fmax(s.v[3], cn);
      s.v[4] = fmax(s.v[4], fabs(cn - co_));
      nbad += (int)(nonfinite_bits(cn) | nonfinite_bits(pn));
    }
    s.v[5] = (double)nbad;
  }
  const Six mine = six_block(s, red);
  Six tot;
  if (!six_fold(mine, d.part, &d.cnt[0], red, &lastflag, tot)) return;
  const int row = *d.base + s_local + 1;
  const double Nn = (double)L * N;
  if (d.hist) {
    const size_t ld = (size_t)d.hist_ld;
    d.hist[row] = (double)row * d.dt;
    d.hist[row + ld] = tot.v[0] / Nn;
    d.hist[row + 2 * ld] = tot.v[1] / Nn;
    d.hist[row + 3 * ld] = tot.v[2];
    d.hist[row + 4 * ld] = tot.v[3];
    d.hist[row + 5 * ld] = tot.v[4];
  }
  int st = kRunning;
  if (tot.v[5] > 0.0)
    st = kNonFinite;
  else if (tot.v[2] < kCLow || tot.v[3] > kCHigh)
    st = kOutOfBounds;
  else if (tot.v[4] <= d.tol)
    st = kConverged;
  if (st != kRunning) {
    *d.stop_step = row;
    *d.status = st;
  }
}

// ---- strided passes: lines along y or x, W adjacent kz lines per block ------------------
template <class P>
struct LGeom {
  static constexpr int N = P::N, E = P::E, T = P::T, W = kBlock / T;
  static size_t smem() { return ((size_t)host_smpad(N * W - 1) + 1) * sizeof(cpx<double>); }
};

// in-place transforms of na (1 or 2) arrays along a strided axis: element p of
// line (o, kz) at o*ostride + kz + p*estride
template <class P, bool INV>
__global__ void __launch_bounds__(kBlock, cphi_minb_light<P>()) k3_line(const Dev* __restrict__ dp, double2* a0, double2* a1, int na,
                                                  long estride, long ostride) {
  using LG = LGeom<P>;
  constexpr int E = LG::E, T = LG::T, W = LG::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  const Dev& d = *dp;
  if (*(volatile const int*)d.status) return;
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kz = blockIdx.x * W + w;
  const bool active = kz < d.K;
  const long base = (long)blockIdx.y * ostride + kz;
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const ColLayout<W> lay{w};
  for (int a = 0; a < na; ++a) {
    double2* arr = a ? a1 : a0;
    cpx<double> v[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const double2 x = active ? arr[base + (long)(t + T * m) * estride] : make_double2(0.0, 0.0);
      v[m] = mkc<double>(x.x, x.y);
    }
    fft<INV, P>(v, t, sm, lay, PassTable<P, double>{});
    if (active) {
#pragma unroll
      for (int m = 0; m < E; ++m) arr[base + (long)(t + T * m) * estride] = make_double2(v[m].x, v[m].y);
    }
  }
}

// x pass with the spectral operations (lines (j, kz), element kx; o = j = blockIdx.y).
// A step's two x passes (kXMu, kXUpdate) each launch two kernels, one per chain of
// transforms (composition, order parameter): a kernel holds one line's values at a
// time, which fits three blocks per SM (two for the mu chain, which would spill).
enum XOp { kXInit = 0, kXMu = 1, kXUpdate = 2 };
enum XKernel { kXKInit = 0, kXKMu = 1, kXKPhi = 2, kXKUpdC = 3, kXKPhiInv = 4 };

template <class P, int OP>
__global__ void __launch_bounds__(kBlock, OP == kXKMu ? cphi_minb<P>() : cphi_minb_light<P>()) k3_xspec(const Dev* __restrict__ dp, int s_local) {
  using LG = LGeom<P>;
  constexpr int N = LG::N, E = LG::E, T = LG::T, W = LG::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  const Dev& d = *dp;
  if (*(volatile const int*)d.status) return;
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kz = blockIdx.x * W + w;
  const int j = blockIdx.y;
  const bool active = kz < d.K;
  const long estride = (long)d.ny * d.K;
  const long base = (long)j * d.K + kz;
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const ColLayout<W> lay{w};
  const double dkx = 2.0 * 3.14159265358979323846 / ((double)N * d.dx);
  const double dky = 2.0 * 3.14159265358979323846 / ((double)d.ny * d.dy);
  const double dkz = 2.0 * 3.14159265358979323846 / ((double)d.nz * d.dz);
  const double kyz2 = [&] {
    const double ky = wavenumber3(j, d.ny, dky), kzv = wavenumber3(kz, d.nz, dkz);
    return ky * ky + kzv * kzv;
  }();
  auto k2_at = [&](int p) {
    const double kx = wavenumber3(p, N, dkx);
    return kx * kx + kyz2;
  };
  auto load = [&](const double2* arr, cpx<double>(&v)[E]) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const double2 x = active ? arr[base + (long)(t + T * m) * estride] : make_double2(0.0, 0.0);
      v[m] = mkc<double>(x.x, x.y);
    }
  };
  auto store = [&](double2* arr, const cpx<double>(&v)[E]) {
    if (!active) return;
#pragma unroll
    for (int m = 0; m < E; ++m) arr[base + (long)(t + T * m) * estride] = make_double2(v[m].x, v[m].y);
  };
  // L2 prefetch of the tile rows of an array read after a transform (one 128-byte
  // line per 8 complex values of a row)
  auto prefetch = [&](const double2* arr) {
    if (active && (w & 7) == 0) {
#pragma unroll
      for (int m = 0; m < E; ++m) prefetch_l2(arr + base + (long)(t + T * m) * estride);
    }
  };
  cpx<double> v[E];
  if (OP == kXKInit) {
    load(d.D1, v);
    fft<false, P>(v, t, sm, lay, PassTable<P, double>{});
    store(d.Ch, v);
    load(d.D2, v);
    fft<false, P>(v, t, sm, lay, PassTable<P, double>{});
    store(d.Ph, v);
  } else if (OP == kXKMu) {
    // mu^ = FFT(df/dc) + 2 kappa_c k^2 c^ (Compute_mu), back along x
    load(d.D1, v);
    prefetch(d.Ch);
    fft<false, P>(v, t, sm, lay, PassTable<P, double>{});
    const double kc2 = 2.0 * d.p.kappa_c;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int p = t + T * m;
      const double2 ch = active ? d.Ch[base + (long)p * estride] : make_double2(0.0, 0.0);
      const double f = kc2 * k2_at(p);
      v[m] = mkc<double>(v[m].x + f * ch.x, v[m].y + f * ch.y);
    }
    fft<true, P>(v, t, sm, lay, PassTable<P, double>{});
    store(d.D1, v);
  } else if (OP == kXKPhi) {
    // phi^' = (phi^ - L dt FFT(df/dphi)) / (1 + 2 L kappa_phi k^2 dt)
    load(d.D2, v);
    prefetch(d.Ph);
    fft<false, P>(v, t, sm, lay, PassTable<P, double>{});
    const double Ldt = d.p.relax * d.dt, c2 = 2.0 * d.p.relax * d.p.kappa_phi * d.dt;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int p = t + T * m;
      const double2 ph = active ? d.Ph[base + (long)p * estride] : make_double2(0.0, 0.0);
      const double lhse = 1.0 + c2 * k2_at(p);
      v[m] = mkc<double>((ph.x - Ldt * v[m].x) / lhse, (ph.y - Ldt * v[m].y) / lhse);
    }
    store(d.Ph, v);
  } else if (OP == kXKUpdC) {
    // c^' = (dt div^ + lhs c^) / lhs, lhs = 1 + 2 Q kappa_c k^4 dt (kernel_comp_phi)
    load(d.D1, v);
    prefetch(d.Ch);
    fft<false, P>(v, t, sm, lay, PassTable<P, double>{});
    const double c1 = 2.0 * d.p.Q * d.p.kappa_c * d.dt;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int p = t + T * m;
      const double2 ch = active ? d.Ch[base + (long)p * estride] : make_double2(0.0, 0.0);
      const double k2 = k2_at(p);
      const double lhs = 1.0 + c1 * k2 * k2;
      v[m] = mkc<double>((d.dt * v[m].x + lhs * ch.x) / lhs, (d.dt * v[m].y + lhs * ch.y) / lhs);
    }
    if (t == 0 && j == 0 && kz == 0) {
      // mass check on the k = 0 mode, held by slot m = 0 of thread 0 (evolve.cu:145-155)
      const double err = fabs(v[0].x * d.invN - d.scal[0]);
      if (!(err <= d.comperr)) {
        *d.stop_step = *d.base + s_local;
        *d.status = kMassError;
      }
    }
    store(d.Ch, v);
    fft<true, P>(v, t, sm, lay, PassTable<P, double>{});
    store(d.D1, v);
  } else {
    // phi^' back along x
    load(d.Ph, v);
    fft<true, P>(v, t, sm, lay, PassTable<P, double>{});
    store(d.D2, v);
  }
}

// ---- per-size kernel set ------------------------------------------------------------------
// The plans of the coupled kernels are a type of their own.  Kernel and __device__
// variable templates keyed on a plan (the pass-major twiddle table g_pass_tw<P, double>
// and its fill kernel k_fill_pass_tw<P, double>) would otherwise be instantiated both
// here and in the 2-D kernel units of the same size: such instances share one host
// stub, so a launch from one unit could run (and fill the table of) the other unit's
// module, leaving this unit's table unfilled.
template <class Base>
struct CphiPlan : Base {};
// FP64 plans of at most 12 elements per thread: 128 and 256 take the eight-element
// plans (4 4 8 and 4 8 8), whose transforms and twiddle powers fit two 256-thread
// blocks per SM; the other sizes keep their FP64 plan (E <= 12 from 96 up).
template <int N>
struct CphiPlanOf {
  using type = CphiPlan<typename Plan64<N>::type>;
};
template <>
struct CphiPlanOf<128> {
  using type = CphiPlan<Plan<128, 8, Radices<4, 4, 8>>>;
};
template <>
struct CphiPlanOf<256> {
  using type = CphiPlan<Plan<256, 8, Radices<4, 8, 8>>>;
};

struct Set {
  int n;
  size_t zsmem, lsmem;
  int zG, lW;  // z units per block, strided lines per block
  void (*fill_tables)(const void* tw, cudaStream_t);
  cudaError_t (*prepare)();
  void (*zf)(const Dev*, int mode, int blocks, cudaStream_t);
  void (*zi_mu)(const Dev*, int blocks, cudaStream_t);
  void (*zi_final)(const Dev*, int s_local, int blocks, cudaStream_t);
  void (*line)(const Dev*, bool inv, double2* a0, double2* a1, int na, long estride, long ostride, dim3 grid,
               cudaStream_t);
  void (*xspec)(const Dev*, int op, int s_local, dim3 grid, cudaStream_t);
};

template <int N>
struct SetOf {
  using P = typename CphiPlanOf<N>::type;
  using ZG = ZGeom<P>;
  using LG = LGeom<P>;
  static void fill_tables(const void* tw, cudaStream_t st) {
    k_fill_pass_tw<P, double><<<1, 256, 0, st>>>(reinterpret_cast<const cpx<double>*>(tw));
  }
  static cudaError_t prepare() {
    const int zs = (int)ZG::smem(), ls = (int)LG::smem();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k3_zf<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs))) return e;
    if ((e = cudaFuncSetAttribute(k3_zi_mu<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs))) return e;
    if ((e = cudaFuncSetAttribute(k3_zi_final<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs))) return e;
    if ((e = cudaFuncSetAttribute(k3_line<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k3_line<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k3_xspec<P, kXKInit>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k3_xspec<P, kXKMu>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k3_xspec<P, kXKPhi>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k3_xspec<P, kXKUpdC>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls))) return e;
    if ((e = cudaFuncSetAttribute(k3_xspec<P, kXKPhiInv>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls)))
      return e;
    return cudaSuccess;
  }
  static void zf(const Dev* d, int mode, int blocks, cudaStream_t st) {
    k3_zf<P><<<blocks, kBlock, ZG::smem(), st>>>(d, mode);
  }
  static void zi_mu(const Dev* d, int blocks, cudaStream_t st) { k3_zi_mu<P><<<blocks, kBlock, ZG::smem(), st>>>(d); }
  static void zi_final(const Dev* d, int s_local, int blocks, cudaStream_t st) {
    k3_zi_final<P><<<blocks, kBlock, ZG::smem(), st>>>(d, s_local);
  }
  static void line(const Dev* d, bool inv, double2* a0, double2* a1, int na, long es, long os, dim3 grid,
                   cudaStream_t st) {
    if (inv)
      k3_line<P, true><<<grid, kBlock, LG::smem(), st>>>(d, a0, a1, na, es, os);
    else
      k3_line<P, false><<<grid, kBlock, LG::smem(), st>>>(d, a0, a1, na, es, os);
  }
  static void xspec(const Dev* d, int op, int s_local, dim3 grid, cudaStream_t st) {
    if (op == kXInit) {
      k3_xspec<P, kXKInit><<<grid, kBlock, LG::smem(), st>>>(d, s_local);
    } else if (op == kXMu) {
      k3_xspec<P, kXKMu><<<grid, kBlock, LG::smem(), st>>>(d, s_local);
      k3_xspec<P, kXKPhi><<<grid, kBlock, LG::smem(), st>>>(d, s_local);
    } else {
      k3_xspec<P, kXKUpdC><<<grid, kBlock, LG::smem(), st>>>(d, s_local);
      k3_xspec<P, kXKPhiInv><<<grid, kBlock, LG::smem(), st>>>(d, s_local);
    }
  }
  static Set make() {
    Set s;
    s.n = N;
    s.zsmem = ZG::smem();
    s.lsmem = LG::smem();
    s.zG = ZG::G;
    s.lW = LG::W;
    s.fill_tables = &fill_tables;
    s.prepare = &prepare;
    s.zf = &zf;
    s.zi_mu = &zi_mu;
    s.zi_final = &zi_final;
    s.line = &line;
    s.xspec = &xspec;
    return s;
  }
};

}  // namespace cphi
}  // namespace esc

#define ESC_CPHI_DEFINE_SIZE(n) \
  const esc::cphi::Set* esc_cphi_set_##n() { \
    static const esc::cphi::Set s = esc::cphi::SetOf<n>::make(); \
    return &s; \
  }

#define ESC_CPHI_SIZES(X) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
