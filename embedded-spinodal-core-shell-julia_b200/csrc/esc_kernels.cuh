// Fused phase kernels of one stabilised semi-implicit Fourier step of the
// fixed-particle Cahn-Hilliard model (reference core_shell.jl:45-82).
//
// Field layout in HBM (per instance, n x n grid, n even):
//   phi  : real n*n, row y contiguous in x            (the Julia column-major matrix)
//   S    : state, the x-transform of c in the mixed (kx, y) domain,
//          H = n/2 complex values per row y, element (y, kx) at y*H + kx.
//          Slot kx = 0 packs the two real modes: (DC, Nyquist) = (X(0,y), X(n/2,y)).
//   F    : x-transform of f'(c), same packing                       [row A -> col A]
//   G    : pair array (two complex per (y,kx)): x-transforms of
//          (d mu/dx, d mu/dy) written by col A, overwritten in place by
//          row B with the x-transforms of (M d mu/dx, M d mu/dy)     [-> col B]
//
// One time step = four launches:
//   row A : S -> inverse x-FFT -> c ; f'(c), f(c), sum/min/max(c) ; forward x-FFT(f') -> F
//   col A : y-FFT(S) = c^, y-FFT(F) ; kappa sum k^2|c^|^2 ; mu^ ; i k mu^ ; inverse y-FFT -> G
//   row B : inverse x-FFT(G) -> grad mu ; M = M0 h(phi) ; sum M|grad mu|^2 ; forward x-FFT -> G
//   col B : y-FFT(G) ; div^ ; dt div^/(1+2 Q kappa k^4 dt) ; inverse y-FFT ; S += increment
// Precision: SR is the state/reduction type, WR the work type of the f', mu and
// flux transforms (double/double for the FP64 drop-in, double/float for the
// mixed mode).
#pragma once
#include "esc_fft.cuh"

#include <type_traits>

namespace esc {

constexpr int kBlock = 256;

// the mixed precision: FP64 state transforms, FP32 flux transforms (packed in pairs where two run side by side)
template <typename SR, typename WR>
constexpr bool kSplitMixed = std::is_same<SR, double>::value && std::is_same<WR, float>::value;

template <typename R>
struct __align__(4 * sizeof(R)) cpx2 {
  cpx<R> a, b;
};

struct ModelParams {
  double A, B, chi, P, ca, cb, cc, kappa, mobility, Q;
};

// Per-instance descriptor (device resident).  Partial-sum layout in `part`:
//   [0, 5*tiles_row_pairs)                  row A: sum c, min c, max c, sum f, #non-finite
//   [5*tiles_row_pairs, +tiles_col)         col A: sum k^2 |c^|^2 (with Hermitian weights)
//   [.. , +tiles_rows)                      row B: sum M |grad mu|^2
struct InstDev {
  int n;
  int hist_ld;        // rows of the history matrix (steps + 1)
  double dx, dt;
  ModelParams p;
  void* S;
  void* F;
  void* G;
  const void* phi;
  double* hist;       // column-major (hist_ld x 6), may be null (no history)
  double* part;
  unsigned* cnt;      // 4 arrival counters
  double* scal;       // [0] sum f of the current step
  int* status;        // 0 ok, 1 non-finite composition
  long long* bad_step;
  const void* tw_s;   // twiddles e^{-2 pi i j/n} in SR
  const void* tw_w;   // same in WR
  double* cio;        // real FP64 field for init/final (n*n)
  int drop_first_copy; // test knob (ESC_PIPE_DROP_COPY): the TMA pipeline kernels skip their
                       // first copy and their bounded wait for it runs out (ESC_ETIMEOUT)
};

// ---- reductions --------------------------------------------------------------
struct OpSum {
  static __device__ __forceinline__ double ap(double a, double b) { return a + b; }
  static __device__ __forceinline__ double identity() { return 0.0; }
};
struct OpMin {
  static __device__ __forceinline__ double ap(double a, double b) { return fmin(a, b); }
  static __device__ __forceinline__ double identity() { return INFINITY; }
};
struct OpMax {
  static __device__ __forceinline__ double ap(double a, double b) { return fmax(a, b); }
  static __device__ __forceinline__ double identity() { return -INFINITY; }
};

// Fixed-order block reduction (deterministic): warp butterflies then one warp.
template <class Op>
__device__ __forceinline__ double block_reduce(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = Op::ap(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : Op::identity();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = Op::ap(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  __syncthreads();
  if (threadIdx.x == 0) red[0] = v;
  __syncthreads();
  v = red[0];
  __syncthreads();
  return v;
}

// Publish this block's partials; returns true in every thread of the block
// that arrived last.  Partials of all blocks are then readable with __ldcg.
__device__ __forceinline__ bool arrive_last(unsigned* counter, unsigned nblocks, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    *flag = (prev == nblocks - 1) ? 1 : 0;
  }
  __syncthreads();
  const bool last = *flag != 0;
  if (last) __threadfence();
  return last;
}

// Deterministic reduction of `count` partials spaced `stride` apart.
template <class Op>
__device__ __forceinline__ double reduce_partials(const double* p, int count, int stride, double init,
                                                  double* red) {
  double v = init;
  for (int i = threadIdx.x; i < count; i += blockDim.x) v = Op::ap(v, __ldcg(p + (size_t)i * stride));
  return block_reduce<Op>(v, red);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Warp-level arrival: returns true (in every lane) in the warp that arrives
// last among `total` arrivals; its earlier partial writes are then visible.
__device__ __forceinline__ bool warp_arrive_last(unsigned* counter, unsigned total) {
  unsigned last = 0;
  if ((threadIdx.x & 31) == 0) {
    __threadfence();
    last = (atomicAdd(counter, 1u) == total - 1) ? 1u : 0u;
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (last) __threadfence();
  return last != 0;
}

// deterministic warp fold of `count` partials spaced `stride` apart.  The fold
// runs in the last warp of an instance, and the last instance's fold ends the
// launch, so its loads are unrolled to keep several in flight; each lane still
// accumulates in increasing slot order.
template <class Op>
__device__ __forceinline__ double warp_fold(const double* p, int count, int stride, double init) {
  double v = init;
#pragma unroll 8
  for (int i = (threadIdx.x & 31); i < count; i += 32) v = Op::ap(v, __ldcg(p + (size_t)i * stride));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = Op::ap(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---- helpers -----------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R wavenumber(int i, int n, double kunit) {
  return (R)(kunit * (double)(i < n / 2 ? i : i - n));
}

// Full-spectrum value Z(k) = Xa(k) + i Xb(k) of two real rows from their packed
// half-spectra a[0..H), b[0..H).
template <typename R, int N>
__device__ __forceinline__ cpx<R> load_pair_spectrum(const cpx<R>* __restrict__ a, const cpx<R>* __restrict__ b,
                                                     int k) {
  constexpr int H = N / 2;
  int idx = k <= H ? k : N - k;
  if (idx == H) idx = 0;
  const cpx<R> va = ldc(a + idx), vb = ldc(b + idx);
  if (k == 0) return mkc<R>(va.x, vb.x);
  if (k == H) return mkc<R>(va.y, vb.y);
  if (k < H) return mkc<R>(va.x - vb.y, va.y + vb.x);
  return mkc<R>(va.x + vb.y, vb.x - va.y);
}

// pair-array variant (a = component 0, b = component 1 of row y)
template <typename R, int N>
__device__ __forceinline__ cpx<R> load_pair_spectrum2(const cpx2<R>* __restrict__ row, int k) {
  constexpr int H = N / 2;
  int idx = k <= H ? k : N - k;
  if (idx == H) idx = 0;
  const cpx2<R> v = row[idx];
  const cpx<R> va = v.a, vb = v.b;
  if (k == 0) return mkc<R>(va.x, vb.x);
  if (k == H) return mkc<R>(va.y, vb.y);
  if (k < H) return mkc<R>(va.x - vb.y, va.y + vb.x);
  return mkc<R>(va.x + vb.y, vb.x - va.y);
}

// Given the forward DFT Y of (a + i b) at positions t + T m (registers), split it
// into the packed half-spectra of the real rows a and b: returns, for output
// index k = t + T*m (m < E/2), Xa(k) and Xb(k).  Uses the row-layout exchange.
template <class P, typename R>
__device__ __forceinline__ void split_pair(const cpx<R> (&y)[P::E], int t, cpx<R>* sm, const RowLayout<P::N>& lay,
                                           cpx<R> (&xa)[P::E / 2], cpx<R> (&xb)[P::E / 2]) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2;
#pragma unroll
  for (int m = 0; m < E; ++m) sm[lay(t + T * m)] = y[m];
  __syncthreads();
#pragma unroll
  for (int m = 0; m < E / 2; ++m) {
    const int k = t + T * m;
    const cpx<R> y1 = sm[lay(k)];
    if (k == 0) {
      const cpx<R> yh = sm[lay(H)];
      xa[m] = mkc<R>(y1.x, yh.x);
      xb[m] = mkc<R>(y1.y, yh.y);
    } else {
      const cpx<R> y2 = cconj(sm[lay(N - k)]);
      xa[m] = cscale(y1 + y2, (R)0.5);
      xb[m] = cscale(times_negi(y1 - y2), (R)0.5);
    }
  }
  __syncthreads();
}

template <typename SR>
__device__ __forceinline__ void bulk(SR c, SR phi, const ModelParams& p, SR& fprime, SR& fbulk) {
  const SR h = phi * phi * phi * ((SR)10 - (SR)15 * phi + (SR)6 * phi * phi);
  const SR g = phi * phi * ((SR)1 - phi) * ((SR)1 - phi);
  const SR A = (SR)p.A, B = (SR)p.B, chi = (SR)p.chi, P = (SR)p.P;
  const SR ca = (SR)p.ca, cb = (SR)p.cb, cc = (SR)p.cc;
  const SR d_a = c - ca, d_b = c - cb, d_c = c - cc;
  fprime = (SR)2 * A * ((SR)1 - h) * d_a + (SR)2 * B * h * d_b * d_c * ((SR)2 * c - cb - cc) - chi * P * g;
  fbulk = A * ((SR)1 - h) * d_a * d_a + B * h * d_b * d_b * d_c * d_c + P * ((SR)1 - chi * c) * g;
}

// Bulk terms of the mixed precision for two points at once (rows a and b of a
// row pair, one packed lane each).  c arrives in FP64; f'(c) and f(c) are
// evaluated in FP32 at c_hi = fl32(c) and corrected to first order in
// c_lo = fl32(c - c_hi), the part of c below FP32 resolution:
//   f'(c) = f'(c_hi) + f''(c_hi) c_lo,   f(c) = f(c_hi) + f'(c_hi) c_lo.
// The neglected terms are O(c_lo^2) ~ 1e-15 relative.  Same formulas as `bulk`
// (core_shell.jl:45-55), with f'' = 2A(1-h) + 2Bh((c-cc)e + (c-cb)e + 2(c-cb)(c-cc)),
// e = 2c - cb - cc.
__device__ __forceinline__ void bulk_pair_split(double ca, double cb, float pa, float pb, const ModelParams& p,
                                                f2& fprime, f2& fbulk) {
  const f2 hi(__double2float_rn(ca), __double2float_rn(cb));
  const f2 lo(__double2float_rn(ca - (double)hi.v.x), __double2float_rn(cb - (double)hi.v.y));
  const f2 ph(pa, pb);
  const f2 p2 = ph * ph;
  const f2 h = p2 * ph * fma(ph, fma(ph, f2(6.0), f2(-15.0)), f2(10.0));
  const f2 q = ph - p2;
  const f2 g = q * q;
  const f2 Ah = f2(p.A) * (f2(1.0) - h);
  const f2 Bh = f2(p.B) * h;
  const f2 da = hi - f2(p.ca), db = hi - f2(p.cb), dc = hi - f2(p.cc);
  const f2 e = hi + hi - f2(p.cb + p.cc);
  const f2 dbdc = db * dc;
  const f2 fp = fma(f2(2.0) * Ah, da, fma(f2(2.0) * Bh * dbdc, e, f2(-p.chi * p.P) * g));
  const f2 fpp = fma(f2(2.0), Ah, f2(2.0) * Bh * fma(dc + db, e, f2(2.0) * dbdc));
  const f2 fv = fma(Ah * da, da, fma(Bh * dbdc, dbdc, f2(p.P) * fma(f2(-p.chi), hi, f2(1.0)) * g));
  fprime = fma(fpp, lo, fp);
  fbulk = fma(fp, lo, fv);
}

// true when x is +-Inf or NaN (exponent bits all set), by integer test
__device__ __forceinline__ bool nonfinite_bits(double x) {
  return (__double2hiint(x) & 0x7ff00000) == 0x7ff00000;
}

// L1 prefetch of `bytes` bytes from `p` (128-byte lines), lines split over `nthr` threads
__device__ __forceinline__ void prefetch_l1(const void* p, int bytes, int t, int nthr) {
  const char* c = static_cast<const char*>(p);
  for (int l = t; l * 128 < bytes; l += nthr) asm volatile("prefetch.global.L1 [%0];" ::"l"(c + 128 * l));
}

// L2 prefetch of the 128-byte line holding `p`
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <typename R>
__device__ __forceinline__ R mobility_of(R phi, R M0) {
  return M0 * (phi * phi * phi * ((R)10 - (R)15 * phi + (R)6 * phi * phi));
}

__device__ __forceinline__ int step_index(const int* base, int s_local) { return *base + s_local; }

// ---- kernels -----------------------------------------------------------------
// Row tiles: G = kBlock / T groups per block; thread (t, g) with t fastest.
template <class P>
struct RowGeom {
  static constexpr int T = P::T;
  static constexpr int G = kBlock / T;
  static_assert(kBlock % T == 0, "block must hold whole FFT groups");
};
template <class P>
struct ColGeom {
  static constexpr int T = P::T;
  static constexpr int W = kBlock / T;
};
// Resident blocks per SM the column kernels are compiled for: the mixed
// precision's transforms fit 3 blocks at up to 8 elements per thread and 2 at
// up to 16; the FP64 drop-in fits 2 at up to 8; larger plans keep the
// compiler's choice.
// Block size of the forward column kernels: 256 threads, or, in the mixed
// precision, two columns for plans of 256 threads per column (n = 4096), where
// one column per block reads 16-byte halves of 32-byte sectors.  (The FP64
// transforms need more than the 128 registers a 512-thread block leaves.)
template <class P, typename SR, typename WR>
constexpr int col_block() {
  return (kSplitMixed<SR, WR> && P::T >= 256) ? 2 * P::T : kBlock;
}
template <class P, typename SR, typename WR>
struct ColGeomF {
  static constexpr int B = col_block<P, SR, WR>();
  static constexpr int W = B / P::T;
};
template <class P, typename SR, typename WR>
constexpr int col_min_blocks() {
  constexpr int b256 = kSplitMixed<SR, WR> ? (P::E <= 8 ? 3 : (P::E <= 16 ? 2 : 1)) : (P::E <= 8 ? 2 : 1);
  return b256 * kBlock / col_block<P, SR, WR>() > 1 ? b256 * kBlock / col_block<P, SR, WR>() : 1;
}

// init: c (FP64 real) -> S (packed x-transform), one row pair per group
template <class P, typename SR>
__global__ void __launch_bounds__(kBlock) k_init(const InstDev* __restrict__ insts) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<SR>* sm = reinterpret_cast<cpx<SR>*>(smraw);
  const InstDev& I = insts[blockIdx.y];
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;
  const RowLayout<N> lay{g * RowLayout<N>::stride};
  cpx<SR> v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    v[m] = active ? mkc<SR>((SR)I.cio[(size_t)ya * N + x], (SR)I.cio[(size_t)(ya + 1) * N + x])
                  : mkc<SR>(0, 0);
  }
  fft<false, P>(v, t, sm, lay, reinterpret_cast<const cpx<SR>*>(I.tw_s));
  cpx<SR> xa[E / 2], xb[E / 2];
  split_pair<P>(v, t, sm, lay, xa, xb);
  if (active) {
    cpx<SR>* S = reinterpret_cast<cpx<SR>*>(I.S);
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      S[(size_t)ya * H + t + T * m] = xa[m];
      S[(size_t)(ya + 1) * H + t + T * m] = xb[m];
    }
  }
}

// final: S -> c (FP64 real)
template <class P, typename SR>
__global__ void __launch_bounds__(kBlock) k_final(const InstDev* __restrict__ insts) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<SR>* sm = reinterpret_cast<cpx<SR>*>(smraw);
  const InstDev& I = insts[blockIdx.y];
  // an instance stopped on a non-finite field keeps its input c (block-uniform)
  if (*(volatile const int*)I.status) return;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;
  const RowLayout<N> lay{g * RowLayout<N>::stride};
  const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
  cpx<SR> v[E];
#pragma unroll
  for (int m = 0; m < E; ++m)
    v[m] = active ? load_pair_spectrum<SR, N>(S + (size_t)ya * H, S + (size_t)(ya + 1) * H, t + T * m)
                  : mkc<SR>(0, 0);
  fft<true, P>(v, t, sm, lay, reinterpret_cast<const cpx<SR>*>(I.tw_s));
  if (active) {
    const double inv = 1.0 / N;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int x = t + T * m;
      I.cio[(size_t)ya * N + x] = (double)v[m].x * inv;
      I.cio[(size_t)(ya + 1) * N + x] = (double)v[m].y * inv;
    }
  }
}

// row A: c from S, bulk terms, reductions for history columns 1,3,4 (and sum f), F = x-FFT(f')
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(kBlock) k_row_a(const InstDev* __restrict__ insts, const int* __restrict__ base,
                                                  int s_local) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32];
  __shared__ int lastflag;
  const InstDev& I = insts[blockIdx.y];
  if (*I.status) return;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;
  const RowLayout<N> lay{g * RowLayout<N>::stride};

  cpx<SR> v[E];
  {
    const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
#pragma unroll
    for (int m = 0; m < E; ++m)
      v[m] = active ? load_pair_spectrum<SR, N>(S + (size_t)ya * H, S + (size_t)(ya + 1) * H, t + T * m)
                    : mkc<SR>(0, 0);
  }
  fft<true, P>(v, t, reinterpret_cast<cpx<SR>*>(smraw), lay, reinterpret_cast<const cpx<SR>*>(I.tw_s));

  const ModelParams mp = I.p;
  const SR invN = (SR)1 / (SR)N;
  const WR* phi = reinterpret_cast<const WR*>(I.phi);
  double sum_c = 0.0, sum_f = 0.0, mn = INFINITY, mx = -INFINITY, bad = 0.0;
  cpx<WR> w[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    SR fa = 0, fb = 0;
    if (active) {
      const SR ca = v[m].x * invN, cb = v[m].y * invN;
      const SR pa = (SR)__ldg(phi + (size_t)ya * N + x), pb = (SR)__ldg(phi + (size_t)(ya + 1) * N + x);
      SR ea, eb;
      bulk<SR>(ca, pa, mp, fa, ea);
      bulk<SR>(cb, pb, mp, fb, eb);
      sum_c += (double)ca + (double)cb;
      sum_f += (double)ea + (double)eb;
      mn = fmin(mn, fmin((double)ca, (double)cb));
      mx = fmax(mx, fmax((double)ca, (double)cb));
      bad += (isfinite((double)ca) ? 0.0 : 1.0) + (isfinite((double)cb) ? 0.0 : 1.0);
    }
    w[m] = mkc<WR>((WR)fa, (WR)fb);
  }
  cpx<WR>* smw = reinterpret_cast<cpx<WR>*>(smraw);
  fft<false, P>(w, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
  cpx<WR> xa[E / 2], xb[E / 2];
  split_pair<P>(w, t, smw, lay, xa, xb);
  if (active) {
    cpx<WR>* F = reinterpret_cast<cpx<WR>*>(I.F);
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      F[(size_t)ya * H + t + T * m] = xa[m];
      F[(size_t)(ya + 1) * H + t + T * m] = xb[m];
    }
  }
  // block partials
  const double r_sum = block_reduce<OpSum>(sum_c, red);
  const double r_min = block_reduce<OpMin>(mn, red);
  const double r_max = block_reduce<OpMax>(mx, red);
  const double r_f = block_reduce<OpSum>(sum_f, red);
  const double r_bad = block_reduce<OpSum>(bad, red);
  const int tiles = gridDim.x;
  if (threadIdx.x == 0) {
    double* pp = I.part + (size_t)blockIdx.x * 5;
    pp[0] = r_sum;
    pp[1] = r_min;
    pp[2] = r_max;
    pp[3] = r_f;
    pp[4] = r_bad;
  }
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
      I.hist[s + 1 * ld] = a_sum / ((double)N * N);
      I.hist[s + 3 * ld] = a_min;
      I.hist[s + 4 * ld] = a_max;
    }
    I.scal[0] = a_f;
    if (a_bad > 0.0) {
      *I.bad_step = s;
      *I.status = 1;
    }
    I.cnt[0] = 0;
  }
}

// col A: y-FFT of S and F, gradient energy, mu^, inverse y-FFT of i k mu^ -> G
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(col_block<P, SR, WR>(), (col_min_blocks<P, SR, WR>())) k_col_a(const InstDev* __restrict__ insts, const int* __restrict__ base,
                                                  int s_local) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeomF<P, SR, WR>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  const InstDev& I = insts[blockIdx.y];
  const int status = *(volatile const int*)I.status;  // read after the column loads are issued
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * I.dx);
  const double kappa = I.p.kappa;

  // c^ = y-FFT(S) in SR
  cpx<SR> v[E];
  {
    const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = active ? ldc(S + (size_t)(t + T * m) * H + kx) : mkc<SR>(0, 0);
  }
  if (status) return;  // block-uniform: one instance per block
  if (w == 0) {
    // F is read after the S transform: start pulling this block's rows of it into L2
    const cpx<WR>* F = reinterpret_cast<const cpx<WR>*>(I.F) + (size_t)blockIdx.x * W;
#pragma unroll
    for (int m = 0; m < E; ++m) prefetch_l2(F + (size_t)(t + T * m) * H);
  }
  cpx<SR>* sms = reinterpret_cast<cpx<SR>*>(smraw);
  fft<false, P>(v, t, sms, lay, PassTable<P, SR>{});

  const bool packed_tile = blockIdx.x == 0;  // holds kx = 0 (DC + i Nyquist)
  const bool packed = packed_tile && w == 0;
  double gsum = 0.0;
  cpx<WR> u[E];  // 2 kappa k^2 c^ (+ packed-column correction), in WR
  const double kxf = kunit * (double)kx;
  const double kH2 = (kunit * (double)H) * (kunit * (double)H);
  if (packed_tile) {
    // partner exchange for the packed column: B_c(ky) = (P(ky) - conj(P(-ky))) / (2i)
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sms[t + T * m] = v[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<SR> pr = cconj(sms[(N - ky) % N]);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf;
        const cpx<SR> Ac = cscale(v[m] + pr, (SR)0.5);
        const cpx<SR> Bc = cscale(times_negi(v[m] - pr), (SR)0.5);
        gsum += k2a * ((double)Ac.x * Ac.x + (double)Ac.y * Ac.y) +
                (k2a + kH2) * ((double)Bc.x * Bc.x + (double)Bc.y * Bc.y);
        // 2 kappa (k2a * P + i kH2 * Bc)
        const cpx<SR> t1 = cscale(v[m], (SR)(2.0 * kappa * k2a));
        const cpx<SR> t2 = times_i(cscale(Bc, (SR)(2.0 * kappa * kH2)));
        u[m] = ccast<WR>(t1 + t2);
      }
    }
    __syncthreads();
  }
  if (!packed) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const double kyf = kunit * (double)(ky < H ? ky : ky - N);
      const double k2 = kxf * kxf + kyf * kyf;
      if (active) gsum += 2.0 * k2 * ((double)v[m].x * v[m].x + (double)v[m].y * v[m].y);
      u[m] = ccast<WR>(cscale(v[m], (SR)(2.0 * kappa * k2)));
    }
  }

  // f'^ = y-FFT(F) in WR, mu^ = f'^ + u
  cpx<WR> a[E];
  {
    const cpx<WR>* F = reinterpret_cast<const cpx<WR>*>(I.F);
#pragma unroll
    for (int m = 0; m < E; ++m) a[m] = active ? ldc(F + (size_t)(t + T * m) * H + kx) : mkc<WR>(0, 0);
  }
  cpx<WR>* smw = reinterpret_cast<cpx<WR>*>(smraw);
  fft<false, P>(a, t, smw, lay, PassTable<P, WR>{});
  const WR scale = (WR)(1.0 / ((double)N * (double)N));
  const WR kxd = (WR)kxf;  // kx < n/2: never the Nyquist
  if constexpr (kSplitMixed<SR, WR>) {
    // both derivatives in one packed transform (lane 0: x, lane 1: y)
    cpx<f2> q[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const WR kyd = (ky == H) ? (WR)0 : wavenumber<WR>(ky, N, kunit);
      const cpx<WR> mu = cscale(a[m] + u[m], scale);
      q[m] = pack2(times_i(cscale(mu, kxd)), times_i(cscale(mu, kyd)));
    }
    fft<true, P>(q, t, reinterpret_cast<cpx<f2>*>(smraw), lay, PassTableDup<P>{});
#pragma unroll
    for (int m = 0; m < E; ++m) {
      a[m] = lane0(q[m]);
      u[m] = lane1(q[m]);
    }
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const WR kyd = (ky == H) ? (WR)0 : wavenumber<WR>(ky, N, kunit);
      const cpx<WR> mu = cscale(a[m] + u[m], scale);
      a[m] = times_i(cscale(mu, kxd));   // x-derivative
      u[m] = times_i(cscale(mu, kyd));   // y-derivative
    }
    fft<true, P>(a, t, smw, lay, PassTable<P, WR>{});
    fft<true, P>(u, t, smw, lay, PassTable<P, WR>{});
  }
  if (active) {
    cpx2<WR>* Gp = reinterpret_cast<cpx2<WR>*>(I.G);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      cpx2<WR> o;
      o.a = a[m];
      o.b = u[m];
      Gp[(size_t)(t + T * m) * H + kx] = o;
    }
  }
  // per-warp partials and a per-warp arrival: no block-wide barrier at the end
  const double r = warp_sum(gsum);
  const int nw = (int)(blockDim.x >> 5), slots = (int)gridDim.x * nw;
  double* part = I.part + (size_t)5 * ((H + RowGeom<P>::G - 1) / RowGeom<P>::G);
  if ((threadIdx.x & 31) == 0) part[blockIdx.x * nw + (threadIdx.x >> 5)] = r;
  if (!warp_arrive_last(&I.cnt[1], (unsigned)slots)) return;
  const double gr = warp_fold<OpSum>(part, slots, 1, 0.0);
  if ((threadIdx.x & 31) == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) {
      const double e = (I.scal[0] + kappa * gr / ((double)N * N)) * I.dx * I.dx;
      I.hist[s + 2 * (size_t)I.hist_ld] = e;
    }
    I.cnt[1] = 0;
  }
}

// row B: grad mu from G, dissipation, M grad mu, forward x-FFT back into G
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(kBlock) k_row_b(const InstDev* __restrict__ insts, const int* __restrict__ base,
                                                  int s_local) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32];
  __shared__ int lastflag;
  const InstDev& I = insts[blockIdx.y];
  if (*I.status) return;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int y = blockIdx.x * G + g;
  const bool active = y < N;
  const RowLayout<N> lay{g * RowLayout<N>::stride};
  cpx2<WR>* row = reinterpret_cast<cpx2<WR>*>(I.G) + (size_t)(active ? y : 0) * H;
  cpx<WR> v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = active ? load_pair_spectrum2<WR, N>(row, t + T * m) : mkc<WR>(0, 0);
  cpx<WR>* smw = reinterpret_cast<cpx<WR>*>(smraw);
  fft<true, P>(v, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
  const WR* phi = reinterpret_cast<const WR*>(I.phi);
  const WR M0 = (WR)I.p.mobility;
  double dsum = 0.0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    WR M = 0;
    if (active) {
      M = mobility_of<WR>(__ldg(phi + (size_t)y * N + x), M0);
      dsum += (double)M * ((double)v[m].x * v[m].x + (double)v[m].y * v[m].y);
    }
    v[m] = cscale(v[m], M);
  }
  fft<false, P>(v, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
  cpx<WR> xa[E / 2], xb[E / 2];
  split_pair<P>(v, t, smw, lay, xa, xb);
  if (active) {
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      cpx2<WR> o;
      o.a = xa[m];
      o.b = xb[m];
      row[t + T * m] = o;
    }
  }
  const double r = block_reduce<OpSum>(dsum, red);
  const int tiles = gridDim.x;
  double* part = I.part + (size_t)5 * ((H + G - 1) / G) + (H + ColGeom<P>::W - 1) / ColGeom<P>::W;
  if (threadIdx.x == 0) part[blockIdx.x] = r;
  if (!arrive_last(&I.cnt[2], tiles, &lastflag)) return;
  const double d = reduce_partials<OpSum>(part, tiles, 1, 0.0, red);
  if (threadIdx.x == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) I.hist[s + 5 * (size_t)I.hist_ld] = d * I.dx * I.dx;
    I.cnt[2] = 0;
  }
}

// col B: y-FFT of the fluxes, divergence, stabilised increment, inverse y-FFT, S += increment
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(col_block<P, SR, WR>(), (col_min_blocks<P, SR, WR>())) k_col_b(const InstDev* __restrict__ insts) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeomF<P, SR, WR>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32];
  const InstDev& I = insts[blockIdx.y];
  const int status = *(volatile const int*)I.status;  // read after the column loads are issued
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * I.dx);
  const cpx2<WR>* Gp = reinterpret_cast<const cpx2<WR>*>(I.G);
  cpx<WR> a[E], b[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    if (active) {
      const cpx2<WR> o = Gp[(size_t)(t + T * m) * H + kx];
      a[m] = o.a;
      b[m] = o.b;
    } else {
      a[m] = mkc<WR>(0, 0);
      b[m] = mkc<WR>(0, 0);
    }
  }
  if (status) return;  // block-uniform: one instance per block
  if (w == 0) {
    // S is updated after both transforms: start pulling this block's rows of it into L2
    const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S) + (size_t)blockIdx.x * W;
#pragma unroll
    for (int m = 0; m < E; ++m) prefetch_l2(S + (size_t)(t + T * m) * H);
  }
  cpx<WR>* smw = reinterpret_cast<cpx<WR>*>(smraw);
  if constexpr (kSplitMixed<SR, WR>) {
    // both flux components in one packed transform (lane 0: x, lane 1: y)
    cpx<f2> q[E];
#pragma unroll
    for (int m = 0; m < E; ++m) q[m] = pack2(a[m], b[m]);
    fft<false, P>(q, t, reinterpret_cast<cpx<f2>*>(smraw), lay, PassTableDup<P>{});
#pragma unroll
    for (int m = 0; m < E; ++m) {
      a[m] = lane0(q[m]);
      b[m] = lane1(q[m]);
    }
  } else {
    fft<false, P>(a, t, smw, lay, PassTable<P, WR>{});
    fft<false, P>(b, t, smw, lay, PassTable<P, WR>{});
  }
  const double c1 = 2.0 * I.p.Q * I.p.kappa * I.dt;  // den = 1 + c1 k2^2
  const double kxf = kunit * (double)kx;
  const double kH2 = (kunit * (double)H) * (kunit * (double)H);
  const WR dtn = (WR)(I.dt / (double)N);
  const bool packed_tile = blockIdx.x == 0;
  const bool packed = packed_tile && w == 0;
  if (packed_tile) {
    // packed column: kx derivative vanishes for both kx = 0 and kx = n/2;
    // incr = dt i ky (A_y/den_A + i B_y/den_B) / n with B_y from the partner mode
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) smw[t + T * m] = b[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<WR> pr = cconj(smw[(N - ky) % N]);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf, k2b = k2a + kH2;
        const WR ida = (WR)(1.0 / (1.0 + c1 * k2a * k2a)), idb = (WR)(1.0 / (1.0 + c1 * k2b * k2b));
        const WR kyd = (ky == H) ? (WR)0 : (WR)kyf;
        const cpx<WR> Ay = cscale(b[m] + pr, (WR)0.5);
        const cpx<WR> By = cscale(times_negi(b[m] - pr), (WR)0.5);
        const cpx<WR> q = cscale(Ay, ida) + times_i(cscale(By, idb));
        a[m] = times_i(cscale(q, kyd * dtn));
      }
    }
    __syncthreads();
  }
  if (!packed) {
    const WR kxd = (WR)kxf;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const double kyf = kunit * (double)(ky < H ? ky : ky - N);
      const double k2 = kxf * kxf + kyf * kyf;
      WR iden;
      if constexpr (kSplitMixed<SR, WR>)
        iden = __frcp_rn((float)fma(c1 * k2, k2, 1.0));  // FP32 reciprocal of the stabiliser
      else
        iden = (WR)(1.0 / (1.0 + c1 * k2 * k2));
      const WR kyd = (ky == H) ? (WR)0 : (WR)kyf;
      const cpx<WR> div = times_i(cscale(a[m], kxd) + cscale(b[m], kyd));
      a[m] = cscale(div, iden * dtn);
    }
  }
  fft<true, P>(a, t, smw, lay, PassTable<P, WR>{});
  // exact mass conservation: the DC row-mode increments (packed column, real
  // part) must sum to zero over y; remove the rounding residue in FP64.
  double corr = 0.0;
  if (packed_tile) {
    double colsum = 0.0;
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) colsum += (double)a[m].x;
    }
    const double tot = block_reduce<OpSum>(colsum, red);
    if (packed) corr = tot / (double)N;
  }
  if (active) {
    cpx<SR>* S = reinterpret_cast<cpx<SR>*>(I.S);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      cpx<SR>* sp = S + (size_t)(t + T * m) * H + kx;
      const cpx<SR> s0 = *sp;
      *sp = mkc<SR>(s0.x + (SR)((double)a[m].x - corr), s0.y + (SR)a[m].y);
    }
  }
}

}  // namespace esc
