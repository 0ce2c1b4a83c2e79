// In-register / shared-memory FFT engine for the Cahn-Hilliard stepper (sm_100a).
//
// One length-N complex DFT is computed by a group of T = N/E threads.  Thread t
// of the group holds E values in registers, at positions t + T*m (m < E).  The
// transform is a sequence of Stockham radix passes (radices R_0, R_1, ... with
// product N, each dividing E): in every pass a thread performs E/R butterflies
// whose inputs are exactly its own registers, so only the outputs of a
// non-final pass are exchanged through shared memory (scatter, barrier,
// gather, barrier).  The final pass writes back into the same registers, so the
// result is again held at positions t + T*m in natural order.  A P-pass plan
// therefore costs P-1 shared-memory exchanges and no staging of inputs or
// outputs; the pointwise physics runs on the registers between transforms.
//
// The forward transform is the unnormalised DFT X(k) = sum_x x(x) e^{-2 pi i k x / N};
// the inverse uses e^{+...} and is also unnormalised (callers fold 1/N into
// their pointwise scale factors).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace esc {

// Two FP32 lanes processed by one packed sm_100 instruction (FADD2 / FMUL2 /
// FFMA2).  Every lane is rounded exactly like the scalar FP32 operation.  PTX
// has no packed negation, so a - b is fma(b, -1, a) (exact product, one
// rounding: identical to a subtraction) and -a is a * -1.
struct __align__(8) f2 {
  float2 v;
  f2() = default;
  __device__ __forceinline__ constexpr f2(float a, float b) : v{a, b} {}
  __device__ __forceinline__ explicit constexpr f2(double s) : v{(float)s, (float)s} {}
};
__device__ __forceinline__ f2 operator+(f2 a, f2 b) {
  f2 r;
  r.v = __fadd2_rn(a.v, b.v);
  return r;
}
__device__ __forceinline__ f2 operator*(f2 a, f2 b) {
  f2 r;
  r.v = __fmul2_rn(a.v, b.v);
  return r;
}
using ::fma;  // keep the scalar overloads visible beside the packed one
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) {
  f2 r;
  r.v = __ffma2_rn(a.v, b.v, c.v);
  return r;
}
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return fma(b, f2(-1.0f, -1.0f), a); }
__device__ __forceinline__ f2 operator-(f2 a) { return a * f2(-1.0f, -1.0f); }

template <typename R>
struct __align__(2 * sizeof(R)) cpx {
  R x, y;
};

template <typename R>
__device__ __forceinline__ cpx<R> mkc(R x, R y) {
  cpx<R> c;
  c.x = x;
  c.y = y;
  return c;
}
template <typename R>
__device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) { return mkc<R>(a.x + b.x, a.y + b.y); }
template <typename R>
__device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) { return mkc<R>(a.x - b.x, a.y - b.y); }
template <typename R>
__device__ __forceinline__ cpx<R> cmul(cpx<R> a, cpx<R> b) {
  return mkc<R>(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <typename R>
__device__ __forceinline__ cpx<R> cmulconj(cpx<R> a, cpx<R> b) {  // a * conj(b)
  return mkc<R>(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
template <typename R>
__device__ __forceinline__ cpx<R> cscale(cpx<R> a, R s) { return mkc<R>(a.x * s, a.y * s); }
template <typename R>
__device__ __forceinline__ cpx<R> cconj(cpx<R> a) { return mkc<R>(a.x, -a.y); }
template <typename R>
__device__ __forceinline__ cpx<R> times_i(cpx<R> a) { return mkc<R>(-a.y, a.x); }      // a * i
template <typename R>
__device__ __forceinline__ cpx<R> times_negi(cpx<R> a) { return mkc<R>(a.y, -a.x); }   // a * (-i)
template <typename R, typename S>
__device__ __forceinline__ cpx<R> ccast(cpx<S> a) { return mkc<R>((R)a.x, (R)a.y); }

// read-only (non-coherent cache) load of a complex value
template <typename R>
__device__ __forceinline__ cpx<R> ldc(const cpx<R>* p);
template <>
__device__ __forceinline__ cpx<float> ldc<float>(const cpx<float>* p) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return mkc<float>(v.x, v.y);
}
template <>
__device__ __forceinline__ cpx<double> ldc<double>(const cpx<double>* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return mkc<double>(v.x, v.y);
}

// ---- packed pairs of complex values: cpx<f2> holds (x0, x1) + i (y0, y1), two
// independent transforms in the two lanes (twiddles: DupTable below).
__device__ __forceinline__ cpx<f2> cmul(cpx<f2> a, cpx<f2> b) {
  const f2 nby = b.y * f2(-1.0f, -1.0f);
  return mkc<f2>(fma(a.y, nby, a.x * b.x), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ cpx<f2> cmulconj(cpx<f2> a, cpx<f2> b) {  // a * conj(b)
  const f2 nby = b.y * f2(-1.0f, -1.0f);
  return mkc<f2>(fma(a.y, b.y, a.x * b.x), fma(a.x, nby, a.y * b.x));
}
__device__ __forceinline__ cpx<f2> pack2(cpx<float> a, cpx<float> b) {
  return mkc<f2>(f2(a.x, b.x), f2(a.y, b.y));
}
__device__ __forceinline__ cpx<float> lane0(cpx<f2> v) { return mkc<float>(v.x.v.x, v.y.v.x); }
__device__ __forceinline__ cpx<float> lane1(cpx<f2> v) { return mkc<float>(v.x.v.y, v.y.v.y); }

// cos / sin of 2*pi*a/48 for the multiples used by the in-register radices
// (6, 8, 12, 16 all divide 48).  Correctly rounded double constants.
__device__ __forceinline__ constexpr double cos48(int a) {
  switch (((a % 48) + 48) % 48) {
    case 0: return 1.0;
    case 3: return 9.238795325112867384831e-01;
    case 4: return 8.660254037844385965883e-01;
    case 6: return 7.071067811865475727373e-01;
    case 8: return 5.0e-01;
    case 9: return 3.826834323650897817792e-01;
    case 12: return 0.0;
    case 15: return -3.826834323650897817792e-01;
    case 16: return -5.0e-01;
    case 18: return -7.071067811865475727373e-01;
    case 20: return -8.660254037844385965883e-01;
    case 21: return -9.238795325112867384831e-01;
    case 24: return -1.0;
    case 27: return -9.238795325112867384831e-01;
    case 28: return -8.660254037844385965883e-01;
    case 30: return -7.071067811865475727373e-01;
    case 32: return -5.0e-01;
    case 33: return -3.826834323650897817792e-01;
    case 36: return 0.0;
    case 39: return 3.826834323650897817792e-01;
    case 40: return 5.0e-01;
    case 42: return 7.071067811865475727373e-01;
    case 44: return 8.660254037844385965883e-01;
    case 45: return 9.238795325112867384831e-01;
    default: return 0.0;  // not used by any radix
  }
}
__device__ __forceinline__ constexpr double sin48(int a) { return cos48(a - 12); }

// multiply by e^{sign * 2 pi i e / R}, sign = -1 forward, +1 inverse; e, R compile-time after unrolling
template <int R, bool INV, typename Re>
__device__ __forceinline__ cpx<Re> twiddle_const(cpx<Re> v, int e) {
  e %= R;
  if (e == 0) return v;
  if (4 * e == R) return INV ? times_i(v) : times_negi(v);
  if (2 * e == R) return mkc<Re>(-v.x, -v.y);
  if (4 * e == 3 * R) return INV ? times_negi(v) : times_i(v);
  const int a = e * (48 / R);
  const Re c = (Re)cos48(a);
  const Re s = INV ? (Re)sin48(a) : -(Re)sin48(a);
  if constexpr (std::is_same<Re, f2>::value) {
    const Re ns = INV ? (Re)-sin48(a) : (Re)sin48(a);  // no packed negation: fold the sign into the constant
    return mkc<Re>(fma(v.y, ns, v.x * c), fma(v.x, s, v.y * c));
  } else {
    return mkc<Re>(fma(v.x, c, -v.y * s), fma(v.x, s, v.y * c));
  }
}

// ---- small DFTs in registers -------------------------------------------------
template <int R, bool INV, typename Re>
struct DFT;

template <bool INV, typename Re>
struct DFT<2, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) {
    const cpx<Re> a0 = b[0], a1 = b[1];
    b[0] = a0 + a1;
    b[1] = a0 - a1;
  }
};

template <bool INV, typename Re>
struct DFT<3, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) {
    const Re h = (Re)8.660254037844385965883e-01;  // sqrt(3)/2
    const cpx<Re> t1 = b[1] + b[2];
    const cpx<Re> t2 = mkc<Re>(fma((Re)-0.5, t1.x, b[0].x), fma((Re)-0.5, t1.y, b[0].y));
    const cpx<Re> d = b[1] - b[2];
    // forward: X1 = t2 - i h d, X2 = t2 + i h d ; inverse swaps the sign of i
    const Re nh = (Re)-8.660254037844385965883e-01;
    const cpx<Re> ihd = mkc<Re>(nh * d.y, h * d.x);  // i*h*d
    b[0] = b[0] + t1;
    if (INV) {
      b[1] = t2 + ihd;
      b[2] = t2 - ihd;
    } else {
      b[1] = t2 - ihd;
      b[2] = t2 + ihd;
    }
  }
};

template <bool INV, typename Re>
struct DFT<4, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) {
    const cpx<Re> s02 = b[0] + b[2], d02 = b[0] - b[2];
    const cpx<Re> s13 = b[1] + b[3], d13 = b[1] - b[3];
    // b[1] = d02 + r, b[3] = d02 - r with r = -i d13 (forward) or +i d13
    // (inverse), written component-wise so that no negation is needed
    b[0] = s02 + s13;
    b[2] = s02 - s13;
    if (INV) {
      b[1] = mkc<Re>(d02.x - d13.y, d02.y + d13.x);
      b[3] = mkc<Re>(d02.x + d13.y, d02.y - d13.x);
    } else {
      b[1] = mkc<Re>(d02.x + d13.y, d02.y - d13.x);
      b[3] = mkc<Re>(d02.x - d13.y, d02.y + d13.x);
    }
  }
};

// composite DFT of size R1*R2 (input n = R2*n1 + n2, output k = k1 + R1*k2)
template <int R1, int R2, bool INV, typename Re>
__device__ __forceinline__ void dft_composite(cpx<Re>* b) {
  constexpr int R = R1 * R2;
  cpx<Re> y[R];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) {
    cpx<Re> u[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) u[n1] = b[R2 * n1 + n2];
    DFT<R1, INV, Re>::run(u);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) y[k1 * R2 + n2] = twiddle_const<R, INV>(u[k1], n2 * k1);
  }
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    cpx<Re> u[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) u[n2] = y[k1 * R2 + n2];
    DFT<R2, INV, Re>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) b[k1 + R1 * k2] = u[k2];
  }
}

template <bool INV, typename Re>
struct DFT<6, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) { dft_composite<2, 3, INV, Re>(b); }
};
template <bool INV, typename Re>
struct DFT<8, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) { dft_composite<2, 4, INV, Re>(b); }
};
template <bool INV, typename Re>
struct DFT<12, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) { dft_composite<3, 4, INV, Re>(b); }
};
template <bool INV, typename Re>
struct DFT<16, INV, Re> {
  static __device__ __forceinline__ void run(cpx<Re>* b) { dft_composite<4, 4, INV, Re>(b); }
};

// ---- plans -------------------------------------------------------------------
template <int... Rs>
struct Radices {};

template <int N_, int E_, typename RadList>
struct Plan {
  static constexpr int N = N_;
  static constexpr int E = E_;
  static constexpr int T = N_ / E_;
  using List = RadList;
};

// Default plans: E elements per thread, radix sequence (each radix divides E).
// Radices 3, 6 and 12 come last: the last pass exchanges nothing, and every
// earlier pass then has power-of-two strides, which the swizzled exchange
// layout keeps free of shared-memory bank conflicts.
template <int N>
struct DefaultPlan;
#define ESC_PLAN(n, e, ...) \
  template <>               \
  struct DefaultPlan<n> { using type = Plan<n, e, Radices<__VA_ARGS__>>; };
ESC_PLAN(8, 8, 8)
ESC_PLAN(12, 12, 4, 3)
ESC_PLAN(16, 16, 16)
ESC_PLAN(24, 12, 4, 2, 3)
ESC_PLAN(32, 8, 4, 8)
ESC_PLAN(48, 12, 4, 4, 3)
ESC_PLAN(64, 8, 8, 8)
ESC_PLAN(96, 24, 4, 8, 3)
ESC_PLAN(128, 16, 8, 16)
ESC_PLAN(192, 12, 4, 4, 4, 3)
ESC_PLAN(256, 16, 16, 16)
ESC_PLAN(384, 24, 8, 8, 6)
ESC_PLAN(512, 8, 8, 8, 8)
ESC_PLAN(768, 24, 8, 8, 12)
ESC_PLAN(1024, 16, 4, 16, 16)
ESC_PLAN(1536, 24, 8, 8, 8, 3)
ESC_PLAN(2048, 16, 8, 16, 16)
ESC_PLAN(3072, 24, 8, 8, 8, 6)
ESC_PLAN(4096, 16, 16, 16, 16)
#undef ESC_PLAN

// shared-memory padding: one element every 16
__device__ __forceinline__ int smpad(int p) { return p + (p >> 4); }

// Exchange addressing.  Row layout: group g owns a padded region of N elements;
// Col layout: element p of column w sits at linear index p*W + w (then padded).
// `at<RAD, NS>(p)` is the address used by the exchange after a pass of radix
// RAD with NS = product of the earlier radices (scatter and gather alike).
template <int N>
struct RowLayout {
  int base;  // g * stride
  static constexpr int stride = N + N / 16 + 1;
  __device__ __forceinline__ int operator()(int p) const { return base + smpad(p); }
  template <int RAD, int NS>
  __device__ __forceinline__ int at(int p) const { return (*this)(p); }
};
template <int W>
struct ColLayout {
  int w;
  __device__ __forceinline__ int operator()(int p) const { return smpad(p * W + w); }
  template <int RAD, int NS>
  __device__ __forceinline__ int at(int p) const { return (*this)(p); }
};

// Barrier used between the scatter and gather of an exchange: the whole block,
// or only the warp when every FFT group lives inside one warp.
struct BlockSync {
  static __device__ __forceinline__ void sync() { __syncthreads(); }
};
struct WarpSync {
  static __device__ __forceinline__ void sync() { __syncwarp(); }
};

// Twiddle factor j of a table e^{-2 pi i j / N} in global memory (read through
// the non-coherent path).
template <typename Re>
__device__ __forceinline__ cpx<Re> tw_at(const cpx<Re>* tw, int i) { return ldc(tw + i); }
// Packed transforms reading the scalar FP32 table: each factor is loaded once
// (8 bytes) and placed in both lanes.
struct DupTable {
  const cpx<float>* p;
};
__device__ __forceinline__ cpx<f2> tw_at(DupTable tw, int i) {
  const cpx<float> w = ldc(tw.p + i);
  return mkc<f2>(f2(w.x, w.x), f2(w.y, w.y));
}

// Pass-major twiddle tables, one per plan and precision.  The pass with
// radix RAD after earlier radices of product NS needs, for butterfly k < NS,
// the factors w^{s k STEP} (STEP = N / (NS RAD), 0 < s < RAD).  In the plain
// table e^{-2 pi i j / N} the lanes of a warp (consecutive k) read entries
// s STEP apart, one sector each once s STEP reaches 4; here factor s of
// butterfly k sits at OFF + (s - 1) NS + k, so the lanes read consecutive
// entries.  OFF is the sum of (R - 1) NS' over the earlier passes, and the
// passes fill exactly N - 1 entries.  The values are copied from the plain
// table (`k_fill_pass_tw`), so both give the same bits.
template <class P, typename Re>
__device__ cpx<Re> g_pass_tw[P::N];

template <class P, typename Re>
struct PassTable {};  // scalar transforms of plan P read g_pass_tw<P, Re>
template <class P>
struct PassTableDup {};  // packed FP32 transforms of plan P: g_pass_tw<P, float>, broadcast into both lanes

// factor s of butterfly k in the pass (NS, RAD) whose pass-major offset is OFF
template <int N, int NS, int RAD, int OFF, typename Re>
__device__ __forceinline__ cpx<Re> pass_tw(const cpx<Re>* tw, int k, int s) {
  return tw_at(tw, s * k * (N / (NS * RAD)));
}
template <int N, int NS, int RAD, int OFF>
__device__ __forceinline__ cpx<f2> pass_tw(DupTable tw, int k, int s) {
  return tw_at(tw, s * k * (N / (NS * RAD)));
}
template <int N, int NS, int RAD, int OFF, class P, typename Re>
__device__ __forceinline__ cpx<Re> pass_tw(PassTable<P, Re>, int k, int s) {
  return ldc(&g_pass_tw<P, Re>[OFF + (s - 1) * NS + k]);
}
template <int N, int NS, int RAD, int OFF, class P>
__device__ __forceinline__ cpx<f2> pass_tw(PassTableDup<P>, int k, int s) {
  const cpx<float> w = ldc(&g_pass_tw<P, float>[OFF + (s - 1) * NS + k]);
  return mkc<f2>(f2(w.x, w.x), f2(w.y, w.y));
}

// Copies the plain table tw (e^{-2 pi i j / N}, j < N) into g_pass_tw<P, Re>; one block.
template <class P, typename Re, int... Rs>
__device__ __forceinline__ void fill_pass_tw(const cpx<Re>* tw, Radices<Rs...>) {
  constexpr int rs[] = {Rs...};
  int ns = 1, off = 0;
#pragma unroll
  for (int q = 0; q < (int)sizeof...(Rs); ++q) {
    const int r = rs[q], step = P::N / (ns * r);
    for (int e = threadIdx.x; e < (r - 1) * ns; e += blockDim.x) {
      const int s = 1 + e / ns, k = e % ns;
      g_pass_tw<P, Re>[off + e] = tw[s * k * step];
    }
    off += (r - 1) * ns;
    ns *= r;
  }
}
template <class P, typename Re>
__global__ void k_fill_pass_tw(const cpx<Re>* tw) {
  fill_pass_tw<P, Re>(tw, typename P::List{});
}

#ifndef ESC_FP64_TREE
#define ESC_FP64_TREE 1
#endif
// FP64 passes of radix >= 8 load one factor per butterfly and build the others as its powers
constexpr bool kFP64PowerTree = ESC_FP64_TREE != 0;

// One Stockham pass (radix RAD, NS = product of earlier radices, OFF = its
// offset in a pass-major table).
template <bool INV, class P, int RAD, int NS, int OFF, bool LAST, class Sync = BlockSync, typename Re, class L,
          class TW>
__device__ __forceinline__ void stockham_pass(cpx<Re> (&v)[P::E], int t, cpx<Re>* sm, const L& lay, const TW& tw) {
  constexpr int N = P::N, E = P::E, T = P::T;
  constexpr int NB = E / RAD;
  static_assert(E % RAD == 0, "radix must divide E");
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = t + T * q;
    cpx<Re> b[RAD];
#pragma unroll
    for (int s = 0; s < RAD; ++s) b[s] = v[q + s * NB];
    if (NS > 1) {
      const int k = j % NS;
      if constexpr (kFP64PowerTree && std::is_same<Re, double>::value && RAD >= 8) {
        // FP64: one table load per butterfly; the other factors are its powers,
        // built by a product tree of depth <= 4 (a few ulp, far below the tolerances)
        cpx<Re> w[RAD];
        w[1] = pass_tw<N, NS, RAD, OFF>(tw, k, 1);
        w[2] = cmul(w[1], w[1]);
#pragma unroll
        for (int s = 3; s < RAD; ++s) {
          const int hi = 1 << (31 - __builtin_clz(s));  // largest power of two <= s
          w[s] = (s == hi) ? cmul(w[s / 2], w[s / 2]) : cmul(w[hi], w[s - hi]);
        }
#pragma unroll
        for (int s = 1; s < RAD; ++s) b[s] = INV ? cmulconj(b[s], w[s]) : cmul(b[s], w[s]);
      } else {
#pragma unroll
        for (int s = 1; s < RAD; ++s) {
          const cpx<Re> w = pass_tw<N, NS, RAD, OFF>(tw, k, s);
          b[s] = INV ? cmulconj(b[s], w) : cmul(b[s], w);
        }
      }
    }
    DFT<RAD, INV, Re>::run(b);
    if (LAST) {
#pragma unroll
      for (int s = 0; s < RAD; ++s) v[q + s * NB] = b[s];
    } else {
      const int base = (j / NS) * NS * RAD + (j % NS);
#pragma unroll
      for (int s = 0; s < RAD; ++s) sm[lay.template at<RAD, NS>(base + s * NS)] = b[s];
    }
  }
  if (!LAST) {
    Sync::sync();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[lay.template at<RAD, NS>(t + T * m)];
    Sync::sync();
  }
}

template <bool INV, class P, int NS, int OFF, class Sync, typename Re, class L, class TW, int RAD, int... REST>
__device__ __forceinline__ void fft_passes(cpx<Re> (&v)[P::E], int t, cpx<Re>* sm, const L& lay, const TW& tw,
                                           Radices<RAD, REST...>) {
  constexpr bool LAST = sizeof...(REST) == 0;
  stockham_pass<INV, P, RAD, NS, OFF, LAST, Sync>(v, t, sm, lay, tw);
  if constexpr (!LAST) fft_passes<INV, P, NS * RAD, OFF + (RAD - 1) * NS, Sync>(v, t, sm, lay, tw, Radices<REST...>{});
}

// Length-N DFT of the values v[m] at positions t + T*m; result in the same slots.
// tw: table of e^{-2 pi i j / N}, j < N, in global memory (read through L1), the
// same broadcast into both lanes (DupTable), or the plan's pass-major table
// (PassTable, PassTableDup).
// Every thread of the CTA must call this (it contains __syncthreads).
template <bool INV, class P, class Sync = BlockSync, typename Re, class L, class TW>
__device__ __forceinline__ void fft(cpx<Re> (&v)[P::E], int t, cpx<Re>* sm, const L& lay, const TW& tw) {
  fft_passes<INV, P, 1, 0, Sync>(v, t, sm, lay, tw, typename P::List{});
}

// Exchange layout of one warp-local FFT group: n elements at `base`, XOR
// swizzled inside each 128-byte line (with a per-group offset) so that the
// strided scatters and the gathers of one warp hit distinct banks.  Requires
// n to be a multiple of the line length; smaller or odd sizes stay linear.
//
// The exchange after a pass (radix RAD = 2^r, NS = 2^a) scatters element s of
// butterfly j to p = (j >> a) << (a + r) | s << a | (j & (NS - 1)): the lanes
// of one bank phase differ in j, whose low a bits already sit in the low bits
// of p while the rest sit from bit a + r up.  `at` XORs bits from
// S = max(log2 LINE, a + r) upwards into bit a and above, which lands them in
// the bank bits that s occupies (the same for every lane of an instruction),
// so the scatter spreads over all banks; the gather (consecutive p in a phase)
// sees a constant XOR and stays conflict-free.  The map only permutes within a
// line, so it is a bijection.  Other radices use the line-index swizzle.
template <int N, int ELEM_BYTES>
struct SwizzleLayout {
  int base;
  int g;  // group index inside the warp
  static constexpr int LINE = 128 / ELEM_BYTES;  // elements per 128-byte line
  __device__ __forceinline__ int operator()(int p) const {
    if constexpr (N % LINE == 0) {
      return base + (p ^ (((p / LINE) + 4 * g) & (LINE - 1)));
    } else {
      return base + p;
    }
  }
  static constexpr int lg(int v) { return v <= 1 ? 0 : 1 + lg(v / 2); }
  template <int RAD, int NS>
  __device__ __forceinline__ int at(int p) const {
    constexpr bool pow2 = (RAD & (RAD - 1)) == 0 && (NS & (NS - 1)) == 0;
    if constexpr (N % LINE == 0 && pow2) {
      constexpr int a = lg(NS), r = lg(RAD), LL = lg(LINE);
      constexpr int S = (a + r > LL) ? a + r : LL;
      return base + (p ^ ((((p >> S) << a) + 4 * g) & (LINE - 1)));
    } else {
      return (*this)(p);
    }
  }
};

}  // namespace esc
