// Warp-independent row kernels (row A and row B).
//
// Every FFT group (T <= 32 threads, one row pair for row A, one row for row B)
// lives inside a single warp and exchanges through its own swizzled slice of
// shared memory, so the transforms need only __syncwarp.  History partials are
// reduced per warp and the last warp to arrive for an instance folds them.
// No block-wide barrier remains: the warps of a block drift freely, and one
// warp's global loads overlap another warp's transforms.  The numerics are
// those of k_row_a / k_row_b in esc_kernels.cuh, operation for operation.
#pragma once
#include "esc_pipe.cuh"

#include <type_traits>

namespace esc {


// Plans with every group inside a warp (T <= 32) and E <= 16 where possible.
template <int N>
struct WarpPlan {
  using type = typename DefaultPlan<N>::type;
};
#define ESC_WPLAN(n, e, ...) \
  template <>                \
  struct WarpPlan<n> { using type = Plan<n, e, Radices<__VA_ARGS__>>; };
ESC_WPLAN(96, 12, 4, 4, 6)
ESC_WPLAN(384, 12, 4, 4, 4, 6)
ESC_WPLAN(512, 16, 16, 16, 2)
ESC_WPLAN(768, 24, 8, 8, 12)
#undef ESC_WPLAN

// Row A (FP64 inverse transform, bulk terms, FP32 forward transform) prefers
// E8 in 64-thread groups at n = 512: half the registers, 24 warps per SM.
template <int N>
struct WarpPlanA {
  using type = typename WarpPlan<N>::type;
};
template <>
struct WarpPlanA<512> {
  using type = Plan<512, 8, Radices<8, 8, 8>>;
};

// Blocks of the warp-independent kernels: no block-wide barrier ties their
// warps together, so small blocks let every warp start as soon as one retires
// and keep the warps of an SM spread over load and compute phases.
#ifndef ESC_WARP_BLOCK
#define ESC_WARP_BLOCK 32
#endif
constexpr int kWarpBlock = ESC_WARP_BLOCK;
constexpr int kWarpBlocksPerSM = 512 / kWarpBlock;  // 16 warps per SM at up to 128 registers

// Groups of T <= 32 threads live inside one warp (one-warp blocks, __syncwarp).
// Larger groups (64 to 256 threads) are a whole block (__syncthreads): E8 plans
// of the mid sizes, with half the registers per thread of the E16 plans, and
// the E16 plans of n >= 2048.
template <class P>
struct WarpRowGeom {
  static constexpr int N = P::N, T = P::T, H = N / 2;
  static constexpr bool kInWarp = T <= 32;
  static_assert((kInWarp && 32 % T == 0) || T == 64 || T == 128 || T == 256,
                "groups inside one warp, or a block of 64, 128 or 256 threads");
  static constexpr int BLOCK = kInWarp ? kWarpBlock : T;  // threads per block
  // blocks per SM compiled for: 128 registers per thread for T >= 128
  // (whole-warp groups of at most 12 elements fit 20 blocks, 96 registers, without spills: n = 384)
  static constexpr int MINB =
      kInWarp ? ((T == 32 && P::E <= 12) ? 20 : kWarpBlocksPerSM) : (T == 64 ? (P::E <= 8 ? 12 : 8) : 512 / T);
  static constexpr int GPW = kInWarp ? 32 / T : 1;        // groups per warp
  static constexpr int NW = BLOCK / 32;                   // warps per block
  static constexpr int G = kInWarp ? GPW * NW : 1;        // groups per block
  static constexpr int tiles_pairs = (H + G - 1) / G;
  static constexpr int tiles_rows = (N + G - 1) / G;
  using Sync = typename std::conditional<kInWarp, WarpSync, BlockSync>::type;
  static __device__ __forceinline__ void group_sync() { Sync::sync(); }
  // this thread's index inside its group, and the group's index inside the warp and the block
  static __device__ __forceinline__ int thread_in_group() { return kInWarp ? (threadIdx.x & 31) % T : threadIdx.x; }
  static __device__ __forceinline__ int group_in_warp() { return kInWarp ? (threadIdx.x & 31) / T : 0; }
  static __device__ __forceinline__ int group_in_block() {
    return kInWarp ? (threadIdx.x >> 5) * GPW + group_in_warp() : 0;
  }
  template <typename SR>
  static constexpr size_t smem() {
    // the group's exchange slice; a 64-thread group also splits its output through it
    return (size_t)G * (kInWarp ? N : N + N / 16 + 1) * sizeof(cpx<SR>);
  }
};

// Resident blocks per SM row A is compiled for: E8 in 64-thread groups runs
// 16 (mixed) or 14 (FP64) two-warp blocks, a few bytes of spills against 12 at
// 80 registers (row A at n = 512: 4 % and 2 % faster); other plans keep their
// group geometry's figure.
template <class P, typename SR, typename WR>
constexpr int row_a_minb() {
  return (P::T == 64 && P::E <= 8) ? (kSplitMixed<SR, WR> ? 16 : 14) : WarpRowGeom<P>::MINB;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}



// The five row-A folds (sum c, min c, max c, sum f, non-finite count) of slots
// holding five consecutive doubles, in one pass: one slot's five loads are
// issued together, with the per-lane order and the shuffle trees of five
// separate warp_fold calls, so the results are the same bits.
__device__ __forceinline__ void warp_fold_row_a(const double* p, int count, double& a_sum, double& a_min,
                                                double& a_max, double& a_f, double& a_bad) {
  double s0 = 0.0, s1 = INFINITY, s2 = -INFINITY, s3 = 0.0, s4 = 0.0;
#pragma unroll 4
  for (int i = (threadIdx.x & 31); i < count; i += 32) {
    const double* q = p + (size_t)i * 5;
    const double v0 = __ldcg(q), v1 = __ldcg(q + 1), v2 = __ldcg(q + 2), v3 = __ldcg(q + 3), v4 = __ldcg(q + 4);
    s0 = OpSum::ap(s0, v0);
    s1 = OpMin::ap(s1, v1);
    s2 = OpMax::ap(s2, v2);
    s3 = OpSum::ap(s3, v3);
    s4 = OpSum::ap(s4, v4);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 = OpSum::ap(s0, __shfl_xor_sync(0xffffffffu, s0, o));
    s1 = OpMin::ap(s1, __shfl_xor_sync(0xffffffffu, s1, o));
    s2 = OpMax::ap(s2, __shfl_xor_sync(0xffffffffu, s2, o));
    s3 = OpSum::ap(s3, __shfl_xor_sync(0xffffffffu, s3, o));
    s4 = OpSum::ap(s4, __shfl_xor_sync(0xffffffffu, s4, o));
  }
  a_sum = s0;
  a_min = s1;
  a_max = s2;
  a_f = s3;
  a_bad = s4;
}

__device__ __forceinline__ bool warp_instance_running(const int* status) {
  int s = 0;
  if ((threadIdx.x & 31) == 0) s = *(volatile const int*)status;
  return __shfl_sync(0xffffffffu, s, 0) == 0;
}
// The same test split in two: the status load is issued first and read after
// the row loads, so a warp waits for one memory round trip instead of two.  A
// stopped instance's rows are still valid memory; they are loaded and dropped.
__device__ __forceinline__ int warp_status_issue(const int* status) {
  int s = 0;
  if ((threadIdx.x & 31) == 0) s = *(volatile const int*)status;
  return s;
}
__device__ __forceinline__ bool warp_status_running(int s) { return __shfl_sync(0xffffffffu, s, 0) == 0; }

// =====================================================================================
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(WarpRowGeom<P>::BLOCK, (row_a_minb<P, SR, WR>())) k_row_a_w(const InstDev* __restrict__ insts,
                                                       const int* __restrict__ base, int s_local) {
  using WG = WarpRowGeom<P>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, NW = WG::NW, G = WG::G;
  constexpr int tiles = WG::tiles_pairs;
  extern __shared__ __align__(16) unsigned char smraw[];
  const InstDev& I = insts[blockIdx.y];
  const int status = warp_status_issue(I.status);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = WG::thread_in_group(), gw = WG::group_in_warp();  // thread and group inside the warp
  const int g = WG::group_in_block();                               // group inside the block
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;

  cpx<SR> v[E];
  if (active) {
    prefetch_l1(reinterpret_cast<const WR*>(I.phi) + (size_t)ya * N, 2 * N * (int)sizeof(WR), t, T);
    const cpx<SR>* S = reinterpret_cast<const cpx<SR>*>(I.S);
    const cpx<SR>* ra = S + (size_t)ya * H;
    const cpx<SR>* rb = ra + H;
    load_pair_rows<P, SR>(v, t, [&](int idx, cpx<SR>& a, cpx<SR>& b) {
      a = ldc(ra + idx);
      b = ldc(rb + idx);
    });
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = mkc<SR>(0, 0);
  }
  if (!warp_status_running(status)) return;
  cpx<SR>* xs = reinterpret_cast<cpx<SR>*>(smraw);
  const SwizzleLayout<N, sizeof(cpx<SR>)> lay_s{g * N, gw};
  fft<true, P, typename WG::Sync>(v, t, xs, lay_s, PassTable<P, SR>{});

  const ModelParams mp = I.p;
  const SR invN = (SR)1 / (SR)N;
  const WR* phi = reinterpret_cast<const WR*>(I.phi);
  double sum_c = 0.0, sum_f = 0.0, mn = INFINITY, mx = -INFINITY, bad = 0.0;
  cpx<WR> wv[E];
  if constexpr (kSplitMixed<SR, WR>) {
    // FP32 bulk terms with the FP64 remainder of c folded in to first order
    int nbad = 0;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int x = t + T * m;
      f2 fp(0.0f, 0.0f);
      if (active) {
        const double ca = v[m].x * invN, cb = v[m].y * invN;
        f2 fv;
        bulk_pair_split(ca, cb, __ldg(reinterpret_cast<const float*>(phi) + (size_t)ya * N + x),
                        __ldg(reinterpret_cast<const float*>(phi) + (size_t)(ya + 1) * N + x), mp, fp, fv);
        sum_c += ca + cb;
        sum_f += (double)(fv.v.x + fv.v.y);
        mn = fmin(mn, fmin(ca, cb));
        mx = fmax(mx, fmax(ca, cb));
        nbad += (int)(nonfinite_bits(ca) | nonfinite_bits(cb));
      }
      wv[m] = mkc<WR>((WR)fp.v.x, (WR)fp.v.y);
    }
    bad = (double)nbad;
  } else {
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
    wv[m] = mkc<WR>((WR)fa, (WR)fb);
  }
  }
  cpx<WR>* xw = reinterpret_cast<cpx<WR>*>(smraw);
  // the FP32 exchange reuses the group's slice (n elements of the smaller type)
  const SwizzleLayout<N, sizeof(cpx<WR>)> lay_w{g * N * (int)(sizeof(cpx<SR>) / sizeof(cpx<WR>)), gw};
  WG::group_sync();
  fft<false, P, typename WG::Sync>(wv, t, xw, lay_w, PassTable<P, WR>{});
  cpx<WR> xa[E / 2], xb[E / 2];
  split_rows<P, WR>(wv, t, xw, RowLayout<N>{0}, xa, xb);
  if (active) {
    cpx<WR>* F = reinterpret_cast<cpx<WR>*>(I.F) + (size_t)ya * H;
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      F[t + T * m] = xa[m];
      F[H + t + T * m] = xb[m];
    }
  }
  sum_c = warp_sum(sum_c);
  mn = warp_min(mn);
  mx = warp_max(mx);
  sum_f = warp_sum(sum_f);
  bad = warp_sum(bad);
  const int slot = blockIdx.x * NW + warp;
  if (lane == 0) {
    double* pp = I.part + (size_t)slot * 5;
    pp[0] = sum_c;
    pp[1] = mn;
    pp[2] = mx;
    pp[3] = sum_f;
    pp[4] = bad;
  }
  if (!warp_arrive_last(&I.cnt[0], (unsigned)(tiles * NW))) return;
  const int nslots = tiles * NW;
  double a_sum, a_min, a_max, a_f, a_bad;
  warp_fold_row_a(I.part, nslots, a_sum, a_min, a_max, a_f, a_bad);
  if (lane == 0) {
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
      *I.status = kStatusNonFinite;
    }
    I.cnt[0] = 0;
  }
}

// =====================================================================================
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(WarpRowGeom<P>::BLOCK, WarpRowGeom<P>::MINB) k_row_b_w(const InstDev* __restrict__ insts,
                                                       const int* __restrict__ base, int s_local) {
  using WG = WarpRowGeom<P>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, NW = WG::NW, G = WG::G;
  constexpr int tiles = WG::tiles_rows;
  extern __shared__ __align__(16) unsigned char smraw[];
  const InstDev& I = insts[blockIdx.y];
  const int status = warp_status_issue(I.status);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = WG::thread_in_group(), gw = WG::group_in_warp();
  const int g = WG::group_in_block();
  const int y = blockIdx.x * G + g;
  const bool active = y < N;
  cpx2<WR>* row = reinterpret_cast<cpx2<WR>*>(I.G) + (size_t)(active ? y : 0) * H;
  cpx<WR> v[E];
  if (active) {
    prefetch_l1(reinterpret_cast<const WR*>(I.phi) + (size_t)y * N, N * (int)sizeof(WR), t, T);
    load_pair_rows<P, WR>(v, t, [&](int idx, cpx<WR>& a, cpx<WR>& b) {
      const cpx2<WR> q = row[idx];
      a = q.a;
      b = q.b;
    });
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = mkc<WR>(0, 0);
  }
  if (!warp_status_running(status)) return;
  cpx<WR>* xw = reinterpret_cast<cpx<WR>*>(smraw);
  const SwizzleLayout<N, sizeof(cpx<WR>)> lay{g * N, gw};
  fft<true, P, typename WG::Sync>(v, t, xw, lay, PassTable<P, WR>{});
  const WR* phi = reinterpret_cast<const WR*>(I.phi);
  const WR M0 = (WR)I.p.mobility;
  double dsum = 0.0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    WR M = 0;
    if (active) {
      M = mobility_of<WR>(__ldg(phi + (size_t)y * N + t + T * m), M0);
      dsum += (double)M * ((double)v[m].x * v[m].x + (double)v[m].y * v[m].y);
    }
    v[m] = cscale(v[m], M);
  }
  fft<false, P, typename WG::Sync>(v, t, xw, lay, PassTable<P, WR>{});
  cpx<WR> xa[E / 2], xb[E / 2];
  split_rows<P, WR>(v, t, xw, RowLayout<N>{0}, xa, xb);
  WG::group_sync();  // every thread of the group has read its inputs before the row is overwritten
  if (active) {
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      cpx2<WR> o;
      o.a = xa[m];
      o.b = xb[m];
      row[t + T * m] = o;
    }
  }
  dsum = warp_sum(dsum);
  const int slot = blockIdx.x * NW + warp;
  if (lane == 0) I.part[slot] = dsum;
  if (!warp_arrive_last(&I.cnt[2], (unsigned)(tiles * NW))) return;
  const double d = warp_fold<OpSum>(I.part, tiles * NW, 1, 0.0);
  if (lane == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) I.hist[s + 5 * (size_t)I.hist_ld] = d * I.dx * I.dx;
    I.cnt[2] = 0;
  }
}

// =====================================================================================
// Packed row B of the mixed precision: each group transforms two adjacent rows
// at once, one per lane of packed FP32 pairs (cpx<f2>), so every butterfly
// instruction serves both rows and a warp keeps twice the data in flight.
// The numerics are those of k_row_b_w per lane, except that the 1/2 of the
// two-real-fields split is folded into the mobility (an exact scaling).

// Split of the packed DFTs Y = FFT(a + i b) (one per lane) into the packed half
// spectra of a and b, when the data already carry the factor 1/2:
//   Xa(k) = Y(k) + conj Y(n-k),  Xb(k) = -i (Y(k) - conj Y(n-k)),
// slot k = 0 of thread 0 packing (DC, Nyquist) at full scale.
template <class P>
__device__ __forceinline__ void split_rows_packed(const cpx<f2> (&y)[P::E], int t, cpx<f2> (&xa)[P::E / 2],
                                                  cpx<f2> (&xb)[P::E / 2]) {
  constexpr int E = P::E, T = P::T;
  static_assert(T <= 32, "mirror exchange by shuffle");
  const int lane = threadIdx.x & 31;
  const int src = lane - t + ((T - t) & (T - 1));
#pragma unroll
  for (int m = 0; m < E / 2; ++m) {
    const cpx<f2> q = y[E - 1 - m];
    cpx<f2> y2;
    y2.x.v.x = __shfl_sync(0xffffffffu, q.x.v.x, src);
    y2.x.v.y = __shfl_sync(0xffffffffu, q.x.v.y, src);
    y2.y.v.x = __shfl_sync(0xffffffffu, q.y.v.x, src);
    y2.y.v.y = __shfl_sync(0xffffffffu, q.y.v.y, src);
    const cpx<f2> y1 = y[m];
    if (t == 0) {
      if (m == 0) {
        const cpx<f2> yh = y[E / 2];
        xa[0] = mkc<f2>(y1.x + y1.x, yh.x + yh.x);
        xb[0] = mkc<f2>(y1.y + y1.y, yh.y + yh.y);
        continue;
      }
      y2 = y[E - m];
    }
    xa[m] = mkc<f2>(y1.x + y2.x, y1.y - y2.y);
    xb[m] = mkc<f2>(y1.y + y2.y, y2.x - y1.x);
  }
}

// the same split for a block-sized group: the mirror modes go through the group's slice
template <class P>
__device__ __forceinline__ void split_rows_packed_block(const cpx<f2> (&y)[P::E], int t, cpx<f2>* slice,
                                                        cpx<f2> (&xa)[P::E / 2], cpx<f2> (&xb)[P::E / 2]) {
  constexpr int N = P::N, E = P::E, T = P::T;
#pragma unroll
  for (int m = E / 2; m < E; ++m) slice[t + T * m] = y[m];
  __syncthreads();
#pragma unroll
  for (int m = 0; m < E / 2; ++m) {
    const cpx<f2> y1 = y[m];
    cpx<f2> y2 = slice[(N - t - T * m) % N];
    if (t == 0) {
      if (m == 0) {
        const cpx<f2> yh = y[E / 2];
        xa[0] = mkc<f2>(y1.x + y1.x, yh.x + yh.x);
        xb[0] = mkc<f2>(y1.y + y1.y, yh.y + yh.y);
        continue;
      }
      y2 = y[E - m];
    }
    xa[m] = mkc<f2>(y1.x + y2.x, y1.y - y2.y);
    xb[m] = mkc<f2>(y1.y + y2.y, y2.x - y1.x);
  }
}

template <class P>
__global__ void __launch_bounds__(WarpRowGeom<P>::BLOCK, WarpRowGeom<P>::MINB) k_row_b_w2(const InstDev* __restrict__ insts,
                                                        const int* __restrict__ base, int s_local) {
  using WG = WarpRowGeom<P>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, NW = WG::NW, G = WG::G;
  constexpr int tiles = WG::tiles_pairs;
  extern __shared__ __align__(16) unsigned char smraw[];
  const InstDev& I = insts[blockIdx.y];
  const int status = warp_status_issue(I.status);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = WG::thread_in_group(), gw = WG::group_in_warp();
  const int g = WG::group_in_block();
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int y0 = 2 * (active ? pair : 0);
  cpx2<float>* r0 = reinterpret_cast<cpx2<float>*>(I.G) + (size_t)y0 * H;
  cpx2<float>* r1 = r0 + H;
  const float* phi = reinterpret_cast<const float*>(I.phi) + (size_t)y0 * N;
  cpx<f2> v[E];
  if (active) {
    prefetch_l1(phi, 2 * N * (int)sizeof(float), t, T);
    load_pair_rows<P, f2>(v, t, [&](int idx, cpx<f2>& a, cpx<f2>& b) {
      const cpx2<float> q0 = r0[idx], q1 = r1[idx];
      a = pack2(q0.a, q1.a);
      b = pack2(q0.b, q1.b);
    });
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = mkc<f2>(f2(0.0f, 0.0f), f2(0.0f, 0.0f));
  }
  if (!warp_status_running(status)) return;
  cpx<f2>* xs = reinterpret_cast<cpx<f2>*>(smraw);
  const SwizzleLayout<N, sizeof(cpx<f2>)> lay{g * N, gw};
  const PassTableDup<P> twp{};
  fft<true, P, typename WG::Sync>(v, t, xs, lay, twp);
  const f2 Mh(0.5 * I.p.mobility);
  double dsum = 0.0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    f2 M(0.0f, 0.0f);
    if (active) {
      const int x = t + T * m;
      const f2 ph(__ldg(phi + x), __ldg(phi + N + x));
      const f2 p2 = ph * ph;
      M = Mh * (p2 * ph * fma(ph, fma(ph, f2(6.0), f2(-15.0)), f2(10.0)));
      const f2 d = M * fma(v[m].x, v[m].x, v[m].y * v[m].y);
      dsum += (double)d.v.x + (double)d.v.y;
    }
    v[m] = mkc<f2>(v[m].x * M, v[m].y * M);
  }
  WG::group_sync();  // every thread of the group has finished its gathers before the next scatter
  fft<false, P, typename WG::Sync>(v, t, xs, lay, twp);
  cpx<f2> xa[E / 2], xb[E / 2];
  if constexpr (WG::kInWarp)
    split_rows_packed<P>(v, t, xa, xb);
  else
    split_rows_packed_block<P>(v, t, xs, xa, xb);
  if (active) {
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      cpx2<float> o0, o1;
      o0.a = lane0(xa[m]);
      o0.b = lane0(xb[m]);
      o1.a = lane1(xa[m]);
      o1.b = lane1(xb[m]);
      r0[t + T * m] = o0;
      r1[t + T * m] = o1;
    }
  }
  dsum = 2.0 * warp_sum(dsum);
  const int slot = blockIdx.x * NW + warp;
  if (lane == 0) I.part[slot] = dsum;
  if (!warp_arrive_last(&I.cnt[2], (unsigned)(tiles * NW))) return;
  const double d = warp_fold<OpSum>(I.part, tiles * NW, 1, 0.0);
  if (lane == 0) {
    const int s = step_index(base, s_local);
    if (I.hist) I.hist[s + 5 * (size_t)I.hist_ld] = d * I.dx * I.dx;
    I.cnt[2] = 0;
  }
}

}  // namespace esc
