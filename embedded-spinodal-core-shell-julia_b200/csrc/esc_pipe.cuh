// Persistent, TMA-fed versions of the four phase kernels.
//
// Each CTA walks the work items w = blockIdx.x, blockIdx.x + gridDim.x, ...
// of its size group (item = (instance, tile)).  Thread 0 keeps the next tile
// in flight: the input of item k+1 streams into the other of two shared-memory
// stages while item k is computed, so the HBM latency is hidden behind the
// FFTs instead of being paid by every tile.  Row tiles are contiguous rows and
// arrive by 1-D bulk copies; column tiles are strided and arrive by 3-D tiled
// tensor copies (x = interleaved real/imag scalars of kx, y = row, z = instance).
// Every wait on a copy is bounded; a copy that never lands sets status 2 on
// the instance (reported as ESC_ETIMEOUT) and the CTA leaves after draining.
//
// Stage layout: [region X | region Y].  Region X receives the first input and,
// once that input sits in registers, doubles as the FFT exchange buffer; region
// Y holds the second input (phi rows, f' columns or state columns) until it is
// read.  The numerics are those of esc_kernels.cuh, operation for operation.
#pragma once
#include "esc_kernels.cuh"
#include "esc_tma.cuh"

namespace esc {

constexpr int kStatusNonFinite = 1;
constexpr int kStatusTimeout = 2;
constexpr int kStatusLayout = 3;  // a stage was not 1024-byte aligned; no copy was issued
constexpr size_t kStageAlignSlack = 1024;  // extra dynamic shared memory for aligning the stages

// Dynamic shared memory of the pipelined kernels.  The runtime only guarantees
// 16-byte alignment of this region, while tensor copies need 128-byte aligned
// destinations, so every kernel rounds the base up to 1024 bytes itself.
extern __shared__ __align__(16) unsigned char esc_pipe_smem[];

__device__ __forceinline__ unsigned char* pipe_stage_base() {
  const uint32_t a = smem_u32(esc_pipe_smem);
  return esc_pipe_smem + ((1024u - (a & 1023u)) & 1023u);
}

// uniform per-CTA check that the stage base is aligned (it always is after
// pipe_stage_base; the check keeps a layout mistake from reaching the TMA unit)
__device__ __forceinline__ bool pipe_base_ok(const unsigned char* base) {
  return !__syncthreads_or(threadIdx.x == 0 && (smem_u32(base) & 1023u) != 0);
}

constexpr size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }

// ---- merged reductions ------------------------------------------------------------
// sum, min, max, sum, sum in one pass (row A history partials)
__device__ __forceinline__ void block_reduce_ssmxs(double& s0, double& mn, double& mx, double& s1, double& s2,
                                                   double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  __syncthreads();
  if (lane == 0) {
    red[wid] = s0;
    red[32 + wid] = mn;
    red[64 + wid] = mx;
    red[96 + wid] = s1;
    red[128 + wid] = s2;
  }
  __syncthreads();
  const int nw = (int)(blockDim.x >> 5);
  s0 = 0.0;
  mn = INFINITY;
  mx = -INFINITY;
  s1 = 0.0;
  s2 = 0.0;
  for (int i = 0; i < nw; ++i) {  // every thread folds the warp partials in the same order
    s0 += red[i];
    mn = fmin(mn, red[32 + i]);
    mx = fmax(mx, red[64 + i]);
    s1 += red[96 + i];
    s2 += red[128 + i];
  }
  __syncthreads();
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  v = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[i];
  __syncthreads();
  return v;
}

// ---- row helpers -------------------------------------------------------------------
// Z(k) = Xa(k) + i Xb(k) at k = t + T m from packed half-spectra rows in shared
// memory; `get(idx)` returns (Xa[idx], Xb[idx]).  The half (m < E/2 -> k < n/2)
// is known at compile time, so only thread 0 needs the DC / Nyquist patches.
template <class P, typename R, class Get>
__device__ __forceinline__ void load_pair_rows(cpx<R> (&v)[P::E], int t, const Get& get) {
  constexpr int N = P::N, E = P::E, T = P::T;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    if (m < E / 2) {
      cpx<R> a, b;
      get(t + T * m, a, b);
      v[m] = mkc<R>(a.x - b.y, a.y + b.x);
      if (m == 0 && t == 0) v[m] = mkc<R>(a.x, b.x);
    } else {
      int idx = N - t - T * m;
      if (m == E / 2 && t == 0) idx = 0;
      cpx<R> a, b;
      get(idx, a, b);
      v[m] = mkc<R>(a.x + b.y, b.x - a.y);
      if (m == E / 2 && t == 0) v[m] = mkc<R>(a.y, b.y);
    }
  }
}

template <typename R>
__device__ __forceinline__ cpx<R> shfl_c(cpx<R> v, int src) {
  return mkc<R>(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// Split the DFT Y of (a + i b) (registers at t + T m) into the packed
// half-spectra of a and b at k = t + T m, m < E/2.  The mirror mode Y(n-k) sits
// in thread (T-t) mod T, slot E-1-m (thread 0: own slot E-m); groups of at most
// a warp exchange it by shuffle, larger groups through shared memory.
template <class P, typename R>
__device__ __forceinline__ void split_rows(const cpx<R> (&y)[P::E], int t, cpx<R>* xbuf, const RowLayout<P::N>& lay,
                                           cpx<R> (&xa)[P::E / 2], cpx<R> (&xb)[P::E / 2]) {
  constexpr int N = P::N, E = P::E, T = P::T;
  cpx<R> mir[E / 2];
  if constexpr (T <= 32) {
    const int lane = threadIdx.x & 31;
    const int src = lane - t + ((T - t) & (T - 1));
#pragma unroll
    for (int m = 0; m < E / 2; ++m) mir[m] = shfl_c(y[E - 1 - m], src);
  } else {
#pragma unroll
    for (int m = E / 2; m < E; ++m) xbuf[lay(t + T * m)] = y[m];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      const int k = t + T * m;
      mir[m] = (k == 0) ? y[E / 2] : xbuf[lay(N - k)];
    }
    __syncthreads();
  }
#pragma unroll
  for (int m = 0; m < E / 2; ++m) {
    const cpx<R> y1 = y[m];
    if (t == 0) {
      if (m == 0) {
        const cpx<R> yh = y[E / 2];
        xa[m] = mkc<R>(y1.x, yh.x);
        xb[m] = mkc<R>(y1.y, yh.y);
        continue;
      }
      mir[m] = y[E - m];
    }
    const cpx<R> y2 = cconj(mir[m]);
    xa[m] = cscale(y1 + y2, (R)0.5);
    xb[m] = cscale(times_negi(y1 - y2), (R)0.5);
  }
}

// ---- geometry of the pipelined kernels ----------------------------------------------
template <class P, typename SR, typename WR>
struct PipeGeom {
  static constexpr int N = P::N, E = P::E, T = P::T, H = N / 2;
  static constexpr int G = kBlock / T;  // row groups per CTA (kBlock threads)
  static constexpr size_t kMaxSmem = 220 * 1024;
  // column CTAs: 256 threads when two stages of column B fit, else 128
  static constexpr size_t xcol_w(int w) { return ((size_t)N * w + (size_t)N * w / 16 + 1) * sizeof(cpx<SR>); }
  static constexpr size_t stage_cb_w(int w) {
    return align_up(cmax((size_t)N * w * sizeof(cpx2<WR>), xcol_w(w)), 1024);
  }
  static constexpr int CB = (T <= 128 && 2 * stage_cb_w(kBlock / T) > kMaxSmem) ? 128 : kBlock;
  static constexpr int W = CB / T;  // columns per CTA
  static constexpr int tiles_pairs = (H + G - 1) / G;
  static constexpr int tiles_rows = (N + G - 1) / G;
  static constexpr int tiles_cols = (H + W - 1) / W;
  static constexpr int RB = N <= 256 ? N : (N % 256 == 0 ? 256 : 192);  // rows per tensor box
  // exchange buffers
  static constexpr size_t xrow = (size_t)G * RowLayout<N>::stride * sizeof(cpx<SR>);
  static constexpr size_t xcol = xcol_w(W);
  // row A: X = S rows of G pairs, Y = phi rows
  static constexpr size_t ra_x = align_up(cmax((size_t)2 * G * H * sizeof(cpx<SR>), xrow), 1024);
  static constexpr size_t ra_y = align_up((size_t)2 * G * N * sizeof(WR), 1024);
  // row B: X = G pair rows, Y = phi rows
  static constexpr size_t rb_x = align_up(cmax((size_t)G * H * sizeof(cpx2<WR>), xrow), 1024);
  static constexpr size_t rb_y = align_up((size_t)G * N * sizeof(WR), 1024);
  // col A: X = S columns, Y = F columns
  static constexpr size_t ca_x = align_up(cmax((size_t)N * W * sizeof(cpx<SR>), xcol), 1024);
  static constexpr size_t ca_y = align_up((size_t)N * W * sizeof(cpx<WR>), 1024);
  // col B: X = G pair columns (the state columns are prefetched to L2 instead)
  static constexpr size_t cb_x = align_up(cmax((size_t)N * W * sizeof(cpx2<WR>), xcol), 1024);
  static constexpr size_t cb_y = 0;
  static constexpr size_t stage_ra = ra_x + ra_y, stage_rb = rb_x + rb_y;
  static constexpr size_t stage_ca = ca_x + ca_y, stage_cb = cb_x + cb_y;
  // TMA column boxes need 16-byte inner extents and x offsets: W complex of WR
  static constexpr bool col_ok = ((W * sizeof(cpx<WR>)) % 16 == 0) && (2 * stage_ca <= kMaxSmem) &&
                                 (2 * stage_cb <= kMaxSmem) && W >= 1 && 4 * W <= 256 && RB <= 256;
  static constexpr bool row_ok = (2 * stage_ra <= kMaxSmem) && (2 * stage_rb <= kMaxSmem);
};

struct ColMaps {
  CUtensorMap S, F, G;
};

// Uniform give-up path after a failed bounded wait: flag the instance, drain the
// copies of this CTA with bounded waits, leave.
// `k` is the item whose wait failed, `issued` the number of items from k on whose
// copies were issued (1 or 2).
__device__ __forceinline__ void pipe_timeout(int* status, uint64_t* bar, int k, int issued) {
  if (threadIdx.x == 0) {
    atomicExch(status, kStatusTimeout);
    for (int j = 0; j < issued; ++j) mbar_wait_bounded(&bar[(k + j) & 1], ((k + j) >> 1) & 1, kDrainLimitNs);
  }
  __syncthreads();
}

// instance status read once per CTA (uniform branch around barriers)
__device__ __forceinline__ bool instance_running(const int* status) {
  return !__syncthreads_or(threadIdx.x == 0 && *(volatile const int*)status != 0);
}

// =====================================================================================
// row A
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(kBlock, 2) k_row_a_p(const InstDev* __restrict__ insts, int count,
                                                    const int* __restrict__ base, int s_local) {
  using PG = PipeGeom<P, SR, WR>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = PG::G, tiles = PG::tiles_pairs;
  // under the drop_first_copy test knob, a launch after a timed-out one does not wait again
  if (insts[0].drop_first_copy && *(volatile const int*)insts[0].status) return;
  unsigned char* const smraw = pipe_stage_base();
  __shared__ uint64_t bar[2];
  __shared__ double red[160];
  __shared__ int lastflag;
  const int total = count * tiles;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!pipe_base_ok(smraw)) {
    if (threadIdx.x == 0 && (int)blockIdx.x < count) atomicExch(insts[0].status, kStatusLayout);
    return;
  }
  auto issue = [&](int w, int s) {
    const int inst = w / tiles, tile = w - inst * tiles;
    const InstDev& I = insts[inst];
    const int p0 = tile * G, np = min(G, H - p0);
    const uint32_t sb = (uint32_t)(2 * np * H * sizeof(cpx<SR>)), pb = (uint32_t)(2 * np * N * sizeof(WR));
    unsigned char* st = smraw + (size_t)s * PG::stage_ra;
    mbar_arrive_expect_tx(&bar[s], sb + pb);
    bulk_load(st, reinterpret_cast<const cpx<SR>*>(I.S) + (size_t)2 * p0 * H, sb, &bar[s]);
    bulk_load(st + PG::ra_x, reinterpret_cast<const WR*>(I.phi) + (size_t)2 * p0 * N, pb, &bar[s]);
  };
  if (threadIdx.x == 0) {
    // drop_first_copy (a test knob): withhold the first copy, so that its wait runs out
    if ((int)blockIdx.x < total && !insts[0].drop_first_copy) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < total) issue(blockIdx.x + gridDim.x, 1);
  }
  const int s_hist = step_index(base, s_local);
  int k = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x, ++k) {
    const int s = k & 1;
    unsigned char* st = smraw + (size_t)s * PG::stage_ra;
    const int inst = w / tiles, tile = w - inst * tiles;
    const InstDev& I = insts[inst];
    const bool ok = mbar_wait_bounded(&bar[s], (k >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      pipe_timeout(I.status, bar, k, ((w + (int)gridDim.x < total) ? 2 : 1));
      return;
    }
    if (instance_running(I.status)) {
      const int pair = tile * G + g;
      const bool active = pair < H;
      const cpx<SR>* ra = reinterpret_cast<const cpx<SR>*>(st) + (size_t)(2 * g) * H;
      const cpx<SR>* rb = ra + H;
      cpx<SR> v[E];
      if (active) {
        load_pair_rows<P, SR>(v, t, [&](int idx, cpx<SR>& a, cpx<SR>& b) {
          a = ra[idx];
          b = rb[idx];
        });
      } else {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = mkc<SR>(0, 0);
      }
      __syncthreads();  // region X is now the exchange buffer
      const RowLayout<N> lay{g * RowLayout<N>::stride};
      fft<true, P>(v, t, reinterpret_cast<cpx<SR>*>(st), lay, reinterpret_cast<const cpx<SR>*>(I.tw_s));
      const ModelParams mp = I.p;
      const SR invN = (SR)1 / (SR)N;
      const WR* pha = reinterpret_cast<const WR*>(st + PG::ra_x) + (size_t)(2 * g) * N;
      const WR* phb = pha + N;
      double sum_c = 0.0, sum_f = 0.0, mn = INFINITY, mx = -INFINITY, bad = 0.0;
      cpx<WR> wv[E];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int x = t + T * m;
        SR fa = 0, fb = 0;
        if (active) {
          const SR ca = v[m].x * invN, cb = v[m].y * invN;
          SR ea, eb;
          bulk<SR>(ca, (SR)pha[x], mp, fa, ea);
          bulk<SR>(cb, (SR)phb[x], mp, fb, eb);
          sum_c += (double)ca + (double)cb;
          sum_f += (double)ea + (double)eb;
          mn = fmin(mn, fmin((double)ca, (double)cb));
          mx = fmax(mx, fmax((double)ca, (double)cb));
          bad += (isfinite((double)ca) ? 0.0 : 1.0) + (isfinite((double)cb) ? 0.0 : 1.0);
        }
        wv[m] = mkc<WR>((WR)fa, (WR)fb);
      }
      fft<false, P>(wv, t, reinterpret_cast<cpx<WR>*>(st), lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      cpx<WR> xa[E / 2], xb[E / 2];
      split_rows<P, WR>(wv, t, reinterpret_cast<cpx<WR>*>(st), lay, xa, xb);
      if (active) {
        cpx<WR>* F = reinterpret_cast<cpx<WR>*>(I.F) + (size_t)(2 * pair) * H;
#pragma unroll
        for (int m = 0; m < E / 2; ++m) {
          F[t + T * m] = xa[m];
          F[H + t + T * m] = xb[m];
        }
      }
      block_reduce_ssmxs(sum_c, mn, mx, sum_f, bad, red);
      if (threadIdx.x == 0) {
        double* pp = I.part + (size_t)tile * 5;
        pp[0] = sum_c;
        pp[1] = mn;
        pp[2] = mx;
        pp[3] = sum_f;
        pp[4] = bad;
      }
      if (arrive_last(&I.cnt[0], tiles, &lastflag)) {
        const double a_sum = reduce_partials<OpSum>(I.part + 0, tiles, 5, 0.0, red);
        const double a_min = reduce_partials<OpMin>(I.part + 1, tiles, 5, INFINITY, red);
        const double a_max = reduce_partials<OpMax>(I.part + 2, tiles, 5, -INFINITY, red);
        const double a_f = reduce_partials<OpSum>(I.part + 3, tiles, 5, 0.0, red);
        const double a_bad = reduce_partials<OpSum>(I.part + 4, tiles, 5, 0.0, red);
        if (threadIdx.x == 0) {
          if (I.hist) {
            const size_t ld = (size_t)I.hist_ld;
            I.hist[s_hist] = (double)s_hist * I.dt;
            I.hist[s_hist + 1 * ld] = a_sum / ((double)N * N);
            I.hist[s_hist + 3 * ld] = a_min;
            I.hist[s_hist + 4 * ld] = a_max;
          }
          I.scal[0] = a_f;
          if (a_bad > 0.0) {
            *I.bad_step = s_hist;
            *I.status = kStatusNonFinite;
          }
          I.cnt[0] = 0;
        }
      }
    }
    __syncthreads();  // stage s fully consumed
    if (threadIdx.x == 0 && w + 2 * (int)gridDim.x < total) {
      fence_proxy_async_smem();
      issue(w + 2 * gridDim.x, s);
    }
  }
}

// =====================================================================================
// row B
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(kBlock, 2) k_row_b_p(const InstDev* __restrict__ insts, int count,
                                                    const int* __restrict__ base, int s_local) {
  using PG = PipeGeom<P, SR, WR>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = PG::G, tiles = PG::tiles_rows;
  // under the drop_first_copy test knob, a launch after a timed-out one does not wait again
  if (insts[0].drop_first_copy && *(volatile const int*)insts[0].status) return;
  unsigned char* const smraw = pipe_stage_base();
  __shared__ uint64_t bar[2];
  __shared__ double red[32];
  __shared__ int lastflag;
  const int total = count * tiles;
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!pipe_base_ok(smraw)) {
    if (threadIdx.x == 0 && (int)blockIdx.x < count) atomicExch(insts[0].status, kStatusLayout);
    return;
  }
  auto issue = [&](int w, int s) {
    const int inst = w / tiles, tile = w - inst * tiles;
    const InstDev& I = insts[inst];
    const int y0 = tile * G, ny = min(G, N - y0);
    const uint32_t gb = (uint32_t)(ny * H * sizeof(cpx2<WR>)), pb = (uint32_t)(ny * N * sizeof(WR));
    unsigned char* st = smraw + (size_t)s * PG::stage_rb;
    mbar_arrive_expect_tx(&bar[s], gb + pb);
    bulk_load(st, reinterpret_cast<const cpx2<WR>*>(I.G) + (size_t)y0 * H, gb, &bar[s]);
    bulk_load(st + PG::rb_x, reinterpret_cast<const WR*>(I.phi) + (size_t)y0 * N, pb, &bar[s]);
  };
  if (threadIdx.x == 0) {
    // drop_first_copy (a test knob): withhold the first copy, so that its wait runs out
    if ((int)blockIdx.x < total && !insts[0].drop_first_copy) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < total) issue(blockIdx.x + gridDim.x, 1);
  }
  const int s_hist = step_index(base, s_local);
  int k = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x, ++k) {
    const int s = k & 1;
    unsigned char* st = smraw + (size_t)s * PG::stage_rb;
    const int inst = w / tiles, tile = w - inst * tiles;
    const InstDev& I = insts[inst];
    const bool ok = mbar_wait_bounded(&bar[s], (k >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      pipe_timeout(I.status, bar, k, ((w + (int)gridDim.x < total) ? 2 : 1));
      return;
    }
    if (instance_running(I.status)) {
      const int y = tile * G + g;
      const bool active = y < N;
      const cpx2<WR>* row = reinterpret_cast<const cpx2<WR>*>(st) + (size_t)g * H;
      cpx<WR> v[E];
      if (active) {
        load_pair_rows<P, WR>(v, t, [&](int idx, cpx<WR>& a, cpx<WR>& b) {
          const cpx2<WR> q = row[idx];
          a = q.a;
          b = q.b;
        });
      } else {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = mkc<WR>(0, 0);
      }
      __syncthreads();
      const RowLayout<N> lay{g * RowLayout<N>::stride};
      cpx<WR>* xb_ = reinterpret_cast<cpx<WR>*>(st);
      fft<true, P>(v, t, xb_, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      const WR* ph = reinterpret_cast<const WR*>(st + PG::rb_x) + (size_t)g * N;
      const WR M0 = (WR)I.p.mobility;
      double dsum = 0.0;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        WR M = 0;
        if (active) {
          M = mobility_of<WR>(ph[t + T * m], M0);
          dsum += (double)M * ((double)v[m].x * v[m].x + (double)v[m].y * v[m].y);
        }
        v[m] = cscale(v[m], M);
      }
      fft<false, P>(v, t, xb_, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      cpx<WR> xa[E / 2], xbv[E / 2];
      split_rows<P, WR>(v, t, xb_, lay, xa, xbv);
      if (active) {
        cpx2<WR>* out = reinterpret_cast<cpx2<WR>*>(I.G) + (size_t)y * H;
#pragma unroll
        for (int m = 0; m < E / 2; ++m) {
          cpx2<WR> o;
          o.a = xa[m];
          o.b = xbv[m];
          out[t + T * m] = o;
        }
      }
      const double r = block_sum(dsum, red);
      double* part = I.part + (size_t)5 * PG::tiles_pairs + PG::tiles_cols;
      if (threadIdx.x == 0) part[tile] = r;
      if (arrive_last(&I.cnt[2], tiles, &lastflag)) {
        const double d = reduce_partials<OpSum>(part, tiles, 1, 0.0, red);
        if (threadIdx.x == 0) {
          if (I.hist) I.hist[s_hist + 5 * (size_t)I.hist_ld] = d * I.dx * I.dx;
          I.cnt[2] = 0;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && w + 2 * (int)gridDim.x < total) {
      fence_proxy_async_smem();
      issue(w + 2 * gridDim.x, s);
    }
  }
}

// =====================================================================================
// column A
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(PipeGeom<P, SR, WR>::CB, 2) k_col_a_p(const InstDev* __restrict__ insts, int count,
                                                    const int* __restrict__ base, int s_local,
                                                    const __grid_constant__ ColMaps maps) {
  using PG = PipeGeom<P, SR, WR>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = PG::W, tiles = PG::tiles_cols, RB = PG::RB;
  // under the drop_first_copy test knob, a launch after a timed-out one does not wait again
  if (insts[0].drop_first_copy && *(volatile const int*)insts[0].status) return;
  unsigned char* const smraw = pipe_stage_base();
  __shared__ uint64_t bar[2];
  __shared__ double red[32];
  __shared__ int lastflag;
  const int total = count * tiles;
  const int w_ = threadIdx.x % W, t = threadIdx.x / W;
  if (threadIdx.x == 0) {
    prefetch_tensormap(&maps.S);
    prefetch_tensormap(&maps.F);
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!pipe_base_ok(smraw)) {
    if (threadIdx.x == 0 && (int)blockIdx.x < count) atomicExch(insts[0].status, kStatusLayout);
    return;
  }
  auto issue = [&](int w, int s) {
    const int inst = w / tiles, tile = w - inst * tiles;
    unsigned char* st = smraw + (size_t)s * PG::stage_ca;
    mbar_arrive_expect_tx(&bar[s], (uint32_t)((size_t)N * W * (sizeof(cpx<SR>) + sizeof(cpx<WR>))));
    const int x0 = tile * W * 2;
#pragma unroll 1
    for (int r0 = 0; r0 < N; r0 += RB) {
      tma_load_3d(st + (size_t)r0 * W * sizeof(cpx<SR>), &maps.S, x0, r0, inst, &bar[s]);
      tma_load_3d(st + PG::ca_x + (size_t)r0 * W * sizeof(cpx<WR>), &maps.F, x0, r0, inst, &bar[s]);
    }
  };
  if (threadIdx.x == 0) {
    // drop_first_copy (a test knob): withhold the first copy, so that its wait runs out
    if ((int)blockIdx.x < total && !insts[0].drop_first_copy) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < total) issue(blockIdx.x + gridDim.x, 1);
  }
  const int s_hist = step_index(base, s_local);
  int k = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x, ++k) {
    const int s = k & 1;
    unsigned char* st = smraw + (size_t)s * PG::stage_ca;
    const int inst = w / tiles, tile = w - inst * tiles;
    const InstDev& I = insts[inst];
    const bool ok = mbar_wait_bounded(&bar[s], (k >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      pipe_timeout(I.status, bar, k, ((w + (int)gridDim.x < total) ? 2 : 1));
      return;
    }
    if (instance_running(I.status)) {
      const int kx = tile * W + w_;
      const bool active = kx < H;
      const ColLayout<W> lay{w_};
      const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * I.dx);
      const double kappa = I.p.kappa;
      cpx<SR> v[E];
      {
        const cpx<SR>* Sb = reinterpret_cast<const cpx<SR>*>(st);
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = active ? Sb[(t + T * m) * W + w_] : mkc<SR>(0, 0);
      }
      __syncthreads();  // region X becomes the exchange buffer
      cpx<SR>* sms = reinterpret_cast<cpx<SR>*>(st);
      fft<false, P>(v, t, sms, lay, reinterpret_cast<const cpx<SR>*>(I.tw_s));
      const bool packed_tile = tile == 0;
      const bool packed = packed_tile && w_ == 0;
      double gsum = 0.0;
      cpx<WR> u[E];
      const double kxf = kunit * (double)kx;
      const double kH2 = (kunit * (double)H) * (kunit * (double)H);
      if (packed_tile) {
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
      cpx<WR> a[E];
      {
        const cpx<WR>* Fb = reinterpret_cast<const cpx<WR>*>(st + PG::ca_x);
#pragma unroll
        for (int m = 0; m < E; ++m) a[m] = active ? Fb[(t + T * m) * W + w_] : mkc<WR>(0, 0);
      }
      cpx<WR>* smw = reinterpret_cast<cpx<WR>*>(st);
      fft<false, P>(a, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      const WR scale = (WR)(1.0 / ((double)N * (double)N));
      const WR kxd = (WR)kxf;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const WR kyd = (ky == H) ? (WR)0 : wavenumber<WR>(ky, N, kunit);
        const cpx<WR> mu = cscale(a[m] + u[m], scale);
        a[m] = times_i(cscale(mu, kxd));
        u[m] = times_i(cscale(mu, kyd));
      }
      fft<true, P>(a, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      fft<true, P>(u, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
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
      const double r = block_sum(gsum, red);
      double* part = I.part + (size_t)5 * PG::tiles_pairs;
      if (threadIdx.x == 0) part[tile] = r;
      if (arrive_last(&I.cnt[1], tiles, &lastflag)) {
        const double gr = reduce_partials<OpSum>(part, tiles, 1, 0.0, red);
        if (threadIdx.x == 0) {
          if (I.hist)
            I.hist[s_hist + 2 * (size_t)I.hist_ld] = (I.scal[0] + kappa * gr / ((double)N * N)) * I.dx * I.dx;
          I.cnt[1] = 0;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && w + 2 * (int)gridDim.x < total) {
      fence_proxy_async_smem();
      issue(w + 2 * gridDim.x, s);
    }
  }
}

// =====================================================================================
// column B
template <class P, typename SR, typename WR>
__global__ void __launch_bounds__(PipeGeom<P, SR, WR>::CB, 2) k_col_b_p(const InstDev* __restrict__ insts, int count,
                                                    const __grid_constant__ ColMaps maps) {
  using PG = PipeGeom<P, SR, WR>;
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = PG::W, tiles = PG::tiles_cols, RB = PG::RB;
  // under the drop_first_copy test knob, a launch after a timed-out one does not wait again
  if (insts[0].drop_first_copy && *(volatile const int*)insts[0].status) return;
  unsigned char* const smraw = pipe_stage_base();
  __shared__ uint64_t bar[2];
  __shared__ double red[32];
  const int total = count * tiles;
  const int w_ = threadIdx.x % W, t = threadIdx.x / W;
  if (threadIdx.x == 0) {
    prefetch_tensormap(&maps.G);
    prefetch_tensormap(&maps.S);  // used for L2 prefetch only
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!pipe_base_ok(smraw)) {
    if (threadIdx.x == 0 && (int)blockIdx.x < count) atomicExch(insts[0].status, kStatusLayout);
    return;
  }
  auto issue = [&](int w, int s) {
    const int inst = w / tiles, tile = w - inst * tiles;
    unsigned char* st = smraw + (size_t)s * PG::stage_cb;
    mbar_arrive_expect_tx(&bar[s], (uint32_t)((size_t)N * W * sizeof(cpx2<WR>)));
#pragma unroll 1
    for (int r0 = 0; r0 < N; r0 += RB) {
      tma_load_3d(st + (size_t)r0 * W * sizeof(cpx2<WR>), &maps.G, tile * W * 4, r0, inst, &bar[s]);
      tma_prefetch_l2_3d(&maps.S, tile * W * 2, r0, inst);
    }
  };
  if (threadIdx.x == 0) {
    // drop_first_copy (a test knob): withhold the first copy, so that its wait runs out
    if ((int)blockIdx.x < total && !insts[0].drop_first_copy) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < total) issue(blockIdx.x + gridDim.x, 1);
  }
  int k = 0;
  for (int w = blockIdx.x; w < total; w += gridDim.x, ++k) {
    const int s = k & 1;
    unsigned char* st = smraw + (size_t)s * PG::stage_cb;
    const int inst = w / tiles, tile = w - inst * tiles;
    const InstDev& I = insts[inst];
    const bool ok = mbar_wait_bounded(&bar[s], (k >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      pipe_timeout(I.status, bar, k, ((w + (int)gridDim.x < total) ? 2 : 1));
      return;
    }
    if (instance_running(I.status)) {
      const int kx = tile * W + w_;
      const bool active = kx < H;
      const ColLayout<W> lay{w_};
      const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * I.dx);
      cpx<WR> a[E], b[E];
      {
        const cpx2<WR>* Gb = reinterpret_cast<const cpx2<WR>*>(st);
#pragma unroll
        for (int m = 0; m < E; ++m) {
          if (active) {
            const cpx2<WR> o = Gb[(t + T * m) * W + w_];
            a[m] = o.a;
            b[m] = o.b;
          } else {
            a[m] = mkc<WR>(0, 0);
            b[m] = mkc<WR>(0, 0);
          }
        }
      }
      __syncthreads();
      cpx<WR>* smw = reinterpret_cast<cpx<WR>*>(st);
      fft<false, P>(a, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      fft<false, P>(b, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      const double c1 = 2.0 * I.p.Q * I.p.kappa * I.dt;
      const double kxf = kunit * (double)kx;
      const double kH2 = (kunit * (double)H) * (kunit * (double)H);
      const WR dtn = (WR)(I.dt / (double)N);
      const bool packed_tile = tile == 0;
      const bool packed = packed_tile && w_ == 0;
      if (packed_tile) {
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
          const WR iden = (WR)(1.0 / (1.0 + c1 * k2 * k2));
          const WR kyd = (ky == H) ? (WR)0 : (WR)kyf;
          const cpx<WR> div = times_i(cscale(a[m], kxd) + cscale(b[m], kyd));
          a[m] = cscale(div, iden * dtn);
        }
      }
      fft<true, P>(a, t, smw, lay, reinterpret_cast<const cpx<WR>*>(I.tw_w));
      double corr = 0.0;
      if (packed_tile) {
        double colsum = 0.0;
        if (packed) {
#pragma unroll
          for (int m = 0; m < E; ++m) colsum += (double)a[m].x;
        }
        const double tot = block_sum(colsum, red);
        if (packed) corr = tot / (double)N;
      }
      if (active) {
        cpx<SR>* S = reinterpret_cast<cpx<SR>*>(I.S);
#pragma unroll
        for (int m = 0; m < E; ++m) {
          cpx<SR>* sp = S + (size_t)(t + T * m) * H + kx;
          const cpx<SR> s0 = *sp;  // prefetched into L2 when the tile was issued
          *sp = mkc<SR>(s0.x + (SR)((double)a[m].x - corr), s0.y + (SR)a[m].y);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && w + 2 * (int)gridDim.x < total) {
      fence_proxy_async_smem();
      issue(w + 2 * gridDim.x, s);
    }
  }
}

}  // namespace esc
