// Cluster-resident run of one small grid (FP64): the whole time loop of
// run_simulation (core_shell.jl:84-103) in ONE launch of one thread-block
// cluster, with the state kept in the cluster's distributed shared memory.
//
// A single 256^2 or 128^2 particle gives each phase kernel of the launch-per-phase
// path only a few warps per SM, so its steps cost the latency of four dependent
// launches (about 10 us each) rather than their work.  Here C = 16 CTAs share
// the grid: CTA r owns rows y in [r R, r R + R),
// R = n / C, of the state S and of the pair array G (the f' transform F lives in
// the first half of G's slots, which column A reads before it writes them).  The
// four phases of a step are separated by hardware cluster barriers:
//   row A  (own rows, local shared memory)     -> F
//   col A  (own columns kx in [r n/2C, ...), every row gathered from the
//           owners' shared memory; results scattered back) -> G
//   row B  (own rows)                           -> G
//   col B  (own columns; S += increment written back to the owners) -> S
// History partials are folded after the barrier that follows their phase, in
// rank order, so every CTA sees the same totals; a non-finite composition stops
// the loop in every CTA at the same step (uniform control flow: every CTA
// executes the same barriers, none returns early).  The arithmetic per phase is
// that of the FP64 phase kernels (esc_kernels.cuh): the same FFT engine, bulk
// terms, packed DC/Nyquist column, energy, dissipation and DC mass fix.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <mutex>

#include "esc_cluster.h"
#include "esc_dispatch.cuh"

namespace cg = cooperative_groups;

namespace esc {
namespace clu {

// plan types of their own: the pass-major tables and their fill kernel are not
// shared with the 2-D kernel units (instances of one template in two units share
// a host stub)
template <class Base>
struct CPlan : Base {};

// Configuration per grid size: cluster size C and threads per CTA
template <int N>
struct Config;
template <>
struct Config<256> {  // 16 CTAs of 256 threads: row pairs and columns 32 threads x 8 elements, rows 16 x 16
  // (512 threads with 4- and 8-element plans measured slower: 42.1 against 36.4 us per step)
  static constexpr int C = 16, TH = 256;
  using A = CPlan<Plan<256, 8, Radices<8, 8, 4>>>;
  using B = CPlan<Plan<256, 16, Radices<16, 16>>>;
};
template <>
struct Config<128> {  // 16 CTAs of 128 threads: row pairs and columns 32 x 4, rows 16 x 8
  static constexpr int C = 16, TH = 128;
  using A = CPlan<Plan<128, 4, Radices<4, 4, 4, 2>>>;
  using B = CPlan<Plan<128, 8, Radices<8, 8, 2>>>;
};

template <int N>
struct Geo {
  static constexpr int C = Config<N>::C, TH = Config<N>::TH;
  static constexpr int H = N / 2, R = N / C, NP = R / 2, NC = H / C, NW = TH / 32;
  static constexpr int TA = TH / NP, TB = TH / R, TC = TH / NC;
};

// shared-memory layout of one CTA
template <int N>
struct Smem {
  using G_ = Geo<N>;
  static constexpr int H = G_::H, R = G_::R;
  static constexpr size_t s_elems = (size_t)R * H;                       // cpx<double>
  static constexpr size_t g_elems = (size_t)R * H;                       // cpx2<double>
  static constexpr size_t xa = (size_t)G_::NP * N;   // row A / init / final exchange (one swizzled line per group)
  static constexpr size_t xb = (size_t)R * N;          // row B exchange
  static constexpr size_t xc = (size_t)((N * G_::NC - 1) + ((N * G_::NC - 1) >> 4)) + 1;  // column exchange
  static constexpr size_t x_elems = xa > xb ? (xa > xc ? xa : xc) : (xb > xc ? xb : xc);
  static constexpr size_t off_g = s_elems * 16;
  static constexpr size_t off_x = off_g + g_elems * 32;
  static constexpr size_t off_part = off_x + x_elems * 16;
  static constexpr size_t part_doubles = 7 * G_::NW;  // per warp: row A's five sums, energy, dissipation
  static constexpr size_t bytes = off_part + part_doubles * 8;
};

// deterministic block sum (fixed order) of NV values over NW warps; result valid in thread 0
template <int NW, int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* red /* NW * NV */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) red[q * NW + wid] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int w = 0; w < NW; ++w) s += red[q * NW + w];
      v[q] = s;
    }
  }
  __syncthreads();
}
// full spectrum of two real rows a, b from their packed half spectra in shared memory
template <int N>
__device__ __forceinline__ cpx<double> pair_spectrum_sm(const cpx<double>* a, const cpx<double>* b, int k) {
  constexpr int H = N / 2;
  int idx = k <= H ? k : N - k;
  if (idx == H) idx = 0;
  const cpx<double> va = a[idx], vb = b[idx];
  if (k == 0) return mkc<double>(va.x, vb.x);
  if (k == H) return mkc<double>(va.y, vb.y);
  if (k < H) return mkc<double>(va.x - vb.y, va.y + vb.x);
  return mkc<double>(va.x + vb.y, vb.x - va.y);
}

// The persistent cluster kernel: c -> S, then steps s = 0..steps (history row s;
// the update only for s < steps), then S -> c.  One cluster of Config<N>::C CTAs.
template <int N>
__global__ void __launch_bounds__(Config<N>::TH, 1) k_cluster_run(const Args a) {
  using G_ = Geo<N>;
  using SM = Smem<N>;
  using PA = typename Config<N>::A;
  using PB = typename Config<N>::B;
  constexpr int C = G_::C, NW = G_::NW;
  constexpr int H = G_::H, R = G_::R, NC = G_::NC;
  constexpr int EA = PA::E, TA = PA::T, EB = PB::E, TB = PB::T;
  static_assert(TA == G_::TA && TB == G_::TB && TA == G_::TC, "plan geometry");
  static_assert(TA <= 32 && 32 % TA == 0 && TB <= 32 && 32 % TB == 0, "row groups inside one warp");
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[6 * NW];
  __shared__ double fold[8];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  cpx<double>* S = reinterpret_cast<cpx<double>*>(smraw);
  cpx2<double>* Gs = reinterpret_cast<cpx2<double>*>(smraw + SM::off_g);
  cpx<double>* X = reinterpret_cast<cpx<double>*>(smraw + SM::off_x);
  double* part = reinterpret_cast<double*>(smraw + SM::off_part);
  const int y0 = rank * R;
  const double invN = 1.0 / N, NN = (double)N * N;
  const ModelParams mp = a.p;

  // ---- c -> S: row pairs of this CTA (forward x-transform, split) ----
  {
    const int t = threadIdx.x % TA, pr = threadIdx.x / TA;
    const SwizzleLayout<N, sizeof(cpx<double>)> lay{pr * N, (int)((threadIdx.x & 31) / TA)};
    const int ya = y0 + 2 * pr;
    cpx<double> v[EA];
#pragma unroll
    for (int m = 0; m < EA; ++m) {
      const int x = t + TA * m;
      v[m] = mkc<double>(a.c[(size_t)ya * N + x], a.c[(size_t)(ya + 1) * N + x]);
    }
    fft<false, PA, WarpSync>(v, t, X, lay, PassTable<PA, double>{});
    cpx<double> xa[EA / 2], xb[EA / 2];
    split_rows<PA, double>(v, t, X, RowLayout<N>{0}, xa, xb);
#pragma unroll
    for (int m = 0; m < EA / 2; ++m) {
      S[(size_t)(2 * pr) * H + t + TA * m] = xa[m];
      S[(size_t)(2 * pr + 1) * H + t + TA * m] = xb[m];
    }
  }
  cl.sync();

  bool stopped = false;
  for (int s = 0; s <= a.steps; ++s) {
    // ---- row A: c, bulk terms, history partials, F = x-FFT(f') into G.a ----
    {
      const int t = threadIdx.x % TA, pr = threadIdx.x / TA;
      const SwizzleLayout<N, sizeof(cpx<double>)> lay{pr * N, (int)((threadIdx.x & 31) / TA)};
      const int la = 2 * pr, ya = y0 + la;
      cpx<double> v[EA];
#pragma unroll
      for (int m = 0; m < EA; ++m) v[m] = pair_spectrum_sm<N>(S + (size_t)la * H, S + (size_t)(la + 1) * H, t + TA * m);
      fft<true, PA, WarpSync>(v, t, X, lay, PassTable<PA, double>{});
      double sc = 0.0, sf = 0.0, mn = INFINITY, mx = -INFINITY, bad = 0.0;
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int x = t + TA * m;
        const double ca = v[m].x * invN, cb = v[m].y * invN;
        double fa, fb, ea, eb;
        bulk<double>(ca, __ldg(a.phi + (size_t)ya * N + x), mp, fa, ea);
        bulk<double>(cb, __ldg(a.phi + (size_t)(ya + 1) * N + x), mp, fb, eb);
        sc += ca + cb;
        sf += ea + eb;
        mn = fmin(mn, fmin(ca, cb));
        mx = fmax(mx, fmax(ca, cb));
        bad += (double)((int)nonfinite_bits(ca) + (int)nonfinite_bits(cb));
        v[m] = mkc<double>(fa, fb);
      }
      __syncwarp();
      fft<false, PA, WarpSync>(v, t, X, lay, PassTable<PA, double>{});
      cpx<double> xa[EA / 2], xb[EA / 2];
      split_rows<PA, double>(v, t, X, RowLayout<N>{0}, xa, xb);
#pragma unroll
      for (int m = 0; m < EA / 2; ++m) {
        Gs[(size_t)la * H + t + TA * m].a = xa[m];
        Gs[(size_t)(la + 1) * H + t + TA * m].a = xb[m];
      }
      // per-warp partials; the fold after the cluster barrier combines them
      sc = warp_sum(sc);
      sf = warp_sum(sf);
      bad = warp_sum(bad);
      mn = warp_min(mn);
      mx = warp_max(mx);
      if ((threadIdx.x & 31) == 0) {
        const int wid = threadIdx.x >> 5;
        part[0 * NW + wid] = sc;
        part[1 * NW + wid] = mn;
        part[2 * NW + wid] = mx;
        part[3 * NW + wid] = sf;
        part[4 * NW + wid] = bad;
      }
    }
    cl.sync();
    // fold row A's partials in rank order (every CTA the same totals)
    if (threadIdx.x < 32) {
      // lane l folds slots l, l + 32, ... of the C * NW (rank, warp) partials, then a
      // fixed shuffle tree: the same order, hence the same bits, in every CTA
      double tsum = 0.0, tmin = INFINITY, tmax = -INFINITY, tf = 0.0, tbad = 0.0;
      for (int i = threadIdx.x; i < C * NW; i += 32) {
        const double* q = cl.map_shared_rank(part, i / NW);
        const int wq = i % NW;
        tsum += q[0 * NW + wq];
        tmin = fmin(tmin, q[1 * NW + wq]);
        tmax = fmax(tmax, q[2 * NW + wq]);
        tf += q[3 * NW + wq];
        tbad += q[4 * NW + wq];
      }
      tsum = warp_sum(tsum);
      tf = warp_sum(tf);
      tbad = warp_sum(tbad);
      tmin = warp_min(tmin);
      tmax = warp_max(tmax);
      if (threadIdx.x == 0) {
        fold[0] = tsum;
        fold[1] = tmin;
        fold[2] = tmax;
        fold[3] = tf;
        fold[4] = tbad;
        if (rank == 0) {
          const size_t ld = (size_t)a.hist_ld;
          if (a.hist) {
            a.hist[s] = (double)s * a.dt;
            a.hist[s + ld] = tsum / NN;
            a.hist[s + 3 * ld] = tmin;
            a.hist[s + 4 * ld] = tmax;
          }
          if (tbad > 0.0) {
            *a.bad_step = s;
            *a.status = kStatusNonFinite;
          }
        }
      }
    }
    __syncthreads();
    if (fold[4] > 0.0) {  // the same value in every CTA: uniform exit from the loop
      stopped = true;
      break;
    }
    // ---- col A: y-FFT of S and F (gathered from every CTA), energy, mu^,
    //      derivatives, inverse y-FFT; G scattered back to the owners ----
    {
      const int w = threadIdx.x % NC, t = threadIdx.x / NC;
      const int kx = rank * NC + w;
      const ColLayout<NC> lay{w};
      const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * a.dx);
      const double kappa = mp.kappa;
      cpx<double> v[EA];
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int y = t + TA * m;
        const cpx<double>* src = cl.map_shared_rank(S, y / R);
        v[m] = src[(size_t)(y % R) * H + kx];
      }
      fft<false, PA>(v, t, X, lay, PassTable<PA, double>{});
      const bool packed = kx == 0;  // holds kx = 0 (DC + i Nyquist)
      double gsum = 0.0;
      cpx<double> u[EA];
      const double kxf = kunit * (double)kx;
      const double kH2 = (kunit * (double)H) * (kunit * (double)H);
      if (rank == 0) {  // the packed column's partner exchange (one column of CTA 0)
        if (packed) {
#pragma unroll
          for (int m = 0; m < EA; ++m) X[t + TA * m] = v[m];
        }
        __syncthreads();
        if (packed) {
#pragma unroll
          for (int m = 0; m < EA; ++m) {
            const int ky = t + TA * m;
            const cpx<double> pr = cconj(X[(N - ky) % N]);
            const double kyf = kunit * (double)(ky < H ? ky : ky - N);
            const double k2a = kyf * kyf;
            const cpx<double> Ac = cscale(v[m] + pr, 0.5);
            const cpx<double> Bc = cscale(times_negi(v[m] - pr), 0.5);
            gsum += k2a * (Ac.x * Ac.x + Ac.y * Ac.y) + (k2a + kH2) * (Bc.x * Bc.x + Bc.y * Bc.y);
            u[m] = cscale(v[m], 2.0 * kappa * k2a) + times_i(cscale(Bc, 2.0 * kappa * kH2));
          }
        }
        __syncthreads();
      }
      if (!packed) {
#pragma unroll
        for (int m = 0; m < EA; ++m) {
          const int ky = t + TA * m;
          const double kyf = kunit * (double)(ky < H ? ky : ky - N);
          const double k2 = kxf * kxf + kyf * kyf;
          gsum += 2.0 * k2 * (v[m].x * v[m].x + v[m].y * v[m].y);
          u[m] = cscale(v[m], 2.0 * kappa * k2);
        }
      }
      // f'^ = y-FFT(F), F held in G.a of the owners
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int y = t + TA * m;
        const cpx2<double>* src = cl.map_shared_rank(Gs, y / R);
        v[m] = src[(size_t)(y % R) * H + kx].a;
      }
      fft<false, PA>(v, t, X, lay, PassTable<PA, double>{});
      const double scale = 1.0 / NN;
      cpx<double> gy[EA];
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int ky = t + TA * m;
        const double kyd = (ky == H) ? 0.0 : kunit * (double)(ky < H ? ky : ky - N);
        const cpx<double> mu = cscale(v[m] + u[m], scale);
        v[m] = times_i(cscale(mu, kxf));  // x-derivative (kx < n/2: never the Nyquist)
        gy[m] = times_i(cscale(mu, kyd));  // y-derivative, the Nyquist zeroed
      }
      fft<true, PA>(v, t, X, lay, PassTable<PA, double>{});
      fft<true, PA>(gy, t, X, lay, PassTable<PA, double>{});
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int y = t + TA * m;
        cpx2<double>* dst = cl.map_shared_rank(Gs, y / R);
        cpx2<double> o;
        o.a = v[m];
        o.b = gy[m];
        dst[(size_t)(y % R) * H + kx] = o;
      }
      gsum = warp_sum(gsum);
      if ((threadIdx.x & 31) == 0) part[5 * NW + (threadIdx.x >> 5)] = gsum;
    }
    cl.sync();
    if (threadIdx.x < 32 && rank == 0) {
      double gr = 0.0;
      for (int i = threadIdx.x; i < C * NW; i += 32) gr += cl.map_shared_rank(part, i / NW)[5 * NW + i % NW];
      gr = warp_sum(gr);
      if (threadIdx.x == 0 && a.hist) a.hist[s + 2 * (size_t)a.hist_ld] = (fold[3] + mp.kappa * gr / NN) * a.dx * a.dx;
    }
    // ---- row B: grad mu of own rows, M = M0 h(phi), dissipation, M grad mu -> G ----
    {
      const int t = threadIdx.x % TB, ry = threadIdx.x / TB;
      const SwizzleLayout<N, sizeof(cpx<double>)> lay{ry * N, (int)((threadIdx.x & 31) / TB)};
      const int y = y0 + ry;
      cpx2<double>* row = Gs + (size_t)ry * H;
      cpx<double> v[EB];
#pragma unroll
      for (int m = 0; m < EB; ++m) {
        const int k = t + TB * m;
        int idx = k <= H ? k : N - k;
        if (idx == H) idx = 0;
        const cpx<double> va = row[idx].a, vb = row[idx].b;
        if (k == 0)
          v[m] = mkc<double>(va.x, vb.x);
        else if (k == H)
          v[m] = mkc<double>(va.y, vb.y);
        else if (k < H)
          v[m] = mkc<double>(va.x - vb.y, va.y + vb.x);
        else
          v[m] = mkc<double>(va.x + vb.y, vb.x - va.y);
      }
      fft<true, PB, WarpSync>(v, t, X, lay, PassTable<PB, double>{});
      double dsum = 0.0;
#pragma unroll
      for (int m = 0; m < EB; ++m) {
        const double M = mobility_of<double>(__ldg(a.phi + (size_t)y * N + t + TB * m), mp.mobility);
        dsum += M * (v[m].x * v[m].x + v[m].y * v[m].y);
        v[m] = cscale(v[m], M);
      }
      __syncwarp();
      fft<false, PB, WarpSync>(v, t, X, lay, PassTable<PB, double>{});
      cpx<double> xa[EB / 2], xb[EB / 2];
      split_rows<PB, double>(v, t, X, RowLayout<N>{0}, xa, xb);
#pragma unroll
      for (int m = 0; m < EB / 2; ++m) {
        cpx2<double> o;
        o.a = xa[m];
        o.b = xb[m];
        row[t + TB * m] = o;
      }
      dsum = warp_sum(dsum);
      if ((threadIdx.x & 31) == 0) part[6 * NW + (threadIdx.x >> 5)] = dsum;
    }
    cl.sync();
    if (threadIdx.x < 32 && rank == 0) {
      double d = 0.0;
      for (int i = threadIdx.x; i < C * NW; i += 32) d += cl.map_shared_rank(part, i / NW)[6 * NW + i % NW];
      d = warp_sum(d);
      if (threadIdx.x == 0 && a.hist) a.hist[s + 5 * (size_t)a.hist_ld] = d * a.dx * a.dx;
    }
    if (s == a.steps) break;  // the last history row: no update

    // ---- col B: y-FFT of the fluxes, divergence, stabilised increment, inverse
    //      y-FFT, S += increment written back to the owners ----
    {
      const int w = threadIdx.x % NC, t = threadIdx.x / NC;
      const int kx = rank * NC + w;
      const ColLayout<NC> lay{w};
      const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * a.dx);
      cpx<double> fa[EA], fb[EA];
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int y = t + TA * m;
        const cpx2<double> o = cl.map_shared_rank(Gs, y / R)[(size_t)(y % R) * H + kx];
        fa[m] = o.a;
        fb[m] = o.b;
      }
      fft<false, PA>(fa, t, X, lay, PassTable<PA, double>{});
      fft<false, PA>(fb, t, X, lay, PassTable<PA, double>{});
      const double c1 = 2.0 * mp.Q * mp.kappa * a.dt;
      const double kxf = kunit * (double)kx;
      const double kH2 = (kunit * (double)H) * (kunit * (double)H);
      const double dtn = a.dt / (double)N;
      const bool packed = kx == 0;
      if (rank == 0) {
        if (packed) {
#pragma unroll
          for (int m = 0; m < EA; ++m) X[t + TA * m] = fb[m];
        }
        __syncthreads();
        if (packed) {
#pragma unroll
          for (int m = 0; m < EA; ++m) {
            const int ky = t + TA * m;
            const cpx<double> pr = cconj(X[(N - ky) % N]);
            const double kyf = kunit * (double)(ky < H ? ky : ky - N);
            const double k2a = kyf * kyf, k2b = k2a + kH2;
            const double ida = 1.0 / (1.0 + c1 * k2a * k2a), idb = 1.0 / (1.0 + c1 * k2b * k2b);
            const double kyd = (ky == H) ? 0.0 : kyf;
            const cpx<double> Ay = cscale(fb[m] + pr, 0.5);
            const cpx<double> By = cscale(times_negi(fb[m] - pr), 0.5);
            const cpx<double> q = cscale(Ay, ida) + times_i(cscale(By, idb));
            fa[m] = times_i(cscale(q, kyd * dtn));
          }
        }
        __syncthreads();
      }
      if (!packed) {
#pragma unroll
        for (int m = 0; m < EA; ++m) {
          const int ky = t + TA * m;
          const double kyf = kunit * (double)(ky < H ? ky : ky - N);
          const double k2 = kxf * kxf + kyf * kyf;
          const double iden = 1.0 / (1.0 + c1 * k2 * k2);
          const double kyd = (ky == H) ? 0.0 : kyf;
          const cpx<double> div = times_i(cscale(fa[m], kxf) + cscale(fb[m], kyd));
          fa[m] = cscale(div, iden * dtn);
        }
      }
      fft<true, PA>(fa, t, X, lay, PassTable<PA, double>{});
      // exact mass conservation: the DC row-mode increments (packed column, real
      // part) sum to zero over y; the rounding residue is removed in FP64
      double colsum[1] = {0.0};
      if (packed) {
#pragma unroll
        for (int m = 0; m < EA; ++m) colsum[0] += fa[m].x;
      }
      block_sums<NW, 1>(colsum, red);
      if (threadIdx.x == 0) fold[5] = colsum[0];
      __syncthreads();
      const double corr = packed ? fold[5] / (double)N : 0.0;
#pragma unroll
      for (int m = 0; m < EA; ++m) {
        const int y = t + TA * m;
        cpx<double>* dst = cl.map_shared_rank(S, y / R) + (size_t)(y % R) * H + kx;
        const cpx<double> s0 = *dst;
        *dst = mkc<double>(s0.x + (fa[m].x - corr), s0.y + fa[m].y);
      }
    }
    cl.sync();
  }

  // ---- S -> c (own row pairs), unless the run stopped on a non-finite field ----
  if (!stopped) {
    const int t = threadIdx.x % TA, pr = threadIdx.x / TA;
    const SwizzleLayout<N, sizeof(cpx<double>)> lay{pr * N, (int)((threadIdx.x & 31) / TA)};
    const int la = 2 * pr, ya = y0 + la;
    cpx<double> v[EA];
#pragma unroll
    for (int m = 0; m < EA; ++m) v[m] = pair_spectrum_sm<N>(S + (size_t)la * H, S + (size_t)(la + 1) * H, t + TA * m);
    fft<true, PA, WarpSync>(v, t, X, lay, PassTable<PA, double>{});
#pragma unroll
    for (int m = 0; m < EA; ++m) {
      const int x = t + TA * m;
      a.c[(size_t)ya * N + x] = v[m].x * invN;
      a.c[(size_t)(ya + 1) * N + x] = v[m].y * invN;
    }
  }
  // no CTA leaves while another may still read its shared memory
  cl.sync();
}

// ---- host side -----------------------------------------------------------------------
template <int N>
struct Launcher {
  using PA = typename Config<N>::A;
  using PB = typename Config<N>::B;
  static constexpr int C = Config<N>::C, TH = Config<N>::TH;
  static constexpr size_t kSmem = Smem<N>::bytes;
  static cudaLaunchConfig_t config(cudaStream_t st, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(TH, 1, 1);
    cfg.dynamicSmemBytes = kSmem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
  }
  static cudaError_t attributes() {
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_cluster_run<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem)))
      return e;
    if (C > 8 && (e = cudaFuncSetAttribute(k_cluster_run<N>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)))
      return e;
    return cudaSuccess;
  }
  static bool available() {
    if (attributes() != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = config(nullptr, attr);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_cluster_run<N>, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return clusters >= 1;
  }
  static cudaError_t prepare(const void* tw, cudaStream_t st) {
    cudaError_t e;
    if ((e = attributes())) return e;
    k_fill_pass_tw<PA, double><<<1, 256, 0, st>>>(static_cast<const cpx<double>*>(tw));
    k_fill_pass_tw<PB, double><<<1, 256, 0, st>>>(static_cast<const cpx<double>*>(tw));
    return cudaGetLastError();
  }
  static cudaError_t run(const Args& a, cudaStream_t st) {
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = config(st, attr);
    return cudaLaunchKernelEx(&cfg, k_cluster_run<N>, a);
  }
};

std::mutex& avail_mutex() {
  static std::mutex m;
  return m;
}

}  // namespace clu

namespace clu {

bool available(int n) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  static signed char cache[64][2] = {};  // 0 unknown, 1 yes, -1 no; [dev][size index]
  const int si = n == 256 ? 0 : (n == 128 ? 1 : -1);
  if (si < 0) return false;
  std::lock_guard<std::mutex> lock(avail_mutex());
  if (!cache[dev][si]) cache[dev][si] = (si == 0 ? Launcher<256>::available() : Launcher<128>::available()) ? 1 : -1;
  return cache[dev][si] > 0;
}

cudaError_t prepare(int n, const void* tw, cudaStream_t st) {
  if (n == 256) return Launcher<256>::prepare(tw, st);
  if (n == 128) return Launcher<128>::prepare(tw, st);
  return cudaErrorInvalidValue;
}

cudaError_t run(int n, const Args& a, cudaStream_t st) {
  if (n == 256) return Launcher<256>::run(a, st);
  if (n == 128) return Launcher<128>::run(a, st);
  return cudaErrorInvalidValue;
}

}  // namespace clu
}  // namespace esc
