// Adjoint (transposed) step of the stabilised Fourier update, FP64.
//
// With S = IFFT diag(1/den) FFT, L = -IFFT diag(k^2) FFT and
// mu = f'(c) - 2 kappa L c, one forward step is c' = c + dt S div(M grad mu(c)).
// Every operator is real and S, L, div(M grad .) are symmetric, so the
// transposed step that maps lam = dLoss/dc' to dLoss/dc is
//     a = dt S lam,   g = div(M grad a),   lam_prev = lam + f''(c) g - 2 kappa L g,
// and the step's sensitivities to theta = (P, chi, kappa, M0) are
//     P: sum g (-chi gphi)     chi: sum g (-P gphi)
//     kappa: sum g IFFT(2 k^2 c^) + sum lam IFFT((c'^ - c^)(-2 Q k^4 dt)/den)
//     M0: sum lam (c' - c) / M0          (the update is linear in M0).
// Four passes per adjoint step, mirroring the forward kernels:
//   col 1 : y-FFT(Lam), y-FFT(S' - S) ; kappa(den) and M0 sums ; i k dt lam^/den -> G
//   row B : (forward kernel k_row_b) M grad a -> G
//   col 2 : y-FFT(G) -> g^ ; y-FFT(S) ; kappa(mu) sum ; Xg = x-transform of g ;
//           Lam += x-transform of IFFT(2 kappa k^2 g^)
//   row 2 : c and g in real space ; P, chi sums ; Lam += x-FFT(f''(c) g)
// Lam is the adjoint in the mixed (kx, y) domain with the packing of the state.
// Sums are reduced per block, folded by the last block and added to the
// per-instance accumulator `acc` (so successive steps add in a fixed order).
#pragma once
#include "esc_kernels.cuh"

namespace esc {

// Adjoint-side descriptor (device resident, one per instance).
struct AdjDev {
  int n;
  double dx, dt, lamF;
  ModelParams p;
  const double2* S0;   // state c_s      (mixed domain, packed)
  const double2* S1;   // state c_{s+1}
  double2* Lam;        // adjoint (mixed domain, packed)
  double2* Xg;         // x-transform of g (or of mu for the seed)
  const double2* F;    // x-transform of f'(c) (seed only)
  cpx2<double>* G;     // pair array (grad a, then M grad a)
  const double* phi;
  const double* target;  // c_target (real, seed only)
  const void* tw;      // twiddles (FP64)
  double* part;
  unsigned* cnt;       // arrival counters [4]
  double* acc;         // [0] P [1] chi [2] kappa [3] M0 [4] 1/2 sum (c-ct)^2 [5] sum (1-chi c) gphi [6] sum c gphi
  // mixed-precision step kernels (the _m kernels below) only
  cpx2<float>* Gw;     // FP32 pair array (grad a, then M grad a)
  cpx<float>* Xw;      // FP32 x-transform of g
  const float* phiw;   // FP32 particle field
};

template <typename R>
__device__ __forceinline__ R fpp_of(R c, R phi, const ModelParams& p) {
  const R h = phi * phi * phi * ((R)10 - (R)15 * phi + (R)6 * phi * phi);
  const R e = (R)2 * c - (R)p.cb - (R)p.cc;
  const R db = c - (R)p.cb, dc = c - (R)p.cc;
  return (R)2 * (R)p.A * ((R)1 - h) + (R)2 * (R)p.B * h * (dc * e + db * e + (R)2 * db * dc);
}
__device__ __forceinline__ double gphi_of(double phi) { return phi * phi * (1.0 - phi) * (1.0 - phi); }

// block_reduce<OpSum> of NV values at once (same shuffle trees, same bits); red
// holds 32 doubles per value
template <int NV>
__device__ __forceinline__ void block_reduce_n(double (&v)[NV], double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) red[32 * q + wid] = v[q];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      v[q] = (lane < (int)(blockDim.x >> 5)) ? red[32 * q + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) red[32 * q] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = red[32 * q];
  __syncthreads();
}

// fold this block's values into acc[slot..] once every block has arrived
template <int NV>
__device__ __forceinline__ void adj_accumulate(const AdjDev& A, int counter, int part_off, const double (&v)[NV],
                                               const int (&slot)[NV], double* red, int* flag) {
  double r[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) r[q] = v[q];
  block_reduce_n(r, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) A.part[part_off + (size_t)blockIdx.x * NV + q] = r[q];
  }
  if (!arrive_last(&A.cnt[counter], gridDim.x, flag)) return;
  // the NV folds of reduce_partials, in one pass (same order, same bits)
  double tot[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) tot[q] = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] += __ldcg(A.part + part_off + (size_t)i * NV + q);
  }
  block_reduce_n(tot, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) A.acc[slot[q]] += tot[q];
    A.cnt[counter] = 0;
  }
}

// ---- column 1 -------------------------------------------------------------------------
template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 2 : 1)) k_adj_col1(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeom<P>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const PassTable<P, double> tw{};  // pass-major copy of the FP64 table A.tw
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * A.dx);
  const double c1 = 2.0 * A.p.Q * A.p.kappa * A.dt;
  cpx<double> l[E], d[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const size_t o = (size_t)(t + T * m) * H + kx;
    if (active) {
      const double2 a = A.Lam[o], s0 = A.S0[o], s1 = A.S1[o];
      l[m] = mkc<double>(a.x, a.y);
      d[m] = mkc<double>(s1.x - s0.x, s1.y - s0.y);
    } else {
      l[m] = mkc<double>(0, 0);
      d[m] = mkc<double>(0, 0);
    }
  }
  fft<false, P>(l, t, sm, lay, tw);
  fft<false, P>(d, t, sm, lay, tw);
  const bool packed_tile = blockIdx.x == 0, packed = packed_tile && w == 0;
  const double kxf = kunit * (double)kx, kH2 = (kunit * H) * (kunit * H);
  const double invNN = 1.0 / ((double)N * N);
  double s_kap = 0.0, s_m0 = 0.0;
  cpx<double> gx[E], gy[E];
  if (packed_tile) {
    // separate the packed (kx = 0, kx = n/2) columns of lam^ and dc^
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sm[t + T * m] = l[m];
    }
    __syncthreads();
    cpx<double> lB[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const cpx<double> pr = packed ? cconj(sm[(N - ky) % N]) : mkc<double>(0, 0);
      lB[m] = cscale(times_negi(l[m] - pr), 0.5);
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sm[t + T * m] = d[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<double> pd = cconj(sm[(N - ky) % N]);
        const cpx<double> dA = cscale(d[m] + pd, 0.5), dB = cscale(times_negi(d[m] - pd), 0.5);
        // lam_A = lam_P - i lam_B
        const cpx<double> lA = l[m] - times_i(lB[m]);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf, k2b = k2a + kH2;
        const double dena = 1.0 + c1 * k2a * k2a, denb = 1.0 + c1 * k2b * k2b;
        const double reA = lA.x * dA.x + lA.y * dA.y, reB = lB[m].x * dB.x + lB[m].y * dB.y;
        s_m0 += (reA + reB) * invNN;
        s_kap += (reA * (-2.0 * A.p.Q * k2a * k2a * A.dt / dena) + reB * (-2.0 * A.p.Q * k2b * k2b * A.dt / denb)) * invNN;
        // a^ packed = dt (lam_A/den_A + i lam_B/den_B); x-derivative vanishes on both columns
        const cpx<double> ah = cscale(lA, A.dt / dena) + times_i(cscale(lB[m], A.dt / denb));
        const double kyd = (ky == H) ? 0.0 : kyf;
        gx[m] = mkc<double>(0, 0);
        gy[m] = times_i(cscale(ah, kyd * invNN));
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
      const double den = 1.0 + c1 * k2 * k2;
      const double re = l[m].x * d[m].x + l[m].y * d[m].y;
      if (active) {
        s_m0 += 2.0 * re * invNN;
        s_kap += 2.0 * re * (-2.0 * A.p.Q * k2 * k2 * A.dt / den) * invNN;
      }
      const cpx<double> ah = cscale(l[m], A.dt / den);
      const double kyd = (ky == H) ? 0.0 : kyf;
      gx[m] = times_i(cscale(ah, kxf * invNN));
      gy[m] = times_i(cscale(ah, kyd * invNN));
    }
  }
  fft<true, P>(gx, t, sm, lay, tw);
  fft<true, P>(gy, t, sm, lay, tw);
  if (active) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      cpx2<double> o;
      o.a = gx[m];
      o.b = gy[m];
      A.G[(size_t)(t + T * m) * H + kx] = o;
    }
  }
  const double vals[2] = {s_kap, s_m0 / A.p.mobility};
  const int slots[2] = {2, 3};
  adj_accumulate<2>(A, 0, 0, vals, slots, red, &lastflag);
}

// ---- column 2 -------------------------------------------------------------------------
template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 2 : 1)) k_adj_col2(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeom<P>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const PassTable<P, double> tw{};  // pass-major copy of the FP64 table A.tw
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * A.dx);
  cpx<double> fx[E], fy[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    if (active) {
      const cpx2<double> o = A.G[(size_t)(t + T * m) * H + kx];
      fx[m] = o.a;
      fy[m] = o.b;
    } else {
      fx[m] = mkc<double>(0, 0);
      fy[m] = mkc<double>(0, 0);
    }
  }
  fft<false, P>(fx, t, sm, lay, tw);
  fft<false, P>(fy, t, sm, lay, tw);
  const double kxf = kunit * (double)kx, kH2 = (kunit * H) * (kunit * H);
  // g^ = i kx F(M dx a) + i ky F(M dy a); on the packed column only the y part survives
  const bool packed_tile = blockIdx.x == 0, packed = packed_tile && w == 0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int ky = t + T * m;
    const double kyd = (ky == H) ? 0.0 : kunit * (double)(ky < H ? ky : ky - N);
    const double kxd = packed ? 0.0 : kxf;
    fx[m] = times_i(cscale(fx[m], kxd) + cscale(fy[m], kyd));  // fx now holds g^
  }
  // c^ = y-FFT(S)
  cpx<double> ch[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const double2 s = active ? A.S0[(size_t)(t + T * m) * H + kx] : make_double2(0, 0);
    ch[m] = mkc<double>(s.x, s.y);
  }
  fft<false, P>(ch, t, sm, lay, tw);
  const double invNN = 1.0 / ((double)N * N), invN = 1.0 / (double)N;
  const double kappa = A.p.kappa;
  double s_kap = 0.0;
  if (packed_tile) {
    cpx<double> gB[E];
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sm[t + T * m] = fx[m];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const cpx<double> pr = packed ? cconj(sm[(N - ky) % N]) : mkc<double>(0, 0);
      gB[m] = cscale(times_negi(fx[m] - pr), 0.5);
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sm[t + T * m] = ch[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<double> pc = cconj(sm[(N - ky) % N]);
        const cpx<double> cA = cscale(ch[m] + pc, 0.5), cB = cscale(times_negi(ch[m] - pc), 0.5);
        const cpx<double> gA = fx[m] - times_i(gB[m]);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf, k2b = k2a + kH2;
        s_kap += (2.0 * k2a * (gA.x * cA.x + gA.y * cA.y) + 2.0 * k2b * (gB[m].x * cB.x + gB[m].y * cB.y)) * invNN;
        // U = 2 kappa (k2a g_A + i k2b g_B) = 2 kappa (k2a g_P + i kH2 g_B)
        ch[m] = cscale(cscale(fx[m], 2.0 * kappa * k2a) + times_i(cscale(gB[m], 2.0 * kappa * kH2)), invN);
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
      if (active) s_kap += 2.0 * 2.0 * k2 * (fx[m].x * ch[m].x + fx[m].y * ch[m].y) * invNN;
      ch[m] = cscale(fx[m], 2.0 * kappa * k2 * invN);  // ch now holds U / n
    }
  }
#pragma unroll
  for (int m = 0; m < E; ++m) fx[m] = cscale(fx[m], invN);
  fft<true, P>(fx, t, sm, lay, tw);
  fft<true, P>(ch, t, sm, lay, tw);
  if (active) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const size_t o = (size_t)(t + T * m) * H + kx;
      A.Xg[o] = make_double2(fx[m].x, fx[m].y);
      const double2 l = A.Lam[o];
      A.Lam[o] = make_double2(l.x + ch[m].x, l.y + ch[m].y);
    }
  }
  const double vals[1] = {s_kap};
  const int slots[1] = {2};
  adj_accumulate<1>(A, 1, 0, vals, slots, red, &lastflag);
}

// ---- row 2 ----------------------------------------------------------------------------
template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 2 : 1)) k_adj_row2(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;
  const RowLayout<N> lay{g * RowLayout<N>::stride};
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const PassTable<P, double> tw{};  // pass-major copy of the FP64 table A.tw
  const cpx<double>* Xg = reinterpret_cast<const cpx<double>*>(A.Xg);
  const cpx<double>* S = reinterpret_cast<const cpx<double>*>(A.S0);
  cpx<double> gv[E], cv[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    gv[m] = active ? load_pair_spectrum<double, N>(Xg + (size_t)ya * H, Xg + (size_t)(ya + 1) * H, t + T * m)
                   : mkc<double>(0, 0);
    cv[m] = active ? load_pair_spectrum<double, N>(S + (size_t)ya * H, S + (size_t)(ya + 1) * H, t + T * m)
                   : mkc<double>(0, 0);
  }
  fft<true, P>(gv, t, sm, lay, tw);
  fft<true, P>(cv, t, sm, lay, tw);
  const double invN = 1.0 / (double)N;
  double sP = 0.0, sChi = 0.0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    double ha = 0.0, hb = 0.0;
    if (active) {
      const double pa = A.phi[(size_t)ya * N + x], pb = A.phi[(size_t)(ya + 1) * N + x];
      const double ga = gv[m].x * invN, gb = gv[m].y * invN;
      const double ca = cv[m].x * invN, cb = cv[m].y * invN;
      ha = fpp_of<double>(ca, pa, A.p) * ga;
      hb = fpp_of<double>(cb, pb, A.p) * gb;
      const double gpa = gphi_of(pa), gpb = gphi_of(pb);
      sP += -A.p.chi * (ga * gpa + gb * gpb);
      sChi += -A.p.P * (ga * gpa + gb * gpb);
    }
    gv[m] = mkc<double>(ha, hb);
  }
  fft<false, P>(gv, t, sm, lay, tw);
  cpx<double> xa[E / 2], xb[E / 2];
  split_pair<P>(gv, t, sm, lay, xa, xb);
  if (active) {
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      const size_t oa = (size_t)ya * H + t + T * m, ob = oa + H;
      const double2 la = A.Lam[oa], lb = A.Lam[ob];
      A.Lam[oa] = make_double2(la.x + xa[m].x, la.y + xa[m].y);
      A.Lam[ob] = make_double2(lb.x + xb[m].x, lb.y + xb[m].y);
    }
  }
  const double vals[2] = {sP, sChi};
  const int slots[2] = {0, 1};
  adj_accumulate<2>(A, 2, 0, vals, slots, red, &lastflag);
}


// ---- mixed-precision adjoint step ------------------------------------------------------
// For contexts of the mixed precision.  The adjoint lam is kept and y-transformed in FP64,
// like the forward state; the fields derived from it -- grad a, M grad a, g, f'' g, and
// the state difference of the sensitivity sums -- are transformed in FP32, two at a time
// in packed pairs (cpx<f2>) where two transforms run side by side, and their increments are
// added to lam in FP64.  The structure, the packed-column handling and the sums are those
// of k_adj_col1 / k_adj_col2 / k_adj_row2; row B is the mixed forward row B kernel.

template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 2 : 1)) k_adj_col1_m(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeom<P>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  cpx<float>* smf = reinterpret_cast<cpx<float>*>(smraw);
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * A.dx);
  const double c1 = 2.0 * A.p.Q * A.p.kappa * A.dt;
  cpx<double> l[E];
  cpx<float> d[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const size_t o = (size_t)(t + T * m) * H + kx;
    if (active) {
      const double2 a = A.Lam[o], s0 = A.S0[o], s1 = A.S1[o];
      l[m] = mkc<double>(a.x, a.y);
      d[m] = mkc<float>((float)(s1.x - s0.x), (float)(s1.y - s0.y));
    } else {
      l[m] = mkc<double>(0, 0);
      d[m] = mkc<float>(0, 0);
    }
  }
  fft<false, P>(l, t, sm, lay, PassTable<P, double>{});
  fft<false, P>(d, t, smf, lay, PassTable<P, float>{});
  const bool packed_tile = blockIdx.x == 0, packed = packed_tile && w == 0;
  const double kxf = kunit * (double)kx, kH2 = (kunit * H) * (kunit * H);
  const double invNN = 1.0 / ((double)N * N);
  double s_kap = 0.0, s_m0 = 0.0;
  cpx<f2> q[E];  // lane 0: x-derivative of a, lane 1: y-derivative
  if (packed_tile) {
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sm[t + T * m] = l[m];
    }
    __syncthreads();
    cpx<double> lB[E];
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const cpx<double> pr = packed ? cconj(sm[(N - ky) % N]) : mkc<double>(0, 0);
      lB[m] = cscale(times_negi(l[m] - pr), 0.5);
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) smf[t + T * m] = d[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<double> dm = ccast<double>(d[m]), pd = ccast<double>(cconj(smf[(N - ky) % N]));
        const cpx<double> dA = cscale(dm + pd, 0.5), dB = cscale(times_negi(dm - pd), 0.5);
        const cpx<double> lA = l[m] - times_i(lB[m]);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf, k2b = k2a + kH2;
        const double dena = 1.0 + c1 * k2a * k2a, denb = 1.0 + c1 * k2b * k2b;
        const double reA = lA.x * dA.x + lA.y * dA.y, reB = lB[m].x * dB.x + lB[m].y * dB.y;
        s_m0 += (reA + reB) * invNN;
        s_kap += (reA * (-2.0 * A.p.Q * k2a * k2a * A.dt / dena) + reB * (-2.0 * A.p.Q * k2b * k2b * A.dt / denb)) * invNN;
        const cpx<double> ah = cscale(lA, A.dt / dena) + times_i(cscale(lB[m], A.dt / denb));
        const double kyd = (ky == H) ? 0.0 : kyf;
        q[m] = pack2(mkc<float>(0.0f, 0.0f), ccast<float>(times_i(cscale(ah, kyd * invNN))));
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
      const double den = 1.0 + c1 * k2 * k2;
      const double re = l[m].x * (double)d[m].x + l[m].y * (double)d[m].y;
      if (active) {
        s_m0 += 2.0 * re * invNN;
        s_kap += 2.0 * re * (-2.0 * A.p.Q * k2 * k2 * A.dt / den) * invNN;
      }
      const cpx<double> ah = cscale(l[m], A.dt / den);
      const double kyd = (ky == H) ? 0.0 : kyf;
      q[m] = pack2(ccast<float>(times_i(cscale(ah, kxf * invNN))), ccast<float>(times_i(cscale(ah, kyd * invNN))));
    }
  }
  fft<true, P>(q, t, reinterpret_cast<cpx<f2>*>(smraw), lay, PassTableDup<P>{});
  if (active) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      cpx2<float> o;
      o.a = lane0(q[m]);
      o.b = lane1(q[m]);
      A.Gw[(size_t)(t + T * m) * H + kx] = o;
    }
  }
  const double vals[2] = {s_kap, s_m0 / A.p.mobility};
  const int slots[2] = {2, 3};
  adj_accumulate<2>(A, 0, 0, vals, slots, red, &lastflag);
}


template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 3 : 1)) k_adj_col2_m(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeom<P>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  cpx<float>* smf = reinterpret_cast<cpx<float>*>(smraw);
  cpx<f2>* smp = reinterpret_cast<cpx<f2>*>(smraw);
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * A.dx);
  cpx<f2> q[E];  // lane 0: F(M dx a), lane 1: F(M dy a)
  cpx<float> ch[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const size_t o = (size_t)(t + T * m) * H + kx;
    const cpx2<float> gq = active ? A.Gw[o] : cpx2<float>{mkc<float>(0, 0), mkc<float>(0, 0)};
    q[m] = pack2(gq.a, gq.b);
    const double2 sv = active ? A.S0[o] : make_double2(0, 0);
    ch[m] = mkc<float>((float)sv.x, (float)sv.y);
  }
  fft<false, P>(q, t, smp, lay, PassTableDup<P>{});
  const float kxf = (float)(kunit * (double)kx);
  const double kH2 = (kunit * H) * (kunit * H);
  const bool packed_tile = blockIdx.x == 0, packed = packed_tile && w == 0;
  // g^ = i kx F(M dx a) + i ky F(M dy a); on the packed column only the y part survives
  cpx<float> fx[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int ky = t + T * m;
    const float kyd = (ky == H) ? 0.0f : (float)(kunit * (double)(ky < H ? ky : ky - N));
    const float kxd = packed ? 0.0f : kxf;
    fx[m] = times_i(cscale(lane0(q[m]), kxd) + cscale(lane1(q[m]), kyd));
  }
  fft<false, P>(ch, t, smf, lay, PassTable<P, float>{});  // c^ = y-FFT(S)
  const double invNN = 1.0 / ((double)N * N);
  const float invN = 1.0f / (float)N;
  const double kappa = A.p.kappa;
  double s_kap = 0.0;
  if (packed_tile) {
    cpx<float> gB[E];
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) smf[t + T * m] = fx[m];
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const cpx<float> pr = packed ? cconj(smf[(N - ky) % N]) : mkc<float>(0, 0);
      gB[m] = cscale(times_negi(fx[m] - pr), 0.5f);
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) smf[t + T * m] = ch[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<float> pc = cconj(smf[(N - ky) % N]);
        const cpx<float> cA = cscale(ch[m] + pc, 0.5f), cB = cscale(times_negi(ch[m] - pc), 0.5f);
        const cpx<float> gA = fx[m] - times_i(gB[m]);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf, k2b = k2a + kH2;
        s_kap += (2.0 * k2a * ((double)gA.x * cA.x + (double)gA.y * cA.y) +
                  2.0 * k2b * ((double)gB[m].x * cB.x + (double)gB[m].y * cB.y)) * invNN;
        ch[m] = cscale(cscale(fx[m], (float)(2.0 * kappa * k2a)) + times_i(cscale(gB[m], (float)(2.0 * kappa * kH2))),
                       invN);
      }
    }
    __syncthreads();
  }
  if (!packed) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const double kyf = kunit * (double)(ky < H ? ky : ky - N);
      const double kx64 = kunit * (double)kx;
      const double k2 = kx64 * kx64 + kyf * kyf;
      if (active) s_kap += 2.0 * 2.0 * k2 * ((double)fx[m].x * ch[m].x + (double)fx[m].y * ch[m].y) * invNN;
      ch[m] = cscale(fx[m], (float)(2.0 * kappa * k2) * invN);  // ch now holds U / n
    }
  }
#pragma unroll
  for (int m = 0; m < E; ++m) q[m] = pack2(cscale(fx[m], invN), ch[m]);
  fft<true, P>(q, t, smp, lay, PassTableDup<P>{});
  if (active) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const size_t o = (size_t)(t + T * m) * H + kx;
      A.Xw[o] = lane0(q[m]);
      const cpx<float> u = lane1(q[m]);
      const double2 l = A.Lam[o];
      A.Lam[o] = make_double2(l.x + (double)u.x, l.y + (double)u.y);
    }
  }
  const double vals[1] = {s_kap};
  const int slots[1] = {2};
  adj_accumulate<1>(A, 1, 0, vals, slots, red, &lastflag);
}


template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 3 : 1)) k_adj_row2_m(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;
  const RowLayout<N> lay{g * RowLayout<N>::stride};
  cpx<float>* smf = reinterpret_cast<cpx<float>*>(smraw);
  const cpx<float>* Xw = A.Xw;
  const cpx<double>* S = reinterpret_cast<const cpx<double>*>(A.S0);
  // lane 0: g of rows ya, ya+1 (as one complex row); lane 1: c of the same rows
  cpx<f2> q[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    if (active) {
      const cpx<float> gv = load_pair_spectrum<float, N>(Xw + (size_t)ya * H, Xw + (size_t)(ya + 1) * H, t + T * m);
      const cpx<double> cv = load_pair_spectrum<double, N>(S + (size_t)ya * H, S + (size_t)(ya + 1) * H, t + T * m);
      q[m] = pack2(gv, ccast<float>(cv));
    } else {
      q[m] = pack2(mkc<float>(0, 0), mkc<float>(0, 0));
    }
  }
  fft<true, P>(q, t, reinterpret_cast<cpx<f2>*>(smraw), lay, PassTableDup<P>{});
  const float invN = 1.0f / (float)N;
  double sP = 0.0, sChi = 0.0;
  cpx<float> h[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    float ha = 0.0f, hb = 0.0f;
    if (active) {
      const float pa = A.phiw[(size_t)ya * N + x], pb = A.phiw[(size_t)(ya + 1) * N + x];
      const cpx<float> gv = lane0(q[m]), cv = lane1(q[m]);
      const float ga = gv.x * invN, gb = gv.y * invN;
      const float ca = cv.x * invN, cb = cv.y * invN;
      ha = fpp_of<float>(ca, pa, A.p) * ga;
      hb = fpp_of<float>(cb, pb, A.p) * gb;
      const double gpa = gphi_of((double)pa), gpb = gphi_of((double)pb);
      sP += -A.p.chi * ((double)ga * gpa + (double)gb * gpb);
      sChi += -A.p.P * ((double)ga * gpa + (double)gb * gpb);
    }
    h[m] = mkc<float>(ha, hb);
  }
  fft<false, P>(h, t, smf, lay, PassTable<P, float>{});
  cpx<float> xa[E / 2], xb[E / 2];
  split_pair<P>(h, t, smf, lay, xa, xb);
  if (active) {
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      const size_t oa = (size_t)ya * H + t + T * m, ob = oa + H;
      const double2 la = A.Lam[oa], lb = A.Lam[ob];
      A.Lam[oa] = make_double2(la.x + (double)xa[m].x, la.y + (double)xa[m].y);
      A.Lam[ob] = make_double2(lb.x + (double)xb[m].x, lb.y + (double)xb[m].y);
    }
  }
  const double vals[2] = {sP, sChi};
  const int slots[2] = {0, 1};
  adj_accumulate<2>(A, 2, 0, vals, slots, red, &lastflag);
}

// ---- seed: mu of the final field (column) ---------------------------------------------
template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 2 : 1)) k_adj_mu_col(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, W = ColGeom<P>::W;
  extern __shared__ __align__(16) unsigned char smraw[];
  const AdjDev& A = adjs[blockIdx.y];
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int kx = blockIdx.x * W + w;
  const bool active = kx < H;
  const ColLayout<W> lay{w};
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const PassTable<P, double> tw{};  // pass-major copy of the FP64 table A.tw
  const double kunit = 2.0 * 3.14159265358979323846 / ((double)N * A.dx);
  const double kappa = A.p.kappa;
  cpx<double> v[E], f[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const size_t o = (size_t)(t + T * m) * H + kx;
    const double2 s = active ? A.S0[o] : make_double2(0, 0), q = active ? A.F[o] : make_double2(0, 0);
    v[m] = mkc<double>(s.x, s.y);
    f[m] = mkc<double>(q.x, q.y);
  }
  fft<false, P>(v, t, sm, lay, tw);
  fft<false, P>(f, t, sm, lay, tw);
  const bool packed_tile = blockIdx.x == 0, packed = packed_tile && w == 0;
  const double kxf = kunit * (double)kx, kH2 = (kunit * H) * (kunit * H);
  const double invN = 1.0 / (double)N;
  if (packed_tile) {
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) sm[t + T * m] = v[m];
    }
    __syncthreads();
    if (packed) {
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int ky = t + T * m;
        const cpx<double> pr = cconj(sm[(N - ky) % N]);
        const cpx<double> Bc = cscale(times_negi(v[m] - pr), 0.5);
        const double kyf = kunit * (double)(ky < H ? ky : ky - N);
        const double k2a = kyf * kyf;
        f[m] = cscale(f[m] + cscale(v[m], 2.0 * kappa * k2a) + times_i(cscale(Bc, 2.0 * kappa * kH2)), invN);
      }
    }
    __syncthreads();
  }
  if (!packed) {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int ky = t + T * m;
      const double kyf = kunit * (double)(ky < H ? ky : ky - N);
      f[m] = cscale(f[m] + cscale(v[m], 2.0 * kappa * (kxf * kxf + kyf * kyf)), invN);
    }
  }
  fft<true, P>(f, t, sm, lay, tw);
  if (active) {
#pragma unroll
    for (int m = 0; m < E; ++m) A.Xg[(size_t)(t + T * m) * H + kx] = make_double2(f[m].x, f[m].y);
  }
}

// ---- seed: lam_T = (c_T - c_target) + lamF mu dx^2 (row) --------------------------------
template <class P>
__global__ void __launch_bounds__(kBlock, (P::E <= 8 ? 2 : 1)) k_adj_seed_row(const AdjDev* __restrict__ adjs) {
  constexpr int N = P::N, E = P::E, T = P::T, H = N / 2, G = RowGeom<P>::G;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32 * 4];
  __shared__ int lastflag;
  const AdjDev& A = adjs[blockIdx.y];
  const int t = threadIdx.x % T, g = threadIdx.x / T;
  const int pair = blockIdx.x * G + g;
  const bool active = pair < H;
  const int ya = 2 * pair;
  const RowLayout<N> lay{g * RowLayout<N>::stride};
  cpx<double>* sm = reinterpret_cast<cpx<double>*>(smraw);
  const PassTable<P, double> tw{};  // pass-major copy of the FP64 table A.tw
  const cpx<double>* Xm = reinterpret_cast<const cpx<double>*>(A.Xg);
  const cpx<double>* S = reinterpret_cast<const cpx<double>*>(A.S0);
  cpx<double> mv[E], cv[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    mv[m] = active ? load_pair_spectrum<double, N>(Xm + (size_t)ya * H, Xm + (size_t)(ya + 1) * H, t + T * m)
                   : mkc<double>(0, 0);
    cv[m] = active ? load_pair_spectrum<double, N>(S + (size_t)ya * H, S + (size_t)(ya + 1) * H, t + T * m)
                   : mkc<double>(0, 0);
  }
  fft<true, P>(mv, t, sm, lay, tw);
  fft<true, P>(cv, t, sm, lay, tw);
  const double invN = 1.0 / (double)N, dx2 = A.dx * A.dx;
  double sl = 0.0, se = 0.0, sc = 0.0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int x = t + T * m;
    double la = 0.0, lb = 0.0;
    if (active) {
      const double ca = cv[m].x * invN, cb = cv[m].y * invN;
      const double ma = mv[m].x * invN, mb = mv[m].y * invN;
      const double ta = A.target[(size_t)ya * N + x], tb = A.target[(size_t)(ya + 1) * N + x];
      const double pa = A.phi[(size_t)ya * N + x], pb = A.phi[(size_t)(ya + 1) * N + x];
      la = (ca - ta) + A.lamF * ma * dx2;
      lb = (cb - tb) + A.lamF * mb * dx2;
      sl += 0.5 * ((ca - ta) * (ca - ta) + (cb - tb) * (cb - tb));
      const double gpa = gphi_of(pa), gpb = gphi_of(pb);
      se += (1.0 - A.p.chi * ca) * gpa + (1.0 - A.p.chi * cb) * gpb;
      sc += ca * gpa + cb * gpb;
    }
    mv[m] = mkc<double>(la, lb);
  }
  fft<false, P>(mv, t, sm, lay, tw);
  cpx<double> xa[E / 2], xb[E / 2];
  split_pair<P>(mv, t, sm, lay, xa, xb);
  if (active) {
#pragma unroll
    for (int m = 0; m < E / 2; ++m) {
      const size_t oa = (size_t)ya * H + t + T * m;
      A.Lam[oa] = make_double2(xa[m].x, xa[m].y);
      A.Lam[oa + H] = make_double2(xb[m].x, xb[m].y);
    }
  }
  const double vals[3] = {sl, se, sc};
  const int slots[3] = {4, 5, 6};
  adj_accumulate<3>(A, 3, 0, vals, slots, red, &lastflag);
}

}  // namespace esc
