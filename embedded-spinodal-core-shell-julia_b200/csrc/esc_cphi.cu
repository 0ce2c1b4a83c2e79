// Host side of the coupled c-phi model (esc_cphi_* in esc.h): contexts, the
// per-step launch sequence captured in CUDA graphs, the runtime-size stencil
// kernels of the y and x parts of div(M grad mu), and the statistics of the
// input fields.  The step itself is described in esc_cphi.cuh.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "esc.h"
#include "esc_cphi.cuh"

#define ESC_CPHI_DECL(n) const esc::cphi::Set* esc_cphi_set_##n();
ESC_CPHI_SIZES(ESC_CPHI_DECL)
#undef ESC_CPHI_DECL

void esc_set_thread_error(const char* msg);

namespace esc {
namespace cphi {

constexpr int kFdW = 16;     // adjacent z lines per block of the stencil kernels
constexpr int kFdLoads = 8;  // staging sweeps whose loads are in flight together

// div += D_a(M D_a mu) along axis a = x (0) or y (1): each block stages kFdW
// adjacent z lines (n points each) of mu, of M = mobility h(phi) and of the
// current div in shared memory (the loads of kFdLoads sweeps in flight
// together), turns the M tile into q = M D mu in place, then writes
// div + D q.  Runtime n; dynamic shared memory 3 n kFdW doubles.
__global__ void __launch_bounds__(kBlock) k3_fd_line(const Dev* __restrict__ dp, int axis) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Dev& d = *dp;
  if (*(volatile const int*)d.status) return;
  const int n = axis == 0 ? d.nx : d.ny;
  const double h = axis == 0 ? d.dx : d.dy;
  const long estride = axis == 0 ? (long)d.ny * d.nz : (long)d.nz;
  const long ostride = axis == 0 ? (long)d.nz : (long)d.ny * d.nz;
  const int k0 = blockIdx.x * kFdW;
  const long base = (long)blockIdx.y * ostride + k0;
  double* mt = reinterpret_cast<double*>(smraw);
  double* qt = mt + (size_t)n * kFdW;
  double* dt = qt + (size_t)n * kFdW;
  const int total = n * kFdW;
  const double inv12 = 1.0 / (12.0 * h);
  const double M0 = d.p.mobility;
  const double* __restrict__ mu = d.mu;
  const double* __restrict__ phi = d.phi;
  double* __restrict__ div = d.div;
  // neighbour rows p +- 1, p +- 2 with the periodic wrap, without a runtime modulo
  auto row = [n](int p, int o) {
    int r = p + o;
    r += (r < 0) ? n : 0;
    r -= (r >= n) ? n : 0;
    return r * kFdW;
  };
  // kFdLoads sweeps' loads are issued before any of them is stored: 3 kFdLoads
  // loads in flight per thread instead of 3
  for (int i0 = threadIdx.x; i0 < total; i0 += kFdLoads * blockDim.x) {
    double lm[kFdLoads], lp[kFdLoads], ld[kFdLoads];
#pragma unroll
    for (int u = 0; u < kFdLoads; ++u) {
      const int idx = i0 + u * (int)blockDim.x;
      const int p = idx / kFdW, w = idx % kFdW;
      const bool ok = idx < total && k0 + w < d.nz;
      const long a = base + (long)p * estride + w;
      lm[u] = ok ? mu[a] : 0.0;
      lp[u] = ok ? phi[a] : 0.0;
      ld[u] = ok ? div[a] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kFdLoads; ++u) {
      const int idx = i0 + u * (int)blockDim.x;
      if (idx >= total) break;
      const bool ok = k0 + idx % kFdW < d.nz;
      mt[idx] = lm[u];
      qt[idx] = ok ? mobility3(lp[u], M0) : 0.0;
      dt[idx] = ld[u];
    }
  }
  __syncthreads();
  // thread (w, seg) sweeps rows [r0, r1) of line w with a five-point window in
  // registers: one shared-memory load per point and stencil
  const int w = threadIdx.x % kFdW, nseg = blockDim.x / kFdW;
  const int rows = (n + nseg - 1) / nseg;
  const int r0 = (threadIdx.x / kFdW) * rows, r1 = min(n, r0 + rows);
  if (r0 < r1) {
    double m2 = mt[row(r0, -2) + w], m1 = mt[row(r0, -1) + w], m0 = mt[r0 * kFdW + w], p1 = mt[row(r0, 1) + w];
    for (int p = r0; p < r1; ++p) {
      const double p2 = mt[row(p, 2) + w];
      qt[p * kFdW + w] *= fd4(p2, p1, m1, m2, inv12);
      m2 = m1;
      m1 = m0;
      m0 = p1;
      p1 = p2;
    }
  }
  __syncthreads();
  if (r0 < r1 && k0 + w < d.nz) {
    double m2 = qt[row(r0, -2) + w], m1 = qt[row(r0, -1) + w], m0 = qt[r0 * kFdW + w], p1 = qt[row(r0, 1) + w];
    for (int p = r0; p < r1; ++p) {
      const double p2 = qt[row(p, 2) + w];
      div[base + (long)p * estride + w] = dt[p * kFdW + w] + fd4(p2, p1, m1, m2, inv12);
      m2 = m1;
      m1 = m0;
      m0 = p1;
      p1 = p2;
    }
  }
}

// history row 0 and the mass reference (mean of the input c, evolve.cu:36-46)
__global__ void __launch_bounds__(kBlock) k3_stats(const Dev* __restrict__ dp) {
  __shared__ Six red[kBlock / 32];
  __shared__ int lastflag;
  const Dev& d = *dp;
  const long total = (long)d.nx * d.ny * d.nz;
  Six s = six_identity();
  int nbad = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const double cv = d.c[i], pv = d.phi[i];
    s.v[0] += cv;
    s.v[1] += pv;
    s.v[2] = fmin(s.v[2], cv);
    s.v[3] = fmax(s.v[3], cv);
    nbad += (int)(nonfinite_bits(cv) | nonfinite_bits(pv));
  }
  s.v[5] = (double)nbad;
  const Six mine = six_block(s, red);
  Six tot;
  if (!six_fold(mine, d.part, &d.cnt[1], red, &lastflag, tot)) return;
  const double Nn = (double)total;
  d.scal[0] = tot.v[0] / Nn;
  if (d.hist) {
    const size_t ld = (size_t)d.hist_ld;
    d.hist[0] = 0.0;
    d.hist[ld] = tot.v[0] / Nn;
    d.hist[2 * ld] = tot.v[1] / Nn;
    d.hist[3 * ld] = tot.v[2];
    d.hist[4 * ld] = tot.v[3];
    d.hist[5 * ld] = 0.0;
  }
  if (tot.v[5] > 0.0) {
    *d.stop_step = 0;
    *d.status = kNonFinite;
  }
}

__global__ void k3_advance(int* base, int by) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *base += by;
}

const Set* set_for(int n) {
  switch (n) {
#define ESC_CPHI_CASE(v) \
  case v:                \
    return esc_cphi_set_##v();
    ESC_CPHI_SIZES(ESC_CPHI_CASE)
#undef ESC_CPHI_CASE
    default:
      return nullptr;
  }
}

constexpr int kStatsBlocks = 296;
constexpr int kNumChunks = 6;
constexpr int kChunkSteps[kNumChunks] = {32, 16, 8, 4, 2, 1};

std::vector<double> plain_twiddles(int n) {
  std::vector<double> t(2 * (size_t)n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int j = 0; j < n; ++j) {
    const long double a = two_pi * (long double)j / (long double)n;
    t[2 * (size_t)j] = (double)cosl(a);
    t[2 * (size_t)j + 1] = (double)(-sinl(a));
  }
  return t;
}

}  // namespace cphi
}  // namespace esc

using esc::cphi::Dev;
using esc::cphi::Set;

struct esc_cphi {
  int device = 0;
  int nx = 0, ny = 0, nz = 0, K = 0;
  const Set *sx = nullptr, *sy = nullptr, *sz = nullptr;
  cudaStream_t own = nullptr, stream = nullptr;
  Dev h{};
  Dev* d_dev = nullptr;
  double* hist = nullptr;
  size_t hist_cap = 0;
  void* tw[3] = {nullptr, nullptr, nullptr};
  int* status = nullptr;
  long long* stop = nullptr;
  int* base = nullptr;
  cudaGraphExec_t graphs[esc::cphi::kNumChunks] = {};
  std::vector<void*> allocs;
  std::string err;

  esc_status fail(esc_status s, const std::string& m) {
    err = m;
    return s;
  }
  esc_status fail_cuda(const char* what, cudaError_t e) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return ESC_ECUDA;
  }
  template <typename T>
  esc_status alloc(T** p, size_t bytes, const char* what) {
    void* v = nullptr;
    const cudaError_t e = cudaMalloc(&v, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      err = std::string("cudaMalloc (") + what + "): " + cudaGetErrorString(e);
      return ESC_ENOMEM;
    }
    allocs.push_back(v);
    *p = static_cast<T*>(v);
    return ESC_OK;
  }
  void release() {
    for (cudaGraphExec_t& g : graphs) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    if (own) cudaStreamDestroy(own);
    own = nullptr;
  }
};

namespace {

#define CK(call)                                                   \
  do {                                                             \
    const cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return X.fail_cuda(#call, e_);          \
  } while (0)
#define TRY(call)                       \
  do {                                  \
    const esc_status s_ = (call);       \
    if (s_ != ESC_OK) return s_;        \
  } while (0)

struct Guard {
  int prev = -1;
  explicit Guard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~Guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

std::mutex& cphi_mutex() {
  static std::mutex m;
  return m;
}

// One step of the coupled model (twelve stages, fourteen launches), s_local its
// index inside the chunk.  With `ev` (13 events), ev[k] is recorded before stage
// k and ev[12] after the last (per-stage timing).
constexpr int kStepKernels = 12;
void launch_step(esc_cphi& X, int s_local, cudaStream_t st, cudaEvent_t* ev = nullptr) {
  using namespace esc::cphi;
  const Dev* d = X.d_dev;
  const long L = (long)X.nx * X.ny;
  const int zb_line = (int)((L + X.sz->zG - 1) / X.sz->zG);
  const int zb_pair = (int)(((L + 1) / 2 + X.sz->zG - 1) / X.sz->zG);
  const dim3 gy((X.K + X.sy->lW - 1) / X.sy->lW, X.nx);  // y lines (i, kz)
  const dim3 gx((X.K + X.sx->lW - 1) / X.sx->lW, X.ny);  // x lines (j, kz)
  const long ey = X.K, oy = (long)X.ny * X.K;
  const dim3 gfy((X.nz + kFdW - 1) / kFdW, X.nx), gfx((X.nz + kFdW - 1) / kFdW, X.ny);
  int k = 0;
  auto mark = [&]() {
    if (ev) cudaEventRecord(ev[k++], st);
  };
  mark();
  X.sz->zf(d, kZLocal, zb_line, st);
  mark();
  X.sy->line(d, false, X.h.D1, X.h.D2, 2, ey, oy, gy, st);
  mark();
  X.sx->xspec(d, kXMu, s_local, gx, st);
  mark();
  X.sy->line(d, true, X.h.D1, nullptr, 1, ey, oy, gy, st);
  mark();
  X.sz->zi_mu(d, zb_pair, st);
  mark();
  k3_fd_line<<<gfy, esc::kBlock, (size_t)3 * X.ny * kFdW * sizeof(double), st>>>(d, 1);
  mark();
  k3_fd_line<<<gfx, esc::kBlock, (size_t)3 * X.nx * kFdW * sizeof(double), st>>>(d, 0);
  mark();
  X.sz->zf(d, kZDiv, zb_pair, st);
  mark();
  X.sy->line(d, false, X.h.D1, nullptr, 1, ey, oy, gy, st);
  mark();
  X.sx->xspec(d, kXUpdate, s_local, gx, st);
  mark();
  X.sy->line(d, true, X.h.D1, X.h.D2, 2, ey, oy, gy, st);
  mark();
  X.sz->zi_final(d, s_local, zb_line, st);
  mark();
}

esc_status ensure_graphs(esc_cphi& X) {
  using namespace esc::cphi;
  cudaStream_t st = X.stream;
  for (int ci = 0; ci < kNumChunks; ++ci) {
    if (X.graphs[ci]) continue;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < kChunkSteps[ci]; ++s) launch_step(X, s, st);
    k3_advance<<<1, 32, 0, st>>>(X.base, kChunkSteps[ci]);
    const cudaError_t ec = cudaStreamEndCapture(st, &g);
    if (ec != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return X.fail_cuda("cudaStreamEndCapture", ec);
    }
    const cudaError_t ei = cudaGraphInstantiate(&X.graphs[ci], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      X.graphs[ci] = nullptr;
      return X.fail_cuda("cudaGraphInstantiate", ei);
    }
    CK(cudaGraphUpload(X.graphs[ci], st));
  }
  return ESC_OK;
}

esc_status run_impl(esc_cphi& X, double* c, double* phi, bool device_io, int steps, double dt, double tol,
                    double comperr, double* history, int64_t* steps_done, int* stop_reason) {
  using namespace esc::cphi;
  if (steps < 0) return X.fail(ESC_EINVAL, "steps must be >= 0");
  if (!std::isfinite(dt)) return X.fail(ESC_EINVAL, "dt must be finite");
  if (std::isnan(tol) || std::isnan(comperr)) return X.fail(ESC_EINVAL, "tolerance and comperr must not be NaN");
  if (!c || !phi) return X.fail(ESC_EINVAL, "null field pointer");
  Guard dg(X.device);
  cudaStream_t st = X.stream;
  const size_t nn = (size_t)X.nx * X.ny * X.nz;
  const size_t rows = (size_t)steps + 1;
  if (rows * 6 > X.hist_cap) {
    if (X.hist) {
      for (auto it = X.allocs.begin(); it != X.allocs.end(); ++it)
        if (*it == X.hist) {
          X.allocs.erase(it);
          break;
        }
      cudaFree(X.hist);
      X.hist = nullptr;
      X.hist_cap = 0;
    }
    TRY(X.alloc(&X.hist, rows * 6 * sizeof(double), "history"));
    X.hist_cap = rows * 6;
  }
  X.h.dt = dt;
  X.h.tol = tol;
  X.h.comperr = comperr;
  X.h.hist = X.hist;
  X.h.hist_ld = (int)rows;
  CK(cudaMemcpyAsync(X.d_dev, &X.h, sizeof(Dev), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(X.hist, 0, rows * 6 * sizeof(double), st));
  CK(cudaMemsetAsync(X.status, 0, sizeof(int), st));
  CK(cudaMemsetAsync(X.stop, 0xff, sizeof(long long), st));
  CK(cudaMemsetAsync(X.base, 0, sizeof(int), st));
  CK(cudaMemsetAsync(X.h.cnt, 0, 2 * sizeof(unsigned), st));
  const cudaMemcpyKind in = device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(X.h.c, c, nn * sizeof(double), in, st));
  CK(cudaMemcpyAsync(X.h.phi, phi, nn * sizeof(double), in, st));
  TRY(ensure_graphs(X));
  // input statistics, then c^ and phi^ of the input fields
  k3_stats<<<kStatsBlocks, esc::kBlock, 0, st>>>(X.d_dev);
  const long L = (long)X.nx * X.ny;
  X.sz->zf(X.d_dev, kZInit, (int)((L + X.sz->zG - 1) / X.sz->zG), st);
  const dim3 gy((X.K + X.sy->lW - 1) / X.sy->lW, X.nx), gx((X.K + X.sx->lW - 1) / X.sx->lW, X.ny);
  X.sy->line(X.d_dev, false, X.h.D1, X.h.D2, 2, X.K, (long)X.ny * X.K, gy, st);
  X.sx->xspec(X.d_dev, kXInit, 0, gx, st);
  CK(cudaGetLastError());
  int left = steps;
  for (int ci = 0; ci < kNumChunks; ++ci)
    while (left >= kChunkSteps[ci]) {
      CK(cudaGraphLaunch(X.graphs[ci], st));
      left -= kChunkSteps[ci];
    }
  const cudaMemcpyKind out = device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  CK(cudaMemcpyAsync(c, X.h.c, nn * sizeof(double), out, st));
  CK(cudaMemcpyAsync(phi, X.h.phi, nn * sizeof(double), out, st));
  if (history) CK(cudaMemcpyAsync(history, X.hist, rows * 6 * sizeof(double), out, st));
  int status = 0;
  long long stop = -1;
  CK(cudaMemcpyAsync(&status, X.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&stop, X.stop, sizeof(long long), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (steps_done) *steps_done = status ? stop : steps;
  if (stop_reason) *stop_reason = status;
  if (status == kNonFinite)
    return X.fail(ESC_ENONFINITE, "Non-finite composition or order parameter after step " + std::to_string(stop));
  if (status == kMassError)
    return X.fail(ESC_EMASS, "Elements not conserved: the mean composition moved by more than comperr in step " +
                                 std::to_string(stop + 1));
  return ESC_OK;
}

}  // namespace

extern "C" {

void esc_cphi_default_params(esc_cphi_params* p) {
  if (!p) return;
  // original/2023-3d/InputParams:13-22
  p->A = 2.0;
  p->B = 1.0;
  p->chi = 0.5;
  p->P = 6.0;
  p->ca = 0.5;
  p->cb1 = 0.0;
  p->cb2 = 1.0;
  p->A0 = 0.08;
  p->kappa_c = 2.0;
  p->kappa_phi = 10.0;
  p->mobility = 1.0;
  p->relax = 0.001;
  p->Q = 0.5;
}

int esc_cphi_supported_size(int n) { return esc::cphi::set_for(n) != nullptr; }

esc_status esc_cphi_create(esc_cphi** out, int nx, int ny, int nz, double dx, double dy, double dz,
                           const esc_cphi_params* p) {
  using namespace esc::cphi;
  if (!out) {
    esc_set_thread_error("null output pointer");
    return ESC_EINVAL;
  }
  *out = nullptr;
  if (!p) {
    esc_set_thread_error("null parameters");
    return ESC_EINVAL;
  }
  const Set *sx = set_for(nx), *sy = set_for(ny), *sz = set_for(nz);
  if (!sx || !sy || !sz) {
    esc_set_thread_error("unsupported grid size (each of nx, ny, nz must be one of 8, 12, 16, 24, 32, 48, 64, 96, "
                         "128, 192, 256, 384, 512)");
    return ESC_EINVAL;
  }
  if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0) || !std::isfinite(dx) || !std::isfinite(dy) || !std::isfinite(dz)) {
    esc_set_thread_error("grid spacings must be positive and finite");
    return ESC_EINVAL;
  }
  std::lock_guard<std::mutex> lock(cphi_mutex());
  esc_cphi* Xp = new (std::nothrow) esc_cphi();
  if (!Xp) {
    esc_set_thread_error("host allocation failed");
    return ESC_ENOMEM;
  }
  esc_cphi& X = *Xp;
  auto bail = [&](esc_status s) {
    esc_set_thread_error(X.err.c_str());
    X.release();
    delete Xp;
    return s;
  };
  if (cudaGetDevice(&X.device) != cudaSuccess) {
    cudaGetLastError();
    X.err = "no CUDA device";
    return bail(ESC_ECUDA);
  }
  X.nx = nx;
  X.ny = ny;
  X.nz = nz;
  X.K = nz / 2 + 1;
  X.sx = sx;
  X.sy = sy;
  X.sz = sz;
  auto setup = [&]() -> esc_status {
    CK(cudaStreamCreateWithFlags(&X.own, cudaStreamNonBlocking));
    X.stream = X.own;
    for (const Set* s : {sx, sy, sz}) CK(s->prepare());
    CK(cudaFuncSetAttribute(k3_fd_line, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(3 * 512 * kFdW * sizeof(double))));
    const size_t nn = (size_t)nx * ny * nz, nk = (size_t)nx * ny * X.K;
    Dev& h = X.h;
    h.nx = nx;
    h.ny = ny;
    h.nz = nz;
    h.K = X.K;
    h.dx = dx;
    h.dy = dy;
    h.dz = dz;
    h.invN = 1.0 / (double)nn;
    h.p = Params{p->A, p->B, p->chi, p->P, p->ca, p->cb1, p->cb2, p->A0, p->kappa_c, p->kappa_phi, p->mobility,
                 p->relax, p->Q};
    TRY(X.alloc(&h.c, nn * 8, "c"));
    TRY(X.alloc(&h.phi, nn * 8, "phi"));
    TRY(X.alloc(&h.mu, nn * 8, "mu"));
    TRY(X.alloc(&h.div, nn * 8, "div"));
    TRY(X.alloc(&h.Ch, nk * 16, "c spectrum"));
    TRY(X.alloc(&h.Ph, nk * 16, "phi spectrum"));
    TRY(X.alloc(&h.D1, nk * 16, "work spectrum"));
    TRY(X.alloc(&h.D2, nk * 16, "work spectrum"));
    // partial sums: one slot of six per block of the statistics or of the final z pass
    const size_t maxblocks = std::max<size_t>((size_t)kStatsBlocks, (size_t)nx * ny);
    TRY(X.alloc(&h.part, maxblocks * 6 * sizeof(double), "partials"));
    TRY(X.alloc(&h.cnt, 4 * sizeof(unsigned), "counters"));
    TRY(X.alloc(&h.scal, 4 * sizeof(double), "scalars"));
    TRY(X.alloc(&X.status, sizeof(int), "status"));
    TRY(X.alloc(&X.stop, sizeof(long long), "stop step"));
    TRY(X.alloc(&X.base, sizeof(int), "step counter"));
    h.status = X.status;
    h.stop_step = X.stop;
    h.base = X.base;
    TRY(X.alloc(&X.d_dev, sizeof(Dev), "descriptor"));
    CK(cudaMemset(h.cnt, 0, 4 * sizeof(unsigned)));
    // twiddle tables: one plain table per distinct size, copied into the pass-major tables
    const int sizes[3] = {nx, ny, nz};
    const Set* sets[3] = {sx, sy, sz};
    for (int a = 0; a < 3; ++a) {
      bool seen = false;
      for (int b = 0; b < a; ++b) seen |= sizes[b] == sizes[a];
      if (seen) continue;
      const std::vector<double> t = plain_twiddles(sizes[a]);
      TRY(X.alloc(&X.tw[a], t.size() * sizeof(double), "twiddles"));
      CK(cudaMemcpy(X.tw[a], t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
      sets[a]->fill_tables(X.tw[a], X.stream);
    }
    CK(cudaMemcpy(X.d_dev, &h, sizeof(Dev), cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(X.stream));
    CK(cudaGetLastError());
    return ESC_OK;
  };
  const esc_status s = setup();
  if (s != ESC_OK) return bail(s);
  *out = Xp;
  return ESC_OK;
}

esc_status esc_cphi_set_stream(esc_cphi* ctx, void* stream) {
  if (!ctx) {
    esc_set_thread_error("null context");
    return ESC_EINVAL;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
  if (s != ctx->stream) {
    // graphs keep their launch configuration, not the stream: nothing to rebuild
    ctx->stream = s;
  }
  return ESC_OK;
}

esc_status esc_cphi_run(esc_cphi* ctx, double* c, double* phi, int steps, double dt, double tolerance,
                        double comperr, double* history, int64_t* steps_done, int* stop_reason) {
  if (!ctx) {
    esc_set_thread_error("null context");
    return ESC_EINVAL;
  }
  return run_impl(*ctx, c, phi, false, steps, dt, tolerance, comperr, history, steps_done, stop_reason);
}

esc_status esc_cphi_run_device(esc_cphi* ctx, double* c, double* phi, int steps, double dt, double tolerance,
                               double comperr, double* history, int64_t* steps_done, int* stop_reason) {
  if (!ctx) {
    esc_set_thread_error("null context");
    return ESC_EINVAL;
  }
  return run_impl(*ctx, c, phi, true, steps, dt, tolerance, comperr, history, steps_done, stop_reason);
}

esc_status esc_cphi_profile(esc_cphi* ctx, int steps, double* ms) {
  if (!ctx || steps < 1 || !ms) {
    esc_set_thread_error("bad argument");
    return ESC_EINVAL;
  }
  esc_cphi& X = *ctx;
  if (!X.hist) return X.fail(ESC_EINVAL, "profile needs a previous run (it steps the fields that run left)");
  Guard dg(X.device);
  cudaStream_t st = X.stream;
  // step on from the last run's fields: no early stop, history into row 0 of the library's buffer
  X.h.tol = -1.0;
  X.h.comperr = INFINITY;
  X.h.hist_ld = 1;
  CK(cudaMemcpyAsync(X.d_dev, &X.h, sizeof(Dev), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(X.status, 0, sizeof(int), st));
  CK(cudaMemsetAsync(X.base, 0, sizeof(int), st));
  cudaEvent_t ev[kStepKernels + 1];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(kStepKernels, 0.0);
  esc_status rs = ESC_OK;
  for (int s = 0; s < steps && rs == ESC_OK; ++s) {
    CK(cudaMemsetAsync(X.base, 0, sizeof(int), st));
    launch_step(X, 0, st, ev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[kStepKernels]);
    for (int k = 0; k < kStepKernels && e == cudaSuccess; ++k) {
      float t = 0.f;
      e = cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
    if (e != cudaSuccess) rs = X.fail_cuda("profile", e);
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (rs != ESC_OK) return rs;
  for (int k = 0; k < kStepKernels; ++k) ms[k] = acc[k] / steps;
  return ESC_OK;
}

const char* esc_cphi_last_error(const esc_cphi* ctx) { return ctx ? ctx->err.c_str() : esc_last_error(nullptr); }

void esc_cphi_destroy(esc_cphi* ctx) {
  if (!ctx) return;
  {
    Guard dg(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->release();
  }
  delete ctx;
}

}  // extern "C"
