// C ABI host library: contexts, batches, CUDA-graph step chunks.
//
// The public entry points mirror the Julia driver core_shell.jl:84-103
// (run_simulation).  A context is a batch of one.  A batch groups its
// instances by grid size; each group owns contiguous device buffers and a
// device array of instance descriptors, and every phase kernel of a step is one
// launch per group whose grid is (tiles, instances).  Steps are replayed from
// captured CUDA graphs of 32, 16, 8, 4, 2 and 1 steps; a device-side step counter
// gives each launch its history row, so the graphs never need re-instantiation.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "esc.h"
#include "esc_cluster.h"
#include "esc_dispatch.cuh"

#define ESC_DECL(n) const esc::KernelSet* esc_kernels_##n(int prec);
ESC_SIZES(ESC_DECL)
#undef ESC_DECL
// runtime-size kernel sets (esc_generic.cu)
const esc::KernelSet* esc_generic_kernels(int n, int prec);
int esc_generic_supported(int n);

namespace {

// ESC_GENERIC = 1 (a validation knob): use the runtime-size kernels even where a
// tuned kernel set exists, so that tests can compare them with the oracle at any n.
bool force_generic() {
  const char* v = getenv("ESC_GENERIC");
  return v && v[0] == '1';
}

// The tuned, compile-time kernel set of n, else the runtime-size set (any n the
// reference accepts within esc_generic_supported), else null.
const esc::KernelSet* find_kernels(int n, int prec) {
  if (!force_generic()) {
    switch (n) {
#define ESC_CASE(nn) \
  case nn:           \
    return esc_kernels_##nn(prec);
      ESC_SIZES(ESC_CASE)
#undef ESC_CASE
      default:
        break;
    }
  }
  return esc_generic_kernels(n, prec);
}

thread_local std::string tl_err;

// Smooth synthetic composition used only to time kernel variants.
__global__ void k_fill_tuning_field(double* c, int n, int count) {
  const size_t total = (size_t)n * n * count;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % n), y = (int)((i / n) % n);
    c[i] = 0.5 + 0.01 * sin(6.283185307179586 * (3.0 * x + 5.0 * y) / n);
  }
}

// Advances the device-side step counter read by the phase kernels.
__global__ void k_advance(int* base, int by) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *base += by;
}
// Graphs are captured for chunks of 32, 16, 8, 4, 2 and 1 steps, so that any step
// count runs as at most K/32 + 5 graph launches per group.
constexpr int kNumChunks = 6;
constexpr int kChunkSteps[kNumChunks] = {32, 16, 8, 4, 2, 1};

struct Group {
  const esc::KernelSet* ks = nullptr;
  int n = 0;
  std::vector<int> members;  // batch indices, in slot order
  void* S = nullptr;
  void* F = nullptr;
  void* G = nullptr;
  void* phi = nullptr;
  void* tw_s = nullptr;
  void* tw_w = nullptr;
  double* cio = nullptr;
  double* part = nullptr;
  double* scal = nullptr;
  unsigned* cnt = nullptr;
  int* status = nullptr;
  long long* bad = nullptr;
  int* base = nullptr;               // this group's step counter (history row of its next step)
  cudaGraphExec_t gexec[kNumChunks] = {};  // kChunkSteps[i] steps of this group, captured on its own stream
  esc::InstDev* d_inst = nullptr;
  std::vector<esc::InstDev> h_inst;
  esc::ColMaps maps;      // tensor maps of S, F, G for the pipelined column kernels
  bool pipe_rows = false;  // use the persistent TMA-fed row kernels
  bool warp_rows = false;  // use the warp-independent row kernels
  bool pipe_cols = false;  // use the persistent TMA-fed column kernels
  // autotuner outcome: chosen families and measured ms per launch pair
  int row_family = -1, col_family = -1;
  float row_ms[3] = {-1, -1, -1}, col_ms[3] = {-1, -1, -1};
};

// Creating a context touches state shared by every context of the process: the
// tuner's decision cache and its file, the occupancy table of the persistent
// kernels and the tensor-map encoder lookup.  Creations are therefore
// serialised under this lock; running, profiling and destroying contexts take
// no lock.
std::mutex& creation_mutex() {
  static std::mutex m;
  return m;
}

// cuTensorMapEncodeTiled from the driver, looked up once
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 3-D map over `count` instances of n rows of `row_scalars` scalars; box = (box_x, RB, 1)
bool encode_map(CUtensorMap* map, void* base, size_t scalar_bytes, int row_scalars, int rows, int count, int box_x,
                int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const CUtensorMapDataType dt = scalar_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[3] = {(cuuint64_t)row_scalars, (cuuint64_t)rows, (cuuint64_t)count};
  const cuuint64_t strides[2] = {(cuuint64_t)row_scalars * scalar_bytes,
                                 (cuuint64_t)row_scalars * scalar_bytes * (cuuint64_t)rows};
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool pipeline_enabled() {
  const char* v = getenv("ESC_PIPE");
  return !(v && v[0] == '0');
}

// ESC_PIPE_DROP_COPY = 1 (read at creation; a test knob): the TMA pipeline kernels
// withhold their first tile copy, so that the bounded wait for it runs out and the
// run reports ESC_ETIMEOUT.  Nothing is left in flight: no copy was issued for it.
bool drop_copy_knob() {
  const char* v = getenv("ESC_PIPE_DROP_COPY");
  return v && v[0] == '1';
}

// ESC_SPLIT = k: split each grid size with at least 2k particles into k groups
// on their own streams, so that different phases of the same size overlap.
int split_factor() {
  const char* v = getenv("ESC_SPLIT");
  const int k = v ? atoi(v) : 1;
  return k >= 1 && k <= 8 ? k : 1;
}

// ESC_H2D_ORDER = i0,i1,...: the queue order of the groups in a host-buffer batch
// run, as indices into the groups sorted by ascending points (measurement aid;
// an order that does not name every group once is ignored).
bool h2d_order_knob(std::vector<int>& pos, int ng) {
  const char* v = getenv("ESC_H2D_ORDER");
  if (!v) return false;
  pos.clear();
  for (const char* q = v; *q;) {
    char* e = nullptr;
    const long k = strtol(q, &e, 10);
    if (e == q || k < 0 || k >= ng) return false;
    pos.push_back((int)k);
    q = *e == ',' ? e + 1 : e;
    if (*e && *e != ',') return false;
  }
  if ((int)pos.size() != ng) return false;
  std::vector<char> seen(ng, 0);
  for (int k : pos) {
    if (seen[k]) return false;
    seen[k] = 1;
  }
  return true;
}

// ESC_ROWS = warp | pipe | legacy forces one row-kernel family (measurement aid)
int row_family_override() {
  const char* v = getenv("ESC_ROWS");
  if (!v) return -1;
  if (!strcmp(v, "legacy")) return 0;
  if (!strcmp(v, "pipe")) return 1;
  if (!strcmp(v, "warp")) return 2;
  return -1;
}

// ESC_COLS = block | pipe | alt forces one column-kernel family (measurement aid)
int col_family_override() {
  const char* v = getenv("ESC_COLS");
  if (!v) return -1;
  if (!strcmp(v, "block")) return 0;
  if (!strcmp(v, "pipe")) return 1;
  if (!strcmp(v, "alt")) return 2;
  return -1;
}

struct Engine {
  int count = 0;
  int prec = 0;
  int device = 0;
  std::vector<int> n;
  std::vector<double> dx;
  std::vector<esc::ModelParams> p;
  std::vector<Group> groups;
  std::vector<std::pair<int, int>> where;  // instance -> (group, slot)
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  int* base = nullptr;
  double* hist = nullptr;
  size_t hist_cap = 0;  // doubles
  std::vector<cudaStream_t> side;    // per-group streams (their graphs, copies and tails)
  std::vector<cudaEvent_t> side_ev;  // per-group completion / join events
  cudaEvent_t fork_ev = nullptr;
  // statuses of a device-memory run, copied back in stream order (pinned; group-major slots)
  int* h_status = nullptr;
  long long* h_bad = nullptr;
  bool pending = false;  // a device-memory run was queued and not yet waited for
  // a single FP64 grid of a size with a cluster configuration runs its whole loop
  // in one cluster launch (esc_cluster.cu) instead of four launches per step
  bool cluster = false;
  std::vector<void*> allocs;
  std::string err;
  // adjoint resources (allocated on first use; single-instance contexts)
  struct Adj {
    bool ready = false;
    int ckpt_cap = 0, seg_cap = 0;
    const esc::KernelSet* ks64 = nullptr;
    double *phi64 = nullptr, *target = nullptr, *part = nullptr, *scal = nullptr, *hist = nullptr,
           *acc = nullptr, *cout = nullptr;
    double2 *F64 = nullptr, *Lam = nullptr, *Xg = nullptr, *ckpt = nullptr;
    esc::cpx2<double>* G64 = nullptr;
    void* tw64 = nullptr;
    unsigned *cnt = nullptr, *acnt = nullptr;
    int *status = nullptr, *zero = nullptr;
    long long* bad = nullptr;
    esc::InstDev* d_seed = nullptr;  // FP64 shadow instance with a 1-row history
    esc::InstDev* d_bwd = nullptr;   // FP64 shadow instance without history
    esc::InstDev* d_out = nullptr;   // final transform of the adjoint
    // mixed contexts: the adjoint step transforms its derived fields in FP32
    bool mixed = false;
    esc::cpx2<float>* Gw = nullptr;  // FP32 pair array of the mixed step
    esc::cpx<float>* Xw = nullptr;   // FP32 x-transform of g
    esc::InstDev* d_bwd_m = nullptr; // mixed shadow instance for the forward row B kernel
    esc::AdjDev* d_adj = nullptr;    // one per step of a segment, per segment buffer
    double2* seg_buf[2] = {nullptr, nullptr};  // recomputed states of a segment (double-buffered)
    cudaStream_t sweep = nullptr;    // the adjoint sweep runs here, beside the next recompute
    cudaEvent_t recomputed[2] = {nullptr, nullptr}, swept[2] = {nullptr, nullptr};
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;  // (kind * 2 + buffer, steps) -> graph
    size_t pstride = 0;              // partial-sum doubles per instance
  } adj;

  esc_status fail(esc_status s, const std::string& msg) {
    err = msg;
    tl_err = msg;
    return s;
  }
  esc_status fail_cuda(const char* what, cudaError_t e) {
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return fail(e == cudaErrorMemoryAllocation ? ESC_ENOMEM : ESC_ECUDA, buf);
  }

  template <typename T>
  esc_status alloc(T** ptr, size_t bytes, const char* what) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
    if (e != cudaSuccess) return fail_cuda(what, e);
    allocs.push_back(q);
    *ptr = static_cast<T*>(q);
    return ESC_OK;
  }

  void release() {
    for (Group& g : groups)
      for (cudaGraphExec_t& x : g.gexec) {
        if (x) cudaGraphExecDestroy(x);
        x = nullptr;
      }
    if (h_status) cudaFreeHost(h_status);
    if (h_bad) cudaFreeHost(h_bad);
    h_status = nullptr;
    h_bad = nullptr;
    for (auto& kv : adj.graphs) cudaGraphExecDestroy(kv.second);
    adj.graphs.clear();
    for (int b = 0; b < 2; ++b) {
      if (adj.recomputed[b]) cudaEventDestroy(adj.recomputed[b]);
      if (adj.swept[b]) cudaEventDestroy(adj.swept[b]);
      adj.recomputed[b] = adj.swept[b] = nullptr;
    }
    if (adj.sweep) cudaStreamDestroy(adj.sweep);
    adj.sweep = nullptr;
    for (cudaStream_t s : side) cudaStreamDestroy(s);
    side.clear();
    for (cudaEvent_t e : side_ev) cudaEventDestroy(e);
    side_ev.clear();
    if (fork_ev) cudaEventDestroy(fork_ev);
    fork_ev = nullptr;
    for (void* q : allocs) cudaFree(q);
    allocs.clear();
    if (own) cudaStreamDestroy(own);
    own = nullptr;
  }
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

#define CK(call)                                             \
  do {                                                       \
    const cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return E.fail_cuda(#call, e_);    \
  } while (0)
#define TRY(call)                         \
  do {                                    \
    const esc_status s_ = (call);         \
    if (s_ != ESC_OK) return s_;          \
  } while (0)

bool finite_params(const esc_params& q) {
  const double v[10] = {q.A, q.B, q.chi, q.P, q.ca, q.cb, q.cc, q.kappa, q.mobility, q.Q};
  for (double x : v)
    if (!std::isfinite(x)) return false;
  return true;
}

// e^{-2 pi i j / n}, j < n, from long-double trigonometry, written as `real` pairs.
template <typename real>
std::vector<real> twiddles(int n) {
  std::vector<real> t(2 * (size_t)n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int j = 0; j < n; ++j) {
    const long double a = two_pi * (long double)j / (long double)n;
    t[2 * (size_t)j] = (real)cosl(a);
    t[2 * (size_t)j + 1] = (real)(-sinl(a));
  }
  return t;
}

esc_status engine_create(Engine& E, int count, const int* n, const double* dx, const double* const* phi,
                         const esc_params* p, int prec) {
  if (count < 1) return E.fail(ESC_EINVAL, "count must be >= 1");
  if (!n || !dx || !phi || !p) return E.fail(ESC_EINVAL, "null argument");
  if (prec != ESC_FP64 && prec != ESC_MIXED) return E.fail(ESC_EINVAL, "unknown precision");
  for (int i = 0; i < count; ++i) {
    if (!esc_supported_size(n[i]))
      return E.fail(ESC_EINVAL, "unsupported grid size " + std::to_string(n[i]) +
                                    " (need 2 <= n <= 4096 with every prime factor <= 127, or n <= 512)");
    if (!(dx[i] > 0.0) || !std::isfinite(dx[i])) return E.fail(ESC_EINVAL, "spacing must be positive and finite");
    if (!phi[i]) return E.fail(ESC_EINVAL, "null particle field");
    if (!finite_params(p[i])) return E.fail(ESC_EINVAL, "non-finite model parameter");
  }
  CK(cudaGetDevice(&E.device));
  E.count = count;
  E.prec = prec;
  E.n.assign(n, n + count);
  E.dx.assign(dx, dx + count);
  E.p.resize(count);
  for (int i = 0; i < count; ++i) {
    const esc_params& q = p[i];
    E.p[i] = esc::ModelParams{q.A, q.B, q.chi, q.P, q.ca, q.cb, q.cc, q.kappa, q.mobility, q.Q};
  }
  // Groups: one per grid size, or, with ESC_SPLIT = k > 1, sizes with at least 2k
  // particles split into k groups of equal size that advance on their own streams.
  const int split = split_factor();
  std::map<int, int> per_size;
  for (int i = 0; i < count; ++i) ++per_size[n[i]];
  std::map<std::pair<int, int>, int> gi;
  std::map<int, int> seen;
  E.where.resize(count);
  for (int i = 0; i < count; ++i) {
    const int k = (split > 1 && per_size[n[i]] >= 2 * split) ? split : 1;
    const int sub = seen[n[i]]++ % k;
    auto it = gi.find({n[i], sub});
    if (it == gi.end()) {
      it = gi.emplace(std::make_pair(n[i], sub), (int)E.groups.size()).first;
      E.groups.emplace_back();
      E.groups.back().n = n[i];
    }
    Group& g = E.groups[it->second];
    E.where[i] = {it->second, (int)g.members.size()};
    g.members.push_back(i);
  }
  CK(cudaStreamCreateWithFlags(&E.own, cudaStreamNonBlocking));
  E.stream = E.own;
  TRY(E.alloc(&E.base, sizeof(int), "step counter"));
  for (Group& g : E.groups) {
    g.ks = find_kernels(g.n, prec);
    if (!g.ks) return E.fail(ESC_EINVAL, "no kernels for n=" + std::to_string(g.n));
    CK(g.ks->prepare());
    const size_t cnt = g.members.size();
    const size_t nn = (size_t)g.n * g.n;
    const size_t sr = g.ks->sr_bytes, wr = g.ks->wr_bytes;
    const size_t fe = g.ks->cplx_per_field;  // complex elements per field and instance
    TRY(E.alloc(&g.S, cnt * fe * 2 * sr, "state buffer"));
    TRY(E.alloc(&g.F, cnt * fe * 2 * wr, "f' buffer"));
    TRY(E.alloc(&g.G, cnt * fe * 4 * wr, "flux buffer"));
    TRY(E.alloc(&g.phi, cnt * nn * wr, "particle buffer"));
    TRY(E.alloc(&g.tw_s, (size_t)g.n * 2 * sr, "twiddles"));
    TRY(E.alloc(&g.tw_w, (size_t)g.n * 2 * wr, "twiddles"));
    TRY(E.alloc(&g.cio, cnt * nn * sizeof(double), "field staging"));
    TRY(E.alloc(&g.part, cnt * (size_t)g.ks->part_len * sizeof(double), "partials"));
    TRY(E.alloc(&g.scal, cnt * 4 * sizeof(double), "scalars"));
    TRY(E.alloc(&g.cnt, cnt * 4 * sizeof(unsigned), "counters"));
    TRY(E.alloc(&g.status, cnt * sizeof(int), "status"));
    TRY(E.alloc(&g.bad, cnt * sizeof(long long), "bad step"));
    TRY(E.alloc(&g.base, sizeof(int), "step counter"));
    TRY(E.alloc(&g.d_inst, cnt * sizeof(esc::InstDev), "descriptors"));
    // twiddles
    if (sr == 8) {
      auto t = twiddles<double>(g.n);
      CK(cudaMemcpy(g.tw_s, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (wr == 8) {
      auto t = twiddles<double>(g.n);
      CK(cudaMemcpy(g.tw_w, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
      auto t = twiddles<float>(g.n);
      CK(cudaMemcpy(g.tw_w, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    g.ks->fill_tables(g.tw_s, g.tw_w, E.own);
    CK(cudaGetLastError());
    // particle fields in the work precision
    if (wr == 8) {
      for (size_t s = 0; s < cnt; ++s)
        CK(cudaMemcpy(static_cast<double*>(g.phi) + s * nn, phi[g.members[s]], nn * sizeof(double),
                      cudaMemcpyHostToDevice));
    } else {
      std::vector<float> tmp(nn);
      for (size_t s = 0; s < cnt; ++s) {
        const double* src = phi[g.members[s]];
        for (size_t k = 0; k < nn; ++k) tmp[k] = (float)src[k];
        CK(cudaMemcpy(static_cast<float*>(g.phi) + s * nn, tmp.data(), nn * sizeof(float),
                      cudaMemcpyHostToDevice));
      }
    }
    g.h_inst.resize(cnt);
    for (size_t s = 0; s < cnt; ++s) {
      esc::InstDev& d = g.h_inst[s];
      memset(&d, 0, sizeof d);
      const int i = g.members[s];
      d.n = g.n;
      d.dx = E.dx[i];
      d.p = E.p[i];
      d.S = static_cast<char*>(g.S) + s * fe * 2 * sr;
      d.F = static_cast<char*>(g.F) + s * fe * 2 * wr;
      d.G = static_cast<char*>(g.G) + s * fe * 4 * wr;
      d.phi = static_cast<char*>(g.phi) + s * nn * wr;
      d.part = g.part + s * (size_t)g.ks->part_len;
      d.cnt = g.cnt + s * 4;
      d.scal = g.scal + s * 4;
      d.status = g.status + s;
      d.bad_step = g.bad + s;
      d.tw_s = g.tw_s;
      d.tw_w = g.tw_w;
      d.cio = g.cio + s * nn;
      d.drop_first_copy = drop_copy_knob() ? 1 : 0;
    }
    // valid descriptors from creation on (no history, dt = 0 until a run sets them), so that
    // no kernel can ever read an unwritten descriptor
    CK(cudaMemcpy(g.d_inst, g.h_inst.data(), cnt * sizeof(esc::InstDev), cudaMemcpyHostToDevice));
    CK(cudaMemset(g.cnt, 0, cnt * 4 * sizeof(unsigned)));
    CK(cudaMemset(g.status, 0, cnt * sizeof(int)));
    if (g.ks->warp_rows) {
      CK(g.ks->prepare_warp());
      g.warp_rows = true;
    }
    if (pipeline_enabled()) {
      CK(g.ks->prepare_pipe());
      g.pipe_rows = g.ks->pipe_rows;
      if (g.ks->pipe_cols) {
        const int H = g.n / 2, W = g.ks->W, RB = g.ks->RB;
        g.pipe_cols = encode_map(&g.maps.S, g.S, sr, 2 * H, g.n, (int)cnt, 2 * W, RB) &&
                      encode_map(&g.maps.F, g.F, wr, 2 * H, g.n, (int)cnt, 2 * W, RB) &&
                      encode_map(&g.maps.G, g.G, wr, 4 * H, g.n, (int)cnt, 4 * W, RB);
      }
    }
    const int rf = row_family_override();
    if (rf == 0) g.pipe_rows = g.warp_rows = false;
    if (rf == 1) g.warp_rows = false;
    if (rf == 2 && g.warp_rows) g.pipe_rows = false;
  }
  CK(cudaDeviceSynchronize());
  return ESC_OK;
}

// One step of every group: record history row (base + s_local) and advance.
void phase_row_a(Group& g, const int* base, int s_local, cudaStream_t st) {
  const int c = (int)g.members.size();
  if (g.warp_rows)
    g.ks->row_a_w(g.d_inst, c, base, s_local, st);
  else if (g.pipe_rows)
    g.ks->row_a_p(g.d_inst, c, base, s_local, st);
  else
    g.ks->row_a(g.d_inst, c, base, s_local, st);
}
void phase_col_a(Group& g, const int* base, int s_local, cudaStream_t st) {
  const int c = (int)g.members.size();
  if (g.col_family == 2)
    g.ks->col_a_alt(g.d_inst, c, base, s_local, st);
  else if (g.pipe_cols)
    g.ks->col_a_p(g.d_inst, c, base, s_local, st, &g.maps);
  else
    g.ks->col_a(g.d_inst, c, base, s_local, st);
}
void phase_row_b(Group& g, const int* base, int s_local, cudaStream_t st) {
  const int c = (int)g.members.size();
  if (g.warp_rows)
    g.ks->row_b_w(g.d_inst, c, base, s_local, st);
  else if (g.pipe_rows)
    g.ks->row_b_p(g.d_inst, c, base, s_local, st);
  else
    g.ks->row_b(g.d_inst, c, base, s_local, st);
}
void phase_col_b(Group& g, cudaStream_t st) {
  const int c = (int)g.members.size();
  if (g.col_family == 2)
    g.ks->col_b_alt(g.d_inst, c, st);
  else if (g.pipe_cols)
    g.ks->col_b_p(g.d_inst, c, st, &g.maps);
  else
    g.ks->col_b(g.d_inst, c, st);
}

// ---- autotuner -----------------------------------------------------------------
// For every size group it times each available row family (0 legacy block
// kernels, 1 persistent TMA pipeline, 2 warp-independent) on row A + row B and
// each column family (0 legacy, 1 persistent TMA pipeline) on column A + column
// B, on a smooth synthetic state, and keeps the fastest.  Decisions are cached
// per process by (n, precision, instances) and, when ESC_TUNE_CACHE names a
// file, read from / appended to it so that later processes reuse them.
// ESC_TUNE=0 skips timing and takes the warp rows and legacy columns; it and a
// family forced with ESC_ROWS / ESC_COLS bypass the cached decisions.
struct TuneKey {
  int n, prec, count;
  bool operator<(const TuneKey& o) const {
    return n != o.n ? n < o.n : (prec != o.prec ? prec < o.prec : count < o.count);
  }
};
std::map<TuneKey, std::pair<int, int>>& tune_cache() {
  static std::map<TuneKey, std::pair<int, int>> m;
  return m;
}
void load_tune_file() {
  static bool loaded = false;
  if (loaded) return;
  loaded = true;
  const char* path = getenv("ESC_TUNE_CACHE");
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  int n, p, c, r, k;
  while (fscanf(f, " {\"n\": %d, \"prec\": %d, \"count\": %d, \"rows\": %d, \"cols\": %d}", &n, &p, &c, &r, &k) == 5)
    tune_cache()[TuneKey{n, p, c}] = {r, k};
  fclose(f);
}
void save_tune(const TuneKey& key, int r, int k) {
  const char* path = getenv("ESC_TUNE_CACHE");
  if (!path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "{\"n\": %d, \"prec\": %d, \"count\": %d, \"rows\": %d, \"cols\": %d}\n", key.n, key.prec, key.count, r, k);
  fclose(f);
}
bool tuning_enabled() {
  const char* v = getenv("ESC_TUNE");
  return !(v && v[0] == '0');
}

void apply_rows(Group& g, int fam) {
  g.row_family = fam;
  g.warp_rows = fam == 2;
  g.pipe_rows = fam == 1;
}
void apply_cols(Group& g, int fam) {
  g.col_family = fam;
  g.pipe_cols = fam == 1 && g.pipe_cols;
}
// column family 2 (alternative plan) needs no capability beyond the kernel set

esc_status autotune(Engine& E) {
  load_tune_file();
  cudaStream_t st = E.own;
  const bool timing = tuning_enabled() && row_family_override() < 0 && pipeline_enabled();
  bool any = false;
  for (Group& g : E.groups) {
    // the runtime-size kernels have one family each: nothing to time, and their
    // group must neither read nor write the decisions kept for a tuned set of the
    // same (n, precision, count), whose column family 2 they do not have
    if (g.ks->generic) {
      apply_rows(g, 0);
      apply_cols(g, 0);
      continue;
    }
    const bool can_pipe_rows = g.pipe_rows, can_warp = g.warp_rows, can_pipe_cols = g.pipe_cols;
    const TuneKey key{g.n, E.prec, (int)g.members.size()};
    auto hit = tune_cache().find(key);
    // a family forced by ESC_ROWS / ESC_COLS, or ESC_TUNE=0, takes precedence over cached decisions
    const bool use_cache = tuning_enabled() && row_family_override() < 0 && col_family_override() < 0;
    if (use_cache && hit != tune_cache().end()) {
      int r = hit->second.first, k = hit->second.second;
      if ((r == 2 && !can_warp) || (r == 1 && !can_pipe_rows)) r = 0;
      // a decision read from a file may name a family this kernel set lacks
      if ((k == 1 && !can_pipe_cols) || (k == 2 && g.ks->E_alt == g.ks->E) || k < 0 || k > 2) k = 0;
      apply_rows(g, r);
      apply_cols(g, k);
      continue;
    }
    if (!timing) {
      if (row_family_override() < 0) apply_rows(g, can_warp ? 2 : (can_pipe_rows ? 1 : 0));
      else g.row_family = g.warp_rows ? 2 : (g.pipe_rows ? 1 : 0);
      // columns: the block kernels unless ESC_COLS asks for a family this size can run
      const int cfo = col_family_override();
      apply_cols(g, ((cfo == 1 && can_pipe_cols) || (cfo == 2 && g.ks->E_alt != g.ks->E)) ? cfo : 0);
      continue;
    }
    any = true;
  }
  if (!any) return ESC_OK;
  // synthetic state for the groups still to be tuned
  for (Group& g : E.groups) {
    if (g.row_family >= 0) continue;
    for (size_t s = 0; s < g.members.size(); ++s) {
      g.h_inst[s].dt = 0.01;
      g.h_inst[s].hist = nullptr;
      g.h_inst[s].hist_ld = 1;
    }
    CK(cudaMemcpyAsync(g.d_inst, g.h_inst.data(), g.h_inst.size() * sizeof(esc::InstDev), cudaMemcpyHostToDevice, st));
    k_fill_tuning_field<<<1024, 256, 0, st>>>(g.cio, g.n, (int)g.members.size());
    CK(cudaMemsetAsync(g.status, 0, g.members.size() * sizeof(int), st));
    CK(cudaMemsetAsync(g.cnt, 0, g.members.size() * 4 * sizeof(unsigned), st));
    g.ks->init(g.d_inst, (int)g.members.size(), st);
  }
  CK(cudaMemsetAsync(E.base, 0, sizeof(int), st));
  CK(cudaGetLastError());
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int reps = 5;
  auto time_it = [&](auto&& launch) -> float {
    launch();  // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / reps;
  };
  for (Group& g : E.groups) {
    if (g.row_family >= 0) continue;
    const bool can_pipe_rows = g.pipe_rows, can_warp = g.warp_rows, can_pipe_cols = g.pipe_cols;
    // columns first (they leave F/G in place for the rows)
    float best_c = 1e30f;
    int best_cf = 0;
    const int cfo = col_family_override();
    for (int cf = 0; cf < 3; ++cf) {
      if (cfo >= 0 && cf != cfo && !(cf == 0 && ((cfo == 1 && !can_pipe_cols) || (cfo == 2 && g.ks->E_alt == g.ks->E))))
        continue;
      if (cf == 1 && !can_pipe_cols) continue;
      if (cf == 2 && g.ks->E_alt == g.ks->E) continue;  // same plan as family 0
      g.pipe_cols = cf == 1;
      g.col_family = cf;
      const float ms = time_it([&] {
        phase_col_a(g, E.base, 0, st);
        phase_col_b(g, st);
      });
      g.col_ms[cf] = ms;
      if (ms < best_c) {
        best_c = ms;
        best_cf = cf;
      }
    }
    g.pipe_cols = can_pipe_cols;
    g.col_family = -1;
    apply_cols(g, best_cf);
    float best_r = 1e30f;
    int best_rf = 0;
    for (int rf = 0; rf < 3; ++rf) {
      if ((rf == 1 && !can_pipe_rows) || (rf == 2 && !can_warp)) continue;
      g.pipe_rows = rf == 1;
      g.warp_rows = rf == 2;
      const float ms = time_it([&] {
        phase_row_a(g, E.base, 0, st);
        phase_row_b(g, E.base, 0, st);
      });
      g.row_ms[rf] = ms;
      if (ms < best_r) {
        best_r = ms;
        best_rf = rf;
      }
    }
    g.pipe_rows = can_pipe_rows;
    g.warp_rows = can_warp;
    apply_rows(g, best_rf);
    if (col_family_override() < 0) {  // a forced column family is not a decision to keep
      const TuneKey key{g.n, E.prec, (int)g.members.size()};
      tune_cache()[key] = {best_rf, best_cf};
      save_tune(key, best_rf, best_cf);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  // tuning may have flagged nothing, but leave a clean slate for the first run
  for (Group& g : E.groups) {
    CK(cudaMemset(g.status, 0, g.members.size() * sizeof(int)));
    CK(cudaMemset(g.cnt, 0, g.members.size() * 4 * sizeof(unsigned)));
  }
  return ESC_OK;
}

void launch_step(Engine& E, int s_local, cudaStream_t st) {
  for (Group& g : E.groups) {
    phase_row_a(g, E.base, s_local, st);
    phase_col_a(g, E.base, s_local, st);
    phase_row_b(g, E.base, s_local, st);
    phase_col_b(g, st);
  }
}

// Each size group advances on its own stream: captured graphs of 32, 16, ..., 1
// steps of that group with its own step counter.  The groups' chains are independent
// (one instance never reads another), so they overlap on the GPU and fill each
// other's launch tails, and in a run with host buffers one group's copies
// overlap the other groups' steps.
esc_status ensure_graph(Engine& E) {
  const int ng = (int)E.groups.size();
  if ((int)E.side.size() < ng) {
    // stream priority by work: the group with the most points gets the highest
    // priority, so it finishes first and its D2H copies overlap the rest
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    for (int i = (int)E.side.size(); i < ng; ++i) {
      const double work = (double)E.groups[i].members.size() * E.groups[i].n * E.groups[i].n;
      int rank = 0;
      for (int j = 0; j < ng; ++j) {
        const double wj = (double)E.groups[j].members.size() * E.groups[j].n * E.groups[j].n;
        if (wj > work) ++rank;  // groups of equal work share a priority and interleave
      }
      const int prio = std::min(least, greatest + rank);
      cudaStream_t s = nullptr;
      CK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio));
      E.side.push_back(s);
      cudaEvent_t ev = nullptr;
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      E.side_ev.push_back(ev);
    }
    if (!E.fork_ev) CK(cudaEventCreateWithFlags(&E.fork_ev, cudaEventDisableTiming));
  }
  for (int gi = 0; gi < ng; ++gi) {
    Group& g = E.groups[gi];
    cudaStream_t ss = E.side[gi];
    for (int ci = 0; ci < kNumChunks; ++ci) {
      if (g.gexec[ci]) continue;
      const int steps = kChunkSteps[ci];
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(ss, cudaStreamCaptureModeThreadLocal));
      for (int s = 0; s < steps; ++s) {
        phase_row_a(g, g.base, s, ss);
        phase_col_a(g, g.base, s, ss);
        phase_row_b(g, g.base, s, ss);
        phase_col_b(g, ss);
      }
      k_advance<<<1, 32, 0, ss>>>(g.base, steps);
      const cudaError_t ec = cudaStreamEndCapture(ss, &graph);
      if (ec != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return E.fail_cuda("cudaStreamEndCapture", ec);
      }
      const cudaError_t ei = cudaGraphInstantiate(&g.gexec[ci], graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        g.gexec[ci] = nullptr;
        return E.fail_cuda("cudaGraphInstantiate", ei);
      }
      // upload now, so that the first launch of a run does not carry it
      CK(cudaGraphUpload(g.gexec[ci], ss));
    }
    CK(cudaStreamSynchronize(ss));
  }
  if (!E.h_status) {
    CK(cudaMallocHost(reinterpret_cast<void**>(&E.h_status), (size_t)E.count * sizeof(int)));
    CK(cudaMallocHost(reinterpret_cast<void**>(&E.h_bad), (size_t)E.count * sizeof(long long)));
  }
  return ESC_OK;
}

// Queues `steps` steps of group g on stream ss as graph launches (32-step chunks,
// then the binary decomposition of the rest).
esc_status launch_steps(Engine& E, Group& g, int steps, cudaStream_t ss) {
  for (int ci = 0; ci < kNumChunks; ++ci)
    while (steps >= kChunkSteps[ci]) {
      CK(cudaGraphLaunch(g.gexec[ci], ss));
      steps -= kChunkSteps[ci];
    }
  return ESC_OK;
}

// ESC_CLUSTER=0 keeps single grids on the launch-per-phase path, ESC_CLUSTER=1
// takes the cluster path without timing it; unset, the faster of the two is kept
bool cluster_knob() {
  const char* v = getenv("ESC_CLUSTER");
  return !(v && v[0] == '0');
}
bool cluster_forced() {
  const char* v = getenv("ESC_CLUSTER");
  return v && v[0] == '1';
}

// Single FP64 contexts of n = 128 or 256 run in one cluster launch when the
// device can place the cluster: its twiddle tables are filled here, and the
// status words of queued runs come back through the pinned host slots.
esc_status enable_cluster(Engine& E) {
  if (E.count != 1 || E.prec != ESC_FP64 || E.groups.size() != 1 || !cluster_knob()) return ESC_OK;
  Group& g = E.groups[0];
  if (g.ks->generic || !esc::clu::available(g.n)) return ESC_OK;
  DeviceGuard dg(E.device);
  CK(esc::clu::prepare(g.n, g.tw_s, E.own));
  if (!E.h_status) {
    CK(cudaMallocHost(reinterpret_cast<void**>(&E.h_status), sizeof(int)));
    CK(cudaMallocHost(reinterpret_cast<void**>(&E.h_bad), sizeof(long long)));
  }
  CK(cudaStreamSynchronize(E.own));
  E.cluster = true;
  return ESC_OK;
}

// Queues a cluster run of the single grid on the engine's stream: status words,
// the launch, and the status copies into the pinned host slots.
esc_status cluster_enqueue(Engine& E, double* cdev, int steps, double dt, double* hist) {
  Group& g = E.groups[0];
  cudaStream_t st = E.stream;
  CK(cudaMemsetAsync(g.status, 0, sizeof(int), st));
  CK(cudaMemsetAsync(g.bad, 0xff, sizeof(long long), st));
  esc::clu::Args a;
  a.phi = static_cast<const double*>(g.phi);
  a.c = cdev;
  a.hist = hist;
  a.hist_ld = steps + 1;
  a.steps = steps;
  a.dt = dt;
  a.dx = g.h_inst[0].dx;
  a.p = g.h_inst[0].p;
  a.status = g.status;
  a.bad_step = g.bad;
  CK(esc::clu::run(g.n, a, st));
  CK(cudaMemcpyAsync(E.h_status, g.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(E.h_bad, g.bad, sizeof(long long), cudaMemcpyDeviceToHost, st));
  return ESC_OK;
}

// c_in_out: per-instance pointers (host or device per `device_io`);
// hist_host: per-instance host pointers (entries may be null) or null;
// hist_dev: one device array for all instances or null.
esc_status engine_run(Engine& E, double* const* cptr, bool device_io, int steps, double dt,
                      double* const* hist_host, double* hist_dev, int64_t* bad_out, bool leave_bad_unchanged) {
  if (E.pending) return E.fail(ESC_EINVAL, "a queued run has not been waited for");
  if (steps < 0) return E.fail(ESC_EINVAL, "steps must be >= 0");
  if (!std::isfinite(dt)) return E.fail(ESC_EINVAL, "dt must be finite");
  if (!cptr) return E.fail(ESC_EINVAL, "null composition array");
  for (int i = 0; i < E.count; ++i)
    if (!cptr[i]) return E.fail(ESC_EINVAL, "null composition field");
  DeviceGuard dg(E.device);
  const size_t rows = (size_t)steps + 1;
  const size_t per = rows * 6;
  double* hbase = hist_dev;
  if (!hbase) {
    const size_t need = per * (size_t)E.count;
    if (need > E.hist_cap) {
      if (E.hist) {
        for (auto it = E.allocs.begin(); it != E.allocs.end(); ++it)
          if (*it == E.hist) {
            E.allocs.erase(it);
            break;
          }
        cudaFree(E.hist);
        E.hist = nullptr;
        E.hist_cap = 0;
      }
      TRY(E.alloc(&E.hist, need * sizeof(double), "history"));
      E.hist_cap = need;
    }
    hbase = E.hist;
  }
  cudaStream_t st = E.stream;
  if (E.cluster) {
    Group& g = E.groups[0];
    const size_t nn = (size_t)g.n * g.n;
    double* cdev = device_io ? cptr[0] : g.cio;
    if (!device_io) CK(cudaMemcpyAsync(g.cio, cptr[0], nn * sizeof(double), cudaMemcpyHostToDevice, st));
    TRY(cluster_enqueue(E, cdev, steps, dt, hbase));
    CK(cudaStreamSynchronize(st));
    const int status = *E.h_status;
    const long long bad = *E.h_bad;
    if (!device_io && status == 0) CK(cudaMemcpy(cptr[0], g.cio, nn * sizeof(double), cudaMemcpyDeviceToHost));
    if (hist_host && hist_host[0]) CK(cudaMemcpy(hist_host[0], hbase, per * sizeof(double), cudaMemcpyDeviceToHost));
    if (bad_out) bad_out[0] = status ? (int64_t)bad : -1;
    (void)leave_bad_unchanged;
    if (status) return E.fail(ESC_ENONFINITE, "Non-finite composition at step " + std::to_string(bad));
    return ESC_OK;
  }
  for (Group& g : E.groups) {
    const size_t nn = (size_t)g.n * g.n;
    for (size_t s = 0; s < g.members.size(); ++s) {
      const int i = g.members[s];
      esc::InstDev& d = g.h_inst[s];
      d.dt = dt;
      d.hist = hbase + (size_t)i * per;
      d.hist_ld = (int)rows;
      d.cio = device_io ? cptr[i] : g.cio + s * nn;
    }
    CK(cudaMemcpyAsync(g.d_inst, g.h_inst.data(), g.h_inst.size() * sizeof(esc::InstDev),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(g.status, 0, g.members.size() * sizeof(int), st));
    CK(cudaMemsetAsync(g.bad, 0xff, g.members.size() * sizeof(long long), st));
    CK(cudaMemsetAsync(g.cnt, 0, g.members.size() * 4 * sizeof(unsigned), st));
    CK(cudaMemsetAsync(g.base, 0, sizeof(int), st));
  }
  TRY(ensure_graph(E));
  // Every group runs on its own stream, forked from (and joined back into) the
  // caller's stream: H2D of its fields, the steps, the final history row, and
  // (below) its D2H copies.  The groups are queued in ascending size, so that steps
  // start while the other fields are still being copied in, except that the largest
  // group comes before the second largest; the largest group has the highest stream
  // priority and finishes first.
  const int ng = (int)E.groups.size();
  std::vector<int> order(ng);
  for (int gi = 0; gi < ng; ++gi) order[gi] = gi;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const Group &ga = E.groups[a], &gb = E.groups[b];
    return (double)ga.members.size() * ga.n * ga.n < (double)gb.members.size() * gb.n * gb.n;
  });
  // then the largest group before the second largest: with the highest priority it
  // finishes before the second largest, whose last steps cover its D2H copies
  std::vector<int> pos;
  if (h2d_order_knob(pos, ng)) {
    std::vector<int> asc = order;
    for (int k = 0; k < ng; ++k) order[k] = asc[pos[k]];
  } else if (ng > 2) {
    std::swap(order[ng - 2], order[ng - 1]);
  }
  CK(cudaEventRecord(E.fork_ev, st));
  for (int gi : order) {
    Group& g = E.groups[gi];
    cudaStream_t ss = E.side[gi];
    const int cnt = (int)g.members.size();
    const size_t nn = (size_t)g.n * g.n;
    CK(cudaStreamWaitEvent(ss, E.fork_ev, 0));
    if (!device_io) {
      for (int s = 0; s < cnt; ++s)
        CK(cudaMemcpyAsync(g.cio + s * nn, cptr[g.members[s]], nn * sizeof(double), cudaMemcpyHostToDevice, ss));
    }
    g.ks->init(g.d_inst, cnt, ss);
    TRY(launch_steps(E, g, steps, ss));
    // history row `steps` of the final field (no update)
    phase_row_a(g, g.base, 0, ss);
    phase_col_a(g, g.base, 0, ss);
    phase_row_b(g, g.base, 0, ss);
    g.ks->fin(g.d_inst, cnt, ss);
    CK(cudaGetLastError());
    CK(cudaEventRecord(E.side_ev[gi], ss));
  }
  // As each group finishes: read its statuses, then queue its D2H copies on its
  // stream, beside the groups still stepping; the caller's stream joins them.
  std::vector<int> status(E.count, 0);
  std::vector<long long> bad(E.count, -1);
  std::vector<char> pending(ng, 1);
  for (int left = ng; left > 0;) {
    bool progressed = false;
    for (int gi : order) {
      if (!pending[gi]) continue;
      const cudaError_t q = cudaEventQuery(E.side_ev[gi]);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return E.fail_cuda("cudaEventQuery", q);
      Group& g = E.groups[gi];
      cudaStream_t ss = E.side[gi];
      const size_t cnt = g.members.size(), nn = (size_t)g.n * g.n;
      std::vector<int> sg(cnt);
      std::vector<long long> bg(cnt);
      CK(cudaMemcpyAsync(sg.data(), g.status, cnt * sizeof(int), cudaMemcpyDeviceToHost, ss));
      CK(cudaMemcpyAsync(bg.data(), g.bad, cnt * sizeof(long long), cudaMemcpyDeviceToHost, ss));
      CK(cudaStreamSynchronize(ss));
      for (size_t k = 0; k < cnt; ++k) {
        status[g.members[k]] = sg[k];
        bad[g.members[k]] = bg[k];
      }
      if (!device_io) {
        for (size_t k = 0; k < cnt; ++k) {
          const int i = g.members[k];
          if (status[i] && leave_bad_unchanged) continue;
          CK(cudaMemcpyAsync(cptr[i], g.cio + k * nn, nn * sizeof(double), cudaMemcpyDeviceToHost, ss));
        }
      }
      if (hist_host) {
        for (size_t k = 0; k < cnt; ++k) {
          const int i = g.members[k];
          if (hist_host[i])
            CK(cudaMemcpyAsync(hist_host[i], hbase + (size_t)i * per, per * sizeof(double), cudaMemcpyDeviceToHost,
                               ss));
        }
      }
      CK(cudaEventRecord(E.side_ev[gi], ss));
      CK(cudaStreamWaitEvent(st, E.side_ev[gi], 0));
      pending[gi] = 0;
      --left;
      progressed = true;
    }
    if (!progressed && left > 0) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  bool any_bad = false;
  for (int i = 0; i < E.count; ++i) {
    if (status[i]) any_bad = true;
    if (bad_out) bad_out[i] = status[i] ? (int64_t)bad[i] : -1;
  }
  CK(cudaStreamSynchronize(st));
  if (any_bad) {
    for (int i = 0; i < E.count; ++i)
      if (status[i] == esc::kStatusLayout)
        return E.fail(ESC_ECUDA, "internal error: a shared-memory stage was misaligned; no copy was issued");
    for (int i = 0; i < E.count; ++i)
      if (status[i] == esc::kStatusTimeout)
        return E.fail(ESC_ETIMEOUT, "a bounded wait for a tile copy gave up (instance " + std::to_string(i) + ")");
    for (int i = 0; i < E.count; ++i)
      if (status[i])
        return E.fail(ESC_ENONFINITE, "Non-finite composition at step " + std::to_string(bad[i]) +
                                          (E.count > 1 ? " (instance " + std::to_string(i) + ")" : ""));
  }
  return ESC_OK;
}

// Device-memory run, queued without waiting: descriptors, fork into the groups'
// streams, every group's steps (graph launches), final history row and final
// field, each group's status words copied into pinned host memory, and the join
// back into the caller's stream.  engine_wait reports the outcome.  A stopped
// instance keeps its device c (the final-field kernel skips it).
esc_status engine_enqueue_device(Engine& E, double* const* cptr, int steps, double dt, double* hist_dev) {
  if (E.pending) return E.fail(ESC_EINVAL, "a queued run has not been waited for");
  if (steps < 0) return E.fail(ESC_EINVAL, "steps must be >= 0");
  if (!std::isfinite(dt)) return E.fail(ESC_EINVAL, "dt must be finite");
  if (!cptr) return E.fail(ESC_EINVAL, "null composition array");
  for (int i = 0; i < E.count; ++i)
    if (!cptr[i]) return E.fail(ESC_EINVAL, "null composition field");
  DeviceGuard dg(E.device);
  const size_t rows = (size_t)steps + 1;
  const size_t per = rows * 6;
  double* hbase = hist_dev;
  if (!hbase) {
    const size_t need = per * (size_t)E.count;
    if (need > E.hist_cap) {
      if (E.hist) {
        for (auto it = E.allocs.begin(); it != E.allocs.end(); ++it)
          if (*it == E.hist) {
            E.allocs.erase(it);
            break;
          }
        cudaFree(E.hist);
        E.hist = nullptr;
        E.hist_cap = 0;
      }
      TRY(E.alloc(&E.hist, need * sizeof(double), "history"));
      E.hist_cap = need;
    }
    hbase = E.hist;
  }
  cudaStream_t st = E.stream;
  if (E.cluster) {
    TRY(cluster_enqueue(E, cptr[0], steps, dt, hbase));
    E.pending = true;
    return ESC_OK;
  }
  TRY(ensure_graph(E));
  for (Group& g : E.groups) {
    for (size_t s = 0; s < g.members.size(); ++s) {
      const int i = g.members[s];
      esc::InstDev& d = g.h_inst[s];
      d.dt = dt;
      d.hist = hbase + (size_t)i * per;
      d.hist_ld = (int)rows;
      d.cio = cptr[i];
    }
    CK(cudaMemcpyAsync(g.d_inst, g.h_inst.data(), g.h_inst.size() * sizeof(esc::InstDev),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(g.status, 0, g.members.size() * sizeof(int), st));
    CK(cudaMemsetAsync(g.bad, 0xff, g.members.size() * sizeof(long long), st));
    CK(cudaMemsetAsync(g.cnt, 0, g.members.size() * 4 * sizeof(unsigned), st));
    CK(cudaMemsetAsync(g.base, 0, sizeof(int), st));
  }
  CK(cudaEventRecord(E.fork_ev, st));
  size_t off = 0;
  for (int gi = 0; gi < (int)E.groups.size(); ++gi) {
    Group& g = E.groups[gi];
    cudaStream_t ss = E.side[gi];
    const int cnt = (int)g.members.size();
    CK(cudaStreamWaitEvent(ss, E.fork_ev, 0));
    g.ks->init(g.d_inst, cnt, ss);
    TRY(launch_steps(E, g, steps, ss));
    phase_row_a(g, g.base, 0, ss);
    phase_col_a(g, g.base, 0, ss);
    phase_row_b(g, g.base, 0, ss);
    g.ks->fin(g.d_inst, cnt, ss);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(E.h_status + off, g.status, cnt * sizeof(int), cudaMemcpyDeviceToHost, ss));
    CK(cudaMemcpyAsync(E.h_bad + off, g.bad, cnt * sizeof(long long), cudaMemcpyDeviceToHost, ss));
    off += cnt;
    CK(cudaEventRecord(E.side_ev[gi], ss));
    CK(cudaStreamWaitEvent(st, E.side_ev[gi], 0));
  }
  E.pending = true;
  return ESC_OK;
}

// Waits for the queued device-memory run and reports it like engine_run.
esc_status engine_wait(Engine& E, int64_t* bad_out) {
  if (!E.pending) return E.fail(ESC_EINVAL, "no queued run to wait for");
  DeviceGuard dg(E.device);
  E.pending = false;
  CK(cudaStreamSynchronize(E.stream));
  std::vector<int> status(E.count, 0);
  std::vector<long long> bad(E.count, -1);
  size_t off = 0;
  for (const Group& g : E.groups) {
    for (size_t k = 0; k < g.members.size(); ++k) {
      status[g.members[k]] = E.h_status[off + k];
      bad[g.members[k]] = E.h_bad[off + k];
    }
    off += g.members.size();
  }
  bool any_bad = false;
  for (int i = 0; i < E.count; ++i) {
    if (status[i]) any_bad = true;
    if (bad_out) bad_out[i] = status[i] ? (int64_t)bad[i] : -1;
  }
  if (any_bad) {
    for (int i = 0; i < E.count; ++i)
      if (status[i] == esc::kStatusLayout)
        return E.fail(ESC_ECUDA, "internal error: a shared-memory stage was misaligned; no copy was issued");
    for (int i = 0; i < E.count; ++i)
      if (status[i] == esc::kStatusTimeout)
        return E.fail(ESC_ETIMEOUT, "a bounded wait for a tile copy gave up (instance " + std::to_string(i) + ")");
    for (int i = 0; i < E.count; ++i)
      if (status[i])
        return E.fail(ESC_ENONFINITE, "Non-finite composition at step " + std::to_string(bad[i]) +
                                          (E.count > 1 ? " (instance " + std::to_string(i) + ")" : ""));
  }
  return ESC_OK;
}

// Times 16 steps of the cluster path and of the launch-per-phase path on a smooth
// synthetic field and keeps the faster for this context (the decision is cached
// per grid size and device; creations are serialised).
esc_status choose_cluster(Engine& E) {
  if (!E.cluster || cluster_forced()) return ESC_OK;
  static std::map<std::pair<int, int>, bool> decided;
  Group& g = E.groups[0];
  const auto key = std::make_pair(g.n, E.device);
  auto it = decided.find(key);
  if (it != decided.end()) {
    E.cluster = it->second;
    return ESC_OK;
  }
  DeviceGuard dg(E.device);
  cudaStream_t st = E.stream;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto time_path = [&](bool cluster, float* ms) -> esc_status {
    E.cluster = cluster;
    double* cp[1] = {g.cio};
    for (int rep = 0; rep < 2; ++rep) {  // the first run builds and uploads what the path needs
      k_fill_tuning_field<<<1024, 256, 0, st>>>(g.cio, g.n, 1);
      CK(cudaEventRecord(e0, st));
      TRY(engine_enqueue_device(E, cp, 16, 0.01, nullptr));
      CK(cudaEventRecord(e1, st));
      TRY(engine_wait(E, nullptr));
    }
    CK(cudaEventElapsedTime(ms, e0, e1));
    return ESC_OK;
  };
  float t_cluster = 0.f, t_phases = 0.f;
  esc_status rs = time_path(true, &t_cluster);
  if (rs == ESC_OK) rs = time_path(false, &t_phases);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rs != ESC_OK) return rs;
  E.cluster = t_cluster < t_phases;
  decided[key] = E.cluster;
  return ESC_OK;
}

esc_status engine_run_device(Engine& E, double* const* cptr, int steps, double dt, double* hist_dev,
                             int64_t* bad_out) {
  const esc_status s = engine_enqueue_device(E, cptr, steps, dt, hist_dev);
  if (s != ESC_OK) return s;
  return engine_wait(E, bad_out);
}

}  // namespace

// ---- adjoint driver -----------------------------------------------------------------
// L = 1/2 sum (c_T - c_target)^2 + lamF F[c_T]; gradients w.r.t. c0 and
// theta = (P, chi, kappa, M0).  Forward pass in the context's precision with a
// checkpoint every `K` steps; backward pass recomputes each segment (storing its
// states) and applies the FP64 adjoint step (esc_adjoint.cuh) from the last step
// to the first.
// Captures the launches `issue(stream)` makes as a CUDA graph, once per
// (kind, segment buffer, steps), and returns the cached executable.  Kinds:
// 0 forward steps, 1 recompute of a segment into a segment buffer, 2 adjoint
// sweep over a segment buffer.
template <class Issue>
esc_status adjoint_graph(Engine& E, int kind, int buf, int len, cudaGraphExec_t* out, Issue&& issue) {
  auto& A = E.adj;
  const auto key = std::make_pair(kind * 2 + buf, len);
  const auto it = A.graphs.find(key);
  if (it != A.graphs.end()) {
    *out = it->second;
    return ESC_OK;
  }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(E.own, cudaStreamCaptureModeThreadLocal));
  issue(E.own);
  const cudaError_t ec = cudaStreamEndCapture(E.own, &graph);
  if (ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return E.fail_cuda("cudaStreamEndCapture", ec);
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) return E.fail_cuda("cudaGraphInstantiate", ei);
  const cudaError_t eu = cudaGraphUpload(ex, E.own);
  if (eu != cudaSuccess) {
    cudaGraphExecDestroy(ex);
    return E.fail_cuda("cudaGraphUpload", eu);
  }
  A.graphs[key] = ex;
  *out = ex;
  return ESC_OK;
}

esc_status engine_adjoint(Engine& E, const double* const* c0, int steps, double dt, const double* const* c_target,
                          double lamF, int K, double* const* dL_dc0, double* dL_dparams, double* Lout) {
  if (E.groups.size() != 1) return E.fail(ESC_EINVAL, "the adjoint needs all particles of one grid size");
  if (steps < 1 || !c0 || !c_target) return E.fail(ESC_EINVAL, "bad adjoint arguments");
  if (!std::isfinite(dt) || !std::isfinite(lamF)) return E.fail(ESC_EINVAL, "dt and lambda_F must be finite");
  Group& g = E.groups[0];
  const int cnt = (int)g.members.size();
  for (int s = 0; s < cnt; ++s)
    if (!c0[g.members[s]] || !c_target[g.members[s]]) return E.fail(ESC_EINVAL, "null field in the adjoint inputs");
  if (K < 1) K = (int)std::ceil(std::sqrt((double)steps));
  if (K > steps) K = steps;
  DeviceGuard dg(E.device);
  const int n = g.n, H = n / 2;
  const size_t nn = (size_t)n * n;
  const size_t hn = (size_t)H * n;  // complex values of one instance's mixed-domain field
  auto& A = E.adj;
  cudaStream_t st = E.stream;
  const int nck = (steps + K - 1) / K;
  if (!A.ready) {
    A.ks64 = find_kernels(n, ESC_FP64);
    if (!A.ks64 || !A.ks64->adj_col1) return E.fail(ESC_EINVAL, "no adjoint kernels for this size");
    CK(A.ks64->prepare());
    CK(A.ks64->prepare_adj());
    if (A.ks64->warp_rows) CK(A.ks64->prepare_warp());
    A.mixed = g.ks->wr_bytes == 4 && A.ks64->adj_col1_m != nullptr;
    A.pstride = (size_t)std::max(A.ks64->part_len, g.ks->part_len) + 8 * 4096;
    TRY(E.alloc(&A.phi64, cnt * nn * 8, "adjoint phi"));
    TRY(E.alloc(&A.target, cnt * nn * 8, "adjoint target"));
    TRY(E.alloc(&A.cout, cnt * nn * 8, "adjoint output"));
    TRY(E.alloc(&A.F64, cnt * hn * 16, "adjoint F"));
    TRY(E.alloc(&A.Lam, cnt * hn * 16, "adjoint state"));
    TRY(E.alloc(&A.Xg, cnt * hn * 16, "adjoint Xg"));
    TRY(E.alloc(&A.G64, cnt * hn * 32, "adjoint G"));
    TRY(E.alloc(&A.tw64, (size_t)n * 16, "adjoint twiddles"));
    TRY(E.alloc(&A.part, cnt * A.pstride * 8, "adjoint partials"));
    TRY(E.alloc(&A.scal, cnt * 8 * 8, "adjoint scalars"));
    TRY(E.alloc(&A.hist, cnt * 6 * 8, "adjoint history row"));
    TRY(E.alloc(&A.acc, cnt * 8 * 8, "adjoint accumulators"));
    TRY(E.alloc(&A.cnt, cnt * 4 * 4, "adjoint counters"));
    TRY(E.alloc(&A.acnt, cnt * 4 * 4, "adjoint counters"));
    TRY(E.alloc(&A.status, cnt * 4, "adjoint status"));
    TRY(E.alloc(&A.zero, 4, "zero"));
    TRY(E.alloc(&A.bad, cnt * 8, "adjoint bad step"));
    TRY(E.alloc(&A.d_seed, cnt * sizeof(esc::InstDev), "adjoint descriptor"));
    TRY(E.alloc(&A.d_bwd, cnt * sizeof(esc::InstDev), "adjoint descriptor"));
    TRY(E.alloc(&A.d_out, cnt * sizeof(esc::InstDev), "adjoint descriptor"));
    // FP64 particle fields and twiddles
    if (g.ks->wr_bytes == 8) {
      CK(cudaMemcpy(A.phi64, g.phi, cnt * nn * 8, cudaMemcpyDeviceToDevice));
    } else {
      std::vector<float> pf(cnt * nn);
      std::vector<double> pd(cnt * nn);
      CK(cudaMemcpy(pf.data(), g.phi, cnt * nn * 4, cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < cnt * nn; ++k) pd[k] = (double)pf[k];
      CK(cudaMemcpy(A.phi64, pd.data(), cnt * nn * 8, cudaMemcpyHostToDevice));
    }
    if (g.ks->sr_bytes == 8) CK(cudaMemcpy(A.tw64, g.tw_s, (size_t)n * 16, cudaMemcpyDeviceToDevice));
    A.ks64->fill_tables(A.tw64, A.tw64, st);
    if (A.mixed) {
      TRY(E.alloc(&A.Gw, cnt * hn * 16, "adjoint G (FP32)"));
      TRY(E.alloc(&A.Xw, cnt * hn * 8, "adjoint Xg (FP32)"));
      TRY(E.alloc(&A.d_bwd_m, cnt * sizeof(esc::InstDev), "adjoint descriptor"));
      A.ks64->fill_adj32(g.tw_w, st);
      if (g.ks->warp_rows) CK(g.ks->prepare_warp());
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    CK(cudaMemset(A.zero, 0, 4));
    A.ready = true;
  }
  if (nck > A.ckpt_cap) {
    TRY(E.alloc(&A.ckpt, (size_t)nck * cnt * hn * 16, "adjoint checkpoints"));
    A.ckpt_cap = nck;
  }
  if (K + 1 > A.seg_cap) {
    // the cached graphs of kinds 1 and 2 address the old segment buffers and descriptors
    for (auto it = A.graphs.begin(); it != A.graphs.end();) {
      if (it->first.first >= 2) {
        cudaGraphExecDestroy(it->second);
        it = A.graphs.erase(it);
      } else {
        ++it;
      }
    }
    TRY(E.alloc(&A.seg_buf[0], (size_t)(K + 1) * cnt * hn * 16, "adjoint segment"));
    TRY(E.alloc(&A.seg_buf[1], (size_t)(K + 1) * cnt * hn * 16, "adjoint segment"));
    TRY(E.alloc(&A.d_adj, (size_t)2 * K * cnt * sizeof(esc::AdjDev), "adjoint step descriptors"));
    A.seg_cap = K + 1;
  }
  if (!A.sweep) {
    CK(cudaStreamCreateWithFlags(&A.sweep, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      CK(cudaEventCreateWithFlags(&A.recomputed[b], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&A.swept[b], cudaEventDisableTiming));
    }
  }
  const size_t sbytes = (size_t)cnt * hn * 16;  // the whole group's state
  double2* S = static_cast<double2*>(g.S);
  // ---- forward pass with checkpoints ----
  for (int s = 0; s < cnt; ++s) {
    esc::InstDev& d = g.h_inst[s];
    d.dt = dt;
    d.hist = nullptr;
    d.hist_ld = 1;
    d.cio = g.cio + s * nn;
    CK(cudaMemcpyAsync(g.cio + s * nn, c0[g.members[s]], nn * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(A.target + s * nn, c_target[g.members[s]], nn * 8, cudaMemcpyHostToDevice, st));
  }
  CK(cudaMemcpyAsync(g.d_inst, g.h_inst.data(), cnt * sizeof(esc::InstDev), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(g.status, 0, cnt * sizeof(int), st));
  CK(cudaMemsetAsync(g.cnt, 0, cnt * 4 * sizeof(unsigned), st));
  CK(cudaMemsetAsync(E.base, 0, sizeof(int), st));
  g.ks->init(g.d_inst, cnt, st);
  for (int c = 0; c < nck; ++c) {
    const int len = std::min(steps, (c + 1) * K) - c * K;
    CK(cudaMemcpyAsync(A.ckpt + (size_t)c * cnt * hn, S, sbytes, cudaMemcpyDeviceToDevice, st));
    cudaGraphExec_t gx = nullptr;
    TRY(adjoint_graph(E, 0, 0, len, &gx, [&](cudaStream_t cs) {
      for (int j = 0; j < len; ++j) launch_step(E, 0, cs);
    }));
    CK(cudaGraphLaunch(gx, st));
  }
  CK(cudaGetLastError());
  // ---- seed: energy, mu and lam_T at the final fields ----
  const esc::KernelSet* k64 = A.ks64;
  std::vector<esc::InstDev> sd((size_t)cnt), bd((size_t)cnt), od((size_t)cnt), bm((size_t)cnt);
  std::vector<esc::AdjDev> ad((size_t)cnt);
  for (int s = 0; s < cnt; ++s) {
    esc::InstDev& q = sd[s];
    memset(&q, 0, sizeof q);
    q.n = n;
    q.hist_ld = 1;
    q.dx = g.h_inst[s].dx;
    q.dt = dt;
    q.p = g.h_inst[s].p;
    q.S = S + s * hn;
    q.F = A.F64 + s * hn;
    q.G = A.G64 + s * hn;
    q.phi = A.phi64 + s * nn;
    q.hist = A.hist + 6 * s;
    q.part = A.part + s * A.pstride;
    q.cnt = A.cnt + 4 * s;
    q.scal = A.scal + 8 * s;
    q.status = A.status + s;
    q.bad_step = A.bad + s;
    q.tw_s = A.tw64;
    q.tw_w = A.tw64;
    q.cio = A.cout + s * nn;
    bd[s] = q;
    bd[s].hist = nullptr;
    od[s] = q;
    od[s].S = A.Lam + s * hn;
    od[s].hist = nullptr;
    // the mixed forward row B kernel on the FP32 pair array and the FP32 particle field
    bm[s] = bd[s];
    if (A.mixed) {
      bm[s].G = A.Gw + s * hn;
      bm[s].phi = static_cast<const float*>(g.phi) + s * nn;
      bm[s].tw_s = g.tw_s;
      bm[s].tw_w = g.tw_w;
    }
    esc::AdjDev& a = ad[s];
    memset(&a, 0, sizeof a);
    a.n = n;
    a.dx = q.dx;
    a.dt = dt;
    a.lamF = lamF;
    a.p = q.p;
    a.S0 = S + s * hn;
    a.S1 = S + s * hn;
    a.Lam = A.Lam + s * hn;
    a.Xg = A.Xg + s * hn;
    a.F = A.F64 + s * hn;
    a.G = A.G64 + s * hn;
    a.phi = A.phi64 + s * nn;
    a.target = A.target + s * nn;
    a.tw = A.tw64;
    a.part = A.part + s * A.pstride;
    a.cnt = A.acnt + 4 * s;
    a.acc = A.acc + 8 * s;
    if (A.mixed) {
      a.Gw = A.Gw + s * hn;
      a.Xw = A.Xw + s * hn;
      a.phiw = static_cast<const float*>(g.phi) + s * nn;
    }
  }
  CK(cudaMemcpyAsync(A.d_seed, sd.data(), cnt * sizeof(esc::InstDev), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(A.d_bwd, bd.data(), cnt * sizeof(esc::InstDev), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(A.d_out, od.data(), cnt * sizeof(esc::InstDev), cudaMemcpyHostToDevice, st));
  if (A.mixed)
    CK(cudaMemcpyAsync(A.d_bwd_m, bm.data(), cnt * sizeof(esc::InstDev), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(A.cnt, 0, cnt * 16, st));
  CK(cudaMemsetAsync(A.acnt, 0, cnt * 16, st));
  CK(cudaMemsetAsync(A.status, 0, cnt * 4, st));
  CK(cudaMemsetAsync(A.acc, 0, cnt * 64, st));
  k64->row_a(A.d_seed, cnt, A.zero, 0, st);
  k64->col_a(A.d_seed, cnt, A.zero, 0, st);
  CK(cudaMemcpyAsync(A.d_adj, ad.data(), cnt * sizeof(esc::AdjDev), cudaMemcpyHostToDevice, st));
  k64->adj_mu_col(A.d_adj, cnt, st);
  k64->adj_seed_row(A.d_adj, cnt, st);
  std::vector<double> hist_rows((size_t)cnt * 6), scal((size_t)cnt * 8);
  CK(cudaMemcpyAsync(hist_rows.data(), A.hist, cnt * 6 * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(scal.data(), A.scal, cnt * 8 * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaGetLastError());
  // ---- backward over segments ----
  // Segment buffers alternate: while the sweep stream runs the adjoint over
  // segment k (reading its buffer), the context stream recomputes segment k-1
  // into the other buffer.  The two touch disjoint memory: the recompute uses
  // the forward state and scratch, the sweep the adjoint's own buffers.
  // Step j of buffer b, instance s: descriptor (b*K + j)*cnt + s, states at
  // seg_buf[b] + (j*cnt + s)*hn and (j+1).
  std::vector<esc::AdjDev> steps_desc((size_t)2 * K * cnt);
  for (int b = 0; b < 2; ++b)
    for (int j = 0; j < K; ++j)
      for (int s = 0; s < cnt; ++s) {
        esc::AdjDev& q = steps_desc[((size_t)b * K + j) * cnt + s];
        q = ad[s];
        q.S0 = A.seg_buf[b] + ((size_t)j * cnt + s) * hn;
        q.S1 = A.seg_buf[b] + ((size_t)(j + 1) * cnt + s) * hn;
      }
  CK(cudaMemcpyAsync(A.d_adj, steps_desc.data(), steps_desc.size() * sizeof(esc::AdjDev), cudaMemcpyHostToDevice,
                     st));
  auto seg_len = [&](int seg) { return std::min(steps, (seg + 1) * K) - seg * K; };
  auto recompute = [&](int seg, int b) -> esc_status {
    const int len = seg_len(seg);
    const double2* ck = A.ckpt + (size_t)seg * cnt * hn;
    CK(cudaStreamWaitEvent(st, A.swept[b], 0));  // the sweep that last read this buffer is done
    CK(cudaMemcpyAsync(A.seg_buf[b], ck, sbytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(S, ck, sbytes, cudaMemcpyDeviceToDevice, st));
    cudaGraphExec_t gx = nullptr;
    TRY(adjoint_graph(E, 1, b, len, &gx, [&](cudaStream_t cs) {
      for (int j = 1; j <= len; ++j) {
        launch_step(E, 0, cs);
        cudaMemcpyAsync(A.seg_buf[b] + (size_t)j * cnt * hn, S, sbytes, cudaMemcpyDeviceToDevice, cs);
      }
    }));
    CK(cudaGraphLaunch(gx, st));
    CK(cudaEventRecord(A.recomputed[b], st));
    return ESC_OK;
  };
  int b = 0;
  TRY(recompute(nck - 1, b));
  for (int seg = nck - 1; seg >= 0; --seg) {
    const int len = seg_len(seg);
    CK(cudaStreamWaitEvent(A.sweep, A.recomputed[b], 0));
    cudaGraphExec_t gx = nullptr;
    esc::AdjDev* dd = A.d_adj + (size_t)b * K * cnt;
    TRY(adjoint_graph(E, 2, b, len, &gx, [&](cudaStream_t cs) {
      for (int j = len - 1; j >= 0; --j) {
        if (A.mixed) {
          k64->adj_col1_m(dd + (size_t)j * cnt, cnt, cs);
          if (g.ks->warp_rows)
            g.ks->row_b_w(A.d_bwd_m, cnt, A.zero, 0, cs);  // M grad a: the mixed forward row B
          else
            g.ks->row_b(A.d_bwd_m, cnt, A.zero, 0, cs);
          k64->adj_col2_m(dd + (size_t)j * cnt, cnt, cs);
          k64->adj_row2_m(dd + (size_t)j * cnt, cnt, cs);
          continue;
        }
        k64->adj_col1(dd + (size_t)j * cnt, cnt, cs);
        if (k64->warp_rows)
          k64->row_b_w(A.d_bwd, cnt, A.zero, 0, cs);  // M grad a: the forward row B, warp-independent form
        else
          k64->row_b(A.d_bwd, cnt, A.zero, 0, cs);
        k64->adj_col2(dd + (size_t)j * cnt, cnt, cs);
        k64->adj_row2(dd + (size_t)j * cnt, cnt, cs);
      }
    }));
    CK(cudaGraphLaunch(gx, A.sweep));
    CK(cudaEventRecord(A.swept[b], A.sweep));
    if (seg > 0) TRY(recompute(seg - 1, 1 - b));
    if (seg == 0) CK(cudaStreamWaitEvent(st, A.swept[b], 0));
    b = 1 - b;
  }
  CK(cudaGetLastError());
  k64->fin(A.d_out, cnt, st);
  std::vector<double> acc((size_t)cnt * 8);
  CK(cudaMemcpyAsync(acc.data(), A.acc, cnt * 64, cudaMemcpyDeviceToHost, st));
  for (int s = 0; s < cnt; ++s)
    if (dL_dc0 && dL_dc0[g.members[s]])
      CK(cudaMemcpyAsync(dL_dc0[g.members[s]], A.cout + s * nn, nn * 8, cudaMemcpyDeviceToHost, st));
  std::vector<int> fstatus((size_t)cnt);
  CK(cudaMemcpyAsync(fstatus.data(), g.status, cnt * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int s = 0; s < cnt; ++s)
    if (fstatus[s]) return E.fail(ESC_ENONFINITE, "Non-finite composition during the adjoint's forward pass");
  for (int s = 0; s < cnt; ++s) {
    const int i = g.members[s];
    const double dx2 = sd[s].dx * sd[s].dx;
    const double E_T = hist_rows[6 * s + 2];
    const double scal0 = scal[8 * s];
    const double* a = &acc[8 * s];
    const esc::ModelParams& p = sd[s].p;
    if (dL_dparams) {
      dL_dparams[4 * i + 0] = a[0] + lamF * a[5] * dx2;
      dL_dparams[4 * i + 1] = a[1] + lamF * (-p.P * a[6] * dx2);
      dL_dparams[4 * i + 2] = a[2] + lamF * ((E_T - scal0 * dx2) / p.kappa);
      dL_dparams[4 * i + 3] = a[3];
    }
    if (Lout) Lout[i] = a[4] + lamF * E_T;
  }
  return ESC_OK;
}

// Lets other translation units of the library report through esc_last_error(NULL).
void esc_set_thread_error(const char* msg) { tl_err = msg ? msg : ""; }

struct esc_ctx {
  Engine e;
};
struct esc_batch {
  Engine e;
};

extern "C" {

void esc_default_params(esc_params* p) {
  if (!p) return;
  p->A = 2.0;
  p->B = 4.0;
  p->chi = 0.5;
  p->P = 5.0;
  p->ca = 0.5;
  p->cb = 0.0;
  p->cc = 1.0;
  p->kappa = 2.0;
  p->mobility = 1.0;
  p->Q = 0.5;
}

int esc_supported_size(int n) { return find_kernels(n, ESC_FP64) != nullptr ? 1 : 0; }

const char* esc_version(void) { return "esc-b200 0.1.0 (sm_100a)"; }

esc_status esc_create(esc_ctx** out, int n, double dx, const double* phi, const esc_params* p, esc_precision prec) {
  if (!out) {
    tl_err = "null output pointer";
    return ESC_EINVAL;
  }
  *out = nullptr;
  esc_ctx* c = new (std::nothrow) esc_ctx();
  if (!c) {
    tl_err = "host allocation failed";
    return ESC_ENOMEM;
  }
  const double* phis[1] = {phi};
  esc_status s;
  {
    std::lock_guard<std::mutex> lock(creation_mutex());
    s = engine_create(c->e, 1, &n, &dx, phis, p, (int)prec);
    if (s == ESC_OK) s = autotune(c->e);
    if (s == ESC_OK) s = enable_cluster(c->e);
    if (s == ESC_OK) s = choose_cluster(c->e);
    if (s == ESC_OK) s = ensure_graph(c->e);
  }
  if (s != ESC_OK) {
    tl_err = c->e.err;
    c->e.release();
    delete c;
    return s;
  }
  *out = c;
  return ESC_OK;
}

esc_status esc_run(esc_ctx* ctx, double* c, int steps, double dt, double* history, int64_t* bad_step) {
  if (!ctx) {
    tl_err = "null context";
    return ESC_EINVAL;
  }
  double* cs[1] = {c};
  double* hs[1] = {history};
  int64_t b = -1;
  const esc_status s = engine_run(ctx->e, cs, false, steps, dt, hs, nullptr, &b, true);
  if (bad_step) *bad_step = b;
  return s;
}

esc_status esc_run_device(esc_ctx* ctx, double* c, int steps, double dt, double* history, int64_t* bad_step) {
  if (!ctx) {
    tl_err = "null context";
    return ESC_EINVAL;
  }
  double* cs[1] = {c};
  int64_t b = -1;
  const esc_status s = engine_run_device(ctx->e, cs, steps, dt, history, &b);
  if (bad_step) *bad_step = b;
  return s;
}

esc_status esc_run_device_async(esc_ctx* ctx, double* c, int steps, double dt, double* history) {
  if (!ctx) {
    tl_err = "null context";
    return ESC_EINVAL;
  }
  double* cs[1] = {c};
  return engine_enqueue_device(ctx->e, cs, steps, dt, history);
}

esc_status esc_wait(esc_ctx* ctx, int64_t* bad_step) {
  if (!ctx) {
    tl_err = "null context";
    return ESC_EINVAL;
  }
  int64_t b = -1;
  const esc_status s = engine_wait(ctx->e, &b);
  if (bad_step) *bad_step = b;
  return s;
}

int esc_uses_cluster(const esc_ctx* ctx) { return ctx && ctx->e.cluster ? 1 : 0; }

esc_status esc_set_stream(esc_ctx* ctx, void* stream) {
  if (!ctx) return ESC_EINVAL;
  ctx->e.stream = stream ? static_cast<cudaStream_t>(stream) : ctx->e.own;
  return ESC_OK;
}

const char* esc_last_error(const esc_ctx* ctx) { return ctx ? ctx->e.err.c_str() : tl_err.c_str(); }

void esc_destroy(esc_ctx* ctx) {
  if (!ctx) return;
  {
    DeviceGuard dg(ctx->e.device);
    if (ctx->e.pending) cudaStreamSynchronize(ctx->e.stream);
    ctx->e.release();
  }
  delete ctx;
}

esc_status esc_batch_create(esc_batch** out, int count, const int* n, const double* dx, const double* const* phi,
                            const esc_params* p, esc_precision prec) {
  if (!out) {
    tl_err = "null output pointer";
    return ESC_EINVAL;
  }
  *out = nullptr;
  esc_batch* b = new (std::nothrow) esc_batch();
  if (!b) {
    tl_err = "host allocation failed";
    return ESC_ENOMEM;
  }
  esc_status s;
  {
    std::lock_guard<std::mutex> lock(creation_mutex());
    s = engine_create(b->e, count, n, dx, phi, p, (int)prec);
    if (s == ESC_OK) s = autotune(b->e);
    if (s == ESC_OK) s = ensure_graph(b->e);
  }
  if (s != ESC_OK) {
    tl_err = b->e.err;
    b->e.release();
    delete b;
    return s;
  }
  *out = b;
  return ESC_OK;
}

esc_status esc_batch_run(esc_batch* b, double* const* c, int steps, double dt, double* const* history,
                         int64_t* bad_steps) {
  if (!b) {
    tl_err = "null batch";
    return ESC_EINVAL;
  }
  return engine_run(b->e, c, false, steps, dt, history, nullptr, bad_steps, true);
}

esc_status esc_batch_run_device(esc_batch* b, double* const* c, int steps, double dt, double* history,
                                int64_t* bad_steps) {
  if (!b) {
    tl_err = "null batch";
    return ESC_EINVAL;
  }
  return engine_run_device(b->e, c, steps, dt, history, bad_steps);
}

esc_status esc_batch_run_device_async(esc_batch* b, double* const* c, int steps, double dt, double* history) {
  if (!b) {
    tl_err = "null batch";
    return ESC_EINVAL;
  }
  return engine_enqueue_device(b->e, c, steps, dt, history);
}

esc_status esc_batch_wait(esc_batch* b, int64_t* bad_steps) {
  if (!b) {
    tl_err = "null batch";
    return ESC_EINVAL;
  }
  return engine_wait(b->e, bad_steps);
}

esc_status esc_batch_profile_phases(esc_batch* b, int steps, int* n_groups, int* group_n, int* group_count,
                                    double* ms) {
  if (!b || steps < 1 || !n_groups) {
    tl_err = "bad argument";
    return ESC_EINVAL;
  }
  Engine& E = b->e;
  DeviceGuard dg(E.device);
  const int ng = (int)E.groups.size();
  *n_groups = ng;
  if (!group_n || !group_count || !ms) return ESC_OK;
  cudaStream_t st = E.stream;
  // write history row 0 into the library's own buffer, never into caller memory
  const size_t need = 6 * (size_t)E.count;
  if (need > E.hist_cap) {
    for (auto it = E.allocs.begin(); it != E.allocs.end(); ++it)
      if (*it == E.hist) {
        E.allocs.erase(it);
        break;
      }
    if (E.hist) cudaFree(E.hist);
    E.hist = nullptr;
    E.hist_cap = 0;
    TRY(E.alloc(&E.hist, need * sizeof(double), "history"));
    E.hist_cap = need;
  }
  for (Group& g : E.groups) {
    for (size_t s = 0; s < g.members.size(); ++s) {
      g.h_inst[s].hist = E.hist + (size_t)g.members[s] * 6;
      g.h_inst[s].hist_ld = 1;
    }
    CK(cudaMemcpyAsync(g.d_inst, g.h_inst.data(), g.h_inst.size() * sizeof(esc::InstDev),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(g.status, 0, g.members.size() * sizeof(int), st));
  }
  std::vector<cudaEvent_t> ev(4 * ng + 1);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  std::vector<double> acc(4 * (size_t)ng, 0.0);
  for (int s = 0; s < steps; ++s) {
    CK(cudaMemsetAsync(E.base, 0, sizeof(int), st));
    for (int gi = 0; gi < ng; ++gi) {
      Group& g = E.groups[gi];
      const int c = (int)g.members.size();
      (void)c;
      CK(cudaEventRecord(ev[4 * gi], st));
      phase_row_a(g, E.base, 0, st);
      CK(cudaEventRecord(ev[4 * gi + 1], st));
      phase_col_a(g, E.base, 0, st);
      CK(cudaEventRecord(ev[4 * gi + 2], st));
      phase_row_b(g, E.base, 0, st);
      CK(cudaEventRecord(ev[4 * gi + 3], st));
      phase_col_b(g, st);
      CK(cudaEventRecord(gi + 1 < ng ? ev[4 * (gi + 1)] : ev[4 * ng], st));
    }
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev[4 * ng]));
    for (int k = 0; k < 4 * ng; ++k) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      acc[k] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int gi = 0; gi < ng; ++gi) {
    group_n[gi] = E.groups[gi].n;
    group_count[gi] = (int)E.groups[gi].members.size();
    for (int k = 0; k < 4; ++k) ms[4 * gi + k] = acc[4 * gi + k] / steps;
  }
  return ESC_OK;
}

esc_status esc_adjoint(esc_ctx* ctx, const double* c0, int steps, double dt, const double* c_target,
                       double lambda_F, int ckpt_every, double* dL_dc0, double* dL_dparams, double* L) {
  if (!ctx) {
    tl_err = "null context";
    return ESC_EINVAL;
  }
  const double* c0s[1] = {c0};
  const double* tgs[1] = {c_target};
  double* outs[1] = {dL_dc0};
  return engine_adjoint(ctx->e, c0s, steps, dt, tgs, lambda_F, ckpt_every, outs, dL_dparams, L);
}

esc_status esc_batch_adjoint(esc_batch* b, const double* const* c0, int steps, double dt,
                             const double* const* c_target, double lambda_F, int ckpt_every, double* const* dL_dc0,
                             double* dL_dparams, double* L) {
  if (!b) {
    tl_err = "null batch";
    return ESC_EINVAL;
  }
  return engine_adjoint(b->e, c0, steps, dt, c_target, lambda_F, ckpt_every, dL_dc0, dL_dparams, L);
}

int esc_batch_describe(const esc_batch* b, char* buf, int buflen) {
  if (!b) return -1;
  std::string out = "[";
  static const char* rows[3] = {"block", "tma-pipeline", "warp"};
  static const char* cols[3] = {"block", "tma-pipeline", "block-alt-plan"};
  for (size_t i = 0; i < b->e.groups.size(); ++i) {
    const Group& g = b->e.groups[i];
    char tmp[512];
    snprintf(tmp, sizeof tmp,
             "%s{\"n\": %d, \"instances\": %zu, \"rows\": \"%s\", \"cols\": \"%s\", \"row_ms\": [%.4f, %.4f, %.4f], "
             "\"col_ms\": [%.4f, %.4f, %.4f], \"E\": %d, \"E_alt\": %d}",
             i ? ", " : "", g.n, g.members.size(), g.row_family >= 0 ? rows[g.row_family] : "?",
             g.col_family >= 0 ? cols[g.col_family] : "?", g.row_ms[0], g.row_ms[1], g.row_ms[2], g.col_ms[0],
             g.col_ms[1], g.col_ms[2], g.ks->E, g.ks->E_alt);
    out += tmp;
  }
  out += "]";
  if (buf && buflen > 0) {
    strncpy(buf, out.c_str(), (size_t)buflen - 1);
    buf[buflen - 1] = 0;
  }
  return (int)out.size() + 1;
}

esc_status esc_batch_set_stream(esc_batch* b, void* stream) {
  if (!b) return ESC_EINVAL;
  b->e.stream = stream ? static_cast<cudaStream_t>(stream) : b->e.own;
  return ESC_OK;
}

const char* esc_batch_last_error(const esc_batch* b) { return b ? b->e.err.c_str() : tl_err.c_str(); }

void esc_batch_destroy(esc_batch* b) {
  if (!b) return;
  {
    DeviceGuard dg(b->e.device);
    if (b->e.pending) cudaStreamSynchronize(b->e.stream);
    b->e.release();
  }
  delete b;
}

}  // extern "C"
