// esc_run_noalloc: a single-particle FP64 run that allocates no memory.
//
// Who needs it: callers that are not allowed to call cudaMalloc -- for example
// a host application whose device memory is fully owned by another allocator
// (a framework's caching pool, a fixed real-time budget), or a latency-bound
// loop that cannot accept the device-wide synchronisation cudaMalloc/cudaFree
// may cause.  They pass device buffers for the inputs and outputs; every
// intermediate of the step (the mixed-domain state, the f' and flux
// transforms, twiddles, partial sums, counters and the instance descriptor)
// lives in one file-scope __device__ array of fixed size, g_noalloc_scratch.
//
// Limits and contract:
//   * grid sizes up to kNoAllocMaxN = 256 (FP64 only); larger sizes are
//     rejected with ESC_EINVAL before any work is queued;
//   * the array is shared by every call in the process on that device and keeps
//     the contents of the last call: the counters, status words and step
//     counter are cleared at the start of each call, and everything else is
//     fully rewritten before it is read;
//   * calls that overlap on the GPU (different host threads or streams at the
//     same time) race on the array and must be serialised by the caller;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current);
//   * no call may run inside a stream capture: each call copies its small
//     descriptor from host memory and waits for its stream, neither of which a
//     capture allows, so a call on a capturing stream returns ESC_EINVAL
//     without touching the stream;
//   * the pass-major twiddle tables of a grid size are process-wide __device__
//     arrays; the first call for a size on a device fills them, later calls
//     reuse them.  Creating a context of the same size refills them with
//     identical values, so a kernel reading them meanwhile sees the same bits.
// The array is part of the library image: every GPU that loads libesc.so
// holds it (about 2.1 MiB) until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "esc.h"
#include "esc_dispatch.cuh"

#define ESC_DECL(n) const esc::KernelSet* esc_kernels_##n(int prec);
ESC_SIZES(ESC_DECL)
#undef ESC_DECL

// Defined in esc_api.cu: records the message returned by esc_last_error(NULL).
void esc_set_thread_error(const char* msg);

namespace {

constexpr int kNoAllocMaxN = 256;
constexpr size_t kNN = (size_t)kNoAllocMaxN * kNoAllocMaxN;
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
// byte offsets inside the scratch array (FP64: complex = 16 B)
constexpr size_t kOffS = 0;
constexpr size_t kOffF = kOffS + align256(kNN * 8);        // H*n complex doubles = 8 n^2 bytes
constexpr size_t kOffG = kOffF + align256(kNN * 8);
constexpr size_t kOffTw = kOffG + align256(kNN * 16);      // pair array: 16 n^2 bytes
constexpr size_t kOffPart = kOffTw + align256((size_t)kNoAllocMaxN * 16);
constexpr size_t kPartDoubles = 5 * 256 + 256 + 256;       // >= part_len for every n <= 256
constexpr size_t kOffScal = kOffPart + align256(kPartDoubles * 8);
constexpr size_t kOffCnt = kOffScal + 256;
constexpr size_t kOffStatus = kOffCnt + 256;
constexpr size_t kOffBad = kOffStatus + 256;
constexpr size_t kOffBase = kOffBad + 256;
constexpr size_t kOffInst = kOffBase + 256;
constexpr size_t kScratchBytes = kOffInst + align256(sizeof(esc::InstDev));

const esc::KernelSet* lookup(int n) {
  switch (n) {
#define ESC_CASE(nn) \
  case nn:           \
    return esc_kernels_##nn(esc::kFP64);
    ESC_SIZES(ESC_CASE)
#undef ESC_CASE
    default:
      return nullptr;
  }
}

}  // namespace

// The scratch of esc_run_noalloc (see the file comment).  In host code this
// name is only a handle: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};
bool g_tables_filled[kMaxDevices][kNoAllocMaxN + 1] = {};  // pass-major tables of size n filled on a device

esc_status fail(esc_status s, const char* what, cudaError_t e = cudaSuccess) {
  char msg[256];
  if (e != cudaSuccess)
    snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
  else
    snprintf(msg, sizeof msg, "%s", what);
  esc_set_thread_error(msg);
  return s;
}

}  // namespace

extern "C" esc_status esc_run_noalloc(int n, double dx, const double* phi, const esc_params* p, double* c,
                                      int steps, double dt, double* history, int64_t* bad_step, void* stream) {
  if (bad_step) *bad_step = -1;
  if (n > kNoAllocMaxN)
    return fail(ESC_EINVAL, "esc_run_noalloc: grid size above the fixed scratch limit of 256");
  const esc::KernelSet* ks = lookup(n);
  if (!ks) return fail(ESC_EINVAL, "esc_run_noalloc: unsupported grid size (needs a tuned size: 8, 12, 16, 24, 32, 48, 64, 96, 128, 192 or 256)");
  if (!phi || !c || !p) return fail(ESC_EINVAL, "esc_run_noalloc: null argument");
  if (!(dx > 0.0) || !std::isfinite(dx) || !std::isfinite(dt) || steps < 0)
    return fail(ESC_EINVAL, "esc_run_noalloc: bad spacing, dt or step count");
  if ((size_t)ks->part_len > kPartDoubles) return fail(ESC_EINVAL, "esc_run_noalloc: partial-sum area too small");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ESC_ECUDA, "cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return fail(ESC_EINVAL, "esc_run_noalloc: device index out of range");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) return fail(ESC_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch)", e);
      g_scratch_ptr[dev] = static_cast<unsigned char*>(ptr);
    }
    base = g_scratch_ptr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess) return fail(ESC_ECUDA, "cudaStreamIsCapturing", e);
    if (cs != cudaStreamCaptureStatusNone)
      return fail(ESC_EINVAL, "esc_run_noalloc: cannot be called while the stream is being captured");
  }
  if ((e = ks->prepare()) != cudaSuccess) return fail(ESC_ECUDA, "kernel attributes", e);

  // twiddles e^{-2 pi i j/n} in long double, staged on the host stack
  double tw[2 * kNoAllocMaxN];
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int j = 0; j < n; ++j) {
    const long double a = two_pi * (long double)j / (long double)n;
    tw[2 * j] = (double)cosl(a);
    tw[2 * j + 1] = (double)(-sinl(a));
  }
  esc::InstDev d;
  memset(&d, 0, sizeof d);
  d.n = n;
  d.hist_ld = steps + 1;
  d.dx = dx;
  d.dt = dt;
  d.p = esc::ModelParams{p->A, p->B, p->chi, p->P, p->ca, p->cb, p->cc, p->kappa, p->mobility, p->Q};
  d.S = base + kOffS;
  d.F = base + kOffF;
  d.G = base + kOffG;
  d.phi = phi;
  d.hist = history;
  d.part = reinterpret_cast<double*>(base + kOffPart);
  d.cnt = reinterpret_cast<unsigned*>(base + kOffCnt);
  d.scal = reinterpret_cast<double*>(base + kOffScal);
  d.status = reinterpret_cast<int*>(base + kOffStatus);
  d.bad_step = reinterpret_cast<long long*>(base + kOffBad);
  d.tw_s = base + kOffTw;
  d.tw_w = base + kOffTw;
  d.cio = c;
  int* step_base = reinterpret_cast<int*>(base + kOffBase);
  const esc::InstDev* dinst = reinterpret_cast<const esc::InstDev*>(base + kOffInst);

#define NA_CK(call)                                      \
  do {                                                   \
    const cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return fail(ESC_ECUDA, #call, e_); \
  } while (0)
  NA_CK(cudaMemcpyAsync(base + kOffTw, tw, (size_t)n * 16, cudaMemcpyHostToDevice, st));
  {
    // the pass-major tables are fixed __device__ arrays too: filled by the first call of this size
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_tables_filled[dev][n]) {
      ks->fill_tables(base + kOffTw, base + kOffTw, st);
      NA_CK(cudaGetLastError());
      g_tables_filled[dev][n] = true;
    }
  }
  NA_CK(cudaMemcpyAsync(base + kOffInst, &d, sizeof d, cudaMemcpyHostToDevice, st));
  // state that must start at zero: counters, status, bad step (-1), step counter
  NA_CK(cudaMemsetAsync(base + kOffCnt, 0, 256, st));
  NA_CK(cudaMemsetAsync(base + kOffStatus, 0, 256, st));
  NA_CK(cudaMemsetAsync(base + kOffBad, 0xff, 256, st));
  NA_CK(cudaMemsetAsync(step_base, 0, sizeof(int), st));
  ks->init(dinst, 1, st);
  for (int s = 0; s < steps; ++s) {
    ks->row_a(dinst, 1, step_base, s, st);
    ks->col_a(dinst, 1, step_base, s, st);
    ks->row_b(dinst, 1, step_base, s, st);
    ks->col_b(dinst, 1, st);
  }
  ks->row_a(dinst, 1, step_base, steps, st);
  ks->col_a(dinst, 1, step_base, steps, st);
  ks->row_b(dinst, 1, step_base, steps, st);
  int status = 0;
  long long bad = -1;
  NA_CK(cudaGetLastError());
  NA_CK(cudaMemcpyAsync(&status, base + kOffStatus, sizeof status, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaMemcpyAsync(&bad, base + kOffBad, sizeof bad, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  if (status == esc::kStatusLayout)
    return fail(ESC_ECUDA, "esc_run_noalloc: internal error: a shared-memory stage was misaligned");
  if (status == esc::kStatusTimeout) return fail(ESC_ETIMEOUT, "esc_run_noalloc: a bounded device-side wait gave up");
  if (status) {
    if (bad_step) *bad_step = bad;
    char msg[96];
    snprintf(msg, sizeof msg, "Non-finite composition at step %lld", bad);
    esc_set_thread_error(msg);
    return ESC_ENONFINITE;
  }
  // final field c = inverse x-transform of the state, only when it stayed finite
  ks->fin(dinst, 1, st);
  NA_CK(cudaGetLastError());
  NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
  return ESC_OK;
}
