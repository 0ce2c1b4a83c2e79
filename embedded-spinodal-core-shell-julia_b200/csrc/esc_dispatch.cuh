// Per-size kernel sets: launch wrappers and launch geometry for one grid size n
// and one precision mode.  Each esc_size_<n>.cu instantiates the two modes.
#pragma once
#include "esc_kernels.cuh"

namespace esc {

enum Prec { kFP64 = 0, kMixed = 1 };

struct KernelSet {
  int n, prec, T, E;
  int tiles_pairs, tiles_rows, tiles_cols;
  int part_len;  // partial-sum doubles per instance
  size_t smem;   // dynamic shared memory per block
  size_t sr_bytes, wr_bytes;  // sizeof(real) of the state and work types
  cudaError_t (*prepare)();
  void (*init)(const InstDev*, int, cudaStream_t);
  void (*fin)(const InstDev*, int, cudaStream_t);
  void (*row_a)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*col_a)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*row_b)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*col_b)(const InstDev*, int, cudaStream_t);
};

// FP64 plans keep E <= 16 so that two register arrays of double2 fit.
template <int N>
struct Plan64 {
  using type = typename DefaultPlan<N>::type;
};
#define ESC_PLAN64(n, e, ...) \
  template <>                 \
  struct Plan64<n> { using type = Plan<n, e, Radices<__VA_ARGS__>>; };
ESC_PLAN64(96, 12, 6, 4, 4)
ESC_PLAN64(384, 12, 6, 4, 4, 4)
ESC_PLAN64(768, 12, 12, 4, 4, 4)
ESC_PLAN64(1536, 12, 6, 4, 4, 4, 4)
ESC_PLAN64(3072, 12, 12, 4, 4, 4, 4)
#undef ESC_PLAN64

inline int host_smpad(int p) { return p + (p >> 4); }

template <class P, typename SR, typename WR>
struct KS {
  static constexpr int N = P::N, T = P::T, E = P::E, H = N / 2;
  static constexpr int G = kBlock / T, W = kBlock / T;
  static constexpr int tiles_pairs = (H + G - 1) / G;
  static constexpr int tiles_rows = (N + G - 1) / G;
  static constexpr int tiles_cols = (H + W - 1) / W;
  static_assert(T <= kBlock, "plan needs more threads than a block");
  static size_t smem() {
    const size_t row = (size_t)G * RowLayout<N>::stride;
    const size_t col = (size_t)host_smpad(N * W - 1) + 1;
    const size_t el = row > col ? row : col;
    return el * sizeof(cpx<SR>);
  }
  static cudaError_t prepare() {
    const int bytes = (int)smem();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_init<P, SR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(k_final<P, SR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(k_row_a<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
      return e;
    if ((e = cudaFuncSetAttribute(k_col_a<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
      return e;
    if ((e = cudaFuncSetAttribute(k_row_b<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
      return e;
    if ((e = cudaFuncSetAttribute(k_col_b<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
      return e;
    return cudaSuccess;
  }
  static void init(const InstDev* d, int count, cudaStream_t st) {
    k_init<P, SR><<<dim3(tiles_pairs, count), kBlock, smem(), st>>>(d);
  }
  static void fin(const InstDev* d, int count, cudaStream_t st) {
    k_final<P, SR><<<dim3(tiles_pairs, count), kBlock, smem(), st>>>(d);
  }
  static void row_a(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    k_row_a<P, SR, WR><<<dim3(tiles_pairs, count), kBlock, smem(), st>>>(d, base, s);
  }
  static void col_a(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    k_col_a<P, SR, WR><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(d, base, s);
  }
  static void row_b(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    k_row_b<P, SR, WR><<<dim3(tiles_rows, count), kBlock, smem(), st>>>(d, base, s);
  }
  static void col_b(const InstDev* d, int count, cudaStream_t st) {
    k_col_b<P, SR, WR><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(d);
  }
  static KernelSet make(int prec) {
    KernelSet k;
    k.n = N;
    k.prec = prec;
    k.T = T;
    k.E = E;
    k.tiles_pairs = tiles_pairs;
    k.tiles_rows = tiles_rows;
    k.tiles_cols = tiles_cols;
    k.part_len = 5 * tiles_pairs + tiles_cols + tiles_rows;
    k.smem = smem();
    k.sr_bytes = sizeof(SR);
    k.wr_bytes = sizeof(WR);
    k.prepare = &prepare;
    k.init = &init;
    k.fin = &fin;
    k.row_a = &row_a;
    k.col_a = &col_a;
    k.row_b = &row_b;
    k.col_b = &col_b;
    return k;
  }
};

}  // namespace esc

// Defines esc_kernels_<n>(prec) in the translation unit that uses it.
#define ESC_DEFINE_SIZE(n)                                                                            \
  const esc::KernelSet* esc_kernels_##n(int prec) {                                                   \
    static const esc::KernelSet fp64 = esc::KS<esc::Plan64<n>::type, double, double>::make(esc::kFP64); \
    static const esc::KernelSet mixed =                                                               \
        esc::KS<esc::DefaultPlan<n>::type, double, float>::make(esc::kMixed);                         \
    return prec == esc::kFP64 ? &fp64 : &mixed;                                                       \
  }

#define ESC_SIZES(X) \
  X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024) X(1536) X(2048) X(3072) X(4096)
