// Per-size kernel sets: launch wrappers and launch geometry for one grid size n
// and one precision mode.  Each esc_size_<n>.cu instantiates the two modes.
#pragma once
#include <type_traits>
#include "esc_warp.cuh"
#include "esc_adjoint.cuh"

namespace esc {

enum Prec { kFP64 = 0, kMixed = 1 };

struct KernelSet {
  int n, prec, T, E;
  int tiles_pairs, tiles_rows, tiles_cols;
  int part_len;  // partial-sum doubles per instance
  size_t smem;   // dynamic shared memory per block
  size_t sr_bytes, wr_bytes;  // sizeof(real) of the state and work types
  size_t cplx_per_field;      // complex elements of S (and of F; G holds twice as many) per instance
  bool generic;               // runtime-size kernels (esc_generic.cu): no tuned families, no adjoint
  cudaError_t (*prepare)();
  cudaError_t (*prepare_pipe)();
  // fills the pass-major twiddle tables of every plan the set uses from the
  // plain tables (state and work precision), in stream order
  void (*fill_tables)(const void*, const void*, cudaStream_t);
  void (*init)(const InstDev*, int, cudaStream_t);
  void (*fin)(const InstDev*, int, cudaStream_t);
  void (*row_a)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*col_a)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*row_b)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*col_b)(const InstDev*, int, cudaStream_t);
  // persistent TMA-fed launchers (available when pipe_rows / pipe_cols)
  bool pipe_rows, pipe_cols;
  int W, RB;  // columns per tile and rows per tensor box of the column kernels
  void (*row_a_p)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*row_b_p)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*col_a_p)(const InstDev*, int, const int*, int, cudaStream_t, const ColMaps*);
  void (*col_b_p)(const InstDev*, int, cudaStream_t, const ColMaps*);
  // warp-independent row kernels (groups inside one warp), when warp_rows
  bool warp_rows;
  void (*row_a_w)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*row_b_w)(const InstDev*, int, const int*, int, cudaStream_t);
  cudaError_t (*prepare_warp)();
  // column kernels with the alternative (fewer elements per thread) plan
  void (*col_a_alt)(const InstDev*, int, const int*, int, cudaStream_t);
  void (*col_b_alt)(const InstDev*, int, cudaStream_t);
  int E_alt;
  // adjoint step kernels (FP64 kernel sets only; null in the mixed sets)
  cudaError_t (*prepare_adj)();
  void (*adj_col1)(const AdjDev*, int, cudaStream_t);
  void (*adj_col2)(const AdjDev*, int, cudaStream_t);
  void (*adj_row2)(const AdjDev*, int, cudaStream_t);
  void (*adj_mu_col)(const AdjDev*, int, cudaStream_t);
  void (*adj_seed_row)(const AdjDev*, int, cudaStream_t);
  // mixed-precision adjoint step kernels (FP64 kernel sets; for mixed contexts) and the
  // fill of their FP32 pass-major twiddle tables from the plain FP32 table
  void (*adj_col1_m)(const AdjDev*, int, cudaStream_t);
  void (*adj_col2_m)(const AdjDev*, int, cudaStream_t);
  void (*adj_row2_m)(const AdjDev*, int, cudaStream_t);
  void (*fill_adj32)(const void*, cudaStream_t);
};

// Alternative column plans: fewer elements per thread (more passes, fewer
// registers, more resident warps).  The autotuner times them against the
// default plan.
template <int N>
struct AltPlan {
  using type = typename DefaultPlan<N>::type;
};
#define ESC_ALTPLAN(n, e, ...) \
  template <>                  \
  struct AltPlan<n> { using type = Plan<n, e, Radices<__VA_ARGS__>>; };
ESC_ALTPLAN(128, 8, 4, 4, 8)
ESC_ALTPLAN(256, 8, 4, 8, 8)
ESC_ALTPLAN(384, 12, 4, 4, 4, 6)
ESC_ALTPLAN(768, 12, 4, 4, 4, 12)
ESC_ALTPLAN(512, 16, 16, 16, 2)
ESC_ALTPLAN(1024, 8, 4, 4, 8, 8)
#undef ESC_ALTPLAN

// FP64 plans keep E <= 16 so that two register arrays of double2 fit.
template <int N>
struct Plan64 {
  using type = typename DefaultPlan<N>::type;
};
#define ESC_PLAN64(n, e, ...) \
  template <>                 \
  struct Plan64<n> { using type = Plan<n, e, Radices<__VA_ARGS__>>; };
ESC_PLAN64(96, 12, 4, 4, 6)
ESC_PLAN64(384, 12, 4, 4, 4, 6)
ESC_PLAN64(768, 12, 4, 4, 4, 12)
ESC_PLAN64(1536, 12, 4, 4, 4, 4, 6)
ESC_PLAN64(3072, 12, 4, 4, 4, 4, 12)
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
  // forward column kernels (ColGeomF: col_block<P>() threads, CW columns per block)
  static constexpr int CB = ColGeomF<P, SR, WR>::B, CW = ColGeomF<P, SR, WR>::W;
  static constexpr int ctiles = (H + CW - 1) / CW;
  static size_t col_smem() {
    const size_t col = (size_t)host_smpad(N * CW - 1) + 1;
    const size_t row = (size_t)G * RowLayout<N>::stride;
    return (row > col ? row : col) * sizeof(cpx<SR>);
  }
  static cudaError_t prepare() {
    const int bytes = (int)smem();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_init<P, SR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(k_final<P, SR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    if ((e = cudaFuncSetAttribute(k_row_a<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
      return e;
    if ((e = cudaFuncSetAttribute(k_col_a<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem())))
      return e;
    if ((e = cudaFuncSetAttribute(k_row_b<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
      return e;
    if ((e = cudaFuncSetAttribute(k_col_b<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem())))
      return e;
    return prepare_alt();
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
    k_col_a<P, SR, WR><<<dim3(ctiles, count), CB, col_smem(), st>>>(d, base, s);
  }
  static void row_b(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    k_row_b<P, SR, WR><<<dim3(tiles_rows, count), kBlock, smem(), st>>>(d, base, s);
  }
  static void col_b(const InstDev* d, int count, cudaStream_t st) {
    k_col_b<P, SR, WR><<<dim3(ctiles, count), CB, col_smem(), st>>>(d);
  }
  using PG = PipeGeom<P, SR, WR>;
  // occupancy (blocks per SM) of the persistent kernels and the SM count, set by prepare()
  static int& occ(int i) {
    static int v[4] = {1, 1, 1, 1};
    return v[i];
  }
  static int& sms() {
    static int v = 148;
    return v;
  }
  static int grid_for(int total, int which) {
    const int cap = occ(which) * sms();
    return total < cap ? total : cap;
  }
  static cudaError_t prepare_pipe() {
    cudaError_t e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev))) return e;
    if ((e = cudaDeviceGetAttribute(&sms(), cudaDevAttrMultiProcessorCount, dev))) return e;
    if constexpr (PG::row_ok) {
      const int ba = (int)(2 * PG::stage_ra + kStageAlignSlack), bb = (int)(2 * PG::stage_rb + kStageAlignSlack);
      if ((e = cudaFuncSetAttribute(k_row_a_p<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, ba)))
        return e;
      if ((e = cudaFuncSetAttribute(k_row_b_p<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bb)))
        return e;
      if ((e = cudaFuncSetAttribute(k_row_a_p<P, SR, WR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared)))
        return e;
      if ((e = cudaFuncSetAttribute(k_row_b_p<P, SR, WR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared)))
        return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ(0), k_row_a_p<P, SR, WR>, kBlock, ba))) return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ(2), k_row_b_p<P, SR, WR>, kBlock, bb))) return e;
    }
    if constexpr (PG::col_ok) {
      const int ba = (int)(2 * PG::stage_ca + kStageAlignSlack), bb = (int)(2 * PG::stage_cb + kStageAlignSlack);
      if ((e = cudaFuncSetAttribute(k_col_a_p<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, ba)))
        return e;
      if ((e = cudaFuncSetAttribute(k_col_b_p<P, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bb)))
        return e;
      if ((e = cudaFuncSetAttribute(k_col_a_p<P, SR, WR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared)))
        return e;
      if ((e = cudaFuncSetAttribute(k_col_b_p<P, SR, WR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared)))
        return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ(1), k_col_a_p<P, SR, WR>, PG::CB, ba))) return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ(3), k_col_b_p<P, SR, WR>, PG::CB, bb))) return e;
    }
    for (int i = 0; i < 4; ++i)
      if (occ(i) < 1) occ(i) = 1;
    return cudaSuccess;
  }
  static void row_a_p(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    if constexpr (PG::row_ok) {
      const int total = count * tiles_pairs;
      k_row_a_p<P, SR, WR><<<grid_for(total, 0), kBlock, 2 * PG::stage_ra + kStageAlignSlack, st>>>(d, count, base, s);
    }
  }
  static void row_b_p(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    if constexpr (PG::row_ok) {
      const int total = count * tiles_rows;
      k_row_b_p<P, SR, WR><<<grid_for(total, 2), kBlock, 2 * PG::stage_rb + kStageAlignSlack, st>>>(d, count, base, s);
    }
  }
  static void col_a_p(const InstDev* d, int count, const int* base, int s, cudaStream_t st, const ColMaps* m) {
    if constexpr (PG::col_ok) {
      const int total = count * PG::tiles_cols;
      k_col_a_p<P, SR, WR><<<grid_for(total, 1), PG::CB, 2 * PG::stage_ca + kStageAlignSlack, st>>>(d, count, base, s, *m);
    }
  }
  static void col_b_p(const InstDev* d, int count, cudaStream_t st, const ColMaps* m) {
    if constexpr (PG::col_ok) {
      const int total = count * PG::tiles_cols;
      k_col_b_p<P, SR, WR><<<grid_for(total, 3), PG::CB, 2 * PG::stage_cb + kStageAlignSlack, st>>>(d, count, *m);
    }
  }
  // ---- warp-independent rows (their own plans: groups inside one warp, or 64-thread blocks) ----
  using WPA = typename WarpPlanA<N>::type;  // row A
  using WP = typename WarpPlan<N>::type;    // row B (and the adjoint's row B)
  template <class Q>
  static constexpr bool group_ok() {
    return ((Q::T <= 32) && (32 % Q::T == 0)) || Q::T == 64 || Q::T == 128 || Q::T == 256;
  }
  static constexpr bool warp_ok = group_ok<WPA>() && group_ok<WP>();
  static size_t warp_smem_a() {
    if constexpr (warp_ok) return WarpRowGeom<WPA>::template smem<SR>();
    return 0;
  }
  static size_t warp_smem() {
    if constexpr (warp_ok) return WarpRowGeom<WP>::template smem<SR>();
    return 0;
  }
  static int warp_partials() {  // partial slots of the row kernels (row A holds 5 per slot)
    if constexpr (warp_ok) {
      const int a = 5 * WarpRowGeom<WPA>::tiles_pairs * WarpRowGeom<WPA>::NW;
      const int b = WarpRowGeom<WP>::tiles_rows * WarpRowGeom<WP>::NW;
      return a > b ? a : b;
    }
    return 0;
  }
  static cudaError_t prepare_warp() {
    if constexpr (warp_ok) {
      cudaError_t e;
      const int a = (int)warp_smem_a(), b = (int)warp_smem();
      if ((e = cudaFuncSetAttribute(k_row_a_w<WPA, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, a))) return e;
      if ((e = cudaFuncSetAttribute(k_row_b_w<WP, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
      if constexpr (kPackedRows)
        if ((e = cudaFuncSetAttribute(k_row_b_w2<WP>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
    }
    return cudaSuccess;
  }
  static void row_a_w(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    if constexpr (warp_ok)
      k_row_a_w<WPA, SR, WR><<<dim3(WarpRowGeom<WPA>::tiles_pairs, count), WarpRowGeom<WPA>::BLOCK, warp_smem_a(),
                                st>>>(d, base, s);
  }
  // the mixed precision transforms two rows per group in packed FP32 pairs
  static constexpr bool kPackedRows = std::is_same<SR, double>::value && std::is_same<WR, float>::value;
  static void row_b_w(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    if constexpr (warp_ok) {
      if constexpr (kPackedRows)
        k_row_b_w2<WP><<<dim3(WarpRowGeom<WP>::tiles_pairs, count), WarpRowGeom<WP>::BLOCK, warp_smem(), st>>>(d, base, s);
      else
        k_row_b_w<WP, SR, WR><<<dim3(WarpRowGeom<WP>::tiles_rows, count), WarpRowGeom<WP>::BLOCK, warp_smem(), st>>>(d, base, s);
    }
  }
  // ---- alternative column plan ----
  using AP = typename AltPlan<N>::type;
  static constexpr int alt_tiles_cols = (H + ColGeomF<AP, SR, WR>::W - 1) / ColGeomF<AP, SR, WR>::W;
  static size_t alt_smem() {
    constexpr int Ga = kBlock / AP::T, Wa = ColGeomF<AP, SR, WR>::W;
    const size_t row = (size_t)Ga * RowLayout<N>::stride;
    const size_t col = (size_t)host_smpad(N * Wa - 1) + 1;
    return (row > col ? row : col) * sizeof(cpx<SR>);
  }
  static cudaError_t prepare_alt() {
    const int b = (int)alt_smem();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_col_a<AP, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
    if ((e = cudaFuncSetAttribute(k_col_b<AP, SR, WR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
    return cudaSuccess;
  }
  static void col_a_alt(const InstDev* d, int count, const int* base, int s, cudaStream_t st) {
    k_col_a<AP, SR, WR><<<dim3(alt_tiles_cols, count), ColGeomF<AP, SR, WR>::B, alt_smem(), st>>>(d, base, s);
  }
  static void col_b_alt(const InstDev* d, int count, cudaStream_t st) {
    k_col_b<AP, SR, WR><<<dim3(alt_tiles_cols, count), ColGeomF<AP, SR, WR>::B, alt_smem(), st>>>(d);
  }
  // ---- pass-major twiddle tables ----
  template <class Q, typename Re>
  static void fill_one(const void* tw, cudaStream_t st) {
    k_fill_pass_tw<Q, Re><<<1, 256, 0, st>>>(static_cast<const cpx<Re>*>(tw));
  }
  static void fill_tables(const void* tw_s, const void* tw_w, cudaStream_t st) {
    fill_one<P, SR>(tw_s, st);
    fill_one<P, WR>(tw_w, st);
    fill_one<AP, SR>(tw_s, st);
    fill_one<AP, WR>(tw_w, st);
    if constexpr (warp_ok) {
      fill_one<WPA, SR>(tw_s, st);
      fill_one<WPA, WR>(tw_w, st);
      fill_one<WP, WR>(tw_w, st);
    }
  }
  // ---- adjoint (FP64) ----
  static constexpr bool adj_ok = std::is_same<SR, double>::value && std::is_same<WR, double>::value;
  static cudaError_t prepare_adj() {
    if constexpr (adj_ok) {
      const int bytes = (int)smem();
      cudaError_t e;
      if ((e = cudaFuncSetAttribute(k_adj_col1<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
      if ((e = cudaFuncSetAttribute(k_adj_col2<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
      if ((e = cudaFuncSetAttribute(k_adj_row2<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
      if ((e = cudaFuncSetAttribute(k_adj_mu_col<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
      if ((e = cudaFuncSetAttribute(k_adj_seed_row<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
        return e;
      if ((e = cudaFuncSetAttribute(k_adj_col1_m<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
      if ((e = cudaFuncSetAttribute(k_adj_col2_m<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
      if ((e = cudaFuncSetAttribute(k_adj_row2_m<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))) return e;
    }
    return cudaSuccess;
  }
  static void adj_col1_m(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_col1_m<P><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(a);
  }
  static void adj_col2_m(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_col2_m<P><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(a);
  }
  static void adj_row2_m(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_row2_m<P><<<dim3(tiles_pairs, count), kBlock, smem(), st>>>(a);
  }
  static void fill_adj32(const void* tw32, cudaStream_t st) {
    if constexpr (adj_ok) fill_one<P, float>(tw32, st);
  }
  static void adj_col1(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_col1<P><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(a);
  }
  static void adj_col2(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_col2<P><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(a);
  }
  static void adj_row2(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_row2<P><<<dim3(tiles_pairs, count), kBlock, smem(), st>>>(a);
  }
  static void adj_mu_col(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_mu_col<P><<<dim3(tiles_cols, count), kBlock, smem(), st>>>(a);
  }
  static void adj_seed_row(const AdjDev* a, int count, cudaStream_t st) {
    if constexpr (adj_ok) k_adj_seed_row<P><<<dim3(tiles_pairs, count), kBlock, smem(), st>>>(a);
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
    {
      // partial sums are scratch of one launch; size for the largest user
      int need = 5 * tiles_pairs + (tiles_cols > PG::tiles_cols ? tiles_cols : PG::tiles_cols) + tiles_rows;
      // the alternative column plan's partials sit after 5 * (its own row tiles)
      const int alt_need = 5 * ((H + kBlock / AP::T - 1) / (kBlock / AP::T)) + alt_tiles_cols +
                           (N + kBlock / AP::T - 1) / (kBlock / AP::T);
      if (alt_need > need) need = alt_need;
      const int wab = warp_partials();
      if (wab > need) need = wab;
      // column A keeps one partial per warp after the row-A area (both column plans)
      const int ca = 5 * tiles_pairs + ctiles * (CB / 32);
      if (ca > need) need = ca;
      const int caa = 5 * ((H + kBlock / AP::T - 1) / (kBlock / AP::T)) + alt_tiles_cols * (ColGeomF<AP, SR, WR>::B / 32);
      if (caa > need) need = caa;
      k.part_len = need;
    }
    k.smem = smem();
    k.sr_bytes = sizeof(SR);
    k.wr_bytes = sizeof(WR);
    k.cplx_per_field = (size_t)N * N / 2;  // H x n, the (DC, Nyquist) pair packed in slot 0
    k.generic = false;
    k.prepare = &prepare;
    k.fill_tables = &fill_tables;
    k.init = &init;
    k.fin = &fin;
    k.row_a = &row_a;
    k.col_a = &col_a;
    k.row_b = &row_b;
    k.col_b = &col_b;
    k.pipe_rows = PG::row_ok;
    k.pipe_cols = PG::col_ok;
    k.W = PG::W;
    k.RB = PG::RB;
    k.row_a_p = &row_a_p;
    k.row_b_p = &row_b_p;
    k.col_a_p = &col_a_p;
    k.col_b_p = &col_b_p;
    k.prepare_pipe = &prepare_pipe;
    k.warp_rows = warp_ok;
    k.row_a_w = &row_a_w;
    k.row_b_w = &row_b_w;
    k.prepare_warp = &prepare_warp;
    k.prepare_adj = &prepare_adj;
    k.col_a_alt = &col_a_alt;
    k.col_b_alt = &col_b_alt;
    k.E_alt = AP::E;
    k.adj_col1 = adj_ok ? &adj_col1 : nullptr;
    k.adj_col2 = adj_ok ? &adj_col2 : nullptr;
    k.adj_row2 = adj_ok ? &adj_row2 : nullptr;
    k.adj_col1_m = adj_ok ? &adj_col1_m : nullptr;
    k.adj_col2_m = adj_ok ? &adj_col2_m : nullptr;
    k.adj_row2_m = adj_ok ? &adj_row2_m : nullptr;
    k.fill_adj32 = adj_ok ? &fill_adj32 : nullptr;
    k.adj_mu_col = adj_ok ? &adj_mu_col : nullptr;
    k.adj_seed_row = adj_ok ? &adj_seed_row : nullptr;
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
