// Cluster-resident single-grid runs (esc_cluster.cu): the interface the engine
// (esc_api.cu) uses.  One thread-block cluster runs the whole time loop of one
// FP64 grid of a supported size; see esc_cluster.cu.
#pragma once
#include <cuda_runtime.h>

#include "esc_kernels.cuh"

namespace esc {
namespace clu {

struct Args {
  const double* phi;  // n*n FP64 particle field (device)
  double* c;          // n*n composition (device): input, and output unless the run stopped
  double* hist;       // column-major (hist_ld x 6), rows 0..steps (device)
  int hist_ld, steps;
  double dt, dx;
  ModelParams p;
  int* status;        // set to 1 (non-finite) by a stopped run
  long long* bad_step;
};

// true when n has a cluster configuration and this device can place one such
// cluster (queried once per size and device)
bool available(int n);
// fills the pass-major twiddle tables of n's cluster plans from the plain FP64 table
// e^{-2 pi i j / n} (device), in stream order
cudaError_t prepare(int n, const void* tw_plain, cudaStream_t st);
// queues one run (one cluster launch)
cudaError_t run(int n, const Args& a, cudaStream_t st);

}  // namespace clu
}  // namespace esc
