// Learned initial guess: the interface the solver context uses (cnn.cu).
#pragma once
#include <cuda_runtime.h>

#include "cgli_dev.cuh"

struct cgli_cnn;

namespace cgli {

// grid of the network matches the context's interior grid
bool cnn_matches(const cgli_cnn *n, int nx, int ny, int nz);
// U_ (interior) = 3 U - 3 Uq + Uqq + correction(U, Uq, Uqq) / J on stream s
cudaError_t cnn_predict(cgli_cnn *n, const Dev &d, cudaStream_t s);
// appends the context's current level U (Q^n after the time-level shift) as
// physical Q to the network's stored levels
int cnn_store_level(cgli_cnn *n, const Dev &d, cudaStream_t s);
// mean device time of `reps` inferences on the context's levels
int cnn_time_inference(cgli_cnn *n, const Dev &d, cudaStream_t s, int reps, float *ms);

}  // namespace cgli
