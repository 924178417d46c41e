// Learned rank predictor (predictor.cu): box features and the BF16 MLP.
#pragma once
#include "common.cuh"

namespace flam {

constexpr int kPredFeatures = 16;

// 16 features per task of a step (slf ids already gathered), FP32, row-major.
void launch_box_features(const CompressTask* tasks, int ntask, const int64_t* ipool, const Problem& P, float neg_log_tol,
                         float* out, cudaStream_t s);
size_t mlp_smem_bytes();
// Forward over nsamp samples (X: nsamp x 16 row-major); yhat may be null.  With train:
// also the backward pass, gradient sums of mean-squared error scaled by inv_batch added to
// grad, and the sum of squared errors added to *loss.
void launch_mlp(const float* X, const float* y, int64_t nsamp, const float* w, float* yhat, float* grad, float* loss,
                float inv_batch, int train, cudaStream_t s);
void launch_adam(float* w, float* m, float* v, float* grad, float lr, int step, cudaStream_t s);

}  // namespace flam
