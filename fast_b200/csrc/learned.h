// learned.h - private types of the learned load-step predictor: the BF16
// tensor-core MLP (mlp.cu), the FP64 POD kernels (pod.cu) and the predictor
// object behind the fast_gpu_ws_* entry points (warmstart.cu).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace fastgpu {

// ---------------------------------------------------------------- mlp.cu
// Epilogues of the tensor-core GEMM C = op(A) op(B)^T (FP32 out):
enum GemmEpi : int {
  kEpiStore = 0,     // C = acc
  kEpiBias = 1,      // C = acc + bias[n]
  kEpiBiasTanh = 2,  // C = tanh(acc + bias[n])
  kEpiDTanh = 3,     // C = acc * (1 - aux[m][n]^2)   (tanh backward)
};

// C[M x N] (row-major, ldc) = sum_k opA(m, k) * opB(n, k) on the tcgen05
// tensor cores: operands are read as FP32, rounded to BF16 into shared memory,
// accumulated in FP32 in tensor memory.
//   opA(m, k) = ta ? A[k * lda + m] : A[m * lda + k]
//   opB(n, k) = tb ? B[k * ldb + n] : B[n * ldb + k]
// A wait that does not finish within its limit sets *status = 1.
// With ws (>= splits * M * N floats, see gemm_splits) a store-epilogue GEMM
// with few output tiles and a long K is split over K across CTAs and the
// partial tiles are summed in a fixed order by a second kernel.
cudaError_t gemm_bf16(cudaStream_t s, int M, int N, int K, const float *A, int lda, bool ta, const float *B,
                      int ldb, bool tb, float *C, int ldc, int epi, const float *bias, const float *aux,
                      int ldaux, int32_t *status, float *ws = nullptr);
int gemm_splits(int M, int N, int K, int epi);

struct MlpRow;  // mlp_row.cuh

// Fully connected tanh network: dims[0] -> dims[1] -> ... -> dims[L] with
// tanh on the hidden layers and a linear output.  Parameters are FP32
// (layer l: W_l [dims[l+1]][dims[l]] row-major, then b_l [dims[l+1]]).
struct Mlp {
  std::vector<int> dims;
  std::vector<int64_t> w_off, b_off;
  int64_t nparams = 0;
  float *d_params = nullptr, *d_grads = nullptr, *d_m = nullptr, *d_v = nullptr;
  int cap = 0;                    // batch capacity of the activation buffers
  std::vector<float *> d_h;       // h[0] input, h[l] output of layer l   [cap][dims[l]]
  std::vector<float *> d_g;       // dLoss / d(pre-activation of layer l) [cap][dims[l]]
  float *d_target = nullptr;      // [cap][dims[L]]
  float *d_part = nullptr;        // loss partial sums
  float *d_loss = nullptr;        // [1]
  float *d_splitws = nullptr;     // split-K partial tiles of the weight gradients
  int32_t *d_status = nullptr;
  int64_t adam_t = 0;
  int64_t launches = 0;

  int layers() const { return (int)dims.size() - 1; }
  cudaError_t init(const std::vector<int> &d, uint64_t seed);   // allocates params, Xavier init
  cudaError_t reserve(int batch);
  void release();
  // h[0] must hold the input rows; output in h[L]
  cudaError_t forward(cudaStream_t s, int batch);
  // one row (batch 1) through the network on the CUDA cores by one CTA
  // (mlp_row.cuh): h[0] row 0 -> h[L] row 0, one launch
  cudaError_t forward_row(cudaStream_t s);
  // the layer sizes and offsets the single-row forward reads; false when the
  // network is deeper or wider than it takes
  bool row_layout(MlpRow &r) const;
  // after forward: loss vs d_target (mean squared error), gradients in d_grads
  cudaError_t backward(cudaStream_t s, int batch);
  cudaError_t adam(cudaStream_t s, float lr, float beta1, float beta2, float eps);
};

// ---------------------------------------------------------------- pod.cu
// FP64 C[M x N] = opA(A) opB(B) with opA(m, k) = ta ? A[k lda + m] : A[m lda + k],
// opB(k, n) = tb ? B[n ldb + k] : B[k ldb + n].  Split over K into fixed
// slices summed in a fixed order (deterministic); ws holds >= splits*M*N
// doubles when splits > 1 (dgemm_splits gives the count).
int dgemm_splits(int M, int N, int K);
cudaError_t dgemm(cudaStream_t s, int M, int N, int K, const double *A, int lda, bool ta, const double *B, int ldb,
                  bool tb, double *C, int ldc, double *ws);

// C[p][q] (row-major, ldc) = sum_i A[i lda + a] B[i ldb + b] over the n rows
// of two tall, thin row-major matrices (p q <= kSkinnyMaxOut): one pass over
// the rows by kSkinnyBlocks blocks, partials (ws >= kSkinnyBlocks p q
// doubles) summed in a fixed order.  Two launches.
constexpr int kSkinnyBlocks = 296;
constexpr int kSkinnyMaxOut = 4096;
cudaError_t skinny_atb(cudaStream_t s, int64_t n, int p, int q, const double *A, int lda, const double *B, int ldb,
                       double *C, int ldc, double *ws);

// symmetric eigen-decomposition (cyclic Jacobi) of a small n x n matrix:
// eigenvalues descending in w, eigenvectors as columns of V (row-major n x n)
void sym_eig(int n, std::vector<double> a, std::vector<double> &w, std::vector<double> &V);

}  // namespace fastgpu
