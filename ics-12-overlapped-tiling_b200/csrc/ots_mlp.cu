// ots_mlp.cu -- the learned tile-configuration cost model.
//
// The reference predicts the best (T, block, E) with a Weka k-NN model trained
// on runtime features (scripts/extract-features.py:40-127,
// scripts/run-weka.py:49-150).  Here the model is a small multi-layer
// perceptron trained and evaluated on the GPU by the kernels in this file:
//
//   x -> normalise -> [Linear -> SiLU] x (layers - 1) -> Linear -> y
//
// Every kernel is deterministic (fixed reduction order, no atomics), so a
// given seed gives bit-identical training runs.  One training epoch (all
// minibatches: gather, forward, loss, backward, AdamW) is captured once as a
// CUDA graph and replayed per epoch; only the epoch's permutation is copied
// in before each replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/ots.h"


// Shared with ots_runtime.cu: the message ots_last_error() returns.
void ots_set_last_error(const char* msg);

namespace {

ots_status mfail(ots_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  ots_set_last_error(buf);
  return s;
}

#define MLP_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return mfail(e_ == cudaErrorMemoryAllocation ? OTS_ERR_OUT_OF_MEMORY : OTS_ERR_CUDA, \
                   "%s: %s", #call, cudaGetErrorString(e_));                        \
  } while (0)

// C[M x N] = op(A)[M x K] * op(B)[K x N] (+ bias[n] per column).
// op(A)(m,k) = transA ? A[k*lda + m] : A[m*lda + k]; likewise B.
// 16 x 16 tiles through shared memory; each C element is one thread's
// fixed-order sum, so results are deterministic.
constexpr int TB = 16;
__global__ void k_gemm(int M, int N, int K, const float* __restrict__ A, int lda, int transA,
                       const float* __restrict__ B, int ldb, int transB, float* __restrict__ C,
                       int ldc, const float* __restrict__ bias) {
  __shared__ float As[TB][TB + 1];
  __shared__ float Bs[TB][TB + 1];
  const int m = blockIdx.y * TB + threadIdx.y;
  const int n = blockIdx.x * TB + threadIdx.x;
  float acc = 0.0f;
  for (int k0 = 0; k0 < K; k0 += TB) {
    {
      const int mm = blockIdx.y * TB + threadIdx.y, kk = k0 + threadIdx.x;
      float v = 0.0f;
      if (mm < M && kk < K) v = transA ? A[(size_t)kk * lda + mm] : A[(size_t)mm * lda + kk];
      As[threadIdx.y][threadIdx.x] = v;
    }
    {
      const int kk = k0 + threadIdx.y, nn = blockIdx.x * TB + threadIdx.x;
      float v = 0.0f;
      if (kk < K && nn < N) v = transB ? B[(size_t)nn * ldb + kk] : B[(size_t)kk * ldb + nn];
      Bs[threadIdx.y][threadIdx.x] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TB; ++kk) acc += As[threadIdx.y][kk] * Bs[kk][threadIdx.x];
    __syncthreads();
  }
  if (m < M && n < N) C[(size_t)m * ldc + n] = acc + (bias ? bias[n] : 0.0f);
}

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

__global__ void k_silu(const float* __restrict__ Z, float* __restrict__ A, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[i] = Z[i] * sigmoid(Z[i]);
}

// In place: A = silu(A) (one pointer, no aliasing promise).
__global__ void k_silu_inplace(float* A, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float z = A[i];
    A[i] = z * sigmoid(z);
  }
}

// dZ = dA * silu'(Z), silu'(z) = s(z) (1 + z (1 - s(z)))
__global__ void k_silu_bwd(const float* __restrict__ dA, const float* __restrict__ Z,
                           float* __restrict__ dZ, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float s = sigmoid(Z[i]);
    dZ[i] = dA[i] * (s * (1.0f + Z[i] * (1.0f - s)));
  }
}

__global__ void k_normalize(const float* __restrict__ X, const float* __restrict__ mean,
                            const float* __restrict__ inv_std, float* __restrict__ Y, int n, int f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n * f) {
    const int c = i % f;
    Y[i] = (X[i] - mean[c]) * inv_std[c];
  }
}

// Rows perm[off .. off+B) of X (already normalised) and y into the batch.
__global__ void k_gather(const float* __restrict__ X, const float* __restrict__ y,
                         const int* __restrict__ perm, int off, int B, int f,
                         float* __restrict__ Xb, float* __restrict__ yb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B * f) {
    const int r = i / f, c = i - r * f;
    Xb[i] = X[(size_t)perm[off + r] * f + c];
  }
  if (i < B) yb[i] = y[perm[off + i]];
}

// MSE on normalised targets: loss = mean((p - t)^2), dP = 2 (p - t) / B.
// One block; fixed-order tree reduction.
__global__ void k_mse(const float* __restrict__ p, const float* __restrict__ t, int B,
                      float* __restrict__ dP, float* __restrict__ loss_out) {
  __shared__ float red[1024];
  float acc = 0.0f;
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    const float d = p[i] - t[i];
    dP[i] = 2.0f * d / (float)B;
    acc += d * d;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss_out) *loss_out = red[0] / (float)B;
}

// db[o] = sum_b dZ[b, o] (fixed order)
__global__ void k_colsum(const float* __restrict__ dZ, int B, int O, float* __restrict__ db) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < O) {
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += dZ[(size_t)b * O + o];
    db[o] = s;
  }
}

// Step counter and bias corrections for Adam (one thread).
__global__ void k_adam_prep(int* step, float* corr, float b1, float b2) {
  const int t = ++(*step);
  corr[0] = 1.0f - powf(b1, (float)t);
  corr[1] = 1.0f - powf(b2, (float)t);
}

// AdamW (decoupled weight decay on every parameter).
__global__ void k_adamw(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                        float* __restrict__ v, const float* __restrict__ corr, int n, float lr,
                        float b1, float b2, float eps, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / corr[0], vh = vi / corr[1];
    w[i] = w[i] - lr * (mh / (sqrtf(vh) + eps) + wd * w[i]);
  }
}

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

// y = z * scale + shift (undo the target standardisation)
__global__ void k_affine(const float* __restrict__ z, float* __restrict__ y, int n, float scale,
                         float shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = z[i] * scale + shift;
}

// Fixed-size working memory of ots_mlp_predict_noalloc: two ping-pong
// activation buffers of kNoAllocRows x kNoAllocWidth floats (2 MiB in all).
// It lives in the module image, so every GPU that loads libots holds it until
// the process exits; no call allocates it.
constexpr int kNoAllocRows = 4096;
constexpr int kNoAllocWidth = 64;
__device__ __align__(256) float g_noalloc_scratch[2 * kNoAllocRows * kNoAllocWidth];

// Device address of g_noalloc_scratch, looked up once per device.
constexpr int kMaxDevices = 64;
float* g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mu;

}  // namespace

struct ots_mlp {
  int device = 0;
  int n_in = 0, hidden = 0, layers = 0;
  std::vector<int> dims;        // layer widths: n_in, hidden..., 1
  std::vector<size_t> w_off, b_off;
  size_t n_params = 0;
  cudaStream_t stream = nullptr;
  float *d_params = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr;
  float *d_mean = nullptr, *d_inv_std = nullptr;
  float y_mean = 0.0f, y_std = 1.0f;
  int* d_step = nullptr;
  float* d_corr = nullptr;
  // activations for a batch of up to cap rows
  int cap = 0;
  std::vector<float*> Z, A, dA;  // per layer outputs (pre/post activation) and grads
  float* d_in = nullptr;         // normalised input batch
  float* d_dout = nullptr;       // d loss / d prediction
  float* d_loss = nullptr;       // per-minibatch losses
  int loss_cap = 0;
};

namespace {

void free_acts(ots_mlp* m) {
  for (float* p : m->Z) cudaFree(p);
  for (float* p : m->A) cudaFree(p);
  for (float* p : m->dA) cudaFree(p);
  m->Z.clear();
  m->A.clear();
  m->dA.clear();
  cudaFree(m->d_in);
  cudaFree(m->d_dout);
  m->d_in = m->d_dout = nullptr;
  m->cap = 0;
}

ots_status ensure_acts(ots_mlp* m, int rows) {
  if (rows <= m->cap) return OTS_OK;
  free_acts(m);
  const int L = m->layers;
  m->Z.assign(L, nullptr);
  m->A.assign(L, nullptr);
  m->dA.assign(L, nullptr);
  for (int l = 0; l < L; ++l) {
    const size_t sz = (size_t)rows * m->dims[l + 1] * sizeof(float);
    MLP_CUDA(cudaMalloc(&m->Z[l], sz));
    MLP_CUDA(cudaMalloc(&m->A[l], sz));
    MLP_CUDA(cudaMalloc(&m->dA[l], sz));
  }
  MLP_CUDA(cudaMalloc(&m->d_in, (size_t)rows * m->n_in * sizeof(float)));
  MLP_CUDA(cudaMalloc(&m->d_dout, (size_t)rows * sizeof(float)));
  m->cap = rows;
  return OTS_OK;
}

void gemm(cudaStream_t s, int M, int N, int K, const float* A, int lda, int tA, const float* B,
          int ldb, int tB, float* C, int ldc, const float* bias) {
  dim3 blk(TB, TB), grd(cdiv(N, TB), cdiv(M, TB));
  k_gemm<<<grd, blk, 0, s>>>(M, N, K, A, lda, tA, B, ldb, tB, C, ldc, bias);
}

// Forward on rows already normalised in `x` (rows x n_in); output in A[L-1].
void forward(ots_mlp* m, const float* x, int rows) {
  const float* in = x;
  for (int l = 0; l < m->layers; ++l) {
    const int I = m->dims[l], O = m->dims[l + 1];
    gemm(m->stream, rows, O, I, in, I, 0, m->d_params + m->w_off[l], I, 1, m->Z[l], O,
         m->d_params + m->b_off[l]);
    const bool last = l == m->layers - 1;
    if (!last) {
      k_silu<<<cdiv(rows * O, 256), 256, 0, m->stream>>>(m->Z[l], m->A[l], rows * O);
      in = m->A[l];
    } else {
      in = m->Z[l];
    }
  }
}

// Backward from d_dout (rows x 1) into d_grad.
void backward(ots_mlp* m, const float* x, int rows) {
  const int L = m->layers;
  const float* dz = m->d_dout;  // dL/dZ of the last (linear) layer
  for (int l = L - 1; l >= 0; --l) {
    const int I = m->dims[l], O = m->dims[l + 1];
    const float* in = l == 0 ? x : m->A[l - 1];
    // dW[O x I] = dZ^T[O x rows] * in[rows x I]
    gemm(m->stream, O, I, rows, dz, O, 1, in, I, 0, m->d_grad + m->w_off[l], I, nullptr);
    k_colsum<<<cdiv(O, 128), 128, 0, m->stream>>>(dz, rows, O, m->d_grad + m->b_off[l]);
    if (l > 0) {
      // dA_{l-1}[rows x I] = dZ[rows x O] * W[O x I]; then through SiLU
      gemm(m->stream, rows, I, O, dz, O, 0, m->d_params + m->w_off[l], I, 0, m->dA[l - 1], I,
           nullptr);
      k_silu_bwd<<<cdiv(rows * I, 256), 256, 0, m->stream>>>(m->dA[l - 1], m->Z[l - 1],
                                                              m->dA[l - 1], rows * I);
      dz = m->dA[l - 1];
    }
  }
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

ots_status ots_mlp_create(int32_t n_in, int32_t hidden, int32_t layers, uint64_t seed,
                          int32_t device, ots_mlp** out) {
  if (!out || n_in < 1 || hidden < 1 || layers < 1 || layers > 8)
    return mfail(OTS_ERR_INVALID_ARGUMENT, "bad MLP shape");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return mfail(OTS_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= ndev) return mfail(OTS_ERR_INVALID_ARGUMENT, "bad device");
  MLP_CUDA(cudaSetDevice(device));
  ots_mlp* m = new ots_mlp();
  m->device = device;
  m->n_in = n_in;
  m->hidden = hidden;
  m->layers = layers;
  m->dims.push_back(n_in);
  for (int l = 0; l < layers - 1; ++l) m->dims.push_back(hidden);
  m->dims.push_back(1);
  size_t off = 0;
  for (int l = 0; l < layers; ++l) {
    m->w_off.push_back(off);
    off += (size_t)m->dims[l] * m->dims[l + 1];
    m->b_off.push_back(off);
    off += m->dims[l + 1];
  }
  m->n_params = off;
  // Glorot-uniform weights from a seeded splitmix64 stream, zero biases.
  std::vector<float> h(m->n_params, 0.0f);
  uint64_t s = seed;
  for (int l = 0; l < layers; ++l) {
    const int I = m->dims[l], O = m->dims[l + 1];
    const double a = std::sqrt(6.0 / (I + O));
    for (size_t i = 0; i < (size_t)I * O; ++i) {
      const double u = (splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
      h[m->w_off[l] + i] = (float)((2.0 * u - 1.0) * a);
    }
  }
  const size_t pb = m->n_params * sizeof(float);
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_params, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_grad, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_m, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_v, pb);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_mean, n_in * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->d_inv_std, n_in * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->d_step, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&m->d_corr, 2 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(m->d_params, h.data(), pb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(m->d_m, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(m->d_v, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(m->d_step, 0, sizeof(int));
  if (e == cudaSuccess) {
    std::vector<float> zero(n_in, 0.0f), one(n_in, 1.0f);
    e = cudaMemcpy(m->d_mean, zero.data(), n_in * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(m->d_inv_std, one.data(), n_in * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    ots_mlp_destroy(m);
    return mfail(OTS_ERR_CUDA, "MLP allocation: %s", cudaGetErrorString(e));
  }
  *out = m;
  return OTS_OK;
}

void ots_mlp_destroy(ots_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  free_acts(m);
  cudaFree(m->d_params);
  cudaFree(m->d_grad);
  cudaFree(m->d_m);
  cudaFree(m->d_v);
  cudaFree(m->d_mean);
  cudaFree(m->d_inv_std);
  cudaFree(m->d_step);
  cudaFree(m->d_corr);
  cudaFree(m->d_loss);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

ots_status ots_mlp_num_params(const ots_mlp* m, int64_t* n) {
  if (!m || !n) return mfail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  *n = (int64_t)m->n_params;
  return OTS_OK;
}

ots_status ots_mlp_get_params(const ots_mlp* m, float* params) {
  if (!m || !params) return mfail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  MLP_CUDA(cudaSetDevice(m->device));
  MLP_CUDA(cudaMemcpy(params, m->d_params, m->n_params * sizeof(float), cudaMemcpyDeviceToHost));
  return OTS_OK;
}

ots_status ots_mlp_set_params(ots_mlp* m, const float* params) {
  if (!m || !params) return mfail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  MLP_CUDA(cudaSetDevice(m->device));
  MLP_CUDA(cudaMemcpy(m->d_params, params, m->n_params * sizeof(float), cudaMemcpyHostToDevice));
  return OTS_OK;
}

ots_status ots_mlp_set_normalization(ots_mlp* m, const float* mean, const float* inv_std,
                                     float y_mean, float y_std) {
  if (!m || !mean || !inv_std || !(y_std > 0.0f))
    return mfail(OTS_ERR_INVALID_ARGUMENT, "bad normalisation");
  MLP_CUDA(cudaSetDevice(m->device));
  MLP_CUDA(cudaMemcpy(m->d_mean, mean, m->n_in * sizeof(float), cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(m->d_inv_std, inv_std, m->n_in * sizeof(float), cudaMemcpyHostToDevice));
  m->y_mean = y_mean;
  m->y_std = y_std;
  return OTS_OK;
}

// Loss (on normalised targets) and the full-batch gradient, for checks.
ots_status ots_mlp_loss_grad(ots_mlp* m, const float* X, const float* y, int32_t n, float* loss,
                             float* grad) {
  if (!m || !X || !y || n < 1 || n > 4096)
    return mfail(OTS_ERR_INVALID_ARGUMENT, "bad arguments (1 <= n <= 4096)");
  MLP_CUDA(cudaSetDevice(m->device));
  ots_status st = ensure_acts(m, n);
  if (st != OTS_OK) return st;
  float *dX = nullptr, *dy = nullptr, *dl = nullptr;
  MLP_CUDA(cudaMalloc(&dX, (size_t)n * m->n_in * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dy, (size_t)n * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dl, sizeof(float)));
  std::vector<float> yn(n);
  for (int i = 0; i < n; ++i) yn[i] = (y[i] - m->y_mean) / m->y_std;
  cudaMemcpyAsync(dX, X, (size_t)n * m->n_in * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  cudaMemcpyAsync(dy, yn.data(), n * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  k_normalize<<<cdiv(n * m->n_in, 256), 256, 0, m->stream>>>(dX, m->d_mean, m->d_inv_std, m->d_in,
                                                             n, m->n_in);
  forward(m, m->d_in, n);
  k_mse<<<1, 1024, 0, m->stream>>>(m->Z[m->layers - 1], dy, n, m->d_dout, dl);
  backward(m, m->d_in, n);
  float hl = 0.0f;
  cudaMemcpyAsync(&hl, dl, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
  if (grad)
    cudaMemcpyAsync(grad, m->d_grad, m->n_params * sizeof(float), cudaMemcpyDeviceToHost,
                    m->stream);
  cudaError_t e = cudaStreamSynchronize(m->stream);
  cudaFree(dX);
  cudaFree(dy);
  cudaFree(dl);
  if (e != cudaSuccess) return mfail(OTS_ERR_CUDA, "loss_grad: %s", cudaGetErrorString(e));
  if (loss) *loss = hl;
  return OTS_OK;
}

ots_status ots_mlp_train(ots_mlp* m, const float* X, const float* y, int32_t n, int32_t epochs,
                         int32_t batch, float lr, float weight_decay, uint64_t seed,
                         float* final_loss) {
  if (!m || !X || !y || n < 1 || epochs < 0 || batch < 1 || batch > 1024)
    return mfail(OTS_ERR_INVALID_ARGUMENT, "bad training arguments (1 <= batch <= 1024)");
  MLP_CUDA(cudaSetDevice(m->device));
  if (batch > n) batch = n;
  const int nb = n / batch;  // full minibatches per epoch (the remainder rotates)
  ots_status st = ensure_acts(m, batch);
  if (st != OTS_OK) return st;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float *dXall = nullptr, *dXn = nullptr, *dyall = nullptr, *dXb = nullptr, *dyb = nullptr;
  int* dperm = nullptr;
  MLP_CUDA(cudaMalloc(&dXall, (size_t)n * m->n_in * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dXn, (size_t)n * m->n_in * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dyall, (size_t)n * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dXb, (size_t)batch * m->n_in * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dyb, (size_t)batch * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dperm, (size_t)n * sizeof(int)));
  if (m->loss_cap < nb) {
    cudaFree(m->d_loss);
    MLP_CUDA(cudaMalloc(&m->d_loss, (size_t)std::max(1, nb) * sizeof(float)));
    m->loss_cap = nb;
  }
  std::vector<float> yn(n);
  for (int i = 0; i < n; ++i) yn[i] = (y[i] - m->y_mean) / m->y_std;
  cudaMemcpyAsync(dXall, X, (size_t)n * m->n_in * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  cudaMemcpyAsync(dyall, yn.data(), n * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  k_normalize<<<cdiv(n * m->n_in, 256), 256, 0, m->stream>>>(dXall, m->d_mean, m->d_inv_std, dXn,
                                                             n, m->n_in);

  // Capture one epoch.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int b = 0; b < nb; ++b) {
      k_gather<<<cdiv(batch * m->n_in, 256), 256, 0, m->stream>>>(dXn, dyall, dperm, b * batch,
                                                                   batch, m->n_in, dXb, dyb);
      forward(m, dXb, batch);
      k_mse<<<1, 1024, 0, m->stream>>>(m->Z[m->layers - 1], dyb, batch, m->d_dout, m->d_loss + b);
      backward(m, dXb, batch);
      k_adam_prep<<<1, 1, 0, m->stream>>>(m->d_step, m->d_corr, b1, b2);
      k_adamw<<<cdiv((int)m->n_params, 256), 256, 0, m->stream>>>(
          m->d_params, m->d_grad, m->d_m, m->d_v, m->d_corr, (int)m->n_params, lr, b1, b2, eps,
          weight_decay);
    }
    e = cudaStreamEndCapture(m->stream, &graph);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  std::mt19937_64 rng(seed);
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::vector<int> pinned_perm(n);
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    pinned_perm = perm;
    e = cudaMemcpyAsync(dperm, pinned_perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice,
                        m->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);  // pinned_perm reuse
  }
  float last = 0.0f;
  if (e == cudaSuccess && nb > 0) {
    std::vector<float> hl(nb);
    e = cudaMemcpy(hl.data(), m->d_loss, nb * sizeof(float), cudaMemcpyDeviceToHost);
    for (float v : hl) last += v / nb;
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  cudaFree(dXall);
  cudaFree(dXn);
  cudaFree(dyall);
  cudaFree(dXb);
  cudaFree(dyb);
  cudaFree(dperm);
  if (e != cudaSuccess) return mfail(OTS_ERR_CUDA, "training: %s", cudaGetErrorString(e));
  if (final_loss) *final_loss = last;
  return OTS_OK;
}

ots_status ots_mlp_predict(ots_mlp* m, const float* X, int32_t n, float* y_out) {
  if (!m || !X || !y_out || n < 1) return mfail(OTS_ERR_INVALID_ARGUMENT, "bad arguments");
  MLP_CUDA(cudaSetDevice(m->device));
  const int chunk = 4096;
  ots_status st = ensure_acts(m, std::min(n, chunk));
  if (st != OTS_OK) return st;
  float* dX = nullptr;
  MLP_CUDA(cudaMalloc(&dX, (size_t)std::min(n, chunk) * m->n_in * sizeof(float)));
  std::vector<float> yn(n);
  cudaError_t e = cudaSuccess;
  for (int o = 0; o < n && e == cudaSuccess; o += chunk) {
    const int r = std::min(chunk, n - o);
    cudaMemcpyAsync(dX, X + (size_t)o * m->n_in, (size_t)r * m->n_in * sizeof(float),
                    cudaMemcpyHostToDevice, m->stream);
    k_normalize<<<cdiv(r * m->n_in, 256), 256, 0, m->stream>>>(dX, m->d_mean, m->d_inv_std,
                                                               m->d_in, r, m->n_in);
    forward(m, m->d_in, r);
    cudaMemcpyAsync(yn.data() + o, m->Z[m->layers - 1], r * sizeof(float), cudaMemcpyDeviceToHost,
                    m->stream);
    e = cudaStreamSynchronize(m->stream);
  }
  cudaFree(dX);
  if (e != cudaSuccess) return mfail(OTS_ERR_CUDA, "predict: %s", cudaGetErrorString(e));
  for (int i = 0; i < n; ++i) y_out[i] = yn[i] * m->y_std + m->y_mean;
  return OTS_OK;
}

// Inference with no allocation (see include/ots.h).  X and y are device
// pointers; the activations live in g_noalloc_scratch, whose device address
// is looked up with cudaGetSymbolAddress on the first call on each device.
ots_status ots_mlp_predict_noalloc(const ots_mlp* m, const float* X, int32_t n, float* y,
                                   void* stream) {
  if (!m || !X || !y) return mfail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (n < 1 || n > kNoAllocRows)
    return mfail(OTS_ERR_INVALID_ARGUMENT,
                 "ots_mlp_predict_noalloc: n = %d rows; the fixed scratch holds 1..%d rows", n,
                 kNoAllocRows);
  for (int l = 0; l <= m->layers; ++l)
    if (m->dims[l] > kNoAllocWidth)
      return mfail(OTS_ERR_UNSUPPORTED,
                   "ots_mlp_predict_noalloc: layer width %d exceeds the fixed scratch width %d",
                   m->dims[l], kNoAllocWidth);
  int dev = -1;
  MLP_CUDA(cudaGetDevice(&dev));
  if (dev != m->device)
    return mfail(OTS_ERR_INVALID_ARGUMENT,
                 "ots_mlp_predict_noalloc: current device %d is not the model's device %d", dev,
                 m->device);
  if (dev < 0 || dev >= kMaxDevices)
    return mfail(OTS_ERR_UNSUPPORTED, "ots_mlp_predict_noalloc: device %d out of range", dev);
  float* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return mfail(OTS_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s",
                     cudaGetErrorString(e));
      g_noalloc_ptr[dev] = static_cast<float*>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* buf[2] = {scratch, scratch + (size_t)kNoAllocRows * kNoAllocWidth};
  // every element read below is written first in this call, so the previous
  // call's contents never leak into the result
  k_normalize<<<cdiv(n * m->n_in, 256), 256, 0, s>>>(X, m->d_mean, m->d_inv_std, buf[0], n,
                                                     m->n_in);
  int cur = 0;
  for (int l = 0; l < m->layers; ++l) {
    const int I = m->dims[l], O = m->dims[l + 1];
    gemm(s, n, O, I, buf[cur], I, 0, m->d_params + m->w_off[l], I, 1, buf[cur ^ 1], O,
         m->d_params + m->b_off[l]);
    if (l < m->layers - 1)
      k_silu_inplace<<<cdiv(n * O, 256), 256, 0, s>>>(buf[cur ^ 1], n * O);
    cur ^= 1;
  }
  k_affine<<<cdiv(n, 256), 256, 0, s>>>(buf[cur], y, n, m->y_std, m->y_mean);
  MLP_CUDA(cudaGetLastError());
  return OTS_OK;
}

ots_status ots_mlp_topk(ots_mlp* m, const float* X, int32_t n, int32_t k, int32_t* idx_out) {
  if (!m || !X || !idx_out || n < 1 || k < 1) return mfail(OTS_ERR_INVALID_ARGUMENT, "bad arguments");
  std::vector<float> p(n);
  ots_status st = ots_mlp_predict(m, X, n, p.data());
  if (st != OTS_OK) return st;
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  k = std::min(k, n);
  std::partial_sort(idx.begin(), idx.begin() + k, idx.end(), [&](int a, int b) {
    return p[a] > p[b] || (p[a] == p[b] && a < b);
  });
  std::copy(idx.begin(), idx.begin() + k, idx_out);
  return OTS_OK;
}

}  // extern "C"
