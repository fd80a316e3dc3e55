// Learned SpMV variant selector for sm_100a: matrix features and a small MLP
// cost model (12 -> 64 -> 64 -> V, FP32, ReLU), with its training kernels.
//
// Features (all from integer accumulators, so they do not depend on the
// order of the atomics): for a CSR matrix, one warp per row accumulates the
// row length, its square, the row maximum, empty rows, the largest and the
// summed |column - row|, diagonal entries, and "segments" -- runs of entries
// that fall in the same 8-column block -- from which twelve numbers are
// derived (selector_finalize below).
//
// The MLP predicts, per variant, the log of the run time relative to the
// matrix's mean over variants; the variant with the smallest prediction is
// picked.  Training is full-batch Adam on mean squared error; every gradient
// sum runs in a fixed order (one thread per weight, samples in order), so a
// training run is reproducible bit for bit.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kIn = ASCB_SELECTOR_FEATURES;    // 12
constexpr int kHidden = ASCB_SELECTOR_HIDDEN;  // 64

// accumulator slots
enum { kSumLen2 = 0, kMaxLen, kEmpty, kMaxDist, kSumDist, kDiag, kSegments, kAccCount };

__global__ void features_accumulate(const int64_t* __restrict__ ptr,
                                    const int64_t* __restrict__ idx, int64_t rows,
                                    unsigned long long* __restrict__ acc) {
  __shared__ unsigned long long block_acc[kAccCount];
  if (threadIdx.x < kAccCount) block_acc[threadIdx.x] = 0ull;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  unsigned long long len2 = 0, maxlen = 0, empty = 0, maxdist = 0, sumdist = 0, diag = 0,
                     segs = 0;
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += warps) {
    const int64_t b = __ldg(ptr + r);
    const int64_t e = __ldg(ptr + r + 1);
    const unsigned long long len = static_cast<unsigned long long>(e - b);
    if (lane == 0) {
      len2 += len * len;
      maxlen = len > maxlen ? len : maxlen;
      empty += len == 0 ? 1ull : 0ull;
    }
    for (int64_t q = b + lane; q < e; q += 32) {
      const int64_t c = __ldg(idx + q);
      const unsigned long long d = static_cast<unsigned long long>(c > r ? c - r : r - c);
      maxdist = d > maxdist ? d : maxdist;
      sumdist += d;
      diag += c == r ? 1ull : 0ull;
      const bool starts = q == b || (__ldg(idx + q - 1) >> 3) != (c >> 3);
      segs += starts ? 1ull : 0ull;
    }
  }
  atomicAdd(&block_acc[kSumLen2], len2);
  atomicMax(&block_acc[kMaxLen], maxlen);
  atomicAdd(&block_acc[kEmpty], empty);
  atomicMax(&block_acc[kMaxDist], maxdist);
  atomicAdd(&block_acc[kSumDist], sumdist);
  atomicAdd(&block_acc[kDiag], diag);
  atomicAdd(&block_acc[kSegments], segs);
  __syncthreads();
  if (threadIdx.x < kAccCount) {
    const unsigned long long v = block_acc[threadIdx.x];
    if (threadIdx.x == kMaxLen || threadIdx.x == kMaxDist) {
      atomicMax(acc + threadIdx.x, v);
    } else {
      atomicAdd(acc + threadIdx.x, v);
    }
  }
}

__global__ void selector_finalize(const unsigned long long* __restrict__ acc, int64_t rows,
                                  int64_t cols, int64_t nnz, int element_bytes,
                                  float* __restrict__ f) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double n = static_cast<double>(rows > 0 ? rows : 1);
  const double c = static_cast<double>(cols > 0 ? cols : 1);
  const double z = static_cast<double>(nnz);
  const double mean = z / n;
  const double var = static_cast<double>(acc[kSumLen2]) / n - mean * mean;
  const double cv = mean > 0.0 ? sqrt(var > 0.0 ? var : 0.0) / mean : 0.0;
  const double mn = static_cast<double>(rows < cols ? rows : cols);
  f[0] = static_cast<float>(log2(1.0 + static_cast<double>(rows)));
  f[1] = static_cast<float>(log2(1.0 + static_cast<double>(cols)));
  f[2] = static_cast<float>(log2(1.0 + z));
  f[3] = static_cast<float>(log2(1.0 + mean));
  f[4] = static_cast<float>(log2(1.0 + static_cast<double>(acc[kMaxLen])));
  f[5] = static_cast<float>(log2(1.0 + cv));
  f[6] = static_cast<float>(static_cast<double>(acc[kMaxDist]) / c);
  f[7] = static_cast<float>(z > 0.0 ? static_cast<double>(acc[kSumDist]) / z / c : 0.0);
  f[8] = static_cast<float>(mn > 0.0 ? static_cast<double>(acc[kDiag]) / mn : 0.0);
  f[9] = static_cast<float>(acc[kSegments] > 0
                                ? z / (8.0 * static_cast<double>(acc[kSegments])) : 0.0);
  f[10] = static_cast<float>(static_cast<double>(acc[kEmpty]) / n);
  f[11] = element_bytes >= 8 ? 1.0f : 0.0f;
}

// ---- MLP -------------------------------------------------------------------
// Parameter layout: W1[64][12] b1[64] W2[64][64] b2[64] W3[V][64] b3[V].
struct Params {
  const float* w1;
  const float* b1;
  const float* w2;
  const float* b2;
  const float* w3;
  const float* b3;
};

__host__ __device__ inline int64_t param_count(int v) {
  return int64_t{kHidden} * kIn + kHidden + int64_t{kHidden} * kHidden + kHidden +
         int64_t{v} * kHidden + v;
}

__host__ __device__ inline Params split(const float* p, int v) {
  Params q;
  q.w1 = p;
  q.b1 = q.w1 + kHidden * kIn;
  q.w2 = q.b1 + kHidden;
  q.b2 = q.w2 + kHidden * kHidden;
  q.w3 = q.b2 + kHidden;
  q.b3 = q.w3 + v * kHidden;
  return q;
}

// out[s][u] = act(b[u] + sum_k w[u][k] in[s][k]), one thread per (s, u).
__global__ void dense_forward(const float* __restrict__ in, int n_in, const float* __restrict__ w,
                              const float* __restrict__ b, int n_out, int64_t batch, int relu,
                              float* __restrict__ out) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= batch * n_out) return;
  const int64_t s = t / n_out;
  const int u = static_cast<int>(t - s * n_out);
  float acc = b[u];
  for (int k = 0; k < n_in; ++k) acc = fmaf(w[u * n_in + k], in[s * n_in + k], acc);
  out[t] = relu && acc < 0.0f ? 0.0f : acc;
}

// dy[s][v] = 2 (y - target) / (batch * V); loss[s] = sum_v (y - target)^2 / V.
__global__ void mse_grad(const float* __restrict__ y, const float* __restrict__ target,
                         int n_out, int64_t batch, float* __restrict__ dy,
                         float* __restrict__ loss) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= batch) return;
  float l = 0.0f;
  for (int v = 0; v < n_out; ++v) {
    const float d = y[s * n_out + v] - target[s * n_out + v];
    l = fmaf(d, d, l);
    dy[s * n_out + v] = 2.0f * d / static_cast<float>(batch * n_out);
  }
  if (loss != nullptr) loss[s] = l / static_cast<float>(n_out);
}

// din[s][k] = relu'(act[s][k]) * sum_u dout[s][u] w[u][k], where act is the
// layer input's post-activation value (no mask when act is null).
__global__ void dense_backward_input(const float* __restrict__ dout, int n_out,
                                     const float* __restrict__ w, int n_in,
                                     const float* __restrict__ act, int64_t batch,
                                     float* __restrict__ din) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= batch * n_in) return;
  const int64_t s = t / n_in;
  const int k = static_cast<int>(t - s * n_in);
  float acc = 0.0f;
  for (int u = 0; u < n_out; ++u) acc = fmaf(dout[s * n_out + u], w[u * n_in + k], acc);
  din[t] = (act != nullptr && act[t] <= 0.0f) ? 0.0f : acc;
}

// gw[u][k] = sum_s dout[s][u] in[s][k]; gb[u] = sum_s dout[s][u].  One thread
// per weight (and per bias), samples in order.
__global__ void dense_weight_grad(const float* __restrict__ dout, int n_out,
                                  const float* __restrict__ in, int n_in, int64_t batch,
                                  float* __restrict__ gw, float* __restrict__ gb) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nw = static_cast<int64_t>(n_out) * n_in;
  if (t < nw) {
    const int u = static_cast<int>(t / n_in);
    const int k = static_cast<int>(t - static_cast<int64_t>(u) * n_in);
    float acc = 0.0f;
    for (int64_t s = 0; s < batch; ++s) acc = fmaf(dout[s * n_out + u], in[s * n_in + k], acc);
    gw[t] = acc;
  } else if (t < nw + n_out) {
    const int u = static_cast<int>(t - nw);
    float acc = 0.0f;
    for (int64_t s = 0; s < batch; ++s) acc += dout[s * n_out + u];
    gb[u] = acc;
  }
}

__global__ void adam_update(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, int64_t n, float lr,
                            float beta1, float beta2, float eps, float c1, float c2) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
  const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// index of the smallest of y[0..n) (first on ties)
__global__ void argmin_kernel(const float* __restrict__ y, int n, int* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int best = 0;
  for (int i = 1; i < n; ++i) {
    if (y[i] < y[best]) best = i;
  }
  *out = best;
}

unsigned Blocks(int64_t n, int threads) {
  const int64_t b = (n + threads - 1) / threads;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

}  // namespace
}  // namespace ascb

extern "C" int64_t ascb_mlp_param_count(int n_variants) { return ascb::param_count(n_variants); }

extern "C" int ascb_matrix_features(void* stream, const ascb_csr* a, int element_bytes,
                                    unsigned long long* acc, float* features, int sm_count) {
  auto s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(acc, 0, 8 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (a->rows > 0) {
    int64_t blocks = (a->rows * 32 + 255) / 256;
    const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
    if (blocks > cap) blocks = cap;
    ascb::features_accumulate<<<static_cast<unsigned>(blocks), 256, 0, s>>>(a->ptr, a->idx,
                                                                           a->rows, acc);
  }
  ascb::selector_finalize<<<1, 32, 0, s>>>(acc, a->rows, a->cols, a->nnz, element_bytes,
                                           features);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_mlp_forward(void* stream, int n_variants, const float* params,
                                const float* x, int64_t batch, float* hidden, float* y) {
  using namespace ascb;
  auto s = static_cast<cudaStream_t>(stream);
  if (batch <= 0) return 0;
  const Params p = split(params, n_variants);
  float* h1 = hidden;
  float* h2 = hidden + batch * kHidden;
  dense_forward<<<Blocks(batch * kHidden, 256), 256, 0, s>>>(x, kIn, p.w1, p.b1, kHidden, batch,
                                                             1, h1);
  dense_forward<<<Blocks(batch * kHidden, 256), 256, 0, s>>>(h1, kHidden, p.w2, p.b2, kHidden,
                                                             batch, 1, h2);
  dense_forward<<<Blocks(batch * n_variants, 256), 256, 0, s>>>(h2, kHidden, p.w3, p.b3,
                                                                n_variants, batch, 0, y);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_mlp_backward(void* stream, int n_variants, const float* params,
                                 const float* x, int64_t batch, const float* hidden,
                                 const float* y, const float* target, float* grads,
                                 float* loss, float* scratch) {
  using namespace ascb;
  auto s = static_cast<cudaStream_t>(stream);
  if (batch <= 0) return 0;
  const int V = n_variants;
  const Params p = split(params, V);
  const float* h1 = hidden;
  const float* h2 = hidden + batch * kHidden;
  float* dy = scratch;                 // batch * V
  float* dh2 = dy + batch * V;         // batch * 64
  float* dh1 = dh2 + batch * kHidden;  // batch * 64
  float* gw1 = grads;
  float* gb1 = gw1 + kHidden * kIn;
  float* gw2 = gb1 + kHidden;
  float* gb2 = gw2 + kHidden * kHidden;
  float* gw3 = gb2 + kHidden;
  float* gb3 = gw3 + V * kHidden;
  mse_grad<<<Blocks(batch, 256), 256, 0, s>>>(y, target, V, batch, dy, loss);
  dense_weight_grad<<<Blocks(int64_t{V} * kHidden + V, 256), 256, 0, s>>>(dy, V, h2, kHidden,
                                                                          batch, gw3, gb3);
  dense_backward_input<<<Blocks(batch * kHidden, 256), 256, 0, s>>>(dy, V, p.w3, kHidden, h2,
                                                                    batch, dh2);
  dense_weight_grad<<<Blocks(int64_t{kHidden} * kHidden + kHidden, 256), 256, 0, s>>>(
      dh2, kHidden, h1, kHidden, batch, gw2, gb2);
  dense_backward_input<<<Blocks(batch * kHidden, 256), 256, 0, s>>>(dh2, kHidden, p.w2, kHidden,
                                                                    h1, batch, dh1);
  dense_weight_grad<<<Blocks(int64_t{kHidden} * kIn + kHidden, 256), 256, 0, s>>>(
      dh1, kHidden, x, kIn, batch, gw1, gb1);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_adam_step(void* stream, float* params, const float* grads, float* m, float* v,
                              int64_t n, float lr, float beta1, float beta2, float eps,
                              int step) {
  if (n <= 0) return 0;
  const float c1 = 1.0f - powf(beta1, static_cast<float>(step));
  const float c2 = 1.0f - powf(beta2, static_cast<float>(step));
  ascb::adam_update<<<ascb::Blocks(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grads, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_argmin(void* stream, const float* y, int n, int* out) {
  ascb::argmin_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(y, n, out);
  return static_cast<int>(cudaGetLastError());
}
