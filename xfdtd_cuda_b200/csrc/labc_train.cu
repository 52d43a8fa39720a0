// Training of the learned absorbing boundary's MLP on the device (see
// labc.cuh for the network).  Hand-written kernels: a fused forward and
// backward pass over chunks of samples (activations in shared memory; every
// block walks a fixed set of chunks and keeps its weight gradients in
// registers), a reduction of the per-block gradients in block order (so a
// training run is reproducible bit for bit), BF16 rounding of the FP32 master
// weights for the forward pass, and Adam.
// No counterpart in the reference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/xfdtd_b200.h"
#include "labc.cuh"

namespace xfb {
namespace {

constexpr int kChunk = 32;     // samples per chunk
constexpr int kThreads = 256;
constexpr int kGradBlocks = 4 * 148;  // blocks of the gradient pass (at most)
constexpr int kPerThread = (kMlpParams + kThreads - 1) / kThreads;  // gradient slots per thread

// Blocks of the gradient pass for n samples (a function of n only, so the
// summation order is fixed).
inline int grad_blocks(int n) {
  const int chunks = (n + kChunk - 1) / kChunk;
  return chunks < kGradBlocks ? chunks : kGradBlocks;
}

thread_local std::string g_mlp_err;

int mlp_fail(int code, const std::string& m) {
  g_mlp_err = m;
  return code;
}

// Master FP32 weights -> the BF16 values the forward pass uses (widened back
// to float so the kernels read one type).
__global__ void k_round_bf16(const float* w, float* wq, int n) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) wq[q] = __bfloat162float(__float2bfloat16_rn(w[q]));
}

// Loss (sum of squared errors / n) and gradient over the chunks blockIdx.x,
// blockIdx.x + gridDim.x, ... of the samples: per block into lpart[block] and
// gpart[block][kMlpParams] (gradients w.r.t. the rounded weights, used for
// the master weights: straight-through rounding).
__global__ void __launch_bounds__(kThreads) k_mlp_grad(const float* wq, const float* x, const float* y, int n,
                                                       double* lpart, float* gpart) {
  extern __shared__ float sm[];
  float* w = sm;                            // kMlpParams
  float* xs = w + kMlpParams;               // [kChunk][8]
  float* h1 = xs + kChunk * kMlpIn;         // [kChunk][64]
  float* h2 = h1 + kChunk * kMlpHid;        // [kChunk][64]
  float* d2 = h2 + kChunk * kMlpHid;        // [kChunk][64] dL/dz2
  float* d1 = d2 + kChunk * kMlpHid;        // [kChunk][64] dL/dz1
  float* dy = d1 + kChunk * kMlpHid;        // [kChunk]
  const int tid = threadIdx.x;
  const int chunks = (n + kChunk - 1) / kChunk;
  for (int q = tid; q < kMlpParams; q += kThreads) w[q] = wq[q];
  float acc[kPerThread];
#pragma unroll
  for (int r = 0; r < kPerThread; ++r) acc[r] = 0.f;
  double loss = 0.0;  // thread 0
  for (int ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    const int s0 = ch * kChunk;
    const int ns = min(kChunk, n - s0);
    __syncthreads();  // the previous chunk's last reads are done
    for (int q = tid; q < kChunk * kMlpIn; q += kThreads)
      xs[q] = q / kMlpIn < ns ? x[static_cast<long long>(s0) * kMlpIn + q] : 0.f;
    __syncthreads();
    // layer 1
    for (int q = tid; q < kChunk * kMlpHid; q += kThreads) {
      const int sm_ = q / kMlpHid, j = q % kMlpHid;
      float a = w[kMlpB1 + j];
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) a = fmaf(w[kMlpW1 + j * kMlpIn + k], xs[sm_ * kMlpIn + k], a);
      h1[q] = tanhf(a);
    }
    __syncthreads();
    // layer 2
    for (int q = tid; q < kChunk * kMlpHid; q += kThreads) {
      const int sm_ = q / kMlpHid, j = q % kMlpHid;
      float a = w[kMlpB2 + j];
      for (int k = 0; k < kMlpHid; ++k) a = fmaf(w[kMlpW2 + j * kMlpHid + k], h1[sm_ * kMlpHid + k], a);
      h2[q] = tanhf(a);
    }
    __syncthreads();
    // output and loss; dL/dy = 2 (y - t) / n
    if (tid < kChunk) {
      float e = 0.f;
      if (tid < ns) {
        float o = w[kMlpB3];
        for (int j = 0; j < kMlpHid; ++j) o = fmaf(w[kMlpW3 + j], h2[tid * kMlpHid + j], o);
        e = o - y[s0 + tid];
      }
      dy[tid] = 2.f * e / static_cast<float>(n);
      double se = static_cast<double>(e) * e;
      for (int o = 16; o > 0; o >>= 1) se += __shfl_down_sync(0xffffffffu, se, o);
      if (tid == 0) loss += se / n;
    }
    __syncthreads();
    // dL/dz2 = dy * w3 * (1 - h2^2)
    for (int q = tid; q < kChunk * kMlpHid; q += kThreads) {
      const int sm_ = q / kMlpHid, j = q % kMlpHid;
      const float t = h2[q];
      d2[q] = dy[sm_] * w[kMlpW3 + j] * (1.f - t * t);
    }
    __syncthreads();
    // dL/dz1 = (W2^T d2) * (1 - h1^2)
    for (int q = tid; q < kChunk * kMlpHid; q += kThreads) {
      const int sm_ = q / kMlpHid, k = q % kMlpHid;
      float a = 0.f;
      for (int j = 0; j < kMlpHid; ++j) a = fmaf(w[kMlpW2 + j * kMlpHid + k], d2[sm_ * kMlpHid + j], a);
      const float t = h1[q];
      d1[q] = a * (1.f - t * t);
    }
    __syncthreads();
    // weight gradients of this chunk, parameters tid, tid + kThreads, ...
#pragma unroll
    for (int r = 0; r < kPerThread; ++r) {
      const int p = tid + r * kThreads;
      if (p >= kMlpParams) break;
      float g = 0.f;
      if (p < kMlpB1) {                       // W1[j][k]
        const int j = p / kMlpIn, k = p % kMlpIn;
        for (int q = 0; q < ns; ++q) g = fmaf(d1[q * kMlpHid + j], xs[q * kMlpIn + k], g);
      } else if (p < kMlpW2) {                // b1[j]
        const int j = p - kMlpB1;
        for (int q = 0; q < ns; ++q) g += d1[q * kMlpHid + j];
      } else if (p < kMlpB2) {                // W2[j][k]
        const int j = (p - kMlpW2) / kMlpHid, k = (p - kMlpW2) % kMlpHid;
        for (int q = 0; q < ns; ++q) g = fmaf(d2[q * kMlpHid + j], h1[q * kMlpHid + k], g);
      } else if (p < kMlpW3) {                // b2[j]
        const int j = p - kMlpB2;
        for (int q = 0; q < ns; ++q) g += d2[q * kMlpHid + j];
      } else if (p < kMlpB3) {                // w3[j]
        const int j = p - kMlpW3;
        for (int q = 0; q < ns; ++q) g = fmaf(dy[q], h2[q * kMlpHid + j], g);
      } else {                                // b3
        for (int q = 0; q < ns; ++q) g += dy[q];
      }
      acc[r] += g;
    }
  }
#pragma unroll
  for (int r = 0; r < kPerThread; ++r) {
    const int p = tid + r * kThreads;
    if (p < kMlpParams) gpart[static_cast<long long>(blockIdx.x) * kMlpParams + p] = acc[r];
  }
  if (tid == 0) lpart[blockIdx.x] = loss;
}

// Sum of the per-block parts in block order: grad[p] and, for the thread
// with p == kMlpParams, the loss.
__global__ void k_mlp_reduce(const double* lpart, const float* gpart, int blocks, double* loss, float* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) {
    float g = 0.f;
    for (int b = 0; b < blocks; ++b) g += gpart[static_cast<long long>(b) * kMlpParams + p];
    grad[p] = g;
  } else if (p == kMlpParams) {
    double l = 0.0;
    for (int b = 0; b < blocks; ++b) l += lpart[b];
    *loss = l;
  }
}

__global__ void k_adam(float* w, float* m, float* v, const float* g, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float gq = g[q];
  const float mq = b1 * m[q] + (1.f - b1) * gq;
  const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  w[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

constexpr size_t kGradSmem =
    (kMlpParams + kChunk * kMlpIn + 4 * kChunk * kMlpHid + kChunk) * sizeof(float);

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
};

#define MLP_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) return mlp_fail(XFB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int upload_samples(const float* x, const float* y, int n, DevBuf& dx, DevBuf& dy) {
  MLP_CUDA(cudaMalloc(&dx.p, static_cast<size_t>(n) * kMlpIn * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dy.p, static_cast<size_t>(n) * sizeof(float)));
  MLP_CUDA(cudaMemcpy(dx.p, x, static_cast<size_t>(n) * kMlpIn * sizeof(float), cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemcpy(dy.p, y, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice));
  return XFB_OK;
}

// Per-block partial sums of the gradient pass for n samples.
struct GradParts {
  DevBuf l, g;
  int blocks = 0;
};

int alloc_parts(int n, GradParts& gp) {
  gp.blocks = grad_blocks(n);
  MLP_CUDA(cudaMalloc(&gp.l.p, static_cast<size_t>(gp.blocks) * sizeof(double)));
  MLP_CUDA(cudaMalloc(&gp.g.p, static_cast<size_t>(gp.blocks) * kMlpParams * sizeof(float)));
  return XFB_OK;
}

int launch_grad(const float* wq, const float* x, const float* y, int n, GradParts& gp, double* loss, float* grad) {
  static bool attr = false;
  if (!attr) {
    MLP_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kGradSmem)));
    attr = true;
  }
  double* lp = static_cast<double*>(gp.l.p);
  float* gq = static_cast<float*>(gp.g.p);
  k_mlp_grad<<<gp.blocks, kThreads, kGradSmem>>>(wq, x, y, n, lp, gq);
  k_mlp_reduce<<<(kMlpParams + 1 + 255) / 256, 256>>>(lp, gq, gp.blocks, loss, grad);
  MLP_CUDA(cudaGetLastError());
  return XFB_OK;
}

}  // namespace
}  // namespace xfb

using namespace xfb;

extern "C" {

int xfb_mlp_param_count(void) { return kMlpParams; }

const char* xfb_mlp_last_error(void) { return g_mlp_err.c_str(); }

int xfb_mlp_loss_grad(const float* x, const float* y, int n, const float* w, double* loss, float* grad) {
  if (!x || !y || !w || !loss || !grad || n <= 0) return mlp_fail(XFB_ERR_INVALID, "null argument or n <= 0");
  DevBuf dx, dy, dw, dwq, dl, dg;
  GradParts gp;
  int rc;
  if ((rc = upload_samples(x, y, n, dx, dy))) return rc;
  if ((rc = alloc_parts(n, gp))) return rc;
  MLP_CUDA(cudaMalloc(&dw.p, kMlpParams * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dwq.p, kMlpParams * sizeof(float)));
  MLP_CUDA(cudaMalloc(&dl.p, sizeof(double)));
  MLP_CUDA(cudaMalloc(&dg.p, kMlpParams * sizeof(float)));
  MLP_CUDA(cudaMemcpy(dw.p, w, kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
  k_round_bf16<<<(kMlpParams + 255) / 256, 256>>>(static_cast<float*>(dw.p), static_cast<float*>(dwq.p), kMlpParams);
  if ((rc = launch_grad(static_cast<float*>(dwq.p), static_cast<float*>(dx.p), static_cast<float*>(dy.p), n, gp,
                        static_cast<double*>(dl.p), static_cast<float*>(dg.p))))
    return rc;
  MLP_CUDA(cudaMemcpy(loss, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
  MLP_CUDA(cudaMemcpy(grad, dg.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
  return XFB_OK;
}

int xfb_mlp_train(const float* x, const float* y, int n, int iters, float lr, const float* w_init, float* w_out,
                  double* loss_curve) {
  if (!x || !y || !w_init || !w_out || n <= 0 || iters < 0) return mlp_fail(XFB_ERR_INVALID, "null argument or bad size");
  DevBuf dx, dy, dw, dwq, dm, dv, dl, dg;
  GradParts gp;
  int rc;
  if ((rc = upload_samples(x, y, n, dx, dy))) return rc;
  if ((rc = alloc_parts(n, gp))) return rc;
  const size_t wb = kMlpParams * sizeof(float);
  MLP_CUDA(cudaMalloc(&dw.p, wb));
  MLP_CUDA(cudaMalloc(&dwq.p, wb));
  MLP_CUDA(cudaMalloc(&dm.p, wb));
  MLP_CUDA(cudaMalloc(&dv.p, wb));
  MLP_CUDA(cudaMalloc(&dg.p, wb));
  MLP_CUDA(cudaMalloc(&dl.p, sizeof(double)));
  MLP_CUDA(cudaMemcpy(dw.p, w_init, wb, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemset(dm.p, 0, wb));
  MLP_CUDA(cudaMemset(dv.p, 0, wb));
  float* w = static_cast<float*>(dw.p);
  const float b1 = 0.9f, b2 = 0.999f;
  double c1 = 1, c2 = 1;
  for (int it = 0; it < iters; ++it) {
    k_round_bf16<<<(kMlpParams + 255) / 256, 256>>>(w, static_cast<float*>(dwq.p), kMlpParams);
    if ((rc = launch_grad(static_cast<float*>(dwq.p), static_cast<float*>(dx.p), static_cast<float*>(dy.p), n, gp,
                          static_cast<double*>(dl.p), static_cast<float*>(dg.p))))
      return rc;
    c1 *= b1;
    c2 *= b2;
    k_adam<<<(kMlpParams + 255) / 256, 256>>>(w, static_cast<float*>(dm.p), static_cast<float*>(dv.p),
                                             static_cast<float*>(dg.p), kMlpParams, lr, b1, b2, 1e-8f,
                                             static_cast<float>(1 - c1), static_cast<float>(1 - c2));
    if (loss_curve) MLP_CUDA(cudaMemcpy(&loss_curve[it], dl.p, sizeof(double), cudaMemcpyDeviceToHost));
  }
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaMemcpy(w_out, w, wb, cudaMemcpyDeviceToHost));
  return XFB_OK;
}

}  // extern "C"
