// Learned absorbing boundary: a small MLP that predicts the tangential E of
// every outer-wall cell at step n+1 from a 3-cell-deep stencil (the wall
// plane and the two planes inside it) at steps n-1, n and n+1, replacing a
// CPML layer.  No counterpart in the reference.
//
// Network (the same one for every face and component, in the face's local
// frame, s = the inward direction along the face normal):
//   features f0..f7 = E(w, n), E(w+s, n), E(w+2s, n), E(w+s, n+1),
//                     E(w+2s, n+1), E(w, n-1), E(w+s, n-1),
//                     transverse 4-neighbour Laplacian of E(w+s, n)
//   scale   = max |f0..f6| (the features and the target are divided by it,
//             so the operator is homogeneous of degree one)
//   h1 = tanh(W1 x + b1)   (64),  h2 = tanh(W2 h1 + b2)  (64),
//   y  = w3 . h2 + b3
//   E(w, n+1) = scale * (x1 + k (x3 - x0) + y)
// The network learns the residual of the first-order Mur boundary
// E(w, n+1) = E(w+s, n) + k (E(w+s, n+1) - E(w, n)), k = (c dt - d)/(c dt + d)
// for the cell size d along the face normal (Mur, IEEE Trans. EMC 23, 1981),
// which keeps the closed loop anchored to a stable operator; with all
// weights zero the boundary is exactly that Mur boundary.
// Weights are stored in BF16 and every product is accumulated in FP32.
#pragma once

#include <cuda_bf16.h>

#include "kernels.cuh"

namespace xfb {

constexpr int kMlpIn = 8, kMlpHid = 64;
// parameter layout: W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpHid * kMlpIn, kMlpW2 = kMlpB1 + kMlpHid,
              kMlpB2 = kMlpW2 + kMlpHid * kMlpHid, kMlpW3 = kMlpB2 + kMlpHid, kMlpB3 = kMlpW3 + kMlpHid,
              kMlpParams = kMlpB3 + 1;

// y = MLP(x) with the weights in shared memory (already widened to float).
// (h1 stays in registers: both loops over it are fully unrolled)
__device__ __forceinline__ float mlp_forward(const float* w, const float x[kMlpIn]) {
  float h1[kMlpHid];
#pragma unroll
  for (int j = 0; j < kMlpHid; ++j) {
    float a = w[kMlpB1 + j];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) a = fmaf(w[kMlpW1 + j * kMlpIn + k], x[k], a);
    h1[j] = tanhf(a);
  }
  float y = w[kMlpB3];
  for (int j = 0; j < kMlpHid; ++j) {
    float a = w[kMlpB2 + j];
#pragma unroll
    for (int k = 0; k < kMlpHid; ++k) a = fmaf(w[kMlpW2 + j * kMlpHid + k], h1[k], a);
    y = fmaf(w[kMlpW3 + j], tanhf(a), y);
  }
  return y;
}

// Geometry of the learned boundary: for face f (XN..ZP) the tangential
// components a = (c+1)%3, b = (c+2)%3 of the normal axis c, in an [n0 x n1]
// grid of wall cells (n0 cells along the component's own axis, n1 interior
// nodes along the other tangential axis: the box's edges stay PEC, so no
// cell a thread reads inward is another face's wall cell).  History planes
// E(w, n-1) and E(w+s, n-1) per face and component.
struct LabcP {
  const __nv_bfloat16* w;  // kMlpParams BF16 weights
  float* hist;             // per (face, comp): [2][n0][n1]
  long long hist_off[6][2];
  int n0[6][2], n1[6][2];  // extents of the wall cells of each (face, comp)
  long long off[13];       // prefix sums of cells over (face, comp), launch indexing
  float mur_k[3];          // first-order Mur coefficient per normal axis
};

// Wall cells of every face and tangential component of an nx x ny x nz box
// (edges left out) and the layout of their history planes.
inline LabcP labc_layout(int nx, int ny, int nz) {
  LabcP p{};
  const int n[3] = {nx, ny, nz};
  long long off = 0, hoff = 0;
  for (int f = 0; f < 6; ++f) {
    const int c = f / 2, a = (c + 1) % 3, b = (c + 2) % 3;
    for (int w = 0; w < 2; ++w) {
      const int comp = w == 0 ? a : b, other = w == 0 ? b : a;
      p.n0[f][w] = n[comp];
      p.n1[f][w] = n[other] > 1 ? n[other] - 1 : 0;
      p.off[2 * f + w] = off;
      p.hist_off[f][w] = hoff;
      const long long cells = static_cast<long long>(p.n0[f][w]) * p.n1[f][w];
      off += cells;
      hoff += 2 * cells;
    }
  }
  p.off[12] = off;
  return p;
}

template <typename T>
__device__ __forceinline__ T* comp_ptr(const GridP<T>& g, int comp) {
  return comp == 0 ? g.ex : comp == 1 ? g.ey : g.ez;
}

// One thread per wall cell of every face and tangential component.  Reads
// E^n from `s` (the set the step read) and E^{n+1} of the interior from `d`,
// writes E^{n+1} of the wall cell to `d` and rolls the history planes.
template <typename T>
__global__ void k_labc_apply(GridP<T> s, GridP<T> d, LabcP lp) {
  __shared__ float w[kMlpParams];
  for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x) w[q] = __bfloat162float(lp.w[q]);
  __syncthreads();
  const long long gid = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (gid >= lp.off[12]) return;
  int fc = 0;
  while (gid >= lp.off[fc + 1]) ++fc;
  const int face = fc >> 1, which = fc & 1;
  const long long r = gid - lp.off[fc];
  const int n1 = lp.n1[face][which];
  const int u = static_cast<int>(r / n1), v = static_cast<int>(r % n1);
  const int c = face >> 1, side = face & 1;
  const int a = (c + 1) % 3, b = (c + 2) % 3;
  const int comp = which == 0 ? a : b, other = which == 0 ? b : a;
  auto stride = [&](int ax) { return ax == 0 ? s.sx : ax == 1 ? s.sy : 1LL; };
  auto extent = [&](int ax) { return ax == 0 ? s.nx : ax == 1 ? s.ny : s.nz; };
  // the wall node along c, cell u along the component's own axis, node v+1
  // along the other tangential axis
  const long long sn = side ? -stride(c) : stride(c);  // inward step
  const long long sc_ = stride(comp), so = stride(other);
  const long long idx = (side ? extent(c) : 0) * stride(c) + u * sc_ + (v + 1) * so;
  const T* e_old = comp_ptr(s, comp);
  T* e_new = comp_ptr(d, comp);
  float* h0 = lp.hist + lp.hist_off[face][which];
  float* h1p = h0 + static_cast<long long>(lp.n0[face][which]) * n1;
  const long long hi = r;
  // transverse Laplacian of E(w+s, n), neighbours clamped at the face's edges
  const long long p1 = idx + sn;
  const int ncomp = extent(comp);
  const float e1 = static_cast<float>(e_old[p1]);
  const float lap = static_cast<float>(e_old[p1 + (u + 1 < ncomp ? sc_ : 0)]) +
                    static_cast<float>(e_old[p1 - (u > 0 ? sc_ : 0)]) + static_cast<float>(e_old[p1 + so]) +
                    static_cast<float>(e_old[p1 - so]) - 4.0f * e1;
  float f[kMlpIn];
  f[0] = static_cast<float>(e_old[idx]);
  f[1] = e1;
  f[2] = static_cast<float>(e_old[idx + 2 * sn]);
  f[3] = static_cast<float>(e_new[idx + sn]);
  f[4] = static_cast<float>(e_new[idx + 2 * sn]);
  f[5] = h0[hi];
  f[6] = h1p[hi];
  f[7] = lap;
  float scale = 0.0f;
#pragma unroll
  for (int q = 0; q < 7; ++q) scale = fmaxf(scale, fabsf(f[q]));
  // Mur estimate in field units; the network's correction only where the
  // stencil's scale is a normal number (1/scale stays finite)
  float out = f[1] + lp.mur_k[c] * (f[3] - f[0]);
  if (scale > 1e-30f) {
    const float inv = 1.0f / scale;
#pragma unroll
    for (int q = 0; q < kMlpIn; ++q) f[q] *= inv;
    out = fmaf(scale, mlp_forward(w, f), out);
  }
  h0[hi] = static_cast<float>(e_old[idx]);
  h1p[hi] = e1;
  e_new[idx] = static_cast<T>(out);
}

}  // namespace xfb
