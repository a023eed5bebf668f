// proposal.cu -- where refs-mode insertions go.  No reference counterpart:
// erdst places the test particle's centre of mass uniformly in the cell
// (insertion.F90:152-162).  The learned proposal keeps that as a component
// and as the yardstick: the cell is cut into G^3 voxels of fractional size 1/G,
//
//   q_v = eps / V + (1 - eps) * softmax(s)_v,   V = G^3,
//
// where s_v is the network's logit for voxel v from its local solvent
// density.  An insertion picks voxel v with probability q_v and a uniform
// point inside it, and carries the importance weight p/q = (1/V) / q_v into
// every histogram and ecorr increment, so the accumulated distributions
// estimate the uniform-insertion ones without bias (eps > 0 keeps q > 0).
//
//   k_density    solvent molecules' first sites on an F^3 fractional grid
//                (F feature cells per side), integer atomics (order-independent)
//   k_features   per voxel, the 4x4x4 feature cells centred on it, standardised
//                as Poisson counts, (n - <n>) / sqrt(<n>): the network's 64 inputs
//   k_prop_cdf   one block: softmax, mixture and CDF over the voxels in FP64,
//                fixed-order block scan
#include <cuda_bf16.h>

#include <cmath>

#include "engine.cuh"

namespace erm {

__global__ void k_density(FrameArgs a, int gf, const float* __restrict__ posraw, const int* __restrict__ molbeg,
                          int* __restrict__ dens) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.slvmax) return;
  const int at = molbeg[k];
  const float x = posraw[3 * at], y = posraw[3 * at + 1], z = posraw[3 * at + 2];
  int c[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    float f = a.g.invcl[m][0] * x + a.g.invcl[m][1] * y + a.g.invcl[m][2] * z;
    f -= floorf(f);
    int i = (int)(f * (float)gf);
    c[m] = i >= gf ? gf - 1 : (i < 0 ? 0 : i);
  }
  atomicAdd(&dens[(c[2] * gf + c[1]) * gf + c[0]], 1);
}

__global__ void k_features(int gv, int gf, float mean, float inv_sd, const int* __restrict__ dens,
                           float* __restrict__ feat) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int V = gv * gv * gv;
  if (idx >= V * kMlpIn) return;
  const int v = idx / kMlpIn, t = idx - v * kMlpIn;
  const int vx = v % gv, vy = (v / gv) % gv, vz = v / (gv * gv);
  const int dx = t & 3, dy = (t >> 2) & 3, dz = t >> 4;
  auto wrap = [gf](int i) { return (i % gf + gf) % gf; };
  // first of the 4 cells nearest to the voxel centre (v + 1/2) gf / gv along each axis
  auto start = [gv, gf](int v) { return (int)floor((double)(2 * v + 1) * gf / (2.0 * gv) - 1.5); };
  const int fx = wrap(start(vx) + dx), fy = wrap(start(vy) + dy), fz = wrap(start(vz) + dz);
  feat[idx] = ((float)dens[(fz * gf + fy) * gf + fx] - mean) * inv_sd;
}

constexpr int kCdfThreads = 1024;

// cdf[v] = sum_{u <= v} q_u (FP64), q[v] = q_v as FP32
__global__ void __launch_bounds__(kCdfThreads) k_prop_cdf(int V, double eps, const float* __restrict__ logit,
                                                          double* __restrict__ cdf, float* __restrict__ q) {
  __shared__ double red[32];
  __shared__ double bmax, bsum;
  const int tid = threadIdx.x;
  const int per = (V + kCdfThreads - 1) / kCdfThreads;
  const int v0 = tid * per, v1 = min(V, v0 + per);
  // max logit
  double mx = -1e300;
  for (int v = v0; v < v1; ++v) mx = fmax(mx, (double)logit[v]);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) red[tid >> 5] = mx;
  __syncthreads();
  if (tid < 32) {
    double m2 = red[tid];
    for (int o = 16; o > 0; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    if (tid == 0) bmax = m2;
  }
  __syncthreads();
  // sum of exp in a fixed order: per thread, then warp, then block
  double loc = 0.0;
  for (int v = v0; v < v1; ++v) loc += exp((double)logit[v] - bmax);
  double ws = warp_sum(loc);
  if ((tid & 31) == 0) red[tid >> 5] = ws;
  __syncthreads();
  if (tid < 32) {
    const double s2 = warp_sum(red[tid]);
    if (tid == 0) bsum = s2;
  }
  __syncthreads();
  // q and the inclusive prefix sum over threads (warp scan, then scan of warp totals)
  const double inv = 1.0 / bsum, mixu = eps / (double)V;
  double run = 0.0;
  for (int v = v0; v < v1; ++v) run += mixu + (1.0 - eps) * exp((double)logit[v] - bmax) * inv;
  double incl = run;
  const int lane = tid & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  __syncthreads();
  if (lane == 31) red[tid >> 5] = incl;
  __syncthreads();
  if (tid < 32) {
    double w = red[tid], wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, wi, o);
      if (tid >= o) wi += y;
    }
    red[tid] = wi - w;   // exclusive prefix of the warp totals
  }
  __syncthreads();
  double acc = red[tid >> 5] + (incl - run);
  for (int v = v0; v < v1; ++v) {
    const double qv = mixu + (1.0 - eps) * exp((double)logit[v] - bmax) * inv;
    acc += qv;
    cdf[v] = acc;
    q[v] = (float)qv;
  }
}

// per insertion, the features of its voxel (training data)
__global__ void k_gather_ins_features(int n, const int* __restrict__ vox, const float* __restrict__ feat,
                                      float* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * kMlpIn) return;
  const int i = idx / kMlpIn, t = idx - i * kMlpIn;
  out[idx] = feat[(size_t)vox[i] * kMlpIn + t];
}

int launch_proposal(const FrameArgs& a, const DeviceState& d, int gv, int gf, float eps, bool learned,
                    cudaStream_t s) {
  const int V = gv * gv * gv;
  if (cudaMemsetAsync(d.dens, 0, sizeof(int) * (size_t)gf * gf * gf, s) != cudaSuccess) return -1;
  int nl = 0;
  if (a.slvmax > 0) {
    k_density<<<(a.slvmax + 255) / 256, 256, 0, s>>>(a, gf, d.posraw, d.molbeg, d.dens);
    ++nl;
  }
  // counts standardised as Poisson variables: (n - <n>) / sqrt(<n>)
  const double mean = (double)a.slvmax / ((double)gf * gf * gf);
  const float inv_sd = mean > 0.0 ? (float)(1.0 / std::sqrt(mean)) : 0.f;
  k_features<<<(V * kMlpIn + 255) / 256, 256, 0, s>>>(gv, gf, (float)mean, inv_sd, d.dens, d.feat);
  ++nl;
  if (learned) {
    mlp_forward(d.mlp_b, d.mlp_f, d.feat, V, nullptr, d.vlogit, &d.status->flags, s);
    k_prop_cdf<<<1, kCdfThreads, 0, s>>>(V, (double)eps, d.vlogit, d.vcdf, d.vq);
    nl += mlp_forward_launches() + 1;
  }
  return nl;
}

void launch_gather_ins_features(const DeviceState& d, int n, float* out, cudaStream_t s) {
  k_gather_ins_features<<<(n * kMlpIn + 255) / 256, 256, 0, s>>>(n, d.ins_voxel, d.feat, out);
}

}  // namespace erm
