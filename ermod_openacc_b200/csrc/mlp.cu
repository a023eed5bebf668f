// mlp.cu -- the learned insertion proposal's network: a 64-128-128-128-1
// multilayer perceptron over a voxel's 4x4x4 local solvent-density grid,
// BF16 weights with FP32 accumulation, trained on the device by the kernels
// below (no library GEMM, no autograd).  No reference counterpart: erdst
// inserts uniformly (insertion.F90:152-162); the proposal only changes where
// insertions go and carries the importance weight p/q that keeps every
// histogram and ecorr increment unbiased.
//
//   forward   h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), h3 = relu(W3 h2 + b3),
//             s = w4 . h3 + b4                      (the voxel's logit)
//   loss      mean binary cross-entropy with logits, softplus(s) - y s
//   backward  the chain rule through the same BF16 weights; every gradient
//             element is one thread's fixed-order sum over the batch, so the
//             gradients are bitwise reproducible
//   update    Adam on FP32 master weights, rounded to BF16 for the next pass
//
// Parameter vector layout (FP32, ERMOD_MLP_NPARAMS entries):
//   W1[128][64] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] w4[128] b4
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"
#include "tc_sm100.cuh"

namespace erm {

namespace {

constexpr int kTile = 64, kTileK = 16, kGemmThreads = 256;

template <class T>
__device__ __forceinline__ float ldf(const T* p) { return (float)*p; }
template <>
__device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]) (relu) (* [R[m][n] > 0]), FP32 accumulation in k order.
// A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn], C row-major with row stride ldc.
template <class TA, class TB>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(int M, int N, int K, const TA* __restrict__ A, int sam, int sak,
    const TB* __restrict__ B, int sbk, int sbn, float* __restrict__ C, int ldc, const float* __restrict__ bias,
    int relu, const float* __restrict__ R, int ldr) {
  __shared__ float As[kTileK][kTile + 1];
  __shared__ float Bs[kTileK][kTile + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kTileK) {
    for (int x = threadIdx.x; x < kTileK * kTile; x += kGemmThreads) {
      const int kk = x / kTile, r = x - kk * kTile;
      const int m = m0 + r, n = n0 + r, k = k0 + kk;
      As[kk][r] = (m < M && k < K) ? ldf(A + (size_t)m * sam + (size_t)k * sak) : 0.f;
      Bs[kk][r] = (n < N && k < K) ? ldf(B + (size_t)k * sbk + (size_t)n * sbn) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTileK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) { a[i] = As[kk][ty * 4 + i]; b[i] = Bs[kk][tx * 4 + i]; }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j];
      if (bias) v += bias[n];
      if (relu) v = fmaxf(v, 0.f);
      if (R && !(R[(size_t)m * ldr + n] > 0.f)) v = 0.f;
      C[(size_t)m * ldc + n] = v;
    }
  }
}

template <class TA, class TB>
void gemm(int M, int N, int K, const TA* A, int sam, int sak, const TB* B, int sbk, int sbn, float* C, int ldc,
          const float* bias, int relu, const float* R, int ldr, cudaStream_t s) {
  const dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  k_gemm<TA, TB><<<grid, kGemmThreads, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, bias, relu, R, ldr);
}

// column sums of a row-major [n][w] matrix, one thread per column, rows in order
__global__ void k_colsum(int n, int w, const float* __restrict__ X, float* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= w) return;
  float acc = 0.f;
  for (int i = 0; i < n; ++i) acc += X[(size_t)i * w + j];
  out[j] = acc;
}

// dL/ds = (sigmoid(s) - y) / n and the per-sample loss softplus(s) - y s
__global__ void k_bce(int n, const float* __restrict__ s, const float* __restrict__ y, float* __restrict__ g,
                      float* __restrict__ l) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = s[i];
  const float sp = z > 0.f ? z + log1pf(expf(-z)) : log1pf(expf(z));
  const float sig = 1.f / (1.f + expf(-z));
  g[i] = (sig - y[i]) / (float)n;
  l[i] = sp - y[i] * z;
}

__global__ void k_sum_loss(int n, const float* __restrict__ l, double* __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += (double)l[i];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) *out = v / (double)n;
  }
}

__global__ void k_to_bf16(int n, const float* __restrict__ src, __nv_bfloat16* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

__global__ void k_adam(int n, float lr, float b1, float b2, float eps, float c1, float c2, float* __restrict__ w,
                       float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       __nv_bfloat16* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float upd = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] -= upd;
  wb[i] = __float2bfloat16_rn(w[i]);
}

// ---- the forward pass on the tensor cores (tcgen05, kind::tf32) -----------
// One CTA per 128 samples, 128 threads.  The three hidden layers are 128 x 128 x K
// MMAs (K = 64, 128, 128) with the samples on the M side: A = the layer's input
// rows, B = the weight matrix [out][in], both K-major in 128-byte-swizzled shared
// memory (32 TF32 per 128-byte row, one 16 KB atom per 32 of K).  The BF16 weights
// are exact in TF32; the inputs are rounded to TF32 (nearest, ties away) as they
// are staged.  The FP32 accumulator (TMEM, 128 lanes x 128 columns) gets the FP32
// bias and the ReLU in the epilogue, which stores the activation in FP32 (the
// backward pass reads it) and stages it, rounded, as the next layer's A.  The
// output layer is a 128-term FP32 dot product per sample, in column order.  Every
// mbarrier wait has an iteration limit; on expiry the kernel sets *err and skips.
constexpr int kFwdRows = 128;
constexpr int kFwdAtoms = kMlpHidden / 32;            // K atoms of a 128-wide input

struct FwdSmem {
  uint32_t a[kFwdAtoms][kFwdRows * 32];               // layer input, TF32 bits, 4 x 16 KB
  uint32_t b[kFwdAtoms][kMlpHidden * 32];             // weights, TF32 bits, 4 x 16 KB
  uint64_t bar;
  uint32_t tmem_base;
};
constexpr size_t kFwdSmemBytes = sizeof(FwdSmem) + 1024;

// instruction descriptor: kind::tf32, D = F32, A = B = TF32, both K-major, M = 128, N = 128
__host__ __device__ constexpr uint32_t idesc_tf32() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kMlpHidden >> 3) << 17) | ((uint32_t)(kFwdRows >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  const uint32_t idesc = idesc_tf32();
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// element (row, k) of a K-major swizzled operand of `atoms` x 16 KB: 32 TF32 per atom row
__device__ __forceinline__ uint32_t* tf32_slot(uint32_t (*op)[kFwdRows * 32], int row, int k) {
  const int atom = k >> 5, kk = k & 31;
  return (uint32_t*)((unsigned char*)op[atom] + tc::swz(row, kk >> 2)) + (kk & 3);
}

// Operand staging with 16-byte loads, kStageBatch in flight per thread: x rows (FP32, 4 per
// load) and weight rows (BF16, 8 per load) into the swizzled TF32 layout; every group of four
// consecutive k lands in one 16-byte chunk of a row.  Unaligned sources take the scalar loop.
constexpr int kStageBatch = 16;

__device__ __forceinline__ void stage_x(uint32_t (*a)[kFwdRows * 32], const float* __restrict__ x, int r0, int n,
                                        int tid) {
  constexpr int Q = kMlpIn / 4, TOT = kFwdRows * Q;            // float4 per row, per tile
  if (((uintptr_t)x & 15) == 0) {
#pragma unroll 1
    for (int e0 = 0; e0 < TOT; e0 += kStageBatch * kFwdRows) {
      float4 v[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * kFwdRows + tid, row = e / Q;
        v[u] = (e < TOT && r0 + row < n) ? __ldg((const float4*)(x + (size_t)(r0 + row) * kMlpIn) + (e - row * Q))
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * kFwdRows + tid, row = e / Q;
        if (e < TOT)
          *(uint4*)tf32_slot(a, row, (e - row * Q) * 4) =
              make_uint4(to_tf32(v[u].x), to_tf32(v[u].y), to_tf32(v[u].z), to_tf32(v[u].w));
      }
    }
  } else {
    for (int e = tid; e < kFwdRows * kMlpIn; e += kFwdRows) {
      const int row = e / kMlpIn, k = e - row * kMlpIn;
      const float v = (r0 + row < n) ? x[(size_t)(r0 + row) * kMlpIn + k] : 0.f;
      *tf32_slot(a, row, k) = to_tf32(v);
    }
  }
}

template <int K>
__device__ __forceinline__ void stage_w(uint32_t (*b)[kMlpHidden * 32], const __nv_bfloat16* __restrict__ w, int tid) {
  constexpr int Q = K / 8, TOT = kMlpHidden * Q;               // 16-byte groups per row, per matrix
  if (((uintptr_t)w & 15) == 0) {
#pragma unroll 1
    for (int e0 = 0; e0 < TOT; e0 += kStageBatch * kFwdRows) {
      uint4 v[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * kFwdRows + tid;
        v[u] = e < TOT ? __ldg((const uint4*)w + e) : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * kFwdRows + tid, o = e / Q, k = (e - o * Q) * 8;
        if (e < TOT) {
          // a BF16 is the high half of its FP32 (and TF32) pattern
          const uint32_t p[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
          *(uint4*)tf32_slot(b, o, k) = make_uint4(p[0] << 16, p[0] & 0xffff0000u, p[1] << 16, p[1] & 0xffff0000u);
          *(uint4*)tf32_slot(b, o, k + 4) = make_uint4(p[2] << 16, p[2] & 0xffff0000u, p[3] << 16, p[3] & 0xffff0000u);
        }
      }
    }
  } else {
    for (int e = tid; e < kMlpHidden * K; e += kFwdRows) {
      const int o = e / K, k = e - o * K;
      *tf32_slot(b, o, k) = __float_as_uint(__bfloat162float(w[e]));
    }
  }
}

__global__ void __launch_bounds__(kFwdRows, 1) k_mlp_fwd_tc(const __nv_bfloat16* __restrict__ pw,
    const float* __restrict__ pf, const float* __restrict__ x, int n, float* __restrict__ act,
    float* __restrict__ logits, int* __restrict__ err, MlpLayout L) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char fsm_raw[];
  FwdSmem& S = *reinterpret_cast<FwdSmem*>((void*)(((uintptr_t)fsm_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.x * kFwdRows;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(kMlpHidden));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&S.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // layer 1 input: x rows, rounded to TF32 (rows past n are zero)
  stage_x(S.a, x, r0, n, tid);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  bool ok = true;
  const int row = r0 + warp * 32 + lane;              // this thread's sample (TMEM lane)
  float out = 0.f;
  const int woff[3] = {L.w1, L.w2, L.w3}, boff[3] = {L.b1, L.b2, L.b3}, kin[3] = {kMlpIn, kMlpHidden, kMlpHidden};
  for (int layer = 0; layer < 3; ++layer) {
    const int K = kin[layer];
    // weights [out][K] (BF16, exact in TF32) as the B operand
    if (K == kMlpIn) stage_w<kMlpIn>(S.b, pw + woff[layer], tid);
    else stage_w<kMlpHidden>(S.b, pw + woff[layer], tid);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      for (int atom = 0; atom < K / 32; ++atom) {
        const uint64_t da = smem_desc(smem_u32(S.a[atom])), db = smem_desc(smem_u32(S.b[atom]));
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)   // K = 8 TF32 (32 bytes) per MMA
          mma_tf32(tmem, da + (uint64_t)(ks * 2), db + (uint64_t)(ks * 2), (atom > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(&S.bar);
    }
    const bool done = mbar_wait(&S.bar, (uint32_t)(layer & 1));
    ok = __syncthreads_and(done && ok) != 0;
    if (!ok) break;
    tc_fence_after();
    float* h = act ? act + (size_t)layer * n * kMlpHidden : nullptr;
    for (int c0 = 0; c0 < kMlpHidden; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int col = c0 + e;
        const float z = fmaxf(__uint_as_float(v[e]) + pf[boff[layer] + col], 0.f);
        if (act && row < n) h[(size_t)row * kMlpHidden + col] = z;
        if (layer < 2) *tf32_slot(S.a, warp * 32 + lane, col) = to_tf32(z);
        else out = fmaf(z, __bfloat162float(pw[L.w4 + col]), out);
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  if (ok && row < n) logits[row] = out + pf[L.b4];
  if (!ok) {
    if (tid == 0 && err) atomicOr(err, kErrTimeout);
    mbar_wait(&S.bar, 0u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMlpHidden));
}

}  // namespace

// ---- shared by the engine: inference over the voxels of a frame ----------

MlpLayout mlp_layout() {
  MlpLayout L;
  L.w1 = 0;
  L.b1 = L.w1 + kMlpHidden * kMlpIn;
  L.w2 = L.b1 + kMlpHidden;
  L.b2 = L.w2 + kMlpHidden * kMlpHidden;
  L.w3 = L.b2 + kMlpHidden;
  L.b3 = L.w3 + kMlpHidden * kMlpHidden;
  L.w4 = L.b3 + kMlpHidden;
  L.b4 = L.w4 + kMlpHidden;
  L.n = L.b4 + 1;
  return L;
}

// Biases stay FP32 (the FP32 copy of the parameters is passed as `pf`); the
// weight matrices are read as BF16.  act: [3][n][128] hidden activations for the
// backward pass, or NULL (inference); logits: [n].  err (device, may be NULL):
// kErrTimeout is or-ed in if a tensor-core wait gave up.
void mlp_forward(const __nv_bfloat16* pw, const float* pf, const float* x, int n, float* act, float* logits,
                 int* err, cudaStream_t s) {
  if (n <= 0) return;
  raise_smem_limit(k_mlp_fwd_tc, kFwdSmemBytes);
  k_mlp_fwd_tc<<<(n + kFwdRows - 1) / kFwdRows, kFwdRows, kFwdSmemBytes, s>>>(pw, pf, x, n, act, logits, err,
                                                                             mlp_layout());
}

int mlp_forward_launches() { return 1; }

}  // namespace erm

// ---- the trainer (C-ABI) -----------------------------------------------------

using namespace erm;

struct ermod_mlp {
  int device = 0, max_batch = 0;
  cudaStream_t st = nullptr;
  float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;   // FP32 master, Adam moments, gradient
  __nv_bfloat16* wb = nullptr;                                     // BF16 weights used by every pass
  float *x = nullptr, *y = nullptr, *act = nullptr, *s = nullptr, *gs = nullptr, *l = nullptr;
  float *d3 = nullptr, *d2 = nullptr, *d1 = nullptr;
  double* loss = nullptr;
  int* dev_err = nullptr;        // set by the tensor-core forward if a wait gave up
  long long t = 0;
  std::string err;
};

namespace {
// the tensor-core forward's error word, read (and cleared) after the stream is synchronised
int take_dev_err(ermod_mlp* p) {
  int e = 0;
  if (cudaMemcpy(&e, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (e == 0) return ERMOD_OK;
  cudaMemset(p->dev_err, 0, sizeof(int));
  p->err = "tc_wait";
  return ERMOD_ERR_CUDA;
}

void mlp_free(ermod_mlp* p) {
  void* ptrs[] = {p->w, p->m, p->v, p->g, p->wb, p->x, p->y, p->act, p->s, p->gs, p->l, p->d3, p->d2, p->d1, p->loss,
                  p->dev_err};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (p->st) cudaStreamDestroy(p->st);
}

// x and y (host) into the device batch buffers
int stage(ermod_mlp* p, const float* x, const float* y, int n) {
  if (cudaMemcpyAsync(p->x, x, sizeof(float) * (size_t)n * kMlpIn, cudaMemcpyHostToDevice, p->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  if (y && cudaMemcpyAsync(p->y, y, sizeof(float) * n, cudaMemcpyHostToDevice, p->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  return ERMOD_OK;
}

// forward + loss + backward into p->g for a staged batch of n samples
void backward(ermod_mlp* p, int n) {
  const MlpLayout L = mlp_layout();
  cudaStream_t s = p->st;
  const __nv_bfloat16* wb = p->wb;
  mlp_forward(wb, p->w, p->x, n, p->act, p->s, p->dev_err, s);
  float* h1 = p->act;
  float* h2 = p->act + (size_t)n * kMlpHidden;
  float* h3 = h2 + (size_t)n * kMlpHidden;
  k_bce<<<(n + 255) / 256, 256, 0, s>>>(n, p->s, p->y, p->gs, p->l);
  k_sum_loss<<<1, 1024, 0, s>>>(n, p->l, p->loss);
  float* g = p->g;
  const int H = kMlpHidden;
  // output layer: dw4[j] = sum_i gs_i h3[i][j], db4 = sum_i gs_i
  gemm(1, H, n, p->gs, 0, 1, h3, H, 1, g + L.w4, H, (const float*)nullptr, 0, (const float*)nullptr, 0, s);
  k_colsum<<<1, 32, 0, s>>>(n, 1, p->gs, g + L.b4);
  // d3 = gs w4^T masked by h3 > 0
  gemm(n, H, 1, p->gs, 1, 1, wb + L.w4, 0, 1, p->d3, H, (const float*)nullptr, 0, h3, H, s);
  // layer 3: dW3 = d3^T h2, db3 = colsum(d3), d2 = (d3 W3) masked by h2 > 0
  gemm(H, H, n, p->d3, 1, H, h2, H, 1, g + L.w3, H, (const float*)nullptr, 0, (const float*)nullptr, 0, s);
  k_colsum<<<1, H, 0, s>>>(n, H, p->d3, g + L.b3);
  gemm(n, H, H, p->d3, H, 1, wb + L.w3, H, 1, p->d2, H, (const float*)nullptr, 0, h2, H, s);
  // layer 2
  gemm(H, H, n, p->d2, 1, H, h1, H, 1, g + L.w2, H, (const float*)nullptr, 0, (const float*)nullptr, 0, s);
  k_colsum<<<1, H, 0, s>>>(n, H, p->d2, g + L.b2);
  gemm(n, H, H, p->d2, H, 1, wb + L.w2, H, 1, p->d1, H, (const float*)nullptr, 0, h1, H, s);
  // layer 1
  gemm(H, kMlpIn, n, p->d1, 1, H, p->x, kMlpIn, 1, g + L.w1, kMlpIn, (const float*)nullptr, 0,
       (const float*)nullptr, 0, s);
  k_colsum<<<1, H, 0, s>>>(n, H, p->d1, g + L.b1);
}
}  // namespace

extern "C" {

int32_t ermod_mlp_create(ermod_mlp** out, int32_t device, int32_t max_batch, const float* init_params) {
  if (!out || max_batch <= 0 || !init_params) return ERMOD_ERR_ARG;
  *out = nullptr;
  ermod_mlp* p = new ermod_mlp();
  p->device = device;
  p->max_batch = max_batch;
  const int np = mlp_layout().n;
  const size_t B = (size_t)max_batch;
  auto A = [&](auto** q, size_t n) { return cudaMalloc((void**)q, sizeof(**q) * std::max<size_t>(n, 1)); };
  bool ok = cudaSetDevice(device) == cudaSuccess && cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking) == 0 &&
            A(&p->w, np) == 0 && A(&p->m, np) == 0 && A(&p->v, np) == 0 && A(&p->g, np) == 0 &&
            A(&p->wb, np) == 0 && A(&p->x, B * kMlpIn) == 0 && A(&p->y, B) == 0 &&
            A(&p->act, 3 * B * kMlpHidden) == 0 && A(&p->s, B) == 0 && A(&p->gs, B) == 0 && A(&p->l, B) == 0 &&
            A(&p->d3, B * kMlpHidden) == 0 && A(&p->d2, B * kMlpHidden) == 0 && A(&p->d1, B * kMlpHidden) == 0 &&
            A(&p->loss, 1) == 0 && A(&p->dev_err, 1) == 0;
  if (ok) {
    ok = cudaMemcpyAsync(p->w, init_params, sizeof(float) * np, cudaMemcpyHostToDevice, p->st) == cudaSuccess &&
         cudaMemsetAsync(p->m, 0, sizeof(float) * np, p->st) == cudaSuccess &&
         cudaMemsetAsync(p->v, 0, sizeof(float) * np, p->st) == cudaSuccess &&
         cudaMemsetAsync(p->dev_err, 0, sizeof(int), p->st) == cudaSuccess;
    k_to_bf16<<<(np + 255) / 256, 256, 0, p->st>>>(np, p->w, p->wb);
    ok = ok && cudaStreamSynchronize(p->st) == cudaSuccess && cudaGetLastError() == cudaSuccess;
  }
  if (!ok) {
    mlp_free(p);
    delete p;
    return ERMOD_ERR_CUDA;
  }
  *out = p;
  return ERMOD_OK;
}

int32_t ermod_mlp_nparams(void) { return mlp_layout().n; }

// logits of n samples x[n][64] (host) with the current BF16 weights
int32_t ermod_mlp_forward(ermod_mlp* p, const float* x, int32_t n, float* logits) {
  if (!p || !x || !logits || n <= 0 || n > p->max_batch) return ERMOD_ERR_ARG;
  if (cudaSetDevice(p->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  int rc = stage(p, x, nullptr, n);
  if (rc != ERMOD_OK) return rc;
  mlp_forward(p->wb, p->w, p->x, n, p->act, p->s, p->dev_err, p->st);
  if (cudaMemcpyAsync(logits, p->s, sizeof(float) * n, cudaMemcpyDeviceToHost, p->st) != cudaSuccess ||
      cudaStreamSynchronize(p->st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return ERMOD_ERR_CUDA;
  return take_dev_err(p);
}

// the hidden activations [3][n][128] (FP32, after bias and ReLU) of the last
// forward or gradient pass over n samples
int32_t ermod_mlp_activations(ermod_mlp* p, int32_t n, float* act) {
  if (!p || !act || n <= 0 || n > p->max_batch) return ERMOD_ERR_ARG;
  if (cudaSetDevice(p->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (cudaMemcpyAsync(act, p->act, sizeof(float) * 3 * (size_t)n * kMlpHidden, cudaMemcpyDeviceToHost, p->st) !=
          cudaSuccess ||
      cudaStreamSynchronize(p->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  return ERMOD_OK;
}

// mean loss and its gradient (FP32, ERMOD_MLP_NPARAMS) for a batch, no update
int32_t ermod_mlp_gradients(ermod_mlp* p, const float* x, const float* y, int32_t n, float* grad, double* loss) {
  if (!p || !x || !y || n <= 0 || n > p->max_batch) return ERMOD_ERR_ARG;
  if (cudaSetDevice(p->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  int rc = stage(p, x, y, n);
  if (rc != ERMOD_OK) return rc;
  backward(p, n);
  if (grad && cudaMemcpyAsync(grad, p->g, sizeof(float) * mlp_layout().n, cudaMemcpyDeviceToHost, p->st) != 0)
    return ERMOD_ERR_CUDA;
  if (loss && cudaMemcpyAsync(loss, p->loss, sizeof(double), cudaMemcpyDeviceToHost, p->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  if (cudaStreamSynchronize(p->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ERMOD_ERR_CUDA;
  if (take_dev_err(p) != ERMOD_OK) return ERMOD_ERR_CUDA;
  return ERMOD_OK;
}

// one Adam step on a batch; returns the batch's mean loss before the step
int32_t ermod_mlp_train_step(ermod_mlp* p, const float* x, const float* y, int32_t n, float lr, double* loss) {
  if (!p || !x || !y || n <= 0 || n > p->max_batch || !(lr > 0.f)) return ERMOD_ERR_ARG;
  if (cudaSetDevice(p->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  int rc = stage(p, x, y, n);
  if (rc != ERMOD_OK) return rc;
  backward(p, n);
  ++p->t;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - (float)std::pow((double)b1, (double)p->t), c2 = 1.f - (float)std::pow((double)b2, (double)p->t);
  const int np = mlp_layout().n;
  k_adam<<<(np + 255) / 256, 256, 0, p->st>>>(np, lr, b1, b2, 1e-8f, c1, c2, p->w, p->m, p->v, p->g, p->wb);
  if (loss && cudaMemcpyAsync(loss, p->loss, sizeof(double), cudaMemcpyDeviceToHost, p->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  if (cudaStreamSynchronize(p->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ERMOD_ERR_CUDA;
  if (take_dev_err(p) != ERMOD_OK) return ERMOD_ERR_CUDA;
  return ERMOD_OK;
}

// FP32 master parameters (host)
int32_t ermod_mlp_get_params(ermod_mlp* p, float* params) {
  if (!p || !params) return ERMOD_ERR_ARG;
  if (cudaSetDevice(p->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (cudaMemcpyAsync(params, p->w, sizeof(float) * mlp_layout().n, cudaMemcpyDeviceToHost, p->st) != cudaSuccess ||
      cudaStreamSynchronize(p->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  return ERMOD_OK;
}

void ermod_mlp_destroy(ermod_mlp* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->st) cudaStreamSynchronize(p->st);
  mlp_free(p);
  delete p;
}

}  // extern "C"

namespace erm {
void launch_to_bf16(int n, const float* src, __nv_bfloat16* dst, cudaStream_t s) {
  k_to_bf16<<<(n + 255) / 256, 256, 0, s>>>(n, src, dst);
}
}  // namespace erm
