// ecorr_tc.cu -- ecorr accumulation as exact INT8 tensor-core GEMMs (tcgen05, sm_100a).
//
// The reference adds, per insertion, engnmfc * k_i * k_j to ecorr(j, i) over
// every pair of non-empty bins of that insertion's count vector
// (erdst/engproc.F90:948-962).  Over a batch of insertions that is
//     ecorr += C^T diag(w) C,        C[cnt][bin] = counts, w = engnmfc.
// Counts are small integers, so C^T X C with integer X is exact on the INT8
// tensor cores (u8 x u8 -> s32).  The FP64 weights are made integer by
//     w_cnt = w_min + m_cnt * q,   m_cnt in [0, 2^P - 1],  q = (w_max - w_min) / (2^P - 1)
// with P chosen per batch so that |w - (w_min + m q)| <= 2^-25 w_min, and
//     C^T diag(w) C = w_min C^T C + q sum_d 2^d C^T diag(bit_d(m)) C :
// one plain GEMM plus P GEMMs whose A operand has the insertions without
// bit d masked out.  Counts above 255 occur in few bins (far solvent piles
// up near zero energy): the GEMM multiplies the low bytes l = c mod 256 and
// k_ecorr_high adds sum_i w_i (c_b c_h - l_b l_h) for those bins in FP64 with
// the exact weights; past kMaxHigh such bins the GEMM instead adds the
// base-256 limb products (c = 256 h + l: h-l, l-h, h-h).  Every GEMM is exact
// in INT32 (at most 4096 * 255^2 per entry); the FP64 combination runs in a
// fixed order, so the result is deterministic.
//
// Kernel structure: a CTA per 128 x 64 tile of the upper triangle of ecorr
// (the epilogue also writes the mirror).  Per K tile of 128
// insertions the CTA stages A (128 bin rows x 128 bytes) and up to eight
// masked copies of B (64 bin rows x 128 bytes, one per term of the group)
// in shared memory in the 128-byte-swizzled K-major layout, in one of two
// stages so that the next K tile is staged while the tensor cores work on
// the current one.  One thread issues the tcgen05.mma instructions (M=128,
// N=64, K=32 each) into up to eight TMEM accumulators (8 x 64 columns) and a
// tcgen05.commit signals the stage's mbarrier.  The epilogue reads the
// accumulators with tcgen05.ld and adds scale * value into ecorr.  Every wait
// on an mbarrier has an iteration limit; on expiry the kernel records an
// error, waits (again bounded) for its MMAs in flight, frees its TMEM and
// returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "engine.cuh"
#include "tc_sm100.cuh"

namespace erm {

namespace {

using namespace tc;

constexpr int kTileM = 128;          // bins of the A side (TMEM lanes)
constexpr int kTileN = 64;           // bins of the B side (TMEM columns per accumulator)
constexpr int kTileK = 128;          // insertions per K tile (one 128-byte swizzle row)
constexpr int kMaxGroup = 8;         // accumulators per pass: 8 x 64 = 512 TMEM columns
constexpr int kThreads = 256;
constexpr int kMaxDigits = 30;
constexpr int kMaxHigh = 64;         // bins with counts above 255 handled by the FP64 correction

struct QuantParams {
  int P;              // weight digits
  int has_high;       // some count > 255 in the batch
  int kpad;           // insertions rounded up to kTileK
  int pad;
  double wmin, q;     // w = wmin + m * q
};

// instruction descriptor: kind::i8, D = s32, A = B = u8, both K-major, M = 128, N = 64
__host__ __device__ constexpr uint32_t idesc_i8() {
  return (2u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(kTileN >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  const uint32_t idesc = idesc_i8();
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// 4 mask bits -> 4 bytes of 0x00 / 0xFF
__device__ __forceinline__ uint32_t expand4(uint32_t b) {
  return ((b & 1u) ? 0x000000FFu : 0u) | ((b & 2u) ? 0x0000FF00u : 0u) | ((b & 4u) ? 0x00FF0000u : 0u) |
         ((b & 8u) ? 0xFF000000u : 0u);
}

// ---- preparation --------------------------------------------------------
// counts[cnt][bin] (u32, batch rows) -> CT_l / CT_h [bin][kpad] (u8, insertions contiguous)
__global__ void k_counts_to_ct(int n, int kpad, int ermax_pad, const uint32_t* __restrict__ counts,
                               uint8_t* __restrict__ ctl, uint8_t* __restrict__ cth, int* __restrict__ high,
                               int* __restrict__ hbin) {
  __shared__ uint32_t tile[32][33];
  const int b0 = blockIdx.x * 32, c0 = blockIdx.y * 32;  // bins, insertions
  const int tx = threadIdx.x, ty = threadIdx.y;          // (32, 8)
  for (int j = 0; j < 32; j += 8) {
    const int cnt = c0 + ty + j, bin = b0 + tx;
    tile[ty + j][tx] = (cnt < n && bin < ermax_pad) ? counts[(size_t)cnt * ermax_pad + bin] : 0u;
  }
  __syncthreads();
  int hi = 0;
  for (int j = 0; j < 32; j += 8) {
    const int bin = b0 + ty + j, cnt = c0 + tx;
    if (bin < ermax_pad && cnt < kpad) {
      const uint32_t v = tile[tx][ty + j];
      ctl[(size_t)bin * kpad + cnt] = (uint8_t)(v & 255u);
      cth[(size_t)bin * kpad + cnt] = (uint8_t)((v >> 8) & 255u);
      if (v > 255u) {
        hi = 1;
        atomicOr(&hbin[bin], 1);
      }
    }
  }
  if (__syncthreads_or(hi) && tx == 0 && ty == 0) atomicOr(high, 1);
}

// Bins with a count above 255 in the batch, in bin order (one block: ballot
// and a fixed-order scan of the per-warp counts).  Up to kMaxHigh of them go
// to the FP64 correction below and the GEMM then multiplies the low bytes only;
// beyond that the GEMM adds the base-256 limb products instead (*high stays 1).
constexpr int kListThreads = 1024;

__global__ void __launch_bounds__(kListThreads) k_high_list(int ermax, const int* __restrict__ hbin,
                                                            int* __restrict__ hl, int* __restrict__ nh,
                                                            int* __restrict__ high) {
  __shared__ int wcount[32];
  __shared__ int base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base = 0;
  __syncthreads();
  for (int b0 = 0; b0 < ermax; b0 += kListThreads) {
    const int b = b0 + tid;
    const bool f = b < ermax && hbin[b] != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcount[warp] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += wcount[w];
    off += __popc(bal & ((1u << lane) - 1u));
    if (f && off < kMaxHigh) hl[off] = b;
    __syncthreads();
    if (tid == 0) {
      int t = 0;
      for (int w = 0; w < kListThreads / 32; ++w) t += wcount[w];
      base += t;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (base <= kMaxHigh) {
      *nh = base;
      *high = 0;
    } else {
      *nh = 0;
    }
  }
}

// ecorr += sum_i w_i (C_ib C_ih - L_ib L_ih) for the high bins h (C: counts,
// L = C mod 256, the part the low-byte GEMM added), over every bin b, and the
// mirror element for b outside the high list.  A CTA per (32 bins, high bin):
// lane = bin, each warp a contiguous slice of the insertions, the warps'
// partial sums added in warp order -- FP64 with the exact weights,
// deterministic.
constexpr int kHighWarps = 16;

__global__ void __launch_bounds__(kHighWarps * 32) k_ecorr_high(int n, int ermax, int ermax_pad,
    const uint32_t* __restrict__ counts, const double* __restrict__ w, const int* __restrict__ hbin,
    const int* __restrict__ hl, const int* __restrict__ nh, double* __restrict__ ecorr) {
  __shared__ double red[kHighWarps][32];
  const int hi = blockIdx.y;
  if (hi >= *nh) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = blockIdx.x * 32 + lane;
  const int h = hl[hi];
  const int per = (n + kHighWarps - 1) / kHighWarps;
  const int i0 = warp * per, i1 = min(n, i0 + per);
  double acc = 0.0;
  if (b < ermax) {
    // branch-free and four insertions deep, so that the loads of a group are in flight together;
    // c_b c_h - l_b l_h is an exact integer below 2^53, summed in insertion order
    int i = i0;
    for (; i + 4 <= i1; i += 4) {
      uint32_t ch[4], cb[4];
      double wi[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        ch[u] = counts[(size_t)(i + u) * ermax_pad + h];
        cb[u] = counts[(size_t)(i + u) * ermax_pad + b];
        wi[u] = w[i + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint64_t full = (uint64_t)cb[u] * ch[u], low = (uint64_t)(cb[u] & 255u) * (ch[u] & 255u);
        acc += wi[u] * (double)(full - low);
      }
    }
    for (; i < i1; ++i) {
      const uint32_t ch = counts[(size_t)i * ermax_pad + h], cb = counts[(size_t)i * ermax_pad + b];
      const uint64_t full = (uint64_t)cb * ch, low = (uint64_t)(cb & 255u) * (ch & 255u);
      acc += w[i] * (double)(full - low);
    }
  }
  red[warp][lane] = acc;
  __syncthreads();
  if (warp == 0 && b < ermax) {
    double t = 0.0;
    for (int k = 0; k < kHighWarps; ++k) t += red[k][lane];
    ecorr[(size_t)b * ermax + h] += t;
    if (!hbin[b]) ecorr[(size_t)h * ermax + b] += t;
  }
}

// weights -> (wmin, q, P, m_cnt), one CTA, fixed-order reductions
__global__ void k_quantize(int base, int n, int kpad, int bits, const double* __restrict__ w,
                           uint32_t* __restrict__ m, uint16_t* __restrict__ gbits, QuantParams* qp,
                           const int* __restrict__ high) {
  __shared__ double smin[32], smax[32];
  double lo = 1e300, hi = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    lo = fmin(lo, w[base + i]);
    hi = fmax(hi, w[base + i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) { smin[threadIdx.x >> 5] = lo; smax[threadIdx.x >> 5] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) { lo = fmin(lo, smin[i]); hi = fmax(hi, smax[i]); }
    lo = fmin(lo, smin[0]);
    hi = fmax(hi, smax[0]);
    const double span = hi - lo;
    int P = 0;
    if (span > 0.0) {
      if (lo > 0.0) P = (int)ceil((double)bits + 1.0 + log2(span / lo));
      else P = kMaxDigits;
      P = P < 1 ? 1 : (P > kMaxDigits ? kMaxDigits : P);
    }
    qp->P = P;
    qp->has_high = *high;
    qp->kpad = kpad;
    qp->wmin = lo;
    qp->q = P > 0 ? span / (double)((1u << P) - 1u) : 0.0;
    smin[0] = lo;
    smax[0] = qp->q;
  }
  __syncthreads();
  const double wmin = smin[0], q = smax[0];
  for (int i = threadIdx.x; i < kpad; i += blockDim.x)
    m[i] = (i < n && q > 0.0) ? (uint32_t)llrint((w[base + i] - wmin) / q) : 0u;
  __syncthreads();
  // mask bits per (K tile, term, 16-insertion chunk): term 0 = every insertion,
  // term d >= 1 = insertions whose digit d-1 is set
  const int P = qp->P;
  const int nk = kpad / kTileK;
  for (int x = threadIdx.x; x < nk * (kMaxDigits + 1) * 8; x += blockDim.x) {
    const int kt = x / ((kMaxDigits + 1) * 8), rem = x % ((kMaxDigits + 1) * 8);
    const int d = rem / 8, c = rem % 8;
    uint32_t v = 0;
    if (d <= P)
      for (int e = 0; e < 16; ++e) {
        const uint32_t mm = m[kt * kTileK + c * 16 + e];
        v |= (d == 0 ? 1u : ((mm >> (d - 1)) & 1u)) << e;
      }
    gbits[x] = (uint16_t)v;
  }
}

// ---- the GEMM ------------------------------------------------------------
// Two shared-memory stages, each holding the unmasked A tile and one masked
// copy of the B tile per term of the group: while the tensor cores run the
// MMAs of one K tile, the threads load the next K tile from global memory
// into registers and then fill the other stage.
constexpr int kStages = 2;
constexpr int kBitRows = kMaxDigits + 1;   // term 0 (all insertions) + digits 1..P

struct TcStage {
  uint8_t b[kMaxGroup][kTileN * kTileK];   // masked B copies, 8 KB each (1024-B aligned)
  uint8_t a[kTileM * kTileK];              // A tile, 16 KB
};

struct TcSmem {
  TcStage st[kStages];
  uint64_t bar[kStages];
  uint32_t tmem_base;
};

__global__ void __launch_bounds__(kThreads, 1) k_ecorr_tc(int ermax, int kpad, const uint8_t* __restrict__ ctl,
    const uint8_t* __restrict__ cth, const uint16_t* __restrict__ gbits, const QuantParams* __restrict__ qp,
    double* __restrict__ ecorr, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>((void*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i0 = blockIdx.y * kTileM, j0 = blockIdx.x * kTileN;
  // ecorr is symmetric: tiles whose columns all lie below the diagonal are the
  // mirror of tiles computed elsewhere
  if (j0 + kTileN <= i0) return;
  const QuantParams Q = *qp;
  if (!Q.has_high) return;   // at most kMaxHigh bins above 255: k_ecorr_tma serves the batch
  const int P = Q.P;
  const int nk = kpad / kTileK;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&S.bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  uint32_t phase[kStages] = {0u, 0u};
  bool used[kStages] = {false, false};
  bool ok = true;
  // this thread's share of a K tile: 4 A chunks (rows tid/8 + 32 q), 2 B chunks
  // (rows tid/8, tid/8 + 32), all in 16-byte chunk column c = tid % 8
  const int c = tid & 7, r0 = tid >> 3;
  uint4 ra[4], rb[2];
  uint32_t rbits[kMaxGroup];

  const int npairs = Q.has_high ? 4 : 1;
  const int nterms = 1 + P;
  for (int pair = 0; pair < npairs && ok; ++pair) {
    const uint8_t* A = (pair == 0 || pair == 1) ? ctl : cth;   // 0: l-l, 1: l-h, 2: h-l, 3: h-h
    const uint8_t* B = (pair == 0 || pair == 2) ? ctl : cth;
    const double limb = pair == 0 ? 1.0 : (pair == 3 ? 65536.0 : 256.0);
    for (int t0 = 0; t0 < nterms && ok; t0 += kMaxGroup) {
      const int G = min(kMaxGroup, nterms - t0);
      auto load_tile = [&](int kt) {
        const int k0 = kt * kTileK;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = r0 + 32 * q;
          ra[q] = (i0 + r < ermax) ? *reinterpret_cast<const uint4*>(A + (size_t)(i0 + r) * kpad + k0 + c * 16)
                                   : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int r = r0 + 32 * q;
          rb[q] = (j0 + r < ermax) ? *reinterpret_cast<const uint4*>(B + (size_t)(j0 + r) * kpad + k0 + c * 16)
                                   : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int g = 0; g < kMaxGroup; ++g)
          rbits[g] = g < G ? (uint32_t)gbits[((size_t)kt * kBitRows + t0 + g) * 8 + c] : 0u;
      };
      load_tile(0);
      for (int kt = 0; kt < nk; ++kt) {
        const int s = kt & 1;
        if (used[s]) {  // the MMAs that last read this stage must be done
          const bool done = mbar_wait(&S.bar[s], phase[s]);
          phase[s] ^= 1u;
          used[s] = false;
          ok = __syncthreads_and(done) != 0;
          if (!ok) break;
        }
        TcStage& T = S.st[s];
#pragma unroll
        for (int q = 0; q < 4; ++q) *reinterpret_cast<uint4*>(T.a + swz(r0 + 32 * q, c)) = ra[q];
        for (int g = 0; g < G; ++g) {
          const uint32_t bits = rbits[g];
          const uint32_t m0 = expand4(bits & 15u), m1 = expand4((bits >> 4) & 15u);
          const uint32_t m2 = expand4((bits >> 8) & 15u), m3 = expand4((bits >> 12) & 15u);
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            uint4 v = rb[q];
            v.x &= m0; v.y &= m1; v.z &= m2; v.w &= m3;
            *reinterpret_cast<uint4*>(T.b[g] + swz(r0 + 32 * q, c)) = v;
          }
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
          tc_fence_after();
          const uint64_t da0 = smem_desc(smem_u32(T.a));
          for (int g = 0; g < G; ++g) {
            const uint64_t db0 = smem_desc(smem_u32(T.b[g]));
#pragma unroll
            for (int ks = 0; ks < kTileK / 32; ++ks)   // K = 32 bytes per MMA: advance 32 B = 2 x 16 B
              mma_i8(tmem + (uint32_t)(g * kTileN), da0 + (uint64_t)(ks * 2), db0 + (uint64_t)(ks * 2),
                     (kt > 0 || ks > 0) ? 1u : 0u);
          }
          mma_commit(&S.bar[s]);
        }
        used[s] = true;
        if (kt + 1 < nk) load_tile(kt + 1);   // global loads overlap the MMAs just issued
      }
      // drain both stages
      for (int s = 0; s < kStages && ok; ++s)
        if (used[s]) {
          const bool done = mbar_wait(&S.bar[s], phase[s]);
          phase[s] ^= 1u;
          used[s] = false;
          ok = __syncthreads_and(done) != 0;
        }
      if (!ok) break;
      // epilogue: warps 0-3 own TMEM lanes 32w..32w+31 = rows i0 + 32w + lane
      tc_fence_after();
      if (warp < 4) {
        const int row = i0 + warp * 32 + lane;
        for (int cc = 0; cc < kTileN; cc += 32) {
          double acc[32];
#pragma unroll
          for (int e = 0; e < 32; ++e) acc[e] = 0.0;
          for (int g = 0; g < G; ++g) {
            const int term = t0 + g;
            const double scale = limb * (term == 0 ? Q.wmin : ldexp(Q.q, term - 1));
            uint32_t v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(g * kTileN + cc), v);
#pragma unroll
            for (int e = 0; e < 32; ++e) acc[e] += scale * (double)(int32_t)v[e];
          }
          if (row < ermax) {
            // upper triangle and its mirror; the diagonal once
#pragma unroll
            for (int e = 0; e < 32; ++e) {
              const int col = j0 + cc + e;
              if (col >= ermax || col < row) continue;
              ecorr[(size_t)row * ermax + col] += acc[e];
              if (col > row) ecorr[(size_t)col * ermax + row] += acc[e];
            }
          }
        }
      }
      tc_fence_before();
      __syncthreads();
    }
  }
  if (!ok) {
    // record the failure and give the MMAs still in flight a bounded time to finish
    // before the TMEM they write is released
    if (tid == 0) atomicOr(err, kErrTimeout);
    for (int s = 0; s < kStages; ++s)
      if (used[s]) mbar_wait(&S.bar[s], phase[s]);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

constexpr size_t kSmemBytes = sizeof(TcSmem) + 1024;

// ---- byte-digit terms, fed by TMA ---------------------------------------
// With m = sum_d 256^d b_d (b_d = byte d of the integer weight), the low-byte part is
//   sum_k w_k L_ik L_jk = wmin (L^T L)_ij + q sum_d 256^d (256 (L^T X_d)_ij + (L^T Y_d)_ij),
// where b_dk L_jk = 256 X_djk + Y_djk splits the (at most 16-bit) product into two exact
// bytes.  So 1 + 2 ceil(P / 8) INT8 GEMMs replace the 1 + P masked ones, and every operand
// is a plain byte array that TMA can stream: T[term][bin][insertion], term 0 = L,
// 1 + 2d = X_d, 2 + 2d = Y_d.
constexpr int kMaxBytes = (kMaxDigits + 7) / 8;   // 4
constexpr int kMaxTerms = 1 + 2 * kMaxBytes;      // 9
constexpr int kTmaStages = 3;
constexpr int kTmaGroup = 4;                      // terms per pass: 4 x 64 TMEM columns
constexpr int kTmaThreads = 128;

__global__ void k_ecorr_terms(int rows, int kpad, const uint8_t* __restrict__ L, const uint32_t* __restrict__ m,
                              const QuantParams* __restrict__ qp, const int* __restrict__ high,
                              uint8_t* __restrict__ XY) {
  if (*high) return;
  const int nd = (qp->P + 7) / 8;
  const size_t slab = (size_t)rows * kpad;
  const size_t i16 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;   // 16-insertion chunk of one bin
  if (i16 * 16 >= slab) return;
  const size_t off = i16 * 16;
  const int k0 = (int)(off % (size_t)kpad);
  const uint4 lv = *reinterpret_cast<const uint4*>(L + off);
  const uint8_t* l = reinterpret_cast<const uint8_t*>(&lv);
  for (int d = 0; d < nd; ++d) {
    alignas(16) uint8_t x[16], y[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const uint32_t v = ((m[k0 + e] >> (8 * d)) & 255u) * (uint32_t)l[e];
      x[e] = (uint8_t)(v >> 8);
      y[e] = (uint8_t)(v & 255u);
    }
    *reinterpret_cast<uint4*>(XY + (size_t)(2 * d) * slab + off) = *reinterpret_cast<const uint4*>(x);
    *reinterpret_cast<uint4*>(XY + (size_t)(2 * d + 1) * slab + off) = *reinterpret_cast<const uint4*>(y);
  }
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// TMA tile loads of this GPU's own memory into shared memory (no multicast)
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

struct TmaStage {
  uint8_t a[kTileM * kTileK];              // L tile, 16 KB (1024-B aligned)
  uint8_t b[kTmaGroup][kTileN * kTileK];   // term tiles, 8 KB each
};
constexpr int kTilePitch = kTileN + 1;             // doubles per row of the accumulated tile
struct TmaSmem {
  TmaStage st[kTmaStages];
  double tile[kTileM * kTilePitch];                 // the tile's FP64 sum over the passes
  uint64_t full[kTmaStages], empty[kTmaStages], done;
  uint32_t tmem_base;
};
constexpr size_t kTmaSmemBytes = sizeof(TmaSmem) + 1024;

// A CTA per 128 x 64 tile of the upper triangle; thread 0 streams the tiles of every K step
// (the L rows of the tile's 128 bins, the term rows of its 64 bins) into a ring of
// kTmaStages stages, thread 32 issues the MMAs of each full stage into kTmaGroup TMEM
// accumulators and commits the stage back, and the four warps read the accumulators
// (lanes = rows) once the pass is done.  Every mbarrier wait has an iteration limit.
__global__ void __launch_bounds__(kTmaThreads, 1) k_ecorr_tma(int ermax, int kpad,
    const __grid_constant__ CUtensorMap tmapA, const __grid_constant__ CUtensorMap tmapB,
    const QuantParams* __restrict__ qp, double* __restrict__ ecorr, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm_raw[];
  TmaSmem& S = *reinterpret_cast<TmaSmem*>((void*)(((uintptr_t)tsm_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i0 = blockIdx.y * kTileM, j0 = blockIdx.x * kTileN;
  if (j0 + kTileN <= i0) return;                 // the mirror of a tile computed elsewhere
  const QuantParams Q = *qp;
  if (Q.has_high) return;                        // k_ecorr_tc's limb products serve this batch
  const int nterms = 1 + 2 * ((Q.P + 7) / 8);
  const int nk = kpad / kTileK;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(kTmaGroup * kTileN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kTmaStages; ++s) { mbar_init(&S.full[s], 1); mbar_init(&S.empty[s], 1); }
    mbar_init(&S.done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  bool ok = true;
  int it = 0;                                    // K steps streamed so far (both roles count alike)
  int pass = 0;
  for (int t0 = 0; t0 < nterms && ok; t0 += kTmaGroup, ++pass) {
    const int G = min(kTmaGroup, nterms - t0);
    const uint32_t bytes = (uint32_t)(kTileM * kTileK + G * kTileN * kTileK);
    if (tid == 0) {                              // producer
      for (int kt = 0; kt < nk && ok; ++kt) {
        const int i = it + kt, s = i % kTmaStages;
        if (i >= kTmaStages && !mbar_wait(&S.empty[s], (uint32_t)((i / kTmaStages - 1) & 1))) { ok = false; break; }
        mbar_expect_tx(&S.full[s], bytes);
        tma_load_2d(S.st[s].a, &tmapA, kt * kTileK, i0, &S.full[s]);
        for (int g = 0; g < G; ++g) tma_load_3d(S.st[s].b[g], &tmapB, kt * kTileK, j0, t0 + g, &S.full[s]);
      }
    } else if (tid == 32) {                      // MMA issuer
      for (int kt = 0; kt < nk && ok; ++kt) {
        const int i = it + kt, s = i % kTmaStages;
        if (!mbar_wait(&S.full[s], (uint32_t)((i / kTmaStages) & 1))) { ok = false; break; }
        tc_fence_after();
        const uint64_t da0 = smem_desc(smem_u32(S.st[s].a));
        for (int g = 0; g < G; ++g) {
          const uint64_t db0 = smem_desc(smem_u32(S.st[s].b[g]));
#pragma unroll
          for (int ks = 0; ks < kTileK / 32; ++ks)
            mma_i8(tmem + (uint32_t)(g * kTileN), da0 + (uint64_t)(ks * 2), db0 + (uint64_t)(ks * 2),
                   (kt > 0 || ks > 0) ? 1u : 0u);
        }
        mma_commit(&S.empty[s]);
      }
      if (ok) mma_commit(&S.done);
    }
    it += nk;
    ok = __syncthreads_and(ok) != 0;
    if (!ok) break;
    ok = __syncthreads_and(mbar_wait(&S.done, (uint32_t)(pass & 1))) != 0;
    if (!ok) break;
    // the pass's terms into the tile: warp w owns TMEM lanes 32w..32w+31 = tile rows
    tc_fence_after();
    {
      double* trow = S.tile + (warp * 32 + lane) * kTilePitch;
      for (int cc = 0; cc < kTileN; cc += 32) {
        double acc[32];
#pragma unroll
        for (int e = 0; e < 32; ++e) acc[e] = pass == 0 ? 0.0 : trow[cc + e];
        for (int g = 0; g < G; ++g) {
          const int term = t0 + g;
          const int d = (term - 1) >> 1;
          const double scale = term == 0 ? Q.wmin : ldexp(Q.q, 8 * d + (((term - 1) & 1) ? 0 : 8));
          uint32_t v[32];
          tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(g * kTileN + cc), v);
#pragma unroll
          for (int e = 0; e < 32; ++e) acc[e] += scale * (double)(int32_t)v[e];
        }
#pragma unroll
        for (int e = 0; e < 32; ++e) trow[cc + e] = acc[e];
      }
    }
    tc_fence_before();
    __syncthreads();                             // TMEM free for the next pass
  }
  if (ok) {
    // ecorr += the tile (upper triangle, diagonal once) and its mirror, every element owned by
    // one thread; eight values loaded before they are added and stored, so the loads overlap.
    // Upper part: a warp per row in turn, lanes over the columns (256-byte rows).
    for (int r0 = warp * 8; r0 < kTileM; r0 += 4 * 8) {
      double cur[8][2];
      size_t at[8][2];
      bool on[8][2];
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = i0 + r0 + u, col = j0 + lane + 32 * h;
          on[u][h] = row < ermax && col < ermax && col >= row;
          at[u][h] = (size_t)row * ermax + col;
          cur[u][h] = on[u][h] ? ecorr[at[u][h]] : 0.0;
        }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (on[u][h]) ecorr[at[u][h]] = cur[u][h] + S.tile[(r0 + u) * kTilePitch + lane + 32 * h];
    }
    // Mirror: a warp per column in turn, lanes over the rows (256-byte column runs of the
    // row-major matrix): element (col, row) for col > row.
    for (int c0 = warp * 4; c0 < kTileN; c0 += 4 * 4) {
      double cur[4][4];
      size_t at[4][4];
      bool on[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int rb = 0; rb < 4; ++rb) {
          const int row = i0 + rb * 32 + lane, col = j0 + c0 + u;
          on[u][rb] = row < ermax && col < ermax && col > row;
          at[u][rb] = (size_t)col * ermax + row;
          cur[u][rb] = on[u][rb] ? ecorr[at[u][rb]] : 0.0;
        }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int rb = 0; rb < 4; ++rb)
          if (on[u][rb]) ecorr[at[u][rb]] = cur[u][rb] + S.tile[(rb * 32 + lane) * kTilePitch + c0 + u];
    }
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, kErrTimeout);
    mbar_wait(&S.done, (uint32_t)(pass & 1));    // bounded: MMAs in flight finish before TMEM goes
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmaGroup * kTileN));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

// u8 tensor maps over the term array T[kMaxTerms][rows][kpad]: A = term 0 in 128-row boxes,
// B = any term in 64-row boxes; 128-byte rows, 128-byte swizzle (the UMMA K-major layout)
bool make_term_maps(uint8_t* T, int rows, int kpad, CUtensorMap* a, CUtensorMap* b) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dimA[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
  const cuuint64_t strA[1] = {(cuuint64_t)kpad};
  const cuuint32_t boxA[2] = {(cuuint32_t)kTileK, (cuuint32_t)kTileM};
  const cuuint32_t es2[2] = {1, 1};
  if (enc(a, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, T, dimA, strA, boxA, es2, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
      CUDA_SUCCESS)
    return false;
  const cuuint64_t dimB[3] = {(cuuint64_t)kpad, (cuuint64_t)rows, (cuuint64_t)kMaxTerms};
  const cuuint64_t strB[2] = {(cuuint64_t)kpad, (cuuint64_t)rows * kpad};
  const cuuint32_t boxB[3] = {(cuuint32_t)kTileK, (cuuint32_t)kTileN, 1};
  const cuuint32_t es3[3] = {1, 1, 1};
  return enc(b, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, T, dimB, strB, boxB, es3, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace

int ecorr_tc_available() { return 1; }

size_t ecorr_tc_workspace(int n, int ermax) {
  const size_t kpad = (size_t)(n + kTileK - 1) / kTileK * kTileK;
  const size_t ermax_pad = (size_t)(ermax + 127) / 128 * 128;
  return (kMaxTerms + 1) * ermax_pad * kpad + 4 * kpad + (kpad / kTileK) * (kMaxDigits + 1) * 8 * 2 + 256 + 64 +
         sizeof(int) * (ermax_pad + kMaxHigh + 4);
}

// ecorr += C^T diag(w) C for targets [base, base+n) of the batch starting at count_base
int launch_ecorr_tc(const DeviceState& d, int base, int n, int ermax, int ermax_pad, int count_base, int weight_bits,
                    void* work, size_t work_bytes, cudaStream_t s) {
  if (raise_smem_limit(k_ecorr_tc, kSmemBytes) != cudaSuccess) return -1;
  if (raise_smem_limit(k_ecorr_tma, kTmaSmemBytes) != cudaSuccess) return -1;
  const int kpad = (n + kTileK - 1) / kTileK * kTileK;
  const size_t nbits = (size_t)(kpad / kTileK) * (kMaxDigits + 1) * 8;
  const size_t slab = (size_t)ermax_pad * kpad;
  const size_t need = (kMaxTerms + 1) * slab + 4 * (size_t)kpad + 2 * nbits + 256 + 64 +
                      sizeof(int) * (ermax_pad + kMaxHigh + 4);
  if (need > work_bytes) return -2;
  uint8_t* ctl = (uint8_t*)work;                 // term 0 of T[kMaxTerms][ermax_pad][kpad]
  uint8_t* xy = ctl + slab;                      // terms 1 .. kMaxTerms - 1
  uint8_t* cth = ctl + (size_t)kMaxTerms * slab;
  uint32_t* m = (uint32_t*)(cth + slab);
  uint16_t* gbits = (uint16_t*)(m + kpad);
  QuantParams* qp = (QuantParams*)((uint8_t*)(gbits + nbits) + ((16 - (nbits * 2) % 16) % 16));
  int* high = (int*)((uint8_t*)qp + 64);
  int* nh = high + 1;
  int* hl = high + 4;
  int* hbin = hl + kMaxHigh;      // [ermax_pad]
  int* errw = &d.status->flags;   // kErrTimeout if an mbarrier wait expires
  const uint32_t* cnt = d.counts + (size_t)(base - count_base) * ermax_pad;
  cudaMemsetAsync(high, 0, sizeof(int) * (4 + kMaxHigh + ermax_pad), s);
  dim3 tb(32, 8), tg((ermax_pad + 31) / 32, (kpad + 31) / 32);
  k_counts_to_ct<<<tg, tb, 0, s>>>(n, kpad, ermax_pad, cnt, ctl, cth, high, hbin);
  k_high_list<<<1, kListThreads, 0, s>>>(ermax, hbin, hl, nh, high);
  k_quantize<<<1, 1024, 0, s>>>(base, n, kpad, weight_bits > 0 ? weight_bits : 24, d.w, m, gbits, qp, high);
  dim3 gg((ermax_pad + kTileN - 1) / kTileN, (ermax_pad + kTileM - 1) / kTileM);
  CUtensorMap map_a, map_b;
  if (!make_term_maps(ctl, ermax_pad, kpad, &map_a, &map_b)) return -4;
  const size_t chunks = slab / 16;
  k_ecorr_terms<<<(unsigned)((chunks + 255) / 256), 256, 0, s>>>(ermax_pad, kpad, ctl, m, qp, high, xy);
  k_ecorr_tma<<<gg, kTmaThreads, kTmaSmemBytes, s>>>(ermax, kpad, map_a, map_b, qp, d.ecorr, errw);
  k_ecorr_tc<<<gg, kThreads, kSmemBytes, s>>>(ermax, kpad, ctl, cth, gbits, qp, d.ecorr, errw);
  k_ecorr_high<<<dim3((ermax + 31) / 32, kMaxHigh), kHighWarps * 32, 0, s>>>(n, ermax, ermax_pad, cnt, d.w + base,
                                                                              hbin, hl, nh, d.ecorr);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace erm
