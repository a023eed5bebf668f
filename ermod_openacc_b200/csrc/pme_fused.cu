// pme_fused.cu -- the PME solve of a chunk of 32 targets without cuFFT and
// without a spread grid in HBM, for power-of-two meshes of 16..128 points a
// side.
//
// recpcal's per-insertion work (recpcal.F90:380-497 spreading, forward FFT,
// influence multiply, self energy; :592-710 the inverse FFT the gather reads)
// is, for a grid of K3 x K2 x K1 points and the half spectrum k1 < K1/2+1:
//
//   k_pme_plane     CTA = (target, k1 plane).  Forms the B-spline stencils of
//                   the solute sites (recpcal.F90:553-574) and their 1-D
//                   transforms B_m(k) = sum_c w_mc exp(-2 pi i k (g_m - c) / K_m)
//                   in FP64, builds the plane of the solute spectrum
//                   Qhat(k1, k2, k3) -- either directly,
//                   sum_a q_a B1_a(k1) B2_a(k2) B3_a(k3), or by spreading
//                   q_a B1_a(k1) w2 w3 on the (n2, n3) plane and a forward 2-D
//                   FFT -- multiplies by the influence function, adds the
//                   plane's share of the FP64 self energy, and runs the
//                   inverse 2-D FFT over (k2, k3) in shared memory.  The plane
//                   Y[b][k1][n3][n2] is written once (it stays in L2 for the
//                   next kernel).
//   k_pme_lines     a thread per (n3, n2) line and target: the complex-to-real
//                   transform along k1 (a half-length complex FFT of the
//                   Hermitian-packed line) in registers, written straight
//                   into the insertion-fastest potential layout the gather
//                   reads: n1 pairs (phi(2m), phi(2m+1)) per target, 32
//                   targets, for each line n3*K2 + n2
//                   (K1 <= 64; k_pme_rows does K1 = 128 in shared memory).
//
// The FFTs are radix-8/4 Stockham stages (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC08):
// every thread holds its butterflies in registers across one barrier, so a
// stage runs in place in shared memory.  Twiddle tables are FP64 values
// rounded to FP32.  All sums run in a fixed order, so results are bitwise
// reproducible.  The result equals spreading + R2C + influence + C2R of the
// cuFFT path up to FP32 rounding.
#include <algorithm>
#include <cmath>

#include "engine.cuh"
#include "regfft.cuh"
#include "tc_sm100.cuh"

namespace erm {

using namespace fft;

namespace {

// Placement of a batch of 2^LNB transforms of length 2^LN in shared memory:
// transform bt starts at (bt >> LBG) * BPITCH + (bt & (2^LBG - 1)) * BSTRIDE
// and its elements are ES apart.  Everything is a compile-time constant, so
// shared-memory addresses are immediates off one register per butterfly.
template <int LN_, int LNB_, int LBG_, int BPITCH_, int BSTRIDE_, int ES_>
struct FftShape {
  static constexpr int LN = LN_, LNB = LNB_, LBG = LBG_, BPITCH = BPITCH_, BSTRIDE = BSTRIDE_, ES = ES_;
};

// One radix-R Stockham stage (input stride N/R, output groups of Ns = 2^LNS)
// of every transform of the batch, in place: each thread loads its
// butterflies, the block synchronises, then stores.  tw[m] = exp(-2 pi i m / N).
template <class S, int R, int LNS, int NTHR, bool INV>
__device__ __forceinline__ void fft_stage(float2* buf, const float2* __restrict__ tw, int tid) {
  constexpr int LR = R == 8 ? 3 : 2;
  constexpr int NR = 1 << (S::LN - LR), NS = 1 << LNS, LTS = S::LN - LNS - LR;
  constexpr int NBUT = (1 << (S::LN + S::LNB)) / R;
  constexpr int BPT = NBUT / NTHR;
  static_assert(BPT * NTHR == NBUT, "butterflies must divide evenly over the threads");
  float2 v[BPT][R];
  int dst[BPT];
#pragma unroll
  for (int i = 0; i < BPT; ++i) {
    const int idx = tid + i * NTHR;
    const int bt = idx & ((1 << S::LNB) - 1), j = idx >> S::LNB;
    const int off = (bt >> S::LBG) * S::BPITCH + (bt & ((1 << S::LBG) - 1)) * S::BSTRIDE;
    const int k = j & (NS - 1);
    const float2* src = buf + off + j * S::ES;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 x = src[r * NR * S::ES];
      if (LNS > 0 && r > 0) {                      // the first stage has k = 0: unit twiddles
        const float2 w = tw[(k * r) << LTS];
        x = INV ? make_float2(x.x * w.x + x.y * w.y, x.y * w.x - x.x * w.y) : cmul(x, w);
      }
      v[i][r] = x;
    }
    dft<R, INV>(v[i]);
    dst[i] = off + ((j - k) * R + k) * S::ES;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < BPT; ++i)
#pragma unroll
    for (int r = 0; r < R; ++r) buf[dst[i] + r * NS * S::ES] = v[i][r];
  __syncthreads();
}

// All stages of every transform of the batch: radix 8, radix 4 for the
// remaining factors (2^4 = 4 * 4 rather than 8 * 2; lengths are >= 8).
template <class S, int LNS, int NTHR, bool INV>
__device__ __forceinline__ void fft_stages(float2* buf, const float2* __restrict__ tw, int tid) {
  if constexpr (LNS < S::LN) {
    constexpr int REM = S::LN - LNS;
    constexpr int R = (REM >= 3 && REM != 4) ? 8 : 4;
    fft_stage<S, R, LNS, NTHR, INV>(buf, tw, tid);
    fft_stages<S, LNS + (R == 8 ? 3 : 2), NTHR, INV>(buf, tw, tid);
  }
}

template <class S, int NTHR, bool INV>
__device__ __forceinline__ void fft_batch(float2* buf, const float2* __restrict__ tw, int tid) {
  static_assert(S::LN >= 3, "transform length >= 8");
  fft_stages<S, 0, NTHR, INV>(buf, tw, tid);
}

constexpr int kSiteTile = 32;                  // solute sites staged in shared memory at a time (at most)
constexpr int kTabPairs = 8;                   // (target, site) pairs per CTA of k_site_tables
constexpr int kStn = 2 + 2 * kMaxOrder;        // stencil record: g2, g3, w2[kMaxOrder], w3[kMaxOrder]
constexpr int kRowThreads = 512;
constexpr int kLineRows = 4;                   // n2 rows per CTA of k_pme_lines (a warp each): 4 or 8
constexpr int kLoadBatch = 8;                  // global loads a thread keeps in flight while staging

template <int LK2, int LK3>
struct PlaneCfg {
  static constexpr int K2 = 1 << LK2, K3 = 1 << LK3, PITCH = K2 + 1;
  static constexpr int E = LK2 + LK3 <= 12 ? 16 : 32;     // plane points per thread
  static constexpr int NTHR = (K2 * K3) / E;
  static constexpr int MINB = E == 16 ? 3 : 1;
  // plane spreading accumulates in 2^-40 fixed point in shared memory when the
  // int64 plane fits beside the FP32 plane (up to 8192 points)
  static constexpr bool FIXED = K2 * K3 <= 8192;
  static_assert(K3 % E == 0, "a thread owns E consecutive k3 of one k2 column");
};

}  // namespace

// ---------------------------------------------------------------------------
// k_site_tables: per (target, site) of a batch, the B-spline stencil
// (calc_spline_molecule, recpcal.F90:553-574) and its 1-D transforms
//   B_m(k) = sum_c w_mc exp(-2 pi i k (g_m - c) / K_m),
// summed in FP64 as exp(-2 pi i k g / K) times powers of exp(+2 pi i k / K).
// tab[pair][nk]: q B1(k1) for k1 < Kh1, then (direct sums) B2(k2), B3(k3).
// stn[pair][kStn]: g2, g3 (as floats), w2[kMaxOrder], w3[kMaxOrder].
// A CTA takes kTabPairs pairs: stencils first, then every entry of its pairs.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_site_tables(FrameArgs a, int base, int npairs, int nk,
    const float4* __restrict__ tgt_raw, const double2* __restrict__ fft_twd, float2* __restrict__ tab,
    float* __restrict__ stn) {
  __shared__ float sw[kTabPairs][3][kMaxOrder];
  __shared__ int sg[kTabPairs][3];
  __shared__ float sq[kTabPairs];
  const int K1 = a.K1, K2 = a.K2, K3 = a.K3, Kh1 = a.Kh1, n = a.order;
  const int p0 = blockIdx.x * kTabPairs;
  const int np = min(kTabPairs, npairs - p0);
  const float4* sites = tgt_raw + (size_t)base * a.nsite;
  for (int x = threadIdx.x; x < np * 3; x += blockDim.x) {
    const int t = x / 3, m = x - 3 * t;
    const float4 r = sites[p0 + t];
    const int K = m == 0 ? K1 : (m == 1 ? K2 : K3);
    float f = a.g.invcl[m][0] * r.x + a.g.invcl[m][1] * r.y + a.g.invcl[m][2] * r.z;
    f = f - floorf(f);
    f = f * (float)K;
    const int rci = (int)f;
    float w[kMaxOrder];
    spline_weights(f - (float)rci, n, w);
    for (int c = 0; c < kMaxOrder; ++c) sw[t][m][c] = c < n ? w[c] : 0.f;
    sg[t][m] = rci & (K - 1);
    if (m == 0) sq[t] = r.w;
  }
  __syncthreads();
  if (stn) {
    for (int x = threadIdx.x; x < np * kStn; x += blockDim.x) {
      const int t = x / kStn, r = x - t * kStn;
      float v;
      if (r < 2) v = (float)sg[t][1 + r];
      else if (r < 2 + kMaxOrder) v = sw[t][1][r - 2];
      else v = sw[t][2][r - 2 - kMaxOrder];
      stn[(size_t)(p0 + t) * kStn + r] = v;
    }
  }
  for (int x = threadIdx.x; x < np * nk; x += blockDim.x) {
    const int t = x / nk, r = x - t * nk;
    int m, k, K, t0;
    if (r < Kh1) { m = 0; k = r; K = K1; t0 = 0; }
    else if (r < Kh1 + K2) { m = 1; k = r - Kh1; K = K2; t0 = K1; }
    else { m = 2; k = r - Kh1 - K2; K = K3; t0 = K1 + K2; }
    const int g = sg[t][m];
    double2 e = fft_twd[t0 + ((k * g) & (K - 1))];
    const double2 st = fft_twd[t0 + ((K - k) & (K - 1))];   // exp(+2 pi i k / K)
    double re = (double)sw[t][m][0] * e.x, im = (double)sw[t][m][0] * e.y;
    for (int c = 1; c < n; ++c) {
      e = make_double2(e.x * st.x - e.y * st.y, e.x * st.y + e.y * st.x);
      re += (double)sw[t][m][c] * e.x;
      im += (double)sw[t][m][c] * e.y;
    }
    if (m == 0) {
      const double q = (double)sq[t];
      re *= q;
      im *= q;
    }
    tab[(size_t)(p0 + t) * nk + r] = make_float2((float)re, (float)im);
  }
}

// ---------------------------------------------------------------------------
// Direct site sums on the tensor cores (square 64 and 128 planes, up to 64 sites).  For one
// (target, k1) plane X(k3, k2) = sum_s B3_s(k3) D_s(k2), D_s = q_s B1_s(k1) B2_s(k2), is formed
// transposed, as one real product of a 128 x 2s operand A (row k2: Re D, Im D per site) by a
// 2s x 2K operand B (for each k3 the columns (Re B3, -Im B3) and (Im B3, Re B3)): product row
// k2, column 2 k3 + part is the real or imaginary part of X(k3, k2).  Every value is split
// into two TF32 terms (hi = v rounded to TF32, lo = v - hi rounded again) and the three
// products hi*hi, hi*lo and lo*hi are accumulated in FP32 in TMEM (`tcgen05.mma kind::tf32`,
// M = 128, N = 2K, K = 8 a step): the dropped lo*lo term and the split's rounding are below
// 2^-22 of each product, the FP32 level of the CUDA-core sums it replaces.  More than 16
// sites: tiles of 16 sites (K = 32) accumulate in the same TMEM columns, each tile's operands
// staged once the previous tile's MMAs have completed.
// ---------------------------------------------------------------------------
namespace tcs {
constexpr int kK = 32, kTileSites = kK / 2, kMaxSites = 4 * kTileSites;
constexpr int kRows = 128;                                          // M of every MMA
// A KN x KN plane, transposed: product row = k2 (KN = 64: rows 64..127 repeat rows 0..63, so
// that each of the four TMEM lane quarters holds the k2 of the warps that read it), product
// column = 2 k3 + part (part 0: Re, 1: Im), N = 2 KN.
template <int KN>
struct Shape {
  static_assert(KN == 64 || KN == 128, "64 x 64 or 128 x 128 planes");
  static constexpr int kN = 2 * KN;
  static constexpr int kAB = kRows * kK * 4;                      // bytes of the A operand (TF32)
  static constexpr int kBB = kN * kK * 4;                         // bytes of the B operand
  static constexpr int kOperandBytes = 2 * (kAB + kBB);           // hi and lo of each
  static constexpr int kTmemCols = kN;                            // 128 or 256
  static constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kN >> 3) << 17) |
                                     ((uint32_t)(kRows >> 4) << 24);   // kind::tf32, D = F32, K-major
};

__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// element (row, k) of a 128-byte-swizzled K-major tile, 32 TF32 a row
__device__ __forceinline__ uint32_t* slot(unsigned char* tile, int row, int k) {
  return (uint32_t*)(tile + tc::swz(row, k >> 2)) + (k & 3);
}
// the pair (v0, v1) at columns (k, k + 1), k even: one 8-byte store into each of hi and lo
__device__ __forceinline__ void put_split2(unsigned char* hi, unsigned char* lo, int row, int k, float v0, float v1) {
  const uint32_t h0 = tf32_bits(v0), h1 = tf32_bits(v1);
  *reinterpret_cast<uint2*>(slot(hi, row, k)) = make_uint2(h0, h1);
  *reinterpret_cast<uint2*>(slot(lo, row, k)) =
      make_uint2(tf32_bits(v0 - __uint_as_float(h0)), tf32_bits(v1 - __uint_as_float(h1)));
}
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// The staging, MMAs and bounded wait of site_sums; returns the TMEM address of the product,
// which the caller reads and then frees with tmem_release.  Rows 0..KN-1 of A hold D_s(k2) of
// plane k1A of the target whose site tables start at pairA.  KN = 64: rows 64..127 hold those
// of plane k1B of the target at pairB (zero when k1B < 0).  Two targets take two rounds, each
// with its own B3 and the other half's A rows zero, accumulating in the same TMEM columns.
template <int KN, int NTHR>
__device__ uint32_t site_mma(const float2* __restrict__ tab, size_t pairA, int k1A, size_t pairB, int k1B, int s,
                             int nk, int Kh1, unsigned char* opnd, uint64_t* bar, uint32_t* tmem_slot,
                             int* __restrict__ errflags) {
  using Sh = Shape<KN>;
  using namespace tc;
  constexpr int NI = kTileSites * KN / NTHR;           // staging items of a thread per loop, full tile
  static_assert(NI * NTHR == kTileSites * KN, "whole items per thread");
  constexpr int NB = NI < 4 ? NI : 4;                   // items loaded together (registers)
  const int tid = threadIdx.x, warp = tid >> 5;
  unsigned char* ahi = opnd;
  unsigned char* alo = ahi + Sh::kAB;
  unsigned char* bhi = alo + Sh::kAB;
  unsigned char* blo = bhi + Sh::kBB;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(Sh::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  bool ok = true;
  uint32_t tmem = 0;                                   // read once the first tile's barrier has passed (s >= 1)
  int tile = 0;
  const bool cross = KN == 64 && k1B >= 0 && pairB != pairA;
  for (int round = 0; round < (cross ? 2 : 1); ++round)
  for (int t0 = 0; t0 < s && ok; t0 += kTileSites, ++tile) {
    const bool onA = !cross || round == 0, onB = k1B >= 0 && (!cross || round == 1);
    const size_t pb3 = round == 0 ? pairA : pairB;    // the target whose B3 this round multiplies
    const int ns = min(kTileSites, s - t0);
    // K steps of 8 columns that the tile's sites fill; the columns past 2 ns of the last step are zeroed
    const int nks = (2 * ns + 7) / 8;
    if (2 * ns < 8 * nks) {
      const int k0 = 2 * ns, k1e = 8 * nks;                 // zero columns [k0, k1e), even bounds
      const int per = (k1e - k0) / 2;                       // column pairs a row
      for (int x = tid; x < (kRows + Sh::kN) * per; x += NTHR) {
        const int r = x / per, k = k0 + 2 * (x - r * per);
        if (r < kRows) {
          *reinterpret_cast<uint2*>(slot(ahi, r, k)) = make_uint2(0u, 0u);
          *reinterpret_cast<uint2*>(slot(alo, r, k)) = make_uint2(0u, 0u);
        } else {
          *reinterpret_cast<uint2*>(slot(bhi, r - kRows, k)) = make_uint2(0u, 0u);
          *reinterpret_cast<uint2*>(slot(blo, r - kRows, k)) = make_uint2(0u, 0u);
        }
      }
    }
    if constexpr (KN == 128) {
      // 128 x 128 planes (one target, one plane): consecutive lanes take consecutive k2 and k3,
      // so the table reads are 256-byte runs.  Measured on the 60-site chain, this order keeps
      // the plane stage at 43 ms a frame where the bank-conflict-free order below took 48.
      for (int e = tid; e < ns * KN; e += NTHR) {
        const int t = e / KN, q = e - t * KN;
        const float2* row = tab + (pairA + t0 + t) * nk;
        const float2 d = fft::cmul(row[k1A], row[Kh1 + q]);   // q B1(k1) B2(k2 = q)
        put_split2(ahi, alo, q, 2 * t, d.x, d.y);
        const float2 b3 = row[Kh1 + KN + q];                  // B3(k3 = q)
        put_split2(bhi, blo, 2 * q, 2 * t, b3.x, -b3.y);
        put_split2(bhi, blo, 2 * q + 1, 2 * t, b3.y, b3.x);
      }
    } else {
      // The item orders put the 16 lanes of a half warp on 16 distinct (16-byte chunk, half)
      // slots of the swizzled rows, so the 8-byte stores are free of bank conflicts: a lane's
      // chunk is (t / 2) ^ (row mod 8), its half t mod 2.
      // A rows k2 = q: item bits 0-2 q mod 8, bit 3 t mod 2, bits 4.. q / 8, then t / 2.  Each
      // loop loads NB items of the thread at a time, then splits and stores them, so that the
      // table reads are in flight together.
#pragma unroll 1
      for (int u0 = 0; u0 < NI; u0 += NB) {
        const int lim = ((ns + 1) >> 1) * 2 * KN;
        const bool same = pairB == pairA;
        float2 c1v[NB], b2v[NB], c1w[NB], b2w[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          const int x = tid + (u0 + u) * NTHR;
          const int q = (x & 7) | (((x >> 4) & (KN / 8 - 1)) << 3);
          const int t = ((x >> 3) & 1) | ((x / (2 * KN)) << 1);
          const float2 z = make_float2(0.f, 0.f);
          c1v[u] = z; b2v[u] = z; c1w[u] = z; b2w[u] = z;
          if (x < lim && t < ns) {
            const float2* row = tab + (pairA + t0 + t) * nk;
            b2v[u] = row[Kh1 + q];
            if (onA) c1v[u] = row[k1A];
            if (KN == 64 && onB) {
              const float2* rb = same ? row : tab + (pairB + t0 + t) * nk;
              c1w[u] = rb[k1B];
              if (!same) b2w[u] = rb[Kh1 + q];
            }
          }
        }
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          const int x = tid + (u0 + u) * NTHR;
          const int q = (x & 7) | (((x >> 4) & (KN / 8 - 1)) << 3);
          const int t = ((x >> 3) & 1) | ((x / (2 * KN)) << 1);
          if (x < lim && t < ns) {
            const float2 d = fft::cmul(c1v[u], b2v[u]);       // q B1(k1) B2(k2 = q); zero when off
            put_split2(ahi, alo, q, 2 * t, d.x, d.y);
            if (KN == 64) {
              const float2 e = fft::cmul(c1w[u], same ? b2v[u] : b2w[u]);
              put_split2(ahi, alo, 64 + q, 2 * t, e.x, e.y);
            }
          }
        }
      }
      // B row pairs (2 c2, 2 c2 + 1): item bits 0-1 c2 mod 4, bits 2-3 t mod 4, bits 4.. c2 / 4,
      // then t / 4.  Pair c2 holds k3 = c2.
#pragma unroll 1
      for (int u0 = 0; u0 < NI; u0 += NB) {
        const int lim = ((ns + 3) >> 2) * 4 * KN;
        float2 v[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          const int x = tid + (u0 + u) * NTHR;
          const int c2 = (x & 3) | (((x >> 4) & (KN / 4 - 1)) << 2);
          const int t = ((x >> 2) & 3) | ((x / (4 * KN)) << 2);
          const int k3 = c2;
          v[u] = make_float2(0.f, 0.f);
          if (x < lim && t < ns) v[u] = tab[(pb3 + t0 + t) * nk + Kh1 + KN + k3];
        }
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          const int x = tid + (u0 + u) * NTHR;
          const int c2 = (x & 3) | (((x >> 4) & (KN / 4 - 1)) << 2);
          const int t = ((x >> 2) & 3) | ((x / (4 * KN)) << 2);
          if (x < lim && t < ns) {
            put_split2(bhi, blo, 2 * c2, 2 * t, v[u].x, -v[u].y);
            put_split2(bhi, blo, 2 * c2 + 1, 2 * t, v[u].y, v[u].x);
          }
        }
      }
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    tmem = *tmem_slot;
    if (tid == 0) {
      const uint64_t dah = smem_desc(smem_u32(ahi)), dal = smem_desc(smem_u32(alo));
      const uint64_t dbh = smem_desc(smem_u32(bhi)), dbl = smem_desc(smem_u32(blo));
      for (int ks = 0; ks < nks; ++ks)
        mma(tmem, dah + 2 * ks, dbh + 2 * ks, Sh::kIdesc, (round > 0 || t0 > 0 || ks > 0) ? 1u : 0u);
      for (int ks = 0; ks < nks; ++ks) mma(tmem, dah + 2 * ks, dbl + 2 * ks, Sh::kIdesc, 1u);
      for (int ks = 0; ks < nks; ++ks) mma(tmem, dal + 2 * ks, dbh + 2 * ks, Sh::kIdesc, 1u);
      mma_commit(bar);
    }
    // the tile's MMAs complete before its operands are overwritten or TMEM is read (bounded wait;
    // on expiry the error is flagged and the kernel waits once more, bounded, before going on)
    ok = __syncthreads_and(mbar_wait(bar, (uint32_t)(tile & 1))) != 0;
    if (!ok) {
      if (tid == 0) atomicOr(errflags, kErrTimeout);
      mbar_wait(bar, (uint32_t)(tile & 1));
    }
  }
  tc_fence_after();
  return tmem;
}

// every thread's TMEM reads are complete before warp 0 frees the columns
template <int KN>
__device__ __forceinline__ void tmem_release(uint32_t tmem) {
  tc::tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Shape<KN>::kTmemCols));
}

// X(k3, k2) of plane k1 of the target whose site tables start at pair0, straight into the
// calling thread's registers in the plane kernel's layout: acc[e] = X(k30 + e, k2) with
// k2 = tid mod KN, k30 = E (tid / KN).  The product is X^T: A(k2, 2 s + c) = (Re, Im) of
// D_s(k2) = q B1_s(k1) B2_s(k2); B(2 k3 + p, 2 s + c) = (Re B3, -Im B3) for p = 0 and
// (Im B3, Re B3) for p = 1.  Thread lane l of warp w reads TMEM lane 32 (w mod 4) + l, which
// holds k2 = (32 w + l) mod KN, and the 2 E columns of its k3 range.  `opnd`
// (Shape<KN>::kOperandBytes, 1024-byte aligned) may alias the plane buffer, which this
// function does not write.  NTHR = KN * KN / E threads.
template <int KN, int E, int NTHR>
__device__ void site_sums(const float2* __restrict__ tab, size_t pair0, int s, int nk, int Kh1, int k1, int k30,
                          unsigned char* opnd, uint64_t* bar, uint32_t* tmem_slot, int* __restrict__ errflags,
                          float2 (&acc)[E]) {
  static_assert(NTHR == KN * KN / E && (2 * E) % 32 == 0, "whole 32-column TMEM loads");
  const uint32_t tmem = site_mma<KN, NTHR>(tab, pair0, k1, pair0, k1, s, nk, Kh1, opnd, bar, tmem_slot, errflags);
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 2 * E; c += 32) {
    uint32_t v[32];
    tc::tmem_ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(2 * k30 + c), v);
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[c / 2 + j] = make_float2(__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1]));
  }
  tmem_release<KN>(tmem);
}
}  // namespace tcs

// ---------------------------------------------------------------------------
// k_pme_plane<LK2, LK3, DIRECT>: grid (k1max + 1, targets), K2*K3/E threads.  Thread
// tid owns the points (k2 = tid mod K2, k3 = (tid / K2) * E + e), e < E.
// Solute sites are staged ts at a time from the batch's site tables.
// ---------------------------------------------------------------------------
template <int LK2, int LK3, bool DIRECT, bool TCS = false>
__global__ void __launch_bounds__(PlaneCfg<LK2, LK3>::NTHR, PlaneCfg<LK2, LK3>::MINB) k_pme_plane(FrameArgs a,
    int tbase, int ts, const float2* __restrict__ tab, const float* __restrict__ stn,
    const float* __restrict__ engfacT, const float2* __restrict__ fft_tw, float2* __restrict__ Y,
    double* __restrict__ partial, int* __restrict__ errflags) {
  using C = PlaneCfg<LK2, LK3>;
  constexpr int K2 = C::K2, K3 = C::K3, PITCH = C::PITCH, E = C::E, NTHR = C::NTHR;
  extern __shared__ __align__(16) unsigned char psm[];
  const int k1 = blockIdx.x, b = blockIdx.y;
  const int K1 = a.K1, Kh1 = a.Kh1, s = a.nsite, n = a.order;
  const int nk = Kh1 + (DIRECT ? K2 + K3 : 0);
  const int tid = threadIdx.x;
  float2* tw2 = (float2*)psm;                          // [K2]
  float2* tw3 = tw2 + K2;                              // [K3]
  float2* plane = tw3 + K3;                            // [K3][PITCH]
  float2* c1 = plane + K3 * PITCH;                     // [ts] q_a B1_a(k1), padded to even length
  float2* b2 = c1 + ((ts + 1) & ~1);                   // DIRECT: [ts][K2] (16-byte aligned: K's are even)
  float2* b3 = b2 + (DIRECT ? ts * K2 : 0);            // DIRECT: [ts][K3]
  float* sst = (float*)b3;                             // spreading: [ts][kStn] stencils
  long long* facc = (long long*)(((uintptr_t)(sst + ts * kStn) + 15) & ~(uintptr_t)15);   // spreading: [K3*K2]
  for (int p = tid; p < K2 + K3; p += NTHR) tw2[p] = fft_tw[K1 + p];
  const size_t pair0 = (size_t)(tbase + b) * s;       // first (target, site) pair of this target in the tables
  const int k2 = tid & (K2 - 1), k30 = (tid >> LK2) * E;
  float2 acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = make_float2(0.f, 0.f);
  if constexpr (TCS) {
    static_assert(DIRECT && K2 == K3 && K2 == 128, "tensor-core site sums here: 128 x 128 planes (k_pme_plane_pair: 64)");
    __shared__ __align__(8) uint64_t tcs_bar;
    __shared__ uint32_t tcs_tmem;
    unsigned char* opnd = (unsigned char*)(((uintptr_t)plane + 1023) & ~(uintptr_t)1023);
    tcs::site_sums<K2, E, NTHR>(tab, pair0, s, nk, Kh1, k1, k30, opnd, &tcs_bar, &tcs_tmem, errflags, acc);
  } else if (!DIRECT && C::FIXED) {
    // q_a B1_a(k1) w2 w3 scattered on the (n2, n3) plane: a thread per (site, stencil point),
    // integer atomics in 2^-40 fixed point (exact, order-independent), real then imaginary part
    constexpr double kFix = 1099511627776.0, kUnfix = 1.0 / 1099511627776.0;
    for (int part = 0; part < 2; ++part) {
      __syncthreads();
      for (int p = tid; p < K2 * K3; p += NTHR) facc[p] = 0;
      for (int a0 = 0; a0 < s; a0 += ts) {
        const int nt = min(ts, s - a0);
        __syncthreads();
        for (int x = tid; x < nt; x += NTHR) c1[x] = tab[(pair0 + a0 + x) * nk + k1];
        for (int x = tid; x < nt * kStn; x += NTHR) sst[x] = stn[(pair0 + a0) * kStn + x];
        __syncthreads();
        const int nn = n * n;
        for (int x = tid; x < nt * nn; x += NTHR) {
          const int t = x / nn, c = x - t * nn, c3 = c / n, c2 = c - c3 * n;
          const float* st = sst + t * kStn;
          const float v = (part ? c1[t].y : c1[t].x) * st[2 + c2] * st[2 + kMaxOrder + c3];
          const int n2 = ((int)st[0] - c2) & (K2 - 1), n3 = ((int)st[1] - c3) & (K3 - 1);
          atomicAdd((unsigned long long*)&facc[n3 * K2 + n2], (unsigned long long)__double2ll_rn((double)v * kFix));
        }
      }
      __syncthreads();
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float v = (float)((double)facc[(k30 + e) * K2 + k2] * kUnfix);
        if (part) acc[e].y = v; else acc[e].x = v;
      }
    }
  } else {
    for (int a0 = 0; a0 < s; a0 += ts) {
      const int nt = min(ts, s - a0);
      __syncthreads();
      for (int x = tid; x < nt; x += NTHR) c1[x] = tab[(pair0 + a0 + x) * nk + k1];
      if (DIRECT) {
        // B2 then B3 of each site: K2 + K3 consecutive table entries, kLoadBatch loads in flight
        const int per = K2 + K3, tot = nt * per;
        for (int x0 = 0; x0 < tot; x0 += kLoadBatch * NTHR) {
          float2 v[kLoadBatch];
#pragma unroll
          for (int u = 0; u < kLoadBatch; ++u) {
            const int x = x0 + u * NTHR + tid;
            if (x < tot) v[u] = tab[(pair0 + a0 + x / per) * nk + Kh1 + x % per];
          }
#pragma unroll
          for (int u = 0; u < kLoadBatch; ++u) {
            const int x = x0 + u * NTHR + tid;
            if (x < tot) {
              const int t = x / per, r = x - t * per;
              if (r < K2) b2[t * K2 + r] = v[u];
              else b3[t * K3 + r - K2] = v[u];
            }
          }
        }
      } else {
        for (int x = tid; x < nt * kStn; x += NTHR) sst[x] = stn[(pair0 + a0) * kStn + x];
      }
      __syncthreads();
      if (DIRECT) {
        for (int t = 0; t < nt; ++t) {
          const float2 c = cmul(c1[t], b2[t * K2 + k2]);
          const float4* bt = (const float4*)(b3 + t * K3 + k30);   // two k3 per 16-byte load
#pragma unroll
          for (int e = 0; e < E; e += 2) {
            const float4 u = bt[e / 2];
            acc[e].x += c.x * u.x - c.y * u.y;
            acc[e].y += c.x * u.y + c.y * u.x;
            acc[e + 1].x += c.x * u.z - c.y * u.w;
            acc[e + 1].y += c.x * u.w + c.y * u.z;
          }
        }
      } else {
        // large planes: q_a B1_a(k1) w2 w3 accumulated in site order by the point's owner
        for (int t = 0; t < nt; ++t) {
          const float* st = sst + t * kStn;
          const int c2 = ((int)st[0] - k2) & (K2 - 1);
          if (c2 >= n) continue;
          const int g3 = (int)st[1];
          if (((g3 - k30) & (K3 - 1)) >= E + n - 1) continue;   // the site's rows miss this thread's rows
          const float2 c = c1[t];
          const float w2 = st[2 + c2];
          const float2 f = make_float2(c.x * w2, c.y * w2);
          const float* w3 = st + 2 + kMaxOrder;
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const int c3 = (g3 - (k30 + e)) & (K3 - 1);
            if (c3 < n) {
              acc[e].x += f.x * w3[c3];
              acc[e].y += f.y * w3[c3];
            }
          }
        }
      }
    }
  }
  // (DIRECT) acc holds Qhat(k1, k2, k3); otherwise the k1-transformed plane, still in (n2, n3)
  using Rows = FftShape<LK2, LK3, 30, 0, PITCH, 1>;
  using Cols = FftShape<LK3, LK2, 30, 0, 1, PITCH>;
  float2* own = plane + k30 * PITCH + k2;
  if (!DIRECT) {
#pragma unroll
    for (int e = 0; e < E; ++e) own[e * PITCH] = acc[e];
    __syncthreads();
    fft_batch<Rows, NTHR, false>(plane, tw2, tid);
    fft_batch<Cols, NTHR, false>(plane, tw3, tid);
#pragma unroll
    for (int e = 0; e < E; ++e) acc[e] = own[e * PITCH];
  }
  // influence function and the plane's share of the self energy (recpcal.F90:482-497);
  // each mode's G |Qhat|^2 is formed in FP32 (~1e-7 relative) and summed in FP64
  double self = 0.0;
  const float* gk = engfacT + ((size_t)k1 * K3 + k30) * K2 + k2;
  float g[E];
#pragma unroll
  for (int e = 0; e < E; ++e) g[e] = gk[e * K2];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    self += (double)(g[e] * (acc[e].x * acc[e].x + acc[e].y * acc[e].y));
    own[e * PITCH] = make_float2(acc[e].x * g[e], acc[e].y * g[e]);
  }
  if (k1 == 0 || 2 * k1 == K1) self *= 0.5;
  __syncthreads();
  fft_batch<Rows, NTHR, true>(plane, tw2, tid);
  fft_batch<Cols, NTHR, true>(plane, tw3, tid);
  grid_dep_launch();                                  // the k1 transform may start filling the tail
  float2* y = Y + ((size_t)b * Kh1 + k1) * K3 * K2;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int p = tid + e * NTHR;
    y[p] = plane[(p >> LK2) * PITCH + (p & (K2 - 1))];
  }
  // the plane's share of the self energy, reduced in a fixed order; the k1 transform sums
  // the planes of each target (self_energy_sum)
  __shared__ double red[32];
  self = warp_sum(self);
  if ((tid & 31) == 0) red[tid >> 5] = self;
  __syncthreads();
  if (tid < 32) {
    double v = tid < (NTHR >> 5) ? red[tid] : 0.0;
    v = warp_sum(v);
    if (tid == 0) partial[(size_t)b * Kh1 + k1] = v;
  }
  // Launched behind the previous chunk's gather, which reads the potential grid that this
  // chunk's k1 transform overwrites: this grid does not complete before that gather has.
  grid_dep_wait();
}

// ---------------------------------------------------------------------------
// k_pme_plane_pair<LK>: two planes per CTA, K x K planes (K = 2^LK = 64), 2K threads.  The
// chunk's planes (target b, k1 <= k1max) are numbered p = b (k1max + 1) + k1 and CTA c takes
// p = 2c and 2c + 1, so a chunk of 32 targets is at most 32 (k1max + 1) / 2 CTAs, one resident
// wave at 3 CTAs per SM for k1max < 27.  B3 does not depend on k1, so one tensor-core product
// serves two planes of a target: A rows 0..63 hold D(k2) of the first plane, rows 64..127
// those of the second (zero past the chunk's last plane); a pair that spans two targets takes
// two rounds (tcs::site_mma).  TMEM lane quarter w holds the rows that warp w reads.
// Thread (half = tid / K, k2 = tid mod K) takes all K of its column from TMEM, applies G,
// and transforms the column in registers (idft64_reg); one transpose through shared memory
// hands each thread a row n3 for the second axis, and the rows go back through shared
// memory so that each warp store is one 256-byte row of Y.
// Grid ceil(targets (k1max + 1) / 2).
// ---------------------------------------------------------------------------
template <int LK>
__global__ void __launch_bounds__(2 << LK, 3) k_pme_plane_pair(FrameArgs a, int tbase, int nb,
    const float2* __restrict__ tab, const float* __restrict__ engfacT, Tw64 t64, float2* __restrict__ Y,
    double* __restrict__ partial, int* __restrict__ errflags) {
  constexpr int K = 1 << LK, NTHR = 2 * K, P = K + 1;
  static_assert(K == 64, "64 x 64 planes");
  extern __shared__ __align__(16) unsigned char psm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int half = tid >> LK, i = tid & (K - 1);          // plane of the pair; column k2, later row n3
  const int kp = a.k1max + 1, p0 = 2 * blockIdx.x;
  const bool has1 = p0 + 1 < nb * kp;
  const int b0 = p0 / kp, k1a = p0 - b0 * kp;
  const int b1 = has1 ? (p0 + 1) / kp : b0, k1b = has1 ? p0 + 1 - b1 * kp : -1;
  const bool live = half == 0 || has1;
  const int b = half ? b1 : b0, k1 = half && has1 ? k1b : k1a;
  const int Kh1 = a.Kh1, s = a.nsite, nk = Kh1 + 2 * K;
  unsigned char* opnd = (unsigned char*)(((uintptr_t)psm + 1023) & ~(uintptr_t)1023);
  float2* xp = (float2*)opnd + half * K * P;              // this plane's [n][P], over the dead operands
  float gv[K];                                            // G of column k2, prefetched during the staging
  {
    const float* gk = engfacT + (size_t)k1 * K * K + i;
#pragma unroll
    for (int e = 0; e < K; ++e) gv[e] = gk[(size_t)e * K];
  }
  __shared__ __align__(8) uint64_t tcs_bar;
  __shared__ uint32_t tcs_tmem;
  const uint32_t tmem =
      tcs::site_mma<K, NTHR>(tab, (size_t)(tbase + b0) * s, k1a, (size_t)(tbase + b1) * s, k1b, s, nk, Kh1,
                             opnd, &tcs_bar, &tcs_tmem, errflags);
  // influence function and the plane's share of the self energy (recpcal.F90:482-497);
  // each mode's G |Qhat|^2 is formed in FP32 (~1e-7 relative) and summed in FP64
  float2 z[K];
  double self = 0.0;
#pragma unroll
  for (int c = 0; c < 2 * K; c += 32) {
    uint32_t v[32];
    tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int k3 = c / 2 + j;
      const float xr = __uint_as_float(v[2 * j]), xi = __uint_as_float(v[2 * j + 1]), g = gv[k3];
      self += (double)(g * (xr * xr + xi * xi));
      z[k3] = make_float2(xr * g, xi * g);
    }
  }
  if (k1 == 0 || 2 * k1 == a.K1) self *= 0.5;
  tcs::tmem_release<K>(tmem);                             // also: every thread is past the MMAs
  idft64_reg(z, t64);                                     // column k2: n3 = 4 c + d at z[16 d + c]
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 16; ++c) xp[(4 * c + d) * P + i] = z[16 * d + c];
  __syncthreads();
#pragma unroll
  for (int k2 = 0; k2 < K; ++k2) z[k2] = xp[i * P + k2];  // row n3 = i
  idft64_reg(z, t64);                                     // n2 = 4 c + d at z[16 d + c]
  __syncthreads();
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 16; ++c) xp[i * P + 4 * c + d] = z[16 * d + c];
  __syncthreads();
  grid_dep_launch();                                      // the k1 transform may start filling the tail
  if (live) {
    float2* y = Y + ((size_t)b * Kh1 + k1) * K * K + i;
#pragma unroll 8
    for (int e = 0; e < K; ++e) y[(size_t)e * K] = xp[e * P + i];
  }
  // each plane's share of the self energy over its two warps, in a fixed order; the k1
  // transform sums the planes of each target (self_energy_sum)
  __shared__ double red[NTHR / 32];
  self = warp_sum(self);
  if ((tid & 31) == 0) red[warp] = self;
  __syncthreads();
  if (i == 0 && live) partial[(size_t)b * Kh1 + k1] = red[2 * half] + red[2 * half + 1];
  // Launched behind the previous chunk's gather, which reads the potential grid that this
  // chunk's k1 transform overwrites: this grid does not complete before that gather has.
  grid_dep_wait();
}

// selfrec[base + b] = sum over the planes k1 <= k1max of target b's shares, in
// plane order.  Run by the first CTA of the k1 transform: every plane of the
// chunk is complete by then.
__device__ __forceinline__ void self_energy_sum(const FrameArgs& a, int base, int nb, int Kh1,
                                                const double* __restrict__ partial, double* __restrict__ selfrec) {
  if (blockIdx.x != 0 || blockIdx.y != 0 || (int)threadIdx.x >= nb) return;
  const int b = threadIdx.x;
  double sum = 0.0;
  for (int k1 = 0; k1 <= a.k1max; ++k1) sum += partial[(size_t)b * Kh1 + k1];
  selfrec[base + b] = sum;
}

// ---------------------------------------------------------------------------
// k_pme_rows<LM>: grid (K3, K2 / G2), kRowThreads threads, G2 = 256 / M rows
// of n2 for all 32 targets; M = K1 / 2 = 2^LM.  Shared rows k1 = 0..M hold
// Y[b][k1][n3][n2] at column (n2 - n2g) * 33 + b.
// ---------------------------------------------------------------------------
template <int LM>
__global__ void __launch_bounds__(kRowThreads, 2) k_pme_rows(FrameArgs a, int base, int nb, const float2* __restrict__ Y,
    const float2* __restrict__ fft_tw, const double* __restrict__ partial, double* __restrict__ selfrec,
    float* __restrict__ phi) {
  constexpr int M = 1 << LM, K1 = 2 * M, Kh1 = M + 1;
  constexpr int G2 = 256 / M, LG2 = 8 - LM, T = 32 * G2, LT = LG2 + 5, TP = G2 * 33;
  extern __shared__ __align__(16) unsigned char rsm[];
  const int K2 = a.K2, K3 = a.K3;
  const int n3 = blockIdx.x, n2g = blockIdx.y * G2;
  const int tid = threadIdx.x;
  grid_dep_wait();
  self_energy_sum(a, base, nb, Kh1, partial, selfrec);
  float2* twk = (float2*)rsm;          // [K1] exp(-2 pi i m / K1)
  float2* twm = twk + K1;              // [M]  exp(-2 pi i m / M)
  float2* S = twm + M;                 // [Kh1][TP]
  for (int p = tid; p < K1; p += kRowThreads) twk[p] = fft_tw[p];
  for (int p = tid; p < M; p += kRowThreads) twm[p] = fft_tw[K1 + K2 + K3 + p];
  // stage Y with kLoadBatch independent loads in flight per thread
  constexpr int total = T * Kh1;
  for (int x0 = 0; x0 < total; x0 += kLoadBatch * kRowThreads) {
    float2 v[kLoadBatch];
    int dst[kLoadBatch];
#pragma unroll
    for (int u = 0; u < kLoadBatch; ++u) {
      const int x = x0 + u * kRowThreads + tid;
      dst[u] = -1;
      v[u] = make_float2(0.f, 0.f);
      if (x < total) {
        const int j = x & (G2 - 1), r = x >> LG2;   // r = k1 * 32 + b
        const int b = r & 31, k1 = r >> 5;
        dst[u] = k1 * TP + j * 33 + b;
        if (b < nb && k1 <= a.k1max) v[u] = Y[(((size_t)b * Kh1 + k1) * K3 + n3) * K2 + n2g + j];
      }
    }
#pragma unroll
    for (int u = 0; u < kLoadBatch; ++u)
      if (dst[u] >= 0) S[dst[u]] = v[u];
  }
  __syncthreads();
  // Hermitian packing into a length-M complex sequence Z (rows 0..M-1):
  //   Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) exp(+2 pi i k / K1)
  // so that x[2n] = Re z[n], x[2n+1] = Im z[n] for z = inverse DFT_M(Z).
  for (int x = tid; x < T * (M / 2 + 1); x += kRowThreads) {
    const int t = x & (T - 1), k = x >> LT;
    const int c = (t >> 5) * 33 + (t & 31);
    float2 xk = S[k * TP + c], xm = S[(M - k) * TP + c];
    if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
    {
      const float2 cm = make_float2(xm.x, -xm.y);
      const float2 w = make_float2(twk[k].x, -twk[k].y);
      const float2 d = cmul(csub(xk, cm), w);
      S[k * TP + c] = make_float2(xk.x + cm.x - d.y, xk.y + cm.y + d.x);
    }
    if (k != 0 && 2 * k != M) {
      const float2 ck = make_float2(xk.x, -xk.y);
      const float2 w = make_float2(twk[M - k].x, -twk[M - k].y);
      const float2 d = cmul(csub(xm, ck), w);
      S[(M - k) * TP + c] = make_float2(xm.x + ck.x - d.y, xm.y + ck.y + d.x);
    }
  }
  __syncthreads();
  fft_batch<FftShape<LM, LT, 5, 33, 1, TP>, kRowThreads, true>(S, twm, tid);
  // phi in n1 pairs: z[n] = (phi(2n), phi(2n+1)) of line (n3 K2 + n2g + j), target b
  float2* out = (float2*)phi + ((size_t)n3 * K2 + n2g) * M * kChunk;
  for (int x = tid; x < T * M; x += kRowThreads) {
    const int b = x & 31, r = x >> 5;
    const int n = r & (M - 1), j = r >> LM;
    out[((size_t)j * M + n) * kChunk + b] = S[n * TP + j * 33 + b];
  }
}

// ---------------------------------------------------------------------------
// k_pme_lines<LM>: the same transform for K1 = 2M <= 64, a thread per line.
// Grid (K3, K2 / kLineRows), 32 * kLineRows threads; warp j takes row
// n2 = blockIdx.y * kLineRows + j, lane b the target.  The CTA first stages
// the half spectra Y[b][k1][n3][n2], k1 <= k1max, of its kLineRows rows and
// 32 targets in shared memory (16-byte loads along n2), each line's k1 run
// contiguous: S[j JP + b LP + k1], LP = M + 2, JP = 32 LP + 4.  With these
// pitches a half warp's 8-byte staging stores and a quarter warp's 16-byte
// line reads fall on distinct banks, and a thread reads its line in M / 2 + 1
// 16-byte loads.  Each thread then packs its line (hermitian_pack), transforms
// it in registers (idft_reg) and writes the line's M pairs (phi(2n), phi(2n+1)):
// every store of a warp is one 256-byte row of the insertion-fastest layout.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int line_lp(int M) { return M + 2; }
__host__ __device__ constexpr int line_jp(int M) { return 32 * line_lp(M) + 4; }

size_t lines_smem(int M) { return sizeof(float2) * (size_t)kLineRows * line_jp(M); }

template <int LM>
__global__ void __launch_bounds__(32 * kLineRows, 2) k_pme_lines(FrameArgs a, int base, int nb,
    const float2* __restrict__ Y, Tw64 tw, const double* __restrict__ partial, double* __restrict__ selfrec,
    float* __restrict__ phi) {
  constexpr int M = 1 << LM, K1 = 2 * M, Kh1 = M + 1, NT = 32 * kLineRows;
  constexpr int LP = line_lp(M), JP = line_jp(M);
  static_assert(kLineRows == 4, "staging items: 2 row pairs x 2 k1 x 32 targets per 128 threads");
  extern __shared__ __align__(16) float2 S[];              // [kLineRows][32][LP] + pads
  const int K2 = a.K2, K3 = a.K3;
  const int tid = threadIdx.x;
  const int n3 = blockIdx.x, n2g = blockIdx.y * kLineRows;
  const size_t plane = (size_t)K3 * K2;
  const int kmax = a.k1max;
  grid_dep_wait();                                    // the planes of this chunk are complete
  self_energy_sum(a, base, nb, Kh1, partial, selfrec);
  {
    // staging item (u, x = tid): rows 2q, 2q + 1 of target bs at k1 = 2u + kp, one float4;
    // q = x mod 2, kp = bit 1, bs = bits 2-6, so a warp's loads are 16 whole 32-byte sectors
    const int q = tid & 1, kp = (tid >> 1) & 1, bs = ((tid >> 2) & 7) | (((tid >> 5) & 3) << 3);
    const bool on = bs < nb;
    const float4* src = (const float4*)(Y + (size_t)bs * Kh1 * plane + (size_t)n3 * K2 + n2g + 2 * q);
    float2* dst = S + (2 * q) * JP + bs * LP;
    // every load is issued before the first store, from a clamped (always valid) k1, so that
    // they are all in flight together; rows above k1max and targets past nb are not used
    constexpr int NPASS = (M + 2) / 2;                      // k1 = 0..M+1 in pairs
    static_assert(NT == 128, "one k1 pair per pass");
    float4 v[NPASS];
#pragma unroll
    for (int u = 0; u < NPASS; ++u) v[u] = __ldg(src + (size_t)min(2 * u + kp, kmax) * (plane / 2));
#pragma unroll
    for (int u = 0; u < NPASS; ++u) {
      const int k1 = 2 * u + kp;
      if (k1 <= kmax && k1 <= M) {
        const float4 t = on ? v[u] : make_float4(0.f, 0.f, 0.f, 0.f);
        dst[k1] = make_float2(t.x, t.y);
        dst[JP + k1] = make_float2(t.z, t.w);
      }
    }
  }
  __syncthreads();
  grid_dep_launch();                                  // the gather may start filling the tail
  const int b = tid & 31, j = tid >> 5;
  const float4* line = reinterpret_cast<const float4*>(S + j * JP + b * LP);
  float2 Z[M];
#pragma unroll
  for (int kk = 0; kk < M / 2; ++kk) {
    const float4 w = line[kk];
    Z[2 * kk] = 2 * kk <= kmax ? make_float2(w.x, w.y) : make_float2(0.f, 0.f);
    Z[2 * kk + 1] = 2 * kk + 1 <= kmax ? make_float2(w.z, w.w) : make_float2(0.f, 0.f);
  }
  float2 xM = make_float2(0.f, 0.f);
  if (M <= kmax) {
    const float4 w = line[M / 2];
    xM = make_float2(w.x, w.y);
  }
  hermitian_pack<LM>(Z, xM, tw);
  idft_reg<LM>(Z, tw);
  // z[n] = (phi(2n), phi(2n+1)): one 8-byte store per pair, a 256-byte row per warp
  float2* o = (float2*)phi + (size_t)(n3 * K2 + n2g + j) * M * kChunk + b;
#pragma unroll
  for (int n = 0; n < M; ++n) o[n * kChunk] = Z[n];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
Tw64 make_tw64() {
  Tw64 t;
  for (int m = 0; m < 64; ++m) {
    const double ang = 2.0 * kPi * (double)m / 64.0;
    t.w[m] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
  }
  return t;
}

bool pow2_in(int k, int lo, int hi) { return k >= lo && k <= hi && (k & (k - 1)) == 0; }
int lg(int k) { int l = 0; while ((1 << l) < k) ++l; return l; }

int plane_elems(const FrameArgs& a) { return a.K2 * a.K3 <= 4096 ? 16 : 32; }

int site_tile(const FrameArgs& a) { return std::min(a.nsite, kSiteTile); }
int site_table_entries(const FrameArgs& a, bool direct) { return a.Kh1 + (direct ? a.K2 + a.K3 : 0); }

size_t plane_smem(const FrameArgs& a, bool direct) {
  const size_t ts = site_tile(a), tsa = (ts + 1) & ~(size_t)1;
  const size_t pts = (size_t)a.K2 * a.K3;
  const size_t tile = sizeof(float2) * tsa + (direct ? sizeof(float2) * ts * (a.K2 + a.K3)
                                                     : sizeof(float) * ts * kStn + 16 + (pts <= 8192 ? 8 * pts : 0));
  return sizeof(float2) * (size_t)(a.K2 + a.K3) + sizeof(float2) * (size_t)a.K3 * (a.K2 + 1) + tile;
}

// the tensor-core site-sum variant (64 x 64 planes): twiddles, then the plane or the TF32
// operands aliased over it, 1024-byte aligned
template <int KN>
size_t plane_smem_tcs() {
  const size_t plane = sizeof(float2) * KN * (KN + 1);
  return sizeof(float2) * 2 * KN + 1024 + std::max(plane, (size_t)tcs::Shape<KN>::kOperandBytes);
}

// k_pme_plane_pair<LK>: the TF32 operands and, aliased over them, the two planes' K (K + 1)
// float2 rows, 1024-byte aligned
template <int LK>
size_t plane_smem_pair() {
  constexpr int K = 1 << LK;
  const size_t rows = sizeof(float2) * (size_t)(2 * K * (K + 1));
  return 1024 + std::max(rows, (size_t)tcs::Shape<K>::kOperandBytes);
}

size_t rows_smem(const FrameArgs& a) {
  const int M = a.K1 / 2, G2 = 256 / M;
  return sizeof(float2) * (size_t)(a.K1 + M) + sizeof(float2) * (size_t)a.Kh1 * G2 * 33;
}

// Compile-time plane sizes: every (K2, K3) in {16..128}^2 with K2 K3 >= 512.
#define ERM_PLANE_SIZES(X) \
  X(4, 5) X(4, 6) X(4, 7) X(5, 4) X(5, 5) X(5, 6) X(5, 7) X(6, 4) X(6, 5) X(6, 6) X(6, 7) X(7, 4) X(7, 5) X(7, 6) X(7, 7)

template <int L2, int L3>
cudaError_t plane_attr(const FrameArgs& a) {
  cudaError_t e = raise_smem_limit(k_pme_plane<L2, L3, true>, plane_smem(a, true));
  if (e == cudaSuccess) e = raise_smem_limit(k_pme_plane<L2, L3, false>, plane_smem(a, false));
  if constexpr (L2 == 7 && L3 == 7)
    if (e == cudaSuccess) e = raise_smem_limit(k_pme_plane<L2, L3, true, true>, plane_smem_tcs<(1 << L2)>());
  if constexpr (L2 == 6 && L3 == 6)
    if (e == cudaSuccess) e = raise_smem_limit(k_pme_plane_pair<6>, plane_smem_pair<6>());
  return e;
}

template <int L2, int L3>
void plane_launch(const FrameArgs& a, const DeviceState& d, int tbase, int nb, bool direct, bool pdl, cudaStream_t s) {
  using C = PlaneCfg<L2, L3>;
  const dim3 grid(a.k1max + 1, nb);   // planes above k1max carry no influence-function weight
  const int ts = site_tile(a);
  int* err = d.status ? &d.status->flags : nullptr;
  if constexpr (L2 == 6 && L3 == 6) {
    if (direct && a.nsite <= tcs::kMaxSites) {   // site sums on the tensor cores, two planes per CTA
      static const Tw64 t64 = make_tw64();
      const int npairs = (nb * (a.k1max + 1) + 1) / 2;
      launch_k(pdl, dim3(npairs), 2 << L2, plane_smem_pair<6>(), s, k_pme_plane_pair<6>, a, tbase, nb,
               (const float2*)d.sitetab, (const float*)d.engfacT, t64, d.spec, d.partial, err);
      return;
    }
  }
  if constexpr (L2 == 7 && L3 == 7) {
    if (direct && a.nsite <= tcs::kMaxSites) {   // site sums on the tensor cores
      launch_k(pdl, grid, C::NTHR, plane_smem_tcs<(1 << L2)>(), s, k_pme_plane<L2, L3, true, true>, a, tbase, ts,
               (const float2*)d.sitetab, (const float*)d.sitestn, (const float*)d.engfacT,
               (const float2*)d.fft_tw, d.spec, d.partial, err);
      return;
    }
  }
  if (direct)
    launch_k(pdl, grid, C::NTHR, plane_smem(a, true), s, k_pme_plane<L2, L3, true>, a, tbase, ts,
             (const float2*)d.sitetab, (const float*)d.sitestn, (const float*)d.engfacT, (const float2*)d.fft_tw,
             d.spec, d.partial, err);
  else
    launch_k(pdl, grid, C::NTHR, plane_smem(a, false), s, k_pme_plane<L2, L3, false>, a, tbase, ts,
             (const float2*)d.sitetab, (const float*)d.sitestn, (const float*)d.engfacT, (const float2*)d.fft_tw,
             d.spec, d.partial, err);
}
}  // namespace

bool fused_supported(const FrameArgs& a) {
  if (!a.pme) return false;
  if (!pow2_in(a.K1, 16, 128) || !pow2_in(a.K2, 16, 128) || !pow2_in(a.K3, 16, 128)) return false;
  const int M = a.K1 / 2, G2 = 256 / M;
  if (G2 > a.K2) return false;                       // one CTA of k_pme_rows spans G2 rows of n2
  if (a.K2 * a.K3 < 512) return false;               // at least 32 threads per plane
  if (a.K3 % plane_elems(a) != 0) return false;      // a thread owns E consecutive k3
  return plane_smem(a, true) <= 220 * 1024 && plane_smem(a, false) <= 220 * 1024 && rows_smem(a) <= 220 * 1024;
}

int setup_fused(const FrameArgs& a) {
  if (!fused_supported(a)) return -1;
  const int l2 = lg(a.K2), l3 = lg(a.K3);
  cudaError_t e = cudaErrorInvalidValue;
#define ERM_ATTR(L2, L3) if (l2 == L2 && l3 == L3) e = plane_attr<L2, L3>(a);
  ERM_PLANE_SIZES(ERM_ATTR)
#undef ERM_ATTR
  if (e != cudaSuccess) return -1;
  const int lm = lg(a.K1 / 2);
  const int sm = (int)rows_smem(a);
  if (lm == 3) e = raise_smem_limit(k_pme_lines<3>, lines_smem(8));
  if (lm == 4) e = raise_smem_limit(k_pme_lines<4>, lines_smem(16));
  if (lm == 5) e = raise_smem_limit(k_pme_lines<5>, lines_smem(32));
  if (lm == 6) e = raise_smem_limit(k_pme_rows<6>, (size_t)sm);
  return e == cudaSuccess ? 0 : -1;
}

size_t fused_sitetab_elems(const FrameArgs& a, int batch, bool direct) {
  return (size_t)batch * a.nsite * site_table_entries(a, direct);
}
size_t fused_sitestn_elems(const FrameArgs& a, int batch) { return (size_t)batch * a.nsite * kStn; }

void fused_twiddles(int K1, int K2, int K3, std::vector<float2>& tw, std::vector<double2>& twd) {
  // tw:  [K1 | K2 | K3 | K1/2] tables of exp(-2 pi i m / N), FP64 rounded to FP32
  // twd: [K1 | K2 | K3] the same in FP64
  tw.clear();
  twd.clear();
  const int Ns[4] = {K1, K2, K3, K1 / 2};
  for (int t = 0; t < 4; ++t)
    for (int m = 0; m < Ns[t]; ++m) {
      const double ang = 2.0 * kPi * (double)m / (double)Ns[t];
      const double c = std::cos(ang), sn = -std::sin(ang);
      tw.push_back(make_float2((float)c, (float)sn));
      if (t < 3) twd.push_back(make_double2(c, sn));
    }
}

void launch_site_tables(const FrameArgs& a, const DeviceState& d, int bb, int nbatch, bool direct, cudaStream_t s) {
  const int npairs = nbatch * a.nsite;
  k_site_tables<<<(npairs + kTabPairs - 1) / kTabPairs, 256, 0, s>>>(a, bb, npairs, site_table_entries(a, direct),
                                                                     d.tgt_raw, d.fft_twd, d.sitetab,
                                                                     direct ? nullptr : d.sitestn);
}

void launch_pme_plane(const FrameArgs& a, const DeviceState& d, int tbase, int nb, bool direct, bool pdl,
                      cudaStream_t s) {
  const int l2 = lg(a.K2), l3 = lg(a.K3);
#define ERM_LAUNCH(L2, L3) if (l2 == L2 && l3 == L3) plane_launch<L2, L3>(a, d, tbase, nb, direct, pdl, s);
  ERM_PLANE_SIZES(ERM_LAUNCH)
#undef ERM_LAUNCH
}

void launch_pme_rows(const FrameArgs& a, const DeviceState& d, int base, int nb, bool pdl, cudaStream_t s) {
  static const Tw64 tw = make_tw64();
  const dim3 lgrid(a.K3, a.K2 / kLineRows);
  switch (lg(a.K1 / 2)) {
    case 3:
      launch_k(pdl, lgrid, 32 * kLineRows, lines_smem(1 << 3), s, k_pme_lines<3>, a, base, nb, (const float2*)d.spec,
               tw, (const double*)d.partial, d.selfrec, d.phi);
      return;
    case 4:
      launch_k(pdl, lgrid, 32 * kLineRows, lines_smem(1 << 4), s, k_pme_lines<4>, a, base, nb, (const float2*)d.spec,
               tw, (const double*)d.partial, d.selfrec, d.phi);
      return;
    case 5:
      launch_k(pdl, lgrid, 32 * kLineRows, lines_smem(1 << 5), s, k_pme_lines<5>, a, base, nb, (const float2*)d.spec,
               tw, (const double*)d.partial, d.selfrec, d.phi);
      return;
    default: break;
  }
  const int M = a.K1 / 2, G2 = 256 / M;
  const dim3 grid(a.K3, a.K2 / G2);
  const size_t sm = rows_smem(a);
  switch (lg(M)) {
    default: k_pme_rows<6><<<grid, kRowThreads, sm, s>>>(a, base, nb, d.spec, d.fft_tw, d.partial, d.selfrec, d.phi); break;
  }
}

}  // namespace erm
