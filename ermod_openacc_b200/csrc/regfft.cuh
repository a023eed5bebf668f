// regfft.cuh -- complex arithmetic and short DFTs on float2 values, for the
// fused PME kernels.  Everything is __host__ __device__ and header-only so the
// same code runs in a host test against a direct DFT.
#pragma once

#include <cuda_runtime.h>

namespace erm {
namespace fft {

#define ERM_HD __host__ __device__ __forceinline__

constexpr float kRsqrt2 = 0.70710678118654752f;

ERM_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
ERM_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
ERM_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
ERM_HD float2 conj(float2 a) { return make_float2(a.x, -a.y); }

// a * (+i) for the inverse direction, a * (-i) for the forward one
template <bool INV>
ERM_HD float2 rot90(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// X[q] = sum_r v[r] w^(rq), w = exp(-+2 pi i / 4)
template <bool INV>
ERM_HD void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
  const float2 a0 = cadd(v0, v2), a1 = csub(v0, v2);
  const float2 b0 = cadd(v1, v3), b1 = rot90<INV>(csub(v1, v3));
  v0 = cadd(a0, b0);
  v2 = csub(a0, b0);
  v1 = cadd(a1, b1);
  v3 = csub(a1, b1);
}

// X[q] = sum_r v[r] w^(rq), w = exp(-+2 pi i / R), in place
template <int R, bool INV>
ERM_HD void dft(float2 (&v)[R]) {
  static_assert(R == 4 || R == 8, "radix 4 or 8");
  if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else {
    // radix 8 as two radix-4 transforms of the even and odd inputs
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // o_q *= w8^q, w8 = exp(-+2 pi i / 8)
    const float s = INV ? 1.f : -1.f;
    o1 = make_float2((o1.x - s * o1.y) * kRsqrt2, (o1.y + s * o1.x) * kRsqrt2);
    o2 = rot90<INV>(o2);
    o3 = make_float2((-o3.x - s * o3.y) * kRsqrt2, (-o3.y + s * o3.x) * kRsqrt2);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
  }
}

// exp(-2 pi i m / 64), m < 64, FP64 values rounded to FP32: the twiddles of
// every power-of-two length up to 64.  Passed to kernels by value, so that
// compile-time indices become constant-bank operands.
struct Tw64 {
  float2 w[64];
};

// exp(+2 pi i m / N) for N dividing 64
template <int N>
ERM_HD float2 wplus(const Tw64& t, int m) {
  static_assert(N >= 1 && N <= 64 && (64 % N) == 0, "N divides 64");
  return conj(t.w[(m & (N - 1)) * (64 / N)]);
}

// In-register inverse DFT of length M = 2^LM, 3 <= LM <= 5:
//   z[n] = sum_k Z[k] exp(+2 pi i k n / M), in place, unnormalised.
// M = P * 4 (P = M / 4; M = 8 is a single radix-8 DFT): with k = 4 ka + kb
// and n = na + P nb,
//   z[na + P nb] = sum_kb exp(2 pi i kb nb / 4) w_M^(kb na) sum_ka Z[4 ka + kb] exp(2 pi i ka na / P).
template <int LM>
ERM_HD void idft_reg(float2 (&Z)[1 << LM], const Tw64& t) {
  static_assert(LM >= 3 && LM <= 5, "lengths 8, 16, 32");
  constexpr int M = 1 << LM;
  if constexpr (M == 8) {
    dft<8, true>(Z);
  } else {
    constexpr int Q = 4, P = M / Q;
    float2 A[Q][P];
#pragma unroll
    for (int kb = 0; kb < Q; ++kb) {
      float2 v[P];
#pragma unroll
      for (int ka = 0; ka < P; ++ka) v[ka] = Z[Q * ka + kb];
      dft<P, true>(v);
#pragma unroll
      for (int na = 0; na < P; ++na) A[kb][na] = (kb == 0 || na == 0) ? v[na] : cmul(v[na], wplus<M>(t, kb * na));
    }
#pragma unroll
    for (int na = 0; na < P; ++na) {
      float2 u[Q];
#pragma unroll
      for (int kb = 0; kb < Q; ++kb) u[kb] = A[kb][na];
      dft<Q, true>(u);
#pragma unroll
      for (int nb = 0; nb < Q; ++nb) Z[na + P * nb] = u[nb];
    }
  }
}

// In-register inverse DFT of length 64, unnormalised, with the outputs in a 4 x 16 order:
//   x(4 c + d) = sum_k Z[k] exp(+2 pi i k (4 c + d) / 64) is left in Z[16 d + c].
// One radix-4 step over k = a + 16 b (b < 4) with the twiddle w_64^(a d), then a length-16
// DFT of each d group:  x(4c + d) = sum_a w_16^(a c) w_64^(a d) sum_b w_4^(b d) Z[a + 16 b].
ERM_HD void idft64_reg(float2 (&Z)[64], const Tw64& t) {
#pragma unroll
  for (int a = 0; a < 16; ++a) {
    float2 v0 = Z[a], v1 = Z[a + 16], v2 = Z[a + 32], v3 = Z[a + 48];
    dft4<true>(v0, v1, v2, v3);
    Z[a] = v0;
    Z[a + 16] = a == 0 ? v1 : cmul(v1, wplus<64>(t, a));
    Z[a + 32] = a == 0 ? v2 : cmul(v2, wplus<64>(t, 2 * a));
    Z[a + 48] = a == 0 ? v3 : cmul(v3, wplus<64>(t, 3 * a));
  }
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    float2 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = Z[16 * d + c];
    idft_reg<4>(v, t);
#pragma unroll
    for (int c = 0; c < 16; ++c) Z[16 * d + c] = v[c];
  }
}

// Hermitian packing of a half spectrum X[0..M] (X[0], X[M] real) of a real
// sequence of length K1 = 2M into a length-M complex sequence Z:
//   Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) exp(+2 pi i k / K1),
// so that for z = inverse DFT_M(Z), x[2n] = Re z[n] and x[2n+1] = Im z[n] is
// the inverse real DFT of length K1.  Z holds X[0..M-1] on entry, xM = X[M].
template <int LM>
ERM_HD void hermitian_pack(float2 (&Z)[1 << LM], float2 xM, const Tw64& t) {
  constexpr int M = 1 << LM, K1 = 2 * M;
#pragma unroll
  for (int k = 0; k <= M / 2; ++k) {
    float2 xk = Z[k], xm = k == 0 ? xM : Z[M - k];
    if (k == 0) {
      xk.y = 0.f;
      xm.y = 0.f;
    }
    const float2 cm = conj(xm);
    const float2 d = cmul(csub(xk, cm), wplus<K1>(t, k));
    Z[k] = make_float2(xk.x + cm.x - d.y, xk.y + cm.y + d.x);
    if (k != 0 && 2 * k != M) {
      const float2 ck = conj(xk);
      const float2 d2 = cmul(csub(xm, ck), wplus<K1>(t, M - k));
      Z[M - k] = make_float2(xm.x + ck.x - d2.y, xm.y + ck.y + d2.x);
    }
  }
}

#undef ERM_HD

}  // namespace fft
}  // namespace erm
