// common.cuh -- device-side building blocks shared by the engine's kernels.
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>

namespace erm {

constexpr double kPi = 3.1415926535897932;   // erdst/engmain.F90:249

// Normalised periodic cell, the state realcal_prepare / normalize_periodic
// leave in module realcal (erdst/realcal.F90:22-27, 859-896), plus the
// inverted raw cell used by the PME splines (engproc.F90:1049-1070).
struct CellGeom {
  float cn[3][3];     // cell_normal(i,j): row i, column j
  float inv[3];       // invcell_normal
  float len[3];       // cell_len_normal
  float half[3];      // 0.5 * cell_len_normal
  float rot[3][3];    // Q of the QR step (applied as Q^T x) when `rotated`
  float invcl[3][3];  // inverse of the raw cell
  float cell[3][3];   // raw cell
  float volume;
  int rotated, cuboid, periodic;
};

// Constants of the pair energy of realcal (erdst/realcal.F90:62-96, 131-197).
struct PairParams {
  float lw, up, lw2, up2, lw3, up3, lw6, up6;
  float repA, repB, repC, attA, attB, attC;
  float reelcut;      // elecut when periodic, FLT_MAX otherwise
  float screen;
  int ljswitch;
  int bare;           // cltype == bare Coulomb (realcal_bare)
};

// Minimum image of a difference of normalised coordinates (realcal.F90:115-128).
// The cuboid case picks the image the reference's half - |half - |dx|| picks (realcal.F90:
// 243-250), as dx - L rint(dx / L): a displacement shorter than half the box is left exact,
// where the folded form rounds it to the ulp of half the box (~1e-6 A in a 50 A box, which
// is 1e-5 of an r^-12 repulsion at contact).
__device__ __forceinline__ void min_image(const CellGeom& g, float& x, float& y, float& z) {
  if (!g.periodic) return;
  if (g.cuboid) {
    x = fmaf(-g.len[0], rintf(x * g.inv[0]), x);
    y = fmaf(-g.len[1], rintf(y * g.inv[1]), y);
    z = fmaf(-g.len[2], rintf(z * g.inv[2]), z);
  } else {
    float f = roundf(z * g.inv[2]);
    x -= g.cn[0][2] * f; y -= g.cn[1][2] * f; z -= g.cn[2][2] * f;
    f = roundf(y * g.inv[1]);
    x -= g.cn[0][1] * f; y -= g.cn[1][1] * f; z -= g.cn[2][1] * f;
    f = roundf(x * g.inv[0]);
    x -= g.cn[0][0] * f; y -= g.cn[1][0] * f; z -= g.cn[2][0] * f;
  }
}

// Lennard-Jones with the four switching forms plus real-space Ewald (or bare)
// Coulomb for one site pair at squared distance dis2 (realcal.F90:129-197).
// FP32, as the reference's default build.  erfcf replaces 1-erf (more
// accurate for large arguments; the difference is below FP32 resolution of
// the pair energy).  One correctly rounded reciprocal square root replaces the
// reference's sqrt and its two divisions: r = dis2 / sqrt(dis2), sigma^2 / r^2 and
// q q' erfc / r are products with it, each within two FP32 roundings of the
// divided form.
__device__ __forceinline__ float pair_energy(const PairParams& P, float dis2, float ljeps, float ljsgm2,
                                             float qq) {
  const float rinv = __frsqrt_rn(dis2);
  const float rst = dis2 > 0.0f ? dis2 * rinv : 0.0f;   // coincident sites: r = 0, as sqrt gives
  float eplj = 0.0f;
  if (!(rst > P.up)) {
    const float invr2 = ljsgm2 * (rinv * rinv);
    const float invr6 = invr2 * invr2 * invr2;
    if (P.ljswitch <= 1) {
      eplj = 4.0f * ljeps * invr6 * (invr6 - 1.0f);
      if (rst > P.lw) {
        float swth;
        if (P.ljswitch == 0) {
          const float d = P.up2 - P.lw2;
          const float e = dis2 - P.up2;
          swth = (2.0f * dis2 + P.up2 - 3.0f * P.lw2) * (e * e) / (d * d * d);
        } else {
          const float s = (rst - P.lw) / (P.up - P.lw);
          const float s3 = s * s * s;
          swth = 1.0f - 10.0f * s3 + 15.0f * (s3 * s) - 6.0f * (s3 * s * s);
        }
        eplj = swth * eplj;
      }
    } else if (P.ljswitch == 2) {
      const float ljsgm6 = ljsgm2 * ljsgm2 * ljsgm2;
      float vdwa, vdwb;
      if (rst <= P.lw) {
        vdwa = invr6 * invr6 - ljsgm6 * ljsgm6 / (P.lw6 * P.up6);
        vdwb = invr6 - ljsgm6 / (P.lw3 * P.up3);
      } else {
        const float invr3 = sqrtf(invr6), ljsgm3 = sqrtf(ljsgm6);
        const float a = invr6 - ljsgm6 / P.up6, b = invr3 - ljsgm3 / P.up3;
        vdwa = P.up6 / (P.up6 - P.lw6) * (a * a);
        vdwb = P.up3 / (P.up3 - P.lw3) * (b * b);
      }
      eplj = 4.0f * ljeps * (vdwa - vdwb);
    } else {
      const float ljsgm6 = ljsgm2 * ljsgm2 * ljsgm2;
      float vdwa, vdwb;
      if (rst <= P.lw) {
        vdwa = invr6 * invr6 - ljsgm6 * ljsgm6 * P.repC;
        vdwb = invr6 - ljsgm6 * P.attC;
      } else {
        const float s = rst - P.lw, s3 = s * s * s, s4 = s3 * s;
        vdwa = invr6 * invr6 - ljsgm6 * ljsgm6 * (P.repA * s3 + P.repB * s4 + P.repC);
        vdwb = invr6 - ljsgm6 * (P.attA * s3 + P.attB * s4 + P.attC);
      }
      eplj = 4.0f * ljeps * (vdwa - vdwb);
    }
  }
  float epcl = 0.0f;
  if (rst < P.reelcut) epcl = P.bare ? qq * rinv : qq * erfcf(P.screen * rst) * rinv;
  return eplj + epcl;
}

// Philox4x32-10 (Salmon et al., SC'11); the insertion stream is keyed by
// (iseed, "ERMD") with counter (insertion, stnum, attempt, purpose).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k.x += 0x9E3779B9u; k.y += 0xBB67AE85u; }
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
  }
  return c;
}
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
constexpr uint32_t kStreamTag = 0x45524D44u;

// Cardinal B-spline weights w[c] = M_n(u + c), c = 0..n-1, of a site at
// fractional grid offset u in [0, 1): the stencil of calc_spline_molecule
// (recpcal.F90:506-574).  The reference evaluates M_n by the truncated-power
// sum of spline.F90:45-58, sum_i (-1)^i n/(i!(n-i)!) (x-i)^(n-1), whose terms
// reach ~3e2 at order 8 while M_n is O(1), so FP32 loses ~1e-5 absolute
// there.  The same function is formed here by the Cox-de Boor recursion
// M_k(x) = (x M_{k-1}(x) + (k-x) M_{k-1}(x-1)) / (k-1) (Essmann et al.,
// J. Chem. Phys. 103, 8577 (1995), eq. 4.1), whose terms are all positive.
__device__ __forceinline__ void spline_weights(float u, int order, float* w) {
  w[0] = 1.0f;                                  // M_1(u)
  for (int k = 2; k <= order; ++k) {
    const float rk = 1.0f / (float)(k - 1);
    w[k - 1] = (1.0f - u) * w[k - 2] * rk;      // x = u + k - 1: x M(x) term vanishes (M_{k-1}(x) = 0)
    for (int c = k - 2; c >= 1; --c)
      w[c] = ((u + (float)c) * w[c] + ((float)k - u - (float)c) * w[c - 1]) * rk;
    w[0] = u * w[0] * rk;
  }
}

// grid index r in [-(order-1), K] wrapped into [0, K) (the reference's modulo, recpcal.F90:388-390)
__device__ __forceinline__ int wrapk(int r, int K) {
  r += (r < 0) ? K : 0;
  return r - ((r >= K) ? K : 0);
}

// Programmatic dependent launch (PTX griddepcontrol): a kernel launched with
// programmatic stream serialisation may start while its predecessor in the
// stream is still running.  grid_dep_wait() blocks until the predecessor has
// completed and its memory is visible (a no-op without such a predecessor);
// grid_dep_launch() lets the successor start once every CTA of this grid has
// called it or exited.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// float atomics through the ordered integer images of IEEE floats
__device__ __forceinline__ void atomic_min_f(float* a, float v) {
  if (v >= 0.0f) atomicMin((int*)a, __float_as_int(v));
  else atomicMax((unsigned int*)a, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float* a, float v) {
  if (v >= 0.0f) atomicMax((int*)a, __float_as_int(v));
  else atomicMin((unsigned int*)a, __float_as_uint(v));
}

// Device error word bits (set by kernels, read by the host after a frame).
enum : int {
  kErrEngMin = 1,     // eng_min
  kErrEngSft = 2,     // eng_sft
  kErrEngCns = 4,     // eng_cns
  kWarnMbin = 8,      // mbin warning
  kErrOverflow = 16,  // internal capacity exceeded
  kErrGrid = 32,      // a PME grid index outside the grid
  kErrTimeout = 64,   // a bounded wait on an mbarrier expired
  kErrInsRej = 128,   // an insertion found no configuration in the RMSD window within kInsTries
};

struct DevStatus {
  int flags;
  int first_bad_mol;
  int first_bad_ins;
  float first_bad_value;
};

__device__ __forceinline__ void report(DevStatus* st, int bit, int mol, int ins, float v) {
  const int old = atomicOr(&st->flags, bit);
  if ((old & bit) == 0) {
    st->first_bad_mol = mol;
    st->first_bad_ins = ins;
    st->first_bad_value = v;
  }
}

}  // namespace erm
