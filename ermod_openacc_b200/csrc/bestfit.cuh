// bestfit.cuh -- weighted rigid superposition (the reference's bestfit module,
// bestfit.F90:114-336) for one thread: centres of mass, the rotation that
// best maps one centred point set onto another, RMSD without fitting.
//
// The rotation is the unit quaternion of Horn, "Closed-form solution of
// absolute orientation using unit quaternions", J. Opt. Soc. Am. A 4, 629
// (1987): with S_ab = sum_i w_i x_i,a y_i,b over the centred moving points x
// and reference points y, q is the eigenvector of the largest eigenvalue of
// the symmetric 4x4 matrix N(S), and y ~ q (0, x) q*.  The eigenvector comes
// from cyclic Jacobi rotations in FP64 (at most kJacobiSweeps sweeps).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace erm {
namespace fit {

#define ERM_HD __host__ __device__ __forceinline__

constexpr int kJacobiSweeps = 50;

// res = q (0, v) conj(q)
ERM_HD void rotate(const double q[4], const double v[3], double res[3]) {
  const double t0 = -(q[1] * v[0] + q[2] * v[1] + q[3] * v[2]);
  const double t1 = q[0] * v[0] + q[2] * v[2] - q[3] * v[1];
  const double t2 = q[0] * v[1] + q[3] * v[0] - q[1] * v[2];
  const double t3 = q[0] * v[2] + q[1] * v[1] - q[2] * v[0];
  // (t0, t) * (q0, -qv): vector part
  res[0] = -t0 * q[1] + q[0] * t1 - (t2 * q[3] - t3 * q[2]);
  res[1] = -t0 * q[2] + q[0] * t2 - (t3 * q[1] - t1 * q[3]);
  res[2] = -t0 * q[3] + q[0] * t3 - (t1 * q[2] - t2 * q[1]);
}

// Eigenvector of the largest eigenvalue of the symmetric 4x4 matrix a (overwritten).
ERM_HD void max_eigenvector4(double a[4][4], double v[4]) {
  double e[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) e[i][j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < kJacobiSweeps; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < 4; ++i) {
      diag += a[i][i] * a[i][i];
      for (int j = i + 1; j < 4; ++j) off += a[i][j] * a[i][j];
    }
    if (off <= 1e-30 * (diag + 1e-300)) break;
    for (int p = 0; p < 3; ++p)
      for (int q = p + 1; q < 4; ++q) {
        if (a[p][q] == 0.0) continue;
        // rotation angle zeroing a[p][q] (Rutishauser's form)
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 4; ++k) {   // a <- J^T a J
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 4; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 4; ++k) {   // eigenvectors: e <- e J
          const double ekp = e[k][p], ekq = e[k][q];
          e[k][p] = c * ekp - s * ekq;
          e[k][q] = s * ekp + c * ekq;
        }
      }
  }
  int best = 0;
  for (int i = 1; i < 4; ++i)
    if (a[i][i] > a[best][best]) best = i;
  double n = 0.0;
  for (int k = 0; k < 4; ++k) n += e[k][best] * e[k][best];
  n = sqrt(n);
  for (int k = 0; k < 4; ++k) v[k] = e[k][best] / n;
}

// Unit quaternion rotating the centred moving points onto the centred reference
// points, from S[a][b] = sum_i w_i x_i,a y_i,b (x moving, y reference).
ERM_HD void rotation_from_s(const double S[3][3], double q[4]) {
  const double xx = S[0][0], xy = S[0][1], xz = S[0][2], yx = S[1][0], yy = S[1][1], yz = S[1][2];
  const double zx = S[2][0], zy = S[2][1], zz = S[2][2];
  double N[4][4] = {{xx + yy + zz, yz - zy, zx - xz, xy - yx},
                    {yz - zy, xx - yy - zz, xy + yx, zx + xz},
                    {zx - xz, xy + yx, -xx + yy - zz, yz + zy},
                    {xy - yx, zx + xz, yz + zy, -xx - yy + zz}};
  max_eigenvector4(N, q);
}

// fit_a_rotate_b (bestfit.F90:309-336) for point sets held as float triples:
// the rotation that best maps `a` onto `refa` (weights w, n points) applied to
// the nb points `b` about a's centre, placed at refa's centre.
ERM_HD void fit_a_rotate_b(int n, const float* refa, const float* a, const float* w, int nb, const float* b,
                           float* bout) {
  double cr[3] = {0.0, 0.0, 0.0}, ca[3] = {0.0, 0.0, 0.0}, ws = 0.0;
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      cr[k] += (double)w[i] * refa[3 * i + k];
      ca[k] += (double)w[i] * a[3 * i + k];
    }
    ws += w[i];
  }
  for (int k = 0; k < 3; ++k) { cr[k] /= ws; ca[k] /= ws; }
  double S[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  for (int i = 0; i < n; ++i)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        S[r][c] += (double)w[i] * ((double)a[3 * i + r] - ca[r]) * ((double)refa[3 * i + c] - cr[c]);
  double q[4];
  rotation_from_s(S, q);
  for (int i = 0; i < nb; ++i) {
    const double v[3] = {(double)b[3 * i] - ca[0], (double)b[3 * i + 1] - ca[1], (double)b[3 * i + 2] - ca[2]};
    double r[3];
    rotate(q, v, r);
    for (int k = 0; k < 3; ++k) bout[3 * i + k] = (float)(r[k] + cr[k]);
  }
}

// rmsd_bestfit (bestfit.F90:339-346) without a buffer for the fitted points: the rotation
// that best maps x onto ref (weights w), each fitted point rounded to FP32 as fit_a_rotate_b
// stores it, then the weighted RMSD from ref.  Returns -1 when the weights sum to zero.
ERM_HD double rmsd_bestfit(int n, const float* ref, const float* x, const float* w) {
  double cr[3] = {0.0, 0.0, 0.0}, cx[3] = {0.0, 0.0, 0.0}, ws = 0.0;
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      cr[k] += (double)w[i] * ref[3 * i + k];
      cx[k] += (double)w[i] * x[3 * i + k];
    }
    ws += w[i];
  }
  if (ws == 0.0) return -1.0;
  for (int k = 0; k < 3; ++k) { cr[k] /= ws; cx[k] /= ws; }
  double S[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  for (int i = 0; i < n; ++i)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        S[r][c] += (double)w[i] * ((double)x[3 * i + r] - cx[r]) * ((double)ref[3 * i + c] - cr[c]);
  double q[4];
  rotation_from_s(S, q);
  double d = 0.0;
  for (int i = 0; i < n; ++i) {
    const double v[3] = {(double)x[3 * i] - cx[0], (double)x[3 * i + 1] - cx[1], (double)x[3 * i + 2] - cx[2]};
    double r[3];
    rotate(q, v, r);
    double t = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double e = (double)ref[3 * i + k] - (double)(float)(r[k] + cr[k]);
      t += e * e;
    }
    d += (double)w[i] * t;
  }
  return sqrt(d / ws);
}

// rmsd_nofit (bestfit.F90:349-364)
ERM_HD double rmsd_nofit(int n, const float* x, const float* y, const float* w) {
  double d = 0.0, ws = 0.0;
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double t = (double)y[3 * i + k] - (double)x[3 * i + k];
      s += t * t;
    }
    d += (double)w[i] * s;
    ws += w[i];
  }
  return sqrt(d / ws);
}

#undef ERM_HD

}  // namespace fit
}  // namespace erm
