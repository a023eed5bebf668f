"""The in-register DFTs of the fused PME kernels (csrc/regfft.cuh), run on the host.

The header is __host__ __device__, so the same code that the plane and k1-line kernels run
is compiled here as host code and checked against numpy's FFT:
- idft_reg<LM> (lengths 8, 16, 32) and idft64_reg, the inverse complex DFTs;
- hermitian_pack followed by idft_reg, the inverse real DFT of length 2M that the k1 line
  transform computes (recpcal.F90's complex-to-real FFT of the influence-weighted spectrum).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "ermod_openacc_b200", "csrc", "regfft.cuh")

SRC = r"""
#include <cmath>
#include <cstdio>
#include "regfft.cuh"
using namespace erm::fft;

static Tw64 tw64() {
  Tw64 t;
  for (int m = 0; m < 64; ++m) {
    const double a = 2.0 * M_PI * m / 64.0;
    t.w[m] = make_float2((float)std::cos(a), (float)-std::sin(a));
  }
  return t;
}

template <int LM>
static void run_idft(const Tw64& t, FILE* in, FILE* out) {
  constexpr int M = 1 << LM;
  float2 z[M];
  for (int k = 0; k < M; ++k) fscanf(in, "%f %f", &z[k].x, &z[k].y);
  idft_reg<LM>(z, t);
  for (int n = 0; n < M; ++n) fprintf(out, "%.9g %.9g\n", z[n].x, z[n].y);
}

template <int LM>
static void run_c2r(const Tw64& t, FILE* in, FILE* out) {
  constexpr int M = 1 << LM;
  float2 z[M], xm;
  for (int k = 0; k < M; ++k) fscanf(in, "%f %f", &z[k].x, &z[k].y);
  fscanf(in, "%f %f", &xm.x, &xm.y);
  hermitian_pack<LM>(z, xm, t);
  idft_reg<LM>(z, t);
  for (int n = 0; n < M; ++n) fprintf(out, "%.9g %.9g\n", z[n].x, z[n].y);
}

int main(int argc, char** argv) {
  const Tw64 t = tw64();
  FILE* in = fopen(argv[1], "r");
  FILE* out = fopen(argv[2], "w");
  char kind[16];
  int lm;
  while (fscanf(in, "%15s %d", kind, &lm) == 2) {
    if (kind[0] == 'c') {
      if (lm == 3) run_c2r<3>(t, in, out);
      if (lm == 4) run_c2r<4>(t, in, out);
      if (lm == 5) run_c2r<5>(t, in, out);
    } else if (lm == 6) {
      float2 z[64];
      for (int k = 0; k < 64; ++k) fscanf(in, "%f %f", &z[k].x, &z[k].y);
      idft64_reg(z, t);
      for (int n = 0; n < 64; ++n) {
        const float2 v = z[16 * (n & 3) + (n >> 2)];   // x(4c + d) sits at z[16 d + c]
        fprintf(out, "%.9g %.9g\n", v.x, v.y);
      }
    } else {
      if (lm == 3) run_idft<3>(t, in, out);
      if (lm == 4) run_idft<4>(t, in, out);
      if (lm == 5) run_idft<5>(t, in, out);
    }
  }
  fclose(out);
  return 0;
}
"""


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


@pytest.fixture(scope="module")
def regfft_exe(tmp_path_factory):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not found")
    d = tmp_path_factory.mktemp("regfft")
    src = d / "regfft_host.cu"
    src.write_text(SRC)
    exe = d / "regfft_host"
    subprocess.run([nvcc, "-x", "cu", "-O2", "-I", os.path.dirname(HDR), "-o", str(exe), str(src)], check=True,
                   capture_output=True)
    return exe


def _run(exe, tmp_path, cases):
    """cases: [("idft", lm, complex array)] -> the transforms, in order."""
    inp, out = tmp_path / "in.txt", tmp_path / "out.txt"
    with open(inp, "w") as f:
        for kind, lm, z in cases:
            f.write(f"{kind} {lm}\n")
            for v in z:
                f.write(f"{float(np.float32(v.real))!r} {float(np.float32(v.imag))!r}\n")
    subprocess.run([str(exe), str(inp), str(out)], check=True)
    vals = np.loadtxt(out).reshape(-1, 2)
    res, i = [], 0
    for _, lm, _ in cases:
        n = 1 << lm
        res.append(vals[i:i + n, 0] + 1j * vals[i:i + n, 1])
        i += n
    return res


def test_inverse_dfts_match_numpy(regfft_exe, tmp_path):
    rng = np.random.default_rng(7)
    cases = []
    for lm in (3, 4, 5, 6):
        for _ in range(3):
            z = (rng.standard_normal(1 << lm) + 1j * rng.standard_normal(1 << lm)).astype(np.complex64)
            cases.append(("idft", lm, z))
    got = _run(regfft_exe, tmp_path, cases)
    for (_, lm, z), g in zip(cases, got):
        n = 1 << lm
        ref = np.fft.ifft(z.astype(np.complex128)) * n            # sum_k Z[k] exp(+2 pi i k n / N)
        err = np.abs(g - ref).max() / np.abs(ref).max()
        assert err < 2e-6, (lm, err)


def test_hermitian_pack_gives_the_inverse_real_dft(regfft_exe, tmp_path):
    """The k1 line transform: a half spectrum X[0..M] of a real sequence of length 2M,
    packed and transformed at length M, gives x[2n] = Re z[n], x[2n+1] = Im z[n]."""
    rng = np.random.default_rng(11)
    cases, halves = [], []
    for lm in (3, 4, 5):
        m = 1 << lm
        x = rng.standard_normal(2 * m)
        X = np.fft.rfft(x)                                          # X[0..M], X[0] and X[M] real
        halves.append(x)
        cases.append(("c2r", lm, np.concatenate([X[:m], X[m:m + 1]]).astype(np.complex64)))
    inp, out = tmp_path / "in.txt", tmp_path / "out.txt"
    with open(inp, "w") as f:
        for kind, lm, z in cases:
            f.write(f"c {lm}\n")
            for v in z:
                f.write(f"{float(np.float32(v.real))!r} {float(np.float32(v.imag))!r}\n")
    subprocess.run([str(regfft_exe), str(inp), str(out)], check=True)
    vals = np.loadtxt(out).reshape(-1, 2)
    i = 0
    for (_, lm, _), x in zip(cases, halves):
        m = 1 << lm
        z = vals[i:i + m]
        i += m
        got = np.empty(2 * m)
        got[0::2], got[1::2] = z[:, 0], z[:, 1]
        ref = x * (2 * m)                                           # unnormalised inverse
        assert np.abs(got - ref).max() / np.abs(ref).max() < 2e-6, lm
