// ermod_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// CPU restatement of the reference's per-frame energy-distribution path
// (drmaruyama/ermod-openacc, erdst), used only as the checker by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg.  Nothing in the
// shipped library links, loads or calls this file.
//
// The reference is Fortran + OpenACC built by nvfortran; no Fortran
// compiler exists in this environment, so the reference cannot be run here
// and ships no golden vectors or tests of its own.  PARITY UNPINNED by the
// reference: this restatement is pinned instead by published known-answer
// values (Random123 Philox vectors, cardinal B-spline values, the NaCl
// Madelung constant and the simple-cubic Wigner constant) and by the
// reference's own mesh sizes, see tests/test_oracle_golden.py.
//
// The real type T selects the build: double restates the reference built
// with --enable-double (erdst/configure.ac:141-182), float the default
// single-precision build.  The algorithm is the reference's, step for
// step: brute-force pair loop over all site pairs (realcal.F90:207-364),
// one PME solve per insertion (recpcal.F90:429-502) with a radix-2 /
// direct DFT written here, binary-search binning (engproc.F90:1078-1171)
// and a per-insertion sparse ecorr update (engproc.F90:943-962).  Energies
// of different insertions are computed on OpenMP threads; the histogram
// updates run in insertion order as in the reference.
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/ermod_b200.h"

namespace {

constexpr double kPi = 3.1415926535897932;  // engmain.F90:249

// ---------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).  The reference
// draws insertions from the compiler's random_number (insertion.F90:549-584),
// whose stream is compiler specific; both this oracle and the library use
// this published generator with the stream layout documented in
// orc_insertion_uniforms below.
// ---------------------------------------------------------------------
void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
  }
  for (int i = 0; i < 4; ++i) out[i] = c[i];
}
// 24-bit uniform in [0,1), exact in float.
inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

constexpr uint32_t kStreamTag = 0x45524D44u;  // "ERMD"

// ---------------------------------------------------------------------
// spline.F90:25-58
// ---------------------------------------------------------------------
template <class T> struct Spline {
  int order = 0;
  std::vector<T> coeff;
  void init(int n) {
    order = n;
    coeff.assign(n + 1, T(0));
    for (int i = 0; i <= n; ++i) {
      T f = T(1);
      for (int k = 1; k <= i; ++k) f *= T(k);
      for (int k = 1; k <= n - i; ++k) f *= T(k);
      f = T(n) / f;
      if (i % 2 == 1) f = -f;
      coeff[i] = f;
    }
  }
  T value(T x) const {
    T f = T(0);
    if (x > T(0) && x < T(order)) {
      const int k = (int)x;
      for (int i = 0; i <= k; ++i) {
        T d = x - T(i), p = T(1);
        for (int e = 0; e < order - 1; ++e) p *= d;
        f += coeff[i] * p;
      }
    }
    return f;
  }
};

// ---------------------------------------------------------------------
// FFT: unnormalised, forward e^{-2 pi i}, inverse e^{+2 pi i} (the cuFFT
// R2C / C2R conventions that fft_iface.F90:38-98 relies on).  Radix-2 for
// powers of two, direct DFT otherwise.
// ---------------------------------------------------------------------
template <class T> struct FFT1 {
  int n = 0;
  bool pow2 = false;
  std::vector<std::complex<T>> tw;  // e^{-2 pi i k/n}
  std::vector<int> rev;
  void init(int n_) {
    n = n_;
    pow2 = (n & (n - 1)) == 0;
    tw.resize(n);
    for (int k = 0; k < n; ++k) {
      const double a = -2.0 * kPi * (double)k / (double)n;
      tw[k] = std::complex<T>((T)std::cos(a), (T)std::sin(a));
    }
    if (pow2) {
      rev.resize(n);
      int lg = 0;
      while ((1 << lg) < n) ++lg;
      for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
        rev[i] = r;
      }
    }
  }
  // in-place transform of x[0..n-1]; sign = -1 forward, +1 inverse
  void run(std::complex<T>* x, int sign, std::complex<T>* scratch) const {
    if (pow2) {
      for (int i = 0; i < n; ++i) if (i < rev[i]) std::swap(x[i], x[rev[i]]);
      for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = n / len;
        for (int i = 0; i < n; i += len)
          for (int j = 0; j < half; ++j) {
            std::complex<T> w = tw[j * step];
            if (sign > 0) w = std::conj(w);
            const std::complex<T> u = x[i + j], v = x[i + j + half] * w;
            x[i + j] = u + v;
            x[i + j + half] = u - v;
          }
      }
    } else {
      for (int k = 0; k < n; ++k) {
        std::complex<T> s(0, 0);
        for (int j = 0; j < n; ++j) {
          std::complex<T> w = tw[(int)(((long)j * k) % n)];
          if (sign > 0) w = std::conj(w);
          s += x[j] * w;
        }
        scratch[k] = s;
      }
      for (int k = 0; k < n; ++k) x[k] = scratch[k];
    }
  }
};

// 3D transform of a complex grid g[z][y][x] (x fastest), K1 x K2 x K3.
template <class T>
void fft3(std::complex<T>* g, int K1, int K2, int K3, const FFT1<T>& f1, const FFT1<T>& f2,
          const FFT1<T>& f3, int sign, std::vector<std::complex<T>>& line,
          std::vector<std::complex<T>>& scratch) {
  const int Kmax = std::max(K1, std::max(K2, K3));
  line.resize(Kmax);
  scratch.resize(Kmax);
  for (int z = 0; z < K3; ++z)
    for (int y = 0; y < K2; ++y) f1.run(g + ((size_t)z * K2 + y) * K1, sign, scratch.data());
  for (int z = 0; z < K3; ++z)
    for (int x = 0; x < K1; ++x) {
      for (int y = 0; y < K2; ++y) line[y] = g[((size_t)z * K2 + y) * K1 + x];
      f2.run(line.data(), sign, scratch.data());
      for (int y = 0; y < K2; ++y) g[((size_t)z * K2 + y) * K1 + x] = line[y];
    }
  for (int y = 0; y < K2; ++y)
    for (int x = 0; x < K1; ++x) {
      for (int z = 0; z < K3; ++z) line[z] = g[((size_t)z * K2 + y) * K1 + x];
      f3.run(line.data(), sign, scratch.data());
      for (int z = 0; z < K3; ++z) g[((size_t)z * K2 + y) * K1 + x] = line[z];
    }
}

inline int fmodulo(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

// ---------------------------------------------------------------------
// The oracle context: the state engmain / engproc / realcal / reciprocal
// keep in module variables.
// ---------------------------------------------------------------------
template <class T> struct Oracle {
  ermod_params p{};
  // topology
  int nummol = 0, numatm = 0, numatm_phys = 0, slvmax = 0, numslt = 0, nsite_slt = 0;
  std::vector<int> numsite, sluvid, uvspec, molbeg, tagpt, sltlist;
  std::vector<T> charge, sitemass, mol_charge;
  std::vector<int> ljtype;
  int ljtype_max = 0;
  std::vector<T> ljene_mat, ljlensq_mat;
  std::vector<T> bfcoord;
  // mesh
  int numslv = 0, ermax = 0, esmax = 0;
  std::vector<double> uvcrd, escrd;
  std::vector<int> uvmax, uvsoft;
  // accumulators
  std::vector<double> edens, ecorr, eself;
  std::vector<T> slnuv, minuv, maxuv;
  double avslf = 0, engnorm = 0, engsmpl = 0, voffset = 0;
  bool voffset_initialized = false;
  bool warn_bin_firsttime = true;
  // cell
  T cell[3][3]{}, invcl[3][3]{}, volume = 0;
  T cell_normal[3][3]{}, invcell_normal[3]{}, cell_len_normal[3]{};
  bool is_cuboid = true;
  // PME
  bool pme_initialized = false;
  T prevcl[3][3]{};
  int K1 = 0, K2 = 0, K3 = 0, cce = 0;
  Spline<T> spl;
  std::vector<T> splfc1, splfc2, splfc3, engfac;
  FFT1<T> f1, f2, f3;
  // realcal force-switch constants (realcal.F90:237-251)
  T lwljcut3 = 0, upljcut3 = 0, lwljcut6 = 0, upljcut6 = 0;
  T repA = 0, repB = 0, repC = 0, attA = 0, attB = 0, attC = 0;
  // self-energy reuse (engproc.F90:839-851)
  T usreal = 0;
  uint64_t solute_hash = 0;
  // last frame
  int maxdst = 0;
  std::vector<T> pos;          // sitepos for physical atoms + maxdst solute copies (refs)
  std::vector<T> posn;         // sitepos_normal
  std::vector<double> uvengy;  // [maxdst][slvmax] stored molecule-fastest
  std::vector<double> uvengy0;
  std::vector<double> insw;    // per-insertion structure weight
  std::vector<float> flceng;   // [maxdst][numslv]
  int nthreads = 1;
  std::string err;

  int fail(int code, const char* name) { err = name; return code; }

  static void gmx_force_params(int pw, T lw, T up, T& a, T& b, T& c) {  // realcal.F90:899-915
    const T df = up - lw;
    T uppw2 = T(1), uppw = T(1);
    for (int i = 0; i < pw + 2; ++i) uppw2 *= up;
    for (int i = 0; i < pw; ++i) uppw *= up;
    a = -T(pw) * (T(pw + 4) * up - T(pw + 1) * lw) / (uppw2 * (df * df)) / T(3);
    b = T(pw) * (T(pw + 3) * up - T(pw + 1) * lw) / (uppw2 * (df * df * df)) / T(4);
    c = T(1) / uppw - a * (df * df * df) - b * (df * df * df * df);
  }

  int create(const ermod_params* pp, const ermod_topology* t, const ermod_mesh* m, int nth) {
    p = *pp;
    nthreads = nth > 0 ? nth : 1;
    nummol = t->nummol;
    numsite.assign(t->numsite, t->numsite + nummol);
    sluvid.assign(t->sluvid, t->sluvid + nummol);
    uvspec.assign(t->uvspec, t->uvspec + nummol);
    molbeg.resize(nummol + 1);
    molbeg[0] = 0;
    for (int i = 0; i < nummol; ++i) molbeg[i + 1] = molbeg[i] + numsite[i];
    numatm = molbeg[nummol];
    charge.resize(numatm); sitemass.resize(numatm); ljtype.resize(numatm);
    for (int a = 0; a < numatm; ++a) {
      charge[a] = (T)t->charge[a]; sitemass[a] = (T)t->sitemass[a]; ljtype[a] = t->ljtype[a];
    }
    ljtype_max = t->ljtype_max;
    ljene_mat.resize(ljtype_max * ljtype_max); ljlensq_mat.resize(ljtype_max * ljtype_max);
    for (int i = 0; i < ljtype_max * ljtype_max; ++i) {
      ljene_mat[i] = (T)t->ljene_mat[i]; ljlensq_mat[i] = (T)t->ljlensq_mat[i];
    }
    mol_charge.resize(nummol);
    for (int i = 0; i < nummol; ++i) {
      T s = 0;
      for (int a = molbeg[i]; a < molbeg[i + 1]; ++a) s += charge[a];
      mol_charge[i] = s;
    }
    // engconst :391-399, enginit :72-80
    tagpt.clear(); sltlist.clear(); numatm_phys = 0;
    for (int i = 0; i < nummol; ++i) {
      if (sluvid[i] == ERMOD_PT_SOLVENT || sluvid[i] == ERMOD_PT_SOLUTE) {
        tagpt.push_back(i);
        numatm_phys += numsite[i];
      }
      if (sluvid[i] > 0) sltlist.push_back(i);
    }
    slvmax = (int)tagpt.size();
    numslt = (int)sltlist.size();
    if (numslt <= 0) return fail(ERMOD_ERR_ARG, "eng_num");
    if (p.slttype != ERMOD_SLT_SOLN) {
      if (numslt != 1 || sltlist[0] != nummol - 1) return fail(ERMOD_ERR_ARG, "eng_ins");
      nsite_slt = numsite[nummol - 1];
      if (t->bfcoord) bfcoord.assign(t->bfcoord, t->bfcoord + 3 * nsite_slt);
      else bfcoord.assign(3 * nsite_slt, T(0));
      maxdst = p.maxins;
      if (maxdst < 1) return fail(ERMOD_ERR_ARG, "set_ins");   // setconf.F90:352
    } else {
      maxdst = numslt;
    }
    numslv = m->numslv; ermax = m->ermax; esmax = m->esmax;
    uvcrd.assign(m->uvcrd, m->uvcrd + ermax);
    uvmax.assign(m->uvmax, m->uvmax + numslv);
    uvsoft.assign(m->uvsoft, m->uvsoft + numslv);
    if (m->escrd && esmax > 0) escrd.assign(m->escrd, m->escrd + esmax);
    edens.assign(ermax, 0.0);
    if (p.corrcal) ecorr.assign((size_t)ermax * ermax, 0.0);
    if (p.selfcal) eself.assign(esmax, 0.0);
    slnuv.assign(numslv, T(0));
    minuv.assign(numslv + 1, std::numeric_limits<T>::max());
    maxuv.assign(numslv + 1, -std::numeric_limits<T>::max());
    voffset = -(double)std::numeric_limits<T>::max();
    if (p.ljswitch == ERMOD_LJSWT_FRC_CHM) {
      lwljcut3 = (T)p.lwljcut * (T)p.lwljcut * (T)p.lwljcut;
      upljcut3 = (T)p.upljcut * (T)p.upljcut * (T)p.upljcut;
      lwljcut6 = lwljcut3 * lwljcut3; upljcut6 = upljcut3 * upljcut3;
    }
    if (p.ljswitch == ERMOD_LJSWT_FRC_GMX) {
      gmx_force_params(12, (T)p.lwljcut, (T)p.upljcut, repA, repB, repC);
      gmx_force_params(6, (T)p.lwljcut, (T)p.upljcut, attA, attB, attC);
    }
    if (p.cltype == ERMOD_EL_PME || p.cltype == ERMOD_EL_PPPM) {
      // recpcal.F90:250-251: the PPPM denominator needs an even order
      if (p.cltype == ERMOD_EL_PPPM && p.splodr % 2 != 0) return fail(ERMOD_ERR_ARG, "pppm_odr");
      K1 = p.ms1max; K2 = p.ms2max; K3 = p.ms3max; cce = K1 / 2;
      spl.init(p.splodr);
      f1.init(K1); f2.init(K2); f3.init(K3);
      init_spline_axis(K1, splfc1); init_spline_axis(K2, splfc2); init_spline_axis(K3, splfc3);
      if (p.cltype == ERMOD_EL_PPPM) calc_gfb_pppm();
      engfac.assign((size_t)(cce + 1) * K2 * K3, T(0));
    } else if (p.cltype != ERMOD_EL_COULOMB) {
      return fail(ERMOD_ERR_UNSUPPORTED, "set_prs");
    }
    if (!(p.insposition >= ERMOD_INSPOS_RANDOM && p.insposition <= ERMOD_INSPOS_GAUSS))
      return fail(ERMOD_ERR_UNSUPPORTED, "ins_geo");
    if (p.insposition >= ERMOD_INSPOS_SPHERE && p.insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC &&
        !(p.lwreg >= 0.f && p.upreg >= p.lwreg && p.upreg > 0.f && p.hostspec != 0))
      return fail(ERMOD_ERR_ARG, "ins_reg");
    if (p.insposition >= ERMOD_INSPOS_RMSD && !(p.lwreg >= 0.f && p.upreg >= p.lwreg && p.upreg > 0.f))
      return fail(ERMOD_ERR_ARG, "ins_reg");
    if (p.insstructure != ERMOD_INSSTR_NOREJECT && p.insstructure != ERMOD_INSSTR_RMSD)
      return fail(ERMOD_ERR_ARG, "ins_str");
    return ERMOD_OK;
  }

  // recpcal.F90:97-119
  void init_spline_axis(int K, std::vector<T>& splfc) {
    splfc.resize(K);
    for (int rci = 0; rci < K; ++rci) {
      std::complex<T> rcpi(0, 0);
      for (int spi = 0; spi <= p.splodr - 2; ++spi) {
        const T chr = spl.value(T(spi + 1));
        const T rtp2 = T(2) * (T)kPi * T(spi * rci) / T(K);
        rcpi += std::complex<T>(chr * std::cos(rtp2), chr * std::sin(rtp2));
      }
      splfc[rci] = std::real(rcpi * std::conj(rcpi));
    }
  }

  // recpcal.F90:121-163
  void spline_greenfunc() {
    for (int rc3 = 0; rc3 < K3; ++rc3)
      for (int rc2 = 0; rc2 < K2; ++rc2)
        for (int rc1 = 0; rc1 <= cce; ++rc1) {
          T factor = T(0);
          if (rc1 == 0 && rc2 == 0 && rc3 == 0) continue;
          const int rcv[3] = {rc1, rc2, rc3}, kmax[3] = {K1, K2, K3};
          T inm[3];
          bool zero = false;
          for (int mm = 0; mm < 3; ++mm) {
            if ((p.splodr % 2 == 1) && (2 * std::abs(rcv[mm]) == kmax[mm])) { zero = true; break; }
            inm[mm] = rcv[mm] <= kmax[mm] / 2 ? T(rcv[mm]) : T(rcv[mm] - kmax[mm]);
          }
          if (!zero) {
            T xst[3];
            for (int mm = 0; mm < 3; ++mm) xst[mm] = invcl[0][mm] * inm[0] + invcl[1][mm] * inm[1] + invcl[2][mm] * inm[2];
            T rtp2 = xst[0] * xst[0] + xst[1] * xst[1] + xst[2] * xst[2];
            const T chr = (T)(kPi * kPi) * rtp2 / ((T)p.screen * (T)p.screen);
            factor = std::exp(-chr) / rtp2 / (T)kPi / volume;
            rtp2 = splfc1[rc1] * splfc2[rc2] * splfc3[rc3];
            factor = factor / rtp2;
          }
          engfac[((size_t)rc3 * K2 + rc2) * (cce + 1) + rc1] = factor;
        }
    engfac[0] = T(0);
  }

  // calc_gfb_pppm (recpcal.F90:179-198).  gfb[l], l = 0 .. P-1, are the coefficients of
  // sum_n U^2(k + 2 pi n / h) = sum_l gfb[l] z^l, z = sin^2(k h / 2), for the order-P
  // assignment function U(k) = (sin(k h / 2) / (k h / 2))^P: the recurrence of the
  // reference, then the division by (2P - 1)!.
  std::vector<double> gfb;
  void calc_gfb_pppm() {
    const int P = p.splodr;
    gfb.assign(P, 0.0);
    gfb[0] = 1.0;
    for (int m = 1; m < P; ++m) {
      for (int l = m; l >= 1; --l)
        gfb[l] = 4.0 * (gfb[l] * (l - m) * (l - m - 0.5) - gfb[l - 1] * (l - m - 1) * (l - m - 1));
      gfb[0] = 4.0 * (gfb[0] * (-m) * (-m - 0.5));
    }
    double fact = 1.0;
    for (int i = 2; i <= 2 * P - 1; ++i) fact *= i;
    for (int l = 0; l < P; ++l) gfb[l] /= fact;
  }

  // gf_denom (recpcal.F90:201-214): the squared product of the three axes' alias sums
  T gf_denom(const T z[3]) const {
    T s[3] = {T(0), T(0), T(0)};
    for (int l = p.splodr - 1; l >= 0; --l)
      for (int a = 0; a < 3; ++a) s[a] = (T)gfb[l] + s[a] * z[a];
    const T prod = s[0] * s[1] * s[2];
    return prod * prod;
  }

  // Alias range of the PPPM sums (recpcal.F90:230-233, 243-244): m_max per mesh axis
  // from LAMMPS's accuracy form with EPS_HOC = 1e-7, projected on each cell vector,
  // in single precision and truncated as the reference's int().  -1 on a negative range.
  static void pppm_mrange(const float c[3][3], float screen, int K1, int K2, int K3, int out[3]) {
    const float acc = std::pow(-std::log(1.0e-7f), 0.25f);
    const float pi = (float)kPi;
    const float mm[3] = {screen / (pi * (float)K1) * acc, screen / (pi * (float)K2) * acc,
                         screen / (pi * (float)K3) * acc};
    for (int j = 0; j < 3; ++j) {
      const int v = (int)(c[0][j] * mm[0] + c[1][j] * mm[1] + c[2][j] * mm[2]);
      out[j] = v;
    }
  }

  // recpcal_pppm_greenfunc (recpcal.F90:217-337): Hockney and Eastwood's optimal influence
  // function, sum over aliases k_n = k + 2 pi invcl^T (n1 K1, n2 K2, n3 K3), |n_i| <= mmax[i],
  // of (k . k_n) gamma(k_n) U^2(k_n) / |k_n|^2, times 4 pi / (k^2 denom V).  The third alias
  // offset is n3 * K3; the reference's :311 multiplies n3 by K2 instead, which this does not
  // repeat (it differs only when K2 != K3 and mmax[2] > 0).
  int mrange[3] = {0, 0, 0};
  void pppm_greenfunc() {
    const T tp = T(2) * (T)kPi;
    const T sc = (T)p.screen;
    const int Kv[3] = {K1, K2, K3};
    for (int rc3 = 0; rc3 < K3; ++rc3)
      for (int rc2 = 0; rc2 < K2; ++rc2)
        for (int rc1 = 0; rc1 <= cce; ++rc1) {
          if (rc1 == 0 && rc2 == 0 && rc3 == 0) continue;
          const int rcv[3] = {rc1, rc2, rc3};
          T inm[3], z[3];
          for (int a = 0; a < 3; ++a) {
            inm[a] = rcv[a] <= Kv[a] / 2 ? T(rcv[a]) : T(rcv[a] - Kv[a]);
            const T sn = std::sin((T)kPi * inm[a] / T(Kv[a]));
            z[a] = sn * sn;
          }
          T k[3];
          for (int i = 0; i < 3; ++i) k[i] = tp * (invcl[0][i] * inm[0] + invcl[1][i] * inm[1] + invcl[2][i] * inm[2]);
          const T k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
          T factor = T(0);
          if (k2 > T(0)) {
            T sum = T(0);
            T ukm[3];
            auto usq = [&](int a, int n) {
              const T t = (T)kPi * (inm[a] / T(Kv[a]) + T(n));
              if (t == T(0)) return T(1);
              const T x = std::sin(t) / t;
              T r = T(1);
              for (int e = 0; e < 2 * p.splodr; ++e) r *= x;
              return r;
            };
            for (int nx = -mrange[0]; nx <= mrange[0]; ++nx) {
              ukm[0] = usq(0, nx);
              for (int ny = -mrange[1]; ny <= mrange[1]; ++ny) {
                ukm[1] = usq(1, ny);
                for (int nz = -mrange[2]; nz <= mrange[2]; ++nz) {
                  ukm[2] = usq(2, nz);
                  const T mN[3] = {T(nx * K1), T(ny * K2), T(nz * K3)};
                  T km[3];
                  for (int i = 0; i < 3; ++i)
                    km[i] = k[i] + tp * (invcl[0][i] * mN[0] + invcl[1][i] * mN[1] + invcl[2][i] * mN[2]);
                  T gam = T(1);
                  for (int i = 0; i < 3; ++i) gam *= std::exp(T(-0.25) * (km[i] / sc) * (km[i] / sc));
                  const T kk = km[0] * km[0] + km[1] * km[1] + km[2] * km[2];
                  sum += (k[0] * km[0] + k[1] * km[1] + k[2] * km[2]) * gam * (ukm[0] * ukm[1] * ukm[2]) / kk;
                }
              }
            }
            factor = sum * T(4) * (T)kPi / (k2 * gf_denom(z)) / volume;
          }
          engfac[((size_t)rc3 * K2 + rc2) * (cce + 1) + rc1] = factor;
        }
    engfac[0] = T(0);
  }

  // engproc.F90:1049-1070 ; cell(i,j) = row i, column j (column j is the j-th vector)
  void get_inverted_cell() {
    const T(*c)[3] = cell;
    volume = c[0][0] * c[1][1] * c[2][2] + c[0][1] * c[1][2] * c[2][0] + c[0][2] * c[1][0] * c[2][1]
           - c[0][2] * c[1][1] * c[2][0] - c[0][1] * c[1][0] * c[2][2] - c[0][0] * c[1][2] * c[2][1];
    invcl[0][0] = c[1][1] * c[2][2] - c[1][2] * c[2][1];
    invcl[0][1] = c[0][2] * c[2][1] - c[0][1] * c[2][2];
    invcl[0][2] = c[0][1] * c[1][2] - c[0][2] * c[1][1];
    invcl[1][0] = c[1][2] * c[2][0] - c[1][0] * c[2][2];
    invcl[1][1] = c[0][0] * c[2][2] - c[0][2] * c[2][0];
    invcl[1][2] = c[0][2] * c[1][0] - c[0][0] * c[1][2];
    invcl[2][0] = c[1][0] * c[2][1] - c[1][1] * c[2][0];
    invcl[2][1] = c[0][1] * c[2][0] - c[0][0] * c[2][1];
    invcl[2][2] = c[0][0] * c[1][1] - c[0][1] * c[1][0];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) invcl[i][j] /= volume;
  }

  // realcal.F90:776-896
  int normalize_periodic(size_t natoms) {
    posn.assign(pos.begin(), pos.begin() + 3 * natoms);
    if (cell[1][0] == T(0) && cell[2][0] == T(0) && cell[2][1] == T(0)) {
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) cell_normal[i][j] = cell[i][j];
    } else {
      // modified Gram-Schmidt (realcal.F90:794-816)
      T q[3][3]{}, r[3][3]{}, tmp[3][3];
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) tmp[i][j] = cell[i][j];
      for (int i = 0; i < 3; ++i) {
        const T len = std::sqrt(tmp[0][0] * tmp[0][0] + tmp[1][0] * tmp[1][0] + tmp[2][0] * tmp[2][0]);
        for (int k = 0; k < 3; ++k) q[k][i] = tmp[k][i] / len;
        r[i][i] = len;
        for (int j = i + 1; j < 3; ++j) {
          r[i][j] = q[0][i] * tmp[0][j] + q[1][i] * tmp[1][j] + q[2][i] * tmp[2][j];
          for (int k = 0; k < 3; ++k) tmp[k][j] -= r[i][j] * q[k][i];
        }
      }
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) cell_normal[i][j] = r[i][j];
      for (size_t a = 0; a < natoms; ++a) {
        T x[3] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
        for (int i = 0; i < 3; ++i) posn[3 * a + i] = q[0][i] * x[0] + q[1][i] * x[1] + q[2][i] * x[2];
      }
    }
    // normalize_cell_vector (realcal.F90:820-857)
    for (int i = 0; i < 3; ++i)
      if (cell_normal[0][0] < T(0)) for (int k = 0; k < 3; ++k) cell_normal[k][i] = -cell_normal[k][i];
    const T thr = (T)1e-4;
    if (std::abs(cell_normal[0][1]) > T(0.5) * cell_normal[0][0] + thr) {
      const T f = std::round(cell_normal[0][1] * invcell_normal[0]);
      for (int k = 0; k < 3; ++k) cell_normal[k][1] -= cell_normal[k][0] * f;
    }
    if (std::abs(cell_normal[0][2]) > T(0.5) * cell_normal[0][0] + thr) {
      const T f = std::round(cell_normal[0][2] * invcell_normal[0]);
      for (int k = 0; k < 3; ++k) cell_normal[k][2] -= cell_normal[k][0] * f;
    }
    if (std::abs(cell_normal[1][2]) > T(0.5) * cell_normal[1][1] + thr) {
      const T f = std::round(cell_normal[1][2] * invcell_normal[1]);
      for (int k = 0; k < 3; ++k) cell_normal[k][2] -= cell_normal[k][1] * f;
    }
    const T cutoff = std::min((T)p.elecut, (T)p.upljcut);
    for (int i = 0; i < 3; ++i)
      if (cutoff > cell_normal[i][i] * T(0.5)) return fail(ERMOD_ERR_CELL, "cel_siz");
    for (int i = 0; i < 3; ++i) cell_len_normal[i] = std::abs(cell_normal[i][i]);
    for (int i = 0; i < 3; ++i) invcell_normal[i] = T(1) / cell_len_normal[i];
    const T cth = (T)1e-8;
    is_cuboid = !(std::abs(cell[0][1]) > cth || std::abs(cell[0][2]) > cth || std::abs(cell[1][2]) > cth);
    for (size_t a = 0; a < natoms; ++a) {
      T* x = &posn[3 * a];
      for (int d = 2; d >= 0; --d) {
        const T f = std::floor(invcell_normal[d] * x[d]);
        for (int k = 0; k < 3; ++k) x[k] -= cell_normal[k][d] * f;
      }
    }
    return ERMOD_OK;
  }

  inline void min_image(T xst[3]) const {
    if (p.boxshp != ERMOD_SYS_PERIODIC) return;
    if (is_cuboid) {
      for (int k = 0; k < 3; ++k) {
        const T half = T(0.5) * cell_len_normal[k];
        xst[k] = half - std::abs(half - std::abs(xst[k]));
      }
    } else {
      for (int d = 2; d >= 0; --d) {
        const T f = std::round(xst[d] * invcell_normal[d]);
        for (int k = 0; k < 3; ++k) xst[k] -= cell_normal[k][d] * f;
      }
    }
  }

  // one site pair of realcal_soln / realcal_refs / realcal_bare (realcal.F90:114-197)
  inline T pair_energy(const T* xi, const T* xj, int ati, int atj, bool bare) const {
    T xst[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
    min_image(xst);
    const T dis2 = xst[0] * xst[0] + xst[1] * xst[1] + xst[2] * xst[2];
    const T rst = std::sqrt(dis2);
    const T lw = (T)p.lwljcut, up = (T)p.upljcut;
    T eplj;
    if (rst > up) {
      eplj = T(0);
    } else {
      const int lti = ljtype[ati] - 1, ltj = ljtype[atj] - 1;
      const T ljeps = ljene_mat[(size_t)ltj * ljtype_max + lti];
      const T ljsgm2 = ljlensq_mat[(size_t)ltj * ljtype_max + lti];
      const T invr2 = ljsgm2 / dis2;
      const T invr6 = invr2 * invr2 * invr2;
      switch (p.ljswitch) {
        case ERMOD_LJSWT_POT_CHM:
        case ERMOD_LJSWT_POT_GMX: {
          eplj = T(4) * ljeps * invr6 * (invr6 - T(1));
          if (rst > lw) {
            T swth;
            if (p.ljswitch == ERMOD_LJSWT_POT_CHM) {
              const T lw2 = lw * lw, up2 = up * up;
              const T d = up2 - lw2;
              swth = (T(2) * dis2 + up2 - T(3) * lw2) * ((dis2 - up2) * (dis2 - up2)) / (d * d * d);
            } else {
              const T s = (rst - lw) / (up - lw);
              swth = T(1) - T(10) * (s * s * s) + T(15) * (s * s * s * s) - T(6) * (s * s * s * s * s);
            }
            eplj = swth * eplj;
          }
          break;
        }
        case ERMOD_LJSWT_FRC_CHM: {
          const T ljsgm6 = ljsgm2 * ljsgm2 * ljsgm2;
          T vdwa, vdwb;
          if (rst <= lw) {
            vdwa = invr6 * invr6 - ljsgm6 * ljsgm6 / (lwljcut6 * upljcut6);
            vdwb = invr6 - ljsgm6 / (lwljcut3 * upljcut3);
          } else {
            const T invr3 = std::sqrt(invr6), ljsgm3 = std::sqrt(ljsgm6);
            const T a = invr6 - ljsgm6 / upljcut6, b = invr3 - ljsgm3 / upljcut3;
            vdwa = upljcut6 / (upljcut6 - lwljcut6) * (a * a);
            vdwb = upljcut3 / (upljcut3 - lwljcut3) * (b * b);
          }
          eplj = T(4) * ljeps * (vdwa - vdwb);
          break;
        }
        default: {  // ERMOD_LJSWT_FRC_GMX
          const T ljsgm6 = ljsgm2 * ljsgm2 * ljsgm2;
          T vdwa, vdwb;
          if (rst <= lw) {
            vdwa = invr6 * invr6 - ljsgm6 * ljsgm6 * repC;
            vdwb = invr6 - ljsgm6 * attC;
          } else {
            const T s = rst - lw, s3 = s * s * s, s4 = s3 * s;
            vdwa = invr6 * invr6 - ljsgm6 * ljsgm6 * (repA * s3 + repB * s4 + repC);
            vdwb = invr6 - ljsgm6 * (attA * s3 + attB * s4 + attC);
          }
          eplj = T(4) * ljeps * (vdwa - vdwb);
        }
      }
    }
    const T reelcut = p.boxshp == ERMOD_SYS_PERIODIC ? (T)p.elecut : std::numeric_limits<T>::max();
    T epcl;
    if (rst >= reelcut) epcl = T(0);
    else if (bare) epcl = charge[ati] * charge[atj] / rst;
    else epcl = charge[ati] * charge[atj] * (T(1) - std::erf((T)p.screen * rst)) / rst;
    return eplj + epcl;
  }

  // recpcal.F90:504-575: spline weights and grid base of one site at raw position x
  void spline_site(const T* x, T* w /*3*order*/, int* grd) const {
    T inm[3];
    for (int k = 0; k < 3; ++k) {
      T f = invcl[k][0] * x[0] + invcl[k][1] * x[1] + invcl[k][2] * x[2];
      f = f - std::floor(f);
      inm[k] = f;
    }
    const int kmax[3] = {K1, K2, K3};
    for (int m = 0; m < 3; ++m) {
      const T f = inm[m] * T(kmax[m]);
      const int rci = (int)f;
      for (int spi = 0; spi < p.splodr; ++spi) w[m * p.splodr + spi] = spl.value(f - T(rci - spi));
      grd[m] = rci;
    }
  }

  // recpcal_prepare_solute(_refs) (recpcal.F90:359-502) for one solute copy:
  // spread, forward FFT, self energy, influence multiply, inverse FFT.
  // phi receives the real potential grid, returns the reciprocal self energy.
  T pme_solute(const T* spos, const int* satoms, int nsite, std::vector<T>& phi,
               std::vector<std::complex<T>>& g, std::vector<std::complex<T>>& line,
               std::vector<std::complex<T>>& scr) const {
    const int n = p.splodr;
    const size_t NG = (size_t)K1 * K2 * K3;
    g.assign(NG, std::complex<T>(0, 0));
    std::vector<T> w(3 * n);
    int grd[3];
    for (int sid = 0; sid < nsite; ++sid) {
      spline_site(spos + 3 * sid, w.data(), grd);
      const T chr = charge[satoms[sid]];
      for (int c3 = 0; c3 < n; ++c3)
        for (int c2 = 0; c2 < n; ++c2)
          for (int c1 = 0; c1 < n; ++c1) {
            const int r1 = fmodulo(grd[0] - c1, K1), r2 = fmodulo(grd[1] - c2, K2), r3 = fmodulo(grd[2] - c3, K3);
            const T f = chr * w[c1] * w[n + c2] * w[2 * n + c3];
            g[((size_t)r3 * K2 + r2) * K1 + r1] += f;
          }
    }
    fft3(g.data(), K1, K2, K3, f1, f2, f3, -1, line, scr);
    // self energy on the half spectrum (recpcal.F90:482-491)
    T self = T(0);
    for (int r3 = 0; r3 < K3; ++r3)
      for (int r2 = 0; r2 < K2; ++r2)
        for (int r1 = 0; r1 <= cce; ++r1) {
          const std::complex<T> v = g[((size_t)r3 * K2 + r2) * K1 + r1];
          const T e = engfac[((size_t)r3 * K2 + r2) * (cce + 1) + r1] * std::real(v * std::conj(v));
          T wgt;
          if (K1 % 2 == 0) wgt = (r1 == 0 || r1 == cce) ? T(0.5) : T(1);
          else wgt = (r1 == 0) ? T(0.5) : T(1);
          self += wgt * e;
        }
    // influence multiply on the half spectrum, then the C2R transform:
    // rebuild the Hermitian full spectrum from the half and inverse-transform.
    std::vector<std::complex<T>> h((size_t)(cce + 1) * K2 * K3);
    for (int r3 = 0; r3 < K3; ++r3)
      for (int r2 = 0; r2 < K2; ++r2)
        for (int r1 = 0; r1 <= cce; ++r1) {
          const size_t hi = ((size_t)r3 * K2 + r2) * (cce + 1) + r1;
          h[hi] = engfac[hi] * g[((size_t)r3 * K2 + r2) * K1 + r1];
        }
    for (int r3 = 0; r3 < K3; ++r3)
      for (int r2 = 0; r2 < K2; ++r2)
        for (int r1 = 0; r1 < K1; ++r1) {
          std::complex<T> v;
          if (r1 <= cce) v = h[((size_t)r3 * K2 + r2) * (cce + 1) + r1];
          else {
            const int m1 = K1 - r1, m2 = (K2 - r2) % K2, m3 = (K3 - r3) % K3;
            v = std::conj(h[((size_t)m3 * K2 + m2) * (cce + 1) + m1]);
          }
          // C2R treats the self-conjugate planes as real (imaginary part ignored)
          if ((r1 == 0 || (K1 % 2 == 0 && r1 == cce))) {
            const int m2 = (K2 - r2) % K2, m3 = (K3 - r3) % K3;
            const std::complex<T> a = h[((size_t)r3 * K2 + r2) * (cce + 1) + r1];
            const std::complex<T> b = std::conj(h[((size_t)m3 * K2 + m2) * (cce + 1) + r1]);
            v = (a + b) * T(0.5);
          }
          g[((size_t)r3 * K2 + r2) * K1 + r1] = v;
        }
    fft3(g.data(), K1, K2, K3, f1, f2, f3, +1, line, scr);
    phi.resize(NG);
    for (size_t i = 0; i < NG; ++i) phi[i] = std::real(g[i]);
    return self;
  }

  // recpcal_energy_soln / _refs inner sum (recpcal.F90:613-646) for molecule mol
  T pme_gather(int mol, const std::vector<T>& phi, const std::vector<T>& wslv, const std::vector<int>& gslv,
               const std::vector<int>& slvtag) const {
    const int n = p.splodr;
    T pairep = T(0);
    const int svi = slvtag[mol];
    for (int sid = 0; sid < numsite[mol]; ++sid) {
      const int pt = svi + sid;
      const T chr = charge[molbeg[mol] + sid];
      const T* w = &wslv[(size_t)pt * 3 * n];
      const int* gd = &gslv[(size_t)pt * 3];
      for (int c3 = 0; c3 < n; ++c3) {
        const T fac1 = chr * w[2 * n + c3];
        const int r3 = fmodulo(gd[2] - c3, K3);
        for (int c2 = 0; c2 < n; ++c2) {
          const T fac2 = fac1 * w[n + c2];
          const int r2 = fmodulo(gd[1] - c2, K2);
          for (int c1 = 0; c1 < n; ++c1) {
            const T fac3 = fac2 * w[c1];
            const int r1 = fmodulo(gd[0] - c1, K1);
            pairep += fac3 * phi[((size_t)r3 * K2 + r2) * K1 + r1];
          }
        }
      }
    }
    return pairep;
  }

  // realcal_self(_refs) (realcal.F90:669-771) on normalised coordinates xs
  T real_self(const T* xs, const int* satoms, int nsite) const {
    T pairep = T(0);
    if (p.cltype == ERMOD_EL_COULOMB) return pairep;
    const T sqpi = std::sqrt((T)kPi);
    for (int is = 0; is < nsite; ++is) {
      const T qi = charge[satoms[is]];
      pairep += -qi * qi * (T)p.screen / sqpi;
      for (int js = is + 1; js < nsite; ++js) {
        T xst[3] = {xs[3 * is] - xs[3 * js], xs[3 * is + 1] - xs[3 * js + 1], xs[3 * is + 2] - xs[3 * js + 2]};
        if (is_cuboid) {
          for (int k = 0; k < 3; ++k) {
            const T half = T(0.5) * cell_len_normal[k];
            xst[k] = half - std::abs(half - std::abs(xst[k]));
          }
        } else {
          for (int d = 2; d >= 0; --d) {
            const T f = std::round(xst[d] * invcell_normal[d]);
            for (int k = 0; k < 3; ++k) xst[k] -= cell_normal[k][d] * f;
          }
        }
        const T rst = std::sqrt(xst[0] * xst[0] + xst[1] * xst[1] + xst[2] * xst[2]);
        pairep += -qi * charge[satoms[js]] * std::erf((T)p.screen * rst) / rst;
      }
    }
    return pairep;
  }

  // residual_self_ene (engproc.F90:967-977)
  T residual_self(T q) const {
    if (p.cltype == ERMOD_EL_COULOMB) return T(0);
    T e = (T)kPi * q * q / (T)p.screen / (T)p.screen / volume;
    return -(e / T(2));
  }

  static uint64_t hash_coords(const T* x, int n) {  // utility.F90:32-65 / hash_real.c:17-27
    uint64_t h = 0;
    for (int i = 0; i < n; ++i) {
      uint64_t b = 0;
      if (sizeof(T) == 4) { uint32_t u; std::memcpy(&u, &x[i], 4); b = u; }
      else std::memcpy(&b, &x[i], 8);
      h = ((h << 7) | (h >> 57)) ^ b;
    }
    return h;
  }

  // com_aggregate (insertion.F90:587-614): mass-weighted centre of the atoms of the solvent
  // molecules whose species is in hostspec, from the frame's coordinates, summed in FP64.
  void aggregate_center(const float* sitepos) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < nummol; ++i) {
      if (sluvid[i] != ERMOD_PT_SOLVENT || uvspec[i] < 1 || uvspec[i] > 31) continue;
      if (!((p.hostspec >> (uvspec[i] - 1)) & 1)) continue;
      for (int a = molbeg[i]; a < molbeg[i + 1]; ++a) {
        const double m = (double)(float)sitemass[a];
        for (int k = 0; k < 3; ++k) acc[k] += m * (double)sitepos[3 * a + k];
        acc[3] += m;
      }
    }
    for (int k = 0; k < 3; ++k) aggcen[k] = acc[3] > 0.0 ? acc[k] / acc[3] : 0.0;
  }
  double aggcen[3] = {0.0, 0.0, 0.0};

  // ---- RefInfo reference structure (insertion.F90:646-770, bestfit.F90:114-364) ----
  std::vector<int> ref_atom;          // physical atoms of the refspec molecules, molecule order
  std::vector<double> ref_host, ref_host_w, ref_slt, ref_slt_w, ref_bf;
  bool gauss_init = false;
  double gauss_l[3] = {0, 0, 0}, gauss_z0 = 0, gauss_z1 = 0;

  int set_refstructure(int refspec, int nhost, const float* hc, const float* hw, const float* sc, const float* sw) {
    ref_atom.clear();
    for (int i = 0; i < nummol; ++i)
      if (sluvid[i] == ERMOD_PT_SOLVENT && uvspec[i] >= 1 && uvspec[i] <= 31 && ((refspec >> (uvspec[i] - 1)) & 1))
        for (int a = molbeg[i]; a < molbeg[i + 1]; ++a) ref_atom.push_back(a);
    if ((int)ref_atom.size() != nhost) return fail(ERMOD_ERR_ARG, "ins_ref");
    const int s = p.slttype == ERMOD_SLT_SOLN ? numsite[sltlist[0]] : nsite_slt;
    ref_host.assign(hc, hc + 3 * nhost); ref_host_w.assign(hw, hw + nhost);
    ref_slt.assign(sc, sc + 3 * s); ref_slt_w.assign(sw, sw + s);
    ref_bf.assign(3 * s, 0.0);
    return ERMOD_OK;
  }

  // Largest-eigenvalue eigenvector of a symmetric 4x4 matrix: cyclic Jacobi, the rotation
  // angle from tan(2 phi) = 2 a_pq / (a_qq - a_pp), eigenvectors accumulated column-wise.
  static void top_eigvec4(double a[4][4], double out[4]) {
    double v[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
    for (int it = 0; it < 100; ++it) {
      double off = 0;
      for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) if (i != j) off += a[i][j] * a[i][j];
      if (off < 1e-40) break;
      for (int p0 = 0; p0 < 4; ++p0)
        for (int q0 = p0 + 1; q0 < 4; ++q0) {
          if (std::abs(a[p0][q0]) < 1e-300) continue;
          const double phi = 0.5 * std::atan2(2 * a[p0][q0], a[q0][q0] - a[p0][p0]);
          const double c = std::cos(phi), sn = std::sin(phi);
          for (int k = 0; k < 4; ++k) {
            const double x = a[k][p0], y = a[k][q0];
            a[k][p0] = c * x - sn * y; a[k][q0] = sn * x + c * y;
          }
          for (int k = 0; k < 4; ++k) {
            const double x = a[p0][k], y = a[q0][k];
            a[p0][k] = c * x - sn * y; a[q0][k] = sn * x + c * y;
          }
          for (int k = 0; k < 4; ++k) {
            const double x = v[k][p0], y = v[k][q0];
            v[k][p0] = c * x - sn * y; v[k][q0] = sn * x + c * y;
          }
        }
    }
    int b = 0;
    for (int i = 1; i < 4; ++i) if (a[i][i] > a[b][b]) b = i;
    double n = 0;
    for (int k = 0; k < 4; ++k) n += v[k][b] * v[k][b];
    for (int k = 0; k < 4; ++k) out[k] = v[k][b] / std::sqrt(n);
  }
  // q (0, x) conj(q) as a rotation matrix applied to x
  static void qrot(const double q[4], const double x[3], double r[3]) {
    const double w = q[0], a = q[1], b = q[2], c = q[3];
    const double R[3][3] = {{w * w + a * a - b * b - c * c, 2 * (a * b - w * c), 2 * (a * c + w * b)},
                            {2 * (a * b + w * c), w * w - a * a + b * b - c * c, 2 * (b * c - w * a)},
                            {2 * (a * c - w * b), 2 * (b * c + w * a), w * w - a * a - b * b + c * c}};
    for (int i = 0; i < 3; ++i) r[i] = R[i][0] * x[0] + R[i][1] * x[1] + R[i][2] * x[2];
  }
  // fit_a_rotate_b: rotation of the centred `mov` onto the centred `ref` (Horn 1987), applied to
  // the nb points b about mov's centre and placed at ref's centre
  static void fit_rotate(int n, const double* ref, const double* mov, const double* w, int nb, const double* b,
                         double* out) {
    double cr[3] = {0, 0, 0}, cm[3] = {0, 0, 0}, ws = 0;
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) { cr[k] += w[i] * ref[3 * i + k]; cm[k] += w[i] * mov[3 * i + k]; }
      ws += w[i];
    }
    for (int k = 0; k < 3; ++k) { cr[k] /= ws; cm[k] /= ws; }
    double S[3][3] = {};
    for (int i = 0; i < n; ++i)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) S[r][c] += w[i] * (mov[3 * i + r] - cm[r]) * (ref[3 * i + c] - cr[c]);
    double N[4][4] = {{S[0][0] + S[1][1] + S[2][2], S[1][2] - S[2][1], S[2][0] - S[0][2], S[0][1] - S[1][0]},
                      {S[1][2] - S[2][1], S[0][0] - S[1][1] - S[2][2], S[0][1] + S[1][0], S[2][0] + S[0][2]},
                      {S[2][0] - S[0][2], S[0][1] + S[1][0], -S[0][0] + S[1][1] - S[2][2], S[1][2] + S[2][1]},
                      {S[0][1] - S[1][0], S[2][0] + S[0][2], S[1][2] + S[2][1], -S[0][0] - S[1][1] + S[2][2]}};
    double q[4];
    top_eigvec4(N, q);
    for (int i = 0; i < nb; ++i) {
      const double x[3] = {b[3 * i] - cm[0], b[3 * i + 1] - cm[1], b[3 * i + 2] - cm[2]};
      double r[3];
      qrot(q, x, r);
      for (int k = 0; k < 3; ++k) out[3 * i + k] = r[k] + cr[k];
    }
  }
  // reffit's host step: the reference host onto this frame's host atoms, carrying the reference solute
  void reffit_frame(const float* sitepos) {
    const int n = (int)ref_atom.size();
    std::vector<double> cur(3 * (size_t)n);
    for (int i = 0; i < n; ++i) for (int k = 0; k < 3; ++k) cur[3 * i + k] = sitepos[3 * ref_atom[i] + k];
    fit_rotate(n, cur.data(), ref_host.data(), ref_host_w.data(), (int)ref_slt_w.size(), ref_slt.data(), ref_bf.data());
    for (double& x : ref_bf) x = (double)(float)x;
  }

  // instslt('proc') for insposition RANDOM/NOCHANGE/SPHERE/SLAB, insorient RANDOM/NOCHANGE
  // (insertion.F90:86-98, 100-200, 307-375; bestfit.F90:252-297; quaternion rotate
  // bestfit.F90:74-99).  Writes the nsite solute coordinates of insertion cnt.
  void insert_one(int stnum, int cnt, const T* conf, T* out) {
    const int s = nsite_slt;
    const int ab = molbeg[nummol - 1];
    for (int i = 0; i < 3 * s; ++i) out[i] = conf[i];
    auto com_of = [&](T c[3]) {
      T msum = 0;
      for (int a = 0; a < s; ++a) msum += sitemass[ab + a];
      for (int k = 0; k < 3; ++k) {
        T acc = 0;
        for (int a = 0; a < s; ++a) acc += out[3 * a + k] * sitemass[ab + a];
        c[k] = acc / msum;
      }
    };
    const uint32_t key[2] = {(uint32_t)p.iseed, kStreamTag};
    if (p.insposition == ERMOD_INSPOS_RANDOM) {
      T c[3];
      com_of(c);  // set_solute_origin -> set_solute_com(0)
      for (int a = 0; a < s; ++a) for (int k = 0; k < 3; ++k) out[3 * a + k] -= c[k];
      uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)stnum, 0u, 0u}, r4[4];
      philox4x32_10(ctr, key, r4);
      const T r[3] = {(T)u01(r4[0]), (T)u01(r4[1]), (T)u01(r4[2])};
      T com[3];
      for (int k = 0; k < 3; ++k) com[k] = cell[k][0] * r[0] + cell[k][1] * r[1] + cell[k][2] * r[2];
      com_of(c);  // set_solute_com(com)
      for (int a = 0; a < s; ++a) for (int k = 0; k < 3; ++k) out[3 * a + k] = (out[3 * a + k] - c[k]) + com[k];
    } else if (p.insposition >= ERMOD_INSPOS_SPHERE && p.insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC) {
      // insorigin 2: COM to the aggregate centre (insertion.F90:122-124), then set_shift_com (:164-200)
      T c[3];
      com_of(c);
      const T ag[3] = {(T)(float)aggcen[0], (T)(float)aggcen[1], (T)(float)aggcen[2]};
      for (int a = 0; a < s; ++a) for (int k = 0; k < 3; ++k) out[3 * a + k] = (out[3 * a + k] - c[k]) + ag[k];
      uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)stnum, 0u, 0u}, r4[4];
      philox4x32_10(ctr, key, r4);
      T sh[3];
      if (p.insposition == ERMOD_INSPOS_SPHERE) {
        const T lw3 = (T)p.lwreg * (T)p.lwreg * (T)p.lwreg, up3 = (T)p.upreg * (T)p.upreg * (T)p.upreg;
        const T t = std::pow((T)u01(r4[0]) * (up3 - lw3) + lw3, T(1) / T(3));
        T r[3] = {T(1), T(0), T(0)}, nrm = T(1);
        for (uint32_t att = 1; att <= 64; ++att) {
          uint32_t bc[4] = {(uint32_t)cnt, (uint32_t)stnum, att, 2u}, b4[4];
          philox4x32_10(bc, key, b4);
          const T x = (T)u01(b4[0]) * T(2) - T(1), y = (T)u01(b4[1]) * T(2) - T(1), z = (T)u01(b4[2]) * T(2) - T(1);
          const T n2 = x * x + y * y + z * z;
          if (T(0) < n2 && n2 <= T(1)) {
            r[0] = x; r[1] = y; r[2] = z;
            nrm = std::sqrt(n2);
            break;
          }
        }
        for (int k = 0; k < 3; ++k) sh[k] = t * r[k] / nrm;
      } else {
        T t = (T)u01(r4[2]) * ((T)p.upreg - (T)p.lwreg) + (T)p.lwreg;
        if (p.insposition == ERMOD_INSPOS_SLAB_SYMMETRIC && u01(r4[3]) > 0.5f) t = -t;
        const T l3 = std::sqrt(cell[0][2] * cell[0][2] + cell[1][2] * cell[1][2] + cell[2][2] * cell[2][2]);
        const T r[3] = {(T)u01(r4[0]), (T)u01(r4[1]), t / l3};
        for (int k = 0; k < 3; ++k) sh[k] = cell[k][0] * r[0] + cell[k][1] * r[1] + cell[k][2] * r[2];
      }
      for (int a = 0; a < s; ++a) for (int k = 0; k < 3; ++k) out[3 * a + k] += sh[k];
    }
    if (p.insposition == ERMOD_INSPOS_RMSD || p.insposition == ERMOD_INSPOS_GAUSS) {
      insert_refstr(stnum, cnt, conf, out);
      return;
    }
    orient(stnum, cnt, 1u, out);
  }

  // apply_orientation (insertion.F90:348-369) with the counters (cnt, stnum, attempt, tag)
  void orient(int stnum, int cnt, uint32_t tag, T* out) const {
    const int s = nsite_slt;
    const int ab = molbeg[nummol - 1];
    auto com_of = [&](T c[3]) {
      T msum = 0;
      for (int a = 0; a < s; ++a) msum += sitemass[ab + a];
      for (int k = 0; k < 3; ++k) {
        T acc = 0;
        for (int a = 0; a < s; ++a) acc += out[3 * a + k] * sitemass[ab + a];
        c[k] = acc / msum;
      }
    };
    const uint32_t key[2] = {(uint32_t)p.iseed, kStreamTag};
    if (p.insorient == ERMOD_INSROT_RANDOM) {
      T c[3];
      com_of(c);
      for (int a = 0; a < s; ++a) for (int k = 0; k < 3; ++k) out[3 * a + k] -= c[k];
      T q[4] = {T(1), T(0), T(0), T(0)};
      for (uint32_t att = 1; att <= 64; ++att) {
        uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)stnum, att, tag}, r4[4];
        philox4x32_10(ctr, key, r4);
        T t[4], n2 = 0;
        for (int i = 0; i < 4; ++i) { t[i] = (T)u01(r4[i]) * T(2) - T(1); n2 += t[i] * t[i]; }
        if (n2 < T(1)) {
          const T nn = std::sqrt(n2);
          for (int i = 0; i < 4; ++i) q[i] = t[i] / nn;
          break;
        }
      }
      for (int a = 0; a < s; ++a) {
        // res = q (0,v) conj(q), quaternion products as bestfit.F90:48-74
        const T v[3] = {out[3 * a], out[3 * a + 1], out[3 * a + 2]};
        T t0 = -(q[1] * v[0] + q[2] * v[1] + q[3] * v[2]);
        T t1 = q[2] * v[2] - q[3] * v[1] + q[0] * v[0];
        T t2 = q[3] * v[0] - q[1] * v[2] + q[0] * v[1];
        T t3 = q[1] * v[1] - q[2] * v[0] + q[0] * v[2];
        const T cj[4] = {q[0], -q[1], -q[2], -q[3]};
        // p = t * cj ; vector part
        const T r1 = t2 * cj[3] - t3 * cj[2] + t0 * cj[1] + cj[0] * t1;
        const T r2 = t3 * cj[1] - t1 * cj[3] + t0 * cj[2] + cj[0] * t2;
        const T r3 = t1 * cj[2] - t2 * cj[1] + t0 * cj[3] + cj[0] * t3;
        out[3 * a] = r1 + c[0]; out[3 * a + 1] = r2 + c[1]; out[3 * a + 2] = r3 + c[2];
      }
    }
  }

  // insorigin 3 (insertion.F90:86-94, 131-304, 617-643): fit the conformation onto this frame's best-fit
  // reference solute, shift (RMSD: uniform in a cube of half width upreg + 3 r_max; Gaussian: the
  // uniform / Gaussian mixture, weight divided by its density), orient, and retry until the RMSD to
  // the best-fit reference lies in lwreg..upreg (kInsTries attempts).
  void insert_refstr(int stnum, int cnt, const T* conf, T* out) {
    const int s = nsite_slt;
    const int ab = molbeg[nummol - 1];
    const uint32_t key[2] = {(uint32_t)p.iseed, kStreamTag};
    std::vector<double> cf(3 * s), fo(3 * s);
    for (int i = 0; i < 3 * s; ++i) cf[i] = (double)conf[i];
    double wfac = 1.0;
    bool ok = false;
    for (int tr = 0; tr < kInsTries && !ok; ++tr) {
      const uint32_t tg = (uint32_t)tr << 8;
      fit_rotate(s, ref_bf.data(), cf.data(), ref_slt_w.data(), s, cf.data(), fo.data());
      for (int i = 0; i < 3 * s; ++i) out[i] = (T)(float)fo[i];
      T sh[3];
      if (p.insposition == ERMOD_INSPOS_RMSD) {
        T msum = 0, c[3] = {0, 0, 0};
        for (int a = 0; a < s; ++a) msum += sitemass[ab + a];
        for (int k = 0; k < 3; ++k) {
          for (int a = 0; a < s; ++a) c[k] += out[3 * a + k] * sitemass[ab + a];
          c[k] /= msum;
        }
        T maxd = 0;
        for (int a = 0; a < s; ++a) {
          T d2 = 0;
          for (int k = 0; k < 3; ++k) d2 += (out[3 * a + k] - c[k]) * (out[3 * a + k] - c[k]);
          maxd = std::max(maxd, d2);
        }
        const T movmax = (T)p.upreg + T(3) * std::sqrt(maxd);
        uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)stnum, tg, 3u}, r4[4];
        philox4x32_10(ctr, key, r4);
        for (int k = 0; k < 3; ++k) sh[k] = movmax * (T(2) * (T)u01(r4[k]) - T(1));
      } else {
        T sc[3];
        if (((cnt + tr) & 1) == 0) {
          uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)stnum, tg, 4u}, r4[4];
          philox4x32_10(ctr, key, r4);
          for (int k = 0; k < 3; ++k) sc[k] = (T(2) * (T)u01(r4[k]) - T(1)) * (T)gauss_l[k];
        } else {
          for (int k = 0; k < 3; ++k) {
            sc[k] = 0;
            for (uint32_t att = 1; att <= 64; ++att) {
              uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)stnum, tg | att, 5u + (uint32_t)k}, r4[4];
              philox4x32_10(ctr, key, r4);
              const double u1 = std::max((double)u01(r4[0]), 1.0e-7), u2 = (double)u01(r4[1]);
              const double r = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2) * std::sqrt(0.5);
              if (std::abs(r) < gauss_l[k]) { sc[k] = (T)r; break; }
            }
          }
        }
        const T sq = sc[0] * sc[0] + sc[1] * sc[1] + sc[2] * sc[2];
        wfac /= 0.5 / gauss_z0 + 0.5 * std::exp(-(double)sq) / gauss_z1;
        T f[3];
        for (int k = 0; k < 3; ++k) f[k] = sc[k] / (T(2) * (T)gauss_l[k]);
        for (int k = 0; k < 3; ++k) sh[k] = cell[k][0] * f[0] + cell[k][1] * f[1] + cell[k][2] * f[2];
      }
      for (int a = 0; a < s; ++a) for (int k = 0; k < 3; ++k) out[3 * a + k] += sh[k];
      orient(stnum, cnt, 1u | tg, out);
      double d = 0, ws = 0;
      for (int a = 0; a < s; ++a) {
        double t = 0;
        for (int k = 0; k < 3; ++k) t += ((double)out[3 * a + k] - ref_bf[3 * a + k]) * ((double)out[3 * a + k] - ref_bf[3 * a + k]);
        d += ref_slt_w[a] * t;
        ws += ref_slt_w[a];
      }
      const double rmsd = std::sqrt(d / ws);
      ok = !((double)p.lwreg > rmsd || rmsd > (double)p.upreg);
    }
    if (!ok) ins_rejected[cnt] = 1;
    if (p.insposition == ERMOD_INSPOS_GAUSS) insw[cnt] *= wfac;
  }
  std::vector<char> ins_rejected;
  static constexpr int kInsTries = 1024;

  // binsearch + getiduv (engproc.F90:1078-1171).  Returns 0-based bin or <0 error.
  int getiduv(int pti, double engval, int* warn) {
    const double* coord;
    int idmin = 0, idnum;
    if (pti > 0) {
      for (int q = 0; q < pti - 1; ++q) idmin += uvmax[q];
      idnum = uvmax[pti - 1];
      coord = &uvcrd[idmin];
    } else {
      idnum = esmax;
      coord = escrd.data();
    }
    int idpti;
    if (engval < coord[0]) idpti = 0;
    else if (engval > coord[idnum - 1]) idpti = idnum;
    else {
      int rmin = 1, rmax = idnum + 1;
      while (rmax - rmin > 1) {
        const int rmid = (rmin + rmax - 1) >> 1;
        if (engval > coord[rmid - 1]) rmin = rmid + 1; else rmax = rmid + 1;
      }
      idpti = rmin - 1;
    }
    if (idpti <= 0) { err = "eng_min"; return ERMOD_ERR_ENG_MIN; }
    if (p.slttype == ERMOD_SLT_SOLN && pti > 0 && idpti > uvsoft[pti - 1]) { err = "eng_sft"; return ERMOD_ERR_ENG_SFT; }
    if (idpti == idnum && engval < 1.0e3 && warn_bin_firsttime) { *warn = 1; warn_bin_firsttime = false; }
    return idmin + idpti - 1;
  }

  // update_histogram (engproc.F90:858-964) for insertion / solute cnt
  int update_histogram(int cnt, T stat_weight_system, int* warn, std::vector<int>& insdst) {
    double engnmfc;
    const T u0 = (T)uvengy0[cnt];
    if (!p.wgtslf) engnmfc = 1.0;
    else {
      if (!voffset_initialized) { voffset = (double)u0; voffset_initialized = true; }
      const T factor = (T)((double)u0 - voffset);
      engnmfc = p.slttype == ERMOD_SLT_SOLN ? std::exp((double)factor / p.temp) : std::exp(-(double)factor / p.temp);
    }
    T total_weight = stat_weight_system * (T)insw[cnt];
    if (p.estype == ERMOD_ES_NPT) {  // volcorrect (engproc.F90:1022-1038)
      total_weight = total_weight * volume;
      if (p.cltype == ERMOD_EL_EWALD || p.cltype == ERMOD_EL_PME || p.cltype == ERMOD_EL_PPPM) {
        T qt = 0;
        for (int i = 0; i < nummol; ++i)
          if (sluvid[i] == ERMOD_PT_SOLVENT || sluvid[i] == ERMOD_PT_SOLUTE) qt += mol_charge[i];
        const T factor = (T)kPi * (qt * qt) / ((T)p.screen * (T)p.screen) / volume / T(2);
        total_weight = (T)((double)total_weight * std::exp((double)factor / p.temp));
      }
    }
    engnmfc = engnmfc * (double)total_weight;
    engnorm += engnmfc;
    engsmpl += 1.0;
    avslf += (double)total_weight;
    if (p.selfcal) {
      const int id = getiduv(0, (double)u0, warn);
      if (id < 0) return id;
      eself[id] += engnmfc;
    }
    minuv[0] = std::min(minuv[0], u0);
    maxuv[0] = std::max(maxuv[0], u0);
    std::fill(insdst.begin(), insdst.end(), 0);
    float* fl = &flceng[(size_t)cnt * numslv];
    for (int q = 0; q < numslv; ++q) fl[q] = 0.0f;
    const int tagslt = p.slttype == ERMOD_SLT_SOLN ? sltlist[cnt] : nummol - 1;
    std::vector<T> fls(numslv, T(0));
    for (int k = 0; k < slvmax; ++k) {
      const int i = tagpt[k];
      if (i == tagslt) continue;
      const int pti = uvspec[i];
      if (pti <= 0) { err = "eng_cns"; return ERMOD_ERR_ENG_CNS; }
      const double e = uvengy[(size_t)cnt * slvmax + k];
      const T pairep = (T)e;
      const int id = getiduv(pti, sizeof(T) == 4 ? (double)pairep : e, warn);
      if (id < 0) return id;
      insdst[id] += 1;
      fls[pti - 1] += pairep;
      minuv[pti] = std::min(minuv[pti], pairep);
      maxuv[pti] = std::max(maxuv[pti], pairep);
    }
    for (int q = 0; q < numslv; ++q) fl[q] = (float)fls[q];
    if (p.slttype == ERMOD_SLT_SOLN)
      for (int q = 0; q < numslv; ++q) slnuv[q] += (T)((double)fls[q] * engnmfc);
    std::vector<int> nz;
    for (int b = 0; b < ermax; ++b)
      if (insdst[b] != 0) { edens[b] += engnmfc * (double)insdst[b]; nz.push_back(b); }
    if (p.corrcal) {
      for (int bi : nz)
        for (int bj : nz)
          ecorr[(size_t)bi * ermax + bj] += engnmfc * (double)insdst[bi] * (double)insdst[bj];
    }
    return ERMOD_OK;
  }

  int engconst(int stnum, const float* sitepos, const float* cellin, float stat_weight_system,
               const float* ins_conf, const float* ins_weight, float* flceng_out) {
    err.clear();
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) cell[i][j] = (T)cellin[j * 3 + i];
    get_inverted_cell();
    const bool refs = p.slttype != ERMOD_SLT_SOLN;
    const int s = nsite_slt;
    // sitepos: physical atoms first, then maxdst solute copies (refs)
    const size_t next = refs ? (size_t)maxdst * s : 0;
    pos.assign(3 * ((size_t)numatm_phys + next), T(0));
    for (size_t i = 0; i < 3 * (size_t)numatm_phys; ++i) pos[i] = (T)sitepos[i];
    insw.assign(maxdst, 1.0);
    if (refs) {
      if ((p.insposition == ERMOD_INSPOS_RANDOM || p.insposition == ERMOD_INSPOS_SLAB_GENERIC ||
           p.insposition == ERMOD_INSPOS_SLAB_SYMMETRIC) && p.boxshp == ERMOD_SYS_NONPERIODIC)
        return fail(ERMOD_ERR_INS_GEO, "ins_geo");
      if (p.insposition >= ERMOD_INSPOS_SPHERE && p.insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC)
        aggregate_center(sitepos);
      if (p.insposition >= ERMOD_INSPOS_RMSD) {
        if (ref_atom.empty()) return fail(ERMOD_ERR_ARG, "ins_ref");
        reffit_frame(sitepos);
        if (p.insposition == ERMOD_INSPOS_GAUSS && !gauss_init) {   // insertion.F90:268-274, first call
          gauss_z0 = 8.0; gauss_z1 = std::pow(kPi, 1.5);
          for (int k = 0; k < 3; ++k) {
            const double len = std::sqrt((double)cell[0][k] * cell[0][k] + (double)cell[1][k] * cell[1][k] +
                                         (double)cell[2][k] * cell[2][k]);
            gauss_l[k] = (double)(float)(0.5 * len / p.upreg);
            gauss_z0 *= gauss_l[k];
            gauss_z1 *= std::erf(gauss_l[k]);
          }
          gauss_z0 = (double)(float)gauss_z0; gauss_z1 = (double)(float)gauss_z1;
          gauss_init = true;
        }
      }
      if (ins_weight) for (int c = 0; c < maxdst; ++c) insw[c] = ins_weight[c];
      ins_rejected.assign(maxdst, 0);
      std::vector<T> conf(3 * s);
#pragma omp parallel for num_threads(nthreads) firstprivate(conf) schedule(static)
      for (int cnt = 0; cnt < maxdst; ++cnt) {
        const float* src = ins_conf ? ins_conf + (size_t)3 * s * cnt : nullptr;
        for (int i = 0; i < 3 * s; ++i) conf[i] = src ? (T)src[i] : bfcoord[i];
        insert_one(stnum, cnt, conf.data(), &pos[3 * ((size_t)numatm_phys + (size_t)cnt * s)]);
      }
      for (int c = 0; c < maxdst; ++c) if (ins_rejected[c]) return fail(ERMOD_ERR_INS_GEO, "ins_rej");
    }
    // soln: check_mol_configuration (engproc.F90:1197-1324) for sphere / slab regions;
    // a rejected solute gets no energies and no update_histogram (:447-450, 754-755)
    std::vector<char> skip(maxdst, 0);
    if (!refs && p.insposition == ERMOD_INSPOS_RMSD) {   // engproc.F90:1249-1269
      if (ref_atom.empty()) return fail(ERMOD_ERR_ARG, "ins_ref");
      reffit_frame(sitepos);
      const int ns = (int)ref_slt_w.size();
      for (int cnt = 0; cnt < maxdst; ++cnt) {
        const int a0 = molbeg[sltlist[cnt]];
        double d = 0, ws = 0;
        for (int a = 0; a < ns; ++a) {
          double t = 0;
          for (int k = 0; k < 3; ++k) {
            const double x = (double)sitepos[3 * (a0 + a) + k] - ref_bf[3 * a + k];
            t += x * x;
          }
          d += ref_slt_w[a] * t;
          ws += ref_slt_w[a];
        }
        const double rmsd = std::sqrt(d / ws);
        skip[cnt] = ((double)p.lwreg > rmsd || rmsd > (double)p.upreg) ? 1 : 0;
      }
    }
    if (!refs && p.insposition >= ERMOD_INSPOS_SPHERE && p.insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC) {
      const bool slab = p.insposition != ERMOD_INSPOS_SPHERE;
      if (slab && p.boxshp == ERMOD_SYS_NONPERIODIC) return fail(ERMOD_ERR_INS_GEO, "eng_slb");
      aggregate_center(sitepos);
      const T l3 = std::sqrt(cell[0][2] * cell[0][2] + cell[1][2] * cell[1][2] + cell[2][2] * cell[2][2]);
      for (int cnt = 0; cnt < maxdst; ++cnt) {
        const int tagslt = sltlist[cnt];
        double c[3] = {0.0, 0.0, 0.0}, msum = 0.0;   // relative_com (:1300-1323)
        for (int a = molbeg[tagslt]; a < molbeg[tagslt + 1]; ++a) {
          const double m = (double)(float)sitemass[a];
          for (int k = 0; k < 3; ++k) c[k] += m * (double)sitepos[3 * a + k];
          msum += m;
        }
        T dx[3];
        for (int k = 0; k < 3; ++k) dx[k] = (T)(float)(c[k] / msum) - (T)(float)aggcen[k];
        T dist;
        if (!slab) {
          dist = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
        } else {
          dist = (invcl[2][0] * dx[0] + invcl[2][1] * dx[1] + invcl[2][2] * dx[2]) * l3;
          if (p.insposition == ERMOD_INSPOS_SLAB_SYMMETRIC) dist = std::abs(dist);
        }
        skip[cnt] = ((T)p.lwreg > dist || dist > (T)p.upreg) ? 1 : 0;
      }
    }
    if (!refs && p.insstructure == ERMOD_INSSTR_RMSD) {   // engproc.F90:1277-1295
      if (ref_atom.empty()) return fail(ERMOD_ERR_ARG, "ins_ref");
      const int ns = (int)ref_slt_w.size();
      std::vector<double> cf(3 * ns), fo(3 * ns);
      for (int cnt = 0; cnt < maxdst; ++cnt) {
        if (skip[cnt]) continue;                            // the region check came first
        const int a0 = molbeg[sltlist[cnt]];
        for (int i = 0; i < 3 * ns; ++i) cf[i] = (double)sitepos[3 * a0 + i];
        // rmsd_bestfit (bestfit.F90:339-346): fit, the fitted points stored as default reals
        fit_rotate(ns, ref_slt.data(), cf.data(), ref_slt_w.data(), ns, cf.data(), fo.data());
        double d = 0, ws = 0;
        for (int a = 0; a < ns; ++a) {
          double t = 0;
          for (int k = 0; k < 3; ++k) {
            const double x = (double)(float)fo[3 * a + k] - ref_slt[3 * a + k];
            t += x * x;
          }
          d += ref_slt_w[a] * t;
          ws += ref_slt_w[a];
        }
        const double rmsd = std::sqrt(d / ws);
        skip[cnt] = ((double)p.lwstr > rmsd || rmsd > (double)p.upstr) ? 1 : 0;
      }
    }
    // PME setup (engconst :419-437)
    const bool pme = p.cltype == ERMOD_EL_PME || p.cltype == ERMOD_EL_PPPM;
    std::vector<T> wslv;
    std::vector<int> gslv, slvtag(nummol, -1);
    if (pme) {
      bool changed = !pme_initialized;
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) if (prevcl[i][j] != cell[i][j]) changed = true;
      if (changed && p.cltype == ERMOD_EL_PPPM) {
        float cf[3][3];
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) cf[i][j] = (float)cell[i][j];
        pppm_mrange(cf, p.screen, K1, K2, K3, mrange);
        if (mrange[0] < 0 || mrange[1] < 0 || mrange[2] < 0) return fail(ERMOD_ERR_ARG, "pppm_mrg");
        pppm_greenfunc();
      } else if (changed) {
        spline_greenfunc();
      }
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) prevcl[i][j] = cell[i][j];
      pme_initialized = true;
      // recpcal_prepare_solvent (recpcal.F90:340-357)
      int ptrnk = 0;
      for (int k = 0; k < slvmax; ++k) { slvtag[tagpt[k]] = ptrnk; ptrnk += numsite[tagpt[k]]; }
      wslv.resize((size_t)ptrnk * 3 * p.splodr);
      gslv.resize((size_t)ptrnk * 3);
      int pa = 0;
      for (int k = 0; k < slvmax; ++k) {
        const int i = tagpt[k];
        for (int sid = 0; sid < numsite[i]; ++sid, ++pa)
          spline_site(&pos[3 * (size_t)pa], &wslv[(size_t)pa * 3 * p.splodr], &gslv[(size_t)pa * 3]);
      }
    }
    // realcal_prepare (realcal.F90:30-48)
    const size_t natoms = (size_t)numatm_phys + next;
    if (p.boxshp == ERMOD_SYS_PERIODIC) {
      const int rc = normalize_periodic(natoms);
      if (rc != ERMOD_OK) return rc;
    } else {
      posn.assign(pos.begin(), pos.begin() + 3 * natoms);
    }
    // physical atom index of each physical molecule's first site in pos[]
    std::vector<int> physbeg(nummol, -1);
    { int a = 0; for (int k = 0; k < slvmax; ++k) { physbeg[tagpt[k]] = a; a += numsite[tagpt[k]]; } }
    uvengy.assign((size_t)maxdst * slvmax, 0.0);
    uvengy0.assign(maxdst, 0.0);
    flceng.assign((size_t)maxdst * numslv, 0.0f);
    std::vector<T> selfrec(maxdst, T(0)), selfreal(maxdst, T(0));
    const bool bare = p.cltype == ERMOD_EL_COULOMB;
    const T pivol = (T)kPi / (T)p.screen / (T)p.screen / volume;
#pragma omp parallel num_threads(nthreads)
    {
      std::vector<T> phi, xs;
      std::vector<std::complex<T>> g, line, scr;
      std::vector<int> satoms;
#pragma omp for schedule(dynamic, 1)
      for (int cnt = 0; cnt < maxdst; ++cnt) {
        if (skip[cnt]) continue;
        const int tagslt = refs ? nummol - 1 : sltlist[cnt];
        const int ns = numsite[tagslt];
        satoms.resize(ns);
        for (int a = 0; a < ns; ++a) satoms[a] = molbeg[tagslt] + a;
        const size_t sbase = refs ? (size_t)numatm_phys + (size_t)cnt * s : (size_t)physbeg[tagslt];
        const T* spos = &pos[3 * sbase];
        const T* sposn = &posn[3 * sbase];
        if (pme) selfrec[cnt] = pme_solute(spos, satoms.data(), ns, phi, g, line, scr);
        for (int k = 0; k < slvmax; ++k) {
          const int i = tagpt[k];
          if (i == tagslt) continue;
          // realcal: site-pair sums accumulated per solute site (realcal.F90:259-358)
          T e = T(0);
          for (int is = 0; is < ns; ++is) {
            T pairep = T(0);
            for (int js = 0; js < numsite[i]; ++js)
              pairep += pair_energy(sposn + 3 * is, &posn[3 * ((size_t)physbeg[i] + js)], satoms[is], molbeg[i] + js, bare);
            e += pairep;
          }
          if (pme) {
            e += pme_gather(i, phi, wslv, gslv, slvtag);
            e -= pivol * mol_charge[tagslt] * mol_charge[i];  // residual_ene(_refs)
          }
          uvengy[(size_t)cnt * slvmax + k] = (double)e;
        }
        xs.assign(sposn, sposn + 3 * ns);
        selfreal[cnt] = real_self(xs.data(), satoms.data(), ns);
      }
    }
    // uvengy0 (engproc.F90:828-855); rigid refs reuse the first real self energy
    for (int cnt = 0; cnt < maxdst; ++cnt) {
      if (skip[cnt]) continue;
      const int tagslt = refs ? nummol - 1 : sltlist[cnt];
      T pairep;
      if (refs) {
        const uint64_t h = hash_coords(&pos[3 * ((size_t)numatm_phys + (size_t)cnt * s)], 3 * s);
        if (h == solute_hash || (p.slttype == ERMOD_SLT_REFS_RIGID && solute_hash != 0)) pairep = usreal;
        else { pairep = selfreal[cnt]; usreal = pairep; }
        solute_hash = h;
      } else {
        pairep = selfreal[cnt];
      }
      uvengy0[cnt] = (double)(selfrec[cnt] + pairep + residual_self(mol_charge[tagslt]));
    }
    int warn = 0;
    std::vector<int> insdst(ermax);
    for (int cnt = 0; cnt < maxdst; ++cnt) {
      if (skip[cnt]) continue;
      const int rc = update_histogram(cnt, (T)stat_weight_system, &warn, insdst);
      if (rc < 0) return rc;
    }
    if (flceng_out) std::memcpy(flceng_out, flceng.data(), sizeof(float) * flceng.size());
    if (warn) { err = "mbin"; return ERMOD_WARN_MBIN; }
    return ERMOD_OK;
  }

  void engclear() {  // engproc.F90:321-340
    std::fill(edens.begin(), edens.end(), 0.0);
    std::fill(ecorr.begin(), ecorr.end(), 0.0);
    std::fill(eself.begin(), eself.end(), 0.0);
    std::fill(slnuv.begin(), slnuv.end(), T(0));
    avslf = engnorm = engsmpl = 0.0;
  }

  void fetch(ermod_accum* o, bool normalise) const {
    const double nrm = normalise ? engnorm : 1.0;
    if (o->edens) for (int i = 0; i < ermax; ++i) o->edens[i] = edens[i] / nrm;
    if (o->ecorr && p.corrcal) for (size_t i = 0; i < ecorr.size(); ++i) o->ecorr[i] = ecorr[i] / nrm;
    if (o->eself && p.selfcal) for (int i = 0; i < esmax; ++i) o->eself[i] = eself[i] / nrm;
    if (o->slnuv) for (int i = 0; i < numslv; ++i) o->slnuv[i] = (float)(slnuv[i] / nrm);   // aveuv (engproc.F90:622)
    if (o->minuv) for (int i = 0; i <= numslv; ++i) o->minuv[i] = (float)minuv[i];
    if (o->maxuv) for (int i = 0; i <= numslv; ++i) o->maxuv[i] = (float)maxuv[i];
    o->avslf = avslf / nrm;
    o->engnorm = engnorm;
    o->engsmpl = engsmpl;
    o->voffset = voffset;
    o->voffset_initialized = voffset_initialized ? 1 : 0;
  }
};

struct Handle {
  int precision = 8;
  Oracle<double>* d = nullptr;
  Oracle<float>* f = nullptr;
};

// enginit mesh (engproc.F90:171-226, 264-281) for one &hist set
int mesh_one(const ermod_hist* h, int pti, std::vector<double>& ercrd, int* pemax_o, int* pesoft_o) {
  const int rglmax = 5;
  double ecdmin = h->ecdmin, ecfmns = h->ecfmns, ecdcen = h->ecdcen, eccore = h->eccore, ecdmax = h->ecdmax;
  const double eclbin = h->eclbin, ecfbin = h->ecfbin, ec0bin = h->ec0bin, finfac = h->finfac;
  int pecore = h->pecore;
  (void)pti;
  const double ectmvl = finfac * ecfbin;
  ecdmin = ecdmin - ectmvl;
  ecfmns = ecfmns - ectmvl;
  const double ecmns0 = ecdcen - ectmvl;
  const double ecpls0 = 2.0 * ecdcen - ecmns0;
  const double ecfpls = 2.0 * ecdcen - ecfmns;
  eccore = eccore + ecfpls - ecdcen;
  const double cdrgvl[7] = {ecdmin, ecfmns, ecmns0, ecpls0, ecfpls, eccore, ecdmax};
  int uprgcd[7];
  uprgcd[0] = 1;
  for (int regn = 1; regn <= rglmax; ++regn) {
    double factor = (regn == 1 || regn == 5) ? eclbin : (regn == 2 || regn == 4) ? ecfbin : ec0bin;
    const double incre = cdrgvl[regn] - cdrgvl[regn - 1];
    if (incre < factor) return ERMOD_ERR_ENG_ECD;
    const int iduv = (int)std::lround(incre / factor);
    uprgcd[regn] = uprgcd[regn - 1] + iduv;
  }
  const int pesoft = uprgcd[rglmax] - uprgcd[0];
  const int pemax = pesoft + pecore;
  uprgcd[rglmax + 1] = pemax;
  ercrd.assign(std::max(pemax, uprgcd[rglmax]) + 2, 0.0);  // 1-based
  for (int r = 0; r <= rglmax + 1; ++r) ercrd[uprgcd[r]] = cdrgvl[r];
  const int last = pecore == 0 ? rglmax : rglmax + 1;
  for (int regn = 1; regn <= last; ++regn) {
    const int minrg = uprgcd[regn - 1], maxrg = uprgcd[regn];
    double incre = 0.0;
    if (regn <= rglmax) incre = ercrd[maxrg] - ercrd[minrg];
    if (regn == rglmax + 1) incre = std::log(ercrd[maxrg] / ercrd[minrg]);
    const double factor = incre / (double)(maxrg - minrg);
    for (int iduv = minrg; iduv <= maxrg - 1; ++iduv) {
      const double inc = factor * (double)(iduv - minrg);
      if (regn <= rglmax) ercrd[iduv] = ercrd[minrg] + inc;
      if (regn == rglmax + 1) ercrd[iduv] = ercrd[minrg] * std::exp(inc);
    }
  }
  *pemax_o = pemax;
  *pesoft_o = pesoft;
  return ERMOD_OK;
}

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) { philox4x32_10(ctr, key, out); }

// calc_gfb_pppm (recpcal.F90:179-198) for one order: out[0 .. order-1]
void orc_pppm_gfb(int order, double* out) {
  ermod_params p{};
  p.splodr = order;
  Oracle<double> o;
  o.p = p;
  o.calc_gfb_pppm();
  for (int l = 0; l < order; ++l) out[l] = o.gfb[l];
}

double orc_spline_value(int order, double x) {
  Spline<double> s;
  s.init(order);
  return s.value(x);
}

// binsearch (engproc.F90:1078-1108), 0-based count semantics: returns ret as the reference
int orc_binsearch(const double* coord, int n, double v) {
  if (v < coord[0]) return 0;
  if (v > coord[n - 1]) return n;
  int rmin = 1, rmax = n + 1;
  while (rmax - rmin > 1) {
    const int rmid = (rmin + rmax - 1) >> 1;
    if (v > coord[rmid - 1]) rmin = rmid + 1; else rmax = rmid + 1;
  }
  return rmin - 1;
}

int orc_enginit_mesh(const ermod_hist* hist, int numslv, double* uvcrd, int* uvmax, int* uvsoft,
                     double* escrd, int* ermax, int* esmax) {
  std::vector<double> ercrd;
  int pemax = 0, pesoft = 0;
  const int rc = mesh_one(hist, 0, ercrd, &pemax, &pesoft);
  if (rc != ERMOD_OK) return rc;
  if (ermax) *ermax = numslv * pemax;
  if (esmax) *esmax = pesoft;
  for (int q = 0; q < numslv; ++q) {
    if (uvmax) uvmax[q] = pemax;
    if (uvsoft) uvsoft[q] = pesoft;
    if (uvcrd) for (int i = 0; i < pemax; ++i) uvcrd[q * pemax + i] = ercrd[i + 1];
  }
  if (escrd) for (int i = 0; i < pesoft; ++i) escrd[i] = ercrd[i + 1];
  return ERMOD_OK;
}

void* orc_create(const ermod_params* p, const ermod_topology* t, const ermod_mesh* m, int precision,
                 int nthreads, int* status) {
  Handle* h = new Handle();
  h->precision = precision;
  int rc;
  if (precision == 4) { h->f = new Oracle<float>(); rc = h->f->create(p, t, m, nthreads); }
  else { h->d = new Oracle<double>(); rc = h->d->create(p, t, m, nthreads); }
  if (status) *status = rc;
  return h;
}

void orc_destroy(void* hv) {
  Handle* h = (Handle*)hv;
  delete h->d;
  delete h->f;
  delete h;
}

void orc_engclear(void* hv) {
  Handle* h = (Handle*)hv;
  if (h->d) h->d->engclear(); else h->f->engclear();
}

int orc_engconst(void* hv, int stnum, const float* sitepos, const float* cell, float wsys,
                 const float* ins_conf, const float* ins_weight, float* flceng) {
  Handle* h = (Handle*)hv;
  if (h->d) return h->d->engconst(stnum, sitepos, cell, wsys, ins_conf, ins_weight, flceng);
  return h->f->engconst(stnum, sitepos, cell, wsys, ins_conf, ins_weight, flceng);
}

void orc_fetch(void* hv, ermod_accum* out, int normalise) {
  Handle* h = (Handle*)hv;
  if (h->d) h->d->fetch(out, normalise != 0); else h->f->fetch(out, normalise != 0);
}

void orc_get_uvengy(void* hv, double* uvengy, double* uvengy0) {
  Handle* h = (Handle*)hv;
  const std::vector<double>& u = h->d ? h->d->uvengy : h->f->uvengy;
  const std::vector<double>& u0 = h->d ? h->d->uvengy0 : h->f->uvengy0;
  if (uvengy) std::memcpy(uvengy, u.data(), sizeof(double) * u.size());
  if (uvengy0) std::memcpy(uvengy0, u0.data(), sizeof(double) * u0.size());
}

void orc_get_insertions(void* hv, float* ins) {
  Handle* h = (Handle*)hv;
  if (h->d) {
    Oracle<double>& o = *h->d;
    const size_t n = (size_t)3 * o.nsite_slt * o.maxdst;
    for (size_t i = 0; i < n; ++i) ins[i] = (float)o.pos[3 * (size_t)o.numatm_phys + i];
  } else {
    Oracle<float>& o = *h->f;
    const size_t n = (size_t)3 * o.nsite_slt * o.maxdst;
    for (size_t i = 0; i < n; ++i) ins[i] = o.pos[3 * (size_t)o.numatm_phys + i];
  }
}

// engfac half spectrum [K3][K2][K1/2+1] of the last frame
void orc_get_engfac(void* hv, double* out) {
  Handle* h = (Handle*)hv;
  if (h->d) { for (size_t i = 0; i < h->d->engfac.size(); ++i) out[i] = h->d->engfac[i]; }
  else { for (size_t i = 0; i < h->f->engfac.size(); ++i) out[i] = h->f->engfac[i]; }
}

void orc_get_insw(void* hv, double* w) {
  Handle* h = (Handle*)hv;
  const std::vector<double>& v = h->d ? h->d->insw : h->f->insw;
  std::memcpy(w, v.data(), sizeof(double) * v.size());
}

int orc_set_refstructure(void* hv, int refspec, int nhost, const float* hc, const float* hw, const float* sc,
                         const float* sw) {
  Handle* h = (Handle*)hv;
  return h->d ? h->d->set_refstructure(refspec, nhost, hc, hw, sc, sw)
              : h->f->set_refstructure(refspec, nhost, hc, hw, sc, sw);
}

const char* orc_last_error(void* hv) {
  Handle* h = (Handle*)hv;
  return h->d ? h->d->err.c_str() : h->f->err.c_str();
}

}  // extern "C"
