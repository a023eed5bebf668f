// erdst_io.cpp -- erdst's on-disk formats on the host: the DCD trajectory
// reader that stands in for the VMD molfile plugin path (vmdfio.c:132-385),
// and engstore's output files (engproc.F90:630-722) with the reference's
// Fortran edit descriptors as gfortran prints them.
//
// DCD layout (CHARMM / NAMD / X-PLOR), every block a Fortran unformatted
// record framed by a length marker before and after:
//   header  "CORD" + 20 int32 control words (84 bytes).  Word 8 (0-based) is
//           the fixed-atom count, word 10 the unit-cell flag and word 11 the
//           4-D flag of CHARMM files (word 19, the CHARMM version, non-zero);
//           X-PLOR files (word 19 zero) carry neither.
//   title   int32 count + count x 80 characters
//   natoms  one int32
//   frames  [6 FP64 unit cell] + x[natoms] + y[natoms] + z[natoms] FP32
//           (+ a fourth coordinate record in 4-D files, skipped).
// The unit cell holds A, gamma, B, beta, alpha, C; the angles are cosines when
// all three lie in [-1, 1] (CHARMM, NAMD >= 2.5) and degrees otherwise.  The
// cell vectors follow vmdfio.c:355-373: a = (A, 0, 0), b = B (cos g, sin g, 0),
// c = C (u, v, w) with u = cos b, v = (cos a - cos g u) / sin g, w = sqrt(1 - u^2 - v^2).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ermod_io.h"
#include "bestfit.cuh"

namespace {

thread_local const char* g_err = "";

int io_fail(int code, const char* name) {
  g_err = name;
  return code;
}

uint32_t bswap32(uint32_t v) {
  return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}

uint64_t bswap64(uint64_t v) {
  return ((uint64_t)bswap32((uint32_t)v) << 32) | bswap32((uint32_t)(v >> 32));
}

}  // namespace

struct ermod_traj {
  FILE* f = nullptr;
  bool swap = false;         // file byte order differs from the host's
  int marker = 4;            // record-marker width in bytes (4 or 8)
  bool charmm = false, has_cell = false, dim4 = false;
  int32_t natoms = 0, nframes = 0;
  long first_frame = 0;      // file offset of the first frame
  std::vector<float> buf;

  // Reads one record's leading marker; returns its length or -1 at end of file.
  int64_t head() {
    if (marker == 4) {
      uint32_t v;
      if (std::fread(&v, 4, 1, f) != 1) return -1;
      if (swap) v = bswap32(v);
      return (int64_t)(int32_t)v;
    }
    uint64_t v;
    if (std::fread(&v, 8, 1, f) != 1) return -1;
    if (swap) v = bswap64(v);
    return (int64_t)v;
  }
  // Reads a record of exactly n bytes into dst (or skips it when dst is null).
  // 0 on success, ERMOD_TRJ_EOF when the file ends before the record starts.
  int record(void* dst, int64_t n) {
    const int64_t len = head();
    if (len < 0) return ERMOD_TRJ_EOF;
    if (len != n) return io_fail(ERMOD_ERR_FORMAT, "trj_rec");
    if (dst) {
      if (std::fread(dst, 1, (size_t)n, f) != (size_t)n) return io_fail(ERMOD_ERR_FORMAT, "trj_rec");
    } else if (std::fseek(f, (long)n, SEEK_CUR) != 0) {
      return io_fail(ERMOD_ERR_FORMAT, "trj_rec");
    }
    if (head() != n) return io_fail(ERMOD_ERR_FORMAT, "trj_rec");
    return 0;
  }
  void fix32(void* p, size_t count) {
    if (!swap) return;
    uint32_t* w = static_cast<uint32_t*>(p);
    for (size_t i = 0; i < count; ++i) w[i] = bswap32(w[i]);
  }
  void fix64(void* p, size_t count) {
    if (!swap) return;
    uint64_t* w = static_cast<uint64_t*>(p);
    for (size_t i = 0; i < count; ++i) w[i] = bswap64(w[i]);
  }
};

extern "C" int32_t ermod_traj_open(const char* path, ermod_traj** out, int32_t* natoms, int32_t* nframes,
                                   int32_t* has_cell) {
  if (!path || !out) return io_fail(ERMOD_ERR_ARG, "trj_arg");
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return io_fail(ERMOD_ERR_IO, "trj_opn");
  ermod_traj* t = new ermod_traj;
  t->f = f;
  auto bad = [&](int code, const char* name) {
    std::fclose(f);
    delete t;
    return io_fail(code, name);
  };
  // byte order and marker width from the 84-byte header record
  unsigned char m[8];
  if (std::fread(m, 1, 8, f) != 8) return bad(ERMOD_ERR_FORMAT, "trj_hdr");
  uint32_t m32;
  uint64_t m64;
  std::memcpy(&m32, m, 4);
  std::memcpy(&m64, m, 8);
  // the 64-bit forms first: a little-endian 64-bit marker also reads as 84 in its low word
  if (m64 == 84u) { t->marker = 8; t->swap = false; }
  else if (bswap64(m64) == 84u) { t->marker = 8; t->swap = true; }
  else if (m32 == 84u) { t->marker = 4; t->swap = false; }
  else if (bswap32(m32) == 84u) { t->marker = 4; t->swap = true; }
  else return bad(ERMOD_ERR_FORMAT, "trj_hdr");
  std::fseek(f, 0, SEEK_SET);
  unsigned char hdr[84];
  if (t->record(hdr, 84) != 0) return bad(ERMOD_ERR_FORMAT, "trj_hdr");
  if (std::memcmp(hdr, "CORD", 4) != 0) return bad(ERMOD_ERR_FORMAT, "trj_hdr");
  int32_t ic[20];
  std::memcpy(ic, hdr + 4, 80);
  t->fix32(ic, 20);
  t->charmm = ic[19] != 0;
  t->has_cell = t->charmm && ic[10] != 0;
  t->dim4 = t->charmm && ic[11] != 0;
  t->nframes = ic[0];
  if (ic[8] != 0) return bad(ERMOD_ERR_UNSUPPORTED, "trj_fix");
  // title block: int32 count + count x 80 characters
  const int64_t tl = t->head();
  if (tl < 4) return bad(ERMOD_ERR_FORMAT, "trj_ttl");
  if (std::fseek(f, (long)tl, SEEK_CUR) != 0 || t->head() != tl) return bad(ERMOD_ERR_FORMAT, "trj_ttl");
  int32_t na;
  if (t->record(&na, 4) != 0) return bad(ERMOD_ERR_FORMAT, "trj_nat");
  t->fix32(&na, 1);
  if (na <= 0) return bad(ERMOD_ERR_FORMAT, "trj_nat");
  t->natoms = na;
  t->first_frame = std::ftell(f);
  t->buf.resize((size_t)na);
  if (natoms) *natoms = na;
  if (nframes) *nframes = t->nframes;
  if (has_cell) *has_cell = t->has_cell ? 1 : 0;
  *out = t;
  return ERMOD_OK;
}

extern "C" int32_t ermod_traj_read(ermod_traj* t, int32_t natoms, float* crd, float* cell) {
  if (!t || !crd || !cell) return io_fail(ERMOD_ERR_ARG, "trj_arg");
  if (natoms != t->natoms) return io_fail(ERMOD_ERR_ARG, "trj_nat");
  for (int i = 0; i < 9; ++i) cell[i] = 0.f;
  if (t->has_cell) {
    double uc[6];
    const int rc = t->record(uc, 48);
    if (rc != 0) return rc;
    t->fix64(uc, 6);
    // the molfile timestep keeps A, B, C and the angles (degrees) in FP32
    float A = (float)uc[0], B = (float)uc[2], Cc = (float)uc[5], alpha, beta, gamma;
    if (uc[1] >= -1.0 && uc[1] <= 1.0 && uc[3] >= -1.0 && uc[3] <= 1.0 && uc[4] >= -1.0 && uc[4] <= 1.0) {
      const double half_pi = 1.57079632679489661923;
      alpha = (float)(90.0 - std::asin(uc[4]) * 90.0 / half_pi);
      beta = (float)(90.0 - std::asin(uc[3]) * 90.0 / half_pi);
      gamma = (float)(90.0 - std::asin(uc[1]) * 90.0 / half_pi);
    } else {
      alpha = (float)uc[4];
      beta = (float)uc[3];
      gamma = (float)uc[1];
    }
    const double pi = 3.14159265358979323846;
    const double x = std::cos(gamma * pi / 180.0), y = std::sin(gamma * pi / 180.0);
    const double u = std::cos(beta * pi / 180.0);
    const double v = (std::cos(alpha * pi / 180.0) - x * u) / y;
    const double w = std::sqrt(1.0 - u * u - v * v);
    cell[0] = A;
    cell[3] = (float)(B * x);
    cell[4] = (float)(B * y);
    cell[6] = (float)(Cc * u);
    cell[7] = (float)(Cc * v);
    cell[8] = (float)(Cc * w);
  }
  const int64_t n = (int64_t)natoms * 4;
  for (int k = 0; k < 3; ++k) {
    const int rc = t->record(t->buf.data(), n);
    if (rc == ERMOD_TRJ_EOF && (k > 0 || t->has_cell)) return io_fail(ERMOD_ERR_FORMAT, "trj_rec");
    if (rc != 0) return rc;
    t->fix32(t->buf.data(), (size_t)natoms);
    for (int i = 0; i < natoms; ++i) crd[3 * i + k] = t->buf[i];
  }
  if (t->dim4) {
    const int rc = t->record(nullptr, n);
    if (rc != 0) return rc == ERMOD_TRJ_EOF ? io_fail(ERMOD_ERR_FORMAT, "trj_rec") : rc;
  }
  return ERMOD_OK;
}

extern "C" int32_t ermod_traj_rewind(ermod_traj* t) {
  if (!t) return io_fail(ERMOD_ERR_ARG, "trj_arg");
  if (std::fseek(t->f, t->first_frame, SEEK_SET) != 0) return io_fail(ERMOD_ERR_IO, "trj_rwd");
  return ERMOD_OK;
}

extern "C" void ermod_traj_close(ermod_traj* t) {
  if (!t) return;
  if (t->f) std::fclose(t->f);
  delete t;
}

// ---------------------------------------------------------------------------
// Fortran formatted output (the edit descriptors engstore uses), as gfortran
// writes them: right-justified fields, asterisks when a value does not fit,
// the optional leading zero of F and E output dropped only when the field is
// one character short.  Decimal digits come from the C library's correctly
// rounded conversion, as gfortran's own do.
// ---------------------------------------------------------------------------
namespace fmt {

std::string fit(const std::string& s, int w) {
  if ((int)s.size() > w) return std::string((size_t)w, '*');
  return std::string((size_t)(w - (int)s.size()), ' ') + s;
}

// drop the optional zero of "0." / "-0." when the field is one character short
std::string fit_number(std::string s, int w) {
  if ((int)s.size() == w + 1) {
    if (s.compare(0, 2, "0.") == 0) s.erase(0, 1);
    else if (s.compare(0, 3, "-0.") == 0) s.erase(1, 1);
  }
  return fit(s, w);
}

// Iw
std::string I(long v, int w) { return fit(std::to_string(v), w); }

// Aw for output: leading blanks when the string is shorter, its leftmost w characters otherwise
std::string A(const std::string& s, int w) {
  if ((int)s.size() >= w) return s.substr(0, (size_t)w);
  return std::string((size_t)(w - (int)s.size()), ' ') + s;
}

// Fw.d
std::string F(double x, int w, int d) {
  char b[512];
  std::snprintf(b, sizeof(b), "%#.*f", d, x);
  return fit_number(b, w);
}

// d significant digits of |x| and the decimal exponent e with |x| ~ 0.d1d2... x 10^e
void digits(double x, int d, std::string& dig, int& e) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.*e", d - 1, std::fabs(x));
  dig.clear();
  const char* p = b;
  for (; *p && *p != 'e'; ++p)
    if (*p >= '0' && *p <= '9') dig.push_back(*p);
  e = (x == 0.0) ? 0 : std::atoi(p + 1) + 1;
}

// Ew.d: [-]0.d1..dd followed by E+ee, or +eee without the E beyond two digits
std::string E(double x, int w, int d) {
  std::string dig;
  int e;
  digits(x, d, dig, e);
  std::string s = (std::signbit(x) && x != 0.0) ? "-" : "";
  s += "0." + dig;
  char b[16];
  if (std::abs(e) <= 99) std::snprintf(b, sizeof(b), "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
  else std::snprintf(b, sizeof(b), "%c%03d", e < 0 ? '-' : '+', std::abs(e));
  s += b;
  return fit_number(s, w);
}

// Gw.d for output (F2008 10.7.5.2.2): F(w-4).(d-k) and four blanks when the
// value rounded to d digits lies in [0.1, 10^d), k its decimal exponent;
// zero as F(w-4).(d-1) and four blanks; E editing otherwise.
std::string G(double x, int w, int d) {
  if (x == 0.0) return F(0.0, w - 4, d - 1) + "    ";
  std::string dig;
  int e;
  digits(x, d, dig, e);
  if (e >= 0 && e <= d) return F(x, w - 4, d - e) + "    ";
  return E(x, w, d);
}

}  // namespace fmt

namespace {

struct Out {
  FILE* f = nullptr;
  explicit Out(const std::string& path) { f = std::fopen(path.c_str(), "w"); }
  ~Out() { if (f) std::fclose(f); }
  void line(const std::string& s) { std::fputs(s.c_str(), f); std::fputc('\n', f); }
};

std::string join(const char* dir, const std::string& name) {
  std::string p = dir ? dir : ".";
  if (!p.empty() && p.back() != '/') p += '/';
  return p + name;
}

// representative_bin_info (engproc.F90:1355-1387), iduv 1-based
int bin_info(const ermod_store_info& s, int iduv, double& left, double& middle, double& invwt, int& spec) {
  int idmin = 0, cnt = 1;
  for (; cnt <= s.numslv; ++cnt) {
    const int idpt = idmin + s.uvmax[cnt - 1];
    if (iduv <= idpt) break;
    idmin = idpt;
  }
  if (cnt > s.numslv) return -1;
  spec = cnt;
  const int idsoft = s.uvsoft[cnt - 1], idmax = s.uvmax[cnt - 1], idpt = iduv - idmin;
  if (idpt < 1 || idpt > idmax) return -1;
  const double* c = s.uvcrd - 1;   // 1-based
  left = c[iduv];
  if (iduv == s.ermax && idpt <= idsoft) {
    // a linear last bin of the last species (pecore = 0) has no right edge in uvcrd
    middle = c[iduv];
    invwt = 0.0;
  } else if (idpt <= idsoft) {
    middle = (c[iduv] + c[iduv + 1]) / 2.0;
    invwt = 1.0 / (c[iduv + 1] - c[iduv]);
  } else if (idpt < idmax) {
    middle = std::sqrt(c[iduv] * c[iduv + 1]);
    invwt = 1.0 / (c[iduv + 1] - c[iduv]);
  } else {
    middle = c[iduv];
    invwt = 0.0;
  }
  return 0;
}

}  // namespace

extern "C" int32_t ermod_write_engstore(const char* dir, const ermod_store_info* info, const ermod_accum* norm,
                                        const double* avediv, const float* aveuv) {
  if (!info || !norm || !norm->edens || !info->uvcrd || !info->uvmax || !info->uvsoft)
    return io_fail(ERMOD_ERR_ARG, "sto_arg");
  const ermod_store_info& s = *info;
  const bool soln = s.slttype == ERMOD_SLT_SOLN;
  if (s.division < 1 || s.division > s.engdiv || s.engdiv > 99) return io_fail(ERMOD_ERR_ARG, "sto_div");
  if (s.corrcal && !norm->ecorr) return io_fail(ERMOD_ERR_ARG, "sto_arg");
  if (s.selfcal && (!norm->eself || !s.escrd)) return io_fail(ERMOD_ERR_ARG, "sto_arg");
  const bool last = s.division == s.engdiv;
  if (last && (!avediv || !norm->minuv || !norm->maxuv || (soln && !aveuv))) return io_fail(ERMOD_ERR_ARG, "sto_arg");

  if (last) {
    if (soln) {   // aveuv.tt: format(i5, 9999f15.5)
      Out o(join(dir, "aveuv.tt"));
      if (!o.f) return io_fail(ERMOD_ERR_IO, "sto_opn");
      for (int k = 1; k <= s.engdiv; ++k) {
        std::string l = fmt::I(k, 5);
        for (int q = 0; q < s.numslv; ++q) l += fmt::F(aveuv[(size_t)q * s.engdiv + (k - 1)], 15, 5);
        o.line(l);
      }
    }
    {             // weight_soln / weight_refs: (i5,e20.8) or (i5,e20.8,e20.7)
      Out o(join(dir, soln ? "weight_soln" : "weight_refs"));
      if (!o.f) return io_fail(ERMOD_ERR_IO, "sto_opn");
      for (int k = 1; k <= s.engdiv; ++k) {
        std::string l = fmt::I(k, 5) + fmt::E(avediv[k - 1], 20, 8);
        if (s.wgtslf) l += fmt::E(avediv[s.engdiv + k - 1], 20, 7);
        o.line(l);
      }
    }
    {             // uvrange.tt
      Out o(join(dir, "uvrange.tt"));
      if (!o.f) return io_fail(ERMOD_ERR_IO, "sto_opn");
      o.line(" species     minimum        maximum");
      for (int pti = 0; pti <= s.numslv; ++pti) {
        const float mn = norm->minuv[pti], mx = norm->maxuv[pti];
        if (mx < 1.0e5f) o.line(fmt::I(pti, 5) + fmt::F(mn, 15, 5) + fmt::F(mx, 15, 5));
        else o.line(fmt::I(pti, 5) + fmt::F(mn, 15, 5) + fmt::G(mx, 18, 5));
      }
    }
  }
  char suf[8];
  if (s.engdiv == 1) std::snprintf(suf, sizeof(suf), ".tt");
  else std::snprintf(suf, sizeof(suf), ".%02d", s.division);
  {               // engsln / engref: header, then (g15.7,g15.7,i5,g25.15,g25.15)
    Out o(join(dir, std::string(soln ? "engsln" : "engref") + suf));
    if (!o.f) return io_fail(ERMOD_ERR_IO, "sto_opn");
    o.line(fmt::A("# ", 2) + fmt::A("bin_left", 13) + fmt::A("bin_middle", 15) + fmt::A("spec", 5) +
           fmt::A("ratio", 25) + fmt::A("dens", 25));
    for (int iduv = 1; iduv <= s.ermax; ++iduv) {
      double left, middle, invwt;
      int spec;
      if (bin_info(s, iduv, left, middle, invwt, spec) != 0) return io_fail(ERMOD_ERR_ENG_ECD, "eng_ecd");
      const double e = norm->edens[iduv - 1];
      o.line(fmt::G(left, 15, 7) + fmt::G(middle, 15, 7) + fmt::I(spec, 5) + fmt::G(e, 25, 15) +
             fmt::G(e * invwt, 25, 15));
    }
  }
  if (s.corrcal) {  // corsln / corref: one unformatted record of ermax^2 FP64
    const uint64_t bytes = (uint64_t)s.ermax * (uint64_t)s.ermax * 8u;
    // gfortran splits records above 2^31 - 9 bytes into sub-records; ermax <= 16383 stays below
    if (bytes > 2147483639ull) return io_fail(ERMOD_ERR_ARG, "sto_cor");
    FILE* f = std::fopen(join(dir, std::string(soln ? "corsln" : "corref") + suf).c_str(), "wb");
    if (!f) return io_fail(ERMOD_ERR_IO, "sto_opn");
    const int32_t m = (int32_t)bytes;
    bool ok = std::fwrite(&m, 4, 1, f) == 1;
    ok = ok && std::fwrite(norm->ecorr, 8, (size_t)s.ermax * s.ermax, f) == (size_t)s.ermax * s.ermax;
    ok = ok && std::fwrite(&m, 4, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return io_fail(ERMOD_ERR_IO, "sto_wrt");
  }
  if (s.selfcal) {  // slfeng: (g15.7,g25.15) of the FP32 representative energy and eself
    Out o(join(dir, std::string("slfeng") + suf));
    if (!o.f) return io_fail(ERMOD_ERR_IO, "sto_opn");
    for (int iduv = 1; iduv <= s.esmax; ++iduv) {
      // representative_bin_selfenergy (engproc.F90:1344-1353) returns a default real
      const float c = iduv < s.esmax ? (float)((s.escrd[iduv - 1] + s.escrd[iduv]) / 2.0) : (float)s.escrd[s.esmax - 1];
      o.line(fmt::G(c, 15, 7) + fmt::G(norm->eself[iduv - 1], 25, 15));
    }
  }
  return ERMOD_OK;
}

// rmsd_bestfit (bestfit.F90:339-346): fit `crd` onto `ref` with weights w, then the weighted RMSD.
extern "C" double ermod_rmsd_bestfit(int32_t n, const float* ref, const float* crd, const float* w) {
  if (n <= 0 || !ref || !crd || !w) return -1.0;
  return erm::fit::rmsd_bestfit(n, ref, crd, w);   // -1: halt_with_error('bst_zrw') in the reference
}

extern "C" const char* ermod_io_last_error(void) { return g_err; }

extern "C" int32_t ermod_io_format(int32_t kind, double x, int32_t w, int32_t d, char* out, int32_t cap) {
  std::string s;
  switch (kind) {
    case 0: s = fmt::G(x, w, d); break;
    case 1: s = fmt::E(x, w, d); break;
    case 2: s = fmt::F(x, w, d); break;
    case 3: s = fmt::I((long)x, w); break;
    default: return ERMOD_ERR_ARG;
  }
  if ((int)s.size() + 1 > cap) return ERMOD_ERR_ARG;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return ERMOD_OK;
}
