// engine.cu -- C-ABI of the engine: context setup and the per-frame pipeline.
//
// One ermod_engconst call runs, on one CUDA stream:
//   H2D coordinates -> solvent normalisation + splines -> cell list ->
//   insertion placement -> per chunk of `chunk` targets:
//     [PME] zero + spread -> cuFFT R2C -> influence multiply / self energy ->
//           cuFFT C2R into a target-fastest potential grid
//     real space (cell list) -> gather + residual + binning (integer atomics)
//   per batch of targets: weights -> edens -> ecorr
// and reads one status word back.  See kernels.cu for the kernel map to the
// reference routines.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"

using namespace erm;

#define CK(x)                                                   \
  do {                                                          \
    cudaError_t e_ = (x);                                       \
    if (e_ != cudaSuccess) {                                    \
      ctx->err = std::string("cuda: ") + cudaGetErrorString(e_); \
      return ERMOD_ERR_CUDA;                                    \
    }                                                           \
  } while (0)

#define CF(x)                                              \
  do {                                                     \
    cufftResult r_ = (x);                                  \
    if (r_ != CUFFT_SUCCESS) {                             \
      ctx->err = "cufft error " + std::to_string((int)r_); \
      return ERMOD_ERR_CUDA;                               \
    }                                                      \
  } while (0)

// Engine extensions declared in ecorr_tc.cu
namespace erm {
int ecorr_tc_available();
int launch_ecorr_tc(const DeviceState& d, int base, int n, int ermax, int ermax_pad, int count_base,
                    int weight_bits, void* work, size_t work_bytes, cudaStream_t s);
size_t ecorr_tc_workspace(int n, int ermax);
}  // namespace erm

struct ermod_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;            // real space, beside the PME chain of st
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev[9] = {};
  ermod_params p{};
  // host topology
  int nummol = 0, numatm = 0, natoms = 0, slvmax = 0, numslt = 0, s = 0, maxdst = 0;
  int numslv = 0, ermax = 0, esmax = 0, ermax_pad = 0;
  int ljtype_max = 0;
  std::vector<int> numsite, sluvid, uvspec, tagpt, sltlist, molbeg_all, tgt_k;
  std::vector<float> charge, mass;
  double qslt_refs = 0.0;
  std::vector<double> uvcrd, escrd;
  std::vector<int> uvmax, uvsoft;
  DeviceState d;
  int chunk = kChunk, batch = 0, ncell_cap = 0;
  float cell_h = 0.f;                    // cell-list edge picked by the tuner (0: not yet tuned, 4 A)
  int nhost = 0;                      // atoms of the host aggregate (insposition 2..4)
  int nref = 0;                       // atoms of the RefInfo host (insposition 5, 6)
  bool gauss_init = false;            // Gaussian insertion constants fixed at the first frame
  float gauss_l[3] = {0.f, 0.f, 0.f}, gauss_z0 = 0.f, gauss_z1 = 0.f;
  PppmGreen pppm{};                   // PPPM influence function inputs (cltype 3)
  cufftHandle r2c = 0, c2r = 0;
  bool plans = false;
  void* tc_work = nullptr;
  size_t tc_work_bytes = 0;
  // reference state carried between frames
  float invcell_prev[3] = {0.f, 0.f, 0.f};
  float prevcl[9] = {0};
  bool pme_init = false, usreal_init = false, warn_bin_firsttime = true;
  float* h_pin = nullptr;
  size_t h_pin_bytes = 0;
  std::string err;
  // stage timing: events recorded on the stream between stages, read once per frame
  std::vector<cudaEvent_t> pev;
  std::vector<int> ptag;
  int pused = 0;
  float timings[17] = {0};
  long long launches = 0;
  int use_tc = 1;
  int spath = 1;     // PME solve: 1 spread + cuFFT, 2 fused with direct site sums, 3 fused with plane spreading
  int real_threads = 0;           // block size of k_real chosen by the autotuner (0: not tuned yet)
  // the frame as a CUDA graph, re-captured when the frame plan changes
  cudaGraphExec_t gexec = nullptr;
  std::vector<unsigned char> gkey;
  long long graph_launches = 0;
  int* h_frame = nullptr;         // pinned: [0] stnum of the frame being staged
  DevStatus* h_status = nullptr;  // pinned: status word written by the frame
  // insertion proposal: voxels per side (0: off), uniform mixture weight, network loaded
  int prop_gv = 0, prop_gf = 0;
  float prop_eps = 0.1f;
  bool prop_params = false;
};

// With spectrum_path == 0 the fused solve builds the solute spectrum by direct
// site sums up to this many sites and by plane spreading + forward FFT above:
// the sums cost s * K2 * K3 per plane, the FFT a fixed ~K2 * K3 * log(K2 K3).
constexpr int kDirectAutoSites = 16, kDirectAutoSitesTc64 = 32, kDirectAutoSitesTc128 = 64;

enum Stage { kStPrep = 1, kStIns = 2, kStReal = 3, kStSpread = 4, kStR2C = 5, kStInfl = 6, kStC2R = 7,
             kStGather = 8, kStBin = 9, kStWeights = 10, kStEcorr = 11, kStChunks = 12, kStTranspose = 13,
             kStPlane = 14, kStRows = 15, kStSiteTab = 16, kNumTimings = 17 };

namespace {

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  return cudaMalloc((void**)p, n * sizeof(T));
}

template <class T>
cudaError_t h2d(T* dst, const T* src, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  return cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

void free_all(ermod_ctx* c) {
  DeviceState& d = c->d;
  void* ptrs[] = {d.molbeg, d.molspec, d.molq, d.atom_lj, d.atom_q, d.ljene, d.ljlensq, d.slt_lj, d.slt_q,
                  d.slt_mass, d.bfcoord, d.uvcrd, d.spec_off, d.uvsoft, d.escrd, d.posraw, d.slvn, d.spl, d.grd,
                  d.grec, d.mrec, d.anchor, d.cellof, d.cellcount, d.cellstart, d.molsorted, d.rmol, d.ins_conf, d.insw_in,
                  d.tgt_raw, d.tgt_n, d.tgt_c, d.tgt_mol, d.selfreal, d.selfrec, d.u0, d.w, d.etot, d.flceng,
                  d.grid, d.spec, d.phin, d.phi, d.engfac, d.engfacT, d.fft_tw, d.fft_twd, d.sitetab, d.sitestn,
                  d.splfc,
                  d.E, d.Etot, d.tgtq, d.twt, d.sbin, d.gacc,
                  d.boxinfo, d.partial, d.done, d.uvengy, d.counts, d.edens, d.edens_part, d.ecorr, d.eself,
                  d.slnuv, d.minuv, d.maxuv, d.scal, d.status, d.frame_i, d.dens, d.feat, d.mlp_f, d.mlp_b,
                  d.vact, d.vlogit, d.vcdf, d.vq, d.ins_voxel, d.ins_feat, d.host_atom, d.host_mass, d.aggcen,
                  d.atom_mass, d.skip, d.ref_atom, d.ref_host, d.ref_host_w, d.ref_slt, d.ref_slt_w, d.ref_bf,
                  c->tc_work};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->plans) {
    cufftDestroy(c->r2c);
    cufftDestroy(c->c2r);
  }
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->pev)
    if (e) cudaEventDestroy(e);
  if (c->h_pin) cudaFreeHost(c->h_pin);
  if (c->h_frame) cudaFreeHost(c->h_frame);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->st) cudaStreamDestroy(c->st);
}

// spline.F90:25-44
double spline_value_d(int order, double x) {
  double c[kMaxOrder + 1];
  for (int i = 0; i <= order; ++i) {
    double f = 1.0;
    for (int k = 1; k <= i; ++k) f *= k;
    for (int k = 1; k <= order - i; ++k) f *= k;
    f = order / f;
    if (i % 2 == 1) f = -f;
    c[i] = f;
  }
  double r = 0.0;
  if (x > 0.0 && x < order) {
    const int k = (int)x;
    for (int i = 0; i <= k; ++i) r += c[i] * std::pow(x - i, order - 1);
  }
  return r;
}

// init_spline_axis (recpcal.F90:97-119) in FP64
void spline_axis(int K, int order, double* out) {
  for (int rci = 0; rci < K; ++rci) {
    double re = 0.0, im = 0.0;
    for (int spi = 0; spi <= order - 2; ++spi) {
      const double chr = spline_value_d(order, spi + 1.0);
      const double a = 2.0 * kPi * (double)(spi * rci) / (double)K;
      re += chr * std::cos(a);
      im += chr * std::sin(a);
    }
    out[rci] = re * re + im * im;
  }
}

int set_error(ermod_ctx* c, int code, const char* name) {
  c->err = name;
  return code;
}

// record a stage boundary: the time since the previous mark belongs to `tag`
void mark(ermod_ctx* c, int tag) {
  if (c->pused == (int)c->pev.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->pev.push_back(e);
    c->ptag.push_back(0);
  }
  cudaEventRecord(c->pev[c->pused], c->st);
  c->ptag[c->pused] = tag;
  ++c->pused;
}

}  // namespace

extern "C" {

int32_t ermod_abi_version(void) { return ERMOD_ABI_VERSION; }

// enginit mesh (engproc.F90:171-226, 264-281) for one &hist set shared by all species
int32_t ermod_enginit_mesh(const ermod_hist* h, int32_t numslv, double* uvcrd, int32_t* uvmax, int32_t* uvsoft,
                           double* escrd, int32_t* ermax, int32_t* esmax) {
  if (!h || numslv <= 0) return ERMOD_ERR_ARG;
  const int rglmax = 5;
  double ecdmin = h->ecdmin, ecfmns = h->ecfmns, ecdcen = h->ecdcen, eccore = h->eccore, ecdmax = h->ecdmax;
  const double eclbin = h->eclbin, ecfbin = h->ecfbin, ec0bin = h->ec0bin, finfac = h->finfac;
  const int pecore = h->pecore;
  if (pecore == 1) return ERMOD_ERR_ENG_ECD;
  const double ectmvl = finfac * ecfbin;
  ecdmin -= ectmvl;
  ecfmns -= ectmvl;
  const double ecmns0 = ecdcen - ectmvl, ecpls0 = 2.0 * ecdcen - ecmns0, ecfpls = 2.0 * ecdcen - ecfmns;
  eccore = eccore + ecfpls - ecdcen;
  const double v[7] = {ecdmin, ecfmns, ecmns0, ecpls0, ecfpls, eccore, ecdmax};
  int up[7];
  up[0] = 1;
  for (int r = 1; r <= rglmax; ++r) {
    const double f = (r == 1 || r == 5) ? eclbin : (r == 2 || r == 4) ? ecfbin : ec0bin;
    const double inc = v[r] - v[r - 1];
    if (inc < f) return ERMOD_ERR_ENG_ECD;
    up[r] = up[r - 1] + (int)std::lround(inc / f);
  }
  const int pesoft = up[rglmax] - up[0], pemax = pesoft + pecore;
  up[rglmax + 1] = pemax;
  std::vector<double> e(std::max(pemax, up[rglmax]) + 2, 0.0);
  for (int r = 0; r <= rglmax + 1; ++r) e[up[r]] = v[r];
  const int last = pecore == 0 ? rglmax : rglmax + 1;
  for (int r = 1; r <= last; ++r) {
    const int lo = up[r - 1], hi = up[r];
    const double inc = r <= rglmax ? e[hi] - e[lo] : std::log(e[hi] / e[lo]);
    const double f = inc / (double)(hi - lo);
    for (int i = lo; i < hi; ++i) e[i] = r <= rglmax ? e[lo] + f * (i - lo) : e[lo] * std::exp(f * (i - lo));
  }
  if (ermax) *ermax = numslv * pemax;
  if (esmax) *esmax = pesoft;
  for (int q = 0; q < numslv; ++q) {
    if (uvmax) uvmax[q] = pemax;
    if (uvsoft) uvsoft[q] = pesoft;
    if (uvcrd) for (int i = 0; i < pemax; ++i) uvcrd[(size_t)q * pemax + i] = e[i + 1];
  }
  if (escrd) for (int i = 0; i < pesoft; ++i) escrd[i] = e[i + 1];
  return ERMOD_OK;
}

int32_t ermod_create(ermod_ctx** out, int32_t device, const ermod_params* prm, const ermod_topology* t,
                     const ermod_mesh* m) {
  if (!out || !prm || !t || !m) return ERMOD_ERR_ARG;
  *out = nullptr;
  ermod_ctx* ctx = new ermod_ctx();
  ctx->device = device;
  ctx->p = *prm;
  const ermod_params& p = ctx->p;
  auto bad = [&](int code, const char* name) {
    ctx->err = name;
    *out = ctx;
    return code;
  };
  const bool mesh = p.cltype == ERMOD_EL_PME || p.cltype == ERMOD_EL_PPPM;
  if (!mesh && p.cltype != ERMOD_EL_COULOMB) return bad(ERMOD_ERR_UNSUPPORTED, "set_prs");
  if (mesh && (p.splodr < 2 || p.splodr > kMaxOrder)) return bad(ERMOD_ERR_ARG, "set_ewa");
  // recpcal.F90:250-251: the PPPM denominator needs an even order
  if (p.cltype == ERMOD_EL_PPPM && p.splodr % 2 != 0) return bad(ERMOD_ERR_ARG, "pppm_odr");
  if (mesh &&
      (p.ms1max < p.splodr || p.ms2max < p.splodr || p.ms3max < p.splodr || p.ms1max > kMaxGrid ||
       p.ms2max > kMaxGrid || p.ms3max > kMaxGrid))
    return bad(ERMOD_ERR_ARG, "set_ewa");
  if (p.boxshp == ERMOD_SYS_NONPERIODIC && (p.estype == ERMOD_ES_NPT || p.cltype != ERMOD_EL_COULOMB))
    return bad(ERMOD_ERR_ARG, "set_prs");
  if (p.slttype < 1 || p.slttype > 3) return bad(ERMOD_ERR_ARG, "set_slt");
  if (p.slttype != ERMOD_SLT_SOLN &&
      !((p.insposition >= ERMOD_INSPOS_RANDOM && p.insposition <= ERMOD_INSPOS_GAUSS) &&
        (p.insorient == ERMOD_INSROT_RANDOM || p.insorient == ERMOD_INSROT_NOCHANGE)))
    return bad(ERMOD_ERR_UNSUPPORTED, "ins_geo");
  // sphere / slab regions around the host aggregate and RMSD / Gaussian insertion against the
  // RefInfo structure: refs insertion (set_shift_com) and soln configuration checks
  // (check_mol_configuration)
  if (p.slttype == ERMOD_SLT_SOLN && (p.insposition < ERMOD_INSPOS_RANDOM || p.insposition > ERMOD_INSPOS_GAUSS))
    return bad(ERMOD_ERR_UNSUPPORTED, "ins_geo");
  const bool region = p.insposition >= ERMOD_INSPOS_SPHERE && p.insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC;
  if (region && !(p.lwreg >= 0.f && p.upreg >= p.lwreg && p.upreg > 0.f && p.hostspec != 0))
    return bad(ERMOD_ERR_ARG, "ins_reg");
  if (p.insposition >= ERMOD_INSPOS_RMSD && !(p.lwreg >= 0.f && p.upreg >= p.lwreg && p.upreg > 0.f))
    return bad(ERMOD_ERR_ARG, "ins_reg");
  if (p.insstructure != ERMOD_INSSTR_NOREJECT && p.insstructure != ERMOD_INSSTR_RMSD)
    return bad(ERMOD_ERR_ARG, "ins_str");   // "Unknown insstructure" (engproc.F90:1293-1294)
  // topology (setparam / enginit / engconst bookkeeping)
  ctx->nummol = t->nummol;
  ctx->numsite.assign(t->numsite, t->numsite + t->nummol);
  ctx->sluvid.assign(t->sluvid, t->sluvid + t->nummol);
  ctx->uvspec.assign(t->uvspec, t->uvspec + t->nummol);
  ctx->molbeg_all.resize(ctx->nummol + 1, 0);
  for (int i = 0; i < ctx->nummol; ++i) ctx->molbeg_all[i + 1] = ctx->molbeg_all[i] + ctx->numsite[i];
  ctx->numatm = ctx->molbeg_all[ctx->nummol];
  ctx->charge.assign(t->charge, t->charge + ctx->numatm);
  ctx->mass.assign(t->sitemass, t->sitemass + ctx->numatm);
  for (int i = 0; i < ctx->nummol; ++i) {
    if (ctx->sluvid[i] < 0 || ctx->sluvid[i] > 3) return bad(ERMOD_ERR_ARG, "eng_bug");
    if (ctx->sluvid[i] == ERMOD_PT_SOLVENT || ctx->sluvid[i] == ERMOD_PT_SOLUTE) ctx->tagpt.push_back(i);
    if (ctx->sluvid[i] > 0) ctx->sltlist.push_back(i);
  }
  ctx->slvmax = (int)ctx->tagpt.size();
  ctx->numslt = (int)ctx->sltlist.size();
  if (ctx->numslt <= 0 || ctx->slvmax <= 0) return bad(ERMOD_ERR_ARG, "eng_num");
  const bool refs = p.slttype != ERMOD_SLT_SOLN;
  if (refs) {
    if (ctx->numslt != 1 || ctx->sltlist[0] != ctx->nummol - 1) return bad(ERMOD_ERR_ARG, "eng_ins");
    for (int i = 0; i < ctx->nummol; ++i) if (ctx->sluvid[i] == ERMOD_PT_SOLUTE) return bad(ERMOD_ERR_ARG, "eng_par");
    ctx->maxdst = p.maxins;
    if (ctx->maxdst < 1) return bad(ERMOD_ERR_ARG, "set_ins");
  } else {
    for (int i = 0; i < ctx->nummol; ++i) if (ctx->sluvid[i] >= 2) return bad(ERMOD_ERR_ARG, "eng_par");
    ctx->maxdst = ctx->numslt;
  }
  ctx->s = ctx->numsite[ctx->sltlist[0]];
  for (int i : ctx->sltlist) if (ctx->numsite[i] != ctx->s) return bad(ERMOD_ERR_ARG, "set_slt");
  if (ctx->s > kMaxSoluteSites) return bad(ERMOD_ERR_OVERFLOW, "ins_siz");
  ctx->ljtype_max = t->ljtype_max;
  ctx->numslv = m->numslv;
  ctx->ermax = m->ermax;
  ctx->esmax = m->esmax;
  ctx->uvcrd.assign(m->uvcrd, m->uvcrd + m->ermax);
  ctx->uvmax.assign(m->uvmax, m->uvmax + m->numslv);
  ctx->uvsoft.assign(m->uvsoft, m->uvsoft + m->numslv);
  if (p.selfcal && (!m->escrd || m->esmax <= 0)) return bad(ERMOD_ERR_ARG, "eng_ecd");
  if (m->escrd && m->esmax > 0) ctx->escrd.assign(m->escrd, m->escrd + m->esmax);
  for (int i : ctx->tagpt)
    if (ctx->uvspec[i] < 0 || ctx->uvspec[i] > ctx->numslv) return bad(ERMOD_ERR_ARG, "eng_bug");
  ctx->ermax_pad = (ctx->ermax + 127) / 128 * 128;
  {
    int sum = 0;
    for (int q = 0; q < ctx->numslv; ++q) sum += ctx->uvmax[q];
    if (sum != ctx->ermax) return bad(ERMOD_ERR_ARG, "eng_bug");
  }
  // tagpt-order physical atoms
  std::vector<int> molbeg(ctx->slvmax + 1, 0), molspec(ctx->slvmax), atom_lj, tagk(ctx->nummol, -1);
  std::vector<float> molq(ctx->slvmax), atom_q;
  for (int k = 0; k < ctx->slvmax; ++k) {
    const int i = ctx->tagpt[k];
    tagk[i] = k;
    molbeg[k + 1] = molbeg[k] + ctx->numsite[i];
    molspec[k] = ctx->uvspec[i];
    float q = 0.0f;
    for (int a = ctx->molbeg_all[i]; a < ctx->molbeg_all[i + 1]; ++a) {
      q += ctx->charge[a];
      atom_q.push_back(ctx->charge[a]);
      atom_lj.push_back(t->ljtype[a] - 1);
    }
    molq[k] = q;
  }
  ctx->natoms = molbeg[ctx->slvmax];
  // atoms of the host aggregate (com_aggregate, insertion.F90:587-614): molecules of the hostspec species
  std::vector<int> host_atom;
  std::vector<float> host_mass;
  if (region) {
    for (int k = 0; k < ctx->slvmax; ++k) {
      const int i = ctx->tagpt[k], sp = ctx->uvspec[i];
      if (sp < 1 || sp > 31 || !((p.hostspec >> (sp - 1)) & 1)) continue;
      for (int j = 0; j < ctx->numsite[i]; ++j) {
        host_atom.push_back(molbeg[k] + j);
        host_mass.push_back(ctx->mass[ctx->molbeg_all[i] + j]);
      }
    }
    if (host_atom.empty()) return bad(ERMOD_ERR_ARG, "ins_reg");
  }
  ctx->nhost = (int)host_atom.size();
  const int slt = ctx->sltlist[0];
  std::vector<int> slt_lj(ctx->s);
  std::vector<float> slt_q(ctx->s), slt_m(ctx->s);
  float qs = 0.0f;
  for (int a = 0; a < ctx->s; ++a) {
    slt_lj[a] = t->ljtype[ctx->molbeg_all[slt] + a] - 1;
    slt_q[a] = ctx->charge[ctx->molbeg_all[slt] + a];
    slt_m[a] = ctx->mass[ctx->molbeg_all[slt] + a];
    qs += slt_q[a];
  }
  ctx->qslt_refs = qs;
  if (!refs) for (int c = 0; c < ctx->maxdst; ++c) ctx->tgt_k.push_back(tagk[ctx->sltlist[c]]);
  for (int a : atom_lj) if (a < 0 || a >= ctx->ljtype_max) return bad(ERMOD_ERR_ARG, "set_ljt");
  for (int a : slt_lj) if (a < 0 || a >= ctx->ljtype_max) return bad(ERMOD_ERR_ARG, "set_ljt");
  // engine shape
  if (p.ins_chunk != 0 && p.ins_chunk != kChunk) return bad(ERMOD_ERR_ARG, "ins_chk");
  ctx->chunk = kChunk;
  const int K1 = p.ms1max, K2 = p.ms2max, K3 = p.ms3max, Kh1 = K1 / 2 + 1;
  const bool pme = mesh;   // smooth PME and PPPM share the whole pipeline but the influence function
  ctx->batch = p.ecorr_batch > 0 ? p.ecorr_batch : 4096;
  ctx->batch = std::max(ctx->chunk, (ctx->batch + ctx->chunk - 1) / ctx->chunk * ctx->chunk);
  ctx->batch = std::min(ctx->batch, (ctx->maxdst + ctx->chunk - 1) / ctx->chunk * ctx->chunk);
  ctx->ncell_cap = 64 * 64 * 64;
  *out = ctx;

  CK(cudaSetDevice(device));
  {
    // the PME chain on st comes first; real space on st2 fills the SMs it leaves
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&ctx->st, cudaStreamNonBlocking, hi));
    CK(cudaStreamCreateWithPriority(&ctx->st2, cudaStreamNonBlocking, lo));
  }
  CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  for (auto& e : ctx->ev) CK(cudaEventCreate(&e));
  DeviceState& d = ctx->d;
  const size_t NA = ctx->natoms, SM = ctx->slvmax, MD = ctx->maxdst, S = ctx->s;
  const int order = pme ? p.splodr : 1;
  CK(dalloc(&d.molbeg, SM + 1)); CK(dalloc(&d.molspec, SM)); CK(dalloc(&d.molq, SM));
  CK(dalloc(&d.atom_lj, NA)); CK(dalloc(&d.atom_q, NA));
  CK(dalloc(&d.ljene, (size_t)ctx->ljtype_max * ctx->ljtype_max));
  CK(dalloc(&d.ljlensq, (size_t)ctx->ljtype_max * ctx->ljtype_max));
  CK(dalloc(&d.slt_lj, S)); CK(dalloc(&d.slt_q, S)); CK(dalloc(&d.slt_mass, S)); CK(dalloc(&d.bfcoord, 3 * S));
  CK(dalloc(&d.uvcrd, ctx->ermax)); CK(dalloc(&d.spec_off, ctx->numslv + 1)); CK(dalloc(&d.uvsoft, ctx->numslv));
  CK(dalloc(&d.escrd, std::max(1, ctx->esmax)));
  CK(dalloc(&d.posraw, 3 * NA)); CK(dalloc(&d.slvn, NA)); CK(dalloc(&d.spl, NA * 3 * order)); CK(dalloc(&d.grd, NA));
  if (pme && gather_rec_ok(order, K1, K2, K3)) { CK(dalloc(&d.grec, NA * kRecWords)); CK(dalloc(&d.mrec, SM)); }
  CK(dalloc(&d.anchor, SM)); CK(dalloc(&d.cellof, SM)); CK(dalloc(&d.cellcount, ctx->ncell_cap));
  CK(dalloc(&d.cellstart, ctx->ncell_cap + 1)); CK(dalloc(&d.molsorted, SM)); CK(dalloc(&d.rmol, 1));
  CK(dalloc(&d.ins_conf, 3 * S * MD)); CK(dalloc(&d.insw_in, MD));
  CK(dalloc(&d.tgt_raw, MD * S)); CK(dalloc(&d.tgt_n, MD * S)); CK(dalloc(&d.tgt_c, MD)); CK(dalloc(&d.tgt_mol, MD));
  CK(dalloc(&d.selfreal, MD)); CK(dalloc(&d.selfrec, MD)); CK(dalloc(&d.u0, MD)); CK(dalloc(&d.w, MD));
  CK(dalloc(&d.etot, MD)); CK(dalloc(&d.flceng, MD * ctx->numslv));
  const size_t KK = (size_t)K1 * K2 * K3, KH = (size_t)K3 * K2 * Kh1;
  // PME solve path (spectrum_path): the fused solve where the mesh allows it
  FrameArgs fa{};
  fa.pme = pme; fa.K1 = K1; fa.K2 = K2; fa.K3 = K3; fa.Kh1 = Kh1; fa.nsite = ctx->s; fa.order = order;
  fa.ljtype_max = ctx->ljtype_max;
  if (setup_real_smem(fa) != 0) return bad(ERMOD_ERR_CUDA, "real_smem");
  if (setup_insert_smem(ctx->s) != 0) return bad(ERMOD_ERR_CUDA, "ins_smem");
  const bool fused_ok = pme && fused_supported(fa);
  if (p.spectrum_path < 0 || p.spectrum_path > 3) return bad(ERMOD_ERR_ARG, "spc_path");
  if (pme && p.spectrum_path >= 2 && !fused_ok) return bad(ERMOD_ERR_UNSUPPORTED, "spc_path");
  // direct site sums up to 16 sites; on square 64 and 128 planes they run on the tensor cores
  // and beat plane spreading up to about 32 sites (64 x 64: ring-recipe solutes in 4096 waters)
  // and past 60 (128 x 128: the 60-site chain in 32,768 waters, 92.9 against 109.6 ms a frame)
  const int direct_auto = (K2 == 64 && K3 == 64) ? kDirectAutoSitesTc64
                          : (K2 == 128 && K3 == 128) ? kDirectAutoSitesTc128 : kDirectAutoSites;
  if (p.spectrum_path == 0) ctx->spath = fused_ok ? (ctx->s <= direct_auto ? 2 : 3) : 1;
  else ctx->spath = p.spectrum_path;
  if (pme) {
    CK(dalloc(&d.spec, (size_t)ctx->chunk * KH));
    CK(dalloc(&d.phi, (size_t)ctx->chunk * K3 * K2 * 2 * ((K1 + 1) / 2)));   // n1 pairs, see DeviceState::phi
    CK(dalloc(&d.engfac, KH)); CK(dalloc(&d.splfc, K1 + K2 + K3));
    if (ctx->spath == 1) {
      CK(dalloc(&d.grid, (size_t)ctx->chunk * KK));
      CK(cudaMemsetAsync(d.grid, 0, sizeof(float) * ctx->chunk * KK, ctx->st));  // kept zero outside the boxes
      CK(dalloc(&d.phin, (size_t)ctx->chunk * KK));
    } else {
      CK(dalloc(&d.engfacT, KH));
      std::vector<float2> tw;
      std::vector<double2> twd;
      fused_twiddles(K1, K2, K3, tw, twd);
      CK(dalloc(&d.fft_tw, tw.size()));
      CK(dalloc(&d.fft_twd, twd.size()));
      CK(dalloc(&d.sitetab, fused_sitetab_elems(fa, ctx->batch, ctx->spath == 2)));
      if (ctx->spath == 3) CK(dalloc(&d.sitestn, fused_sitestn_elems(fa, ctx->batch)));
      CK(cudaMemcpyAsync(d.fft_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice, ctx->st));
      CK(cudaMemcpyAsync(d.fft_twd, twd.data(), sizeof(double2) * twd.size(), cudaMemcpyHostToDevice, ctx->st));
      CK(cudaStreamSynchronize(ctx->st));
      if (setup_fused(fa) != 0) return bad(ERMOD_ERR_CUDA, "pme_smem");
    }
  }
  CK(dalloc(&d.E, SM * ctx->batch));
  CK(dalloc(&d.Etot, SM * ctx->batch));
  CK(dalloc(&d.tgtq, MD));
  CK(dalloc(&d.twt, MD));
  CK(dalloc(&d.sbin, MD));
  if (pme) {
    if (ctx->spath == 1) CK(dalloc(&d.gacc, (size_t)ctx->chunk * KK));
    CK(dalloc(&d.boxinfo, 2 * (size_t)ctx->chunk));
    CK(dalloc(&d.partial, (size_t)ctx->chunk * std::max(kInflBlocks, Kh1)));
    CK(dalloc(&d.done, (size_t)ctx->chunk));
    CK(cudaMemsetAsync(d.done, 0, sizeof(unsigned int) * ctx->chunk, ctx->st));
    if (setup_spread_smem() != 0) return bad(ERMOD_ERR_CUDA, "spr_smem");
  }
  if (p.keep_uvengy) CK(dalloc(&d.uvengy, MD * SM));
  CK(dalloc(&d.counts, (size_t)ctx->batch * ctx->ermax_pad));
  CK(dalloc(&d.edens, ctx->ermax));
  CK(dalloc(&d.edens_part, (size_t)kEdensSlices * ctx->ermax));
  if (p.corrcal) CK(dalloc(&d.ecorr, (size_t)ctx->ermax * ctx->ermax));
  CK(dalloc(&d.eself, std::max(1, ctx->esmax))); CK(dalloc(&d.slnuv, ctx->numslv));
  CK(dalloc(&d.minuv, ctx->numslv + 1)); CK(dalloc(&d.maxuv, ctx->numslv + 1));
  CK(dalloc(&d.scal, 8)); CK(dalloc(&d.status, 1)); CK(dalloc(&d.frame_i, 4));
  CK(cudaMallocHost((void**)&ctx->h_frame, 4 * sizeof(int)));
  CK(cudaMallocHost((void**)&ctx->h_status, sizeof(DevStatus)));
  if (p.graph_mode < 0 || p.graph_mode > 1 || p.stage_timing < 0 || p.stage_timing > 1) return bad(ERMOD_ERR_ARG, "opt_arg");
  // static uploads
  cudaStream_t st = ctx->st;
  CK(h2d(d.molbeg, molbeg.data(), SM + 1, st)); CK(h2d(d.molspec, molspec.data(), SM, st));
  CK(h2d(d.molq, molq.data(), SM, st)); CK(h2d(d.atom_lj, atom_lj.data(), NA, st));
  CK(h2d(d.atom_q, atom_q.data(), NA, st));
  CK(h2d(d.ljene, t->ljene_mat, (size_t)ctx->ljtype_max * ctx->ljtype_max, st));
  CK(h2d(d.ljlensq, t->ljlensq_mat, (size_t)ctx->ljtype_max * ctx->ljtype_max, st));
  CK(h2d(d.slt_lj, slt_lj.data(), S, st)); CK(h2d(d.slt_q, slt_q.data(), S, st));
  CK(h2d(d.slt_mass, slt_m.data(), S, st));
  if (ctx->nhost > 0) {
    CK(dalloc(&d.host_atom, ctx->nhost)); CK(dalloc(&d.host_mass, ctx->nhost)); CK(dalloc(&d.aggcen, 3));
    CK(h2d(d.host_atom, host_atom.data(), ctx->nhost, st));
    CK(h2d(d.host_mass, host_mass.data(), ctx->nhost, st));
    if (!refs) {   // solute centres of mass for check_mol_configuration, and its verdicts
      std::vector<float> am;
      am.reserve(NA);
      for (int k = 0; k < ctx->slvmax; ++k) {
        const int i = ctx->tagpt[k];
        for (int j = 0; j < ctx->numsite[i]; ++j) am.push_back(ctx->mass[ctx->molbeg_all[i] + j]);
      }
      CK(dalloc(&d.atom_mass, NA));
      CK(h2d(d.atom_mass, am.data(), NA, st));
    }
  }
  // soln: the verdicts of check_mol_configuration (sphere / slab around the aggregate, RMSD to RefInfo)
  if (!refs && (ctx->nhost > 0 || p.insposition == ERMOD_INSPOS_RMSD || p.insstructure == ERMOD_INSSTR_RMSD))
    CK(dalloc(&d.skip, MD));
  std::vector<float> bf(3 * S, 0.0f);
  if (t->bfcoord) std::memcpy(bf.data(), t->bfcoord, sizeof(float) * 3 * S);
  CK(h2d(d.bfcoord, bf.data(), 3 * S, st));
  CK(h2d(d.uvcrd, ctx->uvcrd.data(), ctx->ermax, st));
  std::vector<int> off(ctx->numslv + 1, 0);
  for (int q = 0; q < ctx->numslv; ++q) off[q + 1] = off[q] + ctx->uvmax[q];
  CK(h2d(d.spec_off, off.data(), ctx->numslv + 1, st));
  CK(h2d(d.uvsoft, ctx->uvsoft.data(), ctx->numslv, st));
  if (!ctx->escrd.empty()) CK(h2d(d.escrd, ctx->escrd.data(), ctx->esmax, st));
  std::vector<int> tm(MD, -1);
  if (!refs) for (size_t c = 0; c < MD; ++c) tm[c] = ctx->tgt_k[c];
  CK(h2d(d.tgt_mol, tm.data(), MD, st));
  {  // net solute charge of every target (mol_charge(tagslt), engproc.F90:994, 1014)
    std::vector<double> q(MD, (double)qs);
    if (!refs)
      for (size_t c = 0; c < MD; ++c) {
        float s = 0.f;
        const int i = ctx->sltlist[c];
        for (int at = ctx->molbeg_all[i]; at < ctx->molbeg_all[i + 1]; ++at) s += ctx->charge[at];
        q[c] = s;
      }
    CK(h2d(d.tgtq, q.data(), MD, st));
  }
  {
    BinArgs ba{};
    ba.ermax = ctx->ermax;
    ba.ermax_pad = ctx->ermax_pad;
    if (setup_bin_smem(ba) != 0) return bad(ERMOD_ERR_OVERFLOW, "ermax_lim");
  }
  if (pme) {
    std::vector<double> sf(K1 + K2 + K3);
    spline_axis(K1, p.splodr, sf.data());
    spline_axis(K2, p.splodr, sf.data() + K1);
    spline_axis(K3, p.splodr, sf.data() + K1 + K2);
    CK(h2d(d.splfc, sf.data(), K1 + K2 + K3, st));
  }
  if (p.cltype == ERMOD_EL_PPPM) {
    // calc_gfb_pppm (recpcal.F90:179-198): the alias sum of the order-P assignment function
    // is a polynomial of degree P-1 in sin^2(k h / 2); the reference's recurrence for its
    // coefficients, then the division by (2P-1)!
    PppmGreen& pg = ctx->pppm;
    pg.on = 1;
    const int P = p.splodr;
    for (int l = 0; l < kMaxOrder; ++l) pg.gfb[l] = 0.0;
    pg.gfb[0] = 1.0;
    for (int m = 1; m < P; ++m) {
      for (int l = m; l >= 1; --l)
        pg.gfb[l] = 4.0 * (pg.gfb[l] * (l - m) * (l - m - 0.5) - pg.gfb[l - 1] * (l - m - 1) * (l - m - 1));
      pg.gfb[0] = 4.0 * pg.gfb[0] * m * (m + 0.5);
    }
    double fact = 1.0;
    for (int i = 2; i <= 2 * P - 1; ++i) fact *= i;
    for (int l = 0; l < P; ++l) pg.gfb[l] /= fact;
  }
  if (pme && ctx->spath == 1) {
    int n[3] = {K3, K2, K1};
    int inR[3] = {K3, K2, K1}, onC[3] = {K3, K2, Kh1};
    CF(cufftPlanMany(&ctx->r2c, 3, n, inR, 1, (int)KK, onC, 1, (int)KH, CUFFT_R2C, ctx->chunk));
    int inC[3] = {K3, K2, Kh1}, onR[3] = {K3, K2, K1};
    CF(cufftPlanMany(&ctx->c2r, 3, n, inC, 1, (int)KH, onR, 1, (int)KK, CUFFT_C2R, ctx->chunk));
    ctx->plans = true;
    CF(cufftSetStream(ctx->r2c, st));
    CF(cufftSetStream(ctx->c2r, st));
  }
  ctx->use_tc = (p.corrcal && ecorr_tc_available() && p.ecorr_path == 0) ? 1 : 0;
  if (ctx->use_tc) {
    ctx->tc_work_bytes = ecorr_tc_workspace(ctx->batch, ctx->ermax);
    CK(cudaMalloc(&ctx->tc_work, ctx->tc_work_bytes));
  }
  const int rc = ermod_engclear(ctx);
  if (rc != ERMOD_OK) return rc;
  // minuv / maxuv / voffset start values (enginit, engproc.F90:299-303)
  std::vector<float> mn(ctx->numslv + 1, FLT_MAX), mx(ctx->numslv + 1, -FLT_MAX);
  CK(h2d(d.minuv, mn.data(), mn.size(), st));
  CK(h2d(d.maxuv, mx.data(), mx.size(), st));
  double sc[8] = {0, 0, 0, -(double)FLT_MAX, 0, 0, 0, 0};
  CK(h2d(d.scal, sc, 8, st));
  CK(cudaStreamSynchronize(st));
  return ERMOD_OK;
}

int32_t ermod_set_refstructure(ermod_ctx* ctx, int32_t refspec, int32_t nhost, const float* host_crd,
                               const float* host_w, const float* slt_crd, const float* slt_w) {
  if (!ctx || refspec == 0 || nhost <= 0 || !host_crd || !host_w || !slt_crd || !slt_w) return ERMOD_ERR_ARG;
  ctx->err.clear();
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->st));
  // refhost_specatm (insertion.F90:686-702): every atom of the refspec molecules, in molecule order
  std::vector<int> atoms;
  int off = 0;
  for (int k = 0; k < ctx->slvmax; ++k) {
    const int i = ctx->tagpt[k], sp = ctx->uvspec[i];
    if (sp >= 1 && sp <= 31 && ((refspec >> (sp - 1)) & 1))
      for (int j = 0; j < ctx->numsite[i]; ++j) atoms.push_back(off + j);
    off += ctx->numsite[i];
  }
  if ((int)atoms.size() != nhost) return set_error(ctx, ERMOD_ERR_ARG, "ins_ref");
  double wh = 0.0, wsl = 0.0;
  for (int i = 0; i < nhost; ++i) wh += host_w[i];
  for (int i = 0; i < ctx->s; ++i) wsl += slt_w[i];
  if (!(wh > 0.0) || !(wsl > 0.0)) return set_error(ctx, ERMOD_ERR_ARG, "bst_zrw");   // bestfit.F90:261
  DeviceState& d = ctx->d;
  for (void* q : {(void*)d.ref_atom, (void*)d.ref_host, (void*)d.ref_host_w, (void*)d.ref_slt, (void*)d.ref_slt_w,
                  (void*)d.ref_bf})
    if (q) cudaFree(q);
  const size_t n = nhost, S = ctx->s;
  CK(dalloc(&d.ref_atom, n)); CK(dalloc(&d.ref_host, 3 * n)); CK(dalloc(&d.ref_host_w, n));
  CK(dalloc(&d.ref_slt, 3 * S)); CK(dalloc(&d.ref_slt_w, S)); CK(dalloc(&d.ref_bf, 3 * S));
  CK(h2d(d.ref_atom, atoms.data(), n, ctx->st));
  CK(h2d(d.ref_host, host_crd, 3 * n, ctx->st));
  CK(h2d(d.ref_host_w, host_w, n, ctx->st));
  CK(h2d(d.ref_slt, slt_crd, 3 * S, ctx->st));
  CK(h2d(d.ref_slt_w, slt_w, S, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->nref = nhost;
  ctx->gkey.clear();   // the frame graph holds the old buffers: capture it again
  return ERMOD_OK;
}

int32_t ermod_engclear(ermod_ctx* ctx) {
  if (!ctx) return ERMOD_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  DeviceState& d = ctx->d;
  cudaStream_t st = ctx->st;
  CK(cudaMemsetAsync(d.edens, 0, sizeof(double) * ctx->ermax, st));
  if (d.ecorr) CK(cudaMemsetAsync(d.ecorr, 0, sizeof(double) * ctx->ermax * ctx->ermax, st));
  CK(cudaMemsetAsync(d.eself, 0, sizeof(double) * std::max(1, ctx->esmax), st));
  CK(cudaMemsetAsync(d.slnuv, 0, sizeof(double) * ctx->numslv, st));
  // avslf, engnorm, engsmpl (scal[0..2]); voffset and the self-energy reuse persist
  CK(cudaMemsetAsync(d.scal, 0, sizeof(double) * 3, st));
  CK(cudaStreamSynchronize(st));
  return ERMOD_OK;
}

}  // extern "C"

// ---- the per-frame pipeline ------------------------------------------------
// frame_plan   host: cell normalisation and every per-frame constant (FramePlan);
// frame_enqueue device work of one frame on one stream, no host synchronisation;
//              the frame's inputs (coordinates, stnum) are staged in fixed device
//              buffers beforehand, so the enqueued work can be captured once as a
//              CUDA graph and replayed while the plan stays the same;
// frame_finish host: status word and stage timings after the stream is done.

// Everything the enqueued work depends on besides the staged inputs.  Compared
// bytewise to decide whether a captured graph is still valid, so it is
// zero-filled before use.
struct FramePlan {
  FrameArgs a;
  WeightArgs wa;
  BinArgs ba;
  int ncell, use_conf, selfreal, real_threads;
  int prop_gv, prop_gf, prop_learned;   // proposal voxels and feature cells per side (0: none), network on
  float prop_eps;
};

struct FramePlanHost {
  FramePlan k;
  bool engfac;          // influence function to rebuild before the frame
  double inv[3][3], vold;
};

// Cell grid of the real-space cell list for cells of edge >= hmin on the normalised cuboid
// box (at most 64 a side, at least 3); false when no such grid fits.
constexpr float kCellDefault = 4.0f;
static bool cell_grid(const ermod_ctx* ctx, FrameArgs& a, float hmin, int& ncell) {
  bool ok = true;
  for (int dd = 0; dd < 3; ++dd) {
    a.nc[dd] = std::max(1, std::min(64, (int)std::floor(a.g.len[dd] / hmin)));
    a.ch[dd] = a.g.len[dd] / (float)a.nc[dd];
    if (a.nc[dd] < 3) ok = false;
  }
  ncell = a.nc[0] * a.nc[1] * a.nc[2];
  return ok && ncell <= ctx->ncell_cap;
}

static int frame_plan(ermod_ctx* ctx, const float* cellin, float wsys, bool use_conf, FramePlanHost& ph) {
  const ermod_params& p = ctx->p;
  std::memset(&ph, 0, sizeof(ph));
  FramePlan& fp = ph.k;
  const bool refs = p.slttype != ERMOD_SLT_SOLN;
  const bool pme = p.cltype == ERMOD_EL_PME || p.cltype == ERMOD_EL_PPPM;
  const int K1 = p.ms1max, K2 = p.ms2max, K3 = p.ms3max;
  // ---- cell (engproc.F90:1049-1070, realcal.F90:776-896) ----
  double c[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) c[i][j] = cellin[j * 3 + i];
  float cf[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) cf[i][j] = cellin[j * 3 + i];
  // FP32 as the reference's get_inverted_cell
  const float vol = cf[0][0] * cf[1][1] * cf[2][2] + cf[0][1] * cf[1][2] * cf[2][0] + cf[0][2] * cf[1][0] * cf[2][1] -
                    cf[0][2] * cf[1][1] * cf[2][0] - cf[0][1] * cf[1][0] * cf[2][2] - cf[0][0] * cf[1][2] * cf[2][1];
  const double vold = c[0][0] * c[1][1] * c[2][2] + c[0][1] * c[1][2] * c[2][0] + c[0][2] * c[1][0] * c[2][1] -
                      c[0][2] * c[1][1] * c[2][0] - c[0][1] * c[1][0] * c[2][2] - c[0][0] * c[1][2] * c[2][1];
  double (&inv)[3][3] = ph.inv;
  inv[0][0] = c[1][1] * c[2][2] - c[1][2] * c[2][1];
  inv[0][1] = c[0][2] * c[2][1] - c[0][1] * c[2][2];
  inv[0][2] = c[0][1] * c[1][2] - c[0][2] * c[1][1];
  inv[1][0] = c[1][2] * c[2][0] - c[1][0] * c[2][2];
  inv[1][1] = c[0][0] * c[2][2] - c[0][2] * c[2][0];
  inv[1][2] = c[0][2] * c[1][0] - c[0][0] * c[1][2];
  inv[2][0] = c[1][0] * c[2][1] - c[1][1] * c[2][0];
  inv[2][1] = c[0][1] * c[2][0] - c[0][0] * c[2][1];
  inv[2][2] = c[0][0] * c[1][1] - c[0][1] * c[1][0];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) inv[i][j] /= vold;
  ph.vold = vold;
  FrameArgs& a = fp.a;
  CellGeom& g = a.g;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      g.cell[i][j] = cf[i][j];
      g.invcl[i][j] = (float)inv[i][j];
      g.rot[i][j] = i == j ? 1.f : 0.f;
    }
  g.volume = vol;
  g.periodic = p.boxshp == ERMOD_SYS_PERIODIC;
  if (g.periodic) {
    float cn[3][3];
    if (cf[1][0] == 0.f && cf[2][0] == 0.f && cf[2][1] == 0.f) {
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) cn[i][j] = cf[i][j];
      g.rotated = 0;
    } else {  // modified Gram-Schmidt (realcal.F90:794-816)
      float q[3][3] = {}, r[3][3] = {}, tmp[3][3];
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) tmp[i][j] = cf[i][j];
      for (int i = 0; i < 3; ++i) {
        const float len = std::sqrt(tmp[0][0] * tmp[0][0] + tmp[1][0] * tmp[1][0] + tmp[2][0] * tmp[2][0]);
        for (int k = 0; k < 3; ++k) q[k][i] = tmp[k][i] / len;
        r[i][i] = len;
        for (int j = i + 1; j < 3; ++j) {
          r[i][j] = q[0][i] * tmp[0][j] + q[1][i] * tmp[1][j] + q[2][i] * tmp[2][j];
          for (int k = 0; k < 3; ++k) tmp[k][j] -= r[i][j] * q[k][i];
        }
      }
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { cn[i][j] = r[i][j]; g.rot[i][j] = q[i][j]; }
      g.rotated = 1;
    }
    for (int i = 0; i < 3; ++i)  // normalize_cell_vector (realcal.F90:826-830)
      if (cn[0][0] < 0.f) for (int k = 0; k < 3; ++k) cn[k][i] = -cn[k][i];
    const float thr = 1e-4f;
    if (std::fabs(cn[0][1]) > 0.5f * cn[0][0] + thr) {
      const float f = std::round(cn[0][1] * ctx->invcell_prev[0]);
      for (int k = 0; k < 3; ++k) cn[k][1] -= cn[k][0] * f;
    }
    if (std::fabs(cn[0][2]) > 0.5f * cn[0][0] + thr) {
      const float f = std::round(cn[0][2] * ctx->invcell_prev[0]);
      for (int k = 0; k < 3; ++k) cn[k][2] -= cn[k][0] * f;
    }
    if (std::fabs(cn[1][2]) > 0.5f * cn[1][1] + thr) {
      const float f = std::round(cn[1][2] * ctx->invcell_prev[1]);
      for (int k = 0; k < 3; ++k) cn[k][2] -= cn[k][1] * f;
    }
    const float cut = std::min(p.elecut, p.upljcut);
    for (int i = 0; i < 3; ++i)
      if (cut > cn[i][i] * 0.5f) return set_error(ctx, ERMOD_ERR_CELL, "cel_siz");
    for (int i = 0; i < 3; ++i) {
      g.len[i] = std::fabs(cn[i][i]);
      g.inv[i] = 1.0f / g.len[i];
      g.half[i] = 0.5f * g.len[i];
      ctx->invcell_prev[i] = g.inv[i];
    }
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) g.cn[i][j] = cn[i][j];
    g.cuboid = !(std::fabs(cf[0][1]) > 1e-8f || std::fabs(cf[0][2]) > 1e-8f || std::fabs(cf[1][2]) > 1e-8f);
  } else {
    g.cuboid = 1;
  }
  if (refs && (p.insposition == ERMOD_INSPOS_RANDOM || p.insposition == ERMOD_INSPOS_SLAB_GENERIC ||
               p.insposition == ERMOD_INSPOS_SLAB_SYMMETRIC) && !g.periodic)
    return set_error(ctx, ERMOD_ERR_INS_GEO, "ins_geo");   // insertion.F90:154-156, 185-187
  if (!refs && (p.insposition == ERMOD_INSPOS_SLAB_GENERIC || p.insposition == ERMOD_INSPOS_SLAB_SYMMETRIC) &&
      !g.periodic)
    return set_error(ctx, ERMOD_ERR_INS_GEO, "eng_slb");   // engproc.F90:1238
  if (ctx->nref == 0 && ((p.insposition >= ERMOD_INSPOS_RMSD && (refs || p.insposition == ERMOD_INSPOS_RMSD)) ||
                         (!refs && p.insstructure == ERMOD_INSSTR_RMSD)))
    return set_error(ctx, ERMOD_ERR_ARG, "ins_ref");        // load_refstructure (insertion.F90:676-770)
  if (refs && p.insposition == ERMOD_INSPOS_GAUSS && !ctx->gauss_init) {
    // uniform_gauss_mixture keeps the first call's cell (insertion.F90:268-274): l = (|c_k|/2)/upreg,
    // z0 = 8 l1 l2 l3, z1 = pi^(3/2) erf(l1) erf(l2) erf(l3)
    double z0 = 8.0, z1 = std::pow(kPi, 1.5);
    for (int k = 0; k < 3; ++k) {
      const double len = std::sqrt(c[0][k] * c[0][k] + c[1][k] * c[1][k] + c[2][k] * c[2][k]);
      const double l = 0.5 * len / p.upreg;
      ctx->gauss_l[k] = (float)l;
      z0 *= l;
      z1 *= std::erf(l);
    }
    ctx->gauss_z0 = (float)z0;
    ctx->gauss_z1 = (float)z1;
    ctx->gauss_init = true;
  }
  // ---- pair / PME constants ----
  PairParams& P = a.pp;
  P.lw = p.lwljcut; P.up = p.upljcut; P.lw2 = p.lwljcut * p.lwljcut; P.up2 = p.upljcut * p.upljcut;
  P.lw3 = P.lw2 * p.lwljcut; P.up3 = P.up2 * p.upljcut; P.lw6 = P.lw3 * P.lw3; P.up6 = P.up3 * P.up3;
  auto gmx = [&](int pw, float& A, float& B, float& C) {  // realcal.F90:899-915
    const float lw = p.lwljcut, up = p.upljcut, df = up - lw;
    float uppw2 = 1.f, uppw = 1.f;
    for (int i = 0; i < pw + 2; ++i) uppw2 *= up;
    for (int i = 0; i < pw; ++i) uppw *= up;
    A = -(float)pw * ((float)(pw + 4) * up - (float)(pw + 1) * lw) / (uppw2 * (df * df)) / 3.0f;
    B = (float)pw * ((float)(pw + 3) * up - (float)(pw + 1) * lw) / (uppw2 * (df * df * df)) / 4.0f;
    C = 1.0f / uppw - A * (df * df * df) - B * (df * df * df * df);
  };
  gmx(12, P.repA, P.repB, P.repC);
  gmx(6, P.attA, P.attB, P.attC);
  P.reelcut = g.periodic ? p.elecut : FLT_MAX;
  P.screen = p.screen;
  P.ljswitch = p.ljswitch;
  P.bare = p.cltype == ERMOD_EL_COULOMB;
  a.slvmax = ctx->slvmax; a.natoms = ctx->natoms; a.nsite = ctx->s; a.maxdst = ctx->maxdst;
  a.K1 = K1; a.K2 = K2; a.K3 = K3; a.order = pme ? p.splodr : 1; a.Kh1 = K1 / 2 + 1;
  // Fused solve: planes k1 whose every mode has exp(-pi^2 |k|^2 / screen^2) < kModeCut are not
  // transformed (|k| >= k1 / |a1| in plane k1, a1 the first cell vector).  Their share of any
  // molecule energy is below 1e-9 of the k = 0 Gaussian weight per mode, far under FP32 rounding.
  a.k1max = K1 / 2;
  if (pme) {
    const double a1 = std::sqrt(c[0][0] * c[0][0] + c[1][0] * c[1][0] + c[2][0] * c[2][0]);
    const double mcut = std::sqrt(-std::log(kModeCut)) * (double)p.screen * a1 / kPi;
    a.k1max = std::max(0, std::min(K1 / 2, (int)std::floor(mcut) + 1));
  }
  a.ljtype_max = ctx->ljtype_max;
  a.pme = pme;
  a.pivol = pme ? kPi / ((double)p.screen * (double)p.screen) / vold : 0.0;
  a.rcut = g.periodic ? std::max(p.elecut, p.upljcut) : (P.bare ? FLT_MAX : p.upljcut);
  if (P.bare && !g.periodic) a.rcut = FLT_MAX;
  // cell list only for cuboid periodic boxes
  a.use_cells = 0;
  fp.ncell = 1;
  if (g.periodic && g.cuboid && !g.rotated) {
    a.use_cells = cell_grid(ctx, a, ctx->cell_h > 0.f ? ctx->cell_h : kCellDefault, fp.ncell) ? 1 : 0;
  }
  // ---- influence function when the cell changes (engconst :423-433) ----
  if (pme) {
    bool changed = !ctx->pme_init;
    for (int i = 0; i < 9; ++i) if (ctx->prevcl[i] != cellin[i]) changed = true;
    ph.engfac = changed;
    if (changed && ctx->pppm.on) {
      // alias range (recpcal.F90:230-233, 243-244): LAMMPS's accuracy form with EPS_HOC = 1e-7
      // per mesh axis, projected on each cell vector, in single precision and truncated
      const float acc = std::pow(-std::log(1.0e-7f), 0.25f);
      const float pi = (float)kPi;
      const float mm[3] = {p.screen / (pi * (float)K1) * acc, p.screen / (pi * (float)K2) * acc,
                           p.screen / (pi * (float)K3) * acc};
      for (int j = 0; j < 3; ++j) {
        ctx->pppm.mmax[j] = (int)(cf[0][j] * mm[0] + cf[1][j] * mm[1] + cf[2][j] * mm[2]);
        if (ctx->pppm.mmax[j] < 0) return set_error(ctx, ERMOD_ERR_ARG, "pppm_mrg");
      }
    }
  }
  // ---- real-space self term: per insertion, or once for a rigid solute ----
  const bool rigid = p.slttype == ERMOD_SLT_REFS_RIGID;
  fp.selfreal = P.bare ? 0 : (rigid ? (ctx->usreal_init ? 3 : 1) : 2);
  fp.use_conf = use_conf ? 1 : 0;
  fp.real_threads = ctx->real_threads;
  // ---- insertion proposal (refs mode, random positions only) ----
  const bool learned = refs && p.proposal == ERMOD_PROPOSAL_LEARNED;
  if (learned && (ctx->prop_gv <= 0 || !ctx->prop_params)) return set_error(ctx, ERMOD_ERR_ARG, "prp_set");
  if (learned && p.insposition != ERMOD_INSPOS_RANDOM) return set_error(ctx, ERMOD_ERR_ARG, "prp_pos");
  fp.prop_gv = (refs && p.insposition == ERMOD_INSPOS_RANDOM) ? ctx->prop_gv : 0;
  fp.prop_gf = ctx->prop_gf;
  fp.prop_learned = learned ? 1 : 0;
  fp.prop_eps = ctx->prop_eps;
  // ---- weights ----
  WeightArgs& wa = fp.wa;
  wa.slttype = p.slttype; wa.wgtslf = p.wgtslf; wa.estype = p.estype; wa.selfcal = p.selfcal;
  wa.numslv = ctx->numslv; wa.esmax = ctx->esmax; wa.rigid = rigid && !P.bare;
  wa.temp = p.temp;
  wa.stat_weight_system = wsys;
  double qslt = refs ? ctx->qslt_refs : 0.0;
  if (!refs) {  // soln solutes share one site layout; charge of the first solute
    float q = 0.f;
    const int i = ctx->sltlist[0];
    for (int at = ctx->molbeg_all[i]; at < ctx->molbeg_all[i + 1]; ++at) q += ctx->charge[at];
    qslt = q;
  }
  wa.resid_self = P.bare ? 0.0 : -(kPi * qslt * qslt / (double)p.screen / (double)p.screen / vold) / 2.0;
  wa.npt_factor = 1.0;
  if (p.estype == ERMOD_ES_NPT) {  // volcorrect (engproc.F90:1022-1038)
    double qt = 0.0;
    for (int k = 0; k < ctx->slvmax; ++k) {
      const int i = ctx->tagpt[k];
      float q = 0.f;
      for (int at = ctx->molbeg_all[i]; at < ctx->molbeg_all[i + 1]; ++at) q += ctx->charge[at];
      qt += q;
    }
    double f = vold;
    if (pme) f *= std::exp(kPi * qt * qt / ((double)p.screen * p.screen) / vold / 2.0 / p.temp);
    wa.npt_factor = f;
  }
  BinArgs& ba = fp.ba;
  ba.ermax = ctx->ermax; ba.ermax_pad = ctx->ermax_pad; ba.numslv = ctx->numslv; ba.slttype = p.slttype;
  return ERMOD_OK;
}

// Host-side state the plan consumed, committed once the frame is enqueued.
static void frame_commit(ermod_ctx* ctx, const float* cellin, const FramePlanHost& ph) {
  if (ph.k.a.pme) {
    for (int i = 0; i < 9; ++i) ctx->prevcl[i] = cellin[i];
    ctx->pme_init = true;
  }
  if (ph.k.selfreal == 1) ctx->usreal_init = true;
}

// Block size of k_real: the autotuner's candidates all give bit-identical
// energies (a warp per molecule whatever the block size), so the choice only
// moves time.  Tuned on the first frame with the frame's own data.
static const int kRealCandidates[] = {128, 256, 512};
static const float kCellCandidates[] = {3.0f, 4.0f, 5.0f, 6.0f};

// The real-space autotuner, run on the first frame with that frame's own data: every cell
// edge of kCellCandidates (on cuboid periodic boxes) times every block size of
// kRealCandidates, each timed on the second of two launches; the fastest pair is kept for
// the context's later frames.  A molecule's energy is one fixed-order sum whatever the cell
// grid and block size, so the choice moves only time.  The frame's own cell list is rebuilt
// afterwards, so the rest of this frame runs on the grid it was planned with.
static int tune_real(ermod_ctx* ctx, const FrameArgs& a, int ncell0, int nbatch, cudaStream_t st) {
  float best = 1e30f;
  int pick = 256;
  float hpick = kCellDefault;
  cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1];
  const int nh = a.use_cells ? (int)(sizeof(kCellCandidates) / sizeof(float)) : 1;
  for (int ih = 0; ih < nh; ++ih) {
    FrameArgs b = a;
    if (a.use_cells) {
      int nc = 0;
      if (!cell_grid(ctx, b, kCellCandidates[ih], nc)) continue;
      launch_cells(b, ctx->d, nc, st);
    }
    for (int rep = 0; rep < 2; ++rep)
      for (int nt : kRealCandidates) {
        CK(cudaEventRecord(e0, st));
        launch_real(b, ctx->d, 0, nbatch, ctx->batch, nt, st);
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep == 1 && ms < best) {
          best = ms;
          pick = nt;
          hpick = a.use_cells ? kCellCandidates[ih] : kCellDefault;
        }
      }
  }
  if (a.use_cells) launch_cells(a, ctx->d, ncell0, st);
  ctx->real_threads = pick;
  ctx->cell_h = hpick;
  return ERMOD_OK;
}

// Enqueue the device work of one frame on `st`.  `timed` records stage events
// (direct launches only).  Adds the number of kernel launches to `nl`.
static int frame_enqueue(ermod_ctx* ctx, const FramePlan& fp, cudaStream_t st, bool timed, long long& nl) {
  const ermod_params& p = ctx->p;
  DeviceState& d = ctx->d;
  const FrameArgs& a = fp.a;
  const bool refs = p.slttype != ERMOD_SLT_SOLN;
  const bool pme = a.pme;
  auto M = [&](int tag) { if (timed) mark(ctx, tag); };
  CK(cudaMemsetAsync(d.status, 0, sizeof(DevStatus), st));
  launch_prepare_solvent(a, d, st);
  launch_cells(a, d, fp.ncell, st);
  nl += 1 + (a.slvmax > 0 ? (a.use_cells ? 3 : 2) : 0);
  M(kStPrep);
  // ---- targets ----
  if (refs && fp.prop_gv > 0) {
    const int n = launch_proposal(a, d, fp.prop_gv, fp.prop_gf, fp.prop_eps, fp.prop_learned != 0, st);
    if (n < 0) return set_error(ctx, ERMOD_ERR_CUDA, "prp_run");
    nl += n;
  }
  if (refs && ctx->nhost > 0) {
    launch_aggcen(d, ctx->nhost, st);
    nl += 1;
  }
  if (ctx->nref > 0 && p.insposition >= ERMOD_INSPOS_RMSD) {   // reffit's host fit, once per frame
    launch_reffit(d, ctx->nref, ctx->s, st);
    nl += 1;
  }
  if (refs) {
    InsRegion rg{};
    rg.insposition = p.insposition;
    rg.insorient = p.insorient;
    rg.lwreg = p.lwreg;
    rg.upreg = p.upreg;
    for (int k = 0; k < 3; ++k) rg.gl[k] = ctx->gauss_l[k];
    rg.z0 = ctx->gauss_z0;
    rg.z1 = ctx->gauss_z1;
    launch_insert(a, d, d.frame_i, p.iseed, rg, fp.use_conf, fp.prop_gv, fp.prop_learned, st);
  }
  else launch_targets_soln(a, d, nullptr, st);
  if (!refs && d.skip) {   // check_mol_configuration of every solute
    if (ctx->nhost > 0) {
      launch_aggcen(d, ctx->nhost, st);
      nl += 1;
    }
    const SolnCheck ck{p.insposition, p.lwreg, p.upreg, p.insstructure, p.lwstr, p.upstr};
    launch_soln_region(a, d, ck, st);
    nl += 1;
  }
  CK(cudaMemsetAsync(d.selfrec, 0, sizeof(double) * ctx->maxdst, st));
  CK(cudaMemsetAsync(d.etot, 0, sizeof(double) * ctx->maxdst, st));
  CK(cudaMemsetAsync(d.flceng, 0, sizeof(double) * ctx->maxdst * ctx->numslv, st));
  if (d.uvengy) CK(cudaMemsetAsync(d.uvengy, 0, sizeof(double) * ctx->maxdst * ctx->slvmax, st));
  switch (fp.selfreal) {
    case 0: CK(cudaMemsetAsync(d.selfreal, 0, sizeof(double) * ctx->maxdst, st)); break;
    case 1: launch_selfreal(a, d, 0, 1, (double)p.screen, st); nl += 1; break;
    case 2: launch_selfreal(a, d, 0, ctx->maxdst, (double)p.screen, st); nl += 1; break;
    default: break;   // rigid solute: the first insertion's term is kept (engproc.F90:839-851)
  }
  nl += 1;
  M(kStIns);
  // ---- batches of targets, each in chunks of `chunk` PME solves ----
  const int chunk = ctx->chunk;
  for (int bb = 0; bb < ctx->maxdst; bb += ctx->batch) {
    const int nbatch = std::min(ctx->batch, ctx->maxdst - bb);
    if (ctx->real_threads == 0) {
      const int rc = tune_real(ctx, a, fp.ncell, nbatch, st);
      if (rc != ERMOD_OK) return rc;
    }
    // Real space beside the PME chain: k_real on the second stream, joined before binning (the
    // gather writes the reciprocal part, k_bin adds the real part).  Stage-timed runs keep one
    // stream so that each stage's events bracket it alone; the arithmetic is the same.
    const bool fork = pme && !timed;
    if (fork) {
      CK(cudaEventRecord(ctx->ev_fork, st));
      CK(cudaStreamWaitEvent(ctx->st2, ctx->ev_fork, 0));
    }
    launch_real(a, d, bb, nbatch, ctx->batch, ctx->real_threads, fork ? ctx->st2 : st);
    if (fork) CK(cudaEventRecord(ctx->ev_join, ctx->st2));
    M(kStReal);
    nl += 1;
    if (pme && ctx->spath != 1) {
      launch_site_tables(a, d, bb, nbatch, ctx->spath == 2, st);
      M(kStSiteTab);
      nl += 1;
    }
    // Fused solve, untimed: each chunk kernel may start while its predecessor finishes
    // (programmatic dependent launch; the first plane of a batch follows the site tables).
    const bool pdl = pme && ctx->spath != 1 && !timed;
    for (int cb = bb; cb < bb + nbatch; cb += chunk) {
      const int nb = std::min(chunk, bb + nbatch - cb);
      if (pme && ctx->spath != 1) {
        launch_pme_plane(a, d, cb - bb, nb, ctx->spath == 2, pdl && cb > bb, st);
        M(kStPlane);
        launch_pme_rows(a, d, cb, nb, pdl, st);
        M(kStRows);
        nl += 2;
      } else if (pme) {
        launch_spread(a, d, cb, nb, chunk, st);
        M(kStSpread);
        CF(cufftExecR2C(ctx->r2c, d.grid, (cufftComplex*)d.spec));
        M(kStR2C);
        launch_clear_box(a, d, chunk, st);
        launch_influence(a, d, cb, nb, chunk, st);
        M(kStInfl);
        nl += 3;
        CF(cufftExecC2R(ctx->c2r, (cufftComplex*)d.spec, d.phin));
        M(kStC2R);
        launch_transpose_phi(a, d, st);
        M(kStTranspose);
        nl += 1;
      }
      launch_gather(a, d, cb, bb, nb, chunk, ctx->batch, pdl, st);
      M(kStGather);
      nl += 1;
    }
    if (fork) CK(cudaStreamWaitEvent(st, ctx->ev_join, 0));   // the real-space energies of the batch
    launch_bin(d, fp.ba, bb, nbatch, ctx->slvmax, ctx->batch, st);
    M(kStBin);
    nl += 1;
    if (d.uvengy)
      CK(cudaMemcpyAsync(d.uvengy + (size_t)bb * ctx->slvmax, d.Etot, sizeof(double) * (size_t)nbatch * ctx->slvmax,
                         cudaMemcpyDeviceToDevice, st));
    launch_weights(d, fp.wa, bb, nbatch, st);
    launch_edens(d, bb, nbatch, ctx->ermax, ctx->ermax_pad, bb, st);
    nl += 3;
    M(kStWeights);
    if (p.corrcal) {
      if (ctx->use_tc) {
        const int rc = launch_ecorr_tc(d, bb, nbatch, ctx->ermax, ctx->ermax_pad, bb, p.weight_bits, ctx->tc_work,
                                       ctx->tc_work_bytes, st);
        if (rc != 0) return set_error(ctx, ERMOD_ERR_CUDA, "ecorr_tc");
        nl += 5;   // counts transpose, high-count list, weight digits, GEMM, high-count correction
      } else {
        launch_ecorr_simt(d, bb, nbatch, ctx->ermax, ctx->ermax_pad, bb, st);
        nl += 1;
      }
    }
    M(kStEcorr);
  }
  CK(cudaMemcpyAsync(ctx->h_status, d.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, st));
  return ERMOD_OK;
}

// After the frame's stream work is complete: stage timings and the status word.
static int frame_finish(ermod_ctx* ctx, bool timed, float total_ms) {
  for (float& t : ctx->timings) t = 0.f;
  if (timed) {
    for (int k = 1; k < ctx->pused; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ctx->pev[k - 1], ctx->pev[k]);
      ctx->timings[ctx->ptag[k]] += ms;
      ctx->timings[0] += ms;
    }
  } else {
    ctx->timings[0] = total_ms;
  }
  ctx->timings[kStChunks] = (float)((ctx->maxdst + ctx->chunk - 1) / ctx->chunk);
  const DevStatus hs = *ctx->h_status;
  if (hs.flags & kErrEngCns) return set_error(ctx, ERMOD_ERR_ENG_CNS, "eng_cns");
  if (hs.flags & kErrEngMin) return set_error(ctx, ERMOD_ERR_ENG_MIN, "eng_min");
  if (hs.flags & kErrEngSft) return set_error(ctx, ERMOD_ERR_ENG_SFT, "eng_sft");
  if (hs.flags & kErrOverflow) return set_error(ctx, ERMOD_ERR_OVERFLOW, "ermod_ovf");
  if (hs.flags & kErrGrid) return set_error(ctx, ERMOD_ERR_OVERFLOW, "spr_box");
  if (hs.flags & kErrTimeout) return set_error(ctx, ERMOD_ERR_CUDA, "tc_wait");
  if (hs.flags & kErrInsRej) return set_error(ctx, ERMOD_ERR_INS_GEO, "ins_rej");
  if ((hs.flags & kWarnMbin) && ctx->warn_bin_firsttime) {
    ctx->warn_bin_firsttime = false;
    return set_error(ctx, ERMOD_WARN_MBIN, "mbin");
  }
  return ERMOD_OK;
}

// Capture `body` on `st` as a graph and make `*exec` run it: update the
// existing executable when the topology allows, else instantiate anew.
template <class Body>
static cudaError_t capture_graph(cudaStream_t st, cudaGraphExec_t* exec, Body body, int* body_rc) {
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return e;
  *body_rc = body();
  e = cudaStreamEndCapture(st, &graph);
  if (*body_rc != ERMOD_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return e != cudaSuccess ? e : cudaErrorUnknown;
  }
  if (*exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(*exec, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(*exec);
      *exec = nullptr;
    }
  }
  if (!*exec) e = cudaGraphInstantiate(exec, graph, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(graph);
  return e;
}

// One frame of one context, its inputs already staged on ctx->st.
static int engconst_run(ermod_ctx* ctx, int stnum, const float* cellin, float wsys, bool use_conf) {
  FramePlanHost ph;
  int rc = frame_plan(ctx, cellin, wsys, use_conf, ph);
  if (rc != ERMOD_OK) return rc;
  cudaStream_t st = ctx->st;
  ctx->h_frame[0] = stnum;
  CK(cudaMemcpyAsync(ctx->d.frame_i, ctx->h_frame, sizeof(int), cudaMemcpyHostToDevice, st));
  if (ph.engfac) launch_engfac(ph.k.a, ctx->d, ph.inv, ph.vold, (double)ctx->p.screen, ctx->pppm, st);
  const bool timed = ctx->p.stage_timing != 0;
  const bool graph = !timed && ctx->p.graph_mode == 0 && ctx->real_threads != 0;
  float total = 0.f;
  if (!graph) {
    ctx->pused = 0;
    if (timed) mark(ctx, 0);
    else CK(cudaEventRecord(ctx->ev[2], st));
    long long nl = 0;
    rc = frame_enqueue(ctx, ph.k, st, timed, nl);
    if (rc != ERMOD_OK) return rc;
    if (!timed) CK(cudaEventRecord(ctx->ev[3], st));
    ctx->launches += nl;
  } else {
    if (!ctx->gexec || ctx->gkey.size() != sizeof(FramePlan) ||
        std::memcmp(ctx->gkey.data(), &ph.k, sizeof(FramePlan)) != 0) {
      long long nl = 0;
      int brc = ERMOD_OK;
      const cudaError_t e =
          capture_graph(st, &ctx->gexec, [&]() { return frame_enqueue(ctx, ph.k, st, false, nl); }, &brc);
      if (brc != ERMOD_OK) return brc;
      CK(e);
      ctx->gkey.assign((const unsigned char*)&ph.k, (const unsigned char*)&ph.k + sizeof(FramePlan));
      ctx->graph_launches = nl;
    }
    CK(cudaEventRecord(ctx->ev[2], st));
    CK(cudaGraphLaunch(ctx->gexec, st));
    CK(cudaEventRecord(ctx->ev[3], st));
    ctx->launches += ctx->graph_launches;
  }
  frame_commit(ctx, cellin, ph);
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  if (!timed) CK(cudaEventElapsedTime(&total, ctx->ev[2], ctx->ev[3]));
  return frame_finish(ctx, timed, total);
}

// Stage the host inputs of a frame into the context's device buffers.
static int stage_host_inputs(ermod_ctx* ctx, const float* sitepos, const float* ins_conf, const float* ins_weight,
                             size_t* nconf_out) {
  const bool refs = ctx->p.slttype != ERMOD_SLT_SOLN;
  const size_t npos = 3 * (size_t)ctx->natoms;
  const size_t nconf = (refs && ins_conf) ? 3 * (size_t)ctx->s * ctx->maxdst : 0;
  const size_t need = sizeof(float) * (npos + nconf + ctx->maxdst);
  if (ctx->h_pin_bytes < need) {
    if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
    ctx->h_pin = nullptr;
    CK(cudaMallocHost((void**)&ctx->h_pin, need));
    ctx->h_pin_bytes = need;
  }
  CK(cudaStreamSynchronize(ctx->st));   // the staging buffer may still feed the previous frame's copies
  std::memcpy(ctx->h_pin, sitepos, sizeof(float) * npos);
  CK(cudaMemcpyAsync(ctx->d.posraw, ctx->h_pin, sizeof(float) * npos, cudaMemcpyHostToDevice, ctx->st));
  if (nconf) {
    std::memcpy(ctx->h_pin + npos, ins_conf, sizeof(float) * nconf);
    CK(cudaMemcpyAsync(ctx->d.ins_conf, ctx->h_pin + npos, sizeof(float) * nconf, cudaMemcpyHostToDevice, ctx->st));
  }
  float* hw = ctx->h_pin + npos + nconf;
  for (int i = 0; i < ctx->maxdst; ++i) hw[i] = (refs && ins_weight) ? ins_weight[i] : 1.0f;
  CK(cudaMemcpyAsync(ctx->d.insw_in, hw, sizeof(float) * ctx->maxdst, cudaMemcpyHostToDevice, ctx->st));
  *nconf_out = nconf;
  return ERMOD_OK;
}

extern "C" {

int32_t ermod_engconst(ermod_ctx* ctx, int32_t stnum, const float* sitepos, const float* cell,
                       float stat_weight_system, const float* ins_conf, const float* ins_weight, float* flceng) {
  if (!ctx || !sitepos || !cell) return ERMOD_ERR_ARG;
  ctx->err.clear();
  CK(cudaSetDevice(ctx->device));
  const bool refs = ctx->p.slttype != ERMOD_SLT_SOLN;
  size_t nconf = 0;
  int rc = stage_host_inputs(ctx, sitepos, ins_conf, ins_weight, &nconf);
  if (rc != ERMOD_OK) return rc;
  rc = engconst_run(ctx, stnum, cell, stat_weight_system, nconf > 0);
  if (rc < 0) return rc;
  if (flceng && !refs) {
    std::vector<double> f((size_t)ctx->maxdst * ctx->numslv);
    CK(cudaMemcpy(f.data(), ctx->d.flceng, sizeof(double) * f.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < f.size(); ++i) flceng[i] = (float)f[i];
  }
  return rc;
}

int32_t ermod_engconst_dev(ermod_ctx* ctx, int32_t stnum, const float* sitepos_dev, const float* cell,
                           float stat_weight_system, const float* ins_conf_dev, const float* ins_weight_dev) {
  if (!ctx || !sitepos_dev || !cell) return ERMOD_ERR_ARG;
  ctx->err.clear();
  CK(cudaSetDevice(ctx->device));
  const bool refs = ctx->p.slttype != ERMOD_SLT_SOLN;
  CK(cudaMemcpyAsync(ctx->d.posraw, sitepos_dev, sizeof(float) * 3 * ctx->natoms, cudaMemcpyDeviceToDevice, ctx->st));
  if (refs && ins_conf_dev)
    CK(cudaMemcpyAsync(ctx->d.ins_conf, ins_conf_dev, sizeof(float) * 3 * ctx->s * ctx->maxdst,
                       cudaMemcpyDeviceToDevice, ctx->st));
  if (refs && ins_weight_dev)
    CK(cudaMemcpyAsync(ctx->d.insw_in, ins_weight_dev, sizeof(float) * ctx->maxdst, cudaMemcpyDeviceToDevice, ctx->st));
  else
    launch_fill(ctx->d.insw_in, 1.0f, ctx->maxdst, ctx->st);
  return engconst_run(ctx, stnum, cell, stat_weight_system, refs && ins_conf_dev);
}

// ---- batches of contexts: one graph launch per frame ---------------------
//
// Solutes of different sizes share one solvent frame: every member context
// runs its own unchanged pipeline on its own stream, and the frame of all
// members is captured as ONE CUDA graph with a branch per member, launched
// once per frame.  Each member's results are bit-identical to calling
// ermod_engconst on it alone: the same kernels with the same arguments, no
// state shared between members, every reduction in a fixed order.

}  // extern "C"

struct ermod_batch {
  int device = 0;
  std::vector<ermod_ctx*> m;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec = nullptr;
  std::vector<unsigned char> gkey;
  std::vector<long long> member_launches;   // kernel launches of each member in the captured graph
  float* h_pos = nullptr;
  float* d_pos = nullptr;
  size_t npos = 0;
  float last_ms = 0.f;
  int failed = -1;
  std::string err;
};

extern "C" {

int32_t ermod_batch_create(ermod_batch** out, int32_t n, ermod_ctx* const* members) {
  if (!out || n <= 0 || !members) return ERMOD_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return ERMOD_ERR_ARG;
    if (members[i]->device != members[0]->device || members[i]->natoms != members[0]->natoms)
      return ERMOD_ERR_ARG;   // members share the device and the solvent frame
    for (int j = 0; j < i; ++j)
      if (members[j] == members[i]) return ERMOD_ERR_ARG;
  }
  ermod_batch* b = new ermod_batch();
  b->device = members[0]->device;
  b->m.assign(members, members + n);
  b->npos = 3 * (size_t)members[0]->natoms;
  auto fail = [&]() {
    ermod_batch_destroy(b);
    return ERMOD_ERR_CUDA;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return fail();
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) return fail();
  if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return fail();
  if (cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess) return fail();
  b->join.resize(n, nullptr);
  b->member_launches.assign(n, 0);
  for (auto& e : b->join)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail();
  if (cudaMallocHost((void**)&b->h_pos, sizeof(float) * std::max<size_t>(b->npos, 1)) != cudaSuccess) return fail();
  if (cudaMalloc((void**)&b->d_pos, sizeof(float) * std::max<size_t>(b->npos, 1)) != cudaSuccess) return fail();
  *out = b;
  return ERMOD_OK;
}

static int batch_run(ermod_batch* b, int stnum, const float* cell, float wsys) {
  const int n = (int)b->m.size();
  b->failed = -1;
  b->err.clear();
  auto fail_member = [&](int i, int rc) {
    b->failed = i;
    b->err = "member " + std::to_string(i) + ": " + b->m[i]->err;
    return rc;
  };
  std::vector<FramePlanHost> ph(n);
  bool tuned = true;
  for (int i = 0; i < n; ++i) {
    ermod_ctx* ctx = b->m[i];
    ctx->err.clear();
    const int rc = frame_plan(ctx, cell, wsys, false, ph[i]);
    if (rc != ERMOD_OK) return fail_member(i, rc);
    if (ctx->real_threads == 0) tuned = false;
  }
  // stage every member's inputs on the batch stream, ahead of the graph
  for (int i = 0; i < n; ++i) {
    ermod_ctx* ctx = b->m[i];
    if (cudaMemcpyAsync(ctx->d.posraw, b->d_pos, sizeof(float) * b->npos, cudaMemcpyDeviceToDevice, b->st) !=
        cudaSuccess)
      return ERMOD_ERR_CUDA;
    ctx->h_frame[0] = stnum;
    if (cudaMemcpyAsync(ctx->d.frame_i, ctx->h_frame, sizeof(int), cudaMemcpyHostToDevice, b->st) != cudaSuccess)
      return ERMOD_ERR_CUDA;
    launch_fill(ctx->d.insw_in, 1.0f, ctx->maxdst, b->st);
    if (ph[i].engfac) launch_engfac(ph[i].k.a, ctx->d, ph[i].inv, ph[i].vold, (double)ctx->p.screen, ctx->pppm, b->st);
  }
  if (cudaEventRecord(b->t0, b->st) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (!tuned) {
    // first frame: direct launches on the member streams (the autotuner runs here)
    if (cudaEventRecord(b->fork, b->st) != cudaSuccess) return ERMOD_ERR_CUDA;
    for (int i = 0; i < n; ++i) {
      ermod_ctx* ctx = b->m[i];
      if (cudaStreamWaitEvent(ctx->st, b->fork, 0) != cudaSuccess) return ERMOD_ERR_CUDA;
      long long nl = 0;
      ctx->pused = 0;
      const int rc = frame_enqueue(ctx, ph[i].k, ctx->st, false, nl);
      if (rc != ERMOD_OK) return fail_member(i, rc);
      ctx->launches += nl;
      if (cudaEventRecord(b->join[i], ctx->st) != cudaSuccess) return ERMOD_ERR_CUDA;
      if (cudaStreamWaitEvent(b->st, b->join[i], 0) != cudaSuccess) return ERMOD_ERR_CUDA;
    }
  } else {
    std::vector<unsigned char> key;
    for (int i = 0; i < n; ++i)
      key.insert(key.end(), (const unsigned char*)&ph[i].k, (const unsigned char*)&ph[i].k + sizeof(FramePlan));
    if (!b->gexec || key != b->gkey) {
      long long nl = 0;
      (void)nl;
      int brc = ERMOD_OK, bad = -1;
      const cudaError_t e = capture_graph(b->st, &b->gexec, [&]() {
        if (cudaEventRecord(b->fork, b->st) != cudaSuccess) return (int)ERMOD_ERR_CUDA;
        for (int i = 0; i < n; ++i) {
          ermod_ctx* ctx = b->m[i];
          if (cudaStreamWaitEvent(ctx->st, b->fork, 0) != cudaSuccess) return (int)ERMOD_ERR_CUDA;
          long long nli = 0;
          const int rc = frame_enqueue(ctx, ph[i].k, ctx->st, false, nli);
          if (rc != ERMOD_OK) { bad = i; return rc; }
          b->member_launches[i] = nli;
          nl += nli;
          if (cudaEventRecord(b->join[i], ctx->st) != cudaSuccess) return (int)ERMOD_ERR_CUDA;
          if (cudaStreamWaitEvent(b->st, b->join[i], 0) != cudaSuccess) return (int)ERMOD_ERR_CUDA;
        }
        return (int)ERMOD_OK;
      }, &brc);
      if (brc != ERMOD_OK) return bad >= 0 ? fail_member(bad, brc) : brc;
      if (e != cudaSuccess) {
        b->err = std::string("cuda: ") + cudaGetErrorString(e);
        return ERMOD_ERR_CUDA;
      }
      b->gkey = key;
    }
    if (cudaGraphLaunch(b->gexec, b->st) != cudaSuccess) return ERMOD_ERR_CUDA;
    for (int i = 0; i < n; ++i) b->m[i]->launches += b->member_launches[i];
  }
  if (cudaEventRecord(b->t1, b->st) != cudaSuccess) return ERMOD_ERR_CUDA;
  for (int i = 0; i < n; ++i) frame_commit(b->m[i], cell, ph[i]);
  if (cudaStreamSynchronize(b->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ERMOD_ERR_CUDA;
  cudaEventElapsedTime(&b->last_ms, b->t0, b->t1);
  int worst = ERMOD_OK;
  for (int i = 0; i < n; ++i) {
    const int rc = frame_finish(b->m[i], false, b->last_ms);
    if (rc < 0) return fail_member(i, rc);
    if (rc > 0 && worst == ERMOD_OK) { worst = rc; b->failed = i; b->err = "member " + std::to_string(i) + ": " + b->m[i]->err; }
  }
  return worst;
}

int32_t ermod_batch_engconst(ermod_batch* b, int32_t stnum, const float* sitepos, const float* cell,
                             float stat_weight_system) {
  if (!b || !sitepos || !cell) return ERMOD_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (cudaStreamSynchronize(b->st) != cudaSuccess) return ERMOD_ERR_CUDA;
  std::memcpy(b->h_pos, sitepos, sizeof(float) * b->npos);
  if (cudaMemcpyAsync(b->d_pos, b->h_pos, sizeof(float) * b->npos, cudaMemcpyHostToDevice, b->st) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  return batch_run(b, stnum, cell, stat_weight_system);
}

int32_t ermod_batch_engconst_dev(ermod_batch* b, int32_t stnum, const float* sitepos_dev, const float* cell,
                                 float stat_weight_system) {
  if (!b || !sitepos_dev || !cell) return ERMOD_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (cudaMemcpyAsync(b->d_pos, sitepos_dev, sizeof(float) * b->npos, cudaMemcpyDeviceToDevice, b->st) !=
      cudaSuccess)
    return ERMOD_ERR_CUDA;
  return batch_run(b, stnum, cell, stat_weight_system);
}

float ermod_batch_last_ms(const ermod_batch* b) { return b ? b->last_ms : -1.f; }

const char* ermod_batch_last_error(const ermod_batch* b) { return b ? b->err.c_str() : "null"; }

void ermod_batch_destroy(ermod_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (auto e : b->join) if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->h_pos) cudaFreeHost(b->h_pos);
  if (b->d_pos) cudaFree(b->d_pos);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
}

int32_t ermod_fetch_accum(ermod_ctx* ctx, ermod_accum* o) {
  if (!ctx || !o) return ERMOD_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->st));
  const DeviceState& d = ctx->d;
  if (o->edens) CK(cudaMemcpy(o->edens, d.edens, sizeof(double) * ctx->ermax, cudaMemcpyDeviceToHost));
  if (o->ecorr && d.ecorr)
    CK(cudaMemcpy(o->ecorr, d.ecorr, sizeof(double) * ctx->ermax * ctx->ermax, cudaMemcpyDeviceToHost));
  if (o->eself && ctx->p.selfcal) CK(cudaMemcpy(o->eself, d.eself, sizeof(double) * ctx->esmax, cudaMemcpyDeviceToHost));
  if (o->slnuv) {
    std::vector<double> s(ctx->numslv);
    CK(cudaMemcpy(s.data(), d.slnuv, sizeof(double) * ctx->numslv, cudaMemcpyDeviceToHost));
    for (int i = 0; i < ctx->numslv; ++i) o->slnuv[i] = (float)s[i];
  }
  if (o->minuv) CK(cudaMemcpy(o->minuv, d.minuv, sizeof(float) * (ctx->numslv + 1), cudaMemcpyDeviceToHost));
  if (o->maxuv) CK(cudaMemcpy(o->maxuv, d.maxuv, sizeof(float) * (ctx->numslv + 1), cudaMemcpyDeviceToHost));
  double sc[8];
  CK(cudaMemcpy(sc, d.scal, sizeof(sc), cudaMemcpyDeviceToHost));
  o->avslf = sc[0];
  o->engnorm = sc[1];
  o->engsmpl = sc[2];
  o->voffset = sc[3];
  o->voffset_initialized = sc[4] != 0.0;
  return ERMOD_OK;
}

int32_t ermod_engstore(ermod_ctx* ctx, ermod_accum* o, double* avediv) {
  if (!ctx || !o) return ERMOD_ERR_ARG;
  const int rc = ermod_fetch_accum(ctx, o);
  if (rc != ERMOD_OK) return rc;
  const double nrm = o->engnorm;  // engproc.F90:609-628
  if (o->edens) for (int i = 0; i < ctx->ermax; ++i) o->edens[i] /= nrm;
  if (o->ecorr && ctx->d.ecorr) for (size_t i = 0; i < (size_t)ctx->ermax * ctx->ermax; ++i) o->ecorr[i] /= nrm;
  if (o->eself && ctx->p.selfcal) for (int i = 0; i < ctx->esmax; ++i) o->eself[i] /= nrm;
  // soln: aveuv(division, :) = slnuv / engnorm (engproc.F90:622), returned in slnuv
  if (o->slnuv && ctx->p.slttype == ERMOD_SLT_SOLN)
    for (int i = 0; i < ctx->numslv; ++i) o->slnuv[i] = (float)((double)o->slnuv[i] / nrm);
  const double avslf = o->avslf / nrm;
  if (avediv) {
    avediv[0] = o->engnorm / o->engsmpl;
    avediv[1] = ctx->p.slttype == ERMOD_SLT_SOLN ? o->voffset - ctx->p.temp * std::log(avslf)
                                                 : o->voffset + ctx->p.temp * std::log(avslf);
  }
  o->avslf = avslf;
  return ERMOD_OK;
}

int32_t ermod_get_uvengy(ermod_ctx* ctx, double* uvengy, double* uvengy0) {
  if (!ctx) return ERMOD_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  if (uvengy) {
    if (!ctx->d.uvengy) return set_error(ctx, ERMOD_ERR_ARG, "uv_nokeep");
    CK(cudaMemcpy(uvengy, ctx->d.uvengy, sizeof(double) * ctx->maxdst * ctx->slvmax, cudaMemcpyDeviceToHost));
  }
  if (uvengy0) CK(cudaMemcpy(uvengy0, ctx->d.u0, sizeof(double) * ctx->maxdst, cudaMemcpyDeviceToHost));
  return ERMOD_OK;
}

int32_t ermod_get_insertions(ermod_ctx* ctx, float* ins, double* w) {
  if (!ctx) return ERMOD_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  if (ins) {
    std::vector<float4> t((size_t)ctx->maxdst * ctx->s);
    CK(cudaMemcpy(t.data(), ctx->d.tgt_raw, sizeof(float4) * t.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < t.size(); ++i) { ins[3 * i] = t[i].x; ins[3 * i + 1] = t[i].y; ins[3 * i + 2] = t[i].z; }
  }
  if (w) {
    std::vector<float> f(ctx->maxdst);
    CK(cudaMemcpy(f.data(), ctx->d.insw_in, sizeof(float) * ctx->maxdst, cudaMemcpyDeviceToHost));
    for (int i = 0; i < ctx->maxdst; ++i) w[i] = f[i];
  }
  return ERMOD_OK;
}

int32_t ermod_get_sizes(ermod_ctx* ctx, int32_t* slvmax, int32_t* maxdst, int32_t* ns, int32_t* natoms) {
  if (!ctx) return ERMOD_ERR_ARG;
  if (slvmax) *slvmax = ctx->slvmax;
  if (maxdst) *maxdst = ctx->maxdst;
  if (ns) *ns = ctx->s;
  if (natoms) *natoms = ctx->natoms;
  return ERMOD_OK;
}

const char* ermod_last_error(const ermod_ctx* ctx) { return ctx ? ctx->err.c_str() : "null"; }

int32_t ermod_get_timings(const ermod_ctx* ctx, float* ms, int32_t n) {
  if (!ctx || !ms) return ERMOD_ERR_ARG;
  for (int i = 0; i < n && i < kNumTimings; ++i) ms[i] = ctx->timings[i];
  return ERMOD_OK;
}

int64_t ermod_get_launch_count(const ermod_ctx* ctx) { return ctx ? ctx->launches : -1; }

int32_t ermod_proposal_config(ermod_ctx* ctx, int32_t voxels_per_side, int32_t feature_cells, float mix_uniform,
                              const float* params) {
  if (!ctx) return ERMOD_ERR_ARG;
  if (feature_cells == 0) feature_cells = 2 * voxels_per_side;
  if (voxels_per_side < 2 || voxels_per_side > 64 || feature_cells < 4 || feature_cells > 128 ||
      !(mix_uniform > 0.f) || !(mix_uniform <= 1.f))
    return set_error(ctx, ERMOD_ERR_ARG, "prp_arg");
  if (ctx->p.slttype == ERMOD_SLT_SOLN) return set_error(ctx, ERMOD_ERR_ARG, "prp_sln");
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->st));
  DeviceState& d = ctx->d;
  const int gv = voxels_per_side, V = gv * gv * gv, gf = feature_cells;
  if (gv != ctx->prop_gv || gf != ctx->prop_gf) {
    void* old[] = {d.dens, d.feat, d.vact, d.vlogit, d.vcdf, d.vq};
    for (void* q : old) if (q) cudaFree(q);
    d.dens = nullptr; d.feat = nullptr; d.vact = nullptr; d.vlogit = nullptr; d.vcdf = nullptr; d.vq = nullptr;
    CK(dalloc(&d.dens, (size_t)gf * gf * gf));
    CK(dalloc(&d.feat, (size_t)V * kMlpIn));
    CK(dalloc(&d.vact, (size_t)3 * V * kMlpHidden));
    CK(dalloc(&d.vlogit, V));
    CK(dalloc(&d.vcdf, V));
    CK(dalloc(&d.vq, V));
    if (!d.ins_voxel) CK(dalloc(&d.ins_voxel, ctx->maxdst));
    CK(cudaMemsetAsync(d.ins_voxel, 0, sizeof(int) * ctx->maxdst, ctx->st));   // valid voxels before any frame
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; ctx->gkey.clear(); }
  }
  ctx->prop_gv = gv;
  ctx->prop_gf = gf;
  ctx->prop_eps = mix_uniform;
  if (params) {
    const int np = mlp_layout().n;
    if (!d.mlp_f) CK(dalloc(&d.mlp_f, np));
    if (!d.mlp_b) CK(dalloc(&d.mlp_b, np));
    CK(cudaMemcpyAsync(d.mlp_f, params, sizeof(float) * np, cudaMemcpyHostToDevice, ctx->st));
    launch_to_bf16(np, d.mlp_f, d.mlp_b, ctx->st);
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaGetLastError());
    ctx->prop_params = true;
  }
  return ERMOD_OK;
}

int32_t ermod_get_insertion_samples(ermod_ctx* ctx, float* features, double* etot, int32_t* voxel) {
  if (!ctx) return ERMOD_ERR_ARG;
  if (ctx->prop_gv <= 0 || !ctx->d.ins_voxel) return set_error(ctx, ERMOD_ERR_ARG, "prp_set");
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->st));
  DeviceState& d = ctx->d;
  if (features) {
    if (!d.ins_feat) CK(dalloc(&d.ins_feat, (size_t)ctx->maxdst * kMlpIn));
    launch_gather_ins_features(d, ctx->maxdst, d.ins_feat, ctx->st);
    CK(cudaMemcpyAsync(features, d.ins_feat, sizeof(float) * ctx->maxdst * kMlpIn, cudaMemcpyDeviceToHost, ctx->st));
  }
  if (etot) CK(cudaMemcpyAsync(etot, d.etot, sizeof(double) * ctx->maxdst, cudaMemcpyDeviceToHost, ctx->st));
  if (voxel) CK(cudaMemcpyAsync(voxel, d.ins_voxel, sizeof(int) * ctx->maxdst, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaGetLastError());
  return ERMOD_OK;
}

int32_t ermod_get_paths(const ermod_ctx* ctx, int32_t* spectrum_path, int32_t* ecorr_path) {
  if (!ctx) return ERMOD_ERR_ARG;
  if (spectrum_path) *spectrum_path = (ctx->p.cltype == ERMOD_EL_PME || ctx->p.cltype == ERMOD_EL_PPPM) ? ctx->spath : 0;
  if (ecorr_path) *ecorr_path = ctx->p.corrcal ? (ctx->use_tc ? 0 : 1) : -1;
  return ERMOD_OK;
}

void ermod_destroy(ermod_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  free_all(ctx);
  delete ctx;
}

}  // extern "C"
