// engine.cuh -- device buffers of one engine context and the kernel launchers.
#pragma once
#include <cuda_bf16.h>
#include <cufft.h>
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/ermod_b200.h"
#include "common.cuh"

namespace erm {

constexpr int kMaxOrder = 8;       // PME spline order limit (splodr)
constexpr int kMaxSoluteSites = 1024;
constexpr int kMaxLjTypes = 64;
constexpr int kInflBlocks = 64;    // CTAs per target in the influence multiply
constexpr int kEdensSlices = 32;   // target slices of the edens reduction
constexpr int kMaxGrid = 256;      // largest PME grid dimension (x rows are one CTA dimension)
constexpr int kChunk = 32;         // PME solves per chunk: one warp lane per target
// Fused PME solve: k1 planes whose every mode has a Gaussian factor exp(-pi^2 |k|^2 / screen^2)
// below kModeCut are not transformed (their share of any molecule energy is below 1e-9 of the
// k = 0 weight per mode, far under FP32 rounding).
constexpr double kModeCut = 1e-9;
constexpr int kMlpIn = 64;         // proposal network: 4x4x4 local density inputs
constexpr int kMlpHidden = 128;    // width of its three hidden layers

// Offsets of the proposal network's parameters in its FP32 vector.
struct MlpLayout {
  int w1, b1, w2, b2, w3, b3, w4, b4, n;
};

// Everything the frame kernels read, passed by value.
struct FrameArgs {
  CellGeom g;
  PairParams pp;
  int slvmax, natoms, nsite, maxdst;
  int K1, K2, K3, order, Kh1;      // Kh1 = K1/2+1
  int k1max;                       // last k1 plane the fused PME solve transforms (see frame_plan)
  int ljtype_max;
  int pme;
  double pivol;                    // pi / screen^2 / volume (residual terms, engproc.F90:974,994)
  // cell list (cuboid periodic boxes)
  int use_cells, nc[3];
  float ch[3];                     // cell edge lengths
  float rcut;                      // max(elecut, upljcut): beyond it every pair term is zero
};

// Device-resident state of one context.
// Launch `k` on `s`, with programmatic stream serialisation when `pdl` (the
// kernel orders itself against its predecessor with grid_dep_wait()).
template <class... P, class... A>
cudaError_t launch_k(bool pdl, dim3 grid, dim3 block, size_t smem, cudaStream_t s, void (*k)(P...), A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  // the stream's priority as the launch's own, so that a kernel node captured into a graph keeps it
  int prio = 0;
  cudaStreamGetPriority(s, &prio);
  cudaLaunchAttribute at[2];
  int na = 0;
  at[na].id = cudaLaunchAttributePriority;
  at[na++].val.priority = prio;
  if (pdl) {
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na++].val.programmaticStreamSerializationAllowed = 1;
  }
  cfg.attrs = at;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// A kernel's dynamic shared-memory limit is a per-device attribute that every context of
// the process shares: raise it to `bytes` when below, never lower it (a context set up later
// for a smaller solute or mesh must not make an earlier context's launches fail).
cudaError_t raise_smem_limit_fn(const void* kernel, size_t bytes);
template <class F>
cudaError_t raise_smem_limit(F* kernel, size_t bytes) {
  return raise_smem_limit_fn((const void*)kernel, bytes);
}

// Order-4 gather record of one solvent atom, 16 words (64 bytes): the n1 and n2
// B-spline weights, the atom's charge times the n3 weights (FP32 product), and
// {float offset of phi(gd.x) of row (gd.z, gd.y), target 0, in the pair layout;
// flags; gd.x | gd.y << 10 | gd.z << 20; 0}.  kRecWrap: some stencil index wraps;
// kRecWrapX: an n1 index wraps (a stencil row is then not contiguous in n1).
constexpr int kRecWords = 16, kRecWrap = 1, kRecOdd = 2, kRecWrapX = 4;
// records need the offset in 31 bits and each grid index (0..K) in 10
__host__ __device__ __forceinline__ bool gather_rec_ok(int order, int K1, int K2, int K3) {
  return order == 4 && K1 < 1024 && K2 < 1024 && K3 < 1024 &&
         (double)K3 * K2 * (((K1 + 1) / 2) * 2) * 32 < 2147483647.0;
}

// Float offset of phi(n1) of grid line `line` (= n3 K2 + n2) and target b in the
// pair layout: n1 pairs of kChunk targets, P1 = ceil(K1 / 2) pairs per line.
__host__ __device__ __forceinline__ size_t phi_index(size_t line, int n1, int b, int P1) {
  return ((line * P1 + (size_t)(n1 >> 1)) * kChunk + b) * 2 + (n1 & 1);
}

struct DeviceState {
  // topology (physical molecules in tagpt order)
  int* molbeg = nullptr;     // [slvmax+1]
  int* molspec = nullptr;    // [slvmax] uvspec
  float* molq = nullptr;     // [slvmax] mol_charge
  int* atom_lj = nullptr;    // [natoms] ljtype-1
  float* atom_q = nullptr;   // [natoms]
  float* ljene = nullptr;    // [ljtype_max^2]
  float* ljlensq = nullptr;  // [ljtype_max^2]
  // solute site tables
  int* slt_lj = nullptr;     // [s]
  float* slt_q = nullptr;    // [s]
  float* slt_mass = nullptr; // [s]
  float* bfcoord = nullptr;  // [3s]
  // mesh
  double* uvcrd = nullptr;   // [ermax]
  int* spec_off = nullptr;   // [numslv+1]
  int* uvsoft = nullptr;     // [numslv]
  double* escrd = nullptr;   // [esmax]
  // per frame: solvent
  float* posraw = nullptr;   // [3*natoms]
  float4* slvn = nullptr;    // [natoms] normalised x,y,z + charge
  float* spl = nullptr;      // [natoms*3*order]
  int4* grd = nullptr;       // [natoms]
  float* grec = nullptr;     // [natoms*kRecWords] order-4 gather records, on meshes gather_rec_ok allows
  int4* mrec = nullptr;      // [slvmax] {molecule, first atom, atoms, charge bits} in cell order
  float4* anchor = nullptr;  // [slvmax] first-site position, w = molecule extent
  int* cellof = nullptr;     // [slvmax]
  int* cellcount = nullptr;  // [ncell_cap]
  int* cellstart = nullptr;  // [ncell_cap+1]
  int* molsorted = nullptr;  // [slvmax]
  float* rmol = nullptr;     // [1] max molecule extent
  // per frame: targets (insertions or soln solutes)
  float* ins_conf = nullptr; // [3*s*maxdst] staging of caller conformations
  float* insw_in = nullptr;  // [maxdst]
  float4* tgt_raw = nullptr; // [maxdst*s]
  float4* tgt_n = nullptr;   // [maxdst*s] normalised + charge
  float4* tgt_c = nullptr;   // [maxdst] wrapped COM + radius
  int* tgt_mol = nullptr;    // [maxdst] soln: excluded molecule (k index), refs: -1
  double* selfreal = nullptr;// [maxdst]
  double* selfrec = nullptr; // [maxdst]
  double* u0 = nullptr;      // [maxdst] uvengy0
  double* w = nullptr;       // [maxdst] engnmfc
  double* etot = nullptr;    // [maxdst] sum of solute-solvent energies
  double* flceng = nullptr;  // [maxdst*numslv]
  // PME chunk buffers
  float* grid = nullptr;     // [chunk*K^3]
  float2* spec = nullptr;    // [chunk*K3*K2*Kh1]
  float* phin = nullptr;     // [chunk*K^3] potential grids as the C2R writes them
  float* phi = nullptr;      // potential grids, insertion fastest in n1 pairs: float2 (phi(2m), phi(2m+1)) of
                             // line (n3 K2 + n2) and target b at float2 index (line P1 + m) chunk + b,
                             // P1 = ceil(K1 / 2); see phi_index
  float* engfac = nullptr;   // [K3*K2*Kh1]
  float* engfacT = nullptr;  // [Kh1*K3*K2] influence function, k1-major (fused PME solve)
  float2* fft_tw = nullptr;  // [K1+K2+K3+K1/2] FP32 twiddle tables of the fused PME solve
  double2* fft_twd = nullptr;// [K1+K2+K3] FP64 twiddle tables (stencil transforms)
  float2* sitetab = nullptr; // [batch*s*(Kh1 [+K2+K3])] per (target, site) stencil transforms of a batch
  float* sitestn = nullptr;  // [batch*s*(2+2*kMaxOrder)] per (target, site) stencils (plane spreading)
  double* splfc = nullptr;   // [K1+K2+K3]
  double* E = nullptr;       // [batch*slvmax] real-space energies of the batch, target-major
  double* Etot = nullptr;    // [batch*slvmax] total pair energies of the batch, target-major (uvengy layout)
  double* tgtq = nullptr;    // [maxdst] net charge of each target's solute
  double* twt = nullptr;     // [maxdst] total_weight of each target
  int* sbin = nullptr;       // [maxdst] self-energy bin of each target (-1: none)
  long long* gacc = nullptr; // [chunk*K^3] fixed-point spreading box for large solutes
  int4* boxinfo = nullptr;   // [2*chunk] spreading box origin / extent per target
  double* partial = nullptr; // [chunk*kInflBlocks] self-energy partial sums
  unsigned int* done = nullptr; // [chunk] block counters of the self-energy reduction
  double* uvengy = nullptr;  // [maxdst*slvmax] kept when requested
  uint32_t* counts = nullptr;// [batch*ermax_pad]
  // accumulators
  double* edens = nullptr;   // [ermax]
  double* edens_part = nullptr; // [kEdensSlices*ermax] partial sums (NULL: one-pass edens kernel)
  double* ecorr = nullptr;   // [ermax*ermax]
  double* eself = nullptr;   // [esmax]
  double* slnuv = nullptr;   // [numslv]
  float* minuv = nullptr;    // [numslv+1]
  float* maxuv = nullptr;    // [numslv+1]
  double* scal = nullptr;    // [8]: avslf, engnorm, engsmpl, voffset, voffset_init, usreal, usreal_init
  DevStatus* status = nullptr;
  int* frame_i = nullptr;    // [4] per-frame scalars staged before the frame: [0] stnum
  // insertion proposal (refs mode)
  int* dens = nullptr;       // [F^3] solvent first-site counts on the feature grid
  float* feat = nullptr;     // [G^3][64] per-voxel network inputs
  float* mlp_f = nullptr;    // [nparams] network parameters, FP32 (biases are used from here)
  __nv_bfloat16* mlp_b = nullptr;  // [nparams] the same rounded to BF16 (weight matrices)
  float* vact = nullptr;     // [3][G^3][128] hidden activations of the voxels
  float* vlogit = nullptr;   // [G^3]
  double* vcdf = nullptr;    // [G^3] CDF of the proposal over the voxels
  float* vq = nullptr;       // [G^3] proposal probability of each voxel
  int* host_atom = nullptr;  // [nhost] atoms of the host aggregate (insposition 2..4)
  float* host_mass = nullptr;// [nhost]
  double* aggcen = nullptr;  // [3] mass-weighted centre of the host aggregate, this frame
  float* atom_mass = nullptr;// [natoms] (soln region checks: solute centres of mass)
  // RefInfo reference structure (insposition 5, 6)
  int* ref_atom = nullptr;   // [nref] posraw atoms of the refspec molecules, in molecule order
  float* ref_host = nullptr; // [3*nref] their reference coordinates
  float* ref_host_w = nullptr;  // [nref] fit weights
  float* ref_slt = nullptr;  // [3*s] reference solute coordinates
  float* ref_slt_w = nullptr;// [s]
  float* ref_bf = nullptr;   // [3*s] this frame's best-fit reference solute (reffit)
  int* skip = nullptr;       // [maxdst] soln: 1 where check_mol_configuration rejects the solute this frame
  int* ins_voxel = nullptr;  // [maxdst] voxel of each insertion
  float* ins_feat = nullptr; // [maxdst][64] features of each insertion's voxel (training data, on request)
};

// ---- launchers (kernels.cu) -------------------------------------------
void launch_prepare_solvent(const FrameArgs& a, const DeviceState& d, cudaStream_t s);
void launch_cells(const FrameArgs& a, const DeviceState& d, int ncell, cudaStream_t s);
void launch_aggcen(const DeviceState& d, int nhost, cudaStream_t s);
// check_mol_configuration's inputs for solutes in solution (engproc.F90:1197-1295)
struct SolnCheck {
  int insposition;
  float lwreg, upreg;
  int insstructure;
  float lwstr, upstr;
};
void launch_soln_region(const FrameArgs& a, const DeviceState& d, const SolnCheck& ck, cudaStream_t s);
// Insertion geometry of a frame (set_shift_com, insertion.F90:131-304)
struct InsRegion {
  int insposition, insorient;
  float lwreg, upreg;
  float gl[3];      // Gaussian insertion: (|c_k| / 2) / upreg of the first frame
  float z0, z1;     // its mixture normalisations 8 l1 l2 l3 and pi^(3/2) erf(l1) erf(l2) erf(l3)
};
constexpr int kInsTries = 1024;   // configurations an RMSD-window insertion may try (the reference loops on)
void launch_reffit(const DeviceState& d, int nref, int s, cudaStream_t st);
void launch_insert(const FrameArgs& a, const DeviceState& d, const int* stnum_dev, int iseed, const InsRegion& rg,
                   int use_conf, int gv, int learned, cudaStream_t s);
// proposal (proposal.cu) and its network (mlp.cu)
MlpLayout mlp_layout();
void mlp_forward(const __nv_bfloat16* pw, const float* pf, const float* x, int n, float* act, float* logits,
                 int* err, cudaStream_t s);
int mlp_forward_launches();
void launch_to_bf16(int n, const float* src, __nv_bfloat16* dst, cudaStream_t s);
int launch_proposal(const FrameArgs& a, const DeviceState& d, int gv, int gf, float eps, bool learned,
                    cudaStream_t s);
void launch_gather_ins_features(const DeviceState& d, int n, float* out, cudaStream_t s);
void launch_targets_soln(const FrameArgs& a, const DeviceState& d, const int* tgt_k_host_dev, cudaStream_t s);
void launch_selfreal(const FrameArgs& a, const DeviceState& d, int first, int count, double screen,
                     cudaStream_t s);
void launch_real(const FrameArgs& a, const DeviceState& d, int base, int nb, int chunk, int threads, cudaStream_t s);
int setup_real_smem(const FrameArgs& a);
int setup_insert_smem(int nsite);
void launch_fill(float* p, float v, int n, cudaStream_t s);
// Inputs of the PPPM optimal influence function (recpcal.F90:179-337): the alias sums run
// over |n_i| <= mmax[i]; gfb[l] are the coefficients of the order-P assignment function's
// alias sum as a polynomial in sin^2(k h / 2).  on = 0 selects the smooth-PME function.
struct PppmGreen {
  int on;
  int mmax[3];
  double gfb[kMaxOrder];
};
void launch_engfac(const FrameArgs& a, const DeviceState& d, const double invcl[3][3], double volume,
                   double screen, const PppmGreen& pg, cudaStream_t s);
void launch_spread(const FrameArgs& a, const DeviceState& d, int base, int nb, int chunk, cudaStream_t s);
int setup_spread_smem();
void launch_transpose_phi(const FrameArgs& a, const DeviceState& d, cudaStream_t s);
void launch_clear_box(const FrameArgs& a, const DeviceState& d, int chunk, cudaStream_t s);
// fused PME solve (pme_fused.cu)
bool fused_supported(const FrameArgs& a);
int setup_fused(const FrameArgs& a);
void fused_twiddles(int K1, int K2, int K3, std::vector<float2>& tw, std::vector<double2>& twd);
size_t fused_sitetab_elems(const FrameArgs& a, int batch, bool direct);
size_t fused_sitestn_elems(const FrameArgs& a, int batch);
void launch_site_tables(const FrameArgs& a, const DeviceState& d, int bb, int nbatch, bool direct, cudaStream_t s);
void launch_pme_plane(const FrameArgs& a, const DeviceState& d, int tbase, int nb, bool direct, bool pdl,
                      cudaStream_t s);
void launch_pme_rows(const FrameArgs& a, const DeviceState& d, int base, int nb, bool pdl, cudaStream_t s);
void launch_influence(const FrameArgs& a, const DeviceState& d, int base, int nb, int chunk, cudaStream_t s);

struct BinArgs {
  int ermax, ermax_pad, numslv, slttype;
};
void launch_gather(const FrameArgs& a, const DeviceState& d, int base, int bb, int nb, int chunk, int batch,
                   bool pdl, cudaStream_t s);
// Bins a batch's energy rows; where d.E is set, first adds the real-space energies of the
// batch (d.E, molecule-major with leading dimension `batch`) to Etot and writes the sum back.
void launch_bin(const DeviceState& d, const BinArgs& ba, int bb, int nbatch, int slvmax, int batch,
                cudaStream_t s);
int setup_bin_smem(const BinArgs& ba);

struct WeightArgs {
  int slttype, wgtslf, estype, selfcal, numslv, esmax, rigid;
  double temp, npt_factor;  // exp(pi Q^2/(2 a^2 V)/temp) * V for NPT, else 1
  float stat_weight_system;
  double resid_self;        // residual_self_ene of the solute
};
void launch_weights(const DeviceState& d, const WeightArgs& w, int base, int n, cudaStream_t s);
void launch_edens(const DeviceState& d, int base, int n, int ermax, int ermax_pad, int count_base,
                  cudaStream_t s);
void launch_ecorr_simt(const DeviceState& d, int base, int n, int ermax, int ermax_pad, int count_base,
                       cudaStream_t s);

}  // namespace erm
