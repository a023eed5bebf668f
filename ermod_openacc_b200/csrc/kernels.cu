// kernels.cu -- frame kernels of the energy-distribution engine (sm_100a).
//
// Stage map (reference routine each kernel replaces):
//   k_prepare_solvent  normalize_periodic (realcal.F90:859-896) + solvent splines
//                      (recpcal_prepare_solvent / calc_spline_molecule, recpcal.F90:340-357, 504-538)
//   k_anchor / k_cell_*  cell list of solvent molecules (no reference counterpart:
//                      the reference evaluates every site pair, realcal.F90:257-361)
//   k_insert           instslt('proc') for uniform insertion (insertion.F90:38-375)
//   k_selfreal         realcal_self(_refs) in FP64 (realcal.F90:669-771)
//   k_real             realcal_refs / realcal_soln / realcal_bare (realcal.F90:51-666)
//   k_engfac           recpcal_spline_greenfunc (recpcal.F90:121-163)
//   k_engfac_pppm      recpcal_pppm_greenfunc (recpcal.F90:179-337)
//   k_spread           charge spreading of recpcal_prepare_solute(_refs) (recpcal.F90:380-399, 453-473)
//   k_influence        self energy + influence multiply (recpcal.F90:482-497)
//   k_gather_bin       recpcal_energy_refs/soln (recpcal.F90:592-710) + residual_ene(_refs)
//                      (engproc.F90:979-1020) + getiduv / update_histogram counting
//                      (engproc.F90:917-937, 1111-1171), fused
//   k_weights          update_histogram weights and scalar accumulators (engproc.F90:883-915, 939-941)
//   k_edens            edens += engnmfc * insdst (engproc.F90:943-947)
//   k_ecorr_simt       ecorr += engnmfc * insdst insdst^T (engproc.F90:948-962), FP64 reference kernel
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstdio>

#include "bestfit.cuh"
#include <mutex>

#include "engine.cuh"

namespace erm {

// ---------------------------------------------------------------------------
// solvent preparation
// ---------------------------------------------------------------------------
__global__ void k_prepare_solvent(FrameArgs a, const float* __restrict__ posraw, const float* __restrict__ atom_q,
                                  float4* __restrict__ slvn, float* __restrict__ spl, int4* __restrict__ grd,
                                  float* __restrict__ grec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.natoms) return;
  const float x = posraw[3 * i], y = posraw[3 * i + 1], z = posraw[3 * i + 2];
  const CellGeom& g = a.g;
  if (a.pme) {
    float inm[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float f = g.invcl[k][0] * x + g.invcl[k][1] * y + g.invcl[k][2] * z;
      inm[k] = f - floorf(f);
    }
    const int K[3] = {a.K1, a.K2, a.K3};
    int gi[3];
    float wr[3][kMaxOrder];
    for (int m = 0; m < 3; ++m) {
      const float f = inm[m] * (float)K[m];
      const int rci = (int)f;
      spline_weights(f - (float)rci, a.order, wr[m]);
      for (int spi = 0; spi < a.order; ++spi) spl[((size_t)i * 3 + m) * a.order + spi] = wr[m][spi];
      gi[m] = rci;
    }
    grd[i] = make_int4(gi[0], gi[1], gi[2], 0);
    if (grec) {   // order 4 (gather_rec_ok)
      const float q = atom_q[i];
      const bool wrapx = !(gi[0] >= 3 && gi[0] < a.K1);
      const bool wrap = wrapx || !(gi[1] >= 3 && gi[2] >= 3 && gi[1] < a.K2 && gi[2] < a.K3);
      const int P1 = (a.K1 + 1) / 2;
      const int off = wrap ? 0 : (int)phi_index((size_t)gi[2] * a.K2 + gi[1], gi[0], 0, P1);
      float4* r = reinterpret_cast<float4*>(grec + (size_t)i * kRecWords);
      r[0] = make_float4(wr[0][0], wr[0][1], wr[0][2], wr[0][3]);
      r[1] = make_float4(wr[1][0], wr[1][1], wr[1][2], wr[1][3]);
      r[2] = make_float4(q * wr[2][0], q * wr[2][1], q * wr[2][2], q * wr[2][3]);
      r[3] = make_float4(__int_as_float(off),
                         __int_as_float((wrap ? kRecWrap : 0) | (wrapx ? kRecWrapX : 0) | ((gi[0] & 1) ? kRecOdd : 0)),
                         __int_as_float(gi[0] | gi[1] << 10 | gi[2] << 20), 0.f);
    }
  }
  float nx = x, ny = y, nz = z;
  if (g.periodic) {
    if (g.rotated) {
      nx = g.rot[0][0] * x + g.rot[1][0] * y + g.rot[2][0] * z;
      ny = g.rot[0][1] * x + g.rot[1][1] * y + g.rot[2][1] * z;
      nz = g.rot[0][2] * x + g.rot[1][2] * y + g.rot[2][2] * z;
    }
    float f = floorf(g.inv[2] * nz);
    nx -= g.cn[0][2] * f; ny -= g.cn[1][2] * f; nz -= g.cn[2][2] * f;
    f = floorf(g.inv[1] * ny);
    nx -= g.cn[0][1] * f; ny -= g.cn[1][1] * f; nz -= g.cn[2][1] * f;
    f = floorf(g.inv[0] * nx);
    nx -= g.cn[0][0] * f; ny -= g.cn[1][0] * f; nz -= g.cn[2][0] * f;
  }
  slvn[i] = make_float4(nx, ny, nz, atom_q[i]);
}

__global__ void k_fill(float* __restrict__ p, float v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

void launch_fill(float* p, float v, int n, cudaStream_t s) {
  if (n > 0) k_fill<<<(n + 255) / 256, 256, 0, s>>>(p, v, n);
}

void launch_prepare_solvent(const FrameArgs& a, const DeviceState& d, cudaStream_t s) {
  if (a.natoms <= 0) return;
  k_prepare_solvent<<<(a.natoms + 255) / 256, 256, 0, s>>>(a, d.posraw, d.atom_q, d.slvn, d.spl, d.grd,
                                                           a.pme ? d.grec : nullptr);
}

// ---------------------------------------------------------------------------
// cell list of solvent molecules, keyed by the normalised first site
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_coord(float x, float h, int n) {
  int c = (int)floorf(x / h);
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__global__ void k_anchor(FrameArgs a, const int* __restrict__ molbeg, const float4* __restrict__ slvn,
                         float4* __restrict__ anchor, int* __restrict__ cellof, int* __restrict__ cellcount,
                         float* rmol) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.slvmax) return;
  const int b0 = molbeg[k], b1 = molbeg[k + 1];
  const float4 p0 = slvn[b0];
  float ext = 0.0f;
  for (int at = b0 + 1; at < b1; ++at) {
    const float4 q = slvn[at];
    float dx = q.x - p0.x, dy = q.y - p0.y, dz = q.z - p0.z;
    min_image(a.g, dx, dy, dz);
    ext = fmaxf(ext, sqrtf(dx * dx + dy * dy + dz * dz));
  }
  anchor[k] = make_float4(p0.x, p0.y, p0.z, ext);
  atomicMax((int*)rmol, __float_as_int(ext));
  if (a.use_cells) {
    const int cx = cell_coord(p0.x, a.ch[0], a.nc[0]);
    const int cy = cell_coord(p0.y, a.ch[1], a.nc[1]);
    const int cz = cell_coord(p0.z, a.ch[2], a.nc[2]);
    const int cid = (cz * a.nc[1] + cy) * a.nc[0] + cx;
    cellof[k] = cid;
    atomicAdd(&cellcount[cid], 1);
  }
}

// exclusive scan of the cell counts in one block; leaves cellcount = start (fill cursor)
__global__ void k_cell_scan(int ncell, int* __restrict__ cellcount, int* __restrict__ cellstart) {
  __shared__ int part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (ncell + nt - 1) / nt;
  const int lo = t * per, hi = min(ncell, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += cellcount[i];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - s;
  for (int i = lo; i < hi; ++i) {
    const int c = cellcount[i];
    cellstart[i] = run;
    cellcount[i] = run;
    run += c;
  }
  if (t == nt - 1) cellstart[ncell] = part[nt - 1];
}

__global__ void k_cell_fill(int slvmax, const int* __restrict__ cellof, int* __restrict__ cursor,
                            int* __restrict__ molsorted) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= slvmax) return;
  const int pos = atomicAdd(&cursor[cellof[k]], 1);
  molsorted[pos] = k;
}

__global__ void k_iota(int n, int* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = k;
}

// the gather's molecule records in cell order: {molecule, first atom, atoms, charge bits}
__global__ void k_mol_records(int slvmax, const int* __restrict__ molsorted, const int* __restrict__ molbeg,
                              const float* __restrict__ molq, int4* __restrict__ mrec) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= slvmax) return;
  const int k = molsorted[m];
  mrec[m] = make_int4(k, molbeg[k], molbeg[k + 1] - molbeg[k], __float_as_int(molq[k]));
}

void launch_cells(const FrameArgs& a, const DeviceState& d, int ncell, cudaStream_t s) {
  if (a.slvmax <= 0) return;
  cudaMemsetAsync(d.rmol, 0, sizeof(float), s);
  if (a.use_cells) cudaMemsetAsync(d.cellcount, 0, sizeof(int) * ncell, s);
  k_anchor<<<(a.slvmax + 255) / 256, 256, 0, s>>>(a, d.molbeg, d.slvn, d.anchor, d.cellof, d.cellcount, d.rmol);
  if (a.use_cells) {
    k_cell_scan<<<1, 1024, 0, s>>>(ncell, d.cellcount, d.cellstart);
    k_cell_fill<<<(a.slvmax + 255) / 256, 256, 0, s>>>(a.slvmax, d.cellof, d.cellcount, d.molsorted);
  } else {
    k_iota<<<(a.slvmax + 255) / 256, 256, 0, s>>>(a.slvmax, d.molsorted);
  }
  if (a.pme && d.mrec)
    k_mol_records<<<(a.slvmax + 255) / 256, 256, 0, s>>>(a.slvmax, d.molsorted, d.molbeg, d.molq, d.mrec);
}

// ---------------------------------------------------------------------------
// targets: insertions (refs) or solute molecules taken from the frame (soln)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void wrap_point(const CellGeom& g, float& x, float& y, float& z) {
  if (!g.periodic) return;
  float nx = x, ny = y, nz = z;
  if (g.rotated) {
    nx = g.rot[0][0] * x + g.rot[1][0] * y + g.rot[2][0] * z;
    ny = g.rot[0][1] * x + g.rot[1][1] * y + g.rot[2][1] * z;
    nz = g.rot[0][2] * x + g.rot[1][2] * y + g.rot[2][2] * z;
  }
  float f = floorf(g.inv[2] * nz);
  nx -= g.cn[0][2] * f; ny -= g.cn[1][2] * f; nz -= g.cn[2][2] * f;
  f = floorf(g.inv[1] * ny);
  nx -= g.cn[0][1] * f; ny -= g.cn[1][1] * f; nz -= g.cn[2][1] * f;
  f = floorf(g.inv[0] * nx);
  nx -= g.cn[0][0] * f; ny -= g.cn[1][0] * f; nz -= g.cn[2][0] * f;
  x = nx; y = ny; z = nz;
}

// normalised copies + search sphere (centre = first site, radius = max min-image distance)
__device__ void finish_target(const FrameArgs& a, int cnt, float4* __restrict__ raw, float4* __restrict__ nrm,
                              float4* __restrict__ ctr, const float* __restrict__ qsite) {
  const int s = a.nsite;
  for (int i = 0; i < s; ++i) {
    float4 r = raw[i];
    float x = r.x, y = r.y, z = r.z;
    wrap_point(a.g, x, y, z);
    nrm[i] = make_float4(x, y, z, qsite ? qsite[i] : r.w);
  }
  const float4 c = nrm[0];
  float rad = 0.0f;
  for (int i = 1; i < s; ++i) {
    float dx = nrm[i].x - c.x, dy = nrm[i].y - c.y, dz = nrm[i].z - c.z;
    min_image(a.g, dx, dy, dz);
    rad = fmaxf(rad, sqrtf(dx * dx + dy * dy + dz * dz));
  }
  ctr[cnt] = make_float4(c.x, c.y, c.z, rad);
}

// gv > 0: record each insertion's voxel of the G^3 proposal grid; learned: draw
// the voxel from the proposal CDF and scale the insertion's weight by
// p/q = (1/G^3) / q_v (the position inside the voxel stays uniform).
// com_aggregate (insertion.F90:587-614): the mass-weighted centre of the host
// aggregate's atoms as the frame gives them, one block, FP64 sums in a fixed
// order (per thread, then warps, then the block).
constexpr int kAggThreads = 1024;

__global__ void __launch_bounds__(kAggThreads) k_aggcen(int nhost, const int* __restrict__ host_atom,
                                                       const float* __restrict__ host_mass,
                                                       const float* __restrict__ posraw, double* __restrict__ aggcen) {
  __shared__ double red[4][32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};   // m x, m y, m z, m
  for (int i = tid; i < nhost; i += kAggThreads) {
    const int at = host_atom[i];
    const double m = host_mass[i];
    acc[0] += m * posraw[3 * at];
    acc[1] += m * posraw[3 * at + 1];
    acc[2] += m * posraw[3 * at + 2];
    acc[3] += m;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double v = warp_sum(acc[c]);
    if (lane == 0) red[c][warp] = v;
  }
  __syncthreads();
  if (warp == 0) {
    double t[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) t[c] = warp_sum(lane < kAggThreads / 32 ? red[c][lane] : 0.0);
    if (lane == 0)
      for (int c = 0; c < 3; ++c) aggcen[c] = t[3] > 0.0 ? t[c] / t[3] : 0.0;
  }
}

void launch_aggcen(const DeviceState& d, int nhost, cudaStream_t s) {
  k_aggcen<<<1, kAggThreads, 0, s>>>(nhost, d.host_atom, d.host_mass, d.posraw, d.aggcen);
}

// reffit's first step (insertion.F90:658-666, fit_a_rotate_b bestfit.F90:309-336): the reference
// host is fitted onto this frame's host atoms and the reference solute carried along,
// ref_bf = R (ref_slt - c_ref) + c_frame.  One block, FP64 sums in a fixed order (per thread,
// warps, block); the 4x4 eigenproblem and the carried solute on thread 0.
__global__ void __launch_bounds__(kAggThreads) k_reffit(int nref, int s, const int* __restrict__ ref_atom,
                                                       const float* __restrict__ posraw,
                                                       const float* __restrict__ ref_host,
                                                       const float* __restrict__ ref_host_w,
                                                       const float* __restrict__ ref_slt, float* __restrict__ ref_bf) {
  __shared__ double red[9][32];
  __shared__ double cen[7];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto block_sum = [&](double (&v)[9], int nv) {
    for (int c = 0; c < nv; ++c) {
      const double t = warp_sum(v[c]);
      if (lane == 0) red[c][warp] = t;
    }
    __syncthreads();
    if (warp == 0)
      for (int c = 0; c < nv; ++c) {
        const double t = warp_sum(red[c][lane]);
        if (lane == 0) red[c][0] = t;
      }
    __syncthreads();
  };
  // centres: sum w, sum w x_frame, sum w x_ref
  double v[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = tid; i < nref; i += kAggThreads) {
    const double w = ref_host_w[i];
    const int at = ref_atom[i];
    for (int k = 0; k < 3; ++k) {
      v[1 + k] += w * posraw[3 * at + k];
      v[4 + k] += w * ref_host[3 * i + k];
    }
    v[0] += w;
  }
  block_sum(v, 7);
  if (tid == 0)
    for (int c = 0; c < 7; ++c) cen[c] = c == 0 ? red[0][0] : red[c][0] / red[0][0];
  __syncthreads();
  // S[r][c] = sum w (x_ref - c_ref)_r (x_frame - c_frame)_c: the reference (moving) onto the frame
  for (int c = 0; c < 9; ++c) v[c] = 0.0;
  for (int i = tid; i < nref; i += kAggThreads) {
    const double w = ref_host_w[i];
    const int at = ref_atom[i];
    double xr[3], xf[3];
    for (int k = 0; k < 3; ++k) {
      xr[k] = ref_host[3 * i + k] - cen[4 + k];
      xf[k] = posraw[3 * at + k] - cen[1 + k];
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) v[3 * r + c] += w * xr[r] * xf[c];
  }
  block_sum(v, 9);
  if (tid == 0) {
    double S[3][3], q[4];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) S[r][c] = red[3 * r + c][0];
    fit::rotation_from_s(S, q);
    for (int i = 0; i < s; ++i) {
      const double x[3] = {ref_slt[3 * i] - cen[4], ref_slt[3 * i + 1] - cen[5], ref_slt[3 * i + 2] - cen[6]};
      double r[3];
      fit::rotate(q, x, r);
      for (int k = 0; k < 3; ++k) ref_bf[3 * i + k] = (float)(r[k] + cen[1 + k]);
    }
  }
}

void launch_reffit(const DeviceState& d, int nref, int s, cudaStream_t st) {
  k_reffit<<<1, kAggThreads, 0, st>>>(nref, s, d.ref_atom, d.posraw, d.ref_host, d.ref_host_w, d.ref_slt, d.ref_bf);
}

// check_mol_configuration (engproc.F90:1197-1324) for solutes in solution, sphere
// and slab regions: the solute's centre of mass relative to the host aggregate's
// centre (relative_com :1300-1323) must lie in lwreg..upreg, as a distance
// (sphere) or along the third cell vector (slabs, invcl row 3 . dx * |c3|, its
// absolute value for the symmetric slab).  skip[cnt] = 1 rejects solute cnt for
// this frame: engconst skips its update_histogram (engproc.F90:447-450).
__device__ int region_out(const FrameArgs& a, int insposition, float lwreg, float upreg, int k,
                          const int* __restrict__ molbeg, const float* __restrict__ posraw,
                          const float* __restrict__ atom_mass, const double* __restrict__ aggcen);

// check_mol_configuration (engproc.F90:1197-1295) for every solute in solution: the
// insposition window, then the insstructure RMSD window; skip[cnt] = 1 rejects the solute
__global__ void k_soln_region(FrameArgs a, SolnCheck ck, const int* __restrict__ tgt_mol,
                              const int* __restrict__ molbeg, const float* __restrict__ posraw,
                              const float* __restrict__ atom_mass, const double* __restrict__ aggcen,
                              const float* __restrict__ ref_bf, const float* __restrict__ ref_slt,
                              const float* __restrict__ ref_slt_w, int* __restrict__ skip) {
  const int cnt = blockIdx.x * blockDim.x + threadIdx.x;
  if (cnt >= a.maxdst) return;
  const int k = tgt_mol[cnt];
  const int insposition = ck.insposition;
  const float lwreg = ck.lwreg, upreg = ck.upreg;
  const float* xs = posraw + 3 * molbeg[k];
  int out = 0;
  if (insposition == ERMOD_INSPOS_RMSD) {
    // RMSD of the solute to this frame's best-fit reference solute (engproc.F90:1249-1269)
    const double rmsd = fit::rmsd_nofit(a.nsite, ref_bf, xs, ref_slt_w);
    out = ((double)lwreg > rmsd || rmsd > (double)upreg) ? 1 : 0;
  } else if (insposition >= ERMOD_INSPOS_SPHERE && insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC) {
    out = region_out(a, insposition, lwreg, upreg, k, molbeg, posraw, atom_mass, aggcen);
  }
  if (!out && ck.insstructure == ERMOD_INSSTR_RMSD) {
    // the solute's own structure against RefInfo's solute (engproc.F90:1277-1295)
    const double rmsd = fit::rmsd_bestfit(a.nsite, ref_slt, xs, ref_slt_w);
    out = ((double)ck.lwstr > rmsd || rmsd > (double)ck.upstr) ? 1 : 0;
  }
  skip[cnt] = out;
}

// relative_com of solute k against the aggregate centre and the sphere / slab window
// (engproc.F90:1223-1247); 1 when the solute lies outside [lwreg, upreg]
__device__ int region_out(const FrameArgs& a, int insposition, float lwreg, float upreg, int k,
                          const int* __restrict__ molbeg, const float* __restrict__ posraw,
                          const float* __restrict__ atom_mass, const double* __restrict__ aggcen) {
  double c[3] = {0.0, 0.0, 0.0}, msum = 0.0;
  for (int at = molbeg[k]; at < molbeg[k + 1]; ++at) {
    const double m = atom_mass[at];
    for (int q = 0; q < 3; ++q) c[q] += m * posraw[3 * at + q];
    msum += m;
  }
  float dx[3];
  for (int q = 0; q < 3; ++q) dx[q] = (float)(c[q] / msum) - (float)aggcen[q];
  float dist;
  if (insposition == ERMOD_INSPOS_SPHERE) {
    dist = sqrtf(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
  } else {
    const float l3 = sqrtf(a.g.cell[0][2] * a.g.cell[0][2] + a.g.cell[1][2] * a.g.cell[1][2] +
                           a.g.cell[2][2] * a.g.cell[2][2]);
    dist = (a.g.invcl[2][0] * dx[0] + a.g.invcl[2][1] * dx[1] + a.g.invcl[2][2] * dx[2]) * l3;
    if (insposition == ERMOD_INSPOS_SLAB_SYMMETRIC) dist = fabsf(dist);
  }
  return (lwreg > dist || dist > upreg) ? 1 : 0;
}

void launch_soln_region(const FrameArgs& a, const DeviceState& d, const SolnCheck& ck, cudaStream_t s) {
  k_soln_region<<<(a.maxdst + 127) / 128, 128, 0, s>>>(a, ck, d.tgt_mol, d.molbeg, d.posraw, d.atom_mass, d.aggcen,
                                                       d.ref_bf, d.ref_slt, d.ref_slt_w, d.skip);
}

// Solutes of up to kInsSmemSites sites are placed in shared memory (a slice of an odd number of
// float4 per thread, so that the threads' 16-byte accesses fall in distinct banks) and copied out
// once; larger ones are placed in tgt_raw directly.
constexpr int kInsThreads = 128, kInsSmemSites = 32;
__host__ __device__ inline int ins_pitch(int s) { return s | 1; }
size_t insert_smem(int s) { return s <= kInsSmemSites ? sizeof(float4) * kInsThreads * ins_pitch(s) : 0; }

__global__ void __launch_bounds__(kInsThreads) k_insert(FrameArgs a, const int* __restrict__ stnum_dev, int iseed,
                         InsRegion rg,
                         const double* __restrict__ aggcen, const float* __restrict__ ref_bf,
                         const float* __restrict__ ref_slt_w, DevStatus* st,
                         int use_conf, int gv, int learned, const double* __restrict__ cdf,
                         const float* __restrict__ qv, int* __restrict__ ins_voxel, float* __restrict__ insw,
                         const float* __restrict__ conf_all, const float* __restrict__ bfcoord,
                         const float* __restrict__ mass, const float* __restrict__ qsite,
                         float4* __restrict__ tgt_raw, float4* __restrict__ tgt_n, float4* __restrict__ tgt_c) {
  const int cnt = blockIdx.x * blockDim.x + threadIdx.x;
  if (cnt >= a.maxdst) return;
  const int s = a.nsite;
  const int insposition = rg.insposition, insorient = rg.insorient;
  const float lwreg = rg.lwreg, upreg = rg.upreg;
  const int stnum = *stnum_dev;   // staged per frame, so a captured frame graph replays with the new value
  extern __shared__ float4 ins_site[];
  float4* const gout = tgt_raw + (size_t)cnt * s;
  float4* const out = s <= kInsSmemSites ? ins_site + (size_t)threadIdx.x * ins_pitch(s) : gout;
  const float* conf = use_conf ? conf_all + (size_t)3 * s * cnt : bfcoord;
  float msum = 0.0f;
  for (int i = 0; i < s; ++i) {
    out[i] = make_float4(conf[3 * i], conf[3 * i + 1], conf[3 * i + 2], qsite[i]);
    msum += mass[i];
  }
  auto com = [&](float c[3]) {  // center_of_mass (bestfit.F90:252-266)
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int i = 0; i < s; ++i) { sx += out[i].x * mass[i]; sy += out[i].y * mass[i]; sz += out[i].z * mass[i]; }
    c[0] = sx / msum; c[1] = sy / msum; c[2] = sz / msum;
  };
  const uint2 key = make_uint2((uint32_t)iseed, kStreamTag);
  if (insposition == ERMOD_INSPOS_RANDOM) {
    float c[3];
    com(c);  // set_solute_origin: COM to the origin (insertion.F90:116-119)
    for (int i = 0; i < s; ++i) { out[i].x -= c[0]; out[i].y -= c[1]; out[i].z -= c[2]; }
    const uint4 r4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, 0u, 0u), key);
    float r[3] = {u01(r4.x), u01(r4.y), u01(r4.z)};
    if (gv > 0) {
      const int V = gv * gv * gv;
      int v;
      if (learned) {
        const double target = (double)u01(r4.w) * cdf[V - 1];
        int lo = 0, hi = V - 1;   // first v with cdf[v] > target
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (cdf[mid] > target) hi = mid; else lo = mid + 1;
        }
        v = lo;
        const int vv[3] = {v % gv, (v / gv) % gv, v / (gv * gv)};
        for (int m = 0; m < 3; ++m) r[m] = ((float)vv[m] + r[m]) / (float)gv;
        insw[cnt] *= (float)(1.0 / ((double)V * (double)qv[v]));
      } else {
        int vv[3];
        for (int m = 0; m < 3; ++m) vv[m] = min(gv - 1, (int)(r[m] * (float)gv));
        v = (vv[2] * gv + vv[1]) * gv + vv[0];
      }
      ins_voxel[cnt] = v;
    }
    float cm[3];  // com = cell . r (insertion.F90:157-161)
    for (int k = 0; k < 3; ++k) cm[k] = a.g.cell[k][0] * r[0] + a.g.cell[k][1] * r[1] + a.g.cell[k][2] * r[2];
    com(c);
    for (int i = 0; i < s; ++i) {
      out[i].x = (out[i].x - c[0]) + cm[0];
      out[i].y = (out[i].y - c[1]) + cm[1];
      out[i].z = (out[i].z - c[2]) + cm[2];
    }
  }
  if (insposition >= ERMOD_INSPOS_SPHERE && insposition <= ERMOD_INSPOS_SLAB_SYMMETRIC) {
    // set_solute_origin with insorigin 2: COM to the host aggregate centre (insertion.F90:122-124)
    float c[3];
    com(c);
    const float ag[3] = {(float)aggcen[0], (float)aggcen[1], (float)aggcen[2]};
    for (int i = 0; i < s; ++i) {
      out[i].x = (out[i].x - c[0]) + ag[0];
      out[i].y = (out[i].y - c[1]) + ag[1];
      out[i].z = (out[i].z - c[2]) + ag[2];
    }
    // set_shift_com (insertion.F90:164-200)
    const uint4 r4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, 0u, 0u), key);
    float sh[3];
    if (insposition == ERMOD_INSPOS_SPHERE) {
      // radius uniform in volume over lwreg..upreg, direction uniform by rejection in the unit ball
      const float lw3 = lwreg * lwreg * lwreg, up3 = upreg * upreg * upreg;
      const float t = powf(u01(r4.x) * (up3 - lw3) + lw3, 1.0f / 3.0f);
      float r[3] = {1.f, 0.f, 0.f}, nrm = 1.f;
      for (uint32_t att = 1; att <= 64; ++att) {
        const uint4 b4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, att, 2u), key);
        const float x = u01(b4.x) * 2.f - 1.f, y = u01(b4.y) * 2.f - 1.f, z = u01(b4.z) * 2.f - 1.f;
        const float n2 = x * x + y * y + z * z;
        if (0.f < n2 && n2 <= 1.f) {
          r[0] = x; r[1] = y; r[2] = z;
          nrm = sqrtf(n2);
          break;
        }
      }
      for (int k = 0; k < 3; ++k) sh[k] = t * r[k] / nrm;
    } else {
      // slab: random in the cell's first two directions, dz = lwreg..upreg (either sign when symmetric)
      float t = u01(r4.z) * (upreg - lwreg) + lwreg;
      if (insposition == ERMOD_INSPOS_SLAB_SYMMETRIC && u01(r4.w) > 0.5f) t = -t;
      const float l3 = sqrtf(a.g.cell[0][2] * a.g.cell[0][2] + a.g.cell[1][2] * a.g.cell[1][2] +
                             a.g.cell[2][2] * a.g.cell[2][2]);   // celllen(3), engproc.F90:1045
      const float r[3] = {u01(r4.x), u01(r4.y), t / l3};
      for (int k = 0; k < 3; ++k) sh[k] = a.g.cell[k][0] * r[0] + a.g.cell[k][1] * r[1] + a.g.cell[k][2] * r[2];
    }
    for (int i = 0; i < s; ++i) {   // shift_solute_com
      out[i].x += sh[0];
      out[i].y += sh[1];
      out[i].z += sh[2];
    }
  }
  // apply_orientation (insertion.F90:348-369): a random unit quaternion by rejection in the
  // 4-ball, rotation about the centre of mass; counters (cnt, stnum, attempt, tag)
  auto orient = [&](uint32_t tag) {
    float c[3];
    com(c);
    for (int i = 0; i < s; ++i) { out[i].x -= c[0]; out[i].y -= c[1]; out[i].z -= c[2]; }
    float q0 = 1.f, q1 = 0.f, q2 = 0.f, q3 = 0.f;
    for (uint32_t att = 1; att <= 64; ++att) {
      const uint4 r4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, att, tag), key);
      const float t0 = u01(r4.x) * 2.f - 1.f, t1 = u01(r4.y) * 2.f - 1.f;
      const float t2 = u01(r4.z) * 2.f - 1.f, t3 = u01(r4.w) * 2.f - 1.f;
      const float n2 = t0 * t0 + t1 * t1 + t2 * t2 + t3 * t3;
      if (n2 < 1.f) {
        const float nn = sqrtf(n2);
        q0 = t0 / nn; q1 = t1 / nn; q2 = t2 / nn; q3 = t3 / nn;
        break;
      }
    }
    for (int i = 0; i < s; ++i) {  // q (0,v) q* (bestfit.F90:62-74)
      const float v0 = out[i].x, v1 = out[i].y, v2 = out[i].z;
      const float t0 = -(q1 * v0 + q2 * v1 + q3 * v2);
      const float t1 = q2 * v2 - q3 * v1 + q0 * v0;
      const float t2 = q3 * v0 - q1 * v2 + q0 * v1;
      const float t3 = q1 * v1 - q2 * v0 + q0 * v2;
      const float c1 = -q1, c2 = -q2, c3 = -q3;
      out[i].x = (t2 * c3 - t3 * c2 + t0 * c1 + q0 * t1) + c[0];
      out[i].y = (t3 * c1 - t1 * c3 + t0 * c2 + q0 * t2) + c[1];
      out[i].z = (t1 * c2 - t2 * c1 + t0 * c3 + q0 * t3) + c[2];
    }
  };
  if (insposition == ERMOD_INSPOS_RMSD || insposition == ERMOD_INSPOS_GAUSS) {
    // insorigin 3: try configurations until the RMSD to this frame's best-fit reference solute
    // lies in lwreg..upreg (instslt insertion.F90:86-94, check_solute_configuration :617-643)
    float wfac = 1.0f;
    bool ok = false;
    for (int tr = 0; tr < kInsTries && !ok; ++tr) {
      const uint32_t tg = (uint32_t)tr << 8;
      // set_solute_origin / reffit (:646-673): the conformation fitted onto the best-fit reference
      {
        double cr[3] = {0.0, 0.0, 0.0}, ca[3] = {0.0, 0.0, 0.0}, ws = 0.0;
        for (int i = 0; i < s; ++i) {
          const double w = ref_slt_w[i];
          for (int k = 0; k < 3; ++k) { cr[k] += w * ref_bf[3 * i + k]; ca[k] += w * conf[3 * i + k]; }
          ws += w;
        }
        for (int k = 0; k < 3; ++k) { cr[k] /= ws; ca[k] /= ws; }
        double S[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        for (int i = 0; i < s; ++i)
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
              S[r][c] += (double)ref_slt_w[i] * ((double)conf[3 * i + r] - ca[r]) * ((double)ref_bf[3 * i + c] - cr[c]);
        double q[4];
        fit::rotation_from_s(S, q);
        for (int i = 0; i < s; ++i) {
          const double v[3] = {conf[3 * i] - ca[0], conf[3 * i + 1] - ca[1], conf[3 * i + 2] - ca[2]};
          double r[3];
          fit::rotate(q, v, r);
          out[i].x = (float)(r[0] + cr[0]);
          out[i].y = (float)(r[1] + cr[1]);
          out[i].z = (float)(r[2] + cr[2]);
        }
      }
      // set_shift_com (:201-224 RMSD, :225-300 Gaussian)
      float sh[3];
      if (insposition == ERMOD_INSPOS_RMSD) {
        float c[3];
        com(c);
        float maxd = 0.f;
        for (int i = 0; i < s; ++i) {
          const float dx = out[i].x - c[0], dy = out[i].y - c[1], dz = out[i].z - c[2];
          maxd = fmaxf(maxd, dx * dx + dy * dy + dz * dz);
        }
        const float movmax = upreg + 3.0f * sqrtf(maxd);   // margin_factor 3
        const uint4 r4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, tg, 3u), key);
        sh[0] = movmax * (2.f * u01(r4.x) - 1.f);
        sh[1] = movmax * (2.f * u01(r4.y) - 1.f);
        sh[2] = movmax * (2.f * u01(r4.z) - 1.f);
      } else {
        // uniform_gauss_mixture: alternately uniform over +-l and N(0, 1/2) truncated at l, in
        // units of sigma = upreg; the weight divided by the mixture density (WHAM form)
        float sc[3];
        if (((cnt + tr) & 1) == 0) {
          const uint4 r4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, tg, 4u), key);
          const float u[3] = {u01(r4.x), u01(r4.y), u01(r4.z)};
          for (int k = 0; k < 3; ++k) sc[k] = (2.f * u[k] - 1.f) * rg.gl[k];
        } else {
          for (int k = 0; k < 3; ++k) {
            sc[k] = 0.f;
            for (uint32_t att = 1; att <= 64; ++att) {   // Box-Muller pairs, the first inside +-l
              const uint4 r4 = philox4x32_10(make_uint4((uint32_t)cnt, (uint32_t)stnum, tg | att, 5u + k), key);
              const float u1 = fmaxf(u01(r4.x), 1.0e-7f), u2 = u01(r4.y);
              const float r = sqrtf(-2.f * logf(u1)) * cospif(2.f * u2) * 0.70710678f;
              if (fabsf(r) < rg.gl[k]) { sc[k] = r; break; }
            }
          }
        }
        const float sq = sc[0] * sc[0] + sc[1] * sc[1] + sc[2] * sc[2];
        wfac /= 0.5f / rg.z0 + 0.5f * expf(-sq) / rg.z1;
        const float f[3] = {sc[0] / (2.f * rg.gl[0]), sc[1] / (2.f * rg.gl[1]), sc[2] / (2.f * rg.gl[2])};
        for (int k = 0; k < 3; ++k) sh[k] = a.g.cell[k][0] * f[0] + a.g.cell[k][1] * f[1] + a.g.cell[k][2] * f[2];
      }
      for (int i = 0; i < s; ++i) { out[i].x += sh[0]; out[i].y += sh[1]; out[i].z += sh[2]; }
      if (insorient == ERMOD_INSROT_RANDOM) orient(1u | tg);
      double d = 0.0, ws = 0.0;   // rmsd_nofit (bestfit.F90:349-364)
      for (int i = 0; i < s; ++i) {
        const double dx = (double)out[i].x - ref_bf[3 * i], dy = (double)out[i].y - ref_bf[3 * i + 1];
        const double dz = (double)out[i].z - ref_bf[3 * i + 2];
        d += (double)ref_slt_w[i] * (dx * dx + dy * dy + dz * dz);
        ws += ref_slt_w[i];
      }
      const double rmsd = sqrt(d / ws);
      ok = !((double)lwreg > rmsd || rmsd > (double)upreg);
    }
    if (!ok) report(st, kErrInsRej, -1, cnt, 0.f);
    if (insposition == ERMOD_INSPOS_GAUSS) insw[cnt] *= wfac;
  } else if (insorient == ERMOD_INSROT_RANDOM) {
    orient(1u);
  }
  if (out != gout)
    for (int i = 0; i < s; ++i) gout[i] = out[i];
  finish_target(a, cnt, out, tgt_n + (size_t)cnt * s, tgt_c, qsite);
}

int setup_insert_smem(int nsite) {
  return raise_smem_limit(k_insert, insert_smem(nsite)) == cudaSuccess ? 0 : -1;
}

void launch_insert(const FrameArgs& a, const DeviceState& d, const int* stnum_dev, int iseed, const InsRegion& rg,
                   int use_conf, int gv, int learned, cudaStream_t s) {
  k_insert<<<(a.maxdst + kInsThreads - 1) / kInsThreads, kInsThreads, insert_smem(a.nsite), s>>>(
      a, stnum_dev, iseed, rg, d.aggcen, d.ref_bf, d.ref_slt_w, d.status,
                                                    use_conf, gv, learned, d.vcdf, d.vq, d.ins_voxel, d.insw_in,
                                                    d.ins_conf, d.bfcoord, d.slt_mass, d.slt_q, d.tgt_raw, d.tgt_n,
                                                    d.tgt_c);
}

__global__ void k_targets_soln(FrameArgs a, const int* __restrict__ tgt_mol, const int* __restrict__ molbeg,
                               const float* __restrict__ posraw, const float* __restrict__ atom_q,
                               float4* __restrict__ tgt_raw, float4* __restrict__ tgt_n, float4* __restrict__ tgt_c) {
  const int cnt = blockIdx.x * blockDim.x + threadIdx.x;
  if (cnt >= a.maxdst) return;
  const int k = tgt_mol[cnt], b0 = molbeg[k], s = a.nsite;
  float4* out = tgt_raw + (size_t)cnt * s;
  for (int i = 0; i < s; ++i)
    out[i] = make_float4(posraw[3 * (b0 + i)], posraw[3 * (b0 + i) + 1], posraw[3 * (b0 + i) + 2], atom_q[b0 + i]);
  finish_target(a, cnt, out, tgt_n + (size_t)cnt * s, tgt_c, nullptr);
}

void launch_targets_soln(const FrameArgs& a, const DeviceState& d, const int*, cudaStream_t s) {
  k_targets_soln<<<(a.maxdst + 127) / 128, 128, 0, s>>>(a, d.tgt_mol, d.molbeg, d.posraw, d.atom_q, d.tgt_raw,
                                                          d.tgt_n, d.tgt_c);
}

// realcal_self(_refs) (realcal.F90:669-771), FP64 on normalised coordinates
__global__ void k_selfreal(FrameArgs a, int first, double screen, const float4* __restrict__ tgt_n,
                           double* __restrict__ selfreal) {
  const int cnt = first + blockIdx.x;
  const int s = a.nsite;
  const float4* x = tgt_n + (size_t)cnt * s;
  double acc = 0.0;
  const double sqpi = sqrt(kPi);
  for (int i = threadIdx.x; i < s; i += blockDim.x) acc -= (double)x[i].w * (double)x[i].w * screen / sqpi;
  for (int i = 0; i < s; ++i)
    for (int j = i + 1 + threadIdx.x; j < s; j += blockDim.x) {
      float dx = x[i].x - x[j].x, dy = x[i].y - x[j].y, dz = x[i].z - x[j].z;
      if (a.g.cuboid) {
        dx = a.g.half[0] - fabsf(a.g.half[0] - fabsf(dx));
        dy = a.g.half[1] - fabsf(a.g.half[1] - fabsf(dy));
        dz = a.g.half[2] - fabsf(a.g.half[2] - fabsf(dz));
      } else {
        CellGeom g = a.g;
        g.periodic = 1;
        min_image(g, dx, dy, dz);
      }
      const double r = sqrt((double)dx * dx + (double)dy * dy + (double)dz * dz);
      acc -= (double)x[i].w * (double)x[j].w * erf(screen * r) / r;
    }
  __shared__ double red[32];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) selfreal[cnt] = v;
  }
}

void launch_selfreal(const FrameArgs& a, const DeviceState& d, int first, int count, double screen, cudaStream_t s) {
  if (count <= 0) return;
  k_selfreal<<<count, 128, 0, s>>>(a, first, screen, d.tgt_n, d.selfreal);
}

// ---------------------------------------------------------------------------
// real space: one CTA per target, warps over the cells around it
// ---------------------------------------------------------------------------
constexpr int kRealMaxThreads = 512;

// Small solutes: the lanes of a warp test 32 candidate molecules at a time
// against the cutoff sphere and queue those in range (ballot, per-warp queue
// in shared memory); each batch of up to 32 is then evaluated a molecule per
// lane, all its (site, atom) pairs in turn.  WIDE (large solutes): a warp per
// molecule, lanes over the solute sites, the molecule's atoms in turn, and a
// warp-shuffle reduction.  Either way a molecule's energy is one fixed-order
// FP64 sum.  The solute sites, the LJ tables and the queues sit in shared
// memory (dynamic: s float4 + s int + 2 ljmax^2 float + 64 int per warp).
template <bool WIDE>
__global__ void __launch_bounds__(kRealMaxThreads) k_real(FrameArgs a, int base, int chunk,
    const float4* __restrict__ tgt_n, const float4* __restrict__ tgt_c, const int* __restrict__ tgt_mol,
    const int* __restrict__ slt_lj_tab, const int* __restrict__ molbeg, const float4* __restrict__ slvn,
    const int* __restrict__ atom_lj, const float* __restrict__ ljene, const float* __restrict__ ljlensq,
    const float4* __restrict__ anchor, const int* __restrict__ cellstart, const int* __restrict__ molsorted,
    const float* __restrict__ rmol_p, double* __restrict__ E) {
  extern __shared__ __align__(16) unsigned char rsm_real[];
  const int b = blockIdx.x, cnt = base + b, s = a.nsite;
  const int ljmax = a.ljtype_max;
  float4* ss = (float4*)rsm_real;
  int* slj = (int*)(ss + s);
  float* lje = (float*)(slj + s);
  float* ljs = lje + ljmax * ljmax;
  const float4* tn = tgt_n + (size_t)cnt * s;
  for (int i = threadIdx.x; i < s; i += blockDim.x) {
    ss[i] = tn[i];
    slj[i] = slt_lj_tab ? slt_lj_tab[i] : 0;
  }
  for (int i = threadIdx.x; i < ljmax * ljmax; i += blockDim.x) {
    lje[i] = ljene[i];
    ljs[i] = ljlensq[i];
  }
  const int excl = tgt_mol ? tgt_mol[cnt] : -1;
  // soln: solute site LJ types come from the solute molecule's atoms
  if (excl >= 0)
    for (int i = threadIdx.x; i < s; i += blockDim.x) slj[i] = atom_lj[molbeg[excl] + i];
  __syncthreads();
  const float4 c = tgt_c[cnt];
  const float rmol = *rmol_p;
  const float margin = 1.0e-2f;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // pairs beyond rcut (>= elecut and > upljcut) are zero; the slack keeps r == rcut with pair_energy
  const float rskip2 = a.rcut * a.rcut * 1.0001f;

  // candidate k (-1: none) can have a site pair within the cutoff
  auto in_range = [&](int k) {
    if (k < 0 || k == excl) return false;
    const float4 an = anchor[k];
    float dx = an.x - c.x, dy = an.y - c.y, dz = an.z - c.z;
    min_image(a.g, dx, dy, dz);
    const float lim = a.rcut + c.w + an.w + margin;
    return !(dx * dx + dy * dy + dz * dz > lim * lim);
  };
  // WIDE: molecule k by the whole warp, lanes over the solute sites
  auto do_mol = [&](int k) {
    if (!in_range(k)) return;  // every site pair beyond the cutoff
    const int b0 = molbeg[k], nj = molbeg[k + 1] - b0;
    double acc = 0.0;
    for (int js = 0; js < nj; ++js) {
      const float4 xj = slvn[b0 + js];
      const int lj = atom_lj[b0 + js];
      for (int is = lane; is < s; is += 32) {
        const float4 xi = ss[is];
        float ex = xi.x - xj.x, ey = xi.y - xj.y, ez = xi.z - xj.z;
        min_image(a.g, ex, ey, ez);
        const float dis2 = ex * ex + ey * ey + ez * ez;
        if (dis2 > rskip2) continue;
        const int li = slj[is];
        acc += (double)pair_energy(a.pp, dis2, lje[lj * ljmax + li], ljs[lj * ljmax + li], xi.w * xj.w);
      }
    }
    acc = warp_sum(acc);
    if (lane == 0) E[(size_t)b * a.slvmax + k] = acc;
  };

  // the cells around the target (all cells when the range covers the box)
  (void)rmol;
  int lo[3] = {0, 0, 0}, n[3] = {1, 1, 1};
  int total;
  if (a.use_cells) {
    const float R = a.rcut + c.w + rmol + margin;
    const float cc[3] = {c.x, c.y, c.z};
    for (int d3 = 0; d3 < 3; ++d3) {
      lo[d3] = (int)floorf((cc[d3] - R) / a.ch[d3]);
      const int hi = (int)floorf((cc[d3] + R) / a.ch[d3]);
      n[d3] = hi - lo[d3] + 1;
      if (n[d3] >= a.nc[d3]) { lo[d3] = 0; n[d3] = a.nc[d3]; }
    }
    total = n[0] * n[1] * n[2];
  } else {
    total = (a.slvmax + 7) / 8;   // without cells: runs of 8 molecules
  }
  auto cell_id = [&](int t) {
    const int ix = t % n[0], iy = (t / n[0]) % n[1], iz = t / (n[0] * n[1]);
    int cx = (lo[0] + ix) % a.nc[0]; if (cx < 0) cx += a.nc[0];
    int cy = (lo[1] + iy) % a.nc[1]; if (cy < 0) cy += a.nc[1];
    int cz = (lo[2] + iz) % a.nc[2]; if (cz < 0) cz += a.nc[2];
    return (cz * a.nc[1] + cy) * a.nc[0] + cx;
  };

  if (WIDE) {
    for (int t = warp; t < total; t += nw) {
      if (a.use_cells) {
        const int cid = cell_id(t);
        for (int m = cellstart[cid]; m < cellstart[cid + 1]; ++m) do_mol(molsorted[m]);
      } else {
        for (int k = 8 * t; k < min(8 * t + 8, a.slvmax); ++k) do_mol(k);
      }
    }
    return;
  }

  // Small solutes.  Each lane walks its own cells (t = warp * 32 + lane, then every
  // nw * 32-th), so a ballot step tests up to 32 candidates; molecules in range go to
  // the warp's queue, and every batch of up to 32 is evaluated a molecule per lane at the
  // single call site below (one compiled body: a molecule's sum does not depend on which
  // batch it lands in, and the order of molecules within a cell is not fixed).
  int* q = (int*)(ljs + ljmax * ljmax) + warp * 64;   // this warp's queue of molecules in range
  int qn = 0;                                          // queued (warp-uniform)
  int tc = warp * 32 + lane, m = 0, m1 = 0;            // this lane's cell cursor and candidate range
  auto next_cell = [&]() {
    while (m >= m1 && tc < total) {
      if (a.use_cells) {
        const int cid = cell_id(tc);
        m = cellstart[cid];
        m1 = cellstart[cid + 1];
      } else {
        m = 8 * tc;
        m1 = min(m + 8, a.slvmax);
      }
      tc += nw * 32;
    }
  };
  next_cell();
  for (;;) {
    bool more = __any_sync(0xffffffffu, m < m1);
    while (qn < 32 && more) {
      int kl = -1;
      if (m < m1) {
        kl = a.use_cells ? molsorted[m] : m;
        if (++m >= m1) next_cell();
      }
      const bool in = in_range(kl);
      const unsigned bal = __ballot_sync(0xffffffffu, in);
      if (in) q[qn + __popc(bal & ((1u << lane) - 1u))] = kl;
      qn += __popc(bal);
      more = __any_sync(0xffffffffu, m < m1);
    }
    __syncwarp();
    if (qn == 0) break;
    // lanes past the queue's end repeat entry 0 and store nothing
    const int k = q[lane < qn ? lane : 0];
    const int b0 = molbeg[k], nj = molbeg[k + 1] - b0;
    double acc = 0.0;
    for (int is = 0; is < s; ++is) {
      const float4 xi = ss[is];
      const int li = slj[is];
      for (int js = 0; js < nj; ++js) {
        const float4 xj = slvn[b0 + js];
        float ex = xi.x - xj.x, ey = xi.y - xj.y, ez = xi.z - xj.z;
        min_image(a.g, ex, ey, ez);
        const float dis2 = ex * ex + ey * ey + ez * ez;
        if (dis2 > rskip2) continue;
        const int lj = atom_lj[b0 + js];
        acc += (double)pair_energy(a.pp, dis2, lje[lj * ljmax + li], ljs[lj * ljmax + li], xi.w * xj.w);
      }
    }
    if (lane < qn) E[(size_t)b * a.slvmax + k] = acc;
    __syncwarp();
    if (lane < qn - 32) q[lane] = q[32 + lane];
    qn = qn > 32 ? qn - 32 : 0;
    __syncwarp();
  }
}

// Solutes above this many sites run the WIDE real-space variant (a warp per molecule, lanes
// over the sites); up to it, a molecule a lane is faster (measured on ring-recipe solutes of
// 24 to 60 sites in 4096 waters: real space 3.0 -> 2.0 ms at 28 sites, 4.3 -> 2.9 at 40).
constexpr int kRealWideSites = 64;

size_t real_smem(const FrameArgs& a) {
  return (sizeof(float4) + sizeof(int)) * (size_t)a.nsite + 2 * sizeof(float) * (size_t)a.ljtype_max * a.ljtype_max +
         sizeof(int) * 64 * (kRealMaxThreads / 32);
}

int setup_real_smem(const FrameArgs& a) {
  const int b = (int)real_smem(a);
  if (raise_smem_limit(k_real<true>, (size_t)b) != cudaSuccess) return -1;
  if (raise_smem_limit(k_real<false>, (size_t)b) != cudaSuccess) return -1;
  return 0;
}

// `threads` (a multiple of 32, <= kRealMaxThreads) only changes how many warps
// share a target's molecules: each molecule's energy is one warp's fixed-order
// sum whatever the block size.
void launch_real(const FrameArgs& a, const DeviceState& d, int base, int nb, int chunk, int threads, cudaStream_t s) {
  cudaMemsetAsync(d.E, 0, sizeof(double) * (size_t)a.slvmax * chunk, s);
  if (nb <= 0) return;  // `chunk` is the row stride of E: the batch size
  if (threads <= 0 || threads > kRealMaxThreads || threads % 32) threads = 256;
  const size_t sm = real_smem(a);
  // launch_k: a graph node of this launch keeps the stream's (lower) priority beside the PME chain
#define ERM_REAL(W) launch_k(false, nb, threads, sm, s, k_real<W>, a, base, chunk, d.tgt_n, d.tgt_c, d.tgt_mol, \
      d.slt_lj, d.molbeg, d.slvn, d.atom_lj, d.ljene, d.ljlensq, d.anchor, d.cellstart, d.molsorted, d.rmol, d.E)
  if (a.nsite > kRealWideSites) ERM_REAL(true);
  else ERM_REAL(false);
#undef ERM_REAL
}

// ---------------------------------------------------------------------------
// PME
// ---------------------------------------------------------------------------
struct Mat3d { double m[3][3]; };

__global__ void k_engfac(int K1, int K2, int K3, int Kh1, int order, Mat3d invcl, double volume, double screen,
                         const double* __restrict__ splfc, float* __restrict__ engfac,
                         float* __restrict__ engfacT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = K3 * K2 * Kh1;
  if (i >= n) return;
  const int r1 = i % Kh1, r2 = (i / Kh1) % K2, r3 = i / (Kh1 * K2);
  double factor = 0.0;
  if (!(r1 == 0 && r2 == 0 && r3 == 0)) {
    const int rc[3] = {r1, r2, r3}, K[3] = {K1, K2, K3};
    double inm[3];
    bool zero = false;
    for (int m = 0; m < 3; ++m) {
      if ((order % 2 == 1) && (2 * abs(rc[m]) == K[m])) zero = true;
      inm[m] = rc[m] <= K[m] / 2 ? (double)rc[m] : (double)(rc[m] - K[m]);
    }
    if (!zero) {
      double xs[3];
      for (int m = 0; m < 3; ++m) xs[m] = invcl.m[0][m] * inm[0] + invcl.m[1][m] * inm[1] + invcl.m[2][m] * inm[2];
      const double rtp2 = xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2];
      const double chr = kPi * kPi * rtp2 / (screen * screen);
      factor = exp(-chr) / rtp2 / kPi / volume;
      factor /= splfc[r1] * splfc[K1 + r2] * splfc[K1 + K2 + r3];
    }
  }
  engfac[i] = (float)factor;
  if (engfacT) engfacT[((size_t)r1 * K3 + r3) * K2 + r2] = (float)factor;   // [k1][k3][k2] for k_pme_plane
}

// recpcal_pppm_greenfunc (recpcal.F90:217-337): Hockney and Eastwood's optimal influence
// function for the order-P B-spline assignment.  A thread per half-spectrum point sums, over
// the aliases k_n = k + 2 pi invcl^T (n1 K1, n2 K2, n3 K3) with |n_i| <= mmax[i],
// (k . k_n) exp(-|k_n|^2 / 4 screen^2) U^2(k_n) / |k_n|^2, U^2 = prod_i (sin t_i / t_i)^(2P),
// t_i = pi (m_i / K_i + n_i), and divides by k^2, the squared product of the axes' alias
// polynomials sum_l gfb[l] sin^2(pi m_i / K_i)^l and the volume, times 4 pi.  The third
// alias offset is n3 K3 (the reference's :311 uses K2 there).  FP64, stored as FP32 in the
// same two layouts as the smooth-PME function.
__global__ void k_engfac_pppm(int K1, int K2, int K3, int Kh1, int order, Mat3d invcl, double volume,
                              double screen, PppmGreen pg, float* __restrict__ engfac,
                              float* __restrict__ engfacT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = K3 * K2 * Kh1;
  if (i >= n) return;
  const int r1 = i % Kh1, r2 = (i / Kh1) % K2, r3 = i / (Kh1 * K2);
  double factor = 0.0;
  if (!(r1 == 0 && r2 == 0 && r3 == 0)) {
    const int rc[3] = {r1, r2, r3}, K[3] = {K1, K2, K3};
    double inm[3], den = 1.0;
    for (int m = 0; m < 3; ++m) {
      inm[m] = rc[m] <= K[m] / 2 ? (double)rc[m] : (double)(rc[m] - K[m]);
      const double sn = sin(kPi * inm[m] / K[m]), z = sn * sn;
      double poly = 0.0;
      for (int l = order - 1; l >= 0; --l) poly = pg.gfb[l] + poly * z;
      den *= poly;
    }
    den *= den;
    const double tp = 2.0 * kPi;
    double k[3], step[3][3];   // step[m][c]: component c of the alias step 2 pi invcl^T (K_m e_m)
    for (int c = 0; c < 3; ++c) {
      k[c] = tp * (invcl.m[0][c] * inm[0] + invcl.m[1][c] * inm[1] + invcl.m[2][c] * inm[2]);
      for (int m = 0; m < 3; ++m) step[m][c] = tp * invcl.m[m][c] * K[m];
    }
    const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    const double isc2 = 0.25 / (screen * screen);
    auto usq = [&](int m, int nm) {
      const double t = kPi * (inm[m] / K[m] + nm);
      if (t == 0.0) return 1.0;
      const double x = sin(t) / t, x2 = x * x;
      double r = 1.0;
      for (int e = 0; e < order; ++e) r *= x2;
      return r;
    };
    double sum = 0.0;
    for (int nx = -pg.mmax[0]; nx <= pg.mmax[0]; ++nx) {
      const double u1 = usq(0, nx);
      for (int ny = -pg.mmax[1]; ny <= pg.mmax[1]; ++ny) {
        const double u12 = u1 * usq(1, ny);
        for (int nz = -pg.mmax[2]; nz <= pg.mmax[2]; ++nz) {
          const double u = u12 * usq(2, nz);
          double km[3];
          for (int c = 0; c < 3; ++c) km[c] = k[c] + nx * step[0][c] + ny * step[1][c] + nz * step[2][c];
          const double kk = km[0] * km[0] + km[1] * km[1] + km[2] * km[2];
          sum += (k[0] * km[0] + k[1] * km[1] + k[2] * km[2]) * exp(-kk * isc2) * u / kk;
        }
      }
    }
    factor = sum * 4.0 * kPi / (k2 * den) / volume;
  }
  engfac[i] = (float)factor;
  if (engfacT) engfacT[((size_t)r1 * K3 + r3) * K2 + r2] = (float)factor;
}

void launch_engfac(const FrameArgs& a, const DeviceState& d, const double invcl[3][3], double volume, double screen,
                   const PppmGreen& pg, cudaStream_t s) {
  Mat3d m;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) m.m[i][j] = invcl[i][j];
  const int n = a.K3 * a.K2 * a.Kh1;
  if (pg.on)
    k_engfac_pppm<<<(n + 255) / 256, 256, 0, s>>>(a.K1, a.K2, a.K3, a.Kh1, a.order, m, volume, screen, pg,
                                                d.engfac, d.engfacT);
  else
    k_engfac<<<(n + 255) / 256, 256, 0, s>>>(a.K1, a.K2, a.K3, a.Kh1, a.order, m, volume, screen, d.splfc,
                                           d.engfac, d.engfacT);
}

// ---------------------------------------------------------------------------
// Charge spreading, deterministic.  A CTA per target accumulates the
// order^3 stencil of every solute site into a box around the solute as
// 2^-40 fixed-point integers (shared memory, or a global scratch box when
// the solute is large), so the sum does not depend on the order of the
// additions; the box is written into the grid and k_zero_outside clears the
// rest of the grid.  The reference spreads with FP32 atomics in global
// memory (recpcal.F90:453-473), whose sum order varies from run to run.
// ---------------------------------------------------------------------------
constexpr int kSpreadThreads = 256;
constexpr double kFixScale = 1099511627776.0;   // 2^40
constexpr int kSpreadSmemBytes = 96 * 1024;

// calc_spline_molecule_refs for one site (recpcal.F90:553-574)
__device__ __forceinline__ void site_spline(const FrameArgs& a, float4 r, float w[3][kMaxOrder], int gi[3]) {
  const int K[3] = {a.K1, a.K2, a.K3};
  for (int m = 0; m < 3; ++m) {
    float f = a.g.invcl[m][0] * r.x + a.g.invcl[m][1] * r.y + a.g.invcl[m][2] * r.z;
    f = f - floorf(f);
    f = f * (float)K[m];
    const int rci = (int)f;
    spline_weights(f - (float)rci, a.order, w[m]);
    gi[m] = rci;
  }
}

__device__ __forceinline__ int wrap_half(int d, int K) {  // into (-K/2, K/2]
  d = wrapk(wrapk(d, K), K);
  return d > K / 2 ? d - K : d;
}

// Box coordinate of a site along axis m: the wrapped grid index gi lifted onto
// the branch of the unwrapped coordinate floor(K * invcl.x) of the raw (whole,
// unwrapped) solute coordinates, so a solute of any extent up to the grid gets
// a consistent box; lifted indices equal gi modulo K.
__device__ __forceinline__ int lifted_index(const FrameArgs& a, float4 r, int m, int gi) {
  const int K = m == 0 ? a.K1 : (m == 1 ? a.K2 : a.K3);
  const float f = a.g.invcl[m][0] * r.x + a.g.invcl[m][1] * r.y + a.g.invcl[m][2] * r.z;
  const int gu = (int)floorf(f * (float)K);
  const int d = wrap_half(gi - gu, K);  // ~0 up to rounding at a grid line
  return gu + d;
}

__global__ void __launch_bounds__(kSpreadThreads) k_spread_box(FrameArgs a, int base, int nb, int cap,
    const float4* __restrict__ tgt_raw, float* __restrict__ grid, long long* __restrict__ gacc,
    int4* __restrict__ boxinfo, DevStatus* st) {
  extern __shared__ long long sacc[];
  __shared__ int g0[3], lo[3], hi[3];
  const int b = blockIdx.x;
  const size_t KK = (size_t)a.K1 * a.K2 * a.K3;
  if (b >= nb) {  // empty slot of a partial chunk: its grid stays all zero
    if (threadIdx.x == 0) { boxinfo[2 * b] = make_int4(0, 0, 0, 0); boxinfo[2 * b + 1] = make_int4(0, 0, 0, 0); }
    return;
  }
  const int s = a.nsite, n = a.order;
  const float4* sites = tgt_raw + (size_t)(base + b) * s;
  if (threadIdx.x == 0) {
    float w[3][kMaxOrder];
    int gi[3];
    site_spline(a, sites[0], w, gi);
    for (int m = 0; m < 3; ++m) {
      g0[m] = lifted_index(a, sites[0], m, gi[m]);
      lo[m] = 1 << 30;
      hi[m] = -(1 << 30);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < s; t += blockDim.x) {
    float w[3][kMaxOrder];
    int gi[3];
    site_spline(a, sites[t], w, gi);
    for (int m = 0; m < 3; ++m) {
      const int d = lifted_index(a, sites[t], m, gi[m]) - g0[m];
      atomicMin(&lo[m], d - (n - 1));
      atomicMax(&hi[m], d);
    }
  }
  __syncthreads();
  int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1, n2 = hi[2] - lo[2] + 1;
  // a solute whose stencils span more than the grid wraps onto itself: spread
  // over the whole grid with wrapped indices (the reference's modulo)
  const bool full = n0 > a.K1 || n1 > a.K2 || n2 > a.K3;
  if (full) { n0 = a.K1; n1 = a.K2; n2 = a.K3; }
  const int vol = n0 * n1 * n2;
  long long* acc = (!full && vol <= cap) ? sacc : gacc + (size_t)b * KK;
  for (int i = threadIdx.x; i < vol; i += blockDim.x) acc[i] = 0;
  __syncthreads();
  // a warp per site, lanes over the stencil points
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int n3 = n * n * n;
  for (int t = warp; t < s; t += nw) {
    const float4 r = sites[t];
    float w[3][kMaxOrder];
    int gi[3];
    site_spline(a, r, w, gi);
    int d[3];
    for (int m = 0; m < 3; ++m) d[m] = full ? gi[m] : lifted_index(a, r, m, gi[m]) - g0[m] - lo[m];
    for (int p = lane; p < n3; p += 32) {
      const int c1 = p % n, c2 = (p / n) % n, c3 = p / (n * n);
      const float v = r.w * w[0][c1] * w[1][c2] * w[2][c3];   // recpcal.F90:464-465
      const int idx = full ? (wrapk(d[2] - c3, a.K3) * n1 + wrapk(d[1] - c2, a.K2)) * n0 + wrapk(d[0] - c1, a.K1)
                           : ((d[2] - c3) * n1 + (d[1] - c2)) * n0 + (d[0] - c1);
      atomicAdd((unsigned long long*)&acc[idx], (unsigned long long)llrint((double)v * kFixScale));
    }
  }
  __syncthreads();
  float* gb = grid + (size_t)b * KK;
  auto posmod = [](int x, int K) { const int r = x % K; return r < 0 ? r + K : r; };
  const int o0 = full ? 0 : posmod(g0[0] + lo[0], a.K1), o1 = full ? 0 : posmod(g0[1] + lo[1], a.K2),
            o2 = full ? 0 : posmod(g0[2] + lo[2], a.K3);
  for (int i = threadIdx.x; i < vol; i += blockDim.x) {
    const int x = i % n0, y = (i / n0) % n1, z = i / (n0 * n1);
    const int r1 = wrapk(o0 + x, a.K1), r2 = wrapk(o1 + y, a.K2), r3 = wrapk(o2 + z, a.K3);
    gb[((size_t)r3 * a.K2 + r2) * a.K1 + r1] = (float)((double)acc[i] * (1.0 / kFixScale));
  }
  if (threadIdx.x == 0) {
    boxinfo[2 * b] = make_int4(o0, o1, o2, 1);
    boxinfo[2 * b + 1] = make_int4(n0, n1, n2, 0);
  }
}

// After the forward FFT has read the charge grids, put zeros back where the
// boxes were written, so the grids are all zero again for the next chunk
// (the grids are zeroed once at context creation).
__global__ void k_clear_box(FrameArgs a, const int4* __restrict__ boxinfo, float* __restrict__ grid) {
  const int b = blockIdx.x;
  const int4 o = boxinfo[2 * b], ne = boxinfo[2 * b + 1];
  if (!o.w) return;
  float* gb = grid + (size_t)b * a.K1 * a.K2 * a.K3;
  const int vol = ne.x * ne.y * ne.z;
  for (int i = threadIdx.x; i < vol; i += blockDim.x) {
    const int x = i % ne.x, y = (i / ne.x) % ne.y, z = i / (ne.x * ne.y);
    const int r1 = wrapk(o.x + x, a.K1), r2 = wrapk(o.y + y, a.K2), r3 = wrapk(o.z + z, a.K3);
    gb[((size_t)r3 * a.K2 + r2) * a.K1 + r1] = 0.0f;
  }
}

void launch_spread(const FrameArgs& a, const DeviceState& d, int base, int nb, int chunk, cudaStream_t s) {
  k_spread_box<<<chunk, kSpreadThreads, kSpreadSmemBytes, s>>>(a, base, nb, kSpreadSmemBytes / 8, d.tgt_raw, d.grid,
                                                               d.gacc, d.boxinfo, d.status);
}

void launch_clear_box(const FrameArgs& a, const DeviceState& d, int chunk, cudaStream_t s) {
  k_clear_box<<<chunk, 256, 0, s>>>(a, d.boxinfo, d.grid);
}

int setup_spread_smem() { return raise_smem_limit(k_spread_box, (size_t)kSpreadSmemBytes) == cudaSuccess ? 0 : -1; }

// influence multiply + FP64 self energy of each target (recpcal.F90:482-497).
// The self energy is reduced deterministically: per-block partials, summed in
// block order by the last block of each target.
__global__ void k_influence(FrameArgs a, int base, int nb, float2* __restrict__ spec, const float* __restrict__ engfac,
                            double* __restrict__ partial, unsigned int* __restrict__ done,
                            double* __restrict__ selfrec) {
  const int b = blockIdx.y;
  const int n = a.K3 * a.K2 * a.Kh1;
  float2* sp = spec + (size_t)b * n;
  double acc = 0.0;
  const int even = (a.K1 % 2) == 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 v = sp[i];
    const float e = engfac[i];
    const int r1 = i % a.Kh1;
    const double wgt = (r1 == 0 || (even && r1 == a.Kh1 - 1)) ? 0.5 : 1.0;
    acc += wgt * (double)e * ((double)v.x * v.x + (double)v.y * v.y);
    sp[i] = make_float2(v.x * e, v.y * e);
  }
  __shared__ double red[32];
  __shared__ bool last;
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) {
      partial[(size_t)b * gridDim.x + blockIdx.x] = v;
      __threadfence();
      last = atomicAdd(&done[b], 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double sum = 0.0;
    const volatile double* pp = partial + (size_t)b * gridDim.x;
    for (int i = 0; i < (int)gridDim.x; ++i) sum += pp[i];
    if (b < nb) selfrec[base + b] = sum;
    done[b] = 0u;
  }
}

// potential grids [chunk][K^3] (cuFFT's natural C2R output) -> the gather's
// layout: target fastest, n1 in pairs (phi_index)
__global__ void k_transpose_phi(int KK, int K1, const float* __restrict__ in, float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int p0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // (32, 8)
  const int P1 = (K1 + 1) / 2;
#pragma unroll
  for (int j = 0; j < 32; j += 8) {
    const int b = ty + j, p = p0 + tx;
    tile[b][tx] = p < KK ? in[(size_t)b * KK + p] : 0.0f;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 32; j += 8) {
    const int p = p0 + ty + j;
    if (p < KK) out[phi_index((size_t)(p / K1), p % K1, tx, P1)] = tile[tx][ty + j];
  }
}

void launch_transpose_phi(const FrameArgs& a, const DeviceState& d, cudaStream_t s) {
  const int KK = a.K1 * a.K2 * a.K3;
  k_transpose_phi<<<(KK + 31) / 32, dim3(32, 8), 0, s>>>(KK, a.K1, d.phin, d.phi);
}

void launch_influence(const FrameArgs& a, const DeviceState& d, int base, int nb, int chunk, cudaStream_t s) {
  k_influence<<<dim3(kInflBlocks, chunk), 256, 0, s>>>(a, base, nb, d.spec, d.engfac, d.partial, d.done, d.selfrec);
}

// ---------------------------------------------------------------------------
// PME gather + residual.  A warp per solvent molecule, lane = target of the
// chunk (chunk == 32): the potential grid is stored target-fastest, so each
// stencil point is one coalesced 128-byte row.  Writes the reciprocal-space and
// residual energy of every (target, molecule) pair into Etot[target][molecule]
// (the uvengy layout); k_bin adds the real-space energies, so that k_real runs
// beside the whole PME chain.
// ---------------------------------------------------------------------------
constexpr int kGatherThreads = 128;
constexpr int kMaxDevices = 64;     // per-device caches of launch shapes

// The order-4 stencil rows of CS planes c3 (from c30) of one site, no wrap: v[(cs * 4 + c2) * 4 + c1]
// = phi(gd.x - c1) of row (gd.z - c30 - cs, gd.y - c2).  p0 points at phi(gd.x) of the site's row;
// in the pair layout phi(n - 1) is 1 float back when n is odd, 2 * kChunk - 1 back when n is even.
template <int CS, bool ODD>
__device__ __forceinline__ void gather_rows4(const float* __restrict__ p0, size_t s2, size_t s3, int c30,
                                             float (&v)[CS * 16]) {
#pragma unroll
  for (int cs = 0; cs < CS; ++cs)
#pragma unroll
    for (int c2 = 0; c2 < 4; ++c2) {
      const float* r = p0 - (size_t)(c30 + cs) * s3 - (size_t)c2 * s2;
      float* o = v + (cs * 4 + c2) * 4;
      if (ODD) {   // pairs (gd.x-1, gd.x) and (gd.x-3, gd.x-2)
        const float2 a = *(const float2*)(r - 1), c = *(const float2*)(r - 1 - 2 * kChunk);
        o[0] = a.y; o[1] = a.x; o[2] = c.y; o[3] = c.x;
      } else {     // gd.x alone, pair (gd.x-2, gd.x-1), gd.x-3 alone
        const float2 a = *(const float2*)(r - 2 * kChunk);
        o[0] = r[0]; o[1] = a.y; o[2] = a.x; o[3] = r[-4 * kChunk + 1];
      }
    }
}

// The stencil contraction of CS planes c3 (from c30) of one site, separably: along n1 then
// n2 in FP32 (16 points a plane), each plane's q w3 share added to the FP64 energy.
// v[(cs * NO + c2) * NO + c1] = phi(gd.x - c1, gd.y - c2, gd.z - c30 - cs); w = w1 | w2 | w3.
template <int NO, int CS, class W>
__device__ __forceinline__ void accumulate_planes(const float (&v)[CS * NO * NO], const W& w, int c30, float q,
                                                  double& e) {
  float w1[NO], w2[NO];
#pragma unroll
  for (int c = 0; c < NO; ++c) { w1[c] = w[c]; w2[c] = w[NO + c]; }
#pragma unroll
  for (int cs = 0; cs < CS; ++cs) {
    float plane = 0.0f;
#pragma unroll
    for (int c2 = 0; c2 < NO; ++c2) {
      const float* r = v + (cs * NO + c2) * NO;
      float row = w1[0] * r[0];
#pragma unroll
      for (int c1 = 1; c1 < NO; ++c1) row = fmaf(w1[c1], r[c1], row);
      plane = fmaf(w2[c2], row, plane);
    }
    e += (double)(q * w[2 * NO + c30 + cs]) * (double)plane;
  }
}

template <int NO>
__global__ void __launch_bounds__(kGatherThreads, NO > 0 ? 4 : 8) k_gather(FrameArgs a, int base, int bb, int nb,
    int chunk, int batch, const int* __restrict__ molsorted, const int* __restrict__ molbeg,
    const float* __restrict__ molq, const float* __restrict__ atom_q, const float* __restrict__ spl,
    const int4* __restrict__ grd, const float* __restrict__ phi, const double* __restrict__ tgtq,
    const int* __restrict__ tgt_mol, double* __restrict__ Etot) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwt = (gridDim.x * blockDim.x) >> 5;
  const int b = lane;
  const bool active = b < nb;
  const int cnt = base + b, bi = cnt - bb;
  const double qslt = active ? tgtq[cnt] : 0.0;
  const int excl = (active && tgt_mol) ? tgt_mol[cnt] : -1;
  const int n = NO > 0 ? NO : a.order;
  const int K1 = a.K1, K2 = a.K2, K3 = a.K3, P1 = (K1 + 1) / 2;
  grid_dep_wait();                                    // the potential grid of this chunk is complete
  grid_dep_launch();                                  // the next chunk's planes may start filling the tail
  for (int m = gw; m < a.slvmax; m += nwt) {
    const int k = molsorted[m];
    double e = 0.0;
    const int b0 = molbeg[k], b1 = molbeg[k + 1];
    if (a.pme) {
      for (int at = b0; at < b1; ++at) {
        const float q = atom_q[at];
        const float* w = spl + (size_t)at * 3 * n;
        const int4 gd = grd[at];
        if constexpr (NO > 0) {
          // the stencil rows of CS planes c3 in flight at once (one 128-byte row per load):
          // the whole 4^3 stencil for order 4, one 6^2 plane for order 6
          constexpr int CS = NO <= 4 ? NO : 1;
          if constexpr (NO == 4) if (gd.x >= NO - 1 && gd.y >= NO - 1 && gd.z >= NO - 1 && gd.x < K1 &&
                                     gd.y < K2 && gd.z < K3) {
            // no stencil index wraps (most sites): every point is a fixed offset from phi(gd.x) of
            // this target.  The four n1 values gd.x .. gd.x-3 are two whole pairs when gd.x is odd,
            // else one pair and two single values: two or three loads a row instead of four.
            const float* p0 = phi + phi_index((size_t)gd.z * K2 + gd.y, gd.x, b, P1);
            const size_t s2 = (size_t)P1 * kChunk * 2, s3 = (size_t)K2 * s2;   // floats per n2 row, n3 plane
            const bool odd = gd.x & 1;
#pragma unroll
            for (int c30 = 0; c30 < NO; c30 += CS) {
              float v[CS * NO * NO];
              if (odd) gather_rows4<CS, true>(p0, s2, s3, c30, v);
              else gather_rows4<CS, false>(p0, s2, s3, c30, v);
              accumulate_planes<NO, CS>(v, w, c30, q, e);
            }
            continue;
          }
          int r1[NO];
#pragma unroll
          for (int c1 = 0; c1 < NO; ++c1) r1[c1] = (int)phi_index(0, wrapk(gd.x - c1, K1), b, P1);
#pragma unroll
          for (int c30 = 0; c30 < NO; c30 += CS) {
            float v[CS * NO * NO];
#pragma unroll
            for (int cs = 0; cs < CS; ++cs) {
              const int r3 = wrapk(gd.z - (c30 + cs), K3);
#pragma unroll
              for (int c2 = 0; c2 < NO; ++c2) {
                const float* rowp = phi + phi_index((size_t)r3 * K2 + wrapk(gd.y - c2, K2), 0, 0, P1);
#pragma unroll
                for (int c1 = 0; c1 < NO; ++c1) v[(cs * NO + c2) * NO + c1] = rowp[r1[c1]];
              }
            }
            accumulate_planes<NO, CS>(v, w, c30, q, e);
          }
        } else {
          float w1[kMaxOrder];
          int r1[kMaxOrder];
#pragma unroll
          for (int c1 = 0; c1 < kMaxOrder; ++c1)
            if (c1 < n) { w1[c1] = w[c1]; r1[c1] = (int)phi_index(0, wrapk(gd.x - c1, K1), b, P1); }
          for (int c3 = 0; c3 < n; ++c3) {
            const int r3 = wrapk(gd.z - c3, K3);
            const float fac1 = q * w[2 * n + c3];
            for (int c2 = 0; c2 < n; ++c2) {
              const int r2 = wrapk(gd.y - c2, K2);
              const float fac2 = fac1 * w[n + c2];
              const float* rowp = phi + phi_index((size_t)r3 * K2 + r2, 0, 0, P1);
              float part = 0.0f;
#pragma unroll
              for (int c1 = 0; c1 < kMaxOrder; ++c1)
                if (c1 < n) part += (fac2 * w1[c1]) * rowp[r1[c1]];
              e += (double)part;
            }
          }
        }
      }
      e -= a.pivol * qslt * (double)molq[k];
    }
    if (active) Etot[(size_t)bi * a.slvmax + k] = (k == excl) ? 0.0 : e;
  }
}

// The order-4 gather from per-atom records (k_prepare_solvent) and per-molecule records in
// cell order (k_mol_records): the same stencil sums as k_gather<4>, in the same order, with
// fewer dependent loads.  A warp's first molecule record and the records of its first two
// atoms are fetched before the wait on the k1 transform (they are frame tables, complete
// before the chunk chain starts); lanes 0-15 hold one atom's record, lanes 16-31 the next
// one's, and every record is broadcast from there by shuffles.  The records of the next
// two atoms (or of the next molecule's first two) are in flight while the current ones'
// stencils are summed.
// LK1, LK2 > 0: the mesh's K1 = 2^LK1, K2 = 2^LK2 at compile time, so that every stencil row
// is the site's base pointer plus a constant offset; 0: taken from FrameArgs.
template <int LK1, int LK2>
__global__ void __launch_bounds__(kGatherThreads, 4) k_gather_rec(FrameArgs a, int base, int bb, int nb,
    const int4* __restrict__ mrec, const float* __restrict__ grec, const float* __restrict__ phi,
    const double* __restrict__ tgtq, const int* __restrict__ tgt_mol, double* __restrict__ Etot) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwt = (gridDim.x * blockDim.x) >> 5;
  const int b = lane;
  const bool active = b < nb;
  const int cnt = base + b, bi = cnt - bb;
  const double qslt = active ? tgtq[cnt] : 0.0;
  const int excl = (active && tgt_mol) ? tgt_mol[cnt] : -1;
  const int K1 = LK1 ? 1 << LK1 : a.K1, K2 = LK2 ? 1 << LK2 : a.K2, K3 = a.K3, P1 = (K1 + 1) / 2;
  const size_t s2 = (size_t)P1 * kChunk * 2, s3 = (size_t)K2 * s2;   // floats per n2 row, n3 plane
  const int half = lane >> 4, word = lane & 15;
  int m = gw;
  int4 mr = m < a.slvmax ? mrec[m] : make_int4(0, 0, 0, 0);
  float rv = half < mr.z ? grec[(size_t)(mr.y + half) * kRecWords + word] : 0.f;
  grid_dep_wait();                                    // the potential grid of this chunk is complete
  grid_dep_launch();                                  // the next chunk's planes may start filling the tail
  while (m < a.slvmax) {
    const int mn = m + nwt;
    const int4 mrn = mn < a.slvmax ? mrec[mn] : make_int4(0, 0, 0, 0);
    double e = 0.0;
    if (mr.z <= 0) rv = half < mrn.z ? grec[(size_t)(mrn.y + half) * kRecWords + word] : 0.f;
    for (int p = 0; p < mr.z; p += 2) {
      // the records after this pair: atoms p + 2, p + 3, or the next molecule's first two
      float nxt;
      if (p + 2 < mr.z) nxt = p + 2 + half < mr.z ? grec[(size_t)(mr.y + p + 2 + half) * kRecWords + word] : 0.f;
      else nxt = half < mrn.z ? grec[(size_t)(mrn.y + half) * kRecWords + word] : 0.f;
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        if (p + h >= mr.z) break;
        const int src = h * 16;
        float wl[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) wl[c] = __shfl_sync(0xffffffffu, rv, src + c);
        const int off = __float_as_int(__shfl_sync(0xffffffffu, rv, src + 12));
        const int flags = __float_as_int(__shfl_sync(0xffffffffu, rv, src + 13));
        float v[64];
        if (!(flags & kRecWrap)) {
          const float* p0 = phi + (size_t)off + 2 * b;
          if (flags & kRecOdd) gather_rows4<4, true>(p0, s2, s3, 0, v);
          else gather_rows4<4, false>(p0, s2, s3, 0, v);
        } else if (!(flags & kRecWrapX)) {
          // only n2 or n3 wraps: each row is contiguous in n1, loaded in pairs as above
          const int gp = __float_as_int(__shfl_sync(0xffffffffu, rv, src + 14));
          const int gx = gp & 1023, gy = (gp >> 10) & 1023, gz = gp >> 20;
          const bool odd = flags & kRecOdd;
#pragma unroll
          for (int cs = 0; cs < 4; ++cs) {
            const int r3 = wrapk(gz - cs, K3);
#pragma unroll
            for (int c2 = 0; c2 < 4; ++c2) {
              const float* r = phi + phi_index((size_t)r3 * K2 + wrapk(gy - c2, K2), gx, b, P1);
              float* o = v + (cs * 4 + c2) * 4;
              if (odd) {   // pairs (gx-1, gx) and (gx-3, gx-2)
                const float2 p = *(const float2*)(r - 1), q = *(const float2*)(r - 1 - 2 * kChunk);
                o[0] = p.y; o[1] = p.x; o[2] = q.y; o[3] = q.x;
              } else {     // gx alone, pair (gx-2, gx-1), gx-3 alone
                const float2 p = *(const float2*)(r - 2 * kChunk);
                o[0] = r[0]; o[1] = p.y; o[2] = p.x; o[3] = r[-4 * kChunk + 1];
              }
            }
          }
        } else {
          const int gp = __float_as_int(__shfl_sync(0xffffffffu, rv, src + 14));
          const int gx = gp & 1023, gy = (gp >> 10) & 1023, gz = gp >> 20;
          int r1[4];
#pragma unroll
          for (int c1 = 0; c1 < 4; ++c1) r1[c1] = (int)phi_index(0, wrapk(gx - c1, K1), b, P1);
#pragma unroll
          for (int cs = 0; cs < 4; ++cs) {
            const int r3 = wrapk(gz - cs, K3);
#pragma unroll
            for (int c2 = 0; c2 < 4; ++c2) {
              const float* rowp = phi + phi_index((size_t)r3 * K2 + wrapk(gy - c2, K2), 0, 0, P1);
#pragma unroll
              for (int c1 = 0; c1 < 4; ++c1) v[(cs * 4 + c2) * 4 + c1] = rowp[r1[c1]];
            }
          }
        }
        // wl[8 + c3] is q w3(c3), formed in FP32 as k_gather<4> forms it; times 1.0f it stays exact
        accumulate_planes<4, 4>(v, wl, 0, 1.0f, e);
      }
      rv = nxt;
    }
    e -= a.pivol * qslt * (double)__int_as_float(mr.w);
    if (active) Etot[(size_t)bi * a.slvmax + mr.x] = (mr.x == excl) ? 0.0 : e;
    mr = mrn;
    m = mn;
  }
}

void launch_gather(const FrameArgs& a, const DeviceState& d, int base, int bb, int nb, int chunk, int batch,
                   bool pdl, cudaStream_t s) {
  int blocks = (a.slvmax * 32 + kGatherThreads - 1) / kGatherThreads;
  if (a.pme && a.order == 4 && d.grec) {
    // no more CTAs than are resident at once: every warp fetches its first records early
    static std::atomic<int> resident[kMaxDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    int cap = dev >= 0 && dev < kMaxDevices ? resident[dev].load() : 0;
    if (cap == 0) {
      int per_sm = 0, sms = 0;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather_rec<0, 0>, kGatherThreads, 0);
      cap = std::max(1, per_sm * sms);
      if (dev >= 0 && dev < kMaxDevices) resident[dev].store(cap);
    }
    blocks = std::max(1, std::min(blocks, cap));
#define ERM_GATHER_REC(L1, L2) launch_k(pdl, blocks, kGatherThreads, 0, s, k_gather_rec<L1, L2>, a, base, bb, nb, \
      (const int4*)d.mrec, (const float*)d.grec, (const float*)d.phi, (const double*)d.tgtq, (const int*)d.tgt_mol, \
      d.Etot)
    if (a.K1 == 64 && a.K2 == 64) ERM_GATHER_REC(6, 6);
    else if (a.K1 == 32 && a.K2 == 32) ERM_GATHER_REC(5, 5);
    else if (a.K1 == 128 && a.K2 == 128) ERM_GATHER_REC(7, 7);
    else ERM_GATHER_REC(0, 0);
#undef ERM_GATHER_REC
    return;
  }
  if (blocks > 148 * 2048 / kGatherThreads) blocks = 148 * 2048 / kGatherThreads;   // 2048 threads an SM
  if (blocks < 1) blocks = 1;
#define ERM_GATHER(NO) launch_k(pdl, blocks, kGatherThreads, 0, s, k_gather<NO>, a, base, bb, nb, chunk, batch, \
      (const int*)d.molsorted, (const int*)d.molbeg, (const float*)d.molq, (const float*)d.atom_q,         \
      (const float*)d.spl, (const int4*)d.grd, (const float*)d.phi, (const double*)d.tgtq,                  \
      (const int*)d.tgt_mol, d.Etot)
  if (a.pme && a.order == 4) ERM_GATHER(4);
  else if (a.pme && a.order == 6) ERM_GATHER(6);
  else ERM_GATHER(0);
#undef ERM_GATHER
}

// ---------------------------------------------------------------------------
// binning: a CTA per target, the molecule energies of its row binned into a
// shared-memory histogram (getiduv, engproc.F90:1111-1171; insdst,
// :917-937), written out as that target's count row.
// ---------------------------------------------------------------------------
constexpr int kBinThreads = 256;
constexpr int kMaxSpecSmem = 128;

__global__ void __launch_bounds__(kBinThreads) k_bin(BinArgs ba, int bb, int slvmax, double* __restrict__ Etot,
    const double* __restrict__ Ereal, bool keep_total,
    const int* __restrict__ molspec, const int* __restrict__ spec_off, const double* __restrict__ uvcrd,
    const int* __restrict__ uvsoft, const int* __restrict__ tgt_mol, const int* __restrict__ skip,
    uint32_t* __restrict__ counts, double* __restrict__ etot, double* __restrict__ flceng, float* __restrict__ minuv,
    float* __restrict__ maxuv, DevStatus* st) {
  extern __shared__ unsigned char smem_raw[];
  double* mesh = (double*)smem_raw;                                  // [ermax]
  uint32_t* hist = (uint32_t*)(mesh + ba.ermax);                     // [ermax_pad]
  __shared__ float smin[kMaxSpecSmem], smax[kMaxSpecSmem];
  __shared__ double sfl[kMaxSpecSmem];
  __shared__ double red[32];
  const int bi = blockIdx.x, cnt = bb + bi;
  if (skip && skip[cnt]) {
    // a solute rejected by check_mol_configuration: no energies, no counts (engproc.F90:447-450, 755)
    for (int i = threadIdx.x; i < ba.ermax_pad; i += blockDim.x) counts[(size_t)bi * ba.ermax_pad + i] = 0u;
    for (int k = threadIdx.x; k < slvmax; k += blockDim.x) Etot[(size_t)bi * slvmax + k] = 0.0;
    for (int q = threadIdx.x; q < ba.numslv; q += blockDim.x) flceng[(size_t)cnt * ba.numslv + q] = 0.0;
    if (threadIdx.x == 0) etot[cnt] = 0.0;
    return;
  }
  for (int i = threadIdx.x; i < ba.ermax; i += blockDim.x) mesh[i] = uvcrd[i];
  for (int i = threadIdx.x; i < ba.ermax_pad; i += blockDim.x) hist[i] = 0u;
  for (int i = threadIdx.x; i < kMaxSpecSmem; i += blockDim.x) { smin[i] = FLT_MAX; smax[i] = -FLT_MAX; sfl[i] = 0.0; }
  __syncthreads();
  const int excl = tgt_mol ? tgt_mol[cnt] : -1;
  double* row = Etot + (size_t)bi * slvmax;
  const double* rrow = Ereal ? Ereal + (size_t)bi * slvmax : nullptr;
  double acc = 0.0;
  // a thread's running minimum and maximum of its current species (exact, order-free), flushed
  // to shared memory when the species changes: one atomic pair per run instead of per molecule
  int run_sp = 0;
  float run_min = FLT_MAX, run_max = -FLT_MAX;
  auto flush_run = [&]() {
    if (run_sp > 0 && run_sp < kMaxSpecSmem) {
      atomic_min_f(&smin[run_sp], run_min);
      atomic_max_f(&smax[run_sp], run_max);
    }
    run_min = FLT_MAX;
    run_max = -FLT_MAX;
  };
  for (int k = threadIdx.x; k < slvmax; k += blockDim.x) {
    if (k == excl) continue;
    double e = row[k];
    if (rrow) {   // the real-space energy of the pair, added to the reciprocal part
      e += rrow[k];
      if (keep_total) row[k] = e;
    }
    const int pti = molspec[k];
    if (pti <= 0) { report(st, kErrEngCns, k, cnt, (float)e); continue; }
    const int lo = spec_off[pti - 1], num = spec_off[pti] - lo;
    const double* c = mesh + lo;
    int idp;
    if (e < c[0]) idp = 0;
    else if (e > c[num - 1]) idp = num;
    else {
      int l = 0, h = num;  // first index with c[i] >= e
      while (l < h) { const int mid = (l + h) >> 1; if (c[mid] < e) l = mid + 1; else h = mid; }
      idp = l;
    }
    if (idp <= 0) { report(st, kErrEngMin, k, cnt, (float)e); continue; }
    if (ba.slttype == ERMOD_SLT_SOLN && idp > uvsoft[pti - 1]) { report(st, kErrEngSft, k, cnt, (float)e); continue; }
    if (idp == num && e < 1.0e3) report(st, kWarnMbin, k, cnt, (float)e);
    atomicAdd(&hist[lo + idp - 1], 1u);
    acc += e;
    const float ef = (float)e;
    if (pti < kMaxSpecSmem) {
      if (pti != run_sp) {
        flush_run();
        run_sp = pti;
      }
      run_min = fminf(run_min, ef);
      run_max = fmaxf(run_max, ef);
      if (ba.slttype == ERMOD_SLT_SOLN) atomicAdd(&sfl[pti], e);
    } else {
      atomic_min_f(&minuv[pti], ef);
      atomic_max_f(&maxuv[pti], ef);
      if (ba.slttype == ERMOD_SLT_SOLN) atomicAdd(&flceng[(size_t)cnt * ba.numslv + pti - 1], e);
    }
  }
  flush_run();
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  uint32_t* crow = counts + (size_t)bi * ba.ermax_pad;
  for (int i = threadIdx.x; i < ba.ermax_pad; i += blockDim.x) crow[i] = hist[i];
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) etot[cnt] = v;
  }
  for (int i = threadIdx.x + 1; i < kMaxSpecSmem && i <= ba.numslv; i += blockDim.x) {
    if (smin[i] != FLT_MAX) atomic_min_f(&minuv[i], smin[i]);
    if (smax[i] != -FLT_MAX) atomic_max_f(&maxuv[i], smax[i]);
    if (ba.slttype == ERMOD_SLT_SOLN) flceng[(size_t)cnt * ba.numslv + i - 1] = sfl[i];
  }
}

size_t bin_smem_bytes(const BinArgs& ba) { return sizeof(double) * ba.ermax + sizeof(uint32_t) * ba.ermax_pad; }

void launch_bin(const DeviceState& d, const BinArgs& ba, int bb, int nbatch, int slvmax, int batch,
                cudaStream_t s) {
  if (nbatch <= 0) return;
  // the summed energies go back to Etot only when the per-molecule energies are kept (uvengy)
  k_bin<<<nbatch, kBinThreads, bin_smem_bytes(ba), s>>>(ba, bb, slvmax, d.Etot, d.E, d.uvengy != nullptr, d.molspec,
                                                        d.spec_off,
                                                        d.uvcrd,
                                                        d.uvsoft, d.tgt_mol, d.skip, d.counts, d.etot, d.flceng,
                                                        d.minuv, d.maxuv, d.status);
}

// Shared by every context and the allocation-free entry point: only ever raised.
int setup_bin_smem(const BinArgs& ba) {
  const size_t b = bin_smem_bytes(ba);
  if (b > 200 * 1024) return -1;
  return raise_smem_limit(k_bin, b) == cudaSuccess ? 0 : -1;
}

namespace {
std::mutex g_smem_limit_mu;   // concurrent context set-ups must not interleave get and set
}

cudaError_t raise_smem_limit_fn(const void* kernel, size_t bytes) {
  std::lock_guard<std::mutex> lk(g_smem_limit_mu);
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---------------------------------------------------------------------------
// weights and accumulators
// ---------------------------------------------------------------------------
__global__ void k_offset_init(WeightArgs wa, int base, int n, const int* __restrict__ skip,
                              const double* __restrict__ selfrec, const double* __restrict__ selfreal,
                              double* __restrict__ scal) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int c = base;   // the first target not rejected (engproc.F90:447-450)
  if (skip) while (c < base + n && skip[c]) ++c;
  if (c >= base + n) return;
  if (wa.rigid && scal[6] == 0.0) { scal[5] = selfreal[c]; scal[6] = 1.0; }
  if (wa.wgtslf && scal[4] == 0.0) {
    const double sr = wa.rigid ? scal[5] : selfreal[c];
    scal[3] = selfrec[c] + sr + wa.resid_self;
    scal[4] = 1.0;
  }
}

// per-target weight engnmfc (engproc.F90:883-903, volcorrect :1022-1038)
__global__ void k_weights(WeightArgs wa, int base, int n, const int* __restrict__ skip,
                          const double* __restrict__ selfrec, const double* __restrict__ selfreal,
                          const float* __restrict__ insw,
                          const double* __restrict__ escrd, double* __restrict__ u0, double* __restrict__ w,
                          double* __restrict__ twt, int* __restrict__ sbin, const double* __restrict__ scal,
                          DevStatus* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const int cnt = base + i;
    double tw;
    const double sr = wa.rigid ? scal[5] : selfreal[cnt];
    const double uu = selfrec[cnt] + sr + wa.resid_self;
    u0[cnt] = uu;
    double e = 1.0;
    if (wa.wgtslf) {
      const double f = uu - scal[3];
      e = wa.slttype == ERMOD_SLT_SOLN ? exp(f / wa.temp) : exp(-f / wa.temp);
    }
    tw = (double)wa.stat_weight_system * (double)insw[cnt] * wa.npt_factor;
    e *= tw;
    const bool rej = skip && skip[cnt];   // rejected: no update_histogram (engproc.F90:447-450)
    w[cnt] = rej ? 0.0 : e;
    twt[cnt] = rej ? 0.0 : tw;
    int l = -1;
    if (wa.selfcal && !rej) {  // getiduv(0, uvengy0) (engproc.F90:910-913)
      int lo = 0, h = wa.esmax;
      if (uu < escrd[0]) lo = 0;
      else if (uu > escrd[wa.esmax - 1]) lo = wa.esmax;
      else { while (lo < h) { const int mid = (lo + h) >> 1; if (escrd[mid] < uu) lo = mid + 1; else h = mid; } }
      if (lo <= 0) report(st, kErrEngMin, -1, cnt, (float)uu);
      else {
        if (lo == wa.esmax && uu < 1.0e3) report(st, kWarnMbin, -1, cnt, (float)uu);
        l = lo - 1;
      }
    }
    sbin[cnt] = l;
  }
}

// Scalar accumulators of one batch, summed in a fixed order by one CTA
// (engproc.F90:905-915, 939-941): engnorm, engsmpl, avslf, the self-energy
// histogram, slnuv (soln) and the self-energy min / max.
constexpr int kSumThreads = 1024;

__global__ void __launch_bounds__(kSumThreads) k_wsum(WeightArgs wa, int base, int n, const int* __restrict__ skip,
    const double* __restrict__ w, const double* __restrict__ twt, const double* __restrict__ u0,
    const int* __restrict__ sbin,
    const double* __restrict__ flceng, double* __restrict__ scal, double* __restrict__ eself,
    double* __restrict__ slnuv, float* __restrict__ minuv, float* __restrict__ maxuv) {
  __shared__ double r0[32], r1[32];
  __shared__ float rm[32], rx[32];
  __shared__ int rk[32];
  double a0 = 0.0, a1 = 0.0;
  float mn = FLT_MAX, mx = -FLT_MAX;
  int kept = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (skip && skip[base + i]) continue;
    a0 += w[base + i];
    a1 += twt[base + i];
    const float u = (float)u0[base + i];
    mn = fminf(mn, u);
    mx = fmaxf(mx, u);
    ++kept;
  }
  a0 = warp_sum(a0); a1 = warp_sum(a1); mn = warp_min(mn); mx = warp_max(mx);
  for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
  if ((threadIdx.x & 31) == 0) {
    r0[threadIdx.x >> 5] = a0; r1[threadIdx.x >> 5] = a1; rm[threadIdx.x >> 5] = mn; rx[threadIdx.x >> 5] = mx;
    rk[threadIdx.x >> 5] = kept;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool ok = threadIdx.x < (blockDim.x >> 5);
    a0 = warp_sum(ok ? r0[threadIdx.x] : 0.0);
    a1 = warp_sum(ok ? r1[threadIdx.x] : 0.0);
    mn = warp_min(ok ? rm[threadIdx.x] : FLT_MAX);
    mx = warp_max(ok ? rx[threadIdx.x] : -FLT_MAX);
    kept = ok ? rk[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
    if (threadIdx.x == 0) {
      scal[1] += a0;
      scal[2] += (double)kept;
      scal[0] += a1;
      minuv[0] = fminf(minuv[0], mn);
      maxuv[0] = fmaxf(maxuv[0], mx);
      if (wa.slttype == ERMOD_SLT_SOLN)
        for (int q = 0; q < wa.numslv; ++q) {
          double sq = 0.0;
          for (int i = 0; i < n; ++i) sq += flceng[(size_t)(base + i) * wa.numslv + q] * w[base + i];
          slnuv[q] += sq;
        }
    }
  }
  if (wa.selfcal)
    for (int bin = threadIdx.x; bin < wa.esmax; bin += blockDim.x) {
      double sb = 0.0;
      for (int i = 0; i < n; ++i)
        if (sbin[base + i] == bin) sb += w[base + i];
      eself[bin] += sb;
    }
}

void launch_weights(const DeviceState& d, const WeightArgs& wa, int base, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_offset_init<<<1, 32, 0, s>>>(wa, base, n, d.skip, d.selfrec, d.selfreal, d.scal);
  k_weights<<<(n + 255) / 256, 256, 0, s>>>(wa, base, n, d.skip, d.selfrec, d.selfreal, d.insw_in, d.escrd, d.u0,
                                             d.w, d.twt, d.sbin, d.scal, d.status);
  k_wsum<<<1, kSumThreads, 0, s>>>(wa, base, n, d.skip, d.w, d.twt, d.u0, d.sbin, d.flceng, d.scal, d.eself,
                                   d.slnuv, d.minuv, d.maxuv);
}

__global__ void k_edens(int base, int n, int ermax, int ermax_pad, int count_base, const double* __restrict__ w,
                        const uint32_t* __restrict__ counts, double* __restrict__ edens) {
  const int bin = blockIdx.x * blockDim.x + threadIdx.x;
  if (bin >= ermax) return;
  double acc = 0.0;
  for (int i = 0; i < n; ++i) {
    const uint32_t c = counts[(size_t)(base + i - count_base) * ermax_pad + bin];
    if (c) acc += w[base + i] * (double)c;
  }
  edens[bin] += acc;
}

// edens over kEdensSlices slices of the targets: per-slice partial sums, then
// one fixed-order sum over the slices (deterministic, like the one-pass kernel)
__global__ void k_edens_part(int base, int n, int ermax, int ermax_pad, int count_base, const double* __restrict__ w,
                             const uint32_t* __restrict__ counts, double* __restrict__ part) {
  const int bin = blockIdx.x * blockDim.x + threadIdx.x;
  if (bin >= ermax) return;
  const int sl = blockIdx.y, ns = gridDim.y;
  const int lo = (int)((long long)n * sl / ns), hi = (int)((long long)n * (sl + 1) / ns);
  double acc = 0.0;
  for (int i = lo; i < hi; ++i) {
    const uint32_t c = counts[(size_t)(base + i - count_base) * ermax_pad + bin];
    if (c) acc += w[base + i] * (double)c;
  }
  part[(size_t)sl * ermax + bin] = acc;
}

__global__ void k_edens_sum(int ermax, int ns, const double* __restrict__ part, double* __restrict__ edens) {
  const int bin = blockIdx.x * blockDim.x + threadIdx.x;
  if (bin >= ermax) return;
  double acc = 0.0;
  for (int sl = 0; sl < ns; ++sl) acc += part[(size_t)sl * ermax + bin];
  edens[bin] += acc;
}

void launch_edens(const DeviceState& d, int base, int n, int ermax, int ermax_pad, int count_base, cudaStream_t s) {
  if (n <= 0) return;
  if (!d.edens_part) {
    k_edens<<<(ermax + 127) / 128, 128, 0, s>>>(base, n, ermax, ermax_pad, count_base, d.w, d.counts, d.edens);
    return;
  }
  k_edens_part<<<dim3((ermax + 127) / 128, kEdensSlices), 128, 0, s>>>(base, n, ermax, ermax_pad, count_base, d.w,
                                                                        d.counts, d.edens_part);
  k_edens_sum<<<(ermax + 127) / 128, 128, 0, s>>>(ermax, kEdensSlices, d.edens_part, d.edens);
}

// FP64 CUDA-core ecorr update, 64x64 tile per 256 threads (4x4 per thread)
__global__ void __launch_bounds__(256) k_ecorr_simt(int base, int n, int ermax, int ermax_pad, int count_base,
    const double* __restrict__ w, const uint32_t* __restrict__ counts, double* __restrict__ ecorr) {
  __shared__ double As[16][64];
  __shared__ double Bs[16][64];
  const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < n; k0 += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int kk = t / 64, col = t % 64;
      const int cnt = base + k0 + kk;
      double va = 0.0, vb = 0.0;
      if (k0 + kk < n) {
        const uint32_t* row = counts + (size_t)(cnt - count_base) * ermax_pad;
        if (i0 + col < ermax) va = w[cnt] * (double)row[i0 + col];
        if (j0 + col < ermax) vb = (double)row[j0 + col];
      }
      As[kk][col] = va;
      Bs[kk][col] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      double av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { av[u] = As[kk][ty * 4 + u]; bv[u] = Bs[kk][tx * 4 + u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = i0 + ty * 4 + u, j = j0 + tx * 4 + v;
      if (i < ermax && j < ermax) ecorr[(size_t)i * ermax + j] += acc[u][v];
    }
}

void launch_ecorr_simt(const DeviceState& d, int base, int n, int ermax, int ermax_pad, int count_base, cudaStream_t s) {
  if (n <= 0) return;
  dim3 grid((ermax + 63) / 64, (ermax + 63) / 64);
  k_ecorr_simt<<<grid, 256, 0, s>>>(base, n, ermax, ermax_pad, count_base, d.w, d.counts, d.ecorr);
}

}  // namespace erm
