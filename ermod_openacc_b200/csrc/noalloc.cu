// noalloc.cu -- energy histogram entry point that allocates no device memory.
//
// Some hosts cannot ask the CUDA runtime for memory: a Fortran erdst host
// whose device memory is owned by its OpenACC runtime (data regions and the
// present table decide what lives on the GPU), or an MPI job that fixes
// every rank's GPU footprint up front under a scheduler's memory limit.  For
// them ermod_histogram_noalloc bins per-molecule energies into edens using
// the engine's binning kernel (k_bin) and edens reduction (k_edens), with all
// of their working memory in one fixed array compiled into this library.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "engine.cuh"

namespace {

// The scratch every call works in.  Each GPU that loads the library holds
// these bytes until the process exits.
constexpr size_t kNoallocBytes = ERMOD_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;   // first calls from several host threads look the address up once

// Device address of the scratch array on the current device (host code sees
// only a host-side stand-in for the symbol; the address must be queried).
// Looked up on the first call per device and kept; a failed lookup is retried
// on the next call.
int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return ERMOD_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ERMOD_ERR_CUDA;
    g_scratch_addr[device] = p;
  }
  *out = (unsigned char*)g_scratch_addr[device];
  return ERMOD_OK;
}

size_t align256(size_t n) { return (n + 255) / 256 * 256; }

}  // namespace

extern "C" int32_t ermod_histogram_noalloc(int32_t device, int32_t slttype, const double* uvengy,
                                           int32_t ntarget, int32_t nmol, const int32_t* uvspec,
                                           const double* uvcrd, const int32_t* uvmax, const int32_t* uvsoft,
                                           int32_t numslv, const double* weight, double* edens) {
  using namespace erm;
  const bool soln = slttype == ERMOD_SLT_SOLN;
  if (!uvengy || !uvspec || !uvcrd || !uvmax || !weight || !edens || ntarget <= 0 || nmol <= 0 || numslv <= 0)
    return ERMOD_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return ERMOD_ERR_CUDA;
  unsigned char* base = nullptr;
  int rc = scratch_address(device, &base);
  if (rc != ERMOD_OK) return rc;
  int ermax = 0;
  for (int q = 0; q < numslv; ++q) {
    if (uvmax[q] <= 0) return ERMOD_ERR_ARG;
    ermax += uvmax[q];
  }
  for (int k = 0; k < nmol; ++k)
    if (uvspec[k] < 0 || uvspec[k] > numslv) return ERMOD_ERR_ARG;
  const int ermax_pad = (ermax + 127) / 128 * 128;
  // carve the scratch
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += align256(bytes); return base + o; };
  double* d_E = (double*)take(sizeof(double) * (size_t)ntarget * nmol);
  int* d_spec = (int*)take(sizeof(int) * nmol);
  double* d_uvcrd = (double*)take(sizeof(double) * ermax);
  int* d_off = (int*)take(sizeof(int) * (numslv + 1));
  int* d_soft = (int*)take(sizeof(int) * numslv);
  double* d_w = (double*)take(sizeof(double) * ntarget);
  uint32_t* d_counts = (uint32_t*)take(sizeof(uint32_t) * (size_t)ntarget * ermax_pad);
  double* d_etot = (double*)take(sizeof(double) * ntarget);
  float* d_min = (float*)take(sizeof(float) * (numslv + 1));
  float* d_max = (float*)take(sizeof(float) * (numslv + 1));
  double* d_edens = (double*)take(sizeof(double) * ermax);
  // solutes in solution: k_bin also forms each target's per-species energy sums (flceng)
  double* d_fl = soln ? (double*)take(sizeof(double) * (size_t)ntarget * numslv) : nullptr;
  DevStatus* d_st = (DevStatus*)take(sizeof(DevStatus));
  if (off > kNoallocBytes) return ERMOD_ERR_OVERFLOW;  // beyond ERMOD_NOALLOC_SCRATCH_BYTES
  // inputs into the scratch; outputs and counters start from zero / the
  // reference's initial values (the array keeps the previous call's contents)
  std::vector<int> offs(numslv + 1, 0), soft(numslv);
  for (int q = 0; q < numslv; ++q) {
    offs[q + 1] = offs[q] + uvmax[q];
    soft[q] = uvsoft ? uvsoft[q] : uvmax[q];
  }
  std::vector<float> mn(numslv + 1, FLT_MAX), mx(numslv + 1, -FLT_MAX);
  cudaStream_t s = 0;
  bool ok = true;
  ok &= cudaMemcpyAsync(d_E, uvengy, sizeof(double) * (size_t)ntarget * nmol, cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_spec, uvspec, sizeof(int) * nmol, cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_uvcrd, uvcrd, sizeof(double) * ermax, cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_off, offs.data(), sizeof(int) * (numslv + 1), cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_soft, soft.data(), sizeof(int) * numslv, cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_w, weight, sizeof(double) * ntarget, cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_min, mn.data(), sizeof(float) * (numslv + 1), cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemcpyAsync(d_max, mx.data(), sizeof(float) * (numslv + 1), cudaMemcpyHostToDevice, s) == cudaSuccess;
  ok &= cudaMemsetAsync(d_edens, 0, sizeof(double) * ermax, s) == cudaSuccess;
  if (d_fl) ok &= cudaMemsetAsync(d_fl, 0, sizeof(double) * (size_t)ntarget * numslv, s) == cudaSuccess;
  ok &= cudaMemsetAsync(d_st, 0, sizeof(DevStatus), s) == cudaSuccess;
  if (!ok) return ERMOD_ERR_CUDA;
  DeviceState d;
  d.Etot = d_E;
  d.molspec = d_spec;
  d.spec_off = d_off;
  d.uvcrd = d_uvcrd;
  d.uvsoft = d_soft;
  d.tgt_mol = nullptr;
  d.counts = d_counts;
  d.etot = d_etot;
  d.flceng = d_fl;
  d.minuv = d_min;
  d.maxuv = d_max;
  d.status = d_st;
  d.w = d_w;
  d.edens = d_edens;
  BinArgs ba{};
  ba.ermax = ermax;
  ba.ermax_pad = ermax_pad;
  ba.numslv = numslv;
  ba.slttype = soln ? ERMOD_SLT_SOLN : ERMOD_SLT_REFS_RIGID;
  if (setup_bin_smem(ba) != 0) return ERMOD_ERR_OVERFLOW;
  launch_bin(d, ba, 0, ntarget, nmol, 0, s);
  launch_edens(d, 0, ntarget, ermax, ermax_pad, 0, s);
  DevStatus hs;
  if (cudaMemcpyAsync(&hs, d_st, sizeof(hs), cudaMemcpyDeviceToHost, s) != cudaSuccess) return ERMOD_ERR_CUDA;
  if (cudaMemcpyAsync(edens, d_edens, sizeof(double) * ermax, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return ERMOD_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ERMOD_ERR_CUDA;
  if (hs.flags & kErrEngCns) return ERMOD_ERR_ENG_CNS;
  if (hs.flags & kErrEngMin) return ERMOD_ERR_ENG_MIN;
  if (hs.flags & kErrEngSft) return ERMOD_ERR_ENG_SFT;
  if (hs.flags & kWarnMbin) return ERMOD_WARN_MBIN;
  return ERMOD_OK;
}
