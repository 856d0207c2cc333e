// Stage potential tables without allocating device memory.
//
// Some hosts of this library cannot call cudaMalloc: a Fortran driver that hands
// all of the GPU's memory to its own pool at start-up, or a long-running
// structure-refinement service whose device memory is planned once and must not
// grow or fragment afterwards.  For them trhepd_potential_table_noalloc builds
// the same tables as trhepd_potential_table, but its device scratch (the copies
// of the mod_scpot3 inputs and the table itself) lives in one file-scope device
// array of kNoAllocScratchBytes.  The array is part of the loaded library: every
// GPU that loads it holds those bytes until the process exits.
//
// Calls share the array and it keeps the last call's contents.  Nothing in it
// has to start at zero: every region a call reads is written by that call first.
// Two calls whose GPU work overlaps (from different host threads) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/trhepd_b200.h"
#include "host_model.h"
#include "integrators.h"
#include "kernels.h"

namespace {

using namespace trhepd;

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The device address of the array on the current device.  In host code the
// array's name is only a host-side stand-in, so every call asks the runtime for
// the address on the device that is current for it (the lookup is cheap next to
// the call's synchronous copies, and stays right after a cudaDeviceReset reloads
// the module).
void* scratch_address() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
  return p;
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int trhepd_potential_table_noalloc(const trhepd_pot_state* pot, int int_method,
                                              int ns, double dz, double* v, double* vi,
                                              int* ncol_out) {
  if (!pot || ns < 1) return TRHEPD_EINVAL;
  Integrator I;
  try {
    I = integrator_for(int_method);
  } catch (const std::invalid_argument&) {
    return TRHEPD_EINVAL;
  }
  if (pot->nv < 1 || pot->nelm < 1 || pot->nabr < 1 || pot->nabr + pot->nabi > kMab)
    return TRHEPD_EINVAL;
  if (pot->natms < 0 || pot->natmb < 0 || pot->natms + 2 * pot->natmb > 512)
    return TRHEPD_EINVAL;
  const int nv = pot->nv, nelm = pot->nelm;
  // the stage depths of the integrator's init routine, as trhepd_potential_table
  const std::vector<double> depth = stage_depths(I, ns, dz);
  const int ncol = (int)depth.size();

  // layout of the scratch: inputs, depths, table
  const int first[3] = {pot->natmb, 0, 0};
  const int count[3] = {pot->natms, pot->natmb, pot->natmb};
  const int nk[3] = {nv, pot->nvb, pot->nvb};
  const double* stp[3] = {pot->st0, pot->st1, pot->st2};
  size_t off = 0;
  const size_t o_asf = off;
  off = up256(off + (size_t)nv * kMab * nelm * sizeof(double));
  const size_t o_b = off;
  off = up256(off + (size_t)kMab * nelm * sizeof(double));
  const size_t o_dchg = off;
  off = up256(off + (size_t)nelm * sizeof(double));
  const size_t o_ghk = off;
  off = up256(off + (size_t)nv * sizeof(double));
  size_t o_z[3], o_ocr[3], o_ie[3], o_st[3];
  for (int p = 0; p < 3; ++p) {
    o_z[p] = off;
    off = up256(off + (size_t)count[p] * sizeof(double));
    o_ocr[p] = off;
    off = up256(off + (size_t)count[p] * sizeof(double));
    o_ie[p] = off;
    off = up256(off + (size_t)count[p] * sizeof(int));
    o_st[p] = off;
    off = up256(off + (size_t)nk[p] * count[p] * sizeof(cd));
  }
  const size_t o_depth = off;
  off = up256(off + (size_t)ncol * sizeof(double));
  const size_t o_table = off;
  off = up256(off + (size_t)ncol * nv * sizeof(TableEntry));
  if (off > kNoAllocScratchBytes) return TRHEPD_ENOMEM;  // beyond the static scratch

  unsigned char* base = static_cast<unsigned char*>(scratch_address());
  if (!base) return TRHEPD_ECUDA;

  auto put = [&](size_t o, const void* src, size_t bytes) {
    return bytes == 0 || cudaMemcpy(base + o, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = put(o_asf, pot->asf, (size_t)nv * kMab * nelm * sizeof(double)) &&
            put(o_b, pot->b, (size_t)kMab * nelm * sizeof(double)) &&
            put(o_dchg, pot->dchg, (size_t)nelm * sizeof(double)) &&
            put(o_ghk, pot->Ghk, (size_t)nv * sizeof(double)) &&
            put(o_depth, depth.data(), depth.size() * sizeof(double));
  PotInputs in{};
  in.asf = reinterpret_cast<const double*>(base + o_asf);
  in.b = reinterpret_cast<const double*>(base + o_b);
  in.dchg = reinterpret_cast<const double*>(base + o_dchg);
  in.ghk = reinterpret_cast<const double*>(base + o_ghk);
  in.nv = nv;
  in.nelm = nelm;
  in.nabr = pot->nabr;
  in.nabi = pot->nabi;
  in.mab = kMab;
  const double shift[3] = {-pot->cc, 0.0, pot->cc};
  const double mesh[3] = {1.0, pot->smesh, pot->smesh};
  for (int p = 0; p < 3 && ok; ++p) {
    std::vector<int> ie(count[p]);
    for (int j = 0; j < count[p]; ++j) {
      int e = pot->ielm[first[p] + j];
      if (e < 1 || e > nelm) return TRHEPD_EINVAL;
      ie[j] = e - 1;
    }
    ok = put(o_z[p], pot->z + first[p], count[p] * sizeof(double)) &&
         put(o_ocr[p], pot->ocr + first[p], count[p] * sizeof(double)) &&
         put(o_ie[p], ie.data(), ie.size() * sizeof(int)) &&
         put(o_st[p], stp[p], (size_t)nk[p] * count[p] * sizeof(cd));
    PotPart& P = in.part[p];
    P.z = reinterpret_cast<const double*>(base + o_z[p]);
    P.ocr = reinterpret_cast<const double*>(base + o_ocr[p]);
    P.ielm = reinterpret_cast<const int*>(base + o_ie[p]);
    P.st = reinterpret_cast<const cd*>(base + o_st[p]);
    P.natm = count[p];
    P.nk = nk[p];
    P.zshift = shift[p];
    P.rmesh = mesh[p];
  }
  if (!ok) return TRHEPD_ECUDA;
  TableEntry* table = reinterpret_cast<TableEntry*>(base + o_table);
  launch_potential_table(in, reinterpret_cast<const double*>(base + o_depth), ncol, table, 0);
  if (cudaGetLastError() != cudaSuccess) return TRHEPD_ECUDA;
  std::vector<TableEntry> h((size_t)ncol * nv);
  if (cudaMemcpy(h.data(), table, h.size() * sizeof(TableEntry), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return TRHEPD_ECUDA;
  for (size_t e = 0; e < h.size(); ++e) {  // v = (u + w) / 2, vi = (u - w) / 2
    if (v) {
      v[2 * e] = 0.5 * (h[e].u.x + h[e].w.x);
      v[2 * e + 1] = 0.5 * (h[e].u.y + h[e].w.y);
    }
    if (vi) {
      vi[2 * e] = 0.5 * (h[e].u.x - h[e].w.x);
      vi[2 * e + 1] = 0.5 * (h[e].u.y - h[e].w.y);
    }
  }
  if (ncol_out) *ncol_out = ncol;
  return TRHEPD_OK;
}
