// Host-side setup of the bulk solve: a C++ equivalent of bulkio
// (sim-trhepd-rheed/src/bulkio.f90:10-223) for one domain, positrons or electrons
// (bulkm.f90:21-24: inegpos = 1 or 0).  The reflection records themselves come
// from the GPU.
#pragma once
#include <string>
#include <vector>

#include "common.cuh"
#include "host_model.h"

namespace trhepd {

struct BulkInputs {
  // ---- header records of bulkP.b (bulkio.f90:126-141), as written
  int nh = 1, nk = 1, nb = 0, naz = 1, ng = 1, ml = 100, nsg = 1, nelm = 0, natm = 0;
  int nabr = 4, nabi = 1, iabr = 0;
  int inegpos = 1;                             // 1 positron, 0 electron
  double rdom = 0, be = 10, azi = 0, daz = 0, gi = 0, dg = 0, dz = 0, epsb = 1e-10;
  double aa = 0, bb = 0, gam = 0, cc = 0, dx = 0, dy = 0, zoffset = 0;
  std::vector<int> ih, ik;                     // original beam order (this domain)
  int ndom = 1, domain = 0;                    // domains in bulk.txt; the one described
  std::vector<int> nbd;                        // beams per domain
  std::vector<double> rdom_all;                // domain angles (radians)
  std::vector<int> ih_all, ik_all;             // every domain's beams
  std::vector<double> a_raw, b_raw;            // (nabr+nabi) per element, before asfcrr
  std::vector<double> dth_raw, dtk_raw, dtz_raw, elm, dchg;
  std::vector<int> ielm;                       // 1-based
  std::vector<double> ocr, x, y, z;            // z with zoffset
  // ---- derived
  int ns = 0;                                  // slices per unit layer
  double wn = 0, ghx = 0, ghy = 0, gky = 0;
  std::vector<int> iord, nbg, ihs, iks;        // blkibg (sorted beams)
  int ngr = 0, nbgm = 0, nv = 0;
  std::vector<int> igh, igk, iv;               // blkghk; iv (nbgm, nb) column-major
  std::vector<double> asf, Ghk, bcoef;         // asfcef / asfcrr outputs
  std::vector<double> gh, gk;
  StructureFactorJob stf[3];                   // st at zi (0,0), zi+cc (-dx,-dy), zi-cc (dx,dy)
};

// Parse bulk.txt and derive everything above for domain `domain` (0-based; its
// azimuth is azi + rdom(domain), bulkio.f90:205-207), positrons (inegpos = 1) or
// electrons (0).  Throws std::runtime_error.
void load_bulk_inputs(const std::string& bulk_txt, BulkInputs& B, int inegpos = 1,
                      int domain = 0);

// Write bulkP.b: header records (bulkio.f90:126-141) plus, per domain in order, its
// beam tables (:173-176) and reflection records t4 (per angle, per group, nbf x nbf
// column-major, bulk.f90:122).  B[d] describes domain d.
void write_bulkp(const std::string& path, const std::vector<BulkInputs>& B,
                 const std::vector<std::vector<std::vector<cd>>>& records);

}  // namespace trhepd
