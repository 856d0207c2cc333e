// Host-side problem description of one surface solve: the mod_scpot3 state plus
// the srfref arguments (sim-trhepd-rheed/src/surfio.f90:18-27, surflf.f90:7-8),
// and the C++ surfio equivalent that builds it from the unchanged input files.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace trhepd {

constexpr int kMab = 6;  // surfio.f90:16

// Plane-group images of one structure-factor set (scpot_stf, scpot.f90:100-110):
// st(k, j) = sum_m exp(i (gh_k (dx + x_jm) + gk_k (dy + y_jm))) for k < nk.
struct StructureFactorJob {
  int nk = 0, natm = 0;
  double dx = 0, dy = 0;
  std::vector<double> img;  // natm x 12 x (x, y) in 1x1-lattice units
  std::vector<int> nimg;    // natm
};

// Orbit of atom (x, y) under plane group nsg in the (ma mb; na nb) cell
// (strfac.f90:15-64); writes <= 12 (x, y) pairs, returns the count.
int plane_group_images(int nsg, int ma, int mb, int na, int nb, double x, double y,
                       double* out_xy);

struct SurfaceInputs {
  // ---- mod_scpot3 (surfio.f90:18-27)
  int nv = 0, nvb = 0, natms = 0, natmb = 0, nelm = 0, nabr = 4, nabi = 1;
  std::vector<int> ielm;          // natmb + natms, 1-based element index, bulk atoms first
  double cc = 0, smesh = 1;
  std::vector<double> z, ocr;     // natm
  std::vector<double> dchg;       // nelm
  std::vector<double> Ghk;        // nv
  std::vector<double> b;          // (mab, nelm) column-major
  std::vector<double> asf;        // (nv, mab, nelm) column-major
  std::vector<cd> st0, st1, st2;  // (nv, natms), (nvb, natmb), (nvb, natmb)
  // inputs of the three structure-factor sums (filled by the loader; the sums are
  // formed on the GPU and stored into st0/st1/st2)
  std::vector<double> gh, gk;     // nv
  StructureFactorJob stf[3];
  // ---- srfref arguments (surflf.f90:7-8)
  int nb = 0, ns = 0;
  double dz = 0;
  std::vector<int> iv;            // (nb, nb) column-major, 1-based, entries l > k
  int ngr = 1;
  std::vector<int> nbg, iord, ih, ik;
  double wn = 0, ghx = 0, ghy = 0, gky = 0, azi = 0, daz = 0, gi = 0, dg = 0;
  int naz = 1, ng = 1, int_method = 5;
  std::vector<cd> t1rec;          // bulk records: nrep1*nrep2 angles x sum(nbg^2), file order
  // ---- output header data (surfio.f90:270-288) for the rocking-curve writer and the
  // domain sum (domainsum.f90): every domain's beams, angle and weight
  int ndom = 1, domain = 0;       // domains in the files; the one these inputs describe
  int nh = 1, nk = 1;
  double gam = 0;                 // cell angle (radians)
  std::vector<int> nbd;           // beams per domain
  std::vector<double> rdom, wdom; // domain angles (radians) and weights
  std::vector<int> ih_all, ik_all;  // every domain's beams, domain after domain
};

// surfio (surfio.f90:60-381) for domain `domain` (0-based; srfref is called with
// azimuth azi + rdom(domain), surfio.f90:340): parse bulkP.b and surf.txt, apply the
// surface slicing rule for dz2, and fill every field above.
// Throws std::runtime_error on malformed input.
void load_surface_inputs(const std::string& bulkp, const std::string& surf, double dz2,
                         int int_method, SurfaceInputs& out, int domain = 0);

// Write the rocking-curve file (surfio.f90:270-274 header, surflf.f90:154-165 rows).
void write_rocking_curves(const std::string& path, const SurfaceInputs& in, const double* f2,
                          const double* angle_deg);

}  // namespace trhepd
