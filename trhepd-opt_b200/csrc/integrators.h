// Integrator families of srfref (sim-trhepd-rheed/src/surflf.f90:118-140) and the
// depths of their stage potential tables (host side, shared by the solver and the
// table entry points).
#pragma once
#include <cmath>
#include <stdexcept>
#include <vector>

namespace trhepd {

// Blanes-Moan RKN coefficient tables (surf_prkn.f90:11-52).
inline constexpr double kRkn46[13] = {
    0.0829844064174052,  0.245298957184271,  0.396309801498368,  0.604872665711080,
    -0.0390563049223486, -0.350171622895351, 0.1195241940131508, -0.350171622895351,
    -0.0390563049223486, 0.604872665711080,  0.396309801498368,  0.245298957184271,
    0.0829844064174052};
inline constexpr double kRkn611[23] = {
    0.0414649985182624,  0.123229775946271,  0.198128671918067,  0.290553797799558,
    -0.0400061921041533, -0.127049212625417, 0.0752539843015807, -0.246331761062075,
    -0.0115113874206879, 0.357208872795928,  0.2366699247869311, 0.20477705429147,
    0.2366699247869311,  0.357208872795928,  -0.0115113874206879, -0.246331761062075,
    0.0752539843015807,  -0.127049212625417, -0.0400061921041533, 0.290553797799558,
    0.198128671918067,   0.123229775946271,  0.0414649985182624};

enum Family { kRkn = 0, kLeapfrog = 1, kRk4 = 2, kMagnus2 = 3, kMagnus4 = 4, kMagnus6 = 5 };

struct Integrator {
  int method = 5;
  Family family = kRkn;
  int s = 6;                   // RKN stages per slice
  const double* bab = nullptr; // RKN coefficients (b1, a1, b2, a2, ...)
  bool gs = false;             // RK4 with CholeskyQR re-orthogonalisation (int_method 8)
};

inline Integrator integrator_for(int method) {
  switch (method) {
    case 1: return {1, kMagnus2, 1, nullptr};
    case 2: return {2, kMagnus4, 3, nullptr};
    case 3: return {3, kMagnus6, 3, nullptr};
    case 4: return {4, kLeapfrog, 1, nullptr};
    case 5: return {5, kRkn, 6, kRkn46};
    case 6: return {6, kRkn, 11, kRkn611};
    case 7: return {7, kRk4, 2, nullptr};
    case 8: return {8, kRk4, 2, nullptr, true};  // rk4_intgs: rk4_int_init's table
    default:
      throw std::invalid_argument(
          "int_method must be 1-3 (Magnus 2/4/6), 4 (leapfrog), 5 (RKN-4), 6 (RKN-6), 7 (RK4) or"
          " 8 (RK4 with CholeskyQR)");
  }
}

// Depths of the stage potential table, same arithmetic order as the reference's
// init routines: hp_int_init4/6 (surf_prkn.f90:184-196), m2_int_init
// (surf_magnus.f90:4-20, used by m2 and leapfrog), m4_int_init (:24-42, m4 and m6),
// rk4_int_init (surf_rk.f90:4-25).
inline std::vector<double> stage_depths(const Integrator& I, int ns, double dz) {
  std::vector<double> d;
  switch (I.family) {
    case kRkn:
      d.reserve((size_t)I.s * ns + 1);
      for (int l = 1; l <= ns; ++l) {
        double iz = dz * (l - 1);
        for (int k = 1; k <= I.s; ++k) {
          d.push_back(iz);
          iz = iz + dz * I.bab[2 * k - 1];
        }
      }
      d.push_back(dz * ns);
      break;
    case kLeapfrog:
    case kMagnus2:
      for (int l = 1; l <= ns; ++l) d.push_back(dz * (l - 0.5));
      break;
    case kMagnus4:
    case kMagnus6: {  // m4_int_init (surf_magnus.f90:24-42): the three Gauss points
      const double c0 = (5.0 - std::sqrt(15.0)) / 10, c1 = 0.5, c2 = (5.0 + std::sqrt(15.0)) / 10;
      for (int l = 1; l <= ns; ++l) {
        d.push_back(dz * ((l - 1) + c0));
        d.push_back(dz * ((l - 1) + c1));
        d.push_back(dz * ((l - 1) + c2));
      }
      break;
    }
    case kRk4:
      for (int l = 1; l <= ns; ++l) {
        const double iz = dz * (l - 1);
        d.push_back(iz);
        d.push_back(iz + 0.5 * dz);
      }
      d.push_back(dz * ns);
      break;
  }
  return d;
}

}  // namespace trhepd
