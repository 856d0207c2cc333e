// Host-side setup of the surface solve: a C++ equivalent of surfio for the first
// domain (sim-trhepd-rheed/src/surfio.f90:60-381) that reads the unchanged
// bulkP.b / surf.txt formats and produces the mod_scpot3 state and the srfref
// arguments.  Structure-factor sums run on the GPU (see kernels_f64.cu K2); this
// file only forms the plane-group images.
#include "host_model.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>

#include "fortran_text.h"
#include "scattering_tables.h"

namespace trhepd {

using namespace ftext;

namespace {

const double kPi = std::atan(1.0) * 4.0;

// ------------------------------------------------------------ plane groups
// Orbit of one atom under the 17 plane groups (strfac.f90:88-527).  Each group is a
// list of cases tried in order: a special-position test and the images it keeps.
struct Op {  // x' = a*x + b*y + c ; y' = d*x + e*y + f
  int a, b, d, e;
  double c, f;
};
using Test = std::function<bool(double, double)>;
struct Case {
  Test when;
  std::vector<Op> ops;
};

constexpr double kTol = 2e-4;
bool at(double u, double v) { return std::fabs(u - v) < kTol; }
bool edge(double u) { return at(u, 0.0) || at(u, 0.5); }
const Op I_{1, 0, 0, 1, 0, 0};
Op op(int a, int b, double c, int d, int e, double f) { return Op{a, b, d, e, c, f}; }

const std::vector<Case>& group_cases(int nsg) {
  static std::vector<std::vector<Case>> G;
  if (G.empty()) {
    G.resize(18);
    auto any = [](double, double) { return true; };
    auto c3 = [](double x, double y) {
      return (at(x, 0) && at(y, 0)) || (at(x, 1.0 / 3.0) && at(y, 2.0 / 3.0)) ||
             (at(x, 2.0 / 3.0) && at(y, 1.0 / 3.0));
    };
    auto c3b = [](double x, double y) {
      return (at(x, 1.0 / 3.0) && at(y, 2.0 / 3.0)) || (at(x, 2.0 / 3.0) && at(y, 1.0 / 3.0));
    };
    auto origin = [](double x, double y) { return at(x, 0) && at(y, 0); };
    auto c4 = [](double x, double y) {
      return (at(x, 0) && at(y, 0)) || (at(x, 0.5) && at(y, 0.5));
    };
    auto c2b = [](double x, double y) {
      return (at(x, 0.5) && at(y, 0)) || (at(x, 0) && at(y, 0.5));
    };
    auto c2c = [](double x, double y) {
      return (at(x, 0.5) && at(y, 0)) || (at(x, 0) && at(y, 0.5)) || (at(x, 0.5) && at(y, 0.5));
    };
    auto mirror3 = [](double x, double y) { return at(x, 0) || at(y, 0) || at(x - y, 0); };
    G[1] = {{any, {I_}}};
    G[2] = {{[](double x, double y) { return edge(x) && edge(y); }, {I_}},
            {any, {I_, op(-1, 0, 0, 0, -1, 0)}}};
    G[3] = {{[](double, double y) { return edge(y); }, {I_}}, {any, {I_, op(1, 0, 0, 0, -1, 0)}}};
    G[4] = {{any, {I_, op(1, 0, 0.5, 0, -1, 0)}}};
    G[5] = {{[](double, double y) { return edge(y); }, {I_, op(1, 0, 0.5, 0, -1, 0.5)}},
            {any, {I_, op(1, 0, 0.5, 0, -1, 0.5), op(1, 0, 0, 0, -1, 0), op(1, 0, 0.5, 0, 1, 0.5)}}};
    G[6] = {{[](double x, double y) { return edge(x) && edge(y); }, {I_}},
            {[](double x, double) { return edge(x); }, {I_, op(1, 0, 0, 0, -1, 0)}},
            {[](double, double y) { return edge(y); }, {I_, op(-1, 0, 0, 0, 1, 0)}},
            {any, {I_, op(1, 0, 0, 0, -1, 0), op(-1, 0, 0, 0, 1, 0), op(-1, 0, 0, 0, -1, 0)}}};
    G[7] = {{[](double x, double y) { return edge(x) && edge(y); }, {I_, op(1, 0, 0, 0, -1, 0.5)}},
            {[](double, double y) { return at(y, 0.25) || at(y, 0.75); },
             {I_, op(-1, 0, 0, 0, -1, 0)}},
            {any, {I_, op(1, 0, 0, 0, -1, 0.5), op(-1, 0, 0, 0, -1, 0), op(-1, 0, 0, 0, 1, 0.5)}}};
    G[8] = {{[](double x, double y) { return edge(x) && edge(y); }, {I_, op(-1, 0, 0.5, 0, 1, 0.5)}},
            {any,
             {I_, op(-1, 0, 0.5, 0, 1, 0.5), op(1, 0, 0.5, 0, -1, 0.5), op(-1, 0, 0, 0, -1, 0)}}};
    G[9] = {
        {[](double x, double y) { return edge(x) && edge(y); }, {I_, op(-1, 0, 0.5, 0, 1, 0.5)}},
        {[](double x, double y) {
           return (at(x, 0.25) || at(x, 0.75)) && (at(y, 0.25) || at(y, 0.75));
         },
         {I_, op(1, 0, 0, 0, -1, 0), op(-1, 0, 0, 0, 1, 0), op(-1, 0, 0, 0, -1, 0)}},
        {[](double x, double) { return edge(x); },
         {I_, op(1, 0, 0, 0, -1, 0), op(-1, 0, 0.5, 0, 1, 0.5), op(-1, 0, 0.5, 0, -1, 0.5)}},
        {[](double, double y) { return edge(y); },
         {I_, op(-1, 0, 0, 0, 1, 0), op(1, 0, 0.5, 0, -1, 0.5), op(-1, 0, 0.5, 0, -1, 0.5)}},
        {any,
         {I_, op(1, 0, 0, 0, -1, 0), op(-1, 0, 0, 0, 1, 0), op(-1, 0, 0, 0, -1, 0),
          op(1, 0, 0.5, 0, 1, 0.5), op(1, 0, 0.5, 0, -1, 0.5), op(-1, 0, 0.5, 0, 1, 0.5),
          op(-1, 0, 0.5, 0, -1, 0.5)}}};
    G[10] = {{c4, {I_}},
             {c2b, {I_, op(0, 1, 0, -1, 0, 0)}},
             {any, {I_, op(0, -1, 0, 1, 0, 0), op(-1, 0, 0, 0, -1, 0), op(0, 1, 0, -1, 0, 0)}}};
    G[11] = {{c4, {I_}},
             {c2b, {I_, op(0, 1, 0, 1, 0, 0)}},
             {[](double x, double y) {
                return at(y - x, 0) || at(x + y - 1.0, 0) || edge(x) || edge(y);
              },
              {I_, op(0, -1, 0, 1, 0, 0), op(-1, 0, 0, 0, -1, 0), op(0, 1, 0, -1, 0, 0)}},
             {any,
              {I_, op(0, 1, 0, 1, 0, 0), op(0, -1, 0, 1, 0, 0), op(-1, 0, 0, 0, 1, 0),
               op(-1, 0, 0, 0, -1, 0), op(0, -1, 0, -1, 0, 0), op(0, 1, 0, -1, 0, 0),
               op(1, 0, 0, 0, -1, 0)}}};
    G[12] = {{c4, {I_, op(0, -1, 0.5, -1, 0, 0.5)}},
             {c2b, {I_, op(0, 1, 0, -1, 0, 0)}},
             {[](double x, double y) {
                return at(y - x + 0.5, 0) || at(y - x - 0.5, 0) || at(x + y - 0.5, 0) ||
                       at(x + y - 1.5, 0);
              },
              {I_, op(0, -1, 0, 1, 0, 0), op(-1, 0, 0, 0, -1, 0), op(0, 1, 0, -1, 0, 0)}},
             {any,
              {I_, op(0, -1, 0, 1, 0, 0), op(-1, 0, 0, 0, -1, 0), op(0, 1, 0, -1, 0, 0),
               op(0, -1, 0.5, -1, 0, 0.5), op(1, 0, 0.5, 0, -1, 0.5), op(0, 1, 0.5, 1, 0, 0.5),
               op(-1, 0, 0.5, 0, 1, 0.5)}}};
    G[13] = {{c3, {I_}}, {any, {I_, op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, -1, 0, 0)}}};
    G[14] = {{c3, {I_}},
             {[](double x, double y) {
                return at(x + x - y, 0) || at(y + y - x, 0) || at(x + x - y - 1.0, 0) ||
                       at(y + y - x - 1.0, 0) || at(x + y - 1.0, 0);
              },
              {I_, op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, -1, 0, 0)}},
             {any,
              {I_, op(1, 0, 0, 1, -1, 0), op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, 0, 1, 0),
               op(-1, 1, 0, -1, 0, 0), op(0, -1, 0, -1, 0, 0)}}};
    G[15] = {{origin, {I_}},
             {c3b, {I_, op(0, 1, 0, 1, 0, 0)}},
             {mirror3, {I_, op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, -1, 0, 0)}},
             {any,
              {I_, op(0, 1, 0, 1, 0, 0), op(0, -1, 0, 1, -1, 0), op(-1, 0, 0, -1, 1, 0),
               op(-1, 1, 0, -1, 0, 0), op(1, -1, 0, 0, -1, 0)}}};
    G[16] = {{origin, {I_}},
             {c3b, {I_, op(0, 1, 0, 1, 0, 0)}},
             {c2c, {I_, op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, -1, 0, 0)}},
             {any,
              {I_, op(1, -1, 0, 1, 0, 0), op(0, -1, 0, 1, -1, 0), op(-1, 0, 0, 0, -1, 0),
               op(-1, 1, 0, -1, 0, 0), op(0, 1, 0, -1, 1, 0)}}};
    G[17] = {{origin, {I_}},
             {c3b, {I_, op(0, 1, 0, 1, 0, 0)}},
             {c2c, {I_, op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, -1, 0, 0)}},
             {mirror3,
              {I_, op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, -1, 0, 0), op(-1, 0, 0, 0, -1, 0),
               op(0, 1, 0, -1, 1, 0), op(1, -1, 0, 1, 0, 0)}},
             {any,
              {I_, op(1, 0, 0, 1, -1, 0), op(1, -1, 0, 1, 0, 0), op(0, 1, 0, 1, 0, 0),
               op(0, -1, 0, 1, -1, 0), op(-1, 1, 0, 0, 1, 0), op(-1, 0, 0, 0, -1, 0),
               op(-1, 0, 0, -1, 1, 0), op(-1, 1, 0, -1, 0, 0), op(0, -1, 0, -1, 0, 0),
               op(0, 1, 0, -1, 1, 0), op(1, -1, 0, 0, -1, 0)}}};
  }
  if (nsg < 1 || nsg > 17) throw std::runtime_error("plane group must be 1..17");
  return G[nsg];
}

double wrap01(double x) { return x - std::floor(x + 1e-4); }  // strfac.f90:80-84

// Images of atom (x, y) (1x1 lattice units) in the (ma mb; na nb) surface cell,
// returned in 1x1 units (strfac.f90:15-64).  Returns the image count (<= 12).
}  // namespace

int plane_group_images(int nsg, int ma, int mb, int na, int nb, double x, double y,
                       double* out_xy) {
  double s = (double)(ma * nb - mb * na);
  double xs = wrap01((nb * x - na * y) / s), ys = wrap01((ma * y - mb * x) / s);
  for (const Case& c : group_cases(nsg)) {
    if (!c.when(xs, ys)) continue;
    int m = 0;
    for (const Op& o : c.ops) {
      double u = o.a * xs + o.b * ys + o.c, v = o.d * xs + o.e * ys + o.f;
      u = wrap01(u);
      v = wrap01(v);
      out_xy[2 * m] = ma * u + na * v;
      out_xy[2 * m + 1] = mb * u + nb * v;
      ++m;
    }
    return m;
  }
  return 0;
}

void load_surface_inputs(const std::string& bulkp, const std::string& surf, double dz2,
                         int int_method, SurfaceInputs& S, int domain) {
  Records R(bulkp);
  R.begin();
  S.ndom = R.i4();
  if (S.ndom < 1) throw std::runtime_error("bulkP.b: NDOM < 1");
  if (domain < 0 || domain >= S.ndom) throw std::runtime_error("domain index out of range");
  S.domain = domain;
  R.begin();
  int inegpos = R.i4();
  R.i4();  // isym
  int nh = R.i4(), nk = R.i4(), iabr = R.i4();
  R.i4();  // iabp
  R.i4();  // iabe
  S.nabr = R.i4();
  S.nabi = R.i4();
  R.i4();  // idiag
  R.begin();
  std::vector<int> nbd(S.ndom);
  S.rdom.assign(S.ndom, 0.0);
  int nbt = 0;
  for (int i = 0; i < S.ndom; ++i) {
    nbd[i] = R.i4();
    S.rdom[i] = R.r8();
    nbt += nbd[i];
  }
  S.nbd = nbd;
  S.nh = nh;
  S.nk = nk;
  R.begin();
  std::vector<int> ih(nbt), ik(nbt);
  for (int j = 0; j < nbt; ++j) {
    ih[j] = R.i4();
    ik[j] = R.i4();
  }
  R.begin();
  double be = R.r8();
  S.azi = R.r8();
  S.daz = R.r8();
  S.naz = R.i4();
  S.gi = R.r8();
  S.dg = R.r8();
  S.ng = R.i4();
  R.begin();
  double tem = R.r8(), dzb = R.r8();
  R.i4();  // ml
  R.r8();  // epsb
  R.begin();
  int nsgb = R.i4();
  R.i4();  // mp
  double aa = R.r8(), bb = R.r8(), gam = R.r8();
  S.gam = gam;
  S.cc = R.r8();
  double dxb = R.r8(), dyb = R.r8(), zoffset = R.r8();
  R.begin();
  int nelmb = R.i4();
  S.natmb = R.i4();

  ListInput T(surf);
  int nelms = T.integer();
  S.nelm = nelmb + nelms;
  const int nelm = S.nelm, mab = kMab;
  std::vector<double> a((size_t)mab * nelm, 0.0), c((size_t)mab * nelm, 0.0);
  S.b.assign((size_t)mab * nelm, 0.0);
  std::vector<double> dth(nelm), dtk(nelm), dtz(nelm), elm(nelm);
  S.dchg.assign(nelm, 0.0);
  auto A = [&](int j, int i) -> double& { return a[(size_t)i * mab + j]; };
  auto B = [&](int j, int i) -> double& { return S.b[(size_t)i * mab + j]; };
  for (int i = 0; i < nelmb; ++i) {
    R.begin();
    for (int j = 0; j < S.nabr + S.nabi; ++j) A(j, i) = R.r8();
    for (int j = 0; j < S.nabr + S.nabi; ++j) B(j, i) = R.r8();
    R.begin();
    dth[i] = R.r8();
    dtk[i] = R.r8();
    dtz[i] = R.r8();
    elm[i] = R.r8();
    S.dchg[i] = R.r8();
  }
  for (int i = nelmb; i < nelm; ++i) {
    auto v = T.values(3);
    int iz = std::stoi(v[0]);
    double da1 = ListInput::real(v[1]), sap = ListInput::real(v[2]);
    elm[i] = (iz >= 1 && iz <= 110) ? trhepd_tables::kAtomicMass[iz - 1] : 1000.0;
    double a4[4], b4[4];
    int nr = form_factor_params(iz, iabr, a4, b4);
    if (nr <= 0) throw std::runtime_error("surf.txt: element without scattering factors");
    S.nabr = nr;
    for (int j = 0; j < 4; ++j) {
      A(j, i) = a4[j];
      B(j, i) = b4[j];
    }
    A(0, i) -= da1;  // electron (surfio.f90:151)
    if (inegpos > 0)
      for (int j = 0; j < S.nabr; ++j) A(j, i) = -A(j, i);  // positron (surfio.f90:152)
    S.nabi = 1;
    A(S.nabr, i) = sap;
    B(S.nabr, i) = 0.0;
    auto d = T.values(3);
    dth[i] = std::fabs(ListInput::real(d[0]));
    dtk[i] = std::fabs(ListInput::real(d[1]));
    dtz[i] = std::fabs(ListInput::real(d[2]));
  }
  auto cell = T.values(8);
  int nsgs = std::stoi(cell[0]), msa = std::stoi(cell[1]), msb = std::stoi(cell[2]);
  int nsa = std::stoi(cell[3]), nsb = std::stoi(cell[4]);
  double dthick = ListInput::real(cell[5]), dxs = ListInput::real(cell[6]),
         dys = ListInput::real(cell[7]);
  S.natms = T.integer();
  const int natm = S.natmb + S.natms;
  S.ielm.resize(natm);
  S.ocr.resize(natm);
  S.z.resize(natm);
  std::vector<double> x(natm), y(natm);
  for (int i = 0; i < S.natmb; ++i) {
    R.begin();
    S.ielm[i] = R.i4();
    S.ocr[i] = R.r8();
    x[i] = R.r8();
    y[i] = R.r8();
    S.z[i] = R.r8();
  }
  for (int i = S.natmb; i < natm; ++i) {
    auto v = T.values(5);
    int ie = std::stoi(v[0]);
    S.ocr[i] = ListInput::real(v[1]);
    x[i] = ListInput::real(v[2]);
    y[i] = ListInput::real(v[3]);
    S.z[i] = ListInput::real(v[4]) + zoffset;
    if (ie >= -nelmb && ie <= -1)
      S.ielm[i] = -ie;
    else if (ie >= 1 && ie <= nelms)
      S.ielm[i] = ie + nelmb;
    else
      throw std::runtime_error("surf.txt: atom element index out of range");
  }
  // domain weights (surfio.f90:186-190)
  S.wdom.assign(S.ndom, 1.0);
  if (S.ndom > 1) {
    auto w = T.values(S.ndom);
    for (int i = 0; i < S.ndom; ++i) S.wdom[i] = ListInput::real(w[i]);
  }
  S.ih_all = ih;
  S.ik_all = ik;
  // surface slices (surfio.f90:198-210)
  if (nsgs < 1) {
    S.ns = 0;
    S.dz = dzb;
  } else {
    double zz = 0.0;
    for (int i = S.natmb; i < natm; ++i) zz = std::max(zz, S.z[i]);
    int ns2 = (int)((zz + dthick + S.cc) / dzb) + 1;
    S.ns = (int)std::lround((dzb * ns2) / dz2);
    if (S.ns < 1) throw std::runtime_error("surface slice count < 1");
    S.dz = (dzb * ns2) / S.ns;
  }
  // energy / Debye-Waller correction (asfcrr, scpot.f90:11-58)
  S.smesh = std::fabs((double)(msa * nsb - msb * nsa));
  {
    const double pi = kPi, c2m = 511.001, ek = .262466;
    double area = aa * bb * std::sin(gam) * S.smesh;
    S.wn = std::sqrt(1e3 * be * ek * (1.0 + 0.5 * be / c2m));
    double s4 = 4.0 * pi / area, rel = (1.0 + be / c2m) * s4;
    double rat = std::sqrt(100.0 / be * (1.0 + 50.0 / c2m) / (1.0 + be * 0.5 / c2m)) * s4;
    double vib = 11407.0 * tem;
    for (int i = 0; i < nelm; ++i) {
      double dwz;
      if (tem > 1e-5) {
        dwz = vib / (dtz[i] * dtz[i] * elm[i]);
        dth[i] = std::sqrt((vib + vib) / elm[i]) / (4.0 * pi * dth[i]);
        dtk[i] = std::sqrt((vib + vib) / elm[i]) / (4.0 * pi * dtk[i]);
      } else if (tem < -1e-5) {
        dwz = (8.0 * pi * pi) * dtz[i] * dtz[i];
      } else {
        dwz = dtz[i];
        dth[i] = std::sqrt(dth[i] * 0.5) / (pi + pi);
        dtk[i] = std::sqrt(dtk[i] * 0.5) / (pi + pi);
      }
      for (int j = 0; j < S.nabr; ++j) {
        c[(size_t)i * mab + j] = B(j, i) / (-16.0 * pi * pi);
        A(j, i) = A(j, i) * std::sqrt(4.0 * pi / (B(j, i) + dwz)) * rel;
        B(j, i) = -4.0 * pi * pi / (B(j, i) + dwz);
      }
      if (std::fabs(S.dchg[i]) > 1e-4) S.dchg[i] = S.dchg[i] * 1.88972619 * rel;
      if (S.nabi >= 2)
        for (int j = S.nabr; j < S.nabr + S.nabi; ++j) {
          c[(size_t)i * mab + j] = B(j, i) / (-16.0 * pi * pi);
          A(j, i) = A(j, i) * std::sqrt(4.0 * pi / B(j, i)) * rat;
          B(j, i) = -4.0 * pi * pi / B(j, i);
        }
    }
    S.ghx = (pi + pi) / (aa * nh);
    S.ghy = -(pi + pi) / (aa * std::tan(gam) * nh);
    S.gky = (pi + pi) / (bb * std::sin(gam) * nk);
  }
  // the records of the domains before `domain` (surfio.f90:291-300 and the bulk
  // records srfref reads, surflf.f90:65-72), skipped
  int ibt = 0;
  for (int d = 0; d < domain; ++d) {
    R.begin();  // iord
    R.begin();
    const int ngr = R.i4();
    R.i4();     // nvb
    R.begin();  // nbg
    R.begin();  // igh, igk
    for (int r = 0; r < S.naz * S.ng * ngr; ++r) R.begin();
    ibt += nbd[d];
  }
  S.azi += S.rdom[domain];
  // this domain: beam tables and bulk records
  S.nb = nbd[domain];
  S.ih.assign(ih.begin() + ibt, ih.begin() + ibt + S.nb);
  S.ik.assign(ik.begin() + ibt, ik.begin() + ibt + S.nb);
  R.begin();
  S.iord.resize(S.nb);
  for (int i = 0; i < S.nb; ++i) S.iord[i] = R.i4();
  R.begin();
  S.ngr = R.i4();
  S.nvb = R.i4();
  const int nvm = 1 + S.nb * (S.nb - 1) / 2;
  if (S.nvb > nvm) throw std::runtime_error("bulkP.b: nvb exceeds beam pairs");
  R.begin();
  S.nbg.resize(S.ngr);
  for (int i = 0; i < S.ngr; ++i) S.nbg[i] = R.i4();
  R.begin();
  std::vector<int> igh(nvm, 0), igk(nvm, 0);
  for (int i = 0; i < S.nvb; ++i) {
    igh[i] = R.i4();
    igk[i] = R.i4();
  }
  // srfghk (surfsub.f90:9-41): beam-difference index of every pair l > k
  S.iv.assign((size_t)S.nb * S.nb, 0);
  {
    int nv = S.nvb;
    for (int k = 0; k < S.nb - 1; ++k)
      for (int l = k + 1; l < S.nb; ++l) {
        int dh = S.ih[l] - S.ih[k], dk = S.ik[l] - S.ik[k], m = 1;
        for (; m < nv; ++m)
          if (igh[m] == dh && igk[m] == dk) break;
        if (m == nv) {
          if (nv + 1 > nvm) throw std::runtime_error("srfghk: nv exceeds beam pairs");
          igh[nv] = dh;
          igk[nv] = dk;
          ++nv;
        }
        S.iv[(size_t)k * S.nb + l] = m + 1;
      }
    S.nv = nv;
  }
  // asfcef (scpot.f90:62-95)
  const int nv = S.nv;
  S.asf.assign((size_t)nv * mab * nelm, 0.0);
  S.Ghk.assign(nv, 0.0);
  {
    std::vector<double> s(nv), sj(nv);
    for (int k = 0; k < nv; ++k) {
      double gx = S.ghx * igh[k], gy = S.ghy * igh[k] + S.gky * igk[k];
      s[k] = gx * gx + gy * gy;
    }
    for (int j = 0; j < nelm; ++j) {
      for (int k = 0; k < nv; ++k) {
        double gx = dth[j] * S.ghx * igh[k], gy = dth[j] * S.ghy * igh[k] + dtk[j] * S.gky * igk[k];
        sj[k] = -0.5 * (gx * gx + gy * gy);
      }
      for (int i = 0; i < S.nabr; ++i)
        for (int k = 0; k < nv; ++k)
          S.asf[((size_t)j * mab + i) * nv + k] =
              A(i, j) * std::exp(c[(size_t)j * mab + i] * s[k] + sj[k]);
      if (S.nabi >= 2)
        for (int i = S.nabr; i < S.nabr + S.nabi; ++i)
          for (int k = 0; k < nv; ++k)
            S.asf[((size_t)j * mab + i) * nv + k] =
                A(i, j) * std::exp(c[(size_t)j * mab + i] * s[k] + sj[k] * 0.5);
    }
    for (int k = 0; k < nv; ++k) S.Ghk[k] = std::sqrt(s[k]);
    if (S.nabi == 1)
      for (int j = 0; j < nelm; ++j) S.asf[((size_t)j * mab + S.nabr) * nv] = A(S.nabr, j);
  }
  // plane-group images for the structure factors (scpot_stf, surfio.f90:324-326);
  // the sums themselves are formed on the GPU (trhepd_structure_factors).
  {
    const double pi = kPi;
    S.gh.resize(nv);
    S.gk.resize(nv);
    for (int i = 0; i < nv; ++i) {
      S.gh[i] = (-(pi + pi) / nh) * (double)igh[i];
      S.gk[i] = (-(pi + pi) / nk) * (double)igk[i];
    }
    auto fill = [&](StructureFactorJob& J, int nk_, int first, int count, int nsg, int ma,
                    int mb, int na, int nb_, double dx, double dy) {
      J.nk = nk_;
      J.natm = count;
      J.dx = dx;
      J.dy = dy;
      J.img.assign((size_t)count * 24, 0.0);
      J.nimg.assign(count, 0);
      for (int j = 0; j < count; ++j)
        J.nimg[j] = plane_group_images(nsg, ma, mb, na, nb_, x[first + j], y[first + j],
                                       &J.img[(size_t)j * 24]);
    };
    fill(S.stf[0], nv, S.natmb, S.natms, nsgs, msa, msb, nsa, nsb, dxs + dxb, dys + dyb);
    fill(S.stf[1], S.nvb, 0, S.natmb, nsgb, 1, 0, 0, 1, dxb, dyb);
    fill(S.stf[2], S.nvb, 0, S.natmb, nsgb, 1, 0, 0, 1, 0.0, 0.0);
  }
  // bulk records for every (azimuth, angle) (surflf.f90:65-72)
  {
    size_t per = 0;
    for (int l = 0; l < S.ngr; ++l) per += (size_t)S.nbg[l] * S.nbg[l];
    int nrep = S.naz * S.ng;
    S.t1rec.resize(per * nrep);
    size_t o = 0;
    for (int r = 0; r < nrep; ++r)
      for (int l = 0; l < S.ngr; ++l) {
        R.begin();
        for (size_t e = 0; e < (size_t)S.nbg[l] * S.nbg[l]; ++e) {
          double re = R.r8(), im = R.r8();
          S.t1rec[o++] = cd{re, im};
        }
      }
  }
  S.int_method = int_method;
}

}  // namespace trhepd
