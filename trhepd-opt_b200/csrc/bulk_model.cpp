// bulk.txt parsing and bulkP.b writing for the GPU bulk solve
// (sim-trhepd-rheed/src/bulkio.f90:10-223, bulksub.f90:9-135).
#include "bulk_model.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "fortran_text.h"

namespace trhepd {

using namespace ftext;

namespace {

const double kPi = std::atan(1.0) * 4.0;

class RecWriter {
 public:
  explicit RecWriter(const std::string& p) : f_(std::fopen(p.c_str(), "wb")) {
    if (!f_) throw std::runtime_error("cannot write " + p);
  }
  ~RecWriter() {
    if (f_) std::fclose(f_);
  }
  template <class T>
  void put(T v) {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
    buf_.insert(buf_.end(), b, b + sizeof(T));
  }
  void end() {
    int32_t n = (int32_t)buf_.size();
    std::fwrite(&n, 4, 1, f_);
    if (n) std::fwrite(buf_.data(), 1, buf_.size(), f_);
    std::fwrite(&n, 4, 1, f_);
    buf_.clear();
  }

 private:
  FILE* f_;
  std::vector<unsigned char> buf_;
};

}  // namespace

void load_bulk_inputs(const std::string& path, BulkInputs& B, int inegpos, int domain) {
  B.inegpos = inegpos > 0 ? 1 : 0;
  ListInput T(path);
  auto h3 = T.values(3);
  B.nh = std::stoi(h3[0]);
  B.nk = std::stoi(h3[1]);
  B.ndom = std::stoi(h3[2]);
  if (B.nh < 1 || B.nk < 1) throw std::runtime_error("bulk.txt: NH, NK must be >= 1");
  if (B.ndom < 1) throw std::runtime_error("bulk.txt: NDOM < 1");
  if (domain < 0 || domain >= B.ndom) throw std::runtime_error("domain index out of range");
  B.domain = domain;
  // bulkio.f90:34-50: beams per domain, domain angles, each domain's beams
  auto nbv = T.values(B.ndom);
  B.nbd.resize(B.ndom);
  for (int d = 0; d < B.ndom; ++d) {
    B.nbd[d] = std::stoi(nbv[d]);
    if (B.nbd[d] < 1) throw std::runtime_error("bulk.txt: NB < 1");
  }
  auto rv = T.values(B.ndom);
  B.rdom_all.resize(B.ndom);
  std::vector<double> rdom_deg(B.ndom);
  for (int d = 0; d < B.ndom; ++d) {
    rdom_deg[d] = ListInput::real(rv[d]);
    B.rdom_all[d] = rdom_deg[d] * (kPi / 180.0);
  }
  B.ih_all.clear();
  B.ik_all.clear();
  for (int d = 0; d < B.ndom; ++d) {
    auto bk = T.values(2 * B.nbd[d]);
    for (int j = 0; j < B.nbd[d]; ++j) {
      B.ih_all.push_back(std::stoi(bk[2 * j]));
      B.ik_all.push_back(std::stoi(bk[2 * j + 1]));
    }
  }
  int ibt = 0;
  for (int d = 0; d < domain; ++d) ibt += B.nbd[d];
  B.nb = B.nbd[domain];
  B.rdom = B.rdom_all[domain];
  B.ih.assign(B.ih_all.begin() + ibt, B.ih_all.begin() + ibt + B.nb);
  B.ik.assign(B.ik_all.begin() + ibt, B.ik_all.begin() + ibt + B.nb);
  auto sc = T.values(7);
  double be = ListInput::real(sc[0]), azi = ListInput::real(sc[1]), azf = ListInput::real(sc[2]);
  double daz = ListInput::real(sc[3]), gi = ListInput::real(sc[4]), gf = ListInput::real(sc[5]);
  double dg = ListInput::real(sc[6]);
  auto dm = T.values(2);
  double dz = ListInput::real(dm[0]);
  B.ml = std::stoi(dm[1]);
  if (B.ml < 1 || B.ml > 1000) B.ml = 1000;
  B.be = be;
  // scanrg (bulksub.f90:9-42)
  const double rad = std::atan(1.0) / 45.0;
  B.naz = (std::fabs(daz) < 1e-4) ? 1 : std::min(std::max((int)((azf - azi) / daz + 0.1) + 1, 1), 200);
  B.ng = (std::fabs(dg) < 1e-4) ? 1 : std::min(std::max((int)((gf - gi) / dg + .1) + 1, 1), 200);
  B.azi = azi * rad;
  B.daz = daz * rad;
  B.gi = gi * rad;
  B.dg = dg * rad;
  B.nelm = T.integer();
  if (B.nelm < 1) throw std::runtime_error("bulk.txt: NELM < 1");
  const int nelm = B.nelm, mab = kMab;
  std::vector<double> a((size_t)mab * nelm, 0.0), b((size_t)mab * nelm, 0.0),
      c((size_t)mab * nelm, 0.0);
  B.dth_raw.resize(nelm);
  B.dtk_raw.resize(nelm);
  B.dtz_raw.resize(nelm);
  B.elm.resize(nelm);
  B.dchg.assign(nelm, 0.0);
  for (int i = 0; i < nelm; ++i) {
    auto v = T.values(3);
    int iz = std::stoi(v[0]);
    double da1 = ListInput::real(v[1]), sap = ListInput::real(v[2]);
    B.elm[i] = atomic_mass(iz);
    double a4[4], b4[4];
    int nr = form_factor_params(iz, B.iabr, a4, b4);
    if (nr <= 0) throw std::runtime_error("bulk.txt: element without scattering factors");
    B.nabr = nr;
    for (int j = 0; j < 4; ++j) {
      a[(size_t)i * mab + j] = a4[j];
      b[(size_t)i * mab + j] = b4[j];
    }
    a[(size_t)i * mab] -= da1;                                     // bulkio.f90:73
    if (B.inegpos > 0)                                             // positron: bulkio.f90:74
      for (int j = 0; j < B.nabr; ++j) a[(size_t)i * mab + j] *= -1.0;
    B.nabi = 1;
    a[(size_t)i * mab + B.nabr] = sap;
    b[(size_t)i * mab + B.nabr] = 0.0;
    auto d = T.values(3);
    B.dth_raw[i] = std::fabs(ListInput::real(d[0]));
    B.dtk_raw[i] = std::fabs(ListInput::real(d[1]));
    B.dtz_raw[i] = std::fabs(ListInput::real(d[2]));
  }
  B.a_raw.clear();
  B.b_raw.clear();
  for (int i = 0; i < nelm; ++i)
    for (int j = 0; j < B.nabr + B.nabi; ++j) {
      B.a_raw.push_back(a[(size_t)i * mab + j]);
      B.b_raw.push_back(b[(size_t)i * mab + j]);
    }
  auto st = T.values(7);
  B.nsg = std::stoi(st[0]);
  B.aa = ListInput::real(st[1]);
  B.bb = ListInput::real(st[2]);
  B.gam = ListInput::real(st[3]) * (kPi / 180.0);
  B.cc = ListInput::real(st[4]);
  B.dx = ListInput::real(st[5]);
  B.dy = ListInput::real(st[6]);
  if (B.ndom > 1) {  // rotated domains need a square or hexagonal cell (bulkio.f90:87-99)
    const double gdeg = ListInput::real(st[3]);
    if (std::fabs(B.aa - B.bb) > 1e-4)
      throw std::runtime_error("bulk.txt: NDOM > 1 needs AA = BB");
    const double step = std::fabs(gdeg - 90.0) < 1e-4 ? 90.0
                        : std::fabs(gdeg - 120.0) < 1e-4 ? 60.0 : 0.0;
    if (step == 0.0) throw std::runtime_error("bulk.txt: NDOM > 1 needs GAM = 90 or 120");
    for (int d = 0; d < B.ndom; ++d)
      if (std::fabs(rdom_deg[d] / step - std::nearbyint(rdom_deg[d] / step)) > 1e-4)
        throw std::runtime_error("bulk.txt: domain angle not a multiple of the cell symmetry");
  }
  B.natm = T.integer();
  if (B.natm < 1) throw std::runtime_error("bulk.txt: NATM < 1");
  B.ielm.resize(B.natm);
  B.ocr.resize(B.natm);
  B.x.resize(B.natm);
  B.y.resize(B.natm);
  B.z.resize(B.natm);
  double zmin = 1e10, zmax = -1e10;
  for (int i = 0; i < B.natm; ++i) {
    auto v = T.values(5);
    B.ielm[i] = std::stoi(v[0]);
    B.ocr[i] = ListInput::real(v[1]);
    B.x[i] = ListInput::real(v[2]);
    B.y[i] = ListInput::real(v[3]);
    B.z[i] = ListInput::real(v[4]);
    if (B.ielm[i] < 1 || B.ielm[i] > nelm) throw std::runtime_error("bulk.txt: IELM out of range");
    zmin = std::min(zmin, B.z[i]);
    zmax = std::max(zmax, B.z[i]);
  }
  B.zoffset = 0.5 * (B.cc - zmax - zmin);
  for (double& zz : B.z) zz += B.zoffset;
  B.ns = (int)(B.cc / dz) + 1;
  B.dz = B.cc / B.ns;
  if (B.ns < 2) throw std::runtime_error("bulk.txt: fewer than 2 slices");
  // asfcrr (scpot.f90:11-58) on the 1x1 cell, tem = 0
  {
    const double pi = kPi, c2m = 511.001, ek = .262466;
    B.wn = std::sqrt(1e3 * be * ek * (1.0 + 0.5 * be / c2m));
    double s4 = 4.0 * pi / (B.aa * B.bb * std::sin(B.gam)), rel = (1.0 + be / c2m) * s4;
    std::vector<double> dth(B.dth_raw), dtk(B.dtk_raw);
    for (int i = 0; i < nelm; ++i) {
      double dwz = B.dtz_raw[i];
      dth[i] = std::sqrt(dth[i] * 0.5) / (pi + pi);
      dtk[i] = std::sqrt(dtk[i] * 0.5) / (pi + pi);
      for (int j = 0; j < B.nabr; ++j) {
        double& A = a[(size_t)i * mab + j];
        double& Bc = b[(size_t)i * mab + j];
        c[(size_t)i * mab + j] = Bc / (-16.0 * pi * pi);
        A = A * std::sqrt(4.0 * pi / (Bc + dwz)) * rel;
        Bc = -4.0 * pi * pi / (Bc + dwz);
      }
    }
    B.ghx = (pi + pi) / (B.aa * B.nh);
    B.ghy = -(pi + pi) / (B.aa * std::tan(B.gam) * B.nh);
    B.gky = (pi + pi) / (B.bb * std::sin(B.gam) * B.nk);
    B.bcoef = b;
    // blkibg (bulksub.f90:46-92): groups of coupled beams, sorted beam order
    B.ihs = B.ih;
    B.iks = B.ik;
    B.iord.resize(B.nb);
    for (int i = 0; i < B.nb; ++i) B.iord[i] = i + 1;
    B.nbg.clear();
    if (B.nh == 1 && B.nk == 1) {
      B.nbg.push_back(B.nb);
    } else {
      int j = 1;
      while (true) {
        int i0 = j;
        j = i0 + 1;
        int ih0 = B.ihs[i0 - 1], ik0 = B.iks[i0 - 1];
        for (int k = i0 + 1; k <= B.nb; ++k) {
          if ((B.ihs[k - 1] - ih0) % B.nh == 0 && (B.iks[k - 1] - ik0) % B.nk == 0) {
            if (k > j) {
              int l = B.ihs[k - 1], n = B.iks[k - 1], m = B.iord[k - 1];
              for (int jj = k; jj >= j + 1; --jj) {
                B.ihs[jj - 1] = B.ihs[jj - 2];
                B.iks[jj - 1] = B.iks[jj - 2];
                B.iord[jj - 1] = B.iord[jj - 2];
              }
              B.ihs[j - 1] = l;
              B.iks[j - 1] = n;
              B.iord[j - 1] = m;
            }
            ++j;
          }
        }
        B.nbg.push_back(j - i0);
        if (j > B.nb) break;
      }
    }
    B.ngr = (int)B.nbg.size();
    B.nbgm = *std::max_element(B.nbg.begin(), B.nbg.end());
    // blkghk (bulksub.f90:96-135)
    B.igh.assign(1, 0);
    B.igk.assign(1, 0);
    B.iv.assign((size_t)B.nbgm * B.nb, 0);
    int ibas = 0;
    for (int g = 0; g < B.ngr; ++g) {
      int iend = ibas + B.nbg[g];
      for (int k = ibas; k < iend - 1; ++k)
        for (int l = k + 1; l < iend; ++l) {
          int dh = B.ihs[l] - B.ihs[k], dk = B.iks[l] - B.iks[k], m = 1;
          for (; m < (int)B.igh.size(); ++m)
            if (B.igh[m] == dh && B.igk[m] == dk) break;
          if (m == (int)B.igh.size()) {
            B.igh.push_back(dh);
            B.igk.push_back(dk);
          }
          B.iv[(size_t)k * B.nbgm + (l - ibas)] = m + 1;
        }
      ibas = iend;
    }
    B.nv = (int)B.igh.size();
    // asfcef (scpot.f90:62-95)
    const int nv = B.nv;
    B.asf.assign((size_t)nv * mab * nelm, 0.0);
    B.Ghk.assign(nv, 0.0);
    std::vector<double> s(nv);
    for (int k = 0; k < nv; ++k) {
      double gx = B.ghx * B.igh[k], gy = B.ghy * B.igh[k] + B.gky * B.igk[k];
      s[k] = gx * gx + gy * gy;
    }
    for (int jj = 0; jj < nelm; ++jj) {
      for (int i = 0; i < B.nabr; ++i)
        for (int k = 0; k < nv; ++k) {
          double gx = dth[jj] * B.ghx * B.igh[k];
          double gy = dth[jj] * B.ghy * B.igh[k] + dtk[jj] * B.gky * B.igk[k];
          double sj = -0.5 * (gx * gx + gy * gy);
          B.asf[((size_t)jj * mab + i) * nv + k] =
              a[(size_t)jj * mab + i] * std::exp(c[(size_t)jj * mab + i] * s[k] + sj);
        }
      B.asf[((size_t)jj * mab + B.nabr) * nv] = a[(size_t)jj * mab + B.nabr];
    }
    for (int k = 0; k < nv; ++k) B.Ghk[k] = std::sqrt(s[k]);
    B.gh.resize(nv);
    B.gk.resize(nv);
    for (int k = 0; k < nv; ++k) {
      B.gh[k] = (-(pi + pi) / B.nh) * (double)B.igh[k];
      B.gk[k] = (-(pi + pi) / B.nk) * (double)B.igk[k];
    }
    const double sdx[3] = {0.0, -B.dx, B.dx}, sdy[3] = {0.0, -B.dy, B.dy};
    for (int p = 0; p < 3; ++p) {
      StructureFactorJob& J = B.stf[p];
      J.nk = nv;
      J.natm = B.natm;
      J.dx = sdx[p];
      J.dy = sdy[p];
      J.img.assign((size_t)B.natm * 24, 0.0);
      J.nimg.assign(B.natm, 0);
      for (int j = 0; j < B.natm; ++j)
        J.nimg[j] = plane_group_images(B.nsg, 1, 0, 0, 1, B.x[j], B.y[j], &J.img[(size_t)j * 24]);
    }
  }
}

void write_bulkp(const std::string& path, const std::vector<BulkInputs>& Bd,
                 const std::vector<std::vector<std::vector<cd>>>& records) {
  const BulkInputs& B = Bd.at(0);
  RecWriter W(path);
  W.put<int32_t>(B.ndom);
  W.end();
  for (int v : {B.inegpos, 0, B.nh, B.nk, B.iabr, 1, 0, B.nabr, B.nabi, 3}) W.put<int32_t>(v);
  W.end();
  for (int d = 0; d < B.ndom; ++d) {
    W.put<int32_t>(B.nbd[d]);
    W.put<double>(B.rdom_all[d]);
  }
  W.end();
  for (size_t i = 0; i < B.ih_all.size(); ++i) {
    W.put<int32_t>(B.ih_all[i]);
    W.put<int32_t>(B.ik_all[i]);
  }
  W.end();
  W.put<double>(B.be);
  W.put<double>(B.azi);
  W.put<double>(B.daz);
  W.put<int32_t>(B.naz);
  W.put<double>(B.gi);
  W.put<double>(B.dg);
  W.put<int32_t>(B.ng);
  W.end();
  W.put<double>(0.0);
  W.put<double>(B.dz);
  W.put<int32_t>(B.ml);
  W.put<double>(B.epsb);
  W.end();
  W.put<int32_t>(B.nsg);
  W.put<int32_t>(0);
  for (double v : {B.aa, B.bb, B.gam, B.cc, B.dx, B.dy, B.zoffset}) W.put<double>(v);
  W.end();
  W.put<int32_t>(B.nelm);
  W.put<int32_t>(B.natm);
  W.end();
  const int na = B.nabr + B.nabi;
  for (int i = 0; i < B.nelm; ++i) {
    for (int j = 0; j < na; ++j) W.put<double>(B.a_raw[(size_t)i * na + j]);
    for (int j = 0; j < na; ++j) W.put<double>(B.b_raw[(size_t)i * na + j]);
    W.end();
    for (double v : {B.dth_raw[i], B.dtk_raw[i], B.dtz_raw[i], B.elm[i], B.dchg[i]})
      W.put<double>(v);
    W.end();
  }
  for (int i = 0; i < B.natm; ++i) {
    W.put<int32_t>(B.ielm[i]);
    for (double v : {B.ocr[i], B.x[i], B.y[i], B.z[i]}) W.put<double>(v);
    W.end();
  }
  for (size_t d = 0; d < Bd.size(); ++d) {
    const BulkInputs& D = Bd[d];
    for (int i = 0; i < D.nb; ++i) W.put<int32_t>(D.iord[i]);
    W.end();
    W.put<int32_t>(D.ngr);
    W.put<int32_t>(D.nv);
    W.end();
    for (int g = 0; g < D.ngr; ++g) W.put<int32_t>(D.nbg[g]);
    W.end();
    for (int i = 0; i < D.nv; ++i) {
      W.put<int32_t>(D.igh[i]);
      W.put<int32_t>(D.igk[i]);
    }
    W.end();
    for (const auto& r : records.at(d)) {
      for (const cd& v : r) {
        W.put<double>(v.x);
        W.put<double>(v.y);
      }
      W.end();
    }
  }
}

}  // namespace trhepd
