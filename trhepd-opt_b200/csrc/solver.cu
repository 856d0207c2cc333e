// Batched multislice surface solve and the C ABI (include/trhepd_b200.h).
//
// One launch sequence integrates every (azimuth, glancing angle) of a domain at
// once: the angles' N x N states Q = X^H and P = Y^H are stacked row-wise, the
// shared stage matrix of each integrator stage is gathered once from the
// potential table and applied to all angles by one GEMM whose epilogue performs
// the RKN updates (surf_prkn.f90:278-330).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/trhepd_b200.h"
#include "bulk.h"
#include "magnus.h"
#include "bulk_model.h"
#include "curves.h"
#include "host_model.h"
#include "integrators.h"
#include "kernels.h"
#include "small.h"
#include "cholqr.h"
#include "split_gemm.h"

using namespace trhepd;

namespace {

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess)                                                                 \
      throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_),                     \
                      e_ == cudaErrorMemoryAllocation ? TRHEPD_ENOMEM : TRHEPD_ECUDA);     \
  } while (0)

// Device memory is stream-ordered (cudaMallocAsync / cudaFreeAsync from the
// device's default pool) on the stream of the call in progress: cudaFree would
// synchronise the whole device, so a context growing or freeing a buffer would
// wait for every kernel other contexts have queued (a small serving request
// behind a large one).  Buffers are only used on the stream that allocated them.
thread_local cudaStream_t t_alloc_stream = nullptr;

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  void* ensure(size_t bytes) {
    if (bytes <= n && p) return p;
    if (p) cudaFreeAsync(p, t_alloc_stream);
    p = nullptr;
    n = 0;
    if (bytes == 0) bytes = 256;
    CK(cudaMallocAsync(&p, bytes, t_alloc_stream));
    n = bytes;
    return p;
  }
  void release() {
    if (p) cudaFreeAsync(p, t_alloc_stream);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

template <class T>
T* upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return b.as<T>();
}

}  // namespace

struct trhepd_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  int renorm_policy = 0;
  double renorm_tau = std::log(1e3);
  int split_slices = 5;           // 5 INT8 digits (39 bits) meet 1e-6 per spot at N = 521
  int split_variant = kSplitPersistent;
  int profile = 0;               // 1: time every stage-product launch with events
  int graphs = 1;                // 1: replay resident solves from a captured CUDA graph
  int fused_max_n = kFusedMaxBeams;  // FP64 RKN solves with n <= this run fused (0: never)
  int validate = 0;              // 1: split solves also run the FP64 form (per-curve errors)
  int particle = 0;              // trhepd_bulk_run: 0 positrons, 1 electrons
  int max_ctas = 0;              // persistent split kernels: CTA cap (0: one per SM, -1: one per tile)
  double stats[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<double> curve_err; // 3 per angle of the last validated solve (curves.h)
  std::vector<cudaEvent_t> evpool;
  std::vector<cudaEvent_t> rnpool;  // profile mode: pairs around renormalisations
  // device buffers (grown on demand, reused across calls)
  DevBuf asf, b, dchg, ghk, z[3], ocr[3], ielm[3], st[3], depth, table, pair;
  DevBuf Q0, Q1, P, V, D, gam, F, flags, dval, gj, f2, wnsga2, status, split;
  DevBuf sgh, sgk, simg, snimg, sst;
  DevBuf cva, cvf, cvo;  // rocking-curve convolution of host curves
  DevBuf cerr, cref;     // per-curve errors / distances, reference curves of a comparison
  DevBuf bk[24];  // bulk-solve work arrays
  DevBuf rk[5];   // RK4 / Magnus stage buffers
  DevBuf mg[9];   // Magnus shared matrices
};

namespace {

bool valid_precision(int p) {
  return p == TRHEPD_FP64 || p == TRHEPD_SPLIT_BF16 || p == TRHEPD_SPLIT_INT8;
}

int fail(trhepd_context* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

// Upload mod_scpot3 and build the stage table on the device.
void build_table(trhepd_context* C, const trhepd_pot_state& pot, const std::vector<double>& depth,
                 DevBuf& out, TableEntry** table_out) {
  cudaStream_t st = C->stream;
  const int nv = pot.nv, nelm = pot.nelm;
  const int natm = pot.natmb + pot.natms;
  // the table kernel stages natms + 2*natmb atom factors in shared memory
  if (pot.natms + 2 * pot.natmb > 512)
    throw std::invalid_argument("natms + 2*natmb exceeds 512 (potential table limit)");
  (void)natm;
  if (pot.nabr + pot.nabi > kMab || pot.nabr > 6) throw std::invalid_argument("nabr+nabi > 6");
  auto up = [&](DevBuf& b, const void* src, size_t bytes) {
    b.ensure(std::max<size_t>(bytes, 16));
    if (bytes) CK(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, st));
    return b.p;
  };
  PotInputs in{};
  in.asf = (const double*)up(C->asf, pot.asf, (size_t)nv * kMab * nelm * sizeof(double));
  in.b = (const double*)up(C->b, pot.b, (size_t)kMab * nelm * sizeof(double));
  in.dchg = (const double*)up(C->dchg, pot.dchg, (size_t)nelm * sizeof(double));
  in.ghk = (const double*)up(C->ghk, pot.Ghk, (size_t)nv * sizeof(double));
  in.nv = nv;
  in.nelm = nelm;
  in.nabr = pot.nabr;
  in.nabi = pot.nabi;
  in.mab = kMab;
  // parts: surface at zi - cc (all nv), top bulk at zi, second bulk at zi + cc (nvb)
  const int first[3] = {pot.natmb, 0, 0};
  const int count[3] = {pot.natms, pot.natmb, pot.natmb};
  const double shift[3] = {-pot.cc, 0.0, pot.cc};
  const double mesh[3] = {1.0, pot.smesh, pot.smesh};
  const int nk[3] = {nv, pot.nvb, pot.nvb};
  const double* stp[3] = {pot.st0, pot.st1, pot.st2};
  for (int p = 0; p < 3; ++p) {
    std::vector<int> ie(count[p]);
    for (int j = 0; j < count[p]; ++j) {
      int e = pot.ielm[first[p] + j];
      if (e < 1 || e > nelm) throw std::invalid_argument("ielm out of range");
      ie[j] = e - 1;
    }
    PotPart& P = in.part[p];
    P.z = (const double*)up(C->z[p], pot.z + first[p], count[p] * sizeof(double));
    P.ocr = (const double*)up(C->ocr[p], pot.ocr + first[p], count[p] * sizeof(double));
    P.ielm = upload(C->ielm[p], ie, st);
    P.st = (const cd*)up(C->st[p], stp[p], (size_t)nk[p] * count[p] * sizeof(cd));
    P.natm = count[p];
    P.nk = nk[p];
    P.zshift = shift[p];
    P.rmesh = mesh[p];
  }
  const double* dd = upload(C->depth, depth, st);
  int ncol = (int)depth.size();
  TableEntry* table = (TableEntry*)out.ensure((size_t)ncol * nv * sizeof(TableEntry));
  launch_potential_table(in, dd, ncol, table, st);
  CK(cudaGetLastError());
  *table_out = table;
}

struct SolveArgs {
  const trhepd_pot_state* pot;
  int nb, ns;
  const int32_t* iv;
  double dz;
  int ngr;
  const int32_t *nbg, *iord, *ih, *ik;
  double wn, ghx, ghy, gky, azi, daz, gi, dg;
  int naz, ng, int_method;
  const double* t1;
};

}  // namespace

namespace {

// Device buffers and counters of one integration of a resident problem.
struct RunState {
  int n = 0, ns = 0, nv = 0, nang = 0, ld = 0, kpad = 0;
  bool split = false;
  int split_variant = kSplitPersistent;
  cudaStream_t st = nullptr;
  const TableEntry* table = nullptr;
  const int* pair = nullptr;
  const cd* gam = nullptr;
  const cd* D = nullptr;
  size_t sbytes = 0;
  cd *Q = nullptr, *Qn = nullptr, *P = nullptr, *V = nullptr;
  int* flags = nullptr;
  double* dval = nullptr;
  void* gjs = nullptr;
  unsigned* status = nullptr;
  SplitWorkspace sw{};
  int interval = 1;          // renormalisation interval of the growth-bound policy
  long renorms = 0, products = 0, launches = 0, gj_launches = 0;
  int gj_per = 0;
  bool capturing = false;    // launches go into a CUDA graph: no events on the stream
  long prof_entries = 0;     // event quadruples recorded in profile mode
  long renorm_entries = 0;   // event pairs around renormalisations (profile mode)
  cd* gsx = nullptr;         // int_method 8: power-estimate vectors (nang x n)
  void* gss = nullptr;       // int_method 8: CholeskyQR scratch
  int nprob = 1;             // stacked problems (see trhepd_problem::nprob)
  const TableEntry* const* tables = nullptr;
  StackedRows sr{};          // rows and stage-matrix stride per stacked problem
};

// The device buffers one integration works in: the context's (one solve at a
// time) or a problem's own (problems solved together in a batch).
struct Workspace {
  DevBuf *Q0, *Q1, *P, *V, *flags, *dval, *gj, *status, *split;
};
struct OwnWorkspace {
  DevBuf Q0, Q1, P, V, flags, dval, gj, status, split;
  Workspace view() { return {&Q0, &Q1, &P, &V, &flags, &dval, &gj, &status, &split}; }
  void release() {
    for (DevBuf* b : {&Q0, &Q1, &P, &V, &flags, &dval, &gj, &status, &split}) b->release();
  }
};

}  // namespace

// Device-resident problem: stage table, beam-pair map, bulk boundary, gammas.
// Solving it reads only device memory; the result stays on the device until
// fetched.
struct trhepd_problem {
  int n = 0, ns = 0, nv = 0, nang = 0, ld = 0, nb0 = 0, int_method = 5;
  int nrep2 = 1;               // angles of the inner scan (rows per block of the output)
  // a stacked group (problems of one batch solved as one integration): nprob
  // problems of nang / nprob angles each, their stage tables in `tables` (device)
  int nprob = 1;
  const TableEntry* const* tables = nullptr;
  std::vector<int> pair_host;  // the beam-pair map, to recognise problems that stack
  Integrator I{};
  double dz = 0, kappa_max = 0;
  int ncol = 0;
  DevBuf table, pair, gam, D, F, wnsga2, f2, dang, conv;
  std::vector<double> angle_deg;
  // CUDA graphs of the whole solve, one per option set (`key`: precision form and
  // the options the launch sequence depends on), each valid for the context
  // buffers in its `sig`; `last_sig` holds the buffers of the slot's last
  // uncaptured solve.  A validated split solve alternates two option sets.
  struct GraphSlot {
    std::vector<double> key;
    std::vector<void*> sig, last_sig;
    cudaGraphExec_t exec = nullptr;
    RunState run;
    void drop() {
      if (exec) cudaGraphExecDestroy(exec);
      exec = nullptr;
      sig.clear();
    }
  };
  static constexpr size_t kGraphSlots = 4;
  std::vector<GraphSlot> graphs;
  OwnWorkspace own;            // buffers of batch solves (trhepd_batch_solve)
  DevBuf f2ref;                // FP64 intensities of a validated split solve
  void drop_graph() {
    for (GraphSlot& g : graphs) g.drop();
    graphs.clear();
  }
  // The slot of `key`, made (evicting the oldest) if there is none.
  GraphSlot& slot(const std::vector<double>& key) {
    for (GraphSlot& g : graphs)
      if (g.key == key) return g;
    if (graphs.size() >= kGraphSlots) {
      graphs.front().drop();
      graphs.erase(graphs.begin());
    }
    graphs.emplace_back();
    graphs.back().key = key;
    return graphs.back();
  }
  size_t bytes() const {
    return table.n + pair.n + gam.n + D.n + F.n + wnsga2.n + f2.n + f2ref.n;
  }
  void release() {
    drop_graph();
    own.release();
    for (DevBuf* b : {&table, &pair, &gam, &D, &F, &wnsga2, &f2, &dang, &conv, &f2ref})
      b->release();
  }
};

namespace {

// Upload inputs, build the stage table (K2/K3 outputs) and the per-angle data.
void prepare(trhepd_context* C, const SolveArgs& A, trhepd_problem& Pb) {
  const int n = A.nb, ns = A.ns;
  if (n < 1 || ns < 1) throw std::invalid_argument("nb and ns must be >= 1");
  if (n > kMaxBeams) throw std::invalid_argument("nb exceeds the GPU path limit");
  Pb.I = integrator_for(A.int_method);
  Pb.int_method = A.int_method;
  const std::vector<double> depth = stage_depths(Pb.I, ns, A.dz);
  cudaStream_t st = C->stream;
  TableEntry* table = nullptr;
  build_table(C, *A.pot, depth, Pb.table, &table);
  const int nv = A.pot->nv;
  Pb.n = n;
  Pb.ns = ns;
  Pb.nv = nv;
  Pb.dz = A.dz;
  Pb.ncol = (int)depth.size();

  // beam-pair map for the gather: pair[k*n+j] = iv(max,min) - 1
  std::vector<int> pair((size_t)n * n, 0);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j) {
      if (k == j) continue;
      int hi = std::max(k, j), lo = std::min(k, j);
      int e = A.iv[(size_t)lo * n + hi];
      if (e < 1 || e > nv) throw std::invalid_argument("iv entry out of range");
      pair[(size_t)k * n + j] = e - 1;
    }
  upload(Pb.pair, pair, st);
  Pb.pair_host = pair;

  // angle schedule (surflf.f90:43-92)
  const bool ng_outer = A.ng > A.naz;
  const int nrep1 = ng_outer ? A.naz : A.ng, nrep2 = ng_outer ? A.ng : A.naz;
  const int nang = nrep1 * nrep2;
  const int ld = round_up(n, 16);

  Pb.nang = nang;
  Pb.nrep2 = nrep2;
  Pb.ld = ld;
  std::vector<cd> gam((size_t)nang * n), Dm((size_t)nang * ld, cd{0, 0}), F((size_t)nang * n * n);
  std::vector<double> wnsga2(nang);
  Pb.angle_deg.assign(nang, 0.0);
  size_t per = 0;
  int sum = 0;
  for (int l = 0; l < A.ngr; ++l) {
    if (A.nbg[l] < 1) throw std::invalid_argument("nbg entries must be >= 1");
    per += (size_t)A.nbg[l] * A.nbg[l];
    sum += A.nbg[l];
  }
  if (sum != n) throw std::invalid_argument("sum(nbg) != nb");
  for (int i = 0; i < n; ++i)
    if (A.iord[i] < 1 || A.iord[i] > n) throw std::invalid_argument("iord out of range");
  double kappa_max = 0.0;
  for (int t = 0; t < nang; ++t) {
    int irep1 = t / nrep2, irep2 = t % nrep2;
    double ga, az;
    if (ng_outer) {
      az = A.azi + irep1 * A.daz;
      ga = A.gi + irep2 * A.dg;
    } else {
      ga = A.gi + irep1 * A.dg;
      az = A.azi + irep2 * A.daz;
    }
    double cga = std::cos(ga), sga = std::sin(ga), caz = std::cos(az), saz = std::sin(az);
    wnsga2[t] = A.wn * sga * sga;
    double wnx = A.wn * cga * caz, wny = A.wn * cga * saz;
    for (int i = 0; i < n; ++i) {
      double wgx = A.ghx * A.ih[i] + wnx;
      double wgy = A.ghy * A.ih[i] + A.gky * A.ik[i] + wny;
      double s = A.wn * A.wn - wgx * wgx - wgy * wgy;
      cd g = (s >= 0.0) ? cd{std::sqrt(s), 0.0} : cd{0.0, std::sqrt(-s)};
      gam[(size_t)t * n + i] = g;
      cd g2 = g * g;
      Dm[(size_t)t * ld + i] = cd{-g2.x, g2.y};  // -conj(g^2)
      if (s < 0) kappa_max = std::max(kappa_max, std::sqrt(-s));
    }
    Pb.angle_deg[t] = (ng_outer ? ga : az) * 180.0 / 3.141592654;
    // bulk f permuted by iord (surflf.f90:105-115); F row-major (i, j)
    const double* rec = A.t1 + 2 * per * t;
    cd* Ft = F.data() + (size_t)t * n * n;
    int ib1 = 0;
    size_t o = 0;
    for (int l = 0; l < A.ngr; ++l) {
      int m = A.nbg[l];
      for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i, ++o) {
          int r = A.iord[ib1 + i] - 1, c = A.iord[ib1 + j] - 1;
          Ft[(size_t)r * n + c] = cd{rec[2 * o], rec[2 * o + 1]};
        }
      ib1 += m;
    }
  }
  Pb.kappa_max = kappa_max;
  Pb.nb0 = 0;
  for (int i = 0; i < n; ++i)
    if (A.ih[i] == 0 && A.ik[i] == 0) Pb.nb0 = i;
  upload(Pb.gam, gam, st);
  upload(Pb.D, Dm, st);
  upload(Pb.F, F, st);
  upload(Pb.wnsga2, wnsga2, st);
  Pb.f2.ensure((size_t)nang * n * sizeof(double));
}


// Buffers, the boundary transform invstransh (matcomp.f90:140-172) and the
// renormalisation schedule; Q = I and P = P0 afterwards.
Workspace context_workspace(trhepd_context* C) {
  return {&C->Q0, &C->Q1, &C->P, &C->V, &C->flags, &C->dval, &C->gj, &C->status, &C->split};
}

void begin_run(trhepd_context* C, trhepd_problem& Pb, int precision, int nprod_max, RunState& R,
               const Workspace& W) {
  R.n = Pb.n;
  R.ns = Pb.ns;
  R.nv = Pb.nv;
  R.nang = Pb.nang;
  R.ld = Pb.ld;
  R.kpad = Pb.ld;
  R.st = C->stream;
  R.table = Pb.table.as<TableEntry>();
  R.pair = Pb.pair.as<int>();
  R.gam = Pb.gam.as<cd>();
  R.D = Pb.D.as<cd>();
  const int n = R.n, nang = R.nang, ld = R.ld;
  cudaStream_t st = R.st;
  R.sbytes = (size_t)nang * n * ld * sizeof(cd);
  R.Q = (cd*)W.Q0->ensure(R.sbytes);
  R.Qn = (cd*)W.Q1->ensure(R.sbytes);
  R.P = (cd*)W.P->ensure(R.sbytes);
  R.nprob = Pb.nprob;
  R.tables = Pb.tables;
  if (R.nprob > 1) R.sr = StackedRows{(nang / R.nprob) * n, (long long)(R.kpad + 1) * ld};
  R.V = (cd*)W.V->ensure((size_t)R.nprob * (R.kpad + 1) * ld * sizeof(cd));
  R.flags = (int*)W.flags->ensure(std::max(nang, 4) * sizeof(int));
  R.dval = (double*)W.dval->ensure(std::max(nang, 4) * sizeof(double));
  R.gjs = W.gj->ensure(gj_scratch_bytes(nang, n));
  R.status = (unsigned*)W.status->ensure(16);
  R.split = precision == TRHEPD_SPLIT_BF16 || precision == TRHEPD_SPLIT_INT8;
  R.split_variant = (precision == TRHEPD_SPLIT_INT8) ? kSplitInt8 : C->split_variant;
  if (precision == TRHEPD_SPLIT_BF16 && C->split_slices > 5)
    throw std::invalid_argument("the BF16 split form takes 3 to 5 slices");
  if (R.split)
    R.sw = split_workspace_carve(
        W.split->ensure(split_workspace_bytes(nang, n, C->split_slices, R.nprob)), nang, n,
        C->split_slices, R.status, st, R.nprob);
  R.sw.max_ctas = C->max_ctas;
  R.gj_per = 2 * ceil_div(n, 16);
  if (C->profile && (int)C->evpool.size() < 4 * nprod_max) {
    while ((int)C->evpool.size() < 4 * nprod_max) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      C->evpool.push_back(e);
    }
  }
  if (C->profile && (int)C->rnpool.size() < 2 * (Pb.ns + 2)) {
    while ((int)C->rnpool.size() < 2 * (Pb.ns + 2)) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      C->rnpool.push_back(e);
    }
  }
  if (!R.capturing) CK(cudaEventRecord(C->ev0, st));
  CK(cudaMemsetAsync(R.status, 0, 16, st));
  CK(cudaMemsetAsync(R.Q, 0, R.sbytes, st));
  CK(cudaMemsetAsync(R.Qn, 0, R.sbytes, st));
  CK(cudaMemsetAsync(R.P, 0, R.sbytes, st));
  if (Pb.I.gs) {
    // rk4_intgs (surf_rk.f90:106-109): invstrans, CholeskyQR of every angle, the
    // power-estimate vector initialised
    R.gsx = (cd*)C->mg[1].ensure((size_t)nang * n * sizeof(cd));
    R.gss = C->mg[0].ensure(cholqr_scratch_bytes(nang, n, ld));
    launch_invstrans_build(Pb.F.as<cd>(), R.Q, R.P, R.gam, nang, n, ld, st);
    launch_power_est(R.Q, R.P, R.gsx, R.flags, R.dval, nang, n, ld, -1, st);
    R.launches += 2 + launch_cholqr(R.Q, R.P, R.flags, nang, n, ld, R.gss, R.status, st);
    return;
  }
  // invstransh: Q = I + F^H, P = I - F^H; P <- Q^{-1} P; P <- i P conj(G); Q = I
  launch_invstransh_build(Pb.F.as<cd>(), R.Q, R.P, nang, n, ld, st);
  launch_gauss_jordan(R.Q, R.P, nullptr, nang, n, ld, R.gjs, R.status, st);
  launch_invstransh_finish(R.P, R.gam, nang, n, ld, st);
  launch_set_identity(R.Q, nullptr, nang, n, ld, st);
  R.launches += 4 + R.gj_per;
  if (C->renorm_policy == 1) {
    double kap = Pb.kappa_max + 1.0;
    R.interval = std::max(1, (int)std::floor(C->renorm_tau / (kap * Pb.dz)));
  }
}

// rk4_intgs after each slice (surf_rk.f90:147-152): the power estimate of
// ||[q; p]||^2 (at most nb steps), then CholeskyQR of the angles above 1e2.
void reorthogonalise(trhepd_context* C, RunState& R) {
  cudaEvent_t* ev = (C->profile && 2 * (R.renorm_entries + 1) <= (long)C->rnpool.size())
                        ? &C->rnpool[2 * R.renorm_entries]
                        : nullptr;
  if (ev) CK(cudaEventRecord(ev[0], R.st));
  launch_power_est(R.Q, R.P, R.gsx, R.flags, R.dval, R.nang, R.n, R.ld, R.n, R.st);
  R.launches += 1 + launch_cholqr(R.Q, R.P, R.flags, R.nang, R.n, R.ld, R.gss, R.status, R.st);
  ++R.renorms;  // upper bound; per-angle decisions stay on the device
  if (ev) {
    CK(cudaEventRecord(ev[1], R.st));
    ++R.renorm_entries;
  }
}

// Gather the stage matrix of table column `col` into R.V.
void gather(RunState& R, int col, bool drop_diag) {
  if (R.nprob > 1)
    launch_gather_stage_multi(R.tables, (size_t)col * R.nv, R.pair, R.n, R.kpad, R.ld, drop_diag,
                              R.V, R.sr.vstride, R.nprob, R.st);
  else
    launch_gather_stage(R.table + (size_t)col * R.nv, R.pair, R.n, R.kpad, R.ld, drop_diag, R.V,
                        R.st);
  R.launches += 1;
}

// P += cb (Q M), Qo = Q + ca P with M from R.V (gathered for the chosen form).
void stage_product(trhepd_context* C, RunState& R, const cd* Q, cd* P, cd* Qo, double cb,
                   double ca) {
  const cudaEvent_t* ev = C->profile ? &C->evpool[4 * R.products] : nullptr;
  if (ev) CK(cudaEventRecord(ev[0], R.st));
  if (R.split) {
    R.launches += split_stage(R.sw, Q, P, Qo, R.V, R.D, R.nang, R.n, R.ld, cb, ca,
                              C->split_slices, R.split_variant, ev ? ev + 1 : nullptr, R.st, R.sr);
  } else {
    if (ev) CK(cudaEventRecord(ev[1], R.st));
    launch_stage_gemm_f64(Q, P, Qo, R.V, R.D, R.nang, R.n, R.ld, R.kpad, cb, ca, R.st, R.sr,
                          C->max_ctas);
    if (ev) CK(cudaEventRecord(ev[2], R.st));
    R.launches += 1;
  }
  if (ev) CK(cudaEventRecord(ev[3], R.st));
  ++R.products;
  if (ev) ++R.prof_entries;
}

void renormalise_launch(trhepd_context* C, RunState& R, bool last, int l, bool every_slice);

// End-of-slice renormalisation: the reference's Gershgorin test per angle
// (policy 0, cond_est matcomp.f90:498-528 > 1e3, matAbdivB :53-69) or the
// growth bound every R.interval slices (policy 1); always on the last slice.
void renormalise(trhepd_context* C, RunState& R, int l, bool every_slice) {
  const bool last = (l == R.ns);
  const long gj0 = R.gj_launches;
  cudaEvent_t* ev = (C->profile && 2 * (R.renorm_entries + 1) <= (long)C->rnpool.size())
                        ? &C->rnpool[2 * R.renorm_entries]
                        : nullptr;
  if (ev) CK(cudaEventRecord(ev[0], R.st));
  renormalise_launch(C, R, last, l, every_slice);
  if (ev && R.gj_launches != gj0) {
    CK(cudaEventRecord(ev[1], R.st));
    ++R.renorm_entries;
  }
}

void renormalise_launch(trhepd_context* C, RunState& R, bool last, int l, bool every_slice) {
  if (C->renorm_policy == 0 && !every_slice) {
    launch_cond_est(R.Q, R.nang, R.n, R.ld, last ? 1 : 0, R.flags, R.dval, R.st);
    launch_gauss_jordan(R.Q, R.P, R.flags, R.nang, R.n, R.ld, R.gjs, R.status, R.st,
                        R.split ? kGjFused : kGjFp64Mma);
    launch_set_identity(R.Q, R.flags, R.nang, R.n, R.ld, R.st);
    R.launches += 2 + R.gj_per;
    R.gj_launches += R.gj_per;
    if (!last) ++R.renorms;  // upper bound; per-angle decisions stay on the device
  } else if (last || every_slice || (l % R.interval) == 0) {
    launch_gauss_jordan(R.Q, R.P, nullptr, R.nang, R.n, R.ld, R.gjs, R.status, R.st,
                        R.split ? kGjFused : kGjFp64Mma);
    launch_set_identity(R.Q, nullptr, R.nang, R.n, R.ld, R.st);
    R.launches += 1 + R.gj_per;
    R.gj_launches += R.gj_per;
    if (!last) ++R.renorms;
  }
}

// stransh (matcomp.f90:174-196) and the intensities (surflf.f90:142-151).
void finish_device(trhepd_context* C, trhepd_problem& Pb, RunState& R) {
  cudaStream_t st = R.st;
  const int n = R.n, nang = R.nang, ld = R.ld;
  if (Pb.I.gs)
    launch_strans_build(R.Q, R.P, R.gam, nang, n, ld, st);  // strans + matAdivB2
  else
    launch_stransh_build(R.Q, R.P, R.gam, nang, n, ld, st);
  launch_gauss_jordan(R.Q, R.P, nullptr, nang, n, ld, R.gjs, R.status, st);
  launch_check_finite(R.P, (size_t)nang * n * ld, R.status, st);
  launch_intensities(R.P, R.gam, Pb.wnsga2.as<double>(), nang, n, ld, Pb.nb0,
                     Pb.f2.as<double>(), st);
  R.launches += 3 + R.gj_per;
  if (!R.capturing) CK(cudaEventRecord(C->ev1, st));
  CK(cudaGetLastError());
}

// Status and timing of a finished run (after its launches or its graph).
void finish_host(trhepd_context* C, trhepd_problem& Pb, RunState& R) {
  cudaStream_t st = R.st;
  CK(cudaGetLastError());
  unsigned h_status[4];
  CK(cudaMemcpyAsync(h_status, R.status, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  float ms = 0;
  cudaEventElapsedTime(&ms, C->ev0, C->ev1);
  double prod_ms = 0.0, tensor_ms = 0.0, renorm_ms = 0.0;
  if (C->profile)
    for (long p = 0; p < R.renorm_entries; ++p) {
      float e = 0;
      cudaEventElapsedTime(&e, C->rnpool[2 * p], C->rnpool[2 * p + 1]);
      renorm_ms += e;
    }
  if (C->profile)
    for (long p = 0; p < R.prof_entries; ++p) {
      float e = 0, t = 0;
      cudaEventElapsedTime(&e, C->evpool[4 * p], C->evpool[4 * p + 3]);
      cudaEventElapsedTime(&t, C->evpool[4 * p + 1], C->evpool[4 * p + 2]);
      prod_ms += e;
      tensor_ms += t;
    }
  C->stats[0] = (double)R.renorms;
  C->stats[1] = (double)R.products;
  C->stats[2] = ms;
  C->stats[3] = (double)Pb.ncol;
  C->stats[4] = prod_ms;
  C->stats[5] = (double)R.launches;
  C->stats[6] = (double)R.gj_launches;
  C->stats[7] = tensor_ms;
  C->stats[8] = renorm_ms;
  if (h_status[0] & kStatusTimeout) throw CudaError("device wait timed out", TRHEPD_ETIMEOUT);
  if (h_status[0] & (kStatusNonFinite | kStatusZeroPivot))
    throw CudaError("non-finite value or zero pivot in the surface solve", TRHEPD_ENONFINITE);
}

// The fused-kernel descriptor of a run whose begin_run has been issued.
FusedProblem fused_problem(const RunState& R, double dz, int first_cta) {
  FusedProblem f{};
  f.Q = R.Q;
  f.P = R.P;
  f.table = R.table;
  f.pair = R.pair;
  f.D = R.D;
  f.status = R.status;
  f.n = R.n;
  f.ld = R.ld;
  f.nv = R.nv;
  f.nang = R.nang;
  f.ns = R.ns;
  f.interval = R.interval;
  f.first_cta = first_cta;
  f.dz = dz;
  return f;
}

// Symplectic RKN (hp_int_spa, surf_prkn.f90:278-330) batched over angles.
void run_rkn(trhepd_context* C, trhepd_problem& Pb, int precision, RunState& R) {
  const Integrator& I = Pb.I;
  const double dz = Pb.dz;
  begin_run(C, Pb, precision, I.s * Pb.ns, R, context_workspace(C));
  const bool every_slice = (Pb.n == 1 && Pb.int_method == 6);  // hp_int_spa1d renormalises each slice
  if (!R.split && R.nprob == 1 && Pb.n >= 2 && Pb.n <= std::min(C->fused_max_n, kFusedMaxBeams)) {
    // whole integration in one launch, state in shared memory (small.cu)
    static thread_local FusedLaunch L;  // 17 KB of kernel parameters
    L.nprob = 1;
    L.s = I.s;
    L.policy = C->renorm_policy;
    L.total_ctas = R.nang;
    for (int q = 0; q < 2 * I.s + 1; ++q) L.bab[q] = I.bab[q];
    L.p[0] = fused_problem(R, dz, 0);
    const cudaEvent_t* ev = C->profile ? &C->evpool[0] : nullptr;  // the launch is one entry
    if (ev) {
      CK(cudaEventRecord(ev[0], R.st));
      CK(cudaEventRecord(ev[1], R.st));
    }
    R.launches += launch_fused_rkn(L, R.st);
    if (ev) {
      CK(cudaEventRecord(ev[2], R.st));
      CK(cudaEventRecord(ev[3], R.st));
      R.prof_entries = 1;
    }
    R.products += (long)I.s * R.ns - 1;
    R.renorms += (C->renorm_policy == 1) ? (R.ns - 1) / R.interval : R.ns - 1;
    finish_device(C, Pb, R);
    return;
  }
  for (int l = 1; l <= R.ns; ++l) {
    for (int k = 1; k <= I.s; ++k) {
      const int col = I.s * (l - 1) + k - 1;
      const double ca = I.bab[2 * k - 1] * dz;
      if (l == 1 && k == 1) {  // Q = I: elementwise stage
        gather(R, col, false);
        launch_stage_identity(R.Q, R.P, R.V, R.D, R.nang, R.n, R.ld, I.bab[0] * dz, ca, R.st,
                              R.sr);
        R.launches += 1;
        continue;
      }
      // k == 1, l > 1 merges the end-of-slice half kick of slice l-1 (psave) with the
      // first kick of slice l: both use the same stage column, so cb = 2 b1.
      const double cb = (k == 1) ? 2.0 * I.bab[0] * dz : I.bab[2 * k - 2] * dz;
      gather(R, col, R.split);
      stage_product(C, R, R.Q, R.P, R.Qn, cb, ca);
      std::swap(R.Q, R.Qn);
    }
    // end of slice: renormalisation decision on Q (the reference tests Q after the
    // last stage; the end-of-slice kick does not change Q)
    renormalise(C, R, l, every_slice);
  }
  // final half kick with Q = I: P += b1 dz M(end)
  gather(R, I.s * R.ns, false);
  launch_stage_identity(R.Q, R.P, R.V, R.D, R.nang, R.n, R.ld, I.bab[0] * dz, 0.0, R.st, R.sr);
  R.launches += 1;
  finish_device(C, Pb, R);
}

// Stormer-Verlet leapfrog (lf_int_spa, surf_magnus.f90:46-110) batched over
// angles: Q = I + dz/2 P, then per slice P += dz Q M(l), Q += dz P (dz/2 on the
// last slice).  A renormalised Q = I enters the next product as the identity,
// which gives the reference's Q = I shortcut exactly.
void run_lf(trhepd_context* C, trhepd_problem& Pb, int precision, RunState& R) {
  const double dz = Pb.dz;
  begin_run(C, Pb, precision, Pb.ns, R, context_workspace(C));
  gather(R, 0, false);  // any finite stage matrix: cb = 0 below
  launch_stage_identity(R.Q, R.P, R.V, R.D, R.nang, R.n, R.ld, 0.0, 0.5 * dz, R.st);
  R.launches += 1;
  for (int l = 1; l <= R.ns; ++l) {
    const double dz2 = (l == R.ns) ? dz / 2 : dz;
    gather(R, l - 1, R.split);
    stage_product(C, R, R.Q, R.P, R.Qn, dz, dz2);
    std::swap(R.Q, R.Qn);
    renormalise(C, R, l, false);
  }
  finish_device(C, Pb, R);
}

// Classical RK4 on [Q | P] (rk4_int, surf_rk.f90:27-91) batched over angles:
// k = (P', Q' M) at the stage points, each product Q' M formed by the stage
// kernel into a zeroed buffer (cb = 1, ca = 0).
void run_rk4(trhepd_context* C, trhepd_problem& Pb, int precision, RunState& R) {
  const double dz = Pb.dz;
  begin_run(C, Pb, precision, 4 * Pb.ns, R, context_workspace(C));
  const size_t sb = R.sbytes;
  cd* Qt = (cd*)C->rk[0].ensure(sb);
  cd* Pt = (cd*)C->rk[1].ensure(sb);
  cd* KP = (cd*)C->rk[2].ensure(sb);
  cd* SQ = (cd*)C->rk[3].ensure(sb);
  cd* SP = (cd*)C->rk[4].ensure(sb);
  CK(cudaMemsetAsync(KP, 0, sb, R.st));
  CK(cudaMemsetAsync(Qt, 0, sb, R.st));
  CK(cudaMemsetAsync(Pt, 0, sb, R.st));
  // stage j: (A, column, weight of k_j in the sum, step to the next stage point)
  const double half = 0.5 * dz;
  for (int l = 1; l <= R.ns; ++l) {
    const int c0 = 2 * (l - 1), c1 = 2 * l - 1, c2 = 2 * l;
    const int cols[4] = {c0, c1, c1, c2};
    const double w[4] = {1.0, 2.0, 2.0, 1.0};
    const double step[4] = {half, half, dz, 0.0};
    for (int j = 0; j < 4; ++j) {
      gather(R, cols[j], R.split);
      stage_product(C, R, j == 0 ? R.Q : Qt, KP, R.Qn, 1.0, 0.0);
      launch_rk4_combine(R.Q, R.P, Qt, Pt, KP, SQ, SP, j, w[j], step[j], dz / 6, R.nang, R.n,
                         R.ld, R.st);
      R.launches += 1;
    }
    if (Pb.I.gs)
      reorthogonalise(C, R);
    else
      renormalise(C, R, l, false);
  }
  finish_device(C, Pb, R);
}


// Batched FP64 product C = A B (+ C) over the angles; a zero stride shares the operand.
void bgemm(const cd* A, long long sA, const cd* B, long long sB, cd* Cm, long long sC, int n,
           int ld, int beta, int batch, cudaStream_t st) {
  BatchedGemm g{A, B, Cm, n, n, n, ld, ld, ld, sA, sB, sC, cd{1.0, 0.0}, beta, batch, nullptr};
  launch_zgemm_batched(g, st);
}

// Magnus integrators m2/m4/m6 (m2_int_spa, m4_int_spa, m6_int_spa;
// surf_magnus.f90:114-339) batched over angles.  Each slice forms q and rp from
// hyperbolic_exp4r/6r of the stage matrices (magnus.cu), then P += Q rp and
// Q += P q as batched GEMMs; after a renormalisation Q = I enters those products
// as the identity.  Plain FP64 only.
void run_magnus(trhepd_context* C, trhepd_problem& Pb, int precision, RunState& R) {
  if (precision != TRHEPD_FP64)
    throw std::invalid_argument("the Magnus integrators (int_method 1-3) run in plain FP64 only");
  // the Magnus element kernels index the stacked rows with the grid's y dimension
  if ((long long)Pb.nang * Pb.n > 65535)
    throw std::invalid_argument("Magnus: angles x beams exceeds 65535 stacked rows; split the scan");
  const double dz = Pb.dz;
  const Family fam = Pb.I.family;
  begin_run(C, Pb, precision, 0, R, context_workspace(C));
  const int n = R.n, nang = R.nang, ld = R.ld;
  cudaStream_t st = R.st;
  const size_t sb = R.sbytes, vb = (size_t)(R.kpad + 1) * ld * sizeof(cd);
  const long long sa = (long long)n * ld;
  cd* Qq = (cd*)C->rk[0].ensure(sb);
  cd* RPN = (cd*)C->rk[1].ensure(sb);
  cd* RP = (cd*)C->rk[2].ensure(sb);
  cd* R2 = (cd*)C->rk[3].ensure(sb);
  cd* T = (cd*)C->rk[4].ensure(sb);
  cd* RNEW = (cd*)C->mg[0].ensure(sb);
  cd* V1 = (cd*)C->mg[1].ensure(vb);
  cd* V3 = (cd*)C->mg[2].ensure(vb);
  cd* S = (cd*)C->mg[3].ensure(vb);
  cd* D13 = (cd*)C->mg[4].ensure(vb);
  cd* S13 = (cd*)C->mg[5].ensure(vb);
  cd* Wm = (cd*)C->mg[6].ensure(vb);
  cd* Wp = (cd*)C->mg[7].ensure(vb);
  cd* M3s = (cd*)C->mg[8].ensure(vb);
  CK(cudaMemsetAsync(RP, 0, sb, st));
  const cd* D = R.D;
  auto gather_into = [&](int col, cd* dst) {
    launch_gather_stage(R.table + (size_t)col * R.nv, R.pair, n, R.kpad, ld, false, dst, st);
    R.launches += 1;
  };
  auto update_state = [&]() {  // P += Q RPN; Q += P Qq
    bgemm(R.Q, sa, RPN, sa, R.P, sa, n, ld, 1, nang, st);
    bgemm(R.P, sa, Qq, sa, R.Q, sa, n, ld, 1, nang, st);
    R.launches += 2;
    R.products += 2;
  };
  for (int l = 1; l <= R.ns; ++l) {
    if (fam == kMagnus2) {
      gather_into(l - 1, R.V);
      bgemm(R.V, 0, R.V, 0, S, 0, n, ld, 0, 1, st);
      launch_magnus4_step(R.V, S, nullptr, nullptr, D, nang, n, ld, dz, dz, 0.0, 0.0, Qq, RPN, RP,
                          st);
      R.launches += 2;
      update_state();
    } else if (fam == kMagnus4) {
      const double c0 = std::sqrt(15.0) / 36, c1 = 5.0 / 36;
      gather_into(3 * l - 3, V1);
      gather_into(3 * l - 2, R.V);
      gather_into(3 * l - 1, V3);
      bgemm(R.V, 0, R.V, 0, S, 0, n, ld, 0, 1, st);
      launch_magnus4_step(R.V, S, V1, V3, D, nang, n, ld, dz, dz, c0, c1, Qq, RPN, RP, st);
      R.launches += 2;
      update_state();
    } else {  // kMagnus6
      const double c0 = std::sqrt(15.0) / 180, c1 = 1.0 / 18, c2 = 1.0 / 12960;
      const double d0 = 4.0 / (3.0 * std::sqrt(15.0)), d1 = 1.0 / 6;
      const double h = dz / 2, c0dz = c0 * dz;
      gather_into(3 * l - 3, V1);
      gather_into(3 * l - 2, R.V);
      gather_into(3 * l - 1, V3);
      launch_magnus6_shared(V1, R.V, V3, n, ld, d0, d1, D13, S13, Wm, Wp, st);
      bgemm(D13, 0, D13, 0, M3s, 0, n, ld, 0, 1, st);
      launch_magnus6_m3(M3s, S13, c2 * (dz * dz * dz), c1 * dz, n, ld, st);
      R.launches += 3;
      // first half step: exponent of m2 - d0 m1
      bgemm(Wm, 0, Wm, 0, S, 0, n, ld, 0, 1, st);
      launch_magnus_square(S, Wm, D, nang, n, ld, R2, st);
      bgemm(R2, sa, Wm, 0, T, sa, n, ld, 0, nang, st);
      launch_magnus6_exp(Wm, D, R2, T, nang, n, ld, h, RP, D13, M3s, c0dz, Qq, RPN, RNEW, st);
      R.launches += 4;
      update_state();
      // second half step: exponent of m2 + d0 m1, rp = r(first) + r(second)
      bgemm(Wp, 0, Wp, 0, S, 0, n, ld, 0, 1, st);
      launch_magnus_square(S, Wp, D, nang, n, ld, R2, st);
      bgemm(R2, sa, Wp, 0, T, sa, n, ld, 0, nang, st);
      launch_magnus6_exp(Wp, D, R2, T, nang, n, ld, h, RNEW, nullptr, nullptr, 0.0, Qq, RPN, RNEW,
                         st);
      R.launches += 4;
      update_state();
      launch_magnus6_carry(RNEW, D13, M3s, c0dz, nang, n, ld, RP, st);
      R.launches += 1;
    }
    renormalise(C, R, l, false);
  }
  launch_add(R.P, RP, nang, n, ld, st);  // P += rp
  R.launches += 1;
  finish_device(C, Pb, R);
}

// Every launch of one solve, in stream order, without host synchronisation.
void run_device(trhepd_context* C, trhepd_problem& Pb, int precision, RunState& R) {
  switch (Pb.I.family) {
    case kRkn: run_rkn(C, Pb, precision, R); break;
    case kLeapfrog: run_lf(C, Pb, precision, R); break;
    case kRk4: run_rk4(C, Pb, precision, R); break;
    case kMagnus2:
    case kMagnus4:
    case kMagnus6: run_magnus(C, Pb, precision, R); break;
  }
}

// The context buffers a solve's launches address; a graph stays valid while they do.
std::vector<void*> buffer_signature(const trhepd_context* C) {
  std::vector<void*> s = {C->Q0.p, C->Q1.p, C->P.p, C->V.p, C->flags.p, C->dval.p,
                          C->gj.p, C->status.p, C->split.p};
  for (const DevBuf& b : C->rk) s.push_back(b.p);
  for (const DevBuf& b : C->mg) s.push_back(b.p);
  return s;
}

// Solve a resident problem.  The launch sequence of a solve depends only on the
// problem and the options, so after one uncaptured solve has sized the buffers,
// the next one is captured into a CUDA graph and later solves replay it (one
// launch instead of thousands; changed options, precision or reallocated buffers
// force a new capture).  Profiling runs and TRHEPD_OPT_GRAPHS = 0 launch directly.
void run(trhepd_context* C, trhepd_problem& Pb, int precision) {
  const std::vector<double> key = {(double)precision, (double)C->split_slices,
                                   (double)C->split_variant, (double)C->renorm_policy,
                                   C->renorm_tau, (double)C->fused_max_n, (double)C->max_ctas};
  if (!C->graphs || C->profile) {
    Pb.drop_graph();
    RunState R;
    run_device(C, Pb, precision, R);
    finish_host(C, Pb, R);
    return;
  }
  const std::vector<void*> sig = buffer_signature(C);
  trhepd_problem::GraphSlot& gs = Pb.slot(key);
  if (!gs.exec || gs.sig != sig) {
    gs.drop();
    if (gs.last_sig != sig) {
      // buffers may grow on this solve: run it directly, capture the next one
      RunState R;
      run_device(C, Pb, precision, R);
      gs.last_sig = buffer_signature(C);
      finish_host(C, Pb, R);
      return;
    }
    RunState R;
    R.capturing = true;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(C->stream, cudaStreamCaptureModeThreadLocal));
    try {
      run_device(C, Pb, precision, R);
    } catch (...) {
      cudaStreamEndCapture(C->stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    CK(cudaStreamEndCapture(C->stream, &g));
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    gs.exec = ex;
    gs.sig = sig;
    gs.run = R;
  }
  RunState R = gs.run;
  CK(cudaEventRecord(C->ev0, C->stream));
  CK(cudaGraphLaunch(gs.exec, C->stream));
  CK(cudaEventRecord(C->ev1, C->stream));
  finish_host(C, Pb, R);
}

// A solve in `precision`; with TRHEPD_OPT_VALIDATE set, a split-form solve is
// preceded by the FP64 solve of the same resident problem and followed by a
// per-curve comparison on the device (the statistics stay those of the split solve).
void run_checked(trhepd_context* C, trhepd_problem& Pb, int precision) {
  C->curve_err.clear();
  if (!C->validate || precision == TRHEPD_FP64) {
    run(C, Pb, precision);
    return;
  }
  const size_t bytes = (size_t)Pb.nang * Pb.n * sizeof(double);
  run(C, Pb, TRHEPD_FP64);
  double* ref = (double*)Pb.f2ref.ensure(bytes);
  CK(cudaMemcpyAsync(ref, Pb.f2.p, bytes, cudaMemcpyDeviceToDevice, C->stream));
  run(C, Pb, precision);
  double* e = (double*)C->cerr.ensure((size_t)3 * Pb.nang * sizeof(double));
  launch_curve_errors(Pb.f2.as<double>(), ref, Pb.nang, Pb.n, e, C->stream);
  CK(cudaGetLastError());
  C->curve_err.resize((size_t)3 * Pb.nang);
  CK(cudaMemcpyAsync(C->curve_err.data(), e, C->curve_err.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, C->stream));
  CK(cudaStreamSynchronize(C->stream));
}

// Problems that can be integrated as one stacked solve: same beams and beam-pair
// map, slice count and thickness, integrator and angle count (the candidates of
// one base structure).  Their angles are stacked row-wise; each row tile of the
// stage product reads its own problem's stage matrix.
bool stackable(const trhepd_problem& a, const trhepd_problem& b) {
  return a.n == b.n && a.ns == b.ns && a.dz == b.dz && a.int_method == b.int_method &&
         a.nang == b.nang && a.nv == b.nv && a.ncol == b.ncol && a.nb0 == b.nb0 &&
         a.pair_host == b.pair_host;
}

// One integration of a stacked group; the intensities go back to each problem.
void solve_stacked(trhepd_context* C, const std::vector<trhepd_problem*>& g, int precision,
                   double* stats) {
  cudaStream_t st = C->stream;
  const trhepd_problem& p0 = *g[0];
  const int k = (int)g.size(), n = p0.n, ld = p0.ld, na = p0.nang;
  trhepd_problem M;
  M.n = n;
  M.ns = p0.ns;
  M.nv = p0.nv;
  M.ld = ld;
  M.nb0 = p0.nb0;
  M.int_method = p0.int_method;
  M.I = p0.I;
  M.dz = p0.dz;
  M.ncol = p0.ncol;
  M.nrep2 = p0.nrep2;
  M.nang = k * na;
  M.nprob = k;
  for (const trhepd_problem* p : g) M.kappa_max = std::max(M.kappa_max, p->kappa_max);
  M.pair.p = p0.pair.p;    // borrowed (shared beam-pair map)
  M.table.p = p0.table.p;  // borrowed (the tables array holds every problem's)
  DevBuf tabs;
  auto unborrow = [&]() {
    M.pair.p = nullptr;
    M.table.p = nullptr;
    M.release();
    tabs.release();
  };
  try {
    std::vector<const TableEntry*> tp(k);
    for (int q = 0; q < k; ++q) tp[q] = g[q]->table.as<TableEntry>();
    M.tables = upload(tabs, tp, st);
    auto stack = [&](DevBuf& dst, DevBuf trhepd_problem::*src, size_t per) {
      char* d = (char*)dst.ensure(per * k);
      for (int q = 0; q < k; ++q)
        CK(cudaMemcpyAsync(d + per * q, (g[q]->*src).p, per, cudaMemcpyDeviceToDevice, st));
    };
    stack(M.gam, &trhepd_problem::gam, (size_t)na * n * sizeof(cd));
    stack(M.D, &trhepd_problem::D, (size_t)na * ld * sizeof(cd));
    stack(M.F, &trhepd_problem::F, (size_t)na * n * n * sizeof(cd));
    stack(M.wnsga2, &trhepd_problem::wnsga2, (size_t)na * sizeof(double));
    M.f2.ensure((size_t)M.nang * n * sizeof(double));
    RunState R;
    run_device(C, M, precision, R);
    finish_host(C, M, R);
    for (int q = 0; q < k; ++q)
      CK(cudaMemcpyAsync(g[q]->f2.p, M.f2.as<double>() + (size_t)q * na * n,
                         (size_t)na * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    for (int q = 0; q < 8; ++q) stats[q] = C->stats[q];
  } catch (...) {
    unborrow();
    throw;
  }
  unborrow();
}

// Problems solved together (no counterpart in the reference, whose driver solves
// one structure at a time).  Problems the fused kernel takes (RKN, 2 <= n <= the
// fused limit) are integrated by shared launches, each in its own buffers: one
// launch per integrator and kFusedMaxProblems problems, whatever their beam
// counts, slice counts and angle grids; the boundary kernels of each problem run
// around it.  Other problems are solved one after another (graph replays from
// their second solve on).  The split forms apply to those; fused problems are FP64.
void batch_solve(trhepd_context* C, trhepd_problem* const* probs, int count, int precision) {
  cudaStream_t st = C->stream;
  const int fmax = std::min(C->fused_max_n, kFusedMaxBeams);
  std::vector<trhepd_problem*> fused[2], rest;  // by integrator: RKN-4 (s = 6), RKN-6 (s = 11)
  for (int q = 0; q < count; ++q) {
    trhepd_problem* p = probs[q];
    if (!p) throw std::invalid_argument("null problem in batch");
    if (p->I.family == kRkn && p->n >= 2 && p->n <= fmax)
      fused[p->I.s == 6 ? 0 : 1].push_back(p);
    else
      rest.push_back(p);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  long launches = 0, products = 0, renorms = 0;
  std::vector<unsigned*> statuses;
  try {
    CK(cudaEventRecord(e0, st));
    static thread_local FusedLaunch L;
    for (auto& group : fused)
      for (size_t g0 = 0; g0 < group.size(); g0 += kFusedMaxProblems) {
        const size_t g1 = std::min(group.size(), g0 + (size_t)kFusedMaxProblems);
        std::vector<RunState> runs(g1 - g0);
        const Integrator& I = group[g0]->I;
        L.nprob = (int)(g1 - g0);
        L.s = I.s;
        L.policy = C->renorm_policy;
        for (int q = 0; q < 2 * I.s + 1; ++q) L.bab[q] = I.bab[q];
        int ctas = 0;
        for (size_t q = g0; q < g1; ++q) {
          RunState& R = runs[q - g0];
          R.capturing = true;  // timing events belong to the batch
          begin_run(C, *group[q], TRHEPD_FP64, 0, R, group[q]->own.view());
          L.p[q - g0] = fused_problem(R, group[q]->dz, ctas);
          ctas += R.nang;
          products += (long)I.s * R.ns - 1;
          renorms += (C->renorm_policy == 1) ? (R.ns - 1) / R.interval : R.ns - 1;
        }
        L.total_ctas = ctas;
        launches += launch_fused_rkn(L, st);
        for (size_t q = g0; q < g1; ++q) {
          RunState& R = runs[q - g0];
          finish_device(C, *group[q], R);
          launches += R.launches;
          statuses.push_back(R.status);
        }
      }
    std::vector<unsigned> hs(4 * statuses.size() + 4, 0);
    for (size_t q = 0; q < statuses.size(); ++q)
      CK(cudaMemcpyAsync(&hs[4 * q], statuses[q], 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (size_t q = 0; q < statuses.size(); ++q) {
      if (hs[4 * q] & kStatusTimeout) throw CudaError("device wait timed out", TRHEPD_ETIMEOUT);
      if (hs[4 * q] & (kStatusNonFinite | kStatusZeroPivot))
        throw CudaError("non-finite value or zero pivot in a batch solve", TRHEPD_ENONFINITE);
    }
    // stack the rest into groups (RKN, FP64 or INT8), solve groups of two or more
    // as one integration and the others one by one
    std::vector<bool> done(rest.size(), false);
    const bool stack_ok = precision == TRHEPD_FP64 || precision == TRHEPD_SPLIT_INT8;
    for (size_t q = 0; q < rest.size(); ++q) {
      if (done[q]) continue;
      std::vector<trhepd_problem*> grp = {rest[q]};
      done[q] = true;
      if (stack_ok && rest[q]->I.family == kRkn && rest[q]->n >= 2)
        for (size_t r = q + 1; r < rest.size(); ++r)
          if (!done[r] && stackable(*rest[q], *rest[r]) &&
              (long long)(grp.size() + 1) * rest[q]->nang * rest[q]->n <= (1 << 22)) {
            grp.push_back(rest[r]);
            done[r] = true;
          }
      double st8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (grp.size() > 1) {
        solve_stacked(C, grp, precision, st8);
      } else {
        run(C, *grp[0], precision);
        for (int k = 0; k < 8; ++k) st8[k] = C->stats[k];
      }
      products += (long)st8[1];
      renorms += (long)st8[0];
      launches += (long)st8[5];
    }
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    for (double& v : C->stats) v = 0.0;
    C->stats[0] = (double)renorms;
    C->stats[1] = (double)products;
    C->stats[2] = ms;
    C->stats[5] = (double)launches;
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

void fetch(trhepd_context* C, trhepd_problem& Pb, double* f2, double* angle_deg) {
  if (f2)
    CK(cudaMemcpyAsync(f2, Pb.f2.p, (size_t)Pb.nang * Pb.n * sizeof(double),
                       cudaMemcpyDeviceToHost, C->stream));
  CK(cudaStreamSynchronize(C->stream));
  if (angle_deg) std::copy(Pb.angle_deg.begin(), Pb.angle_deg.end(), angle_deg);
}

// The end-to-end solve behind trhepd_srfref: prepare, run, fetch, release.
void solve(trhepd_context* C, const SolveArgs& A, int precision, double* f2_out,
           double* angle_out) {
  trhepd_problem Pb;
  try {
    prepare(C, A, Pb);
    run_checked(C, Pb, precision);
    fetch(C, Pb, f2_out, angle_out);
  } catch (...) {
    cudaStreamSynchronize(C->stream);
    Pb.release();
    throw;
  }
  Pb.release();
}


// ---------------------------------------------------------------- bulk solve
// blkref (bulk.f90:7-128) for every (angle, group) item at once; see bulk.cu.
void bulk_solve(trhepd_context* C, BulkInputs& B, std::vector<std::vector<cd>>& records,
                double* stats) {
  cudaStream_t st = C->stream;
  const int nv = B.nv, ns = B.ns, ngr = B.ngr, n = B.nbgm;
  if (n > kMaxBeams) throw std::invalid_argument("bulk beam group exceeds the GPU path limit");
  if (3 * B.natm > 512) throw std::invalid_argument("bulk atoms exceed the potential table limit");
  // structure factors (K2) for the three parts
  std::vector<cd> stv[3];
  for (int p = 0; p < 3; ++p) {
    const StructureFactorJob& J = B.stf[p];
    const double* gh = upload(C->sgh, B.gh, st);
    const double* gk = upload(C->sgk, B.gk, st);
    const double* img = upload(C->simg, J.img, st);
    const int* nimg = upload(C->snimg, J.nimg, st);
    cd* out = (cd*)C->sst.ensure((size_t)nv * B.natm * sizeof(cd));
    launch_structure_factor(gh, gk, nv, img, nimg, B.natm, J.dx, J.dy, out, st);
    stv[p].resize((size_t)nv * B.natm);
    CK(cudaMemcpyAsync(stv[p].data(), out, stv[p].size() * sizeof(cd), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  // potential table at the slice centres: parts at zi, zi+cc, zi-cc (bulkio.f90:194-199)
  std::vector<double> depth(ns);
  for (int i = 1; i <= ns; ++i) depth[i - 1] = B.dz * (i - 0.5);
  PotInputs in{};
  in.asf = upload(C->asf, B.asf, st);
  in.b = upload(C->b, B.bcoef, st);
  in.dchg = upload(C->dchg, B.dchg, st);
  in.ghk = upload(C->ghk, B.Ghk, st);
  in.nv = nv;
  in.nelm = B.nelm;
  in.nabr = B.nabr;
  in.nabi = B.nabi;
  in.mab = kMab;
  std::vector<int> ie(B.natm);
  for (int j = 0; j < B.natm; ++j) ie[j] = B.ielm[j] - 1;
  const double shift[3] = {0.0, B.cc, -B.cc};
  for (int p = 0; p < 3; ++p) {
    PotPart& P = in.part[p];
    P.z = upload(C->z[p], B.z, st);
    P.ocr = upload(C->ocr[p], B.ocr, st);
    P.ielm = upload(C->ielm[p], ie, st);
    P.st = upload(C->st[p], stv[p], st);
    P.natm = B.natm;
    P.nk = nv;
    P.zshift = shift[p];
    P.rmesh = 1.0;
  }
  const double* dd = upload(C->depth, depth, st);
  TableEntry* table = (TableEntry*)C->table.ensure((size_t)ns * nv * sizeof(TableEntry));
  launch_potential_table(in, dd, ns, table, st);
  CK(cudaGetLastError());
  std::vector<TableEntry> htab((size_t)ns * nv);
  CK(cudaMemcpyAsync(htab.data(), table, htab.size() * sizeof(TableEntry), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  double vmax = 0.0;
  for (const TableEntry& e : htab)
    vmax = std::max(vmax, std::max(std::hypot(e.u.x, e.u.y), std::hypot(e.w.x, e.w.y)));

  // items: (angle t, group g) -> b = t * ngr + g, padded to n beams
  const bool ng_outer = B.ng > B.naz;
  const int nrep1 = ng_outer ? B.naz : B.ng, nrep2 = ng_outer ? B.ng : B.naz;
  const int nitem = nrep1 * nrep2 * ngr;
  const int ld = round_up(n, 16), n2 = 2 * n, ld2 = round_up(n2, 16);
  std::vector<int> gsize(ngr), goff(ngr + 1, 0);
  for (int g = 0; g < ngr; ++g) {
    gsize[g] = B.nbg[g];
    goff[g + 1] = goff[g] + B.nbg[g];
  }
  std::vector<int> pair((size_t)ngr * n * n, 0);
  for (int g = 0; g < ngr; ++g)
    for (int i = 0; i < gsize[g]; ++i)
      for (int j = 0; j < gsize[g]; ++j) {
        if (i == j) continue;
        int hi = std::max(i, j), lo = std::min(i, j);
        int e = B.iv[(size_t)(goff[g] + lo) * B.nbgm + hi];
        if (e < 1 || e > nv) throw std::invalid_argument("bulk beam-pair index out of range");
        pair[((size_t)g * n + i) * n + j] = e - 1;
      }
  std::vector<cd> gam((size_t)nitem * n, cd{1.0, 0.0}), phase((size_t)nitem * n, cd{1.0, 0.0});
  const double pi2 = std::atan(1.0) * 8.0;
  const bool shifted = std::fabs(B.dx) > 1e-4 || std::fabs(B.dy) > 1e-4;
  const double azr = B.azi + B.rdom;
  double g2max = 0.0;
  for (int t = 0; t < nrep1 * nrep2; ++t) {
    int irep1 = t / nrep2, irep2 = t % nrep2;
    double az, cga;
    if (ng_outer) {
      az = azr + irep1 * B.daz;
      cga = std::cos(B.gi + irep2 * B.dg);
    } else {
      cga = std::cos(B.gi + irep1 * B.dg);
      az = azr + irep2 * B.daz;
    }
    double wnx = B.wn * cga * std::cos(az), wny = B.wn * cga * std::sin(az);
    for (int g = 0; g < ngr; ++g)
      for (int i = 0; i < gsize[g]; ++i) {
        int k = goff[g] + i;
        double wgx = B.ghx * B.ihs[k] + wnx, wgy = B.ghy * B.ihs[k] + B.gky * B.iks[k] + wny;
        double s = B.wn * B.wn - wgx * wgx - wgy * wgy;
        size_t o = ((size_t)t * ngr + g) * n + i;
        gam[o] = (s >= 0.0) ? cd{std::sqrt(s), 0.0} : cd{0.0, std::sqrt(-s)};
        g2max = std::max(g2max, std::fabs(s));
        if (shifted) {
          double a = B.dx * pi2 / B.nh * B.ihs[k] + B.dy * pi2 / B.nk * B.iks[k];
          phase[o] = cd{std::cos(a), std::sin(a)};
        }
      }
  }
  // double-angle steps: ||H|| h^2 <= 1/4 with h = dz / 2^m
  const double hnorm = g2max + (double)n * vmax;
  int m = 0;
  while (hnorm * std::pow(B.dz / std::ldexp(1.0, m), 2) > 0.25) ++m;
  const double h = B.dz / std::ldexp(1.0, m);

  const int* d_pair = upload(C->pair, pair, st);
  const cd* d_gam = upload(C->gam, gam, st);
  const cd* d_ph = upload(C->F, phase, st);
  const int* d_gsize = upload(C->flags, gsize, st);
  const size_t nb1 = (size_t)nitem * n * ld, nb2 = (size_t)nitem * n2 * ld2;
  auto buf1 = [&](int k) { return (cd*)C->bk[k].ensure(nb1 * sizeof(cd)); };
  auto buf2 = [&](int k) { return (cd*)C->bk[k].ensure(nb2 * sizeof(cd)); };
  cd *H = buf1(0), *X = buf1(1), *X2 = buf1(2), *X3 = buf1(3), *X4 = buf1(4), *Cm = buf1(5);
  cd *Sm = buf1(6), *T1 = buf1(7), *T2 = buf1(8), *Hs = buf1(9);
  cd *E = buf2(10), *Et = buf2(11), *En = buf2(12), *Tl = buf2(18);
  if (nitem > 65535) throw std::invalid_argument("too many (angle, group) items for one bulk batch");
  // per-item matrices: n x n at ld (stride s1) or 2n x 2n at ld2 (stride s2)
  const long long s1 = (long long)n * ld, s2 = (long long)n2 * ld2;
  auto gemm1 = [&](const cd* A, const cd* Bm, cd* Cc, int beta, const int* active) {
    BatchedGemm g{A, Bm, Cc, n, n, n, ld, ld, ld, s1, s1, s1, cd{1.0, 0.0}, beta, nitem, active};
    launch_zgemm_batched(g, st);
  };
  auto gemm2 = [&](const cd* A, const cd* Bm, cd* Cc) {
    BatchedGemm g{A, Bm, Cc, n2, n2, n2, ld2, ld2, ld2, s2, s2, s2, cd{1.0, 0.0}, 0, nitem,
                  nullptr};
    launch_zgemm_batched(g, st);
  };
  // T11 R or T21 R: A is the n x n block of T at row offset `row0` (ld2, stride s2)
  auto gemm_t = [&](const cd* Tblk, const cd* Rm, cd* Cc, const int* active) {
    BatchedGemm g{Tblk, Rm, Cc, n, n, n, ld2, ld, ld, s2, s1, s1, cd{1.0, 0.0}, 1, nitem, active};
    launch_zgemm_batched(g, st);
  };
  // Taylor coefficients 1/(2k)! and 1/(2k+1)!, k = 0..8
  double fc[9], fs[9];
  {
    double f = 1.0;
    for (int k = 0; k <= 17; ++k) {
      if (k > 0) f *= k;
      if (k % 2 == 0) fc[k / 2] = 1.0 / f;
      else fs[k / 2] = 1.0 / f;
    }
  }
  CK(cudaEventRecord(C->ev0, st));
  for (int l = 0; l < ns; ++l) {
    launch_bulk_hamiltonian(table + (size_t)l * nv, d_pair, d_gam, d_gsize, ngr, n, ld, nitem,
                            h * h, H, X, st);
    gemm1(X, X, X2, 0, nullptr);
    gemm1(X2, X, X3, 0, nullptr);
    gemm1(X2, X2, X4, 0, nullptr);
    const double c1[5] = {fc[0], fc[1], fc[2], fc[3], 0.0}, c2[5] = {fc[4], fc[5], fc[6], fc[7], fc[8]};
    const double s1[5] = {fs[0], fs[1], fs[2], fs[3], 0.0}, s2[5] = {fs[4], fs[5], fs[6], fs[7], fs[8]};
    launch_bulk_poly(X, X2, X3, nullptr, c1, n, ld, nitem, Cm, st);
    launch_bulk_poly(X, X2, X3, X4, c2, n, ld, nitem, T1, st);
    gemm1(X4, T1, Cm, 1, nullptr);   // C = P1 + X^4 P2
    launch_bulk_poly(X, X2, X3, nullptr, s1, n, ld, nitem, Sm, st);
    launch_bulk_poly(X, X2, X3, X4, s2, n, ld, nitem, T1, st);
    gemm1(X4, T1, Sm, 1, nullptr);
    launch_bulk_axpby(Sm, nullptr, h, 0.0, 0.0, n, ld, nitem, st);  // s = h * series
    for (int q = 0; q < m; ++q) {  // C <- 2C^2 - I, s <- 2 s C
      gemm1(Sm, Cm, T2, 0, nullptr);
      gemm1(Cm, Cm, T1, 0, nullptr);
      launch_bulk_axpby(Cm, T1, 0.0, 2.0, -1.0, n, ld, nitem, st);
      launch_bulk_axpby(Sm, T2, 0.0, 2.0, 0.0, n, ld, nitem, st);
    }
    gemm1(H, Sm, Hs, 0, nullptr);
    launch_bulk_build_e(Cm, Sm, Hs, n, ld, ld2, nitem, E, st);
    // slice transfer matrix T_l = S E_l S^-1 (trmat), then T_tot <- T_l T_tot
    launch_bulk_similarity(E, d_gam, nullptr, d_gsize, ngr, n, ld2, nitem, l == 0 ? Et : Tl, st);
    if (l > 0) {
      gemm2(Tl, Et, En);
      std::swap(Et, En);
    }
  }
  cd* Tm = Et;  // unit-layer transfer matrix
  if (shifted) launch_bulk_phase_cols(Tm, d_ph, d_gsize, ngr, n, ld2, nitem, st);
  // layer recursion with the convergence exit
  std::vector<int> act(nitem, 1);
  int* d_act = upload(C->bk[13], act, st);
  double* r20 = (double*)C->bk[14].ensure((size_t)nitem * n * sizeof(double));
  cd* R = buf1(15);
  cd* Qg = buf1(16);
  cd* Pg = buf1(17);
  unsigned* status = (unsigned*)C->status.ensure(16);
  CK(cudaMemsetAsync(status, 0, 16, st));
  CK(cudaMemsetAsync(R, 0, nb1 * sizeof(cd), st));
  void* gjs = C->gj.ensure(gj_scratch_bytes(nitem, n));
  int layers = 0;
  for (int l = 1; l <= B.ml; ++l) {
    launch_bulk_layer_init(Tm, d_act, n, ld, ld2, nitem, T1, T2, st);
    if (l > 1) {
      gemm_t(Tm, R, T1, d_act);                       // T12 + T11 R
      gemm_t(Tm + (size_t)n * ld2, R, T2, d_act);     // T22 + T21 R
    }
    launch_bulk_transpose_pair(T1, T2, d_act, d_gsize, ngr, n, ld, nitem, Qg, Pg, st);
    launch_gauss_jordan(Qg, Pg, d_act, nitem, n, ld, gjs, status, st);
    launch_bulk_layer_finish(Pg, d_act, d_gsize, ngr, n, ld, nitem, l, B.epsb, r20, R, st);
    layers = l;
    if (l >= 21) {
      CK(cudaMemcpyAsync(act.data(), d_act, nitem * sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      int live = 0;
      for (int a : act) live += a;
      if (!live) break;
    }
  }
  CK(cudaEventRecord(C->ev1, st));
  std::vector<cd> hR(nb1);
  CK(cudaMemcpyAsync(hR.data(), R, nb1 * sizeof(cd), cudaMemcpyDeviceToHost, st));
  unsigned hs[4];
  CK(cudaMemcpyAsync(hs, status, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  float ms = 0;
  cudaEventElapsedTime(&ms, C->ev0, C->ev1);
  if (hs[0] & kStatusZeroPivot) throw CudaError("zero pivot in the bulk layer solve", TRHEPD_ENONFINITE);
  records.assign(nitem, {});
  for (int b = 0; b < nitem; ++b) {
    int g = b % ngr, mg = gsize[g];
    auto& rec = records[b];
    rec.resize((size_t)mg * mg);
    for (int j = 0; j < mg; ++j)
      for (int i = 0; i < mg; ++i) rec[(size_t)j * mg + i] = hR[((size_t)b * n + i) * ld + j];
  }
  if (stats) {
    stats[0] = ms;
    stats[1] = layers;
    stats[2] = m;
    stats[3] = nitem;
  }
}

// Structure factors of SurfaceInputs on the device.
void structure_factors(trhepd_context* C, SurfaceInputs& S) {
  std::vector<cd>* outs[3] = {&S.st0, &S.st1, &S.st2};
  for (int p = 0; p < 3; ++p) {
    const StructureFactorJob& J = S.stf[p];
    outs[p]->assign((size_t)J.nk * J.natm, cd{0, 0});
    if (J.natm == 0 || J.nk == 0) continue;
    const double* gh = upload(C->sgh, S.gh, C->stream);
    const double* gk = upload(C->sgk, S.gk, C->stream);
    const double* img = upload(C->simg, J.img, C->stream);
    const int* nimg = upload(C->snimg, J.nimg, C->stream);
    cd* st = (cd*)C->sst.ensure((size_t)J.nk * J.natm * sizeof(cd));
    launch_structure_factor(gh, gk, J.nk, img, nimg, J.natm, J.dx, J.dy, st, C->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(outs[p]->data(), st, (size_t)J.nk * J.natm * sizeof(cd),
                       cudaMemcpyDeviceToHost, C->stream));
    CK(cudaStreamSynchronize(C->stream));
  }
}

trhepd_pot_state pot_view(const SurfaceInputs& S) {
  trhepd_pot_state p{};
  p.nv = S.nv;
  p.nvb = S.nvb;
  p.natms = S.natms;
  p.natmb = S.natmb;
  p.nelm = S.nelm;
  p.nabr = S.nabr;
  p.nabi = S.nabi;
  p.ielm = S.ielm.data();
  p.cc = S.cc;
  p.smesh = S.smesh;
  p.z = S.z.data();
  p.dchg = S.dchg.data();
  p.Ghk = S.Ghk.data();
  p.ocr = S.ocr.data();
  p.b = S.b.data();
  p.asf = S.asf.data();
  p.st0 = reinterpret_cast<const double*>(S.st0.data());
  p.st1 = reinterpret_cast<const double*>(S.st1.data());
  p.st2 = reinterpret_cast<const double*>(S.st2.data());
  return p;
}

template <class F>
int guarded(trhepd_context* ctx, F&& f) {
  if (!ctx) return TRHEPD_EINVAL;
  try {
    CK(cudaSetDevice(ctx->device));
    t_alloc_stream = ctx->stream;
    f();
    ctx->err.clear();
    return TRHEPD_OK;
  } catch (const CudaError& e) {
    return fail(ctx, e.code, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(ctx, TRHEPD_EINVAL, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(ctx, TRHEPD_ENOMEM, e.what());
  } catch (const std::runtime_error& e) {
    return fail(ctx, TRHEPD_EIO, e.what());
  }
}

// ---- Fortran rocking-curve writer (surfio.f90:270-274, surflf.f90:154-165)
std::string fortran_e(double v, int w, int d) {
  std::string body;
  if (v == 0.0) {
    body = "0." + std::string(d, '0') + "E+00";
  } else {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(v));
    std::string s(buf);
    size_t e = s.find('e');
    std::string digits = s.substr(0, 1) + s.substr(2, e - 2);
    int ex = std::atoi(s.c_str() + e + 1) + 1;
    char eb[16];
    if (std::abs(ex) <= 99)
      std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else
      std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    body = std::string(v < 0 ? "-" : "") + "0." + digits + eb;
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

}  // namespace

namespace {
// '(400I4)' beam list of the header lines (surfio.f90:273, 284-287).
void write_beams(FILE* o, const int* ih, const int* ik, int nb) {
  int cnt = 0;
  for (int j = 0; j < nb; ++j) {
    for (int v : {ih[j], ik[j]}) {
      std::fprintf(o, "%4d", v);
      if (++cnt % 400 == 0 && cnt < 2 * nb) std::fprintf(o, "\n");
    }
  }
  std::fprintf(o, "\n");
}

// One domain's rows (surflf.f90:154-165, domainsum.f90:113-119): per outer scan
// index a block of '(E12.4,200(",",Ew.d))' rows with format reversion after 200
// values, then an empty line.
void write_rows(FILE* o, int naz, int ng, const double* f2, const double* angle_deg, int nb,
                int w, int d) {
  const bool ng_outer = ng > naz;
  const int nrep1 = ng_outer ? naz : ng, nrep2 = ng_outer ? ng : naz;
  for (int r1 = 0; r1 < nrep1; ++r1) {
    for (int r2 = 0; r2 < nrep2; ++r2) {
      const int t = r1 * nrep2 + r2;
      std::string line = fortran_e(angle_deg[t], 12, 4);
      for (int i = 0; i < nb; ++i) {
        if (i > 0 && i % 200 == 0) {
          std::fprintf(o, "%s\n", line.c_str());
          line.clear();
        }
        line += ",";
        line += fortran_e(f2[(size_t)t * nb + i], w, d);
      }
      std::fprintf(o, "%s,\n", line.c_str());
    }
    std::fprintf(o, "\n");
  }
}
}  // namespace

namespace trhepd {
void write_rocking_curves(const std::string& path, const SurfaceInputs& S, const double* f2,
                          const double* angle_deg) {
  FILE* o = std::fopen(path.c_str(), "w");
  if (!o) throw std::runtime_error("cannot write " + path);
  std::fprintf(o, "#azimuths,g-angles,beams\n%4d%4d%4d\n#ih,ik\n", S.naz, S.ng, S.nb);
  write_beams(o, S.ih.data(), S.ik.data(), S.nb);
  write_rows(o, S.naz, S.ng, f2, angle_deg, S.nb, 23, 15);
  std::fclose(o);
}

// The .md file of a multi-domain run (surfio.f90:276-287 header, then each domain's
// srfref rows in domain order): f2[d] (nangles x nbd[d]) and angle_deg[d].
void write_domain_curves(const std::string& path, const SurfaceInputs& S,
                         const std::vector<std::vector<double>>& f2,
                         const std::vector<std::vector<double>>& angle_deg) {
  const double deg = 45.0 / std::atan(1.0);
  FILE* o = std::fopen(path.c_str(), "w");
  if (!o) throw std::runtime_error("cannot write " + path);
  std::fprintf(o, "#azimuths,g-angles,domains,nh,nk,gam\n%4d%4d%4d%4d%4d%10.3f\n", S.naz, S.ng,
               S.ndom, S.nh, S.nk, S.gam * deg);
  std::fprintf(o, "#beams,domain angle,domain weight\n");
  for (int i = 0; i < S.ndom; ++i)
    std::fprintf(o, "%4d%10.3f%s\n", S.nbd[i], S.rdom[i] * deg, fortran_e(S.wdom[i], 12, 3).c_str());
  std::fprintf(o, "#ih,ik\n");
  int ibt = 0;
  for (int i = 0; i < S.ndom; ++i) {
    write_beams(o, S.ih_all.data() + ibt, S.ik_all.data() + ibt, S.nbd[i]);
    ibt += S.nbd[i];
  }
  for (int i = 0; i < S.ndom; ++i)
    write_rows(o, S.naz, S.ng, f2[i].data(), angle_deg[i].data(), S.nbd[i], 23, 15);
  std::fclose(o);
}

// The single-domain file domainsum writes (domainsum.f90:108-119): the reference
// domain's beams, '(E12.4,200(",",E12.4))' rows.
void write_domain_sum(const std::string& path, const SurfaceInputs& S, int idomr,
                      const double* s2, const double* angle_deg) {
  FILE* o = std::fopen(path.c_str(), "w");
  if (!o) throw std::runtime_error("cannot write " + path);
  int ibt = 0;
  for (int i = 0; i < idomr; ++i) ibt += S.nbd[i];
  const int mb = S.nbd[idomr];
  std::fprintf(o, "#azimuths,g-angles,beams\n%4d%4d%4d\n#ih,ik\n", S.naz, S.ng, mb);
  write_beams(o, S.ih_all.data() + ibt, S.ik_all.data() + ibt, mb);
  write_rows(o, S.naz, S.ng, s2, angle_deg, mb, 12, 4);
  std::fclose(o);
}
}  // namespace trhepd

namespace trhepd {
void write_domain_curves(const std::string& path, const SurfaceInputs& S,
                         const std::vector<std::vector<double>>& f2,
                         const std::vector<std::vector<double>>& angle_deg);
void write_domain_sum(const std::string& path, const SurfaceInputs& S, int idomr,
                      const double* s2, const double* angle_deg);
}  // namespace trhepd

namespace {
// A value as it reads back from the Fortran-formatted .md header domainsum parses.
double reread(const std::string& text) { return std::stod(text); }

// surf.exe for NDOM > 1 (surfm.f90:72-90): every domain's srfref (surfio.f90:291-341,
// azimuth azi + rdom(idom)) into its own resident problem, then the weighted sum of
// the rotated domains' curves on the device (domainsum.f90:7-121) with the angles,
// weights and cell angle as domainsum reads them back from the .md header.  Writes
// the .md file (out_path with its extension replaced by .md) and the summed .s file
// (out_path).  f2 receives the summed intensities (nangles x the reference domain's
// beams).
void surf_run_domains(trhepd_context* C, const char* bulkp, const char* surf, double dz2,
                      int int_method, int precision, const SurfaceInputs& S0,
                      const char* out_path, double* f2_out, int max_f2, int* dims) {
  const int ndom = S0.ndom;
  if (ndom > kMaxDomains) throw std::invalid_argument("more domains than the domain sum takes");
  const double rad = std::atan(1.0) / 45.0, deg = 45.0 / std::atan(1.0);
  cudaStream_t st = C->stream;
  std::vector<trhepd_problem*> probs;
  std::vector<SurfaceInputs> Sd(ndom);
  DevBuf dstart, dlist, ds2;
  auto cleanup = [&]() {
    cudaStreamSynchronize(st);
    for (trhepd_problem* p : probs) {
      p->release();
      delete p;
    }
    dstart.release();
    dlist.release();
    ds2.release();
  };
  try {
    for (int d = 0; d < ndom; ++d) {
      load_surface_inputs(bulkp, surf, dz2, int_method, Sd[d], d);
      structure_factors(C, Sd[d]);
      trhepd_pot_state pot = pot_view(Sd[d]);
      const SurfaceInputs& S = Sd[d];
      SolveArgs a{&pot, S.nb, S.ns, S.iv.data(), S.dz, S.ngr, S.nbg.data(), S.iord.data(),
                  S.ih.data(), S.ik.data(), S.wn, S.ghx, S.ghy, S.gky, S.azi, S.daz, S.gi,
                  S.dg, S.naz, S.ng, int_method, reinterpret_cast<const double*>(S.t1rec.data())};
      probs.push_back(new trhepd_problem());
      prepare(C, a, *probs.back());
      run_checked(C, *probs.back(), precision);
    }
    // domainsum.f90:43-56: the reference domain has the most beams (the first such)
    int idomr = 0;
    for (int d = 1; d < ndom; ++d)
      if (S0.nbd[d] > S0.nbd[idomr]) idomr = d;
    const int mb = S0.nbd[idomr];
    const int nang = probs[0]->nang;
    // values as the .md header carries them (F10.3 degrees, E12.3 weights)
    char buf[64];
    auto f103 = [&](double v) {
      std::snprintf(buf, sizeof buf, "%10.3f", v);
      return reread(buf);
    };
    const double gam = f103(S0.gam * deg);
    std::vector<double> rdom(ndom), wdom(ndom);
    for (int d = 0; d < ndom; ++d) {
      rdom[d] = f103(S0.rdom[d] * deg);
      wdom[d] = reread(fortran_e(S0.wdom[d], 12, 3));
    }
    std::vector<int> off(ndom + 1, 0);
    for (int d = 0; d < ndom; ++d) off[d + 1] = off[d] + S0.nbd[d];
    auto reduced = [&](int b, double& gx, double& gy) {  // domainsum.f90:82-86
      gx = (double)S0.ih_all[b] / S0.nh;
      gy = (double)S0.ik_all[b] / S0.nk;
      if (std::fabs(gam - 120.0) < 1e-4) gx = (gx + gx + gy) / std::sqrt(3.0);
    };
    // per domain and reference beam, the domain's beams rotating onto it (:76-101)
    std::vector<int> start((size_t)ndom * (mb + 1), 0), list;
    for (int d = 0; d < ndom; ++d) {
      std::vector<std::vector<int>> onto(mb);
      const double dr = rdom[idomr] - rdom[d];
      const double cdr = std::cos(dr * rad), sdr = std::sin(dr * rad);
      for (int ib = 0; ib < S0.nbd[d]; ++ib) {
        if (d == idomr) {
          onto[ib].push_back(ib);
          continue;
        }
        double gx, gy;
        reduced(off[d] + ib, gx, gy);
        const double gxr = cdr * gx - sdr * gy, gyr = sdr * gx + cdr * gy;
        for (int ibr = 0; ibr < mb; ++ibr) {
          double hx, hy;
          reduced(off[idomr] + ibr, hx, hy);
          if (std::fabs(gxr - hx) < 1e-4 && std::fabs(gyr - hy) < 1e-4) {
            onto[ibr].push_back(ib);
            break;
          }
        }
      }
      for (int ibr = 0; ibr < mb; ++ibr) {
        start[(size_t)d * (mb + 1) + ibr] = (int)list.size();
        list.insert(list.end(), onto[ibr].begin(), onto[ibr].end());
      }
      start[(size_t)d * (mb + 1) + mb] = (int)list.size();
    }
    if (list.empty()) list.push_back(0);
    DomainSumArgs A{};
    A.ndom = ndom;
    for (int d = 0; d < ndom; ++d) {
      A.f2[d] = probs[d]->f2.as<double>();
      A.nb[d] = probs[d]->n;
      A.w[d] = wdom[d];
    }
    A.start = upload(dstart, start, st);
    A.list = upload(dlist, list, st);
    double* s2 = (double*)ds2.ensure((size_t)nang * mb * sizeof(double));
    launch_domain_sum(A, nang, mb, s2, st);
    CK(cudaGetLastError());
    std::vector<double> hs2((size_t)nang * mb);
    CK(cudaMemcpyAsync(hs2.data(), s2, hs2.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    std::vector<std::vector<double>> f2d(ndom), angd(ndom);
    for (int d = 0; d < ndom; ++d) {
      f2d[d].resize((size_t)probs[d]->nang * probs[d]->n);
      angd[d].resize(probs[d]->nang);
      fetch(C, *probs[d], f2d[d].data(), angd[d].data());
    }
    if (out_path) {
      std::string s_path = out_path, md_path = s_path;
      const size_t dot = md_path.find_last_of('.'), slash = md_path.find_last_of('/');
      if (dot != std::string::npos && (slash == std::string::npos || dot > slash))
        md_path.resize(dot);
      md_path += ".md";
      write_domain_curves(md_path, S0, f2d, angd);
      // domainsum reads every domain's angles into one array: the last domain's stay
      write_domain_sum(s_path, S0, idomr, hs2.data(), angd[ndom - 1].data());
    }
    if (f2_out) {
      if ((size_t)max_f2 < hs2.size()) throw std::invalid_argument("f2 buffer too small");
      std::memcpy(f2_out, hs2.data(), hs2.size() * sizeof(double));
    }
    if (dims) {
      dims[0] = mb;
      dims[1] = nang;
      dims[2] = Sd[idomr].ns;
      dims[3] = Sd[idomr].nv;
    }
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
}
}  // namespace

// =============================================================================
// C ABI
// =============================================================================
extern "C" {

int trhepd_create(int device, trhepd_context** out) {
  if (!out) return TRHEPD_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return TRHEPD_ECUDA;
  if (device < 0 || device >= ndev) return TRHEPD_EINVAL;
  auto* c = new trhepd_context();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return TRHEPD_ECUDA;
  }
  // freed buffers stay in the device's default pool for the next allocation
  // instead of going back to the driver at every synchronisation
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  *out = c;
  return TRHEPD_OK;
}

void trhepd_destroy(trhepd_context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  t_alloc_stream = c->stream;
  for (DevBuf& b : c->bk) b.release();
  for (DevBuf& b : c->rk) b.release();
  for (DevBuf& b : c->mg) b.release();
  DevBuf* all[] = {&c->asf, &c->b, &c->dchg, &c->ghk, &c->depth, &c->table, &c->pair,
                   &c->Q0, &c->Q1, &c->P, &c->V, &c->D, &c->gam, &c->F, &c->flags, &c->dval,
                   &c->gj, &c->f2, &c->wnsga2, &c->status, &c->split, &c->sgh, &c->sgk,
                   &c->simg, &c->snimg, &c->sst, &c->cva, &c->cvf, &c->cvo, &c->cerr,
                   &c->cref};
  for (DevBuf* b : all) b->release();
  for (int p = 0; p < 3; ++p) {
    c->z[p].release();
    c->ocr[p].release();
    c->ielm[p].release();
    c->st[p].release();
  }
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaStreamDestroy(c->stream);
  delete c;
}

const char* trhepd_last_error(const trhepd_context* c) { return c ? c->err.c_str() : "no context"; }

int trhepd_set_option(trhepd_context* c, int option, double value) {
  if (!c) return TRHEPD_EINVAL;
  switch (option) {
    case TRHEPD_OPT_RENORM_POLICY:
      if (value != 0.0 && value != 1.0) return fail(c, TRHEPD_EINVAL, "renorm policy must be 0 or 1");
      c->renorm_policy = (int)value;
      return TRHEPD_OK;
    case TRHEPD_OPT_RENORM_TAU:
      if (!(value > 0.0)) return fail(c, TRHEPD_EINVAL, "renorm tau must be > 0");
      c->renorm_tau = value;
      return TRHEPD_OK;
    case TRHEPD_OPT_SPLIT_SLICES:
      if (value < 3 || value > 6) return fail(c, TRHEPD_EINVAL, "split slices must be 3..6");
      c->split_slices = (int)value;
      return TRHEPD_OK;
    case TRHEPD_OPT_PROFILE:
      c->profile = value != 0.0;
      return TRHEPD_OK;
    case TRHEPD_OPT_SPLIT_KERNEL:
      if (value != kSplitPersistent && value != kSplitPerTile)
        return fail(c, TRHEPD_EINVAL, "split kernel must be 0 (persistent) or 1 (per tile)");
      c->split_variant = (int)value;
      return TRHEPD_OK;
    case TRHEPD_OPT_GRAPHS:
      c->graphs = value != 0.0;
      return TRHEPD_OK;
    case TRHEPD_OPT_STREAM_PRIORITY: {
      // replace the context's stream by one of the given priority (graphs are not
      // bound to a stream and stay valid)
      if (value < 0 || value > 1) return fail(c, TRHEPD_EINVAL, "stream priority must be in [0, 1]");
      int least = 0, greatest = 0;
      cudaSetDevice(c->device);
      if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess)
        return fail(c, TRHEPD_ECUDA, "stream priority range unavailable");
      const int prio = least + (int)std::lround(value * (greatest - least));
      cudaStream_t ns = nullptr;
      if (cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, prio) != cudaSuccess)
        return fail(c, TRHEPD_ECUDA, "cudaStreamCreateWithPriority failed");
      cudaStreamSynchronize(c->stream);
      cudaStreamDestroy(c->stream);
      c->stream = ns;
      return TRHEPD_OK;
    }
    case TRHEPD_OPT_FUSED_MAX_N:
      if (value < 0) return fail(c, TRHEPD_EINVAL, "fused beam limit must be >= 0");
      c->fused_max_n = (int)value;
      return TRHEPD_OK;
    case TRHEPD_OPT_VALIDATE:
      c->validate = value != 0.0;
      return TRHEPD_OK;
    case TRHEPD_OPT_MAX_CTAS:
      if (value < -1 || value > 1 << 20 || value != (double)(int)value)
        return fail(c, TRHEPD_EINVAL, "CTA cap must be an integer >= -1");
      c->max_ctas = (int)value;
      return TRHEPD_OK;
    case TRHEPD_OPT_PARTICLE:
      if (value != 0.0 && value != 1.0) return fail(c, TRHEPD_EINVAL, "particle must be 0 or 1");
      c->particle = (int)value;
      return TRHEPD_OK;
  }
  return fail(c, TRHEPD_EINVAL, "unknown option");
}

int trhepd_last_stats(const trhepd_context* c, double* out, int n) {
  if (!c || !out) return TRHEPD_EINVAL;
  for (int i = 0; i < n && i < 9; ++i) out[i] = c->stats[i];
  return TRHEPD_OK;
}

int trhepd_plane_group_images(int nsg, int ma, int mb, int na, int nb, double x, double y,
                              double* out_xy, int* count) {
  if (!out_xy || !count || nsg < 1 || nsg > 17 || ma * nb - mb * na == 0) return TRHEPD_EINVAL;
  *count = trhepd::plane_group_images(nsg, ma, mb, na, nb, x, y, out_xy);
  return TRHEPD_OK;
}

int trhepd_structure_factors(trhepd_context* ctx, int nv, const double* gh, const double* gk,
                             int natm, const double* img, const int32_t* nimg, double dx,
                             double dy, double* st) {
  return guarded(ctx, [&] {
    if (nv < 0 || natm < 0 || (!st && nv * natm > 0)) throw std::invalid_argument("bad sizes");
    for (int j = 0; j < natm; ++j)
      if (nimg[j] < 1 || nimg[j] > 12) throw std::invalid_argument("image count must be 1..12");
    std::vector<double> vgh(gh, gh + nv), vgk(gk, gk + nv), vimg(img, img + (size_t)natm * 24);
    std::vector<int> vn(nimg, nimg + natm);
    const double* a = upload(ctx->sgh, vgh, ctx->stream);
    const double* b = upload(ctx->sgk, vgk, ctx->stream);
    const double* c = upload(ctx->simg, vimg, ctx->stream);
    const int* d = upload(ctx->snimg, vn, ctx->stream);
    cd* out = (cd*)ctx->sst.ensure(std::max<size_t>((size_t)nv * natm * sizeof(cd), 16));
    launch_structure_factor(a, b, nv, c, d, natm, dx, dy, out, ctx->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(st, out, (size_t)nv * natm * sizeof(cd), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  });
}

int trhepd_potential_table(trhepd_context* ctx, const trhepd_pot_state* pot, int int_method,
                           int ns, double dz, double* v, double* vi, int* ncol) {
  return guarded(ctx, [&] {
    if (!pot || ns < 1) throw std::invalid_argument("bad arguments");
    Integrator I = integrator_for(int_method);
    std::vector<double> depth = stage_depths(I, ns, dz);
    TableEntry* table = nullptr;
    build_table(ctx, *pot, depth, ctx->table, &table);
    size_t cnt = depth.size() * (size_t)pot->nv;
    std::vector<TableEntry> h(cnt);
    CK(cudaMemcpyAsync(h.data(), table, cnt * sizeof(TableEntry), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t e = 0; e < cnt; ++e) {  // v = (u + w) / 2, vi = (u - w) / 2
      if (v) {
        v[2 * e] = 0.5 * (h[e].u.x + h[e].w.x);
        v[2 * e + 1] = 0.5 * (h[e].u.y + h[e].w.y);
      }
      if (vi) {
        vi[2 * e] = 0.5 * (h[e].u.x - h[e].w.x);
        vi[2 * e + 1] = 0.5 * (h[e].u.y - h[e].w.y);
      }
    }
    if (ncol) *ncol = (int)depth.size();
  });
}

int trhepd_srfref(trhepd_context* ctx, const trhepd_pot_state* pot, int nb, int ns,
                  const int32_t* iv, double dz, int ngr, const int32_t* nbg, const int32_t* iord,
                  const int32_t* ih, const int32_t* ik, double wn, double ghx, double ghy,
                  double gky, double azi, double daz, int naz, double gi, double dg, int ng,
                  int int_method, const double* t1_records, int precision, double* f2,
                  double* angle_deg) {
  return guarded(ctx, [&] {
    if (!pot || !iv || !nbg || !iord || !ih || !ik || !t1_records || !f2)
      throw std::invalid_argument("null argument");
    if (naz < 1 || ng < 1 || ngr < 1) throw std::invalid_argument("naz, ng, ngr must be >= 1");
    if (!valid_precision(precision))
      throw std::invalid_argument("unknown precision form");
    SolveArgs a{pot, nb, ns, iv, dz, ngr, nbg, iord, ih, ik, wn, ghx, ghy, gky,
                azi, daz, gi, dg, naz, ng, int_method, t1_records};
    solve(ctx, a, precision, f2, angle_deg);
  });
}

int trhepd_problem_create(trhepd_context* ctx, const trhepd_pot_state* pot,
                          const trhepd_srfref_args* a, trhepd_problem** out) {
  if (!out) return TRHEPD_EINVAL;
  *out = nullptr;
  auto* pb = new trhepd_problem();
  int rc = guarded(ctx, [&] {
    if (!pot || !a || !a->iv || !a->nbg || !a->iord || !a->ih || !a->ik || !a->t1_records)
      throw std::invalid_argument("null argument");
    if (a->naz < 1 || a->ng < 1 || a->ngr < 1) throw std::invalid_argument("naz, ng, ngr >= 1");
    SolveArgs s{pot, a->nb, a->ns, a->iv, a->dz, a->ngr, a->nbg, a->iord, a->ih, a->ik,
                a->wn, a->ghx, a->ghy, a->gky, a->azi, a->daz, a->gi, a->dg, a->naz, a->ng,
                a->int_method, a->t1_records};
    prepare(ctx, s, *pb);
    CK(cudaStreamSynchronize(ctx->stream));
  });
  if (rc) {
    pb->release();
    delete pb;
    return rc;
  }
  *out = pb;
  return TRHEPD_OK;
}

int trhepd_problem_solve(trhepd_context* ctx, trhepd_problem* pb, int precision) {
  return guarded(ctx, [&] {
    if (!pb) throw std::invalid_argument("null problem");
    if (!valid_precision(precision))
      throw std::invalid_argument("unknown precision form");
    run_checked(ctx, *pb, precision);
  });
}

int trhepd_last_curve_errors(const trhepd_context* ctx, double* out, int n) {
  if (!ctx || !out) return TRHEPD_EINVAL;
  if (ctx->curve_err.empty() || (size_t)n < ctx->curve_err.size()) return TRHEPD_EINVAL;
  std::copy(ctx->curve_err.begin(), ctx->curve_err.end(), out);
  return TRHEPD_OK;
}

int trhepd_problem_compare(trhepd_context* ctx, trhepd_problem* pb, const double* ref_f2,
                           double* out) {
  return guarded(ctx, [&] {
    if (!pb || !ref_f2 || !out) throw std::invalid_argument("null argument");
    cudaStream_t st = ctx->stream;
    const size_t rows = (size_t)pb->nang, nb = (size_t)pb->n;
    double* dref = (double*)ctx->cref.ensure(rows * nb * sizeof(double));
    CK(cudaMemcpyAsync(dref, ref_f2, rows * nb * sizeof(double), cudaMemcpyHostToDevice, st));
    double* e = (double*)ctx->cerr.ensure(2 * rows * sizeof(double));
    launch_curve_distance(pb->f2.as<double>(), dref, (int)rows, (int)nb, e, st);
    CK(cudaGetLastError());
    std::vector<double> h(2 * rows);
    CK(cudaMemcpyAsync(h.data(), e, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double mm = 0.0;
    for (size_t a = 0; a < rows; ++a) mm = std::max(mm, h[2 * a + 1]);
    for (size_t a = 0; a < rows; ++a) {
      out[2 * a] = h[2 * a] / mm;
      out[2 * a + 1] = h[2 * a] / h[2 * a + 1];
    }
  });
}

int trhepd_rocking_convolution(trhepd_context* ctx, const double* angle_deg, const double* f2,
                               int rows, int scan, int nb, double omega_deg, double* out) {
  return guarded(ctx, [&] {
    if (!angle_deg || !f2 || !out || rows < 2 || scan < 2 || nb < 1 || rows % scan ||
        !(omega_deg > 0))
      throw std::invalid_argument("bad convolution arguments");
    cudaStream_t st = ctx->stream;
    double* da = (double*)ctx->cva.ensure((size_t)rows * sizeof(double));
    double* df = (double*)ctx->cvf.ensure((size_t)rows * nb * sizeof(double));
    double* dout = (double*)ctx->cvo.ensure((size_t)rows * nb * sizeof(double));
    CK(cudaMemcpyAsync(da, angle_deg, (size_t)rows * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(df, f2, (size_t)rows * nb * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_rocking_convolution(da, df, rows, scan, nb, omega_deg, dout, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout, (size_t)rows * nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  });
}

int trhepd_problem_convolve(trhepd_context* ctx, trhepd_problem* pb, double omega_deg,
                            double* out) {
  return guarded(ctx, [&] {
    if (!pb || !out || !(omega_deg > 0)) throw std::invalid_argument("bad convolution arguments");
    if (pb->nrep2 < 2) throw std::invalid_argument("the inner scan has fewer than 2 angles");
    cudaStream_t st = ctx->stream;
    const size_t rows = (size_t)pb->nang, nb = (size_t)pb->n;
    double* da = (double*)pb->dang.ensure(rows * sizeof(double));
    CK(cudaMemcpyAsync(da, pb->angle_deg.data(), rows * sizeof(double), cudaMemcpyHostToDevice,
                       st));
    double* dout = (double*)pb->conv.ensure(rows * nb * sizeof(double));
    launch_rocking_convolution(da, pb->f2.as<double>(), (int)rows, pb->nrep2, (int)nb, omega_deg,
                               dout, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout, rows * nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  });
}

int trhepd_batch_solve(trhepd_context* ctx, trhepd_problem* const* problems, int count,
                       int precision) {
  return guarded(ctx, [&] {
    if (!problems || count < 1) throw std::invalid_argument("empty batch");
    if (!valid_precision(precision)) throw std::invalid_argument("unknown precision form");
    batch_solve(ctx, problems, count, precision);
  });
}

int trhepd_problem_fetch(trhepd_context* ctx, trhepd_problem* pb, double* f2, double* angle_deg) {
  return guarded(ctx, [&] {
    if (!pb) throw std::invalid_argument("null problem");
    fetch(ctx, *pb, f2, angle_deg);
  });
}

int trhepd_problem_info(const trhepd_problem* pb, int64_t* out, int n) {
  if (!pb || !out) return TRHEPD_EINVAL;
  int64_t v[6] = {pb->n, pb->nang, pb->ns, pb->nv, pb->ncol, (int64_t)pb->bytes()};
  for (int i = 0; i < n && i < 6; ++i) out[i] = v[i];
  return TRHEPD_OK;
}

void trhepd_problem_destroy(trhepd_problem* pb) {
  if (!pb) return;
  // every solve and fetch synchronises its stream, so the buffers are idle: free
  // them in the order of the legacy stream, which does not wait for other streams
  t_alloc_stream = nullptr;
  pb->release();
  delete pb;
}

struct trhepd_surface_inputs {
  SurfaceInputs S;
};

int trhepd_surf_load(trhepd_context* ctx, const char* bulkp, const char* surf, double dz2,
                     int int_method, trhepd_surface_inputs** out) {
  if (!out) return TRHEPD_EINVAL;
  *out = nullptr;
  auto* h = new trhepd_surface_inputs();
  int rc = guarded(ctx, [&] {
    if (!bulkp || !surf || !(dz2 > 0)) throw std::invalid_argument("bad arguments");
    load_surface_inputs(bulkp, surf, dz2, int_method, h->S);
    structure_factors(ctx, h->S);
  });
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return TRHEPD_OK;
}

void trhepd_surf_free(trhepd_surface_inputs* in) { delete in; }

int trhepd_surf_views(const trhepd_surface_inputs* in, trhepd_pot_state* pot,
                      trhepd_srfref_args* a) {
  if (!in) return TRHEPD_EINVAL;
  const SurfaceInputs& S = in->S;
  if (pot) *pot = pot_view(S);
  if (a) {
    a->nb = S.nb;
    a->ns = S.ns;
    a->iv = S.iv.data();
    a->dz = S.dz;
    a->ngr = S.ngr;
    a->nbg = S.nbg.data();
    a->iord = S.iord.data();
    a->ih = S.ih.data();
    a->ik = S.ik.data();
    a->wn = S.wn;
    a->ghx = S.ghx;
    a->ghy = S.ghy;
    a->gky = S.gky;
    a->azi = S.azi;
    a->daz = S.daz;
    a->naz = S.naz;
    a->gi = S.gi;
    a->dg = S.dg;
    a->ng = S.ng;
    a->int_method = S.int_method;
    a->t1_records = reinterpret_cast<const double*>(S.t1rec.data());
    const bool ng_outer = S.ng > S.naz;
    a->nrep1 = ng_outer ? S.naz : S.ng;
    a->nrep2 = ng_outer ? S.ng : S.naz;
  }
  return TRHEPD_OK;
}

int trhepd_bulk_run(trhepd_context* ctx, const char* bulk_txt, const char* out_path,
                    double* stats) {
  return guarded(ctx, [&] {
    if (!bulk_txt || !out_path) throw std::invalid_argument("null path");
    const int inegpos = ctx->particle == 1 ? 0 : 1;
    std::vector<BulkInputs> B(1);
    load_bulk_inputs(bulk_txt, B[0], inegpos, 0);
    B.resize(B[0].ndom);
    for (int d = 1; d < B[0].ndom; ++d) load_bulk_inputs(bulk_txt, B[d], inegpos, d);
    std::vector<std::vector<std::vector<cd>>> records(B.size());
    double total[4] = {0, 0, 0, 0};
    for (size_t d = 0; d < B.size(); ++d) {  // one blkref per domain (bulkio.f90:150-214)
      double st[4] = {0, 0, 0, 0};
      bulk_solve(ctx, B[d], records[d], st);
      total[0] += st[0];
      total[1] = std::max(total[1], st[1]);
      total[2] = std::max(total[2], st[2]);
      total[3] += st[3];
    }
    if (stats)
      for (int k = 0; k < 4; ++k) stats[k] = total[k];
    write_bulkp(out_path, B, records);
  });
}

int trhepd_surf_run(trhepd_context* ctx, const char* bulkp, const char* surf, double dz2,
                    int int_method, int precision, const char* out_path, double* f2, int max_f2,
                    int* dims) {
  return guarded(ctx, [&] {
    if (!bulkp || !surf || !(dz2 > 0)) throw std::invalid_argument("bad arguments");
    if (!valid_precision(precision)) throw std::invalid_argument("unknown precision form");
    SurfaceInputs S;
    load_surface_inputs(bulkp, surf, dz2, int_method, S);
    if (S.ndom > 1) {
      surf_run_domains(ctx, bulkp, surf, dz2, int_method, precision, S, out_path, f2, max_f2,
                       dims);
      return;
    }
    structure_factors(ctx, S);
    trhepd_pot_state pot = pot_view(S);
    int nang = S.naz * S.ng;
    std::vector<double> out((size_t)nang * S.nb), ang(nang);
    SolveArgs a{&pot, S.nb, S.ns, S.iv.data(), S.dz, S.ngr, S.nbg.data(), S.iord.data(),
                S.ih.data(), S.ik.data(), S.wn, S.ghx, S.ghy, S.gky, S.azi, S.daz, S.gi, S.dg,
                S.naz, S.ng, int_method, reinterpret_cast<const double*>(S.t1rec.data())};
    solve(ctx, a, precision, out.data(), ang.data());
    if (out_path) write_rocking_curves(out_path, S, out.data(), ang.data());
    if (f2) {
      if ((size_t)max_f2 < out.size()) throw std::invalid_argument("f2 buffer too small");
      std::memcpy(f2, out.data(), out.size() * sizeof(double));
    }
    if (dims) {
      dims[0] = S.nb;
      dims[1] = nang;
      dims[2] = S.ns;
      dims[3] = S.nv;
    }
  });
}

}  // extern "C"
