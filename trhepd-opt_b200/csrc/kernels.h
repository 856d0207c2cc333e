// Launchers for the multislice surface-solve kernels (sm_100a).  All matrices of
// the batched state are complex128, row-major per angle and stacked by angle:
// element (i, j) of angle a lives at [(a * n + i) * ld + j].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace trhepd {

// One atom contribution set of the potential (a "part" of comp_scpot,
// sim-trhepd-rheed/src/surfio.f90:29-41).
struct PotPart {
  const double* z;      // atom heights (device)
  const double* ocr;    // occupancies (device)
  const int* ielm;      // 0-based element indices (device)
  const cd* st;         // structure factors (nk x natm, column-major, device)
  int natm;
  int nk;               // Fourier components this part contributes to
  double zshift;        // depth offset of this part (zi - cc, zi, zi + cc)
  double rmesh;         // area ratio factor (1 or smesh)
};

struct PotInputs {
  PotPart part[3];
  const double* asf;    // (nv, mab, nelm) column-major (device)
  const double* b;      // (mab, nelm) column-major (device)
  const double* dchg;   // (nelm) (device)
  const double* ghk;    // (nv) (device)
  int nv, nelm, nabr, nabi, mab;
};

struct TableEntry {  // per (stage column, Fourier component): u = v + vi, w = v - vi
  cd u, w;
};

// Several problems stacked in one integration: problem b owns the rows_b stacked
// rows from b * rows_b and its stage matrix at V + b * vstride.  rows_b = 0
// (the default): one problem.
struct StackedRows {
  int rows_b = 0;
  long long vstride = 0;
};

// K3: stage potential table T[c * nv + k] for the ncol depths in `depth`.
void launch_potential_table(const PotInputs& in, const double* depth, int ncol, TableEntry* table,
                            cudaStream_t st);

// K2: structure factors st[k + j*nv] = sum over plane-group images.
// img holds (x, y) pairs per atom: img[(j * 12 + m) * 2 + {0,1}], nimg[j] images.
void launch_structure_factor(const double* gh, const double* gk, int nv, const double* img,
                             const int* nimg, int natm, double dx, double dy, cd* st,
                             cudaStream_t stream);

// K4: shared stage matrix V (kpad x ld, row-major) from table column `col`.
// pair[k * n + j] = 0-based table index of beam pair (k, j) (diagonal: 0).
// drop_diag: zero the diagonal (the split path applies it in FP64) and store its
// value at V[kpad * ld]; V must hold (kpad + 1) * ld elements.
void launch_gather_stage(const TableEntry* table_col, const int* pair, int n, int kpad, int ld,
                         bool drop_diag, cd* V, cudaStream_t st);
// The stage matrices of a stacked group (tables[b] + coloff for problem b).
void launch_gather_stage_multi(const TableEntry* const* tables, size_t coloff, const int* pair,
                               int n, int kpad, int ld, bool drop_diag, cd* V, long long vstride,
                               int nprob, cudaStream_t st);

// Elementwise stage with Q = I:  P += cb*(V + diag(D_a));  Q = I + ca*P.
void launch_stage_identity(cd* Q, cd* P, const cd* V, const cd* D, int nang, int n, int ld,
                           double cb, double ca, cudaStream_t st, StackedRows sr = {});

// K5 (FP64 DMMA): P += cb*(Q V + Q o D_a);  Qo = Q + ca*P   (all angles, one launch).
// max_sms > 0: at most two blocks per SM on that many SMs, walking the tiles.
void launch_stage_gemm_f64(const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D, int nang, int n,
                           int ld, int kpad, double cb, double ca, cudaStream_t st,
                           StackedRows sr = {}, int max_sms = 0);

// Q := I for angles whose flag is set (flag == nullptr: all angles).
void launch_set_identity(cd* Q, const int* flag, int nang, int n, int ld, cudaStream_t st);

// K7: Gershgorin estimate per angle (matcomp.f90:498-528); flag[a] = d > 1e3 or force.
void launch_cond_est(const cd* Q, int nang, int n, int ld, int force, int* flag, double* dval,
                     cudaStream_t st);

// Largest beam count of the batched path: the Gauss-Jordan panel keeps n x 16
// complex values plus 12 KB in shared memory (227 KB per block).
constexpr int kMaxBeams = 832;

// K8: Q^{-1} P by blocked Gauss-Jordan with partial pivoting, per flagged angle.
// scratch: gj_scratch_bytes(nang, n) bytes.  arith: the rounding of the complex
// multiply-adds:
//   kGjProductFirst  products formed first, then added (the reference's rounding),
//                    shared-memory panel and one thread per trailing column (the
//                    boundary transforms and the bulk solve),
//   kGjFused         four fused multiply-adds per complex product in the
//                    row-per-thread panel, the trailing update on the FP64 tensor
//                    path (the split forms' renormalisations),
//   kGjFp64Mma       the row-per-thread panel with products formed first, the
//                    trailing update on the FP64 tensor path (the FP64 form's
//                    renormalisations).
// Beyond 640 beams every form takes the shared-memory kernels.
enum GjArith { kGjProductFirst = 0, kGjFused = 1, kGjFp64Mma = 2 };
size_t gj_scratch_bytes(int nang, int n);
void launch_gauss_jordan(cd* Q, cd* P, const int* flag, int nang, int n, int ld, void* scratch,
                         unsigned* status, cudaStream_t st, int arith = kGjProductFirst);

// RK4 stage combination (rk4_int, surf_rk.f90:27-91); see kernels_f64.cu.
void launch_rk4_combine(cd* Q, cd* P, cd* Qt, cd* Pt, cd* KP, cd* SQ, cd* SP, int j, double w,
                        double step, double h6, int nang, int n, int ld, cudaStream_t st);
// invstransh (matcomp.f90:140-172): Q = I + F^H, P = I - F^H, from F (nang x n x n, row-major).
void launch_invstransh_build(const cd* F, cd* Q, cd* P, int nang, int n, int ld, cudaStream_t st);
// P(i,j) = i * P(i,j) * conj(g_i)  (after the solve)
void launch_invstransh_finish(cd* P, const cd* gam, int nang, int n, int ld, cudaStream_t st);
// stransh (matcomp.f90:174-196): Q = conj(G) - iP, P = conj(G) + iP.
void launch_stransh_build(cd* Q, cd* P, const cd* gam, int nang, int n, int ld, cudaStream_t st);
// intensities (surflf.f90:142-151) from R = Q^{-1}P: f2(i) = |R(nb0,i)|^2 wnsga2/Re(g_i)
void launch_intensities(const cd* R, const cd* gam, const double* wnsga2, int nang, int n, int ld,
                        int nb0, double* f2, cudaStream_t st);
// Non-finite scan of a state buffer (sets kStatusNonFinite).
void launch_check_finite(const cd* X, size_t count, unsigned* status, cudaStream_t st);
// Gaussian convolution (FWHM omega, degrees) of rocking curves f2[rows][nb] along
// their angles ang[rows], in blocks of `scan` consecutive rows (make_convolution.py).
void launch_rocking_convolution(const double* ang, const double* f2, int rows, int scan, int nb,
                                double omega, double* out, cudaStream_t st);

}  // namespace trhepd
