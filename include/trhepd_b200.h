/*
 * trhepd_b200.h — C ABI of the B200 multislice surface solve.
 *
 * Drop-in boundary for the per-glancing-angle multislice path of
 * sim-trhepd-rheed (Fortran).  Each entry point replaces one reference routine;
 * the reference interface it stands in for is cited beside it.  Conventions
 * follow the Fortran side: column-major arrays, 1-based beam/element indices,
 * complex(8) passed as interleaved (re, im) doubles, int32 integers.  All host
 * memory stays caller-owned; device memory belongs to the context.
 *
 * Every function returns TRHEPD_OK (0) or a nonzero status; the message of the
 * last failure is available from trhepd_last_error().  A context is not
 * thread-safe and issues its work on one CUDA stream.
 */
#ifndef TRHEPD_B200_H
#define TRHEPD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum trhepd_status {
  TRHEPD_OK = 0,
  TRHEPD_EINVAL = 1,      /* bad argument (sizes, indices, method) */
  TRHEPD_ECUDA = 2,       /* CUDA runtime error */
  TRHEPD_ENONFINITE = 3,  /* NaN/Inf or an exactly zero pivot met on the device */
  TRHEPD_ETIMEOUT = 4,    /* a bounded device wait gave up */
  TRHEPD_ENOMEM = 5,      /* device allocation failed or over the memory budget */
  TRHEPD_EIO = 6          /* input file missing or malformed */
};

/* precision forms of the surface solve */
enum trhepd_precision {
  TRHEPD_FP64 = 0,        /* all-FP64 (DMMA) */
  TRHEPD_SPLIT_BF16 = 1,  /* stage products from BF16 slices on tcgen05 (FP32 accumulators),
                             FP64 elsewhere */
  TRHEPD_SPLIT_INT8 = 2   /* stage products from signed 8-bit digit slices on tcgen05
                             (exact INT32 accumulators, 3 to 6 slices), FP64 elsewhere */
};

/* options (trhepd_set_option) */
enum trhepd_option {
  TRHEPD_OPT_RENORM_POLICY = 1, /* 0: Gershgorin test > 1e3 per angle and slice (reference)
                                   1: growth bound: every floor(tau / ((kappa_max + 1) dz))
                                      slices, kappa_max the largest evanescent decay constant */
  TRHEPD_OPT_RENORM_TAU = 2,    /* growth bound ln(cond) between renormalisations (policy 1) */
  TRHEPD_OPT_SPLIT_SLICES = 3,  /* slices per operand in the split forms (BF16 3..5, INT8 3..6;
                                   each INT8 slice adds 8 bits: 31 at 4, 47 at 6) */
  TRHEPD_OPT_PROFILE = 4,       /* nonzero: time every stage-product launch with CUDA events */
  TRHEPD_OPT_SPLIT_KERNEL = 5,  /* BF16 split kernel: 0 persistent, one CTA per SM, epilogue of
                                   a tile overlapped with the next tile's MMAs (default);
                                   1 one CTA per tile */
  TRHEPD_OPT_GRAPHS = 6,        /* nonzero (default): a resident problem's solve is captured
                                   into a CUDA graph on its second solve with the same
                                   options and replayed afterwards; 0: launch directly */
  TRHEPD_OPT_FUSED_MAX_N = 7,   /* FP64 RKN solves (int_method 5, 6) with 2 <= nb <= this value
                                   (at most 64; default 64, 0 disables) integrate every slice in
                                   one launch, one CTA per angle, state in shared memory */
  TRHEPD_OPT_STREAM_PRIORITY = 8, /* 0 (default, lowest) .. 1 (highest): priority of the
                                   context's stream; the block scheduler starts pending work of
                                   higher-priority streams first when several contexts share a GPU */
  TRHEPD_OPT_VALIDATE = 9,      /* nonzero: every split-form solve (trhepd_srfref,
                                   trhepd_problem_solve) is checked against the plain FP64 form
                                   of the same problem, solved first with the same options; the
                                   per-curve errors are read with trhepd_last_curve_errors.  Costs
                                   one FP64 solve (about 3x the INT8 solve at N = 521) */
  TRHEPD_OPT_PARTICLE = 10,     /* trhepd_bulk_run: 0 positrons (TRHEPD, default), 1 electrons
                                   (RHEED): the program-level switch ep = 'P' / 'E' of bulk.exe
                                   (bulkm.f90:21-24), written to bulkP.b as inegpos; the surface
                                   solve follows the inegpos of the file it reads
                                   (surfio.f90:152) */
  TRHEPD_OPT_MAX_CTAS = 11      /* 0 (default): the stage-product kernels use every SM; k > 0:
                                   the persistent split kernels run at most k CTAs and the FP64
                                   stage kernel at most 2k blocks, leaving the other SMs to
                                   kernels of other contexts (streams) on the same GPU; -1: the
                                   split kernels run one CTA per tile, so higher-priority work of
                                   other contexts starts between tiles */
};

typedef struct trhepd_context trhepd_context;

int trhepd_create(int device, trhepd_context** ctx);
void trhepd_destroy(trhepd_context* ctx);
const char* trhepd_last_error(const trhepd_context* ctx);
int trhepd_set_option(trhepd_context* ctx, int option, double value);
/* counters of the last solve: out[0] renormalisations, out[1] stage products,
   out[2] device milliseconds of the solve, out[3] stage columns, out[4] summed
   device milliseconds of the stage-product kernels (TRHEPD_OPT_PROFILE only),
   out[5] kernels launched, out[6] of which renormalisation kernels, out[7] summed
   device milliseconds of the tensor-core kernel alone inside the stage products
   (TRHEPD_OPT_PROFILE only), out[8] summed device milliseconds of the end-of-slice
   renormalisations (TRHEPD_OPT_PROFILE only) */
int trhepd_last_stats(const trhepd_context* ctx, double* out, int n);
/* Per-curve errors of the last validated split-form solve (TRHEPD_OPT_VALIDATE), one
   rocking curve per angle row: out[3a] = max over every spot of |I - I64| / |I64| (a
   spot with I64 = 0 counts 0 when I = 0 too), out[3a+1] = max |I - I64| over the
   curve's largest |I64|, out[3a+2] = the curve's largest |I64|.  n: capacity of out in
   doubles (at least 3 x angles).  EINVAL when the last solve was not a validated
   split-form solve.  No counterpart in the reference, whose only form is FP64. */
int trhepd_last_curve_errors(const trhepd_context* ctx, double* out, int n);

/*
 * Structure state of the potential, mirroring module mod_scpot3
 * (sim-trhepd-rheed/src/surfio.f90:18-27).  Bulk atoms come first in ielm/z/ocr.
 */
typedef struct trhepd_pot_state {
  int nv, nvb, natms, natmb, nelm, nabr, nabi;
  const int32_t* ielm;  /* natmb+natms, 1-based element index */
  double cc, smesh;
  const double* z;      /* natmb+natms (zoffset applied) */
  const double* dchg;   /* nelm */
  const double* Ghk;    /* nv */
  const double* ocr;    /* natmb+natms */
  const double* b;      /* (6, nelm) */
  const double* asf;    /* (nv, 6, nelm) */
  const double* st0;    /* complex (nv, natms) */
  const double* st1;    /* complex (nvb, natmb) */
  const double* st2;    /* complex (nvb, natmb) */
} trhepd_pot_state;

/*
 * Structure factors of `natm` atoms for `nv` Fourier components on the GPU.
 * Replaces scpot_stf / strfac (sim-trhepd-rheed/src/scpot.f90:100-110,
 * strfac.f90:5-76).  img: per atom 12 (x, y) image pairs in 1x1-lattice units
 * (from trhepd_plane_group_images), nimg: image counts.  st: complex (nv, natm).
 */
int trhepd_structure_factors(trhepd_context* ctx, int nv, const double* gh, const double* gk,
                             int natm, const double* img, const int32_t* nimg, double dx,
                             double dy, double* st);

/* Plane-group orbit of one atom (strfac.f90:15-64, the 17 groups at :88-527). */
int trhepd_plane_group_images(int nsg, int ma, int mb, int na, int nb, double x, double y,
                              double* out_xy, int* count);

/*
 * Stage potential tables of an integrator: v, vi complex (nv, ncol) with
 * ncol = ns for int_method 4, 6*ns+1 for 5, 11*ns+1 for 6 and 2*ns+1 for 7 and 8.
 * Replaces hp_int_init4/6 (sim-trhepd-rheed/src/surf_prkn.f90:174-197),
 * m2_int_init (surf_magnus.f90:4-20), rk4_int_init (surf_rk.f90:4-25) and
 * comp_scpot (surfio.f90:29-41).
 */
int trhepd_potential_table(trhepd_context* ctx, const trhepd_pot_state* pot, int int_method,
                           int ns, double dz, double* v, double* vi, int* ncol);

/*
 * Same tables as trhepd_potential_table (every int_method 1-8), for callers that
 * cannot allocate device memory (a host that hands the whole GPU to its own memory
 * pool at start-up, or a service whose device memory is planned once): no
 * cudaMalloc/cudaFree, no context.  Its device scratch (input copies and the table)
 * is one 32 MiB array inside the library, held by every GPU that loads it until the
 * process exits.  Works on the current device and the legacy default stream,
 * synchronously.  Every call looks up the array's device address on the current
 * device; the first call on a device also loads the library's device code there, so
 * make that first call before any stream capture.  Calls share the array (it keeps
 * the last call's contents; nothing in it has to start at zero, since each call
 * writes what it reads), so calls whose GPU work overlaps race.  Returns
 * TRHEPD_ENOMEM when the inputs and the table need more than the 32 MiB, and
 * TRHEPD_EINVAL for an int_method outside 1-8.
 * This entry point has no counterpart in the reference.
 */
int trhepd_potential_table_noalloc(const trhepd_pot_state* pot, int int_method, int ns,
                                   double dz, double* v, double* vi, int* ncol);

/*
 * Surface solve of every (azimuth, glancing angle) of one domain in one batch.
 * Replaces srfref (sim-trhepd-rheed/src/surflf.f90:7-171) including its
 * integrator call (lf_int_spa surf_magnus.f90:46-110, hp_int4 / hp_int6
 * surf_prkn.f90:123-141, rk4_int surf_rk.f90:27-91, rk4_intgs surf_rk.f90:93-156:
 * int_method 4-8; the Magnus integrators 1-3 as well) and the intensity
 * formula (surflf.f90:142-151).  Arguments keep srfref's names and meaning;
 * t1_records holds the bulk reflection records srfref reads from unit 1
 * (surflf.f90:65-72): nrep1*nrep2 angles, each ngr blocks of nbg(l)^2 complex
 * values in file order.  f2 receives (nb, nrep1*nrep2) intensities,
 * angle_deg the printed angle of each row.
 */
int trhepd_srfref(trhepd_context* ctx, const trhepd_pot_state* pot, int nb, int ns,
                  const int32_t* iv, double dz, int ngr, const int32_t* nbg, const int32_t* iord,
                  const int32_t* ih, const int32_t* ik, double wn, double ghx, double ghy,
                  double gky, double azi, double daz, int naz, double gi, double dg, int ng,
                  int int_method, const double* t1_records, int precision, double* f2,
                  double* angle_deg);

/*
 * C++ equivalent of surfio for the first domain (sim-trhepd-rheed/src/
 * surfio.f90:60-381): parses bulkP.b + surf.txt, applies the slicing rule for
 * dz2, forms the mod_scpot3 state (structure factors summed on the GPU) and the
 * srfref arguments.  The handle owns every array the two views point into.
 */
typedef struct trhepd_surface_inputs trhepd_surface_inputs;

typedef struct trhepd_srfref_args {
  int nb, ns;
  const int32_t* iv;      /* (nb, nb) */
  double dz;
  int ngr;
  const int32_t *nbg, *iord, *ih, *ik;
  double wn, ghx, ghy, gky, azi, daz;
  int naz;
  double gi, dg;
  int ng, int_method;
  const double* t1_records;
  int nrep1, nrep2;       /* angle schedule sizes (surflf.f90:43-49) */
} trhepd_srfref_args;

int trhepd_surf_load(trhepd_context* ctx, const char* bulkp, const char* surf, double dz2,
                     int int_method, trhepd_surface_inputs** out);
void trhepd_surf_free(trhepd_surface_inputs* in);
int trhepd_surf_views(const trhepd_surface_inputs* in, trhepd_pot_state* pot,
                      trhepd_srfref_args* args);

/*
 * Device-resident form of one srfref call, for callers that solve the same
 * structure repeatedly (structure refinement, serving, benchmarking): create
 * uploads the inputs and builds the stage tables in device memory once; solve
 * integrates every angle reading device memory only and leaves the intensities
 * on the device; fetch copies them (and the printed angles) to the host.
 * trhepd_srfref is create + solve + fetch + destroy.
 * info: out[0..5] = nb, nangles, ns, nv, stage columns, device bytes held.
 */
typedef struct trhepd_problem trhepd_problem;
int trhepd_problem_create(trhepd_context* ctx, const trhepd_pot_state* pot,
                          const trhepd_srfref_args* args, trhepd_problem** out);
int trhepd_problem_solve(trhepd_context* ctx, trhepd_problem* pb, int precision);
/* Solve several resident problems together (no counterpart in the reference,
   whose driver solves one structure at a time; this is the candidate-structure
   batch of a refinement step).  Problems with int_method 5 or 6 and
   2 <= nb <= TRHEPD_OPT_FUSED_MAX_N are integrated by shared launches in their own
   buffers: one launch per integrator for up to 192 problems, any mix of beam
   counts, slice counts and angle grids, in plain FP64.  The other problems are
   solved one after another in `precision`.  Each problem's intensities are then
   read with trhepd_problem_fetch; trhepd_last_stats reports the whole batch. */
int trhepd_batch_solve(trhepd_context* ctx, trhepd_problem* const* problems, int count,
                       int precision);

/* Gaussian convolution of rocking curves (make_convolution.py,
   str-lapack/tool/make_convolution.py:21-29, 97-109): f2[rows][nb] with angles
   angle_deg[rows] (degrees) in blocks of `scan` consecutive rows (one block per
   outer loop index of srfref, so scan = the inner scan's angle count);
   out[i][b] = sum_k f2[k][b] g(theta_i - theta_k) dtheta within a block, g the
   normalised Gaussian of FWHM omega_deg, dtheta the block's first angle step. */
int trhepd_rocking_convolution(trhepd_context* ctx, const double* angle_deg, const double* f2,
                               int rows, int scan, int nb, double omega_deg, double* out);
/* The same on a solved resident problem's intensities, on the device (no round
   trip of the intensities); out: (nangles, nb) host buffer.  No counterpart in the
   reference beyond make_convolution.py. */
int trhepd_problem_convolve(trhepd_context* ctx, trhepd_problem* pb, double omega_deg,
                            double* out);
int trhepd_problem_fetch(trhepd_context* ctx, trhepd_problem* pb, double* f2, double* angle_deg);
/* The curve-comparison metric of the reference's regression scripts
   (test/test23/compare.py:50-67) between a solved resident problem's intensities
   (the computed curves, compare.py's first file) and ref_f2 (nangles, nb) host
   curves (its second file), reduced on the device: per angle row a,
   out[2a] = ||I_a - ref_a||_2 / max_b ||I_b||_2 and out[2a+1] = ||I_a - ref_a||_2 /
   ||I_a||_2 (a zero norm counts 1).  out: (nangles, 2) host buffer. */
int trhepd_problem_compare(trhepd_context* ctx, trhepd_problem* pb, const double* ref_f2,
                           double* out);
int trhepd_problem_info(const trhepd_problem* pb, int64_t* out, int n);
void trhepd_problem_destroy(trhepd_problem* pb);

/*
 * bulk.exe (sim-trhepd-rheed/src/bulkm.f90:207-256 + bulkio.f90:10-223 + blkref
 * bulk.f90:7-128) for every domain (NDOM >= 1, each at azimuth azi + rdom), positrons
 * or electrons (TRHEPD_OPT_PARTICLE): reads bulk.txt, computes every
 * (angle, beam group) reflection matrix on the GPU and writes bulkP.b in the
 * reference's record layout.  stats (optional): out[0] device ms, out[1] layers
 * iterated, out[2] double-angle steps, out[3] (angle, group) items.
 */
int trhepd_bulk_run(trhepd_context* ctx, const char* bulk_txt, const char* out_path,
                    double* stats);

/*
 * surf.exe (surfm.f90:6-97 + surfio.f90:60-381): reads bulkP.b and surf.txt,
 * slices the surface for dz2, solves on the GPU and, if out_path is not NULL,
 * writes the rocking-curve file in the reference format.  With NDOM > 1 every
 * domain is solved (azimuth azi + rdom(d)) and the weighted sum of the rotated
 * domains (domainsum.f90:7-121) is formed on the device: out_path receives the
 * summed file (E12.4 rows, the beams of the domain with the most beams) and the
 * same path with the extension .md every domain's rows, as the reference writes
 * them.  f2 (optional) receives (nb, nangles), the summed intensities for
 * NDOM > 1; dims (optional) receives {nb, nangles, ns, nv}.
 */
int trhepd_surf_run(trhepd_context* ctx, const char* bulkp, const char* surf, double dz2,
                    int int_method, int precision, const char* out_path, double* f2,
                    int max_f2, int* dims);

#ifdef __cplusplus
}
#endif
#endif /* TRHEPD_B200_H */
