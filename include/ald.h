/*
 * ald.h -- C ABI of libald, the B200 (sm_100a) implementation of THERMACOND's
 * three-phonon hot path (KeivanS/Anharmonic-lattice-dynamics).
 *
 * Each entry point replaces one Fortran subroutine of the job=1 sequence in
 * THERMACOND/kappa.f90:389-871 and keeps its argument meaning:
 *   - arrays are HOST pointers in the reference's Fortran layout
 *     (column-major, first index fastest) with 1-based index *values*;
 *   - complex arrays are interleaved (re, im) doubles, i.e. complex(8);
 *   - the caller owns every host buffer; the context owns device memory and
 *     never keeps a host pointer past the call;
 *   - every call returns an int status, 0 = success.  The nonzero codes map
 *     the reference's `stop` sites (a Fortran shim turns them into `stop`).
 *
 * Calls on one context are blocking and not thread-safe (the reference runs
 * one thread per MPI rank); separate contexts may run concurrently.
 */
#ifndef ALD_H
#define ALD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum ald_status {
  ALD_OK = 0,
  ALD_ERR_ARG = 1,          /* bad argument, sizes or ksubset                        */
  ALD_ERR_IO = 2,           /* input file missing/malformed: read_params, read_input_fit,
                               read_lattice, read_fc234, read_born stops (rest.f90:2-443,3580) */
  ALD_ERR_NOT_KPOINT = 3,   /* get_k_info: "vector is not a kpoint" (rest.f90:3052-3055)  */
  ALD_ERR_DEN_ZERO = 4,     /* matrix_elt_simplified: den=0 (sub.f90:6002-6004)          */
  ALD_ERR_NBE = 5,          /* nbe: w<=0 or t<=0 (extratools.f90:263-270)                */
  ALD_ERR_INDEX = 6,        /* k-index round trip mismatch (sub.f90:1127-1133,8022-8025) */
  ALD_ERR_CUDA = 7,         /* CUDA runtime or kernel error                              */
  ALD_ERR_UNSUPPORTED = 8,  /* input outside what this build implements (message says)   */
  ALD_ERR_NOMEM = 9,        /* device allocation failed                                  */
  ALD_WARN_CG_MAXITER = 100 /* cg_quadratic reached max_iter; results are still returned */
};

enum ald_delta { ALD_DELTA_TETRA = 0, ALD_DELTA_GAUSS = 1 };
/* ALD_MIXED: the V3 contraction in reduced precision with FP32 accumulation --
 * for 3 bands the phase-class sums, from 9 bands up both eigenvector mode
 * products run on the tensor cores (split-FP16 tcgen05 MMAs), 6 bands in FP32
 * on the CUDA cores; from 9 bands up the pairs that involve a mode of
 * vanishing frequency are formed again in FP64.  ALD_MIXED_FP32 uses the FP32
 * CUDA-core form where one exists.  Inside the pipeline the delta weights and
 * the stored collision matrix are FP32 too; eigensolve, Bose factors, the sums
 * into Q, CG vectors and kappa stay FP64. */
enum ald_precision { ALD_FP64 = 0, ALD_MIXED = 1, ALD_MIXED_FP32 = 2 };
enum ald_cg_stop { ALD_CG_REFERENCE = 0, ALD_CG_RESIDUAL = 1 };

#define ALD_DET_AUTO (-1)

typedef struct ald_options {
  int delta;         /* ALD_DELTA_TETRA (reference, calculate_FGR_mpi2) or ALD_DELTA_GAUSS
                        (extension: delta_g of width `width_cm`, extratools.f90:239)    */
  int precision;     /* ALD_FP64, ALD_MIXED or ALD_MIXED_FP32 (enum ald_precision)      */
  int cg_stop;       /* ALD_CG_REFERENCE: (dv/v)^2 < 10^(-2*cg_ndig) (cg.f90:30,47);
                        ALD_CG_RESIDUAL: |Ax-b|/|b| < cg_tol                            */
  int cg_max_iter;   /* 100 at kappa.f90:846                                            */
  int cg_ndig;       /* 2 at kappa.f90:846                                              */
  double cg_tol;     /* for ALD_CG_RESIDUAL                                             */
  double width_cm;   /* Gaussian width in cm^-1 for ALD_DELTA_GAUSS (<=0: latdyn width) */
  int device;        /* CUDA device ordinal                                             */
  size_t chunk_bytes;/* device bytes for one chunk of |V3|^2 rows (0 = automatic)      */
  int deterministic; /* the pipeline's tetrahedron delta (up to 16 bands):
                        1: sums with the same bits on every run (two passes, the second
                        with fixed-point integer atomics; about 2.4x the delta's time),
                        0: FP64 atomics in arrival order (last bits vary between runs),
                        ALD_DET_AUTO (-1, the default): 1 for ALD_FP64, 0 otherwise    */
} ald_options;

typedef struct ald_ctx ald_ctx;

/* sizes of a loaded system */
typedef struct ald_info {
  int ndyn;          /* 3*natoms0 (bands)             */
  int natoms0;       /* atoms in the primitive cell   */
  int nc[3];         /* q-mesh                        */
  int nkc;           /* nc(1)*nc(2)*nc(3)             */
  int nibz;          /* IBZ size (get_weights rule)   */
  int nterms2, nterms3;
  int natoms;        /* supercell atoms in lat_fc.dat */
  int lattpgcount;   /* lattice point-group order     */
  int born_flag;
  double tempk;      /* tmin of latdyn.params         */
  double width_cm;   /* width of latdyn.params        */
  double volume_r;   /* primitive-cell volume (A^3)   */
} ald_info;

void ald_default_options(ald_options* opt);

/* Message of the last failing call on this thread. */
const char* ald_last_error(void);

/* Reads latdyn.params, structure.params, lat_fc.dat, fc2.dat, fc3.dat and
 * dielectric.params from `dir` with the reference readers' record rules
 * (read_params rest.f90:2, read_input_fit :78, read_lattice :152,
 * read_fc234 :303, read_born :3580), builds the lattice point group
 * (force_constants_init force_constants.f90:3-186), the q-mesh
 * (make_kp_reg modules.f90:1721), e(-q) pairs (get_negatives rest.f90:3208),
 * the IBZ (get_weights modules.f90:2006) and the tetrahedra
 * (make_kp_reg_tet tetrahedron.f90:2), and uploads the tables. */
int ald_create_from_dir(const char* dir, const ald_options* opt, ald_ctx** out);
void ald_destroy(ald_ctx* ctx);
/* Device blocks of any size freed by the library (ald_destroy, workspace
 * resizes) stay reserved in a per-device cache, up to 32 GiB per device, and
 * are reused by later allocations of the same size: a context created after
 * another one skips cudaMalloc.  The cache gives its blocks back when
 * cudaMalloc runs out of memory; ald_release_cached_memory returns all of them
 * to the driver now (no counterpart in the reference). */
void ald_release_cached_memory(void);
int ald_get_info(ald_ctx* ctx, ald_info* info);

/* Host-only: read the input files of `dir` and build the mesh/IBZ tables
 * without touching a GPU (no context).  `info` is filled; any array pointer
 * may be NULL (call once with NULLs to learn nkc and nibz).  Layouts as in
 * ald_get_mesh.  Mirrors the setup part of kappa.f90:185-337. */
int ald_read_mesh(const char* dir, ald_info* info, double* kpc, int* mapibz, int* mapinv, double* kibz,
                  double* wibz);

/* Mesh and IBZ tables (modules.f90:1721-1784, 2006-2160):
 * kpc(3,nkc) Cartesian 1/A including 2*pi (the FP32-fraction mesh that
 * get_frequencies diagonalises on), mapibz(nkc), mapinv(nibz) 1-based,
 * kibz(3,nibz), wibz(nibz).  Any pointer may be NULL. */
int ald_get_mesh(ald_ctx* ctx, double* kpc, int* mapibz, int* mapinv, double* kibz, double* wibz);

/* get_frequencies (rest.f90:2230) on the full mesh followed by subst_eivecs
 * (rest.f90:3262): eigenval(ndyn,nkc) = |omega^2| (eV/A^2/amu),
 * eigenvec(ndyn,ndyn,nkc) complex, veloc(3,ndyn,nkc) in units of c.
 * Outputs may be NULL (then they are only kept on the device). */
int ald_get_frequencies(ald_ctx* ctx, double* eigenval, double* eigenvec, double* veloc);

/* Load eigenpairs and velocities from the host instead of computing them
 * (the module arrays `eigenval`, `eigenvec`, `veloc` the reference passes
 * between stages).  Same layouts as ald_get_frequencies. */
int ald_set_phonons(ald_ctx* ctx, const double* eigenval, const double* eigenvec, const double* veloc);

/* calculate_w3_ibz_split_sq (sub.f90:1050): |V3|^2 in cm^-2 for IBZ rows
 * ksubset(1)..ksubset(2) (1-based, inclusive) against every mesh q2, with
 * q3 = -q1-q2 folded on the mesh.  v33s8(nk1,nkc,ndyn,ndyn,ndyn),
 * nk1 = ksubset(2)-ksubset(1)+1. */
int ald_calculate_w3_ibz_split_sq(ald_ctx* ctx, const int ksubset[2], double* v33s8);

/* calculate_FGR_mpi2 (sub.f90:7199): tetrahedron (or Gaussian) weighted
 * |V3|^2: P1smpi, P2smpi(nk1,nkc,ndyn,ndyn,ndyn).  v33s8 as returned by
 * ald_calculate_w3_ibz_split_sq for the same ksubset. */
int ald_calculate_fgr(ald_ctx* ctx, const int ksubset[2], const double* v33s8, double* P1smpi, double* P2smpi);

/* weight_tet (tetrahedron.f90:188-384, with SSORT tetrahedron.f90:716-738):
 * the linear-tetrahedron weights of every tetrahedron at one energy e, on
 * the device.  The module array tet(:) of the reference becomes two host
 * arrays: w(4,ntet) = tet(i)%p(k)%w (corner energies, REAL(8); rounded to
 * REAL as the reference does) and c(4,ntet) = tet(i)%p(k)%c (out).  fp32 = 0
 * is the arithmetic of the FP64 pipeline, bit for bit the reference's;
 * fp32 = 1 the FP32 weights of the mixed pipeline (a few FP32 ulps per
 * weight).  Synchronous; needs no context. */
int ald_weight_tet(int ntet, const double* w, double e, int fp32, double* c);

/* distribution (sub.f90:1955): frequency(nkc,ndyn) cm^-1, dist(nkc,ndyn). */
int ald_distribution(ald_ctx* ctx, double tempk, double* frequency, double* dist);

/* calculate_tauRTA_mpi2 (sub.f90:7953): Q, Q_N, Q_U(nk1,ndyn) and the
 * Bose-weighted P1, P2(nk1,nkc,ndyn,ndyn,ndyn) (P1/P2 may be NULL). */
int ald_calculate_tau_rta(ald_ctx* ctx, const int ksubset[2], double tempk, const double* P1smpi,
                          const double* P2smpi, double* Q, double* QN, double* QU, double* P1, double* P2);

/* calculate_RTA_distributionfunction (sub.f90:1238) + mode_kappa
 * (sub.f90:1292): FFF(nibz,ndyn,3) and kappa(ndyn,3,3) in W/m/K from
 * Q(nibz,ndyn). */
int ald_rta_kappa(ald_ctx* ctx, double tempk, const double* Q, double* FFF, double* kappa);

/* CollisionMatrix_mpi (sub.f90:3034): Collision_Matrix(nk1*ndyn*3,
 * nibz*ndyn*3) from the Bose-weighted P1, P2 of the same ksubset. */
int ald_collision_matrix(ald_ctx* ctx, const int ksubset[2], const double* P1, const double* P2, double* CM);

/* CollisionMatrix_iso (sub.f90:3387): the collision matrix of iso=1 over all
 * IBZ rows, Collision_Matrix(nibz*ndyn*3, nibz*ndyn*3) column-major, from
 * P1, P2(nibz,nkc,ndyn,ndyn,ndyn) Bose-weighted and Piso(nibz,ndyn).  The
 * diagonal arm takes -(sum(P1 + P2/2) + Piso), every other arm
 * sum_l3 (-P1(arm) + P1(q1+arm) + P2(arm)) + Piso, as the reference does. */
int ald_collision_matrix_iso(ald_ctx* ctx, const double* P1, const double* P2, const double* Piso, double* CM);

/* Isotope scattering (iso=1 in latdyn.params).
 * ald_p_iso_split replaces P_iso_split (sub.f90:4825-4961): Piso(nk1,ndyn)
 * of the IBZ rows ksubset, with g per primitive atom from cal_giso
 * (sub.f90:4695): the mass variance of the element's natural isotopes.
 * The element table covers Ar, C, Cl, Ge, Na, Si; ald_set_isotope_g sets g
 * (natoms0 values) for any other, ald_get_isotope_g reads it back
 * (ALD_ERR_UNSUPPORTED for an element outside the table).  With iso=1 the
 * pipeline adds Piso to Q, Q_N and Q_U (calculate_tauRTA_iso,
 * sub.f90:8311-8549) and builds the collision matrix of
 * ald_collision_matrix_iso.  The iterative solution with isotopes
 * (update_iso) returns ALD_ERR_UNSUPPORTED: kappa_full frees Piso
 * (kappa.f90:1252) before update_iso reads it (sub.f90:2598), so the
 * reference has no defined result there. */
int ald_p_iso_split(ald_ctx* ctx, const int ksubset[2], double* Piso);
int ald_set_isotope_g(ald_ctx* ctx, const double* g);
int ald_get_isotope_g(ald_ctx* ctx, double* g);

/* cal_RHS_IBZ (sub.f90:2618): RHS(nibz*ndyn*3). */
int ald_rhs(ald_ctx* ctx, double tempk, double* RHS);

/* cg_quadratic (cg.f90:19): minimises 1/2 v.a.v - b.v from the initial
 * guess vmin (overwritten), a(n,n) column-major.  Returns ALD_OK or
 * ALD_WARN_CG_MAXITER; *iters receives the iteration count. */
int ald_cg_quadratic(int n, const double* a, const double* b, double* vmin, double* funcmin, int max_iter,
                     int n_dig_accur, int* iters);

/* No counterpart in the reference: cg_quadratic (cg.f90:19) for callers that
 * cannot allocate device memory -- codes whose device memory all comes from
 * their own pool or from another framework's allocator, where a cudaMalloc
 * inside the library breaks the pool's accounting and a cudaFree stalls the
 * whole device.  a(n,n) (column-major), b(n) and vmin(n) are DEVICE pointers
 * on the current device; vmin holds the initial guess and receives the
 * solution.  The work runs on `stream` (a cudaStream_t, NULL = the default
 * stream) and the call returns after it finished.  Nothing is allocated: the
 * CG work vectors live in a fixed __device__ array of the library, so
 * n <= ALD_CG_STATIC_MAX_N (ALD_ERR_ARG otherwise).  The first call on a
 * device looks that array's address up and keeps it for the life of the
 * process; make that first call before any stream capture, and do not reset
 * the device (cudaDeviceReset) between calls.  Every 8 iterations the call
 * reads the stop flag back to the host, synchronising `stream`.  Buffers
 * whose allocation is shorter than n*n (a) or n (b, vmin) doubles are
 * refused with ALD_ERR_ARG.
 * Calls share the array: calls that overlap on one device race.  Returns
 * ALD_OK or ALD_WARN_CG_MAXITER like ald_cg_quadratic. */
#define ALD_CG_STATIC_MAX_N 32768
int ald_cg_quadratic_static(int n, const double* a, const double* b, double* vmin, double* funcmin, int max_iter,
                            int n_dig_accur, int* iters, void* stream);

/* mode_kappa_d (sub.f90:1407): kappa(ndyn,3,3) from the CG solution
 * Fi_x(nibz*ndyn*3) with star-averaged velocities
 * (veloc_avergeIBZ_invsyFBZ sub.f90:5479). */
int ald_mode_kappa_d(ald_ctx* ctx, double tempk, const double* Fi_x, double* kappa);

/* update_mpi (sub.f90:2295-2449), one step of the iterative BTE of job=3:
 * F2mpi(nk1,ndyn,3) = F_RTA + A/Qvalue for IBZ rows ksubset, with A the sum
 * over IBZ q2, its star arms (kstarsinfbz1) and l2, l3 of
 *   P1 (S F(q1+q2,l3) - S F(q2,l2)) + P2/2 (S F(q2,l2) + S F(q1-q2,l3)),
 * S the op that maps the IBZ point onto the arm (syop_f, get_kvecopn2).
 * P1, P2(nk1,nkc,ndyn,ndyn,ndyn) Bose-weighted as ald_calculate_tau_rta
 * returns them; Qvalue(nibz,ndyn); F_RTA, FFF(nibz,ndyn,3). */
int ald_update_mpi(ald_ctx* ctx, const int ksubset[2], const double* P1, const double* P2, const double* Qvalue,
                   const double* F_RTA, const double* FFF, double* F2mpi);

/* The whole job=1 sequence (kappa.f90:389-871) on the device without
 * materialising any (nibz,nkc,ndyn^3) array: phonons (unless injected),
 * V3, delta, Q, RTA kappa, collision matrix, RHS, CG, kappa.  Only the
 * per-mode results come back. */
typedef struct ald_kappa_result {
  double kappa_rta[9];     /* sum over bands, (3,3) column-major, W/m/K  */
  double kappa_cg[9];
  int cg_iters;
  int status_cg;           /* ALD_OK or ALD_WARN_CG_MAXITER              */
  double cg_err;           /* last error measure of the stop rule        */
  /* device time per stage (CUDA events on the context's stream), ms:
     0 phonons+occupations, 1 V3, 2 delta+Bose+band sums, 3 Q reduce,
     4 RTA kappa, 5 collision matrix, 6 RHS, 7 CG, 8 CG kappa, 9 total   */
  double stage_ms[10];
  int launches[10];        /* kernel launches per stage (same indices)   */
  double triplet_bands;    /* nibz*nkc*ndyn^3                            */
  double d2h_bytes;        /* bytes copied back to the host by the call  */
} ald_kappa_result;

/* Run the context's work on a caller-provided cudaStream_t (e.g. one a
 * framework already uses) instead of the context's own stream.  The
 * stream must belong to the context's device; NULL restores the own one. */
int ald_set_stream(ald_ctx* ctx, void* stream);

/* Bytes uploaded to the device when the context was created. */
double ald_h2d_bytes(ald_ctx* ctx);

/* Q, QN, QU (nibz,ndyn), kappa_rta_modes / kappa_cg_modes (ndyn,3,3),
 * x (nibz*ndyn*3, the CG solution) may be NULL.  When one |V3|^2 chunk
 * (ald_options.chunk_bytes, or the autotuner's choice) holds every IBZ row,
 * the context keeps it after the call; a later call with the same eigenpairs
 * (another temperature, as kappa_full's tmin..tmax) reuses it and launches no
 * V3 kernel (res->launches[1] = 0).  New eigenpairs (ald_get_frequencies,
 * ald_set_phonons) or ald_release_workspaces drop it. */
int ald_kappa_pipeline(ald_ctx* ctx, double tempk, ald_kappa_result* res, double* Q, double* QN, double* QU,
                       double* kappa_rta_modes, double* kappa_cg_modes, double* x);

/* ald_kappa_batched: ald_kappa_pipeline on n structures at once (the batched
 * configurations of many cells of uneven size), no reference counterpart:
 * the reference runs one structure per kappa_full run.  A pool of up to 8
 * host threads takes the structures largest first (nibz nkc ndyn^3), each on
 * its context's own stream, so the structures' kernels overlap on the
 * device.  A structure starts only while the estimated pipeline workspaces
 * of the structures running on its device, plus its own, stay within 85 %
 * of the device memory free when the call began (one structure always
 * runs).  When not every structure runs at once, a structure's pipeline
 * workspaces are released after its run (to the library's device-memory
 * cache).  tempk[n], res[n]; status[n] (may be
 * NULL) receives each structure's return code.  Returns ALD_OK, or the first
 * structure's error (ald_last_error names the structure).  The contexts must
 * be distinct; each structure's limits are those of ald_kappa_pipeline (up
 * to 256 bands). */
int ald_kappa_batched(int n, ald_ctx* const* ctx, const double* tempk, ald_kappa_result* res, int* status);

/* No counterpart in the reference (one code path per routine there): the
 * pipeline's autotuner.  ald_autotune times whole ald_kappa_pipeline calls
 * (device time, at the tmin of latdyn.params) over candidate launch shapes,
 * one knob at a time: the |V3|^2 chunk (IBZ rows per V3 and delta launch),
 * for 3-band mixed cells the tensor-core V3's rows per CTA and epilogue
 * warpgroups, for mixed cells of 9 bands and up the pair-batch workspace of
 * the tensor-core mode-product GEMMs.  It keeps the fastest on the context
 * and in the cache file (cache_path; NULL or "": $ALD_TUNE_CACHE; neither:
 * no file), one text line per shape (device, bands, mesh, IBZ rows,
 * precision, delta, deterministic option).  When the file already holds the
 * context's shape, the choice is read from it and nothing is timed.
 * budget_s (<= 0: 10 s) bounds the timing; the knobs change launch shapes
 * only, not results.  ald_set_tuning applies a choice directly (0 fields =
 * the built-in choices). */
typedef struct ald_tuning {
  size_t chunk_bytes;   /* as ald_options.chunk_bytes (0 = automatic)                    */
  int v3_rows_per_cta;  /* 3-band tensor-core V3: IBZ rows per CTA, 1..16 (0 = built-in) */
  int v3_epilogue_wg;   /* 3-band tensor-core V3: epilogue warpgroups, 2 or 3 (0 = 2)    */
  size_t v3_gemm_bytes; /* tensor-core mode-product GEMMs: pair-batch workspace (0 = 2 GiB) */
  double ms;            /* device time of one pipeline call with this choice             */
  int from_cache;       /* 1: read from the cache file, 0: timed by this call            */
  int candidates;       /* pipeline choices timed                                        */
} ald_tuning;
int ald_autotune(ald_ctx* ctx, const char* cache_path, double budget_s, ald_tuning* out);
int ald_set_tuning(ald_ctx* ctx, const ald_tuning* t);

/* No counterpart in the reference: hands a context's pipeline workspaces
 * (R1/R2, the |V3|^2 chunk, the V3 and eigensolver workspaces, the collision
 * matrix) back to the library's device-memory cache; the next pipeline call
 * of any context of the same sizes takes them from there.  For hosts that
 * keep many contexts alive and run them one after another. */
int ald_release_workspaces(ald_ctx* ctx);

/* Row-sharded job=1, one call per rank (one process per GPU): the MPI
 * decomposition of kappa_full (kappa.f90:418-428: nibz/nranks IBZ rows per
 * rank, the last rank also takes the remainder; ald_shard_rows returns a
 * rank's 1-based range).  Each rank computes V3, the delta, Q, Q_N, Q_U and
 * the collision-matrix rows of its own IBZ rows.  Two exchanges replace
 * the reference's MPI_Allgatherv calls (kappa.f90:641-643, 790): Q, Q_N, Q_U
 * once, and in every CG iteration the local rows of the matrix-vector
 * product, so the 3 b nibz x 3 b nibz matrix is never gathered.  `gather`
 * is the caller's all-gather (NCCL, MPI, ...) over host buffers: it
 * receives this rank's `count` values in `mine` and must fill `all` with
 * every rank's values in rank order (counts[k] values of rank k), return 0
 * on success; it is called the same number of times, in the same order,
 * on every rank.  The CG vectors are replicated, so every rank returns the
 * same kappa and the full Q/x.  Outputs as ald_kappa_pipeline; iso=1 is
 * supported, job=3 is not. */
typedef int (*ald_allgather_fn)(void* user, const double* mine, long long count, double* all,
                                const long long* counts, int nranks);
int ald_shard_rows(const ald_ctx* ctx, int rank, int nranks, int ksubset[2]);
/* The same exchange on device buffers, for NCCL-style all-gathers that stay
 * in GPU memory: `mine` (count values) and `all` are device pointers of this
 * rank's GPU, and the gather must be ordered after the work already queued on
 * `stream` (the context's cudaStream_t) and before the work queued after it
 * returns -- e.g. enqueued on that stream; no host copy and no host
 * synchronisation of the exchange is needed.  The CG still reads its stop
 * flag on the host once per iteration, so every rank takes the same steps. */
typedef int (*ald_allgather_dev_fn)(void* user, const double* mine, long long count, double* all,
                                    const long long* counts, int nranks, void* stream);
int ald_kappa_pipeline_sharded(ald_ctx* ctx, double tempk, int rank, int nranks, ald_allgather_fn gather,
                               void* user, ald_kappa_result* res, double* Q, double* QN, double* QU,
                               double* kappa_rta_modes, double* kappa_cg_modes, double* x);
/* ald_kappa_pipeline_sharded with the device all-gather (replaces the same
 * MPI_Allgatherv calls, kappa.f90:641-643, 790). */
int ald_kappa_pipeline_sharded_dev(ald_ctx* ctx, double tempk, int rank, int nranks, ald_allgather_dev_fn gather,
                                   void* user, ald_kappa_result* res, double* Q, double* QN, double* QU,
                                   double* kappa_rta_modes, double* kappa_cg_modes, double* x);

/* The job=3 sequence (kappa.f90:1046-1487): as ald_kappa_pipeline up to the
 * RTA kappa, then from FFF = F_RTA repeat FFF += update_mix (update_mpi(FFF)
 * - FFF) and kappa = mode_kappa(FFF) until sqrt(sum((kappa_new -
 * kappa_old)^2)/(ndyn*9)) < 1e-4 or max_iter iterations (150 and 0.4 in
 * read_params, rest.f90:36-44).  In `res`, kappa_cg holds the iterative kappa,
 * cg_iters the iterations, cg_err the last change and status_cg ALD_OK or
 * ALD_WARN_CG_MAXITER; stage 7 times the iterations, stages 5, 6, 8 are 0.
 * Q(nibz,ndyn), the mode tensors (ndyn,3,3) and FFF(nibz,ndyn,3) may be NULL. */
int ald_kappa_iterative(ald_ctx* ctx, double tempk, int max_iter, double update_mix, ald_kappa_result* res,
                        double* Q, double* kappa_rta_modes, double* kappa_iter_modes, double* FFF);

/* Output files of a job=1 run, as the reference's gfortran build writes
 * them (list-directed records: I11 integers, REAL(8) with 17 significant
 * digits in 25 columns; formatted records: the Fortran Iw/Fw.d/Ew.d/Gw.d
 * rules).
 *
 * ald_tau_eff: tauinv_eff(nibz,ndyn) per mode, the sum mode_kappa
 * (solution = 0, sub.f90:1336-1366; F = FFF(nibz,ndyn,3) of
 * ald_rta_kappa, velocities at mapinv, velocc(j) == 0 -> /0.01) or
 * mode_kappa_d (solution = 1, sub.f90:1497; F = the CG solution
 * Fi_x(nibz*ndyn*3), star-averaged velocities) adds for that mode.
 *
 * ald_qandtau replaces Qandtau (sub.f90:8198-8305): tauinv_N, tauinv_U,
 * tauinv_tot(nibz,ndyn) in 1/s from Q, Q_N, Q_U(nibz,ndyn), and the file
 * Qvalue.dat ("nk,la,Q", then ibz, la, Q, Q/(n(n+1))) when qvalue_path is
 * not NULL.
 *
 * ald_write_kappa replaces write_kappa (sub.f90:1818-1916): kappa_path
 * gets the per-band tensor, tot_kap and the diagonal sums, tau_path one
 * line per IBZ mode (tempk, i, kibz, la, omega, n, 1/tauinv_N,
 * 1/tauinv_U, 1/tauinv_tot, tauinv_eff, veloc at mapinv).  Like the
 * reference it sets zero entries of tauinv_N and tauinv_U to 1e10 in
 * place.  Either path may be NULL.
 *
 * ald_write_job1_files writes, into directory dir, the five files of
 * kappa_full's job=1 block (kappa.f90:559-870) from the outputs of
 * ald_kappa_pipeline (Q, QN, QU, the two per-band tensors and x):
 * Qvalue.dat; tau_RTA.dat and kappa_RTA.dat; tau_RTAandeff-cg.dat and
 * kappa_direct-cg.dat.  tauinv_eff follows the reference's array: mode_kappa
 * clears the whole array before each mode, so the RTA file carries only the
 * last mode's value (nibz, ndyn) and zeros elsewhere; mode_kappa_d adds its
 * sums on top of that.
 *
 * ald_format_value formats one value as the writers do, host only: edit
 * "Iw", "Fw.d", "Ew.d", "Gw.d", "*" (a list-directed REAL(8) field, 25
 * characters, no separator) or "*I" (a list-directed INTEGER field, 11
 * characters).  Returns the length written into out (NUL-terminated), -1
 * for a bad edit or a short buffer. */
int ald_tau_eff(ald_ctx* ctx, double tempk, const double* F, int solution, double* tauinv_eff);
int ald_qandtau(ald_ctx* ctx, double tempk, const double* Q, const double* QN, const double* QU,
                const char* qvalue_path, double* tauinv_N, double* tauinv_U, double* tauinv_tot);
int ald_write_kappa(ald_ctx* ctx, double tempk, const double* kappa, double* tauinv_N, double* tauinv_U,
                    const double* tauinv_tot, const double* tauinv_eff, const char* kappa_path,
                    const char* tau_path);
int ald_write_job1_files(ald_ctx* ctx, const char* dir, double tempk, const double* Q, const double* QN,
                         const double* QU, const double* kappa_rta_modes, const double* kappa_cg_modes,
                         const double* x);
int ald_format_value(const char* edit, double value, char* out, int cap);

/* Three-phonon self-energy at arbitrary q: THERMACOND's job=2 block
 * (kappa.f90:874-1040).
 *
 * ald_make_kp_bs replaces make_kp_bs (modules.f90:1507-1652): the band path
 * of dir/kpbs.params (units 0 = conventional reciprocal coordinates, else
 * primitive; nkdir points per segment; ndir segments), kp_bs(3,nkp_bs)
 * Cartesian (2 pi included) and dk_bs(nkp_bs).  *nkp_bs = ndir*nkdir is
 * always set; kp_bs/dk_bs are filled when not NULL (cap >= nkp_bs).
 *
 * ald_function_self_w replaces function_self_w3 (gauss = 0; Lorentzian
 * of width etaz, four terms, real and imaginary parts; rest.f90:4012) and
 * function_self_w4 (gauss = 1; Gaussian, three terms, imaginary part only;
 * rest.f90:4126) for n jobs: point q(3,n), mode la(n) (1-based), frequency
 * omega(n) and temperature temp, both in cm^-1.  nself, uself (2,n) are
 * the normal and umklapp parts (complex: re, im), already /nkc*pi.  The
 * sum runs over the mesh q2 and the bands at q2 and q3 = -q - q2, whose
 * eigenpairs come from the same eigensolver as the mesh's.  Eigenpairs at q
 * and q3 are taken in |lambda| order (get_frequencies') for both the
 * eigenvalue and the eigenvector.
 *
 * ald_self_energy_bs runs the job=2 block at temperature tempk (K): the path
 * of dir/kpbs.params, omega0(ndyn,nkp_bs) = sqrt|lambda|*cnst at the path
 * points, nself/uself (2,ndyn,nkp_bs) of function_self_w3 (gauss = 0) or
 * function_self_w4 (gauss = 1) at omega = omega0, and, when out_dir is not
 * NULL, lw-selfenergy.dat and lw-selfenergy2.dat there (kappa.f90:1019-1031:
 * isempi = 2 Im(nself + uself), tsempi = 1e10/c_light/isempi). */
int ald_make_kp_bs(ald_ctx* ctx, const char* dir, int* nkp_bs, double* kp_bs, double* dk_bs, int cap);
int ald_function_self_w(ald_ctx* ctx, int n, const double* q, const int* la, const double* omega, double temp,
                        int gauss, double* nself, double* uself);
int ald_self_energy_bs(ald_ctx* ctx, const char* dir, double tempk, int gauss, int nkp_bs, double* omega0,
                       double* nself, double* uself, const char* out_dir);

#ifdef __cplusplus
}
#endif
#endif /* ALD_H */
