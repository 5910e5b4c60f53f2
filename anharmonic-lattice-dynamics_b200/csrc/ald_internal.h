// Internal types of libald.  Host-side tables are built once per context
// from the reference's input files; device buffers live in DevBuf.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ald.h"

#ifdef __CUDACC__
#define ALD_HD __host__ __device__
#else
#define ALD_HD
#endif

namespace ald {

// ------------------------------------------------------------ constants
// THERMACOND/modules.f90:4-23 and kappa.f90:182.  `cnst` is a REAL(8)
// initialised from a default-REAL literal, hence the float rounding.
struct PhysConst {
  static constexpr double pi = 3.14159265358979323846;
  static constexpr double h_plank = 6.62606896e-34;
  static constexpr double k_b = 1.3806504e-23;
  static constexpr double c_light = 2.99792458e+8;
  static constexpr double hbar = 1.054571628e-34;
  static constexpr double ee = 1.60217653e-19;
  static constexpr double uma = 1.66053878e-27;
  static ALD_HD double cnst() { return (double)521.1098918f; }
  static double const33();
};

// Everything the input files define (record layout: rest.f90:2-443).
struct System {
  // latdyn.params
  int nc[3] = {0, 0, 0};
  double shft[3] = {0, 0, 0};
  double width = 0, etaz = 0, tmin = 0, tmax = 0;
  int job = 0, iso = 0, classical = 0;
  // structure.params
  double latp[6] = {0};
  double primlatt[9] = {0};  // column-major (3,3)
  double scale = 0;
  int include_fc[4] = {0};
  std::vector<double> mas;
  std::vector<std::string> atname;  // element name per type
  int nat0 = 0;
  std::vector<int> atype;
  std::vector<double> mass0;
  // lat_fc.dat
  double r[3][3] = {{0}};  // r[a] = primitive vector a (Cartesian, A)
  double g[3][3] = {{0}};  // reciprocal vectors incl. 2*pi
  double volume_r = 0, volume_g = 0;
  int nterms[4] = {0};
  int natoms = 0;
  std::vector<double> atompos;  // 3*natoms
  std::vector<int> cell0;       // natoms, 1-based primitive atom
  std::vector<int> cell;        // 3*natoms, lattice-vector integers
  // fc2 / fc3 (1-based atom and xyz indices as in the files)
  std::vector<int> t2;          // 4*nt2: i, a, j, b
  std::vector<double> f2;
  std::vector<int> t3;          // 6*nt3: i, a, j, b, k, c
  std::vector<double> f3;
  // dielectric.params
  int born_flag = 0;
  double epsil[9] = {0};        // column-major (3,3)
  std::vector<double> charge;   // 9*nat0 column-major charge(i,j) per atom
  // b200.params (optional)
  int delta = -1, precision = -1, cg_stop = -1;
  double cg_tol = -1, width_cm = -1;
};

std::string read_system(const std::string& dir, System& S);

// Mesh / IBZ / symmetry tables (host).
struct Tables {
  int nkc = 0, nibz = 0, b = 0, npg = 0;
  bool shifted = false;            // all mesh divisions even: q = (m/N - 1/2) g
  double opk[48][9];               // op_kmatrix, column-major
  double gconv[3][3];              // reciprocal vectors of the conventional cell, 2 pi included
  std::vector<double> kpc32;       // 3*nkc: mesh of make_kp_reg (FP32 fractions)
  std::vector<int> mapibz;         // nkc, 1-based
  std::vector<int> mapinv;         // nibz, 1-based
  std::vector<double> kibz, wibz;  // 3*nibz, nibz
  std::vector<int> neg_src, neg_dst;  // subst_eivecs copies (0-based)
  // star arms that are mesh points (kstarsinfbz1): CSR over IBZ points
  std::vector<int> arm_off, arm_q, arm_op;   // arm_op 0-based op index
  // all star arms folded onto the mesh (getstar + get_k_info), for the
  // star-averaged velocities of mode_kappa_d
  std::vector<int> star_off, star_q, star_op;
  // tetrahedra: corner mesh indices (6*nkc x 4) and per-point incidences
  std::vector<int> tet_corner;     // 4 per tetrahedron, 0-based
  std::vector<int> tet_inc;        // 24 per point: tet*4 + slot, ascending
  // exact phases: q(m).R_j = 2*pi*t/L with t = sum_a m_a*pc[j][a] + ps[j] (mod L)
  int L = 1;
  std::vector<int> phase_coef;     // 4*natoms: L/N_a*n_a (a=0..2), shift term
};

std::string build_tables(const System& S, Tables& T);

// FC3 regrouped by atom triple (i0, j, k): 27 mass-scaled components per
// triple, triples grouped by the primitive-atom block (i0, j0, k0).
struct Fc3Blocks {
  int ntrip = 0;
  std::vector<int> blk_off;        // nat0^3 + 1
  std::vector<int> trip_j, trip_k; // supercell atom indices (0-based)
  std::vector<double> w;           // 27 per triple: fcs/sqrt(mi*mj*mk), comp = a*9+b*3+c
};
std::string build_fc3(const System& S, Fc3Blocks& F);

// The FC3 triples regrouped for the pair kernel.  With q3 = -q1-q2 on the
// mesh, the phase of triple (i0, j, k) is exp(i q2.(R_j - R_k)) exp(-i q1.R_k),
// so triples that share (j0, k0, R_j - R_k) -- a "class" -- share their
// q2-dependent phase.  Classes are grouped by g = j0*nat0 + k0.
struct V3Classes {
  int ncls = 0;
  std::vector<int> grp_off;   // nat0^2 + 1
  std::vector<int> pc;        // 4 per class: phase coefficients of R_j - R_k (mod L)
  std::vector<int> trip_off;  // ncls + 1: member triples of each class
  std::vector<int> trip;      // member triple (index into Fc3Blocks)
  std::vector<int> trip_i0;   // its primitive atom i0
  std::vector<int> trip_k;    // its supercell atom k (row phase exp(-i q1.R_k))
};
std::string build_v3_classes(const System& S, const Tables& T, const Fc3Blocks& F, V3Classes& C);

// FC2 grouped per dynamical-matrix element (i3, j3) in the file's term
// order (the order set_dynamical_matrix sums them).
struct Fc2Csr {
  std::vector<int> off;            // b*b + 1, element = i3*b + j3 (0-based)
  std::vector<int> atom;           // supercell atom j (0-based)
  std::vector<double> val;         // fcs_2
  std::vector<double> sqm;         // sqrt(mi*mj)
  std::vector<int> uatom;          // the distinct atoms of `atom`, ascending (one phase each per q)
  std::vector<int> uidx;           // per term: index of its atom in uatom
};
std::string build_fc2(const System& S, Fc2Csr& F);

// ------------------------------------------------------------ device side
// Device memory of the library.  Blocks that are freed (of any size) are
// kept per device (after a device synchronisation, so no queued work still
// uses them) and handed out again to an allocation of the same byte size:
// contexts created one after another reuse their workspaces without
// cudaMalloc/cudaFree.  The cache holds at most 32 GiB per device; when
// cudaMalloc runs out of memory the device's cached blocks are released and
// the allocation retried.  dev_trim releases every cached block.
cudaError_t dev_alloc(void** p, size_t bytes);
void dev_free(void* p, size_t bytes);
void dev_trim();
// Held while a stream of the library is being captured into a CUDA graph and
// while dev_free synchronises the device, so that contexts driven from
// different host threads never synchronise the device during a capture.
std::mutex& capture_mutex();

// Raise a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`, never lowering it.  The limit is one process-wide attribute
// per kernel, and contexts on different host threads (ald_kappa_batched)
// launch the same kernels with different sizes: a plain set by one thread
// could shrink the limit under another thread's launch.
cudaError_t raise_smem_limit(const void* func, size_t bytes);

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool view = false;  // p points into a block another DevBuf owns
  cudaError_t alloc(size_t count) {
    if (count == n && p && !view) return cudaSuccess;
    free();
    n = count;
    if (count == 0) return cudaSuccess;
    return dev_alloc((void**)&p, count * sizeof(T));
  }
  // count elements at q, owned elsewhere (never freed through this DevBuf)
  void view_of(T* q, size_t count) {
    free();
    p = q;
    n = count;
    view = true;
  }
  void free() {
    if (p && !view) dev_free(p, n * sizeof(T));
    p = nullptr;
    n = 0;
    view = false;
  }
  ~DevBuf() { free(); }
};

struct Geometry {  // passed by value to kernels
  int nc[3];
  int nkc;
  int b;
  int nat0;
  int shifted;
  int L;
  int L32;  // 1: every phase sum m.pc + pc3 (m < nc, pc < L) fits in 32 bits
};

// kernels (implemented in the .cu files)
struct PhononArgs {
  Geometry geo;
  const double* kpc32;       // 3*nkc
  const double* g;           // 9: g1,g2,g3 rows
  const int* fc2_off;        // b*b+1
  const int* fc2_atom;
  const double* fc2_val;
  const double* fc2_sqm;
  const int* fc2_uatom;      // nuniq distinct atoms of fc2_atom
  const int* fc2_uidx;       // per term: index into fc2_uatom
  int nuniq;
  const double* rr;          // 3*natoms: atompos(j) - atompos(j0)
  int born_flag;
  const double* born;        // epsil(9), charge(9*nat0), masses(nat0), scalars(4): eps_scale, rho2, om0, pad
  double dq;
  int ndisp = 7;             // matrices per point: 7 (the point and its six +-dq, velocities) or 1
  double* w2_all;            // nkc*ndisp*b |lambda| in get_freq order
  double* w2;                // nkc*b eigenval after get_frequencies' sort
  double* evec;              // 2*b*b*nkc (complex) for the central point
  int* err;
  double* he_work = nullptr; // Householder solver: heev_work_doubles(b, he_slots) doubles
  int he_slots = 0;
};
cudaError_t launch_phonons(const PhononArgs& a, cudaStream_t s);
// Householder + implicit QL eigensolver (ald_heev.cu), for cells whose
// matrices do not fit the shared-memory Jacobi (more than 64 bands, up to 256)
constexpr int kHeevMaxBands = 256;
int heev_slots(int nmat);
size_t heev_work_doubles(int b, int slots);
cudaError_t launch_heev(const PhononArgs& a, cudaStream_t s);
cudaError_t launch_phonon_post(const Geometry& geo, const double* w2_all, double dq, double cnst, double* vel,
                               cudaStream_t s);
cudaError_t launch_subst_eivecs(const Geometry& geo, const int* src, const int* dst, int n, double* evec,
                                cudaStream_t s);
cudaError_t launch_freq_dist(const Geometry& geo, const double* w2, double cnst, double temp, int classical,
                             double* freq, double* dist, int* err, cudaStream_t s);

// Three-phonon self-energy at arbitrary q (function_self_w3/w4), ald_self.cu
struct SelfArgs {
  int b, nkc, nat0, np;      // bands, mesh points, primitive atoms, path points of the chunk
  const double* qp;          // 3*np path points (Cartesian, 2 pi included)
  const double* omega;       // np*b target frequencies (cm^-1), [p*b + la]
  const double* evq;         // complex [p][la][comp] eigenvectors at the path points
  const double* wq;          // np*b |lambda| at the path points
  const double* kpc;         // 3*nkc mesh points
  const double* ev2;         // complex [k][l][comp] mesh eigenvectors
  const double* w2;          // nkc*b mesh eigenvalues
  const double* ev3;         // complex [p*nkc + k][l][comp] at k3 = -q - k2
  const double* w3;          // [(p*nkc + k)*b + l] |lambda| at k3
  int ntrip, natoms;
  const int* blk_off;
  const int* trip_j;
  const int* trip_k;
  const double* fc3w;
  const double* rr;          // 3*natoms: atompos(j) - atompos(j0)
  double gd[9];              // dual basis of g1..g3 without 2 pi (make_reciprocal_lattice), rows
  double ghalf[3];           // (g1+g2+g3)/2
  double temp, eta, etacut, cnst, const33, pi, v3thr;
  int classical, gauss;      // gauss: function_self_w4, else function_self_w3
  double* part;              // self_partial_doubles(*this)
  int* err;
};
size_t self_smem_bytes(const SelfArgs& a, int* ppb);
size_t self_partial_doubles(const SelfArgs& a);
cudaError_t launch_k3_points(int np, int nkc, const double* qp, const double* kpc, double* k3, cudaStream_t s);
// out: np*b*4 = nself re, im, uself re, im per (p, la), already /nkc*pi
cudaError_t launch_self(const SelfArgs& a, double* out, cudaStream_t s);

struct V3Args {
  Geometry geo;
  int n1_first;              // first IBZ row of the chunk (0-based)
  int nrows;                 // rows in the chunk
  const int* mapinv;         // 0-based mesh index of IBZ rows
  const double* evec;        // complex (b,b,nkc)
  const double* w2;          // (b,nkc)
  int ntrip;                 // FC3 atom triples
  int natoms;                // supercell atoms (phase table rows)
  const int* blk_off;
  const int* trip_j;
  const int* trip_k;
  const double* fc3w;        // 27*ntrip
  const int* phase_coef;     // 4*natoms
  const double* roots;       // 2*L
  double const33;
  double* v3sq;              // v3_layout 0: [row][q2][l1][l2][l3] (the reference's order, per row)
  int v3_layout;             //           1: [row][l2][l3][l1][q2] (slices of the delta, q2 fastest)
                             //           2: [row][l2][l3][q2][l1] (large cells, tensor-core V3)
  float* v3sq_f32 = nullptr; // the tensor-core V3 writes FP32 here instead of v3sq when set
  int* err;
  // phase classes (pair kernel)
  int ncls;
  const int* cls_grp_off;
  const int* cls_pc;
  const int* cls_trip_off;
  const int* cls_trip;
  const int* cls_trip_i0;
  const int* cls_trip_k;
  void* hbuf;                // row workspace: nrows*ncls*9*b complex (v3_hbuf_bytes)
  // the FP64 GEMMs of ald_v3_dense.cu on a list of pairs (row * nkc + q2, row
  // local to the chunk) instead of every pair of the chunk
  const long long* pair_list = nullptr;
  long long npairs_list = 0;
};
cudaError_t launch_v3_fp64(const V3Args& a, cudaStream_t s);
// pair kernel: bands it handles and the row workspace it needs (0 = not handled)
bool v3_pair_supported(int b, int precision);
size_t v3_hbuf_bytes(int b, int ncls, int nrows, int precision);
cudaError_t launch_v3_pair(const V3Args& a, int precision, cudaStream_t s);
// row stage alone, H in FP32 (for the tensor-core class sums) or FP64
cudaError_t launch_v3_rows_f32(const V3Args& a, cudaStream_t s);
cudaError_t launch_v3_rows_f64(const V3Args& a, cudaStream_t s);
// more than 12 bands (ald_v3_dense.cu): the class sums and both mode products
// as batched complex GEMMs per (q1, q2) pair; hbuf from launch_v3_rows_f64;
// work: v3_dense_work_bytes(b, pairs of the chunk, budget) bytes
bool v3_dense_supported(int b);
size_t v3_dense_work_bytes(int b, long long npairs, size_t budget);
// l1_keep (0 = all): only bands l1 < l1_keep are formed and written
cudaError_t launch_v3_dense(const V3Args& a, void* work, size_t work_bytes, cudaStream_t s, int l1_keep = 0);
// one row's |V3|^2 in the reference's order [q2][l1][l2][l3] (FP64) into row
// `row` of the chunk of a, in a's layout and precision, bands l1 < l1_keep
cudaError_t launch_v3_copy_row(const V3Args& a, int row, const double* src, int l1_keep, cudaStream_t s);
// more than 6 bands, ALD_MIXED (ald_v3_dense_tc.cu): both mode products as
// split-FP16 tcgen05 GEMMs; hbuf from launch_v3_rows_f32; work of
// v3_dense_tc_work_bytes(b, nkc, nrows, pairs) bytes for batches of `pairs`
// pairs; a2_zeroed: the workspace's T2 operand padding is already zero
bool v3_dense_tc_supported(int b);
long long v3_dense_tc_pairs(int b, long long npairs, size_t budget);
size_t v3_dense_tc_work_bytes(int b, int nkc, int nrows, long long pairs);
int v3_dense_tc_launches(long long npairs, long long pairs);
cudaError_t launch_v3_dense_tc(const V3Args& a, void* work, long long pairs, bool a2_zeroed, cudaStream_t s);
// the |V3|^2 layout the pipeline asks V3 for and hands to the delta:
// 0 [row][q2][l1][l2][l3], 1 [row][l2][l3][l1][q2], 2 [row][l2][l3][q2][l1]
int v3_pipeline_layout(int b, int precision);
// 3 bands, ALD_MIXED: class sums on tcgen05 (ald_v3_tc.cu); hbuf from launch_v3_rows_f32
bool v3_tc_supported(int b, int ncls);
// the row-independent phase tiles (split FP16, canonical layout), built once per context
size_t v3_tc_ptile_bytes(int nkc, int ncls);
cudaError_t launch_v3_tc_ptiles(const V3Args& a, void* ptiles, cudaStream_t s);
// btiles: scratch of v3_tc_btile_bytes(nrows, ncls, nkc) (B operands and row data of the
// chunk's rows, per-mode factors and FP32 eigenvectors of the mesh)
size_t v3_tc_btile_bytes(int nrows, int ncls, int nkc);
// rows_per_cta, epilogue_wg: 0 = the built-in choice (up to 16 rows while the
// grid fills the GPU twice; 2 warpgroups), else 1..16 rows and 2 or 3
cudaError_t launch_v3_tc(const V3Args& a, const void* ptiles, void* btiles, cudaStream_t s, int rows_per_cta = 0,
                         int epilogue_wg = 0);

struct CombineArgs {
  Geometry geo;
  int n1_first, nrows;
  const int* mapinv;
  const double* v3sq;        // v3_layout 0: [row][q2][l1][l2][l3]; 1: [row][l2][l3][l1][q2]
  int v3_layout;
  const float* v3sq_f32 = nullptr;  // FP32 |V3|^2 in place of v3sq (band-generic kernels only)
  const double* freq;        // [q][l]
  const double* dist;        // [q][l]
  const int* tet_corner;
  const int* tet_inc;
  int gauss;
  double sigma;
  int f32w;                  // 1: delta weights in FP32 (mixed-precision pipeline), 0: FP64 as the reference
  const double* brange;      // optional [2b]: min / max of omega per band over the mesh (slice skipping)
  double* R1;                // [row][q][l1][l2], row local to the chunk
  double* R2;
  double* R1p;               // optional [row][q][l1][l3] = sum_l2 P1 (update_mpi); nullptr = skip
  double* R2p;
  // the two passes of the deterministic fused delta: per R1/R2/R1p/R2p entry
  // the largest single term (its FP64 bits; every term is >= 0), then the
  // terms as 62-bit fixed point scaled by that bound (delta_fused mode 1, 2)
  unsigned long long* M1 = nullptr;
  unsigned long long* M2 = nullptr;
  unsigned long long* M1p = nullptr;
  unsigned long long* M2p = nullptr;
  double* P1s;               // optional [row][q][l1][l2][l3] (P1smpi)
  double* P2s;
  double* P1;                // optional Bose-weighted
  double* P2;
};
// scratch: the corner energies of the chunk (combine_scratch_bytes)
size_t combine_scratch_bytes(const Geometry& geo, int nrows, int gauss);
cudaError_t launch_combine(const CombineArgs& a, void* scratch, cudaStream_t s);
// tetrahedron delta fused into R1/R2 (pipeline; P1s/P2s/P1/P2 not produced);
// R1/R2 of the chunk must be zero on entry
// mode 0: the terms added with FP64 atomics (arrival order);
// mode 1 and 2 + launch_delta_finalize: the same sums with the same bits on
// every run -- mode 1 records each entry's largest term in M1/M2 (M1p/M2p),
// mode 2 adds every term as an integer, round(term * 2^(62 - e)), with
// 2^e >= kDetTerms(b) x that largest term, and finalize converts the integer
// sums back: R = sum * 2^(e - 62).  R must be zero and M zero on entry.
bool delta_fused_supported(const Geometry& g);
cudaError_t launch_delta_fused(const CombineArgs& a, cudaStream_t s, int mode = 0);
cudaError_t launch_delta_finalize(double* R, const unsigned long long* M, size_t n, int b, cudaStream_t s);
// any number of bands (large cells): the tetrahedron or Gaussian delta into
// R1/R2 and/or P1s/P2s straight from |V3|^2 of the chunk; for the tetrahedron
// R1/R2/P1s/P2s (and R1p/R2p) must be zero on entry; P1/P2 are not produced
constexpr int kDeltaSmallBands = 16;  // up to here the band-templated kernels
cudaError_t launch_delta_any(const CombineArgs& a, cudaStream_t s);
// Q/QN/QU[(n1_first+row)*b + l1] from R1/R2 of rows [0, nrows)
cudaError_t launch_q_from_r(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* R1,
                            const double* R2, double* Q, double* QN, double* QU, int nibz, cudaStream_t s);

struct KappaArgs {
  Geometry geo;
  int nibz;
  const int* mapinv;
  const double* freq;
  const double* dist;
  const double* vel;         // (3,b,nkc)
  const double* w2;
  const int* arm_off;
  const int* arm_q;
  const int* arm_op;
  const int* star_off;
  const int* star_q;
  const int* star_op;
  const double* opk;         // 48*9
  const double* opk_inv;     // 48*9
  double tempk, temp, const1;
  double const2;             // k_b T^2/(h c 100)/c (mode_kappa's tauinv_eff)
  int classical;
  const int* arm_owner;      // per arm (arm_q entry): its IBZ point
  int narm;                  // arm_off[nibz]
  double* part;              // scratch: kappa_partial_doubles(b, narm) (per-CTA partial sums)
  int zero_q_f = 0;          // 1: F_RTA = 0 where Q = 0 (mixed path); 0: the reference's division
};
size_t kappa_partial_doubles(int b, int narm);
cudaError_t launch_rta_F(const KappaArgs& a, const double* Q, double* FFF, cudaStream_t s);
cudaError_t launch_kappa(const KappaArgs& a, const double* F, int averaged, double* kappa_modes, int* err,
                         cudaStream_t s);
cudaError_t launch_rhs(const KappaArgs& a, double* rhs, cudaStream_t s);
// tauinv_eff(nibz, b) [i*b + l] of mode_kappa (averaged = 0, F = F_RTA) or
// mode_kappa_d (averaged = 1, F = the CG solution), both [(i*b + l)*3 + x]
cudaError_t launch_tau_eff(const KappaArgs& a, const double* F, int averaged, double* tauinv_eff,
                           cudaStream_t s);
// CM: double, or float when cm_f32 (mixed-precision pipeline); leading dimension ld.
// piso (optional, [row][l1] of the range): CollisionMatrix_iso's form instead
// of CollisionMatrix_mpi's (Q must then include Piso); mesh_m: 4 mesh integers per point
cudaError_t launch_collision(const Geometry& geo, int nibz, int n1_first, int nrows, const int* mapinv,
                             const int* arm_off, const int* arm_q, const int* arm_op, const double* opk,
                             const double* Q, const double* R1, const double* R2, void* CM, size_t ld, int cm_f32,
                             const double* piso, const int* mesh_m, cudaStream_t s);
// isotope scattering (P_iso_split): Piso[row][l1] of rows n1_first.., and
// Q, Q_N, Q_U += Piso when Q is given; partial: piso_partial_doubles scratch
size_t piso_partial_doubles(const Geometry& geo, int nrows);
cudaError_t launch_piso(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* freq,
                        const double* evec, const int* tet_corner, const double* giso, double* partial,
                        double* Piso, double* Q, double* QN, double* QU, cudaStream_t s);
cudaError_t launch_add(size_t n, double* y, const double* x, cudaStream_t s);
// brange[l] = min_q omega(q,l), brange[b+l] = max_q omega(q,l)
cudaError_t launch_band_range(const Geometry& geo, const double* freq, double* brange, cudaStream_t s);
// weight_tet on a list of tetrahedra (device arrays w, c of 4 doubles each), fp32: the mixed form
cudaError_t launch_weight_tet(int ntet, const double* w, double e, int fp32, double* c, cudaStream_t s);
// the g of cal_g for an element name (false: no isotope data for it), and
// of every primitive atom (cal_giso)
bool isotope_g(const std::string& element, double& g);
std::string isotope_g_atoms(const System& S, std::vector<double>& g);

// layout conversions and the stand-alone stage kernels (ald_util.cu)
// internal 5-index arrays are [row][q][l1][l2][l3]; the reference's are
// Fortran (row,q,l1,l2,l3) with the row index fastest
cudaError_t launch_to_fortran5(const double* src, double* dst, int nr, int nkc, int b, cudaStream_t s);
cudaError_t launch_from_fortran5(const double* src, double* dst, int nr, int nkc, int b, cudaStream_t s);
cudaError_t launch_transpose(const double* src, double* dst, int rows, int cols, cudaStream_t s);
// calculate_tauRTA_mpi2 from given P1smpi/P2smpi (internal layout)
cudaError_t launch_tau(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* P1s,
                       const double* P2s, const double* dist, double* Q, double* QN, double* QU, double* P1,
                       double* P2, cudaStream_t s);
// R1/R2 = sum_l3 P1/P2 and Qd = sum (P1 + P2/2) from Bose-weighted P (internal layout)
cudaError_t launch_collapse(const Geometry& geo, int nrows, const double* P1, const double* P2, double* R1,
                            double* R2, double* Qd, cudaStream_t s);
// Rp = sum_l2 P (internal layout), the band marginal update_mpi needs besides R
cudaError_t launch_marginal_l2(const Geometry& geo, int nrows, const double* P1, const double* P2, double* R1p,
                               double* R2p, cudaStream_t s);
// update_mpi (sub.f90:2295-2449) on band marginals:
//   Ff[q][l][:] = S_op(q) F[ibz(q)][l][:] over the whole mesh (F [n][l][xyz]);
//   F2[n1][l1] = F_RTA[n1][l1] + A/Q[n1][l1],
//   A = sum_q sum_l R1p[q][l1][l] Ff[q1+q][l] - R1[q][l1][l] Ff[q][l]
//             + (R2[q][l1][l] Ff[q][l] + R2p[q][l1][l] Ff[q1-q][l]) / 2;
// with mix > 0 the output is Fout = F + mix (F2 - F) (in place allowed).
// R arrays are local to rows [n1_first, n1_first + nrows); Q, F_RTA, F over
// all IBZ points; Fout local to the rows.
cudaError_t launch_ffull(const Geometry& geo, const int* mapibz, const int* full_op, const double* opk,
                         const double* F, double* Ff, cudaStream_t s);
// part: scratch of update_part_doubles(geo, nrows) doubles
size_t update_part_doubles(const Geometry& geo, int nrows);
cudaError_t launch_update(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* R1,
                          const double* R1p, const double* R2, const double* R2p, const double* Ff, const double* Q,
                          const double* F_RTA, const double* F, double mix, double* Fout, double* part,
                          cudaStream_t s);
// CG workspace: vectors, scalars and the captured CUDA graph of the
// iteration loop, kept across calls and re-captured only when the problem
// (size, pointers, stop rule) changes
struct CgWork {
  DevBuf<double> grad, conj, aux, v0, partial, pnum, p4, fmin;
  DevBuf<double> yloc;  // the local rows of A v (row-sharded CG)
  DevBuf<char> st;
  cudaGraphExec_t exec = nullptr;       // kCgChunk iterations
  cudaGraphExec_t exec_tail = nullptr;  // max_iter % kCgChunk iterations
  int* h_done = nullptr;                // pinned copy of the stop flag
  int n = -1, max_iter = -1, mode = -1;
  double tol = 0;
  const void* A = nullptr;
  size_t ld = 0;
  const double* b = nullptr;
  double* x = nullptr;
  ~CgWork() {
    if (exec) cudaGraphExecDestroy(exec);
    if (exec_tail) cudaGraphExecDestroy(exec_tail);
    if (h_done) cudaFreeHost(h_done);
  }
};
int cg_device(int n, const double* dA /*row-major*/, const double* db, double* dx, int max_iter, int mode,
              double tol, int* iters, double* err_out, double* funcmin, cudaStream_t s, CgWork& w, std::string& msg);
// The exchange of the row-sharded CG: gather this rank's `count` values
// (device) into the full vector `all` (device, rank order); 0 on success.
using CgAllGather = std::function<int(const double* mine, size_t count, double* all)>;
int cg_device_rows(int n, int row0, int nrows, size_t ld, const void* dA, int a_f32, const double* db, double* dx,
                   int max_iter, int mode, double tol, const CgAllGather& gather, int* iters, double* err_out,
                   double* funcmin, cudaStream_t s, CgWork& w, std::string& msg);
// CG iterations whose kernels were launched for a solve that stopped after
// iters (the captured chunks run to their end, as no-ops after the stop)
int cg_launched_iterations(int iters, int max_iter);
// the same on a row-major A of double (a_f32 = 0) or float (a_f32 = 1) with
// leading dimension ld (16-byte aligned rows are read as vectors)
int cg_device_ld(int n, size_t ld, const void* dA, int a_f32, const double* db, double* dx, int max_iter, int mode,
                 double tol, int* iters, double* err_out, double* funcmin, cudaStream_t s, CgWork& w,
                 std::string& msg);

}  // namespace ald
