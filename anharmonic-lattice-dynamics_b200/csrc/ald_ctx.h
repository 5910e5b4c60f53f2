// The context object behind ald_ctx* and the helpers shared by the C ABI
// translation units (ald_capi.cpp, ald_pipeline.cpp).
#pragma once
#include <string>

#include "ald_internal.h"

using namespace ald;

struct ald_ctx {
  System S;
  Tables T;
  Fc3Blocks F3;
  V3Classes VC;
  Fc2Csr F2;
  ald_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;      // stream the work is issued on
  cudaStream_t own_stream = nullptr;  // the context's own stream
  double h2d_bytes = 0;
  Geometry geo;
  // device tables: views into one block (`tables`), uploaded with one copy
  DevBuf<char> tables;
  DevBuf<double> kpc32, rr, fc2_val, fc2_sqm, born, fc3w, roots, opk, opk_inv;
  DevBuf<int> fc2_uatom, fc2_uidx;
  DevBuf<int> fc2_off, fc2_atom, blk_off, trip_j, trip_k, phase_coef, mapinv, neg_src, neg_dst, arm_off, arm_q,
      arm_op, star_off, star_q, star_op, tet_corner, tet_inc, err;
  DevBuf<int> cls_grp_off, cls_pc, cls_trip_off, cls_trip, cls_trip_i0, cls_trip_k;
  DevBuf<int> arm_owner;              // per arm: its IBZ point (kappa over arms)
  DevBuf<int> mesh_m;                 // per mesh point: its three mesh integers (+ 1 pad)
  DevBuf<int> mapibz0, full_op;       // per mesh point: IBZ point and the op of its star arm (job=3)
  bool full_op_ok = false;
  DevBuf<char> w_h;                   // per-row phase-class sums of the pair kernel
  DevBuf<char> w_ptiles;              // phase tiles of the tensor-core V3 (mesh-only, built once)
  DevBuf<char> w_btiles;              // per-row B operands of the tensor-core V3
  DevBuf<char> w_v3work;              // T1/T2 of the large-cell V3 GEMMs
  DevBuf<char> w_h64, w_v3fix;        // mixed path, FP64 V3 near zero frequencies: H and T1/T2
  DevBuf<long long> w_pairs;          // its (row, q2) pair list
  int v3work_tc_b = 0;                // its tensor-core T2 padding is zero for (bands, pairs)
  long long v3work_tc_p = 0;
  bool ptiles_ok = false;
  // phonons and occupations
  DevBuf<double> w2_all, w2, evec, vel, freq, dist;
  // pipeline workspaces, kept across calls (allocation outside the timed work)
  DevBuf<double> w_R1, w_R2, w_Q, w_v3, w_F, w_x, w_rhs, w_kr, w_kc, w_cm;
  DevBuf<double> w_R1p, w_R2p, w_Ff, w_Frta, w_part;  // iterative solution: band marginals, F on the mesh
  // isotope scattering (iso=1): g per primitive atom, Piso [ibz][l1] and its partial sums
  std::vector<double> giso;
  bool giso_ok = false;
  DevBuf<double> giso_d, w_piso, w_piso_part;
  DevBuf<double> w_kpart;   // per-CTA partial sums of kappa
  DevBuf<double> w_brange;  // omega range of every band over the mesh
  DevBuf<char> w_scratch;
  DevBuf<double> w_heev;    // Householder eigensolver workspace (large cells)
  DevBuf<double> w_rmax;    // deterministic delta: each R entry's largest term (FP64 bits)
  // launch shapes chosen by ald_autotune (0 = the built-in choices)
  int tune_v3_rpc = 0, tune_v3_wg = 0;
  size_t tune_gemm_bytes = 0;
  CgWork cg;
  bool have_phonons = false;
  unsigned long long phonon_epoch = 0;  // advanced whenever the eigenpairs change
  // |V3|^2 of every row of [v3c_rb, v3c_re) in w_v3 from one chunk, valid for
  // the eigenpairs of v3c_epoch (0 = nothing kept): a later pipeline call
  // with the same eigenpairs and rows reuses it (|V3|^2 does not depend on T)
  unsigned long long v3c_epoch = 0;
  int v3c_rb = -1, v3c_re = -1, v3c_layout = -1;
  bool v3c_f32 = false;
  const void* v3c_ptr = nullptr;
  size_t v3c_n = 0;
  double dist_tempk = -1;
};

namespace ald {
namespace capi {
int fail(int code, const std::string& msg);
int check_err_flags(ald_ctx* c);
int ensure_phonons(ald_ctx* c);
int ensure_dist(ald_ctx* c, double tempk);
V3Args v3_args(ald_ctx* c, int first, int nrows, double* out);
// nlaunch (optional) += the kernels launched
int run_v3(ald_ctx* c, const V3Args& a, int* nlaunch);
// g of cal_giso on the device (the element table unless ald_set_isotope_g set it)
int ensure_giso(ald_ctx* c);
KappaArgs kappa_args(ald_ctx* c, double tempk);
int delta_mode(ald_ctx* c);
double gauss_width(ald_ctx* c);
int rows_per_chunk(ald_ctx* c);
}  // namespace capi
}  // namespace ald

#define ALD_CK(call)                                                                            \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      return ald::capi::fail(ALD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(_e));   \
  } while (0)
#define ALD_CKA(call)                                                                           \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e == cudaErrorMemoryAllocation)                                                        \
      return ald::capi::fail(ALD_ERR_NOMEM, "device allocation failed: " #call);               \
    if (_e != cudaSuccess)                                                                      \
      return ald::capi::fail(ALD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(_e));   \
  } while (0)
