// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle_core.h).
// Flat C entry points over the restated reference routines, for ctypes.
// Arrays use the reference's Fortran layout; complex arrays are
// interleaved (re, im) doubles.
#include <atomic>
#include <cstring>
#include <stdexcept>
#include <string>

#include "oracle_core.h"

using namespace orc;

namespace orc {
extern std::atomic<long> g_weight_tet_nonperm;
}

extern "C" {

void* orc_load(const char* dir, char* err, int errlen) {
  State* S = new State();
  std::string e = read_inputs(*S, dir);
  if (!e.empty()) {
    std::snprintf(err, errlen, "%s", e.c_str());
    delete S;
    return nullptr;
  }
  return S;
}

void orc_free(void* p) { delete (State*)p; }

// sizes: ndyn nkc nibz nterms2 nterms3 natoms lattpgcount nc1 nc2 nc3 natoms0 npos
int orc_sizes(void* p, int* out) {
  State& S = *(State*)p;
  int v[12] = {S.ndyn, S.nkc, S.nibz, S.nterms[1], S.nterms[2], S.natoms, S.lattpgcount,
               S.nc[0], S.nc[1], S.nc[2], S.natoms0, S.npos};
  std::memcpy(out, v, sizeof v);
  return 0;
}

// lattice: r1 r2 r3 g1 g2 g3 volume_r volume_g const33 cnst (20 doubles)
int orc_lattice(void* p, double* out) {
  State& S = *(State*)p;
  for (int c = 0; c < 3; ++c) {
    out[c] = S.r1[c];
    out[3 + c] = S.r2[c];
    out[6 + c] = S.r3[c];
    out[9 + c] = S.g1[c];
    out[12 + c] = S.g2[c];
    out[15 + c] = S.g3[c];
  }
  out[18] = S.volume_r;
  out[19] = S.volume_g;
  out[20] = S.K.const33;
  out[21] = S.K.cnst;
  return 0;
}

// fc3 terms and the atoms they refer to, as read by read_fc234 / read_lattice
// (rest.f90:164-401): iat (3,nt3), ixyz (3,nt3), fcs (nt3), atompos
// (3,natoms), iatomcell0 (natoms), mass0 (natoms0); 1-based indices
int orc_fc3_terms(void* p, int* iat, int* ixyz, double* fcs, double* atompos, int* cell0, double* mass0) {
  State& S = *(State*)p;
  const int nt = S.nterms[2];
  std::memcpy(iat, S.iatomterm_3.data(), sizeof(int) * 3 * nt);
  std::memcpy(ixyz, S.ixyzterm_3.data(), sizeof(int) * 3 * nt);
  std::memcpy(fcs, S.fcs_3.data(), sizeof(double) * nt);
  std::memcpy(atompos, S.atompos.data(), sizeof(double) * 3 * S.natoms);
  std::memcpy(cell0, S.iatomcell0.data(), sizeof(int) * S.natoms);
  std::memcpy(mass0, S.mass0.data(), sizeof(double) * S.natoms0);
  return nt;
}

int orc_op_kmatrix(void* p, double* out) {
  State& S = *(State*)p;
  for (int i = 0; i < S.lattpgcount; ++i) std::memcpy(out + 9 * i, S.op_kmatrix[i], 9 * sizeof(double));
  return S.lattpgcount;
}

// make_kp_reg + get_negatives + get_weights
int orc_mesh(void* p) {
  State& S = *(State*)p;
  make_kp_reg(S);
  get_negatives(S);
  get_weights(S);
  return S.nibz;
}

int orc_get_kpc(void* p, double* kpc) {
  State& S = *(State*)p;
  std::memcpy(kpc, S.kpc.data(), S.kpc.size() * sizeof(double));
  return 0;
}

int orc_get_ibz(void* p, int* mapibz, int* mapinv, double* kibz, double* wibz, int* mappos) {
  State& S = *(State*)p;
  std::memcpy(mapibz, S.mapibz.data(), S.nkc * sizeof(int));
  std::memcpy(mapinv, S.mapinv.data(), S.nibz * sizeof(int));
  std::memcpy(kibz, S.kibz.data(), 3 * S.nibz * sizeof(double));
  std::memcpy(wibz, S.wibz.data(), S.nibz * sizeof(double));
  if (mappos) std::memcpy(mappos, S.mappos.data(), S.nkc * sizeof(int));
  return 0;
}

int orc_get_k_info(void* p, const double* q, int* out5) {
  State& S = *(State*)p;
  get_k_info(S, q, out5[0], out5[1], out5[2], out5[3], out5[4]);
  return 0;
}

int orc_getstar(void* p, const double* q, double* star, int* ops) {
  State& S = *(State*)p;
  int narms;
  double st[48][3];
  getstar(S, q, narms, st, ops);
  for (int s = 0; s < narms; ++s)
    for (int c = 0; c < 3; ++c) star[3 * s + c] = st[s][c];
  return narms;
}

int orc_kstars(void* p, const double* q, double* star, int* ops) {
  State& S = *(State*)p;
  int narms;
  double st[48][3];
  kstarsinfbz1(S, q, narms, st, ops);
  for (int s = 0; s < narms; ++s)
    for (int c = 0; c < 3; ++c) star[3 * s + c] = st[s][c];
  return narms;
}

int orc_dynmat(void* p, const double* q, double* dyn) {
  State& S = *(State*)p;
  set_dynamical_matrix(S, q, (cplx*)dyn);
  return 0;
}

int orc_get_freq(void* p, const double* q, double* eival, double* eivec) {
  State& S = *(State*)p;
  get_freq(S, q, eival, (cplx*)eivec);
  return 0;
}

int orc_phonons(void* p, int nthreads) {
  State& S = *(State*)p;
  get_frequencies(S, nthreads);
  subst_eivecs(S);
  return 0;
}

int orc_get_phonons(void* p, double* eigenval, double* eigenvec, double* veloc) {
  State& S = *(State*)p;
  if (eigenval) std::memcpy(eigenval, S.eigenval.data(), S.eigenval.size() * sizeof(double));
  if (eigenvec) std::memcpy(eigenvec, S.eigenvec.data(), S.eigenvec.size() * sizeof(cplx));
  if (veloc) std::memcpy(veloc, S.veloc.data(), S.veloc.size() * sizeof(double));
  return 0;
}

int orc_set_phonons(void* p, const double* eigenval, const double* eigenvec, const double* veloc) {
  State& S = *(State*)p;
  size_t n = S.ndyn, nk = S.nkc;
  S.eigenval.assign(eigenval, eigenval + n * nk);
  S.eigenvec.resize(n * n * nk);
  std::memcpy((void*)S.eigenvec.data(), eigenvec, n * n * nk * sizeof(cplx));
  S.veloc.assign(veloc, veloc + 3 * n * nk);
  return 0;
}

int orc_tet(void* p, int* corners) {
  State& S = *(State*)p;
  make_kp_reg_tet(S);
  if (corners)
    for (size_t t = 0; t < S.tet.size(); ++t)
      for (int k = 0; k < 4; ++k) corners[4 * t + k] = S.tet[t].i[k];
  return (int)S.tet.size();
}

int orc_v3(void* p, int k1, int k2, double* v33s8, int nthreads, char* err, int errlen) {
  State& S = *(State*)p;
  try {
    calculate_w3_ibz_split_sq(S, k1, k2, v33s8, nthreads);
  } catch (std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}

int orc_fgr(void* p, int k1, int k2, const double* v33s8, double* P1smpi, double* P2smpi, int gauss,
            int nthreads) {
  State& S = *(State*)p;
  if (gauss)
    calculate_FGR_gauss(S, k1, k2, v33s8, P1smpi, P2smpi, nthreads);
  else
    calculate_FGR_mpi2(S, k1, k2, v33s8, P1smpi, P2smpi, nthreads);
  return 0;
}

long orc_weight_tet_nonperm() { return g_weight_tet_nonperm.load(); }

// one tetrahedron: w[4] corner energies, e -> c[4]
int orc_weight_tet(const double* w, double e, double* c) {
  Tetra T;
  for (int k = 0; k < 4; ++k) {
    T.w[k] = w[k];
    T.c[k] = -12345.0;
  }
  weight_tet_one(T, e);
  for (int k = 0; k < 4; ++k) c[k] = T.c[k];
  return 0;
}

int orc_distribution(void* p, double tempk, double* frequency, double* dist) {
  State& S = *(State*)p;
  int e = distribution(S, tempk);
  if (frequency) std::memcpy(frequency, S.frequency.data(), S.frequency.size() * sizeof(double));
  if (dist) std::memcpy(dist, S.dist.data(), S.dist.size() * sizeof(double));
  return e;
}

int orc_tau(void* p, int k1, int k2, double tempk, const double* P1smpi, const double* P2smpi, double* Q,
            double* QN, double* QU, double* P1, double* P2, int nthreads) {
  State& S = *(State*)p;
  calculate_tauRTA_mpi2(S, k1, k2, tempk, P1smpi, P2smpi, Q, QN, QU, P1, P2, nthreads);
  return 0;
}

int orc_rta(void* p, double tempk, const double* Q, double* FFF, double* kappa) {
  State& S = *(State*)p;
  calculate_RTA_distributionfunction(S, tempk, Q, FFF);
  return mode_kappa(S, tempk, FFF, kappa);
}

int orc_collision(void* p, int k1, int k2, const double* P1, const double* P2, double* CM, int nthreads) {
  State& S = *(State*)p;
  CollisionMatrix_mpi(S, k1, k2, P1, P2, CM, nthreads);
  return 0;
}

int orc_rhs(void* p, double tempk, double* RHS) {
  State& S = *(State*)p;
  cal_RHS_IBZ(S, tempk, RHS);
  return 0;
}

int orc_cg(int n, const double* a, const double* b, double* x, double* fmin, int max_iter, int ndig,
           int nthreads) {
  return cg_quadratic(n, a, b, x, fmin, max_iter, ndig, nthreads);
}

int orc_kappa_d(void* p, double tempk, const double* x, double* kappa) {
  State& S = *(State*)p;
  return mode_kappa_d(S, tempk, x, kappa);
}

// mode_kappa from FFF(nibz,ndn,3) with the module array tauinv_eff(nibz,ndn)
// as it leaves it (teff in/out); keep_all = 1 skips the per-mode clearing,
// so that every mode keeps its own sum
int orc_mode_kappa_teff(void* p, double tempk, const double* FFF, double* kappa, double* teff, int keep_all) {
  State& S = *(State*)p;
  return mode_kappa(S, tempk, FFF, kappa, teff, keep_all == 0);
}

// mode_kappa_d adding to tauinv_eff(nibz,ndn) (teff in/out)
int orc_kappa_d_teff(void* p, double tempk, const double* x, double* kappa, double* teff) {
  State& S = *(State*)p;
  return mode_kappa_d(S, tempk, x, kappa, teff);
}

int orc_update_mpi(void* p, int k1, int k2, const double* P1, const double* P2, const double* Q,
                   const double* F_RTA, const double* FFF, double* F2, int nthreads) {
  State& S = *(State*)p;
  update_mpi(S, k1, k2, P1, P2, Q, F_RTA, FFF, F2, nthreads);
  return 0;
}

int orc_iterative(void* p, double tempk, const double* P1, const double* P2, const double* Q, const double* F_RTA,
                  int max_iter, double mix, double* FFF, double* kappa, int* iters, double* normk, int nthreads) {
  State& S = *(State*)p;
  return iterative_bte(S, tempk, P1, P2, Q, F_RTA, max_iter, mix, FFF, kappa, iters, normk, nthreads);
}

// cal_giso: g per primitive atom; 0, or 1 with the message in err
int orc_giso(void* p, double* g, char* err, int errlen) {
  State& S = *(State*)p;
  std::string e = cal_giso(S, g);
  if (!e.empty()) {
    std::snprintf(err, errlen, "%s", e.c_str());
    return 1;
  }
  return 0;
}

int orc_p_iso(void* p, int k1, int k2, const double* g, double* Piso, int nthreads) {
  State& S = *(State*)p;
  P_iso_split(S, k1, k2, g, Piso, nthreads);
  return 0;
}

int orc_collision_iso(void* p, const double* P1, const double* P2, const double* Piso, double* CM, int nthreads) {
  State& S = *(State*)p;
  CollisionMatrix_iso(S, P1, P2, Piso, CM, nthreads);
  return 0;
}

// make_kp_bs from dir/kpbs.params: *nkp points; kp (3,nkp) and dk (nkp)
// filled when cap >= nkp.  Returns 0, or 1 (message in err).
int orc_make_kp_bs(void* p, const char* dir, int* nkp, double* kp, double* dk, int cap, char* err, int errlen) {
  State& S = *(State*)p;
  std::vector<double> k, d;
  std::string e = make_kp_bs(S, dir, k, d);
  if (!e.empty()) {
    std::snprintf(err, errlen, "%s", e.c_str());
    return 1;
  }
  *nkp = (int)d.size();
  if (cap >= *nkp) {
    std::memcpy(kp, k.data(), k.size() * sizeof(double));
    std::memcpy(dk, d.data(), d.size() * sizeof(double));
  }
  return 0;
}

// get_frequencies at np points: eival (ndyn,np), eivec (ndyn,ndyn,np) complex
int orc_frequencies_at(void* p, int np, const double* kp, double* eival, double* eivec, int nthreads) {
  State& S = *(State*)p;
  frequencies_at(S, np, kp, eival, (cplx*)eivec, nthreads);
  return 0;
}

// function_self_w3 (gauss 0) / function_self_w4 (gauss 1) for each of np
// (point, la, omega) jobs: q (3,np), la (np, 1-based), omega (np), temp in
// cm^-1; out (4,np) = nself re, im, uself re, im.  Returns the first error.
int orc_self_w(void* p, int np, const double* q, const int* la, const double* omega, double temp, int gauss,
               double* out, int nthreads) {
  State& S = *(State*)p;
  std::vector<int> errs(np, 0);
  parfor(0, np - 1, nthreads, [&](int j) {
    cplx ns, us;
    errs[j] = function_self_w(S, &q[3 * j], la[j], omega[j], temp, gauss != 0, ns, us);
    out[4 * j] = ns.real();
    out[4 * j + 1] = ns.imag();
    out[4 * j + 2] = us.real();
    out[4 * j + 3] = us.imag();
  });
  for (int e : errs)
    if (e) return e;
  return 0;
}

int orc_check_inside_bz(void* p, const double* q) { return check_inside_bz(*(State*)p, q); }

}  // extern "C"
