// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle_core.h).  PARITY UNPINNED
// for everything in this file except nbe/distribution/cal_RHS_IBZ: no
// shipped reference output covers V3 and later stages.
//   cal_eiqr2                     THERMACOND/sub.f90:6015-6067
//   calculate_w3_ibz_split_sq     THERMACOND/sub.f90:1050-1233
//   matrix_elt_simplified         THERMACOND/sub.f90:5888-6011
//   weight_tet / ssort            THERMACOND/tetrahedron.f90:188-384, 716-738
//   calculate_FGR_mpi2            THERMACOND/sub.f90:7199-7499
//   nbe / delta_g                 THERMACOND/extratools.f90:239-285
//   distribution / cal_freq       THERMACOND/sub.f90:1955-2006
//   calculate_tauRTA_mpi2         THERMACOND/sub.f90:7953-8194
//   calculate_RTA_distributionfunction THERMACOND/sub.f90:1238-1289
//   mode_kappa / mode_kappa_d     THERMACOND/sub.f90:1292-1401, 1407-1530
//   veloc_avergeIBZ_invsyFBZ      THERMACOND/sub.f90:5479-5537
//   kstarsinfbz1                  THERMACOND/sub.f90:5551-5590
//   syop_f / syop_f2              THERMACOND/sub.f90:2117-2137, 8559-8580
//   CollisionMatrix_mpi           THERMACOND/sub.f90:3034-3210
//   cal_RHS_IBZ                   THERMACOND/sub.f90:2618-2691
//   cg_quadratic                  THERMACOND/cg.f90:19-61
//   get_kvecopn2, update_mpi      THERMACOND/sub.f90:2045-2111, 2295-2449
//   the job=3 mixing loop         THERMACOND/kappa.f90:1390-1487
#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>

#include "oracle_core.h"

namespace orc {

std::atomic<long> g_weight_tet_nonperm{0};

// ---------------------------------------------------------------- V3
void calculate_w3_ibz_split_sq(State& S, int k1, int k2, double* v33s8, int nthreads) {
  int ndn = S.ndyn, nk = S.nkc;
  int max_atomnum = 0;
  for (int t = 0; t < S.nterms[2]; ++t) max_atomnum = std::max(max_atomnum, S.iatomterm_3[1 + 3 * t]);
  // cal_eiqr2: eiqr2(i,j) = exp(i kpc(:,i).(atompos(:,j)-atompos(:,j0)))
  std::vector<cplx> eiqr2((size_t)nk * max_atomnum);
  for (int i = 1; i <= nk; ++i)
    for (int j = 1; j <= max_atomnum; ++j) {
      int j0 = S.iatomcell0[j - 1];
      double x = 0;
      for (int c = 1; c <= 3; ++c) x = x + S.kpc[F2(c, i, 3)] * (S.atompos[F2(c, j, 3)] - S.atompos[F2(c, j0, 3)]);
      eiqr2[F2(i, j, nk)] = cplx(std::cos(x), std::sin(x));
    }
  int nsub = k2 - k1 + 1;
  int nb = ndn / 3;
  std::atomic<int> err{0};
  // jobs: (row, l1, block of q2); each writes its own elements of v33s8, and
  // the arithmetic of every element is the reference's whatever the split
  const int q2blk = 256, nq2b = (nk + q2blk - 1) / q2blk;
  parfor(0, nsub * ndn * nq2b - 1, nthreads, [&](int job) {
    const int n1 = k1 + job / (ndn * nq2b);
    const int l1 = 1 + (job / nq2b) % ndn;
    const int n2lo = 1 + (job % nq2b) * q2blk, n2hi = std::min(nk, n2lo + q2blk - 1);
    int s = n1 - k1 + 1;
    std::vector<cplx> eivec3((size_t)27 * nb * nb * nb);
    double q1[3], q2[3], q3[3];
    for (int c = 0; c < 3; ++c) q1[c] = S.kpc[F2(c + 1, S.mapinv[n1 - 1], 3)];
    int nk1, i1, j1, kk1, inside;
    get_k_info(S, q1, nk1, i1, j1, kk1, inside);
    if (S.mapinv[n1 - 1] != nk1) {
      err = 1;
      return;
    }
    {
      for (int n2 = n2lo; n2 <= n2hi; ++n2) {
        for (int c = 0; c < 3; ++c) q2[c] = S.kpc[F2(c + 1, n2, 3)];
        int nk2, nk3;
        get_k_info(S, q2, nk2, i1, j1, kk1, inside);
        if (n2 != nk2) {
          err = 1;
          continue;
        }
        for (int c = 0; c < 3; ++c) q3[c] = -q2[c] - q1[c];
        get_k_info(S, q3, nk3, i1, j1, kk1, inside);
        for (int l2 = 1; l2 <= ndn; ++l2)
          for (int l3 = 1; l3 <= ndn; ++l3) {
            // matrix_elt_simplified
            for (int x1 = 1; x1 <= 3; ++x1)
              for (int x2 = 1; x2 <= 3; ++x2)
                for (int x3 = 1; x3 <= 3; ++x3)
                  for (int b1 = 1; b1 <= nb; ++b1)
                    for (int b2 = 1; b2 <= nb; ++b2)
                      for (int b3 = 1; b3 <= nb; ++b3) {
                        cplx e1 = S.eigenvec[F3(x1 + 3 * (b1 - 1), l1, nk1, ndn, ndn)];
                        cplx e2 = S.eigenvec[F3(x2 + 3 * (b2 - 1), l2, nk2, ndn, ndn)];
                        cplx e3 = S.eigenvec[F3(x3 + 3 * (b3 - 1), l3, nk3, ndn, ndn)];
                        size_t idx = (x1 - 1) + 3 * ((x2 - 1) + 3 * ((x3 - 1) + 3 * ((b1 - 1) + (size_t)nb *
                                     ((b2 - 1) + (size_t)nb * (b3 - 1)))));
                        eivec3[idx] = cmul(cmul(e1, e2), e3);
                      }
            cplx xx(0, 0);
            for (int t = 1; t <= S.nterms[2]; ++t) {
              int i3 = S.iatomterm_3[0 + 3 * (t - 1)];
              int i0 = S.iatomcell0[i3 - 1];
              if (S.iatomcell0[i3 - 1] != i3) continue;
              int j = S.iatomterm_3[1 + 3 * (t - 1)];
              int k = S.iatomterm_3[2 + 3 * (t - 1)];
              double mi = S.mass0[i0 - 1];
              int j0 = S.iatomcell0[j - 1];
              double mj = S.mass0[j0 - 1];
              int k0 = S.iatomcell0[k - 1];
              double mk = S.mass0[k0 - 1];
              int x1 = S.ixyzterm_3[0 + 3 * (t - 1)], x2 = S.ixyzterm_3[1 + 3 * (t - 1)],
                  x3 = S.ixyzterm_3[2 + 3 * (t - 1)];
              size_t idx = (x1 - 1) + 3 * ((x2 - 1) + 3 * ((x3 - 1) + 3 * ((i0 - 1) + (size_t)nb *
                           ((j0 - 1) + (size_t)nb * (k0 - 1)))));
              double wgt = S.fcs_3[t - 1] / std::sqrt(mi * mj * mk);
              cplx a = cplx(wgt * eiqr2[F2(nk2, j, nk)].real(), wgt * eiqr2[F2(nk2, j, nk)].imag());
              a = cmul(a, eiqr2[F2(nk3, k, nk)]);
              a = cmul(a, eivec3[idx]);
              xx = xx + a;
            }
            double den = std::sqrt(8 * std::sqrt(std::fabs(S.eigenval[F2(l1, nk1, ndn)] *
                                                           S.eigenval[F2(l2, nk2, ndn)] *
                                                           S.eigenval[F2(l3, nk3, ndn)])));
            double v = 0;
            if (den != 0) {
              cplx w33 = cplx(xx.real() / den * S.K.const33, xx.imag() / den * S.K.const33);
              v = (cmul(w33, std::conj(w33))).real();
            } else {
              err = 2;
            }
            v33s8[F5(s, n2, l1, l2, l3, nsub, nk, ndn, ndn)] = v;
          }
      }
    }
  });
  if (err) throw std::runtime_error(err == 2 ? "MATRIX_ELT: den=0" : "V3: index mismatch");
}

// ------------------------------------------------------------- weight_tet
// FP32 internals mirrored exactly: corner energies and differences are
// default REAL; terms that involve the REAL(8) argument e are evaluated in
// double (Fortran promotion rules); c/b temporaries are REAL.  Compiled
// with -ffp-contract=off so no FMA changes the rounding.
void weight_tet_one(Tetra& T, double e) {
  float en[4], en1[4];
  int uns[4];
  for (int k = 0; k < 4; ++k) en[k] = (float)T.w[k];
  for (int k = 0; k < 4; ++k) en1[k] = en[k];
  // ssort: descending by value (tetrahedron.f90:716-738)
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 4; ++j)
      if (en[j] > en[i]) std::swap(en[i], en[j]);
  if (en[0] != en[1] && en[1] != en[2] && en[2] != en[3]) {
    for (int k = 0; k < 4; ++k) {
      if (en[k] == en1[0]) uns[k] = 1;
      else if (en[k] == en1[1]) uns[k] = 2;
      else if (en[k] == en1[2]) uns[k] = 3;
      else if (en[k] == en1[3]) uns[k] = 4;
    }
  } else {
    for (int k = 0; k < 4; ++k) {
      if (en[k] == en1[0]) uns[k] = 1;
      else if (en[k] == en1[1]) uns[k] = 2;
      else if (en[k] == en1[2]) uns[k] = 3;
      else if (en[k] == en1[3]) uns[k] = 4;
      for (int l = 0; l < k; ++l) {
        if (uns[l] == uns[k] && uns[k] == 1) {
          if (en[k] == en1[1]) uns[k] = 2;
          else if (en[k] == en1[2]) uns[k] = 3;
          else if (en[k] == en1[3]) uns[k] = 4;
        } else if (uns[l] == uns[k] && uns[k] == 2) {
          if (en[k] == en1[2]) uns[k] = 3;
          else if (en[k] == en1[3]) uns[k] = 4;
        } else if (uns[l] == uns[k] && uns[k] == 3) {
          uns[k] = 4;
        }
      }
    }
  }
  {
    int seen = 0;
    for (int k = 0; k < 4; ++k) seen |= 1 << (uns[k] - 1);
    if (seen != 15) g_weight_tet_nonperm++;
  }
  float e1 = en[3], e2 = en[2], e3 = en[1], e4 = en[0];
  float e21 = e2 - e1, e31 = e3 - e1, e41 = e4 - e1, e32 = e3 - e2, e42 = e4 - e2, e43 = e4 - e3;
  const double small1 = 1e-10, small2 = 1e-10;
  auto fix = [&](float& x) {
    if (std::fabs((double)x) < small1 && x > 0.0f) x = (float)small2;
    if (std::fabs((double)x) < small1 && x < 0.0f) x = (float)(-small2);
  };
  fix(e21);
  fix(e31);
  fix(e41);
  fix(e42);
  fix(e43);
  double c[4];
  const double E1 = e1, E2 = e2, E3 = e3, E4 = e4;
  const double D21 = e21, D31 = e31, D41 = e41, D32 = e32, D42 = e42, D43 = e43;
  if (e < E1 || e > E4) {
    c[3] = 0;
    c[2] = 0;
    c[1] = 0;
    c[0] = 0;
  } else if (E1 <= e && e <= E2) {
    double x = e - E1;
    c[3] = ((E2 - e) / D21 + (E3 - e) / D31 + (E4 - e) / D41) * (x * x) / (double)((e41 * e31) * e21);
    double x3 = x * (x * x);
    c[2] = x3 / (double)(((e21 * e21) * e31) * e41);
    c[1] = x3 / (double)((e21 * (e31 * e31)) * e41);
    c[0] = x3 / (double)((e21 * e31) * (e41 * e41));
  } else if (E2 <= e && e <= E3) {
    float c11 = (float)((E3 - e) / (double)(e31 * e31));
    float c12 = (float)((E4 - e) / (double)(e41 * e41));
    float c21 = (float)((E3 - e) / (double)(e32 * e32));
    float c22 = (float)((E4 - e) / (double)(e42 * e42));
    float c31 = (float)((e - E2) / (double)(e32 * e32));
    float c32 = (float)((e - E1) / (double)(e31 * e31));
    float c41 = (float)((e - E2) / (double)(e42 * e42));
    float c42 = (float)((e - E1) / (double)(e41 * e41));
    float b11 = (float)((E3 - e) * (e - E2) / (double)(e42 * e32) + (E4 - e) * (e - E1) / (double)(e41 * e42) +
                        (E3 - e) * (e - E1) / (double)(e32 * e41));
    float b12 = (float)((E4 - e) * (e - E1) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e32) +
                        (E3 - e) * (e - E1) / (double)(e31 * e32));
    float b21 = (float)((E3 - e) * (e - E2) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e41) +
                        (E3 - e) * (e - E1) / (double)(e31 * e41));
    float b22 = (float)((E3 - e) * (e - E2) / (double)(e32 * e31) + (E4 - e) * (e - E1) / (double)(e41 * e31) +
                        (E4 - e) * (e - E2) / (double)(e32 * e41));
    float b31 = (float)((E3 - e) * (e - E2) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e41) +
                        (E3 - e) * (e - E1) / (double)(e31 * e41));
    float b32 = (float)((E3 - e) * (e - E2) / (double)(e42 * e32) + (E4 - e) * (e - E1) / (double)(e41 * e42) +
                        (E3 - e) * (e - E1) / (double)(e32 * e41));
    float b41 = (float)((E3 - e) * (e - E2) / (double)(e32 * e31) + (E4 - e) * (e - E1) / (double)(e41 * e31) +
                        (E4 - e) * (e - E2) / (double)(e32 * e41));
    float b42 = (float)((E4 - e) * (e - E1) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e32) +
                        (E3 - e) * (e - E1) / (double)(e31 * e32));
    c[3] = (double)(0.5f * (c11 * b11 + c12 * b12));
    c[2] = (double)(0.5f * (c21 * b21 + c22 * b22));
    c[1] = (double)(0.5f * (c31 * b31 + c32 * b32));
    c[0] = (double)(0.5f * (c41 * b41 + c42 * b42));
  } else {
    double x = E4 - e;
    double x3 = x * (x * x);
    c[3] = x3 / (double)(((e41 * e41) * e42) * e43);
    c[2] = x3 / (double)((e41 * (e42 * e42)) * e43);
    c[1] = x3 / (double)((e41 * e42) * (e43 * e43));
    c[0] = ((e - E3) / D43 + (e - E2) / D42 + (e - E1) / D41) * (x * x) / (double)((e41 * e42) * e43);
  }
  // p(uns(s))%c = c_s  (s=1 highest ... s=4 lowest)
  for (int s = 3; s >= 0; --s) T.c[uns[s] - 1] = c[s];
  (void)D32;
}

// --------------------------------------------------------- FGR (tetra)
static void fgr_core(State& S, int k1, int k2, const double* v33s8, double* P1smpi, double* P2smpi,
                     int nthreads, bool gauss) {
  int ndn = S.ndyn, nkc = S.nkc;
  int nsub = k2 - k1 + 1;
  const int* NC = S.nc;
  // cal_freq
  S.frequency.assign((size_t)nkc * ndn, 0.0);
  for (int i = 1; i <= nkc; ++i)
    for (int ii = 1; ii <= ndn; ++ii)
      S.frequency[F2(i, ii, nkc)] = std::sqrt(S.eigenval[F2(ii, i, ndn)]) * S.K.cnst;
  size_t tot = (size_t)nsub * nkc * ndn * ndn * ndn;
  std::fill(P1smpi, P1smpi + tot, 0.0);
  std::fill(P2smpi, P2smpi + tot, 0.0);
  const double twopi2 = (2 * S.K.pi) * (2 * S.K.pi);
  const double sig = S.width;
  parfor(0, nsub * ndn - 1, nthreads, [&](int job) {
      int n1 = job / ndn + 1, ii = job % ndn + 1;
      std::vector<Tetra> tet = S.tet;  // private copy of the module array
      std::vector<double> F_arbi(nkc);
      int i = S.mapinv[n1 + k1 - 1 - 1];
      double omega1 = S.frequency[F2(i, ii, nkc)];
      for (int jj = 1; jj <= ndn; ++jj)
        for (int kk = 1; kk <= ndn; ++kk) {
          // ---------------- process 1
          for (int j = 1; j <= nkc; ++j) {
            double q1[3], q2[3], q3p[3];
            for (int c = 0; c < 3; ++c) {
              q1[c] = S.kpc[F2(c + 1, i, 3)];
              q2[c] = S.kpc[F2(c + 1, j, 3)];
              q3p[c] = q1[c] + q2[c];
            }
            int nk2, i2, j2, kx2, ins, nk3, i3, j3, k3, ins1;
            get_k_info(S, q2, nk2, i2, j2, kx2, ins);
            get_k_info(S, q3p, nk3, i3, j3, k3, ins1);
            double V3sq1 = v33s8[F5(n1, j, ii, jj, kk, nsub, nkc, ndn, ndn)] * twopi2 / nkc;
            if (jj <= 3 && i2 == NC[0] / 2 + 1 && j2 == NC[1] / 2 + 1 && kx2 == NC[2] / 2 + 1) V3sq1 = 0.0;
            if (kk <= 3 && i3 == NC[0] / 2 + 1 && j3 == NC[1] / 2 + 1 && k3 == NC[2] / 2 + 1) V3sq1 = 0.0;
            if (!gauss) {
              F_arbi[j - 1] = V3sq1;
            } else {
              // Gaussian extension: delta_g(omega1 + omega2 - omega3)
              double x = omega1 + S.frequency[F2(j, jj, nkc)] - S.frequency[F2(nk3, kk, nkc)];
              double d = std::exp(-x * x / 2.0 / sig / sig) / std::sqrt(2 * S.K.pi) / sig;
              P1smpi[F5(n1, j, ii, jj, kk, nsub, nkc, ndn, ndn)] = V3sq1 * d;
            }
          }
          if (!gauss) {
            for (size_t jt = 0; jt < tet.size(); ++jt)
              for (int kt = 0; kt < 4; ++kt) {
                int w = tet[jt].i[kt];
                double q3p[3];
                for (int c = 0; c < 3; ++c) q3p[c] = S.kpc[F2(c + 1, i, 3)] + S.kpc[F2(c + 1, w, 3)];
                int nk3, i3, j3, k3, ins;
                get_k_info(S, q3p, nk3, i3, j3, k3, ins);
                tet[jt].w[kt] = -S.frequency[F2(w, jj, nkc)] + S.frequency[F2(nk3, kk, nkc)];
              }
            for (auto& T : tet) weight_tet_one(T, omega1);
            for (size_t jt = 0; jt < tet.size(); ++jt)
              for (int kt = 0; kt < 4; ++kt) {
                int w = tet[jt].i[kt];
                P1smpi[F5(n1, w, ii, jj, kk, nsub, nkc, ndn, ndn)] += tet[jt].c[kt] / 6.0 * F_arbi[w - 1];
              }
          }
          // ---------------- process 2
          for (int j = 1; j <= nkc; ++j) {
            double q1[3], q2[3], q2n[3], q3p[3];
            for (int c = 0; c < 3; ++c) {
              q1[c] = S.kpc[F2(c + 1, i, 3)];
              q2[c] = S.kpc[F2(c + 1, j, 3)];
              q2n[c] = -S.kpc[F2(c + 1, j, 3)];
              q3p[c] = q1[c] + q2[c];
            }
            int nk2, i2, j2, kx2, ins, nk2n, i2n, j2n, k2n, nk3, i3, j3, k3, ins2;
            get_k_info(S, q2, nk2, i2, j2, kx2, ins);
            get_k_info(S, q2n, nk2n, i2n, j2n, k2n, ins);
            get_k_info(S, q3p, nk3, i3, j3, k3, ins2);
            double V3sq1 = v33s8[F5(n1, j, ii, jj, kk, nsub, nkc, ndn, ndn)] * twopi2 / nkc;
            if (jj <= 3 && i2n == NC[0] / 2 + 1 && j2n == NC[1] / 2 + 1 && k2n == NC[2] / 2 + 1) V3sq1 = 0.0;
            if (kk <= 3 && i3 == NC[0] / 2 + 1 && j3 == NC[1] / 2 + 1 && k3 == NC[2] / 2 + 1) V3sq1 = 0.0;
            if (!gauss) {
              F_arbi[nk2n - 1] = V3sq1;
            } else {
              // point -q2 carries |V3(q1,q2)|^2; delta_g(omega1 - omega2(-q2) - omega3(q1+q2))
              double x = omega1 - S.frequency[F2(nk2n, jj, nkc)] - S.frequency[F2(nk3, kk, nkc)];
              double d = std::exp(-x * x / 2.0 / sig / sig) / std::sqrt(2 * S.K.pi) / sig;
              P2smpi[F5(n1, nk2n, ii, jj, kk, nsub, nkc, ndn, ndn)] = V3sq1 * d;
            }
          }
          if (!gauss) {
            for (size_t jt = 0; jt < tet.size(); ++jt)
              for (int kt = 0; kt < 4; ++kt) {
                int w = tet[jt].i[kt];
                double q3p[3];
                for (int c = 0; c < 3; ++c) q3p[c] = S.kpc[F2(c + 1, i, 3)] - S.kpc[F2(c + 1, w, 3)];
                int nk3, i3, j3, k3, ins;
                get_k_info(S, q3p, nk3, i3, j3, k3, ins);
                tet[jt].w[kt] = S.frequency[F2(w, jj, nkc)] + S.frequency[F2(nk3, kk, nkc)];
              }
            for (auto& T : tet) weight_tet_one(T, omega1);
            for (size_t jt = 0; jt < tet.size(); ++jt)
              for (int kt = 0; kt < 4; ++kt) {
                int w = tet[jt].i[kt];
                P2smpi[F5(n1, w, ii, jj, kk, nsub, nkc, ndn, ndn)] += tet[jt].c[kt] / 6.0 * F_arbi[w - 1];
              }
          }
        }
  });
}

void calculate_FGR_mpi2(State& S, int k1, int k2, const double* v33s8, double* P1smpi, double* P2smpi,
                        int nthreads) {
  fgr_core(S, k1, k2, v33s8, P1smpi, P2smpi, nthreads, false);
}
void calculate_FGR_gauss(State& S, int k1, int k2, const double* v33s8, double* P1smpi, double* P2smpi,
                         int nthreads) {
  fgr_core(S, k1, k2, v33s8, P1smpi, P2smpi, nthreads, true);
}

// ------------------------------------------------------------- Bose
double nbe(double w, double t, int m, int* err) {
  if (t <= 0) {
    *err = 1;
    return 0;
  }
  if (w <= 0) {
    *err = 2;
    return 0;
  }
  double z = w / t, y;
  if (m == 0) {
    if (z > 60)
      y = 0;
    else if (z < (double)0.0010f)
      y = 1 / (z * (1 + z / 2 * (1 + z / 3)));
    else
      y = 1 / (std::exp(z) - 1);
  } else {
    y = 1 / z;
  }
  return y;
}

int distribution(State& S, double tempk) {
  int nk = S.nkc, ndn = S.ndyn;
  double temp = tempk * S.K.k_b / (100 * S.K.h_plank * S.K.c_light);
  S.frequency.assign((size_t)nk * ndn, 0.0);
  S.dist.assign((size_t)nk * ndn, 0.0);
  int err = 0;
  for (int i = 1; i <= nk; ++i)
    for (int ii = 1; ii <= ndn; ++ii) {
      S.frequency[F2(i, ii, nk)] = std::sqrt(S.eigenval[F2(ii, i, ndn)]) * S.K.cnst;
      S.dist[F2(i, ii, nk)] = nbe(S.frequency[F2(i, ii, nk)], temp, S.classical, &err);
    }
  return err;
}

// ------------------------------------------------------------- Q
void calculate_tauRTA_mpi2(State& S, int k1, int k2, double tempk, const double* P1smpi,
                           const double* P2smpi, double* Q, double* QN, double* QU, double* P1, double* P2,
                           int nthreads) {
  int ndn = S.ndyn, nkc = S.nkc;
  int nsub = k2 - k1 + 1;
  (void)tempk;
  parfor(1, nsub, nthreads, [&](int ibz) {
    int i = S.mapinv[ibz + k1 - 1 - 1];
    for (int ii = 1; ii <= ndn; ++ii) {
      double q = 0, qn = 0, qu = 0;
      for (int jj = 1; jj <= ndn; ++jj)
        for (int kk = 1; kk <= ndn; ++kk)
          for (int j = 1; j <= nkc; ++j) {
            double q1[3], q3a[3], q3b[3];
            for (int c = 0; c < 3; ++c) {
              q1[c] = S.kpc[F2(c + 1, i, 3)];
              q3a[c] = q1[c] + S.kpc[F2(c + 1, j, 3)];
              q3b[c] = q1[c] - S.kpc[F2(c + 1, j, 3)];
            }
            int nka, nkb, a1, a2, a3, in1, in2;
            get_k_info(S, q3a, nka, a1, a2, a3, in1);
            get_k_info(S, q3b, nkb, a1, a2, a3, in2);
            size_t idx = F5(ibz, j, ii, jj, kk, nsub, nkc, ndn, ndn);
            double F = S.dist[F2(i, ii, nkc)] * S.dist[F2(j, jj, nkc)] * (S.dist[F2(nka, kk, nkc)] + 1);
            double p1 = P1smpi[idx] * F;
            F = S.dist[F2(i, ii, nkc)] * (S.dist[F2(j, jj, nkc)] + 1) * (S.dist[F2(nkb, kk, nkc)] + 1);
            double p2 = P2smpi[idx] * F;
            if (P1) P1[idx] = p1;
            if (P2) P2[idx] = p2;
            q = q + (p1 + 0.5 * p2);
            if (in1 == 1)
              qn = qn + p1;
            else
              qu = qu + p1;
            if (in2 == 1)
              qn = qn + 0.5 * p2;
            else
              qu = qu + 0.5 * p2;
          }
      Q[F2(ibz, ii, nsub)] = q;
      QN[F2(ibz, ii, nsub)] = qn;
      QU[F2(ibz, ii, nsub)] = qu;
    }
  });
}

// ------------------------------------------------------- RTA and kappa
void calculate_RTA_distributionfunction(State& S, double tempk, const double* Q, double* FFF) {
  int ndn = S.ndyn, nkc = S.nkc, nibz = S.nibz;
  const Consts& K = S.K;
  for (int i = 1; i <= nibz; ++i)
    for (int ii = 1; ii <= ndn; ++ii) {
      double omega = S.frequency[F2(S.mapinv[i - 1], ii, nkc)];
      double nb = S.dist[F2(S.mapinv[i - 1], ii, nkc)];
      for (int iii = 1; iii <= 3; ++iii) {
        double v = S.veloc[F3(iii, ii, S.mapinv[i - 1], 3, ndn)];
        FFF[F3(i, ii, iii, nibz, ndn)] = -((((((K.c_light * v) * K.h_plank) * ((omega * K.c_light) * 100)) * nb) *
                                             (nb + 1)) / (K.k_b * (tempk * tempk)) /
                                            ((Q[F2(i, ii, nibz)] * K.c_light) * 100));
      }
    }
}

void kstarsinfbz1(const State& S, const double q[3], int& ds, double kvecstars[][3], int kvecops[]) {
  int narms, kvecop[48];
  double kvecstar[48][3];
  const double tol = (double)0.0001f;  // params tolerance (rest.f90:32)
  getstar(S, q, narms, kvecstar, kvecop);
  ds = 0;
  for (int s = 1; s <= narms; ++s)
    for (int j = 1; j <= S.nkc; ++j) {
      const double* qk = &S.kpc[F2(1, j, 3)];
      if (std::fabs(qk[0] - kvecstar[s - 1][0]) < tol && std::fabs(qk[1] - kvecstar[s - 1][1]) < tol &&
          std::fabs(qk[2] - kvecstar[s - 1][2]) < tol) {
        ds = ds + 1;
        for (int c = 0; c < 3; ++c) kvecstars[ds - 1][c] = kvecstar[s - 1][c];
        kvecops[ds - 1] = kvecop[s - 1];
      }
    }
}

static void syop_f(const State& S, int s, const double* ff, double* fs) {
  const double* op = S.op_kmatrix[s - 1];
  for (int i = 1; i <= 3; ++i) {
    double x = 0;
    for (int j = 1; j <= 3; ++j) x = x + op[F2(i, j, 3)] * ff[j - 1];
    fs[i - 1] = x;
  }
}

// teff (optional) is the module array tauinv_eff(nibz,ndn): mode_kappa
// (averaged = false) clears all of it before each mode (sub.f90:1337) and
// adds per arm and j const2 F12(j)/omega/velocc(j)/(3 narms), or /0.01 where
// velocc(j) == 0 (sub.f90:1360-1365); mode_kappa_d (averaged = true) adds to
// what it holds, per arm and j, const2 (F12.velocc)/omega/(velocc.velocc)/(3
// narms) (sub.f90:1497).
static int kappa_core(State& S, double tempk, const double* FFF, const double* velsrc, bool averaged,
                      double* kappa, double* teff = nullptr, bool reset = true) {
  int ndn = S.ndyn, nkc = S.nkc, nibz = S.nibz;
  const Consts& K = S.K;
  double temp = tempk * K.k_b / (100 * K.h_plank * K.c_light);
  double const1 = K.h_plank * K.c_light * 100 * K.c_light / (nkc * S.volume_r / 1e30);
  double const2 = K.k_b * (tempk * tempk) / (K.h_plank * K.c_light * 100) / K.c_light;
  std::fill(kappa, kappa + ndn * 9, 0.0);
  int err = 0;
  for (int i = 1; i <= nibz; ++i) {
    double q[3] = {S.kibz[F2(1, i, 3)], S.kibz[F2(2, i, 3)], S.kibz[F2(3, i, 3)]};
    int narms, kvecop[48];
    double kvecstar[48][3];
    kstarsinfbz1(S, q, narms, kvecstar, kvecop);
    for (int ii = 1; ii <= ndn; ++ii) {
      if (teff && !averaged && reset) std::fill(teff, teff + (size_t)nibz * ndn, 0.0);
      for (int s = 1; s <= narms; ++s) {
        double F12[3], velocc[3], f[3], vv[3];
        for (int c = 0; c < 3; ++c) f[c] = FFF[F3(i, ii, c + 1, nibz, ndn)];
        syop_f(S, kvecop[s - 1], f, F12);
        if (averaged)
          for (int c = 0; c < 3; ++c) vv[c] = velsrc[F3(c + 1, ii, i, 3, ndn)];
        else
          for (int c = 0; c < 3; ++c) vv[c] = velsrc[F3(c + 1, ii, S.mapinv[i - 1], 3, ndn)];
        syop_f(S, kvecop[s - 1], vv, velocc);
        int n0, a1, a2, a3, ins;
        get_k_info(S, kvecstar[s - 1], n0, a1, a2, a3, ins);
        double omega = std::sqrt(S.eigenval[F2(ii, n0, ndn)]) * K.cnst;
        double nb0 = nbe(omega, temp, S.classical, &err);
        for (int j = 1; j <= 3; ++j) {
          for (int jj = 1; jj <= 3; ++jj)
            kappa[F3(ii, j, jj, ndn, 3)] = kappa[F3(ii, j, jj, ndn, 3)] -
                                           ((((const1 * omega) * velocc[j - 1]) * nb0) * (nb0 + 1)) * F12[jj - 1];
          if (!teff) continue;
          double& t = teff[F2(i, ii, nibz)];
          if (!averaged) {
            if (velocc[j - 1] == 0.0)
              t = t - const2 * F12[j - 1] / omega / 0.01;
            else
              t = t - const2 * F12[j - 1] / omega / velocc[j - 1] / (narms * 3.0);
          } else {
            double fv = 0, v2 = 0;  // dot_product
            for (int c = 0; c < 3; ++c) fv = fv + F12[c] * velocc[c];
            for (int c = 0; c < 3; ++c) v2 = v2 + velocc[c] * velocc[c];
            t = t - const2 * fv / omega / v2 / (narms * 3.0);
          }
        }
      }
    }
  }
  return err;
}

int mode_kappa(State& S, double tempk, const double* FFF, double* kappa, double* teff, bool reset) {
  return kappa_core(S, tempk, FFF, S.veloc.data(), false, kappa, teff, reset);
}

int mode_kappa_d(State& S, double tempk, const double* Fi_x, double* kappa, double* teff) {
  int ndn = S.ndyn, nibz = S.nibz;
  std::vector<double> FFF((size_t)nibz * ndn * 3);
  int r = 0;
  for (int i1 = 1; i1 <= nibz; ++i1)
    for (int j1 = 1; j1 <= ndn; ++j1)
      for (int j2 = 1; j2 <= 3; ++j2) FFF[F3(i1, j1, j2, nibz, ndn)] = Fi_x[r++];
  // veloc_avergeIBZ_invsyFBZ: star average with inverse operations
  std::vector<double> veloci((size_t)3 * ndn * nibz, 0.0);
  for (int i = 1; i <= nibz; ++i) {
    double qi[3] = {S.kibz[F2(1, i, 3)], S.kibz[F2(2, i, 3)], S.kibz[F2(3, i, 3)]};
    int narms, kvecops[48];
    double kvecstars[48][3];
    getstar(S, qi, narms, kvecstars, kvecops);
    for (int j = 1; j <= ndn; ++j) {
      double veli_a[3] = {0, 0, 0};
      for (int n = 1; n <= narms; ++n) {
        int n0, a1, a2, a3, ins;
        get_k_info(S, kvecstars[n - 1], n0, a1, a2, a3, ins);
        // syop_f2: inverse of op_kmatrix (xmatinv) applied to veloc(:,j,n0)
        double inv[9];
        {
          // op_kmatrix entries are integers with |det|=1: exact inverse by cofactors
          const double* m = S.op_kmatrix[kvecops[n - 1] - 1];
          auto M = [&](int a, int b) { return m[F2(a, b, 3)]; };
          double det = M(1, 1) * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)) -
                       M(1, 2) * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1)) +
                       M(1, 3) * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
          inv[F2(1, 1, 3)] = (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)) / det;
          inv[F2(1, 2, 3)] = (M(1, 3) * M(3, 2) - M(1, 2) * M(3, 3)) / det;
          inv[F2(1, 3, 3)] = (M(1, 2) * M(2, 3) - M(1, 3) * M(2, 2)) / det;
          inv[F2(2, 1, 3)] = (M(2, 3) * M(3, 1) - M(2, 1) * M(3, 3)) / det;
          inv[F2(2, 2, 3)] = (M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1)) / det;
          inv[F2(2, 3, 3)] = (M(1, 3) * M(2, 1) - M(1, 1) * M(2, 3)) / det;
          inv[F2(3, 1, 3)] = (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1)) / det;
          inv[F2(3, 2, 3)] = (M(1, 2) * M(3, 1) - M(1, 1) * M(3, 2)) / det;
          inv[F2(3, 3, 3)] = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) / det;
        }
        double veli[3];
        for (int a = 1; a <= 3; ++a) {
          double x = 0;
          for (int b = 1; b <= 3; ++b) x = x + inv[F2(a, b, 3)] * S.veloc[F3(b, j, n0, 3, ndn)];
          veli[a - 1] = x;
        }
        for (int c = 0; c < 3; ++c) veli_a[c] = veli_a[c] + (veli[c] / narms);
      }
      for (int c = 0; c < 3; ++c) veloci[F3(c + 1, j, i, 3, ndn)] = veli_a[c];
    }
  }
  return kappa_core(S, tempk, FFF.data(), veloci.data(), true, kappa, teff);
}

// ------------------------------------------------------- collision matrix
void CollisionMatrix_mpi(State& S, int k1, int k2, const double* P1, const double* P2, double* CM,
                         int nthreads) {
  int ndn = S.ndyn, nkc = S.nkc, nibz = S.nibz;
  int nsub = k2 - k1 + 1;
  int nrow = nsub * ndn * 3, ncol = nibz * ndn * 3;
  std::fill(CM, CM + (size_t)nrow * ncol, 0.0);
  // arms of every IBZ point (kstarsinfbz1 is called inside the n2 loop in
  // the reference; it depends on n2 only, so it is hoisted unchanged)
  std::vector<int> narms(nibz);
  std::vector<int> armop((size_t)nibz * 48);
  std::vector<double> armq((size_t)nibz * 48 * 3);
  parfor(1, nibz, nthreads, [&](int n2) {
    double q[3] = {S.kibz[F2(1, n2, 3)], S.kibz[F2(2, n2, 3)], S.kibz[F2(3, n2, 3)]};
    int na, ops[48];
    double st[48][3];
    kstarsinfbz1(S, q, na, st, ops);
    narms[n2 - 1] = na;
    for (int s = 0; s < na; ++s) {
      armop[(size_t)(n2 - 1) * 48 + s] = ops[s];
      for (int c = 0; c < 3; ++c) armq[((size_t)(n2 - 1) * 48 + s) * 3 + c] = st[s][c];
    }
  });
  parfor(0, nsub * ndn - 1, nthreads, [&](int job) {
      int n1 = job / ndn + 1, l1 = job % ndn + 1;
      int n1i = S.mapinv[n1 + k1 - 1 - 1];
      int d1 = 3 * ((n1 - 1) * ndn + (l1 - 1)) + 1;
      for (int n2 = 1; n2 <= nibz; ++n2)
        for (int l2 = 1; l2 <= ndn; ++l2) {
          int d2 = 3 * ((n2 - 1) * ndn + (l2 - 1)) + 1;
          for (int ns = 1; ns <= narms[n2 - 1]; ++ns) {
            const double* arm = &armq[((size_t)(n2 - 1) * 48 + ns - 1) * 3];
            int op = armop[(size_t)(n2 - 1) * 48 + ns - 1];
            int n0, a1, a2, a3, ins;
            get_k_info(S, arm, n0, a1, a2, a3, ins);
            double C = 0;
            if (n1i == n0 && l1 == l2) {
              for (int nl2 = 1; nl2 <= ndn; ++nl2)
                for (int l3 = 1; l3 <= ndn; ++l3)
                  for (int n22 = 1; n22 <= nkc; ++n22) {
                    size_t idx = F5(n1, n22, l1, nl2, l3, nsub, nkc, ndn, ndn);
                    C = C + (-P1[idx] - 0.5 * P2[idx]);
                  }
            } else {
              double q1[3] = {S.kibz[F2(1, n1 + k1 - 1, 3)], S.kibz[F2(2, n1 + k1 - 1, 3)],
                              S.kibz[F2(3, n1 + k1 - 1, 3)]};
              double qa[3], qb[3];
              for (int c = 0; c < 3; ++c) {
                qa[c] = q1[c] - arm[c];
                qb[c] = arm[c] - q1[c];
              }
              int nk3_p1, nk3_p2;
              get_k_info(S, qa, nk3_p1, a1, a2, a3, ins);
              get_k_info(S, qb, nk3_p2, a1, a2, a3, ins);
              for (int nl3 = 1; nl3 <= ndn; ++nl3) {
                double t = -P1[F5(n1, n0, l1, l2, nl3, nsub, nkc, ndn, ndn)] +
                           P1[F5(n1, nk3_p2, l1, l2, nl3, nsub, nkc, ndn, ndn)] +
                           0.5 * P2[F5(n1, n0, l1, l2, nl3, nsub, nkc, ndn, ndn)] +
                           0.5 * P2[F5(n1, nk3_p1, l1, l2, nl3, nsub, nkc, ndn, ndn)];
                C = C + t;
              }
            }
            const double* opm = S.op_kmatrix[op - 1];
            for (int i = 1; i <= 3; ++i)
              for (int j = 1; j <= 3; ++j) {
                size_t e = (size_t)(d1 + i - 1 - 1) + (size_t)nrow * (d2 + j - 1 - 1);
                CM[e] = CM[e] + (C * opm[F2(i, j, 3)]);
              }
          }
        }
  });
}

void cal_RHS_IBZ(State& S, double tempk, double* RHS) {
  int ndn = S.ndyn, nkc = S.nkc;
  const Consts& K = S.K;
  int s = 0;
  for (int i = 1; i <= S.nibz; ++i) {
    int n0 = S.mapinv[i - 1];
    for (int ii = 1; ii <= ndn; ++ii) {
      double omega = S.frequency[F2(n0, ii, nkc)];
      double nb0 = S.dist[F2(n0, ii, nkc)];
      for (int iii = 1; iii <= 3; ++iii) {
        double v = S.veloc[F3(iii, ii, n0, 3, ndn)];
        RHS[s++] = ((((((K.c_light * v) * K.h_plank) * ((omega * K.c_light) * 100)) * nb0) * (nb0 + 1)) /
                    (K.k_b * (tempk * tempk))) /
                   (K.c_light * 100);
      }
    }
  }
}

// ------------------------------------------------------------- CG
int cg_quadratic(int n, const double* a, const double* b, double* vmin, double* funcmin, int max_iter,
                 int n_dig_accur, int nthreads) {
  std::vector<double> conj(n), grad(n), aux(n), v0(n);
  double tolerance = 1.0 / std::pow(10.0, 2 * n_dig_accur);
  int iter = 0;
  double err = 9999;
  auto matvec = [&](const double* x, double* y) {
    const int blk = 64;
    parfor(0, (n + blk - 1) / blk - 1, nthreads, [&](int b) {
      for (int i = b * blk; i < std::min(n, (b + 1) * blk); ++i) {
        double s = 0;
        for (int j = 0; j < n; ++j) s = s + a[(size_t)i + (size_t)n * j] * x[j];
        y[i] = s;
      }
    });
  };
  auto dotp = [&](const double* x, const double* y) {
    double s = 0;
    for (int i = 0; i < n; ++i) s = s + x[i] * y[i];
    return s;
  };
  for (int i = 0; i < n; ++i) v0[i] = vmin[i];
  matvec(v0.data(), grad.data());
  for (int i = 0; i < n; ++i) grad[i] = grad[i] - b[i];
  for (int i = 0; i < n; ++i) conj[i] = -grad[i];
  while (iter < max_iter) {
    iter = iter + 1;
    matvec(conj.data(), aux.data());
    double num = dotp(grad.data(), conj.data());
    double den = dotp(aux.data(), conj.data());
    for (int i = 0; i < n; ++i) v0[i] = grad[i];
    for (int i = 0; i < n; ++i) vmin[i] = vmin[i] - num / den * conj[i];
    for (int i = 0; i < n; ++i) grad[i] = grad[i] - num / den * aux[i];
    double v2 = dotp(vmin, vmin);
    err = (num * num / den / den) * dotp(conj.data(), conj.data()) / v2;
    if (err < tolerance) break;
    num = dotp(grad.data(), grad.data());
    den = dotp(v0.data(), v0.data());
    for (int i = 0; i < n; ++i) conj[i] = -grad[i] + num / den * conj[i];
  }
  matvec(vmin, v0.data());
  *funcmin = 0.5 * dotp(vmin, v0.data()) - dotp(vmin, b);
  return iter;
}

// ------------------------------------------------- iterative BTE (job=3)
// kstarsinfbz1 of every IBZ point, computed once (kstarsinfbz1 is a pure
// function of the IBZ vector; update_mpi and get_kvecopn2 call it per arm)
struct IbzArms {
  std::vector<int> narms;
  std::vector<std::array<std::array<double, 3>, 48>> star;
  std::vector<std::array<int, 48>> op;
  std::vector<std::array<int, 48>> idx;  // get_k_info index of each arm
};

static void ibz_arms(const State& S, IbzArms& A) {
  A.narms.assign(S.nibz, 0);
  A.star.resize(S.nibz);
  A.op.resize(S.nibz);
  A.idx.resize(S.nibz);
  for (int n = 1; n <= S.nibz; ++n) {
    double q[3] = {S.kibz[F2(1, n, 3)], S.kibz[F2(2, n, 3)], S.kibz[F2(3, n, 3)]};
    int narms, ops[48];
    double st[48][3];
    kstarsinfbz1(S, q, narms, st, ops);
    A.narms[n - 1] = narms;
    for (int s = 0; s < narms; ++s) {
      for (int c = 0; c < 3; ++c) A.star[n - 1][s][c] = st[s][c];
      A.op[n - 1][s] = ops[s];
      int i3, j3, k3, inside;
      get_k_info(S, st[s], A.idx[n - 1][s], i3, j3, k3, inside);
    }
  }
}

// get_kvecopn2 (sub.f90:2045-2111): the op of the first arm of
// kstarsinfbz1(kibz(n)) whose mesh index equals that of k.  Like the
// reference, spf keeps its previous value when no arm matches.
static void get_kvecopn2(const State& S, const IbzArms& A, int n, const double k[3], int& spf) {
  int sk, i3, j3, k3, inside;
  get_k_info(S, k, sk, i3, j3, k3, inside);
  for (int s = 0; s < A.narms[n - 1]; ++s)
    if (A.idx[n - 1][s] == sk) {
      spf = A.op[n - 1][s];
      return;
    }
}

// update_mpi (sub.f90:2295-2449): F2(n1,l1,:) = F_RTA(n1,l1,:) + A(n1,l1,:)/Q(n1,l1)
// with A = sum over IBZ q2, its arms s and l2, l3 of
//   P1(n1,s,l1,l2,l3) (S_sp1 F(q1+s,l3) - S_sq2 F(q2,l2))
//   + 0.5 P2(n1,s,l1,l2,l3) (S_sq2 F(q2,l2) + S_sp2 F(q1-s,l3)).
// P1, P2: (nk1,nkc,ndn,ndn,ndn) Bose-weighted; Q, F_RTA, FFF over all IBZ
// points; F2mpi(nk1,ndn,3).  The arm data, which do not depend on l1 and
// xyz, are evaluated once per (q1, q2, arm) instead of inside those loops.
void update_mpi(State& S, int k1, int k2, const double* P1, const double* P2, const double* Q,
                const double* F_RTA, const double* FFF, double* F2mpi, int nthreads) {
  const int ndn = S.ndyn, nkc = S.nkc, nibz = S.nibz, nsub = k2 - k1 + 1;
  IbzArms A;
  ibz_arms(S, A);
  parfor(1, nsub, nthreads, [&](int ibz) {
    const int n1 = ibz + k1 - 1;
    const double q1[3] = {S.kibz[F2(1, n1, 3)], S.kibz[F2(2, n1, 3)], S.kibz[F2(3, n1, 3)]};
    struct Arm {
      int n2, ns, sq2, i1, i2, sp1f, sp2f;
    };
    std::vector<Arm> arms;
    int sp1f = 1, sp2f = 1;
    for (int n2 = 1; n2 <= nibz; ++n2)
      for (int s = 0; s < A.narms[n2 - 1]; ++s) {
        const double* ks = A.star[n2 - 1][s].data();
        double q3p1[3], q3p2[3];
        for (int c = 0; c < 3; ++c) {
          q3p1[c] = q1[c] + ks[c];
          q3p2[c] = q1[c] - ks[c];
        }
        int i3, j3, k3, inside, nk3p1, nk3p2;
        get_k_info(S, q3p1, nk3p1, i3, j3, k3, inside);
        get_k_info(S, q3p2, nk3p2, i3, j3, k3, inside);
        const int i1 = S.mapibz[nk3p1 - 1], i2 = S.mapibz[nk3p2 - 1];
        get_kvecopn2(S, A, i1, q3p1, sp1f);
        get_kvecopn2(S, A, i2, q3p2, sp2f);
        arms.push_back({n2, A.idx[n2 - 1][s], A.op[n2 - 1][s], i1, i2, sp1f, sp2f});
      }
    for (int l1 = 1; l1 <= ndn; ++l1)
      for (int xyz = 1; xyz <= 3; ++xyz) {
        double Av = 0;
        for (const Arm& a : arms)
          for (int l2 = 1; l2 <= ndn; ++l2)
            for (int l3 = 1; l3 <= ndn; ++l3) {
              double f[3], Fsq2[3], Fsp1[3], Fsp2[3];
              for (int c = 1; c <= 3; ++c) f[c - 1] = FFF[F3(a.n2, l2, c, nibz, ndn)];
              syop_f(S, a.sq2, f, Fsq2);
              for (int c = 1; c <= 3; ++c) f[c - 1] = FFF[F3(a.i1, l3, c, nibz, ndn)];
              syop_f(S, a.sp1f, f, Fsp1);
              for (int c = 1; c <= 3; ++c) f[c - 1] = FFF[F3(a.i2, l3, c, nibz, ndn)];
              syop_f(S, a.sp2f, f, Fsp2);
              const size_t pi = F5(ibz, a.ns, l1, l2, l3, nsub, nkc, ndn, ndn);
              Av = Av + P1[pi] * (Fsp1[xyz - 1] - Fsq2[xyz - 1]) + 0.5 * P2[pi] * (Fsq2[xyz - 1] + Fsp2[xyz - 1]);
            }
        F2mpi[F3(ibz, l1, xyz, nsub, ndn)] = F_RTA[F3(n1, l1, xyz, nibz, ndn)] + Av / Q[F2(n1, l1, nibz)];
      }
  });
}

// The job=3 iteration (kappa.f90:1390-1487): starting from F = F_RTA and the
// RTA kappa, repeat update_mpi over all IBZ rows, F += update_mix (F2 - F),
// kappa = mode_kappa(F), until sqrt(sum((kappa_new - kappa_old)^2)/(ndn*9)) <
// 1e-4 or max_iter iterations.  Returns the nbe error flag; *iters and
// *normk receive the iteration count and the last change.
int iterative_bte(State& S, double tempk, const double* P1, const double* P2, const double* Q,
                  const double* F_RTA, int max_iter, double update_mix, double* FFF, double* kappa, int* iters,
                  double* normk, int nthreads) {
  const int ndn = S.ndyn, nibz = S.nibz;
  const size_t nf = (size_t)nibz * ndn * 3;
  std::copy(F_RTA, F_RTA + nf, FFF);
  int err = mode_kappa(S, tempk, FFF, kappa);
  std::vector<double> F2(nf), kold(9 * (size_t)ndn);
  *iters = 0;
  *normk = 0;
  for (int i = 1; i <= max_iter; ++i) {
    std::copy(kappa, kappa + 9 * ndn, kold.begin());
    update_mpi(S, 1, nibz, P1, P2, Q, F_RTA, FFF, F2.data(), nthreads);
    for (size_t j = 0; j < nf; ++j) FFF[j] = FFF[j] + update_mix * (F2[j] - FFF[j]);
    err |= mode_kappa(S, tempk, FFF, kappa);
    double e = 0;
    for (int j = 0; j < 9 * ndn; ++j) e = e + (kappa[j] - kold[j]) * (kappa[j] - kold[j]) / (ndn * 3 * 3);
    *iters = i;
    *normk = std::sqrt(e);
    if (*normk < 0.0001) break;
  }
  return err;
}

}  // namespace orc

