// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle_core.h).  PARITY UNPINNED:
// no shipped reference output covers the isotope terms.
//
// Isotope scattering of THERMACOND (iso=1 in latdyn.params):
//   cal_g                 THERMACOND/sub.f90:3766-4693
//   cal_giso              THERMACOND/sub.f90:4695-4725
//   P_iso_split           THERMACOND/sub.f90:4825-4961
//   CollisionMatrix_iso   THERMACOND/sub.f90:3387-3570
//   calculate_tauRTA_iso  THERMACOND/sub.f90:8311-8549 (Q, Q_N, Q_U each + Piso;
//                         done by the callers of this file)
#include <algorithm>
#include <cstring>

#include "oracle_core.h"

namespace orc {

namespace {

// Natural isotopic compositions: (element, isotope mass in amu, abundance
// in percent), the values cal_g tabulates, for the elements covered here.
struct Iso {
  const char* el;
  double m, f;
};
const Iso kIso[] = {
    {"Ar", 35.967546, 0.34},    {"Ar", 37.962732, 0.063},   {"Ar", 39.962383, 99.6},
    {"C", 12.0, 98.9},          {"C", 13.003355, 1.1},      {"Cl", 34.968853, 75.77},
    {"Cl", 36.965903, 24.23},   {"Ge", 69.92425, 20.5},     {"Ge", 71.92208, 27.4},
    {"Ge", 72.923464, 7.8},     {"Ge", 73.921179, 36.5},    {"Ge", 75.921403, 7.8},
    {"Na", 22.98977, 100.0},    {"Si", 27.976928, 92.23},   {"Si", 28.976496, 4.67},
    {"Si", 29.973772, 3.1},
};

}  // namespace

// cal_g: mave = sum_i m_i f_i / 100; g = sum_i f_i (1 - m_i/mave)^2 / 100
// over the isotopes of the element.  False when the element is not covered.
bool cal_g(const std::string& name, double& g) {
  double mave = 0;
  bool found = false;
  for (const Iso& x : kIso)
    if (name == x.el) {
      mave = mave + x.m * x.f;
      found = true;
    }
  if (!found) return false;
  mave = mave / 100;
  g = 0;
  for (const Iso& x : kIso)
    if (name == x.el) g = g + x.f * (1 - (x.m / mave)) * (1 - (x.m / mave));
  g = g / 100;
  return true;
}

// cal_giso: g of every primitive atom from its type's element name
std::string cal_giso(const State& S, double* gis) {
  for (int i = 0; i < S.natoms0; ++i) {
    const int t = S.atom_type[i];
    if (t < 1 || t > (int)S.atname.size()) return "cal_giso: atom type without a name";
    double g = 0;
    if (!cal_g(S.atname[t - 1], g)) return "cal_giso: no isotope data for element " + S.atname[t - 1];
    gis[i] = g;
  }
  return "";
}

// P_iso_split for IBZ rows k1..k2: Piso(nsub, ndn), column-major.
// The reference loops n2 = 1..nkc around a body that does not use n2 (the
// sum is nkc times the body's) and divides by nkc at the end; the loop is
// folded here: Piso = omega1^2 pi/2 sum_l2 sum_tet sum_corner gs c/6, with
// gs = sum_ai g(ai) |e_ai(q1,l1)^H e_ai(w,l2)|^2 and the corner weights c of
// weight_tet at omega1 on the corner energies frequency(w, l2).
void P_iso_split(State& S, int k1, int k2, const double* g, double* Piso, int nthreads) {
  const int ndn = S.ndyn, nkc = S.nkc, nsub = k2 - k1 + 1;
  S.frequency.assign((size_t)nkc * ndn, 0.0);  // cal_freq
  for (int i = 1; i <= nkc; ++i)
    for (int ii = 1; ii <= ndn; ++ii)
      S.frequency[F2(i, ii, nkc)] = std::sqrt(S.eigenval[F2(ii, i, ndn)]) * S.K.cnst;
  parfor(0, nsub * ndn - 1, nthreads, [&](int job) {
    const int n1 = job / ndn + 1, l1 = job % ndn + 1;
    const int i = S.mapinv[n1 + k1 - 1 - 1];
    const double omega1 = S.frequency[F2(i, l1, nkc)];
    std::vector<Tetra> tet = S.tet;  // private copy of the module array
    double sum = 0;
    for (int l2 = 1; l2 <= ndn; ++l2) {
      for (auto& T : tet)
        for (int k = 0; k < 4; ++k) T.w[k] = S.frequency[F2(T.i[k], l2, nkc)];
      for (auto& T : tet) weight_tet_one(T, omega1);
      for (const auto& T : tet)
        for (int k = 0; k < 4; ++k) {
          const int w = T.i[k];
          double gs = 0;
          for (int ai = 1; ai <= S.natoms0; ++ai) {
            cplx d = 0;
            for (int x = 1; x <= 3; ++x) {
              const int c = (ai - 1) * 3 + x;
              d += std::conj(S.eigenvec[F3(c, l1, i, ndn, ndn)]) * S.eigenvec[F3(c, l2, w, ndn, ndn)];
            }
            gs = gs + g[ai - 1] * std::norm(d);
          }
          sum = sum + gs * T.c[k] / 6.0;
        }
    }
    Piso[F2(n1, l1, nsub)] = sum * omega1 * omega1 * S.K.pi / 2;
  });
}

// CollisionMatrix_iso over all IBZ rows: P1, P2 (nibz,nkc,ndn,ndn,ndn)
// Bose-weighted, Piso(nibz,ndn); CM(nibz*ndn*3, nibz*ndn*3) column-major.
// Diagonal arm (n0 = q1, l1 = l2): C = -sum(P1 + P2/2) - Piso; every other
// arm: C = sum_l3 (-P1(q0) + P1(q1+q0) + P2(q0)) + Piso(n1,l1).
void CollisionMatrix_iso(State& S, const double* P1, const double* P2, const double* Piso, double* CM,
                         int nthreads) {
  const int ndn = S.ndyn, nkc = S.nkc, nibz = S.nibz;
  const int n = nibz * ndn * 3;
  std::fill(CM, CM + (size_t)n * n, 0.0);
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
  parfor(0, nibz * ndn - 1, nthreads, [&](int job) {
    const int n1 = job / ndn + 1, l1 = job % ndn + 1;
    const int n1i = S.mapinv[n1 - 1];
    const int d1 = 3 * ((n1 - 1) * ndn + (l1 - 1)) + 1;
    for (int n2 = 1; n2 <= nibz; ++n2)
      for (int l2 = 1; l2 <= ndn; ++l2) {
        const int d2 = 3 * ((n2 - 1) * ndn + (l2 - 1)) + 1;
        for (int ns = 1; ns <= narms[n2 - 1]; ++ns) {
          const double* arm = &armq[((size_t)(n2 - 1) * 48 + ns - 1) * 3];
          const int op = armop[(size_t)(n2 - 1) * 48 + ns - 1];
          int n0, a1, a2, a3, ins;
          get_k_info(S, arm, n0, a1, a2, a3, ins);
          double C = 0;
          if (n1i == n0 && l1 == l2) {
            for (int nl2 = 1; nl2 <= ndn; ++nl2)
              for (int l3 = 1; l3 <= ndn; ++l3)
                for (int n22 = 1; n22 <= nkc; ++n22) {
                  const size_t idx = F5(n1, n22, l1, nl2, l3, nibz, nkc, ndn, ndn);
                  C = C + (-P1[idx] - 0.5 * P2[idx]);
                }
            C = C - Piso[F2(n1, l1, nibz)];
          } else {
            const double q1[3] = {S.kibz[F2(1, n1, 3)], S.kibz[F2(2, n1, 3)], S.kibz[F2(3, n1, 3)]};
            double qp[3];
            for (int c = 0; c < 3; ++c) qp[c] = q1[c] + arm[c];
            int nk3_p1;
            get_k_info(S, qp, nk3_p1, a1, a2, a3, ins);
            for (int nl3 = 1; nl3 <= ndn; ++nl3)
              C = C + (-P1[F5(n1, n0, l1, l2, nl3, nibz, nkc, ndn, ndn)] +
                       P1[F5(n1, nk3_p1, l1, l2, nl3, nibz, nkc, ndn, ndn)] +
                       P2[F5(n1, n0, l1, l2, nl3, nibz, nkc, ndn, ndn)]);
            C = C + Piso[F2(n1, l1, nibz)];
          }
          const double* opm = S.op_kmatrix[op - 1];
          for (int i = 1; i <= 3; ++i)
            for (int j = 1; j <= 3; ++j) {
              const size_t e = (size_t)(d1 + i - 1 - 1) + (size_t)n * (d2 + j - 1 - 1);
              CM[e] = CM[e] + (C * opm[F2(i, j, 3)]);
            }
        }
      }
  });
}

}  // namespace orc
