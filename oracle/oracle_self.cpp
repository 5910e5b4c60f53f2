// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle_core.h).  PARITY UNPINNED:
// no shipped reference output covers the three-phonon self-energy.
//
// Three-phonon self-energy along the band path (THERMACOND job=2):
//   make_kp_bs            THERMACOND/modules.f90:1507-1652 (kpbs.params -> kp_bs, dk_bs)
//   get_direct_components THERMACOND/extratools.f90:561-592
//   check_inside_bz       THERMACOND/extratools.f90:325-341
//   matrix_elt_full       THERMACOND/rest.f90:3664-3719
//   function_self_w3      THERMACOND/rest.f90:4012-4124 (Lorentzian, four terms, real and imaginary)
//   function_self_w4      THERMACOND/rest.f90:4126-4240 (Gaussian, three terms, imaginary only)
//   delta_g, delta_l      THERMACOND/extratools.f90:239-255
//   the job=2 block       THERMACOND/kappa.f90:874-1040 (omega0, isempi, tsempi per path mode)
#include <cmath>
#include <cstdio>
#include <string>

#include "oracle_core.h"

namespace orc {

namespace {

double dot_a(const double* v, const double* w) {  // dotproduct_a: sum(v*w)
  double s = 0;
  for (int i = 0; i < 3; ++i) s = s + v[i] * w[i];
  return s;
}

double delta_l(double x, double w, double pi) { return w / (x * x + w * w) / pi; }

double delta_g(double x, double w, double pi) { return std::exp(-x * x / 2.0 / w / w) / std::sqrt(2 * pi) / w; }

// CMPLX(x, y) without KIND is default COMPLEX: both parts rounded to REAL(4)
double to_real4(double x) { return (double)(float)x; }

}  // namespace

// make_kp_bs: the band path of kpbs.params (units, nkdir, ndir, then ndir+1
// lines "name kx ky kz"; units 0 = conventional reciprocal, else primitive)
std::string make_kp_bs(const State& S, const std::string& dir, std::vector<double>& kp_bs,
                       std::vector<double>& dk_bs) {
  // stdio only: the oracle is loaded next to other C++ runtimes (no iostreams)
  FILE* f = std::fopen((dir + "/kpbs.params").c_str(), "r");
  if (!f) return "MAKE_KP_BS: kpbs.params does not exist";
  std::vector<std::string> lines;
  char buf[1024];
  while (std::fgets(buf, sizeof buf, f)) {
    for (char* c = buf; *c; ++c)
      if (*c == ',') *c = ' ';
    lines.emplace_back(buf);
  }
  std::fclose(f);
  int units = 0, nkdir = 0, ndir = 0;
  if (lines.size() < 3 || std::sscanf(lines[0].c_str(), "%d", &units) != 1 ||
      std::sscanf(lines[1].c_str(), "%d", &nkdir) != 1 || std::sscanf(lines[2].c_str(), "%d", &ndir) != 1)
    return "MAKE_KP_BS: units, nkdir, ndir";
  if (nkdir < 1 || ndir < 1) return "MAKE_KP_BS: nkdir and ndir must be positive";
  if ((int)lines.size() < 3 + ndir + 1) return "MAKE_KP_BS: missing k-point lines";
  std::vector<double> kext((size_t)3 * (ndir + 1));
  for (int i = 0; i < ndir + 1; ++i) {
    char name[256];
    if (std::sscanf(lines[3 + i].c_str(), "%255s %lf %lf %lf", name, &kext[3 * i], &kext[3 * i + 1],
                    &kext[3 * i + 2]) != 4)
      return "MAKE_KP_BS: bad k-point line";
  }
  const double *b1 = units == 0 ? S.g1conv : S.g1, *b2 = units == 0 ? S.g2conv : S.g2,
               *b3 = units == 0 ? S.g3conv : S.g3;
  std::vector<double> ki((size_t)3 * ndir), kf((size_t)3 * ndir);
  for (int i = 0; i < ndir; ++i)
    for (int c = 0; c < 3; ++c) {
      const double* a = &kext[3 * i];
      const double* e = &kext[3 * (i + 1)];
      ki[3 * i + c] = a[0] * b1[c] + a[1] * b2[c] + a[2] * b3[c];
      kf[3 * i + c] = e[0] * b1[c] + e[1] * b2[c] + e[2] * b3[c];
    }
  const int nkp = ndir * nkdir;
  kp_bs.assign((size_t)3 * nkp, 0.0);
  dk_bs.assign(nkp, 0.0);
  int nk = 0;
  for (int i = 0; i < ndir; ++i) {
    double q[3];
    for (int c = 0; c < 3; ++c) q[c] = kf[3 * i + c] - ki[3 * i + c];
    double lk = 0;
    for (int c = 0; c < 3; ++c) lk = lk + q[c] * q[c];  // lengtha
    lk = std::sqrt(lk);
    for (int j = 1; j <= nkdir; ++j) {
      nk = nk + 1;
      if (nk >= 2)
        dk_bs[nk - 1] = j >= 2 ? dk_bs[nk - 2] + lk / (nkdir - 1 + 1e-8) : dk_bs[nk - 2];
      else
        dk_bs[nk - 1] = 0;
      for (int c = 0; c < 3; ++c) kp_bs[3 * (nk - 1) + c] = ki[3 * i + c] + (j - 1) * q[c] / (nkdir - 1 + 1e-8);
    }
  }
  return "";
}

// check_inside_bz: 1 when q + (g1+g2+g3)/2 has direct components in [0,1)
int check_inside_bz(const State& S, const double q[3]) {
  double q2[3];
  for (int c = 0; c < 3; ++c) q2[c] = q[c] + 0.5 * ((S.g1[c] + S.g2[c]) + S.g3[c]);
  RecipNo2pi r = make_reciprocal_lattice(S.g1, S.g2, S.g3);
  const double epsl = 5e-10;
  int inside = 1;
  const double* rr[3] = {r.rr1, r.rr2, r.rr3};
  for (int a = 0; a < 3; ++a) {
    const double x = (q2[0] * rr[a][0] + q2[1] * rr[a][1] + q2[2] * rr[a][2]) + epsl;
    if (x < 0 || x >= 1) inside = 0;
  }
  return inside;
}

// matrix_elt_full: w33 for modes with eigenvectors evq, ev2, ev3 at q, q2, q3
// (no conjugation), frequencies omq, om2, om3 in cm^-1.  Returns false on den == 0.
bool matrix_elt_full(const State& S, const double* q2, const double* q3, double omq, double om2, double om3,
                     const cplx* evq, const cplx* ev2, const cplx* ev3, cplx& w33) {
  cplx xx = 0;
  for (int t = 0; t < S.nterms[2]; ++t) {
    const int i3 = S.iatomterm_3[3 * t];
    const int i0 = S.iatomcell0[i3 - 1];
    if (i0 != i3) continue;
    const int al = S.ixyzterm_3[3 * t], be = S.ixyzterm_3[3 * t + 1], ga = S.ixyzterm_3[3 * t + 2];
    const double mi = S.mass0[i0 - 1];
    const int j1 = S.iatomterm_3[3 * t + 1], j0 = S.iatomcell0[j1 - 1];
    const int k1 = S.iatomterm_3[3 * t + 2], k0 = S.iatomcell0[k1 - 1];
    const double mj = S.mass0[j0 - 1], mk = S.mass0[k0 - 1];
    const int ta1 = al + 3 * (i0 - 1), ta2 = be + 3 * (j0 - 1), ta3 = ga + 3 * (k0 - 1);
    double rr2[3], rr3[3];
    for (int c = 0; c < 3; ++c) {
      rr2[c] = S.atompos[F2(c + 1, j1, 3)] - S.atompos[F2(c + 1, j0, 3)];
      rr3[c] = S.atompos[F2(c + 1, k1, 3)] - S.atompos[F2(c + 1, k0, 3)];
    }
    const double x = dot_a(q2, rr2) + dot_a(q3, rr3);
    const cplx eiqr(std::cos(x), std::sin(x));
    xx = xx + cmul(cmul(cmul(S.fcs_3[t] / std::sqrt(mi * mj * mk) * eiqr, evq[ta1 - 1]), ev2[ta2 - 1]),
                   ev3[ta3 - 1]);
  }
  const double cn = S.K.cnst;
  const double den = std::sqrt(8 * omq * om2 * om3 / (cn * cn * cn));
  if (den == 0) return false;
  w33 = xx / den * S.K.const33;
  return true;
}

// function_self_w3 (gauss = false) / function_self_w4 (gauss = true) at an
// arbitrary q for mode la (1-based), frequency omega and temperature temp
// (both cm^-1).  Uses the mesh eigenpairs of S (eigenval, eigenvec).
// Returns 0, or an error (1 nbe, 2 den = 0).
int function_self_w(const State& S, const double q[3], int la, double omega, double temp, bool gauss,
                    cplx& nself, cplx& uself) {
  const int n = S.ndyn;
  const double pi = S.K.pi, cn = S.K.cnst;
  std::vector<double> eivq(n), eiv3(n);
  std::vector<cplx> evq((size_t)n * n), ev3((size_t)n * n);
  get_freq(S, q, eivq.data(), evq.data());
  const double omq = std::sqrt(std::fabs(eivq[la - 1])) * cn;
  const double eta = S.etaz;
  const double etacut = gauss ? eta * 6 : eta * 3000;
  const double v3_threshold = (double)1e-7f;  // rest.f90:47, a default-REAL literal
  nself = 0;
  uself = 0;
  int err = 0;
  for (int ik = 1; ik <= S.nkc; ++ik) {
    const double* k2 = &S.kpc[F2(1, ik, 3)];
    double k3[3];
    for (int c = 0; c < 3; ++c) k3[c] = -q[c] - k2[c];
    const int inside = check_inside_bz(S, k3);
    get_freq(S, k3, eiv3.data(), ev3.data());
    for (int l2 = 1; l2 <= n; ++l2) {
      const double om2 = std::sqrt(std::fabs(S.eigenval[F2(l2, ik, n)])) * cn;
      const double nb2 = nbe(om2, temp, S.classical, &err);
      for (int l3 = 1; l3 <= n; ++l3) {
        const double om3 = std::sqrt(std::fabs(eiv3[l3 - 1])) * cn;
        const double nb3 = nbe(om3, temp, S.classical, &err);
        double ires = 0, rres = 0, arg;
        if (!gauss) {
          arg = omega - om3 - om2;
          if (std::fabs(arg) < etacut) {
            ires = (nb3 + nb2 + 1) * delta_l(arg, eta, pi);
            rres = (nb3 + nb2 + 1) * arg / (arg * arg + eta * eta);
          }
          arg = omega + om3 + om2;
          if (std::fabs(arg) < etacut) {
            ires = ires - (nb3 + nb2 + 1) * delta_l(arg, eta, pi);
            rres = rres - (nb3 + nb2 + 1) * arg / (arg * arg + eta * eta);
          }
          arg = omega - om3 + om2;
          if (std::fabs(arg) < etacut) {
            ires = ires + (nb2 - nb3) * delta_l(arg, eta, pi);
            rres = rres + (nb2 - nb3) * arg / (arg * arg + eta * eta);
          }
          arg = omega - om2 + om3;
          if (std::fabs(arg) < etacut) {
            ires = ires + (nb3 - nb2) * delta_l(arg, eta, pi);
            rres = rres + (nb3 - nb2) * arg / (arg * arg + eta * eta);
          }
        } else {
          arg = omega - om3 - om2;
          if (std::fabs(arg) < etacut) ires = (nb3 + nb2 + 1) * delta_g(arg, eta, pi);
          arg = omega - om3 + om2;
          if (std::fabs(arg) < etacut) ires = ires + (nb2 - nb3) * delta_g(arg, eta, pi);
          arg = omega - om2 + om3;
          if (std::fabs(arg) < etacut) ires = ires + (nb3 - nb2) * delta_g(arg, eta, pi);
        }
        const cplx self(to_real4(rres), to_real4(ires * pi));
        cplx xx;
        if (!matrix_elt_full(S, k2, k3, omq, om2, om3, &evq[F2(1, la, n)], &S.eigenvec[F3(1, l2, ik, n, n)],
                             &ev3[F2(1, l3, n)], xx))
          return 2;
        if (std::abs(xx) < v3_threshold) continue;
        const double term = (xx * std::conj(xx)).real();
        if (inside == 1)
          nself = nself + term * self;
        else
          uself = uself + term * self;
      }
    }
  }
  nself = nself / (double)S.nkc * pi;
  uself = uself / (double)S.nkc * pi;
  return err ? 1 : 0;
}

// get_frequencies on a list of points: eigenvalues (|lambda|, sorted) and
// eigenvectors, as kappa_full's job=2 block takes them for the path
void frequencies_at(const State& S, int np, const double* kp, double* eival, cplx* eivec, int nthreads) {
  const int n = S.ndyn;
  parfor(0, np - 1, nthreads, [&](int p) {
    std::vector<double> eivl(n), vgr((size_t)3 * n);
    std::vector<cplx> eivc((size_t)n * n);
    std::vector<int> mp(n);
    finitedif_vel(S, &kp[3 * p], vgr.data(), eivl.data(), eivc.data());
    fsort(n, eivl.data(), mp.data());
    for (int j = 1; j <= n; ++j) {
      eival[(size_t)p * n + j - 1] = eivl[mp[j - 1] - 1];
      for (int l = 1; l <= n; ++l) eivec[(size_t)p * n * n + F2(l, j, n)] = eivc[F2(l, mp[j - 1], n)];
    }
  });
}

}  // namespace orc
