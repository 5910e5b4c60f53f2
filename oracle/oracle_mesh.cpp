// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle_core.h).
// Mesh, IBZ, dynamical matrix, eigen-decomposition and group velocities:
//   make_kp_reg            THERMACOND/modules.f90:1721-1784
//   get_k_info             THERMACOND/rest.f90:3024-3058
//   comp1/get_components_g(2)/indexg  THERMACOND/extratools.f90:491-500,592-666
//   make_reciprocal_lattice THERMACOND/extratools.f90:188-207
//   get_negatives          THERMACOND/rest.f90:3208-3260
//   getstar                THERMACOND/force_constants.f90:1748-1784
//   get_weights            THERMACOND/modules.f90:2006-2160
//   set_dynamical_matrix   THERMACOND/rest.f90:445-556
//   diagonalize            THERMACOND/rest.f90:558-598 (ZHEEV, zhegv.f:213)
//   get_freq               THERMACOND/rest.f90:4319-4445
//   finitedif_vel          THERMACOND/rest.f90:2587-2630
//   get_frequencies        THERMACOND/rest.f90:2230-2398
//   subst_eivecs           THERMACOND/rest.f90:3262-3293
//   sort                   THERMACOND/extratools.f90:154-175
//   make_kp_reg_tet        THERMACOND/tetrahedron.f90:2-142
#include <algorithm>
#include <cstring>

#include "oracle_core.h"

namespace orc {

namespace {
inline double dot3(const double* v, const double* w) {  // dotproduct_av (modules.f90:133)
  return v[0] * w[0] + v[1] * w[1] + v[2] * w[2];
}
}  // namespace

RecipNo2pi make_reciprocal_lattice(const double* g1, const double* g2, const double* g3) {
  auto cross = [](const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
  };
  double c23[3], c31[3], c12[3];
  cross(g2, g3, c23);
  cross(g3, g1, c31);
  cross(g1, g2, c12);
  double om = c23[0] * g1[0] + c23[1] * g1[1] + c23[2] * g1[2];
  RecipNo2pi r;
  for (int i = 0; i < 3; ++i) {
    r.rr1[i] = c23[i] / om;
    r.rr2[i] = c31[i] / om;
    r.rr3[i] = c12[i] / om;
  }
  return r;
}

void comp1(const double* q, const double* rr, int n, int& i, int& insid) {
  const double epsl = 5e-10;
  double qdr = dot3(q, rr) + epsl;
  if (qdr < 0 || qdr >= 1) insid = 0;
  double aux = qdr - std::floor(qdr);
  double y = (1 + n * aux);
  i = (int)std::lround(y);
  if (std::fabs(i - y) > 0.01) insid = 2;
  if (i == n + 1) i = 1;
}

// sort (extratools.f90:154-175): ascending, r(mcor(i)) ordered
void fsort(int n, const double* r, int* mcor) {
  for (int i = 1; i <= n; ++i) mcor[i - 1] = i;
  for (int i = 1; i <= n; ++i)
    for (int j = i + 1; j <= n; ++j)
      if (r[mcor[i - 1] - 1] > r[mcor[j - 1] - 1]) std::swap(mcor[i - 1], mcor[j - 1]);
}

void set_k_dual(State& S) {
  RecipNo2pi r = make_reciprocal_lattice(S.g1, S.g2, S.g3);
  for (int c = 0; c < 3; ++c) {
    S.gd1[c] = r.rr1[c];
    S.gd2[c] = r.rr2[c];
    S.gd3[c] = r.rr3[c];
  }
}

void get_k_info(const State& S, const double q[3], int& nk, int& i, int& j, int& k, int& inside) {
  const int* N = S.nc;
  double w[3];
  if (N[0] % 2 == 0 && N[1] % 2 == 0 && N[2] % 2 == 0) {
    // get_components_g2: w = q + 0.5*(g1+g2+g3)
    for (int c = 0; c < 3; ++c) w[c] = q[c] + 0.5 * ((S.g1[c] + S.g2[c]) + S.g3[c]);
  } else {
    for (int c = 0; c < 3; ++c) w[c] = q[c];
  }
  inside = 1;
  comp1(w, S.gd1, N[0], i, inside);
  comp1(w, S.gd2, N[1], j, inside);
  comp1(w, S.gd3, N[2], k, inside);
  nk = k + (j - 1) * N[2] + (i - 1) * N[1] * N[2];  // indexg(i,j,k,1,N1,1,N2,1,N3)
}

void make_kp_reg(State& S) {
  const int* nc = S.nc;
  S.kpc.assign(3 * S.nkc, 0.0);
  double sh[3];
  for (int c = 0; c < 3; ++c) sh[c] = (-0.5) * ((S.g1[c] + S.g2[c]) + S.g3[c]);
  int nk = 0;
  for (int i = 1; i <= nc[0]; ++i)
    for (int j = 1; j <= nc[1]; ++j)
      for (int k = 1; k <= nc[2]; ++k) {
        nk = nk + 1;
        // float(i-1)/nc(1) is a default-real (FP32) quotient
        double f1 = (double)((float)(i - 1) / (float)nc[0]);
        double f2 = (double)((float)(j - 1) / (float)nc[1]);
        double f3 = (double)((float)(k - 1) / (float)nc[2]);
        for (int c = 0; c < 3; ++c) S.kpc[F2(c + 1, nk, 3)] = ((f1 * S.g1[c] + f2 * S.g2[c]) + f3 * S.g3[c]) + 0.0;
      }
  if (nc[0] % 2 == 0 && nc[1] % 2 == 0 && nc[2] % 2 == 0)
    for (int i = 1; i <= nk; ++i)
      for (int c = 0; c < 3; ++c) S.kpc[F2(c + 1, i, 3)] = S.kpc[F2(c + 1, i, 3)] + sh[c];
}

void get_negatives(State& S) {
  int nk = S.nkc;
  S.mappos.assign(nk, 0);
  int nps = 0;
  for (int i = 1; i <= nk; ++i) {
    int k, i1, j1, k1, inside;
    get_k_info(S, &S.kpc[F2(1, i, 3)], k, i1, j1, k1, inside);
    double mq[3] = {-S.kpc[F2(1, i, 3)], -S.kpc[F2(2, i, 3)], -S.kpc[F2(3, i, 3)]};
    int mk;
    get_k_info(S, mq, mk, i1, j1, k1, inside);
    if (mk < i) continue;
    nps = nps + 1;
    S.mappos[nps - 1] = i;
  }
  int cnt = nps;
  std::vector<char> inlist(nk + 1, 0);
  for (int a = 0; a < nps; ++a) inlist[S.mappos[a]] = 1;
  for (int i = 1; i <= nk; ++i)
    if (!inlist[i]) {
      cnt = cnt + 1;
      S.mappos[cnt - 1] = i;
    }
  S.npos = nps;
}

void getstar(const State& S, const double kvec[3], int& narms, double kvecstar[][3], int kvecop[]) {
  double kvecstarp[48][3];
  narms = 0;
  for (int i = 1; i <= S.lattpgcount; ++i) {
    const double* op = S.op_kmatrix[i - 1];
    double v[3], v2[3];
    for (int a = 1; a <= 3; ++a) {  // xvmlt
      double s = 0;
      for (int b = 1; b <= 3; ++b) s = s + op[F2(a, b, 3)] * kvec[b - 1];
      v[a - 1] = s;
    }
    for (int a = 1; a <= 3; ++a) {  // xmatmlt(v,primlatt,v2,1,3,3,1,3,1)
      double s = 0;
      for (int k = 1; k <= 3; ++k) s = s + v[k - 1] * S.primitivelattice[F2(k, a, 3)];
      v2[a - 1] = s;
    }
    bool skip = false;
    for (int j = 1; j <= narms && !skip; ++j) {
      for (int k = 1; k <= 3; ++k) {
        double v3 = v2[k - 1] - kvecstarp[j - 1][k - 1];
        long n = std::lround(v3);
        if (std::fabs(v3 - n) > 1e-6) break;
        if (k == 3) skip = true;
      }
    }
    if (skip) continue;
    narms = narms + 1;
    for (int c = 0; c < 3; ++c) {
      kvecstar[narms - 1][c] = v[c];
      kvecstarp[narms - 1][c] = v2[c];
    }
    kvecop[narms - 1] = i;
  }
}

void get_weights(State& S) {
  int nk = S.nkc;
  std::vector<double> k2(3 * nk), w2(nk, 1.0);
  S.mapibz.assign(nk, 0);
  S.mapinv.assign(nk, 0);
  int nibz = 0;
  for (int i = 1; i <= nk; ++i) {
    int narms, kvecop[48];
    double kvecstar[48][3];
    getstar(S, &S.kpc[F2(1, i, 3)], narms, kvecstar, kvecop);
    bool exists = false;
    for (int l = 1; l <= narms && !exists; ++l) {
      for (int j = 1; j <= nibz; ++j) {
        double d[3];
        for (int c = 0; c < 3; ++c) d[c] = k2[F2(c + 1, j, 3)] - kvecstar[l - 1][c];
        double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (len < 1e-4) {
          exists = true;
          w2[j - 1] = w2[j - 1] + 1.0;
          S.mapibz[i - 1] = j;
          break;
        }
      }
    }
    if (exists) continue;
    nibz = nibz + 1;
    if (nibz == 1) w2[nibz - 1] = 1;
    S.mapibz[i - 1] = nibz;
    S.mapinv[nibz - 1] = i;
    for (int c = 0; c < 3; ++c) k2[F2(c + 1, nibz, 3)] = S.kpc[F2(c + 1, i, 3)];
  }
  S.nibz = nibz;
  S.kibz.assign(k2.begin(), k2.begin() + 3 * nibz);
  S.wibz.assign(w2.begin(), w2.begin() + nibz);
  double sw = 0;
  for (int j = 0; j < nibz; ++j) sw = sw + S.wibz[j];
  for (int j = 0; j < nibz; ++j) S.wibz[j] = S.wibz[j] / sw;
}

void set_dynamical_matrix(const State& S, const double kpt[3], cplx* dynmat) {
  int ndim = S.ndyn;
  for (int e = 0; e < ndim * ndim; ++e) dynmat[e] = cplx(0, 0);
  int nt2 = S.nterms[1];
  for (int i0 = 1; i0 <= S.natoms0; ++i0)
    for (int al = 1; al <= 3; ++al) {
      int i3 = al + 3 * (i0 - 1);
      double mi = S.mass0[i0 - 1];
      for (int t = 1; t <= nt2; ++t) {
        if (i0 == S.iatomterm_2[0 + 2 * (t - 1)] && al == S.ixyzterm_2[0 + 2 * (t - 1)]) {
          int be = S.ixyzterm_2[1 + 2 * (t - 1)];
          int j = S.iatomterm_2[1 + 2 * (t - 1)];
          int j0 = S.iatomcell0[j - 1];
          double mj = S.mass0[j0 - 1];
          int j3 = be + 3 * (j0 - 1);
          double rr[3];
          for (int c = 0; c < 3; ++c) rr[c] = S.atompos[F2(c + 1, j, 3)] - S.atompos[F2(c + 1, j0, 3)];
          double x = kpt[0] * rr[0] + kpt[1] * rr[1] + kpt[2] * rr[2];
          cplx ph(std::cos(x), std::sin(x));
          cplx junk = cplx(S.fcs_2[t - 1] * ph.real(), S.fcs_2[t - 1] * ph.imag());
          double sq = std::sqrt(mi * mj);
          junk = cplx(junk.real() / sq, junk.imag() / sq);
          dynmat[F2(i3, j3, ndim)] += junk;
        }
      }
    }
  // make it hermitian (rest.f90:513-544); note the j loop stops at ndim-1
  for (int t = 1; t <= ndim; ++t) {
    cplx d = dynmat[F2(t, t, ndim)];
    if (std::fabs(d.imag()) > 9e-4 * std::fabs(d.real())) dynmat[F2(t, t, ndim)] = cplx(d.real(), 0.0);
    for (int j = t + 1; j <= ndim - 1; ++j) {
      cplx a = dynmat[F2(t, j, ndim)], b = dynmat[F2(j, t, ndim)];
      double mi = (a.imag() - b.imag()) / 2;
      double mj = (a.real() + b.real()) / 2;
      dynmat[F2(t, j, ndim)] = cplx(mj, mi);
      dynmat[F2(j, t, ndim)] = cplx(mj, -mi);
    }
  }
  double sim = 0, sre = 0;
  for (int e = 0; e < ndim * ndim; ++e) {
    sim += std::fabs(dynmat[e].imag());
    sre += std::fabs(dynmat[e].real());
  }
  sim = sim / (ndim * ndim);
  sre = sre / (ndim * ndim);
  if (sim < sre * 1e-10)
    for (int e = 0; e < ndim * ndim; ++e) dynmat[e] = cplx(dynmat[e].real(), 0.0);
}

// Hermitian eigen-decomposition of the matrix whose upper triangle is given
// (ZHEEV('V','U') reads only the upper triangle and the real diagonal).
// Cyclic complex Jacobi in FP64; eigenvalues returned in the order the
// sweeps leave them (the caller sorts).  Eigenvector bases inside exactly
// degenerate subspaces are arbitrary, as they are for ZHEEV.
void hermitian_eigen(int n, const cplx* upper, double* eival, cplx* eivec) {
  std::vector<cplx> A(n * n);
  for (int i = 1; i <= n; ++i)
    for (int j = 1; j <= n; ++j) {
      if (i == j)
        A[F2(i, i, n)] = cplx(upper[F2(i, i, n)].real(), 0);
      else if (i < j)
        A[F2(i, j, n)] = upper[F2(i, j, n)];
      else
        A[F2(i, j, n)] = std::conj(upper[F2(j, i, n)]);
    }
  for (int e = 0; e < n * n; ++e) eivec[e] = 0;
  for (int i = 1; i <= n; ++i) eivec[F2(i, i, n)] = 1;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0, dia = 0;
    for (int i = 1; i <= n; ++i)
      for (int j = 1; j <= n; ++j) {
        if (i != j)
          off += std::norm(A[F2(i, j, n)]);
        else
          dia += std::norm(A[F2(i, i, n)]);
      }
    if (off == 0.0 || off <= 1e-34 * dia) break;
    for (int p = 1; p < n; ++p)
      for (int q = p + 1; q <= n; ++q) {
        cplx apq = A[F2(p, q, n)];
        double b = std::abs(apq);
        if (b == 0.0) continue;
        double app = A[F2(p, p, n)].real(), aqq = A[F2(q, q, n)].real();
        if (sweep > 4 && std::fabs(app) + 1e3 * b == std::fabs(app) && std::fabs(aqq) + 1e3 * b == std::fabs(aqq)) {
          A[F2(p, q, n)] = 0;
          A[F2(q, p, n)] = 0;
          continue;
        }
        cplx w = apq / b;            // apq = b*w
        double theta = (aqq - app) / (2 * b);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        cplx wc = std::conj(w);
        // V = [[c, s], [-s*conj(w), c*conj(w)]] on (p,q)
        for (int k = 1; k <= n; ++k) {
          if (k == p || k == q) continue;
          cplx akp = A[F2(k, p, n)], akq = A[F2(k, q, n)];
          cplx nkp = c * akp - s * wc * akq;
          cplx nkq = s * akp + c * wc * akq;
          A[F2(k, p, n)] = nkp;
          A[F2(p, k, n)] = std::conj(nkp);
          A[F2(k, q, n)] = nkq;
          A[F2(q, k, n)] = std::conj(nkq);
        }
        A[F2(p, p, n)] = app - t * b;
        A[F2(q, q, n)] = aqq + t * b;
        A[F2(p, q, n)] = 0;
        A[F2(q, p, n)] = 0;
        for (int k = 1; k <= n; ++k) {
          cplx ekp = eivec[F2(k, p, n)], ekq = eivec[F2(k, q, n)];
          eivec[F2(k, p, n)] = c * ekp - s * wc * ekq;
          eivec[F2(k, q, n)] = s * ekp + c * wc * ekq;
        }
      }
  }
  for (int i = 1; i <= n; ++i) eival[i - 1] = A[F2(i, i, n)].real();
}

// nonanal (rest.f90:3517-3578): dipole term added after hermitisation when
// born_flag /= 0; q = 0 is replaced by q + 1d-10 by the caller (get_freq)
static void nonanal(const State& S, const double q[3], cplx* dynmat) {
  const Consts& K = S.K;
  int ndim = S.ndyn;
  double eps_scale = 8.8541878176e-12 / 1e10 / K.ee;
  auto len = [](const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
  double gg = std::pow(len(S.g1) * len(S.g2) * len(S.g3), (double)0.33f);
  double rho = gg / 4.0;
  double rho2 = rho * rho;
  double c12[3] = {S.r1[1] * S.r2[2] - S.r1[2] * S.r2[1], S.r1[2] * S.r2[0] - S.r1[0] * S.r2[2],
                   S.r1[0] * S.r2[1] - S.r1[1] * S.r2[0]};
  double om0 = std::fabs(S.r3[0] * c12[0] + S.r3[1] * c12[1] + S.r3[2] * c12[2]);
  auto E = [&](int i, int j) { return S.epsil[F2(i, j, 3)]; };
  double qeq = (q[0] * (E(1, 1) * q[0] + E(1, 2) * q[1] + E(1, 3) * q[2]) +
                q[1] * (E(2, 1) * q[0] + E(2, 2) * q[1] + E(2, 3) * q[2]) +
                q[2] * (E(3, 1) * q[0] + E(3, 2) * q[1] + E(3, 3) * q[2]));
  double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
  for (int na = 1; na <= S.natoms0; ++na) {
    double ma = S.mass0[na - 1];
    for (int nb = 1; nb <= S.natoms0; ++nb) {
      double mb = S.mass0[nb - 1];
      double zag[3], zbg[3];
      for (int i = 1; i <= 3; ++i) {
        zag[i - 1] = q[0] * S.charge[F3(1, i, na, 3, 3)] + q[1] * S.charge[F3(2, i, na, 3, 3)] +
                     q[2] * S.charge[F3(3, i, na, 3, 3)];
        zbg[i - 1] = q[0] * S.charge[F3(1, i, nb, 3, 3)] + q[1] * S.charge[F3(2, i, nb, 3, 3)] +
                     q[2] * S.charge[F3(3, i, nb, 3, 3)];
      }
      for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j)
          dynmat[F2(i + 3 * (na - 1), j + 3 * (nb - 1), ndim)] +=
              zag[i - 1] * zbg[j - 1] / (qeq * eps_scale) / om0 / std::sqrt(ma * mb) * std::exp(-q2 / rho2);
    }
  }
}

void get_freq(const State& S, const double kp[3], double* eival, cplx* eivec) {
  int n = S.ndyn;
  std::vector<cplx> dyn(n * n), evc(n * n);
  std::vector<double> eivl(n);
  std::vector<int> mp(n);
  set_dynamical_matrix(S, kp, dyn.data());
  if (S.born_flag != 0) {
    double khat[3] = {kp[0], kp[1], kp[2]};
    if (kp[0] == 0.0 && kp[1] == 0.0 && kp[2] == 0.0)
      for (int c = 0; c < 3; ++c) khat[c] = kp[c] + 1.0e-10;
    nonanal(S, khat, dyn.data());
  }
  hermitian_eigen(n, dyn.data(), eivl.data(), evc.data());
  // ZHEEV returns ascending eigenvalues; order the Jacobi output the same way
  // (stable on ties), then apply the reference's own sort
  {
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return eivl[a] < eivl[b]; });
    std::vector<double> l2(n);
    std::vector<cplx> e2(n * n);
    for (int j = 0; j < n; ++j) {
      l2[j] = eivl[ord[j]];
      for (int l = 0; l < n; ++l) e2[l + n * j] = evc[l + n * ord[j]];
    }
    eivl = l2;
    evc = e2;
  }
  fsort(n, eivl.data(), mp.data());
  for (int j = 1; j <= n; ++j) {
    eival[j - 1] = std::fabs(eivl[mp[j - 1] - 1]);
    for (int l = 1; l <= n; ++l) eivec[F2(l, j, n)] = evc[F2(l, mp[j - 1], n)];
  }
  for (int l = 1; l <= n; ++l) {
    double absvec = 0;
    for (int k = 1; k <= n; ++k) absvec += std::fabs(eivec[F2(k, l, n)].real());
    if (absvec < 1e-3)
      for (int k = 1; k <= n; ++k) eivec[F2(k, l, n)] = cmul(cplx(0, 1), eivec[F2(k, l, n)]);
  }
}

void finitedif_vel(const State& S, const double q0[3], double* vgr, double* evl0, cplx* evc0) {
  int n = S.ndyn;
  const double dq = (double)0.001f;
  std::vector<double> evlp(n), evlm(n);
  std::vector<cplx> evct(n * n);
  get_freq(S, q0, evl0, evc0);
  for (int i = 1; i <= 3; ++i) {
    double q1[3] = {q0[0], q0[1], q0[2]};
    q1[i - 1] = q0[i - 1] + dq;
    get_freq(S, q1, evlp.data(), evct.data());
    q1[i - 1] = q0[i - 1] - dq;
    get_freq(S, q1, evlm.data(), evct.data());
    for (int l = 1; l <= n; ++l)
      vgr[F2(i, l, 3)] =
          (evlp[l - 1] - evlm[l - 1]) / 2 / dq / 2 / std::sqrt(evl0[l - 1]) * S.K.cnst * 1e-8 * 2 * S.K.pi;
  }
}

void get_frequencies(State& S, int nthreads) {
  int n = S.ndyn, nk = S.nkc;
  S.eigenval.assign((size_t)n * nk, 0.0);
  S.eigenvec.assign((size_t)n * n * nk, cplx(0, 0));
  S.veloc.assign((size_t)3 * n * nk, 0.0);
  parfor(1, nk, nthreads, [&](int i) {
    std::vector<double> eivl(n);
    std::vector<cplx> eivc(n * n);
    std::vector<int> mp(n);
    finitedif_vel(S, &S.kpc[F2(1, i, 3)], &S.veloc[F3(1, 1, i, 3, n)], eivl.data(), eivc.data());
    fsort(n, eivl.data(), mp.data());
    for (int j = 1; j <= n; ++j) {
      S.eigenval[F2(j, i, n)] = eivl[mp[j - 1] - 1];
      for (int l = 1; l <= n; ++l) S.eigenvec[F3(j, l, i, n, n)] = eivc[F2(j, mp[l - 1], n)];
    }
  });
}

void subst_eivecs(State& S) {
  int n = S.ndyn;
  for (int m = S.npos + 1; m <= S.nkc; ++m) {
    int n3 = S.mappos[m - 1];
    double mq[3] = {-S.kpc[F2(1, n3, 3)], -S.kpc[F2(2, n3, 3)], -S.kpc[F2(3, n3, 3)]};
    int mk3, i1, j1, k1, inside;
    get_k_info(S, mq, mk3, i1, j1, k1, inside);
    for (int la = 1; la <= n; ++la)
      for (int mu = 1; mu <= n; ++mu)
        S.eigenvec[F3(mu, la, mk3, n, n)] = std::conj(S.eigenvec[F3(mu, la, n3, n, n)]);
  }
}

void make_kp_reg_tet(State& S) {
  int nx = S.nc[0], ny = S.nc[1], nz = S.nc[2];
  double sx = S.shft[0], sy = S.shft[1], sz = S.shft[2];
  double sh[3];
  for (int c = 0; c < 3; ++c) sh[c] = (-0.5) * ((S.g1[c] + S.g2[c]) + S.g3[c]);
  const double *g1 = S.g1, *g2 = S.g2, *g3 = S.g3;
  int nk = 0;
  std::vector<double> kpt(3 * S.nkc);
  for (int i = 1; i <= nx; ++i)
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nz; ++k) {
        nk = nk + 1;
        double a = (i - 1 + sx) / nx, b = (j - 1 + sy) / ny, c = (k - 1 + sz) / nz;
        for (int d = 0; d < 3; ++d) kpt[F2(d + 1, nk, 3)] = ((a * g1[d] + b * g2[d]) + c * g3[d]) + 0.0;
      }
  S.tet.assign(6 * (size_t)S.nkc, Tetra());
  int nt = 0;
  for (int i = 1; i <= nx; ++i)
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nz; ++k) {
        for (int l = 1; l <= 6; ++l) {
          double q[8][3];
          double a = (i - 1 + sx) / nx, b = (j - 1 + sy) / ny, c = (k - 1 + sz) / nz;
          double ax = 1.0 / nx, by = 1.0 / ny, cz = 1.0 / nz;
          for (int d = 0; d < 3; ++d) {
            double q1 = ((a * g1[d] + b * g2[d]) + c * g3[d]) + sh[d];
            q[0][d] = q1;
            q[1][d] = q1 + ax * g1[d];
            q[2][d] = q1 + by * g2[d];
            q[3][d] = (q1 + ax * g1[d]) + by * g2[d];
            q[4][d] = q1 + cz * g3[d];
            q[5][d] = (q1 + cz * g3[d]) + ax * g1[d];
            q[6][d] = (q1 + cz * g3[d]) + by * g2[d];
            q[7][d] = ((q1 + cz * g3[d]) + ax * g1[d]) + by * g2[d];
          }
          int pt[8];
          for (int m = 0; m < 8; ++m) {
            int nk1, i1, j1, k1, inside;
            get_k_info(S, q[m], nk1, i1, j1, k1, inside);
            pt[m] = nk1;
          }
          nt = nt + 1;
          static const int corners[6][4] = {{1, 2, 3, 6}, {2, 3, 4, 6}, {1, 3, 5, 6},
                                            {3, 4, 6, 8}, {3, 5, 6, 7}, {3, 6, 7, 8}};
          for (int m = 0; m < 4; ++m) S.tet[nt - 1].i[m] = pt[corners[l - 1][m] - 1];
        }
      }
  if (nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0)
    for (int i = 1; i <= nk; ++i)
      for (int c = 0; c < 3; ++c) kpt[F2(c + 1, i, 3)] = kpt[F2(c + 1, i, 3)] + sh[c];
  S.kpc = kpt;
}

}  // namespace orc
