// ORACLE -- TEST INFRASTRUCTURE ONLY (see oracle_core.h).
// Input readers and lattice symmetry, restated from the reference:
//   read_params     THERMACOND/rest.f90:2-76
//   read_input_fit  THERMACOND/rest.f90:78-149
//   read_lattice    THERMACOND/rest.f90:152-289
//   read_fc234      THERMACOND/rest.f90:303-443
//   read_born       THERMACOND/rest.f90:3580-3601
//   force_constants_init (lattice point group and op_kmatrix only)
//                   THERMACOND/force_constants.f90:3-186, dlatmat2 :1379-1545,
//                   xmatinv/ludcmp/lubksb :1165-1288
#include <algorithm>
#include <cctype>
#include <cstring>
#include <fstream>
#include <sstream>

#include "oracle_core.h"

namespace orc {

namespace {

// Fortran list-directed reading: each READ starts on a new record, takes
// blank/comma separated values across records as needed, then drops the
// rest of the last record it touched.
struct ListReader {
  std::vector<std::string> lines;
  size_t pos = 0;
  bool ok = true;
  std::string err;

  bool open(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string l;
    while (std::getline(f, l)) {
      if (!l.empty() && l.back() == '\r') l.pop_back();
      lines.push_back(l);
    }
    return true;
  }
  static std::vector<std::string> tokens(const std::string& l) {
    std::vector<std::string> t;
    std::string cur;
    for (char c : l) {
      if (c == ' ' || c == '\t' || c == ',') {
        if (!cur.empty()) t.push_back(cur), cur.clear();
      } else if (c == '/') {
        break;
      } else {
        cur.push_back(c);
      }
    }
    if (!cur.empty()) t.push_back(cur);
    return t;
  }
  // read n values of list-directed input
  std::vector<std::string> read(int n) {
    std::vector<std::string> out;
    while ((int)out.size() < n) {
      if (pos >= lines.size()) {
        ok = false;
        err = "end of file";
        return out;
      }
      std::vector<std::string> t = tokens(lines[pos++]);
      for (auto& s : t) {
        if ((int)out.size() < n) out.push_back(s);
      }
    }
    return out;
  }
  std::string read_line() {  // read(u,'(a)')
    if (pos >= lines.size()) {
      ok = false;
      err = "end of file";
      return "";
    }
    return lines[pos++];
  }
  bool eof() const {
    for (size_t p = pos; p < lines.size(); ++p)
      if (!tokens(lines[p]).empty()) return false;
    return true;
  }
};

double fnum(const std::string& s) {
  std::string t = s;
  for (auto& c : t)
    if (c == 'd' || c == 'D') c = 'e';
  return std::strtod(t.c_str(), nullptr);
}
int inum(const std::string& s) { return (int)std::strtol(s.c_str(), nullptr, 10); }
bool lnum(const std::string& s) {
  std::string t;
  for (char c : s)
    if (c != '.') t.push_back((char)std::tolower(c));
  return !t.empty() && t[0] == 't';
}

// ------------------------------------------------- 3x3 helpers (Fortran order)
// xmatmlt: x3 = x1*x2, column-major 3x3 (force_constants.f90:1290-1326)
void xmatmlt3(const double* x1, const double* x2, double* x3) {
  double x[9];
  for (int i = 1; i <= 3; ++i)
    for (int j = 1; j <= 3; ++j) {
      double s = 0;
      for (int k = 1; k <= 3; ++k) s = s + x1[F2(j, k, 3)] * x2[F2(k, i, 3)];
      x[F2(j, i, 3)] = s;
    }
  std::memcpy(x3, x, sizeof x);
}

int ncmp(double x) { return std::fabs(x) > 1e-6 ? 1 : 0; }

// Numerical-Recipes LU as used by xmatinv (force_constants.f90:1165-1288)
void ludcmp(double* a, int n, int* indx, double& d) {
  const double tiny = 1.0e-20;
  double vv[3];
  d = 1;
  int imax = 0;
  for (int i = 1; i <= n; ++i) {
    double aamax = 0;
    for (int j = 1; j <= n; ++j)
      if (std::fabs(a[F2(i, j, 3)]) > aamax) aamax = std::fabs(a[F2(i, j, 3)]);
    if (ncmp(aamax) == 0) {
      d = 0;
      return;
    }
    vv[i - 1] = 1 / aamax;
  }
  for (int j = 1; j <= n; ++j) {
    for (int i = 1; i <= j - 1; ++i) {
      double sum = a[F2(i, j, 3)];
      for (int k = 1; k <= i - 1; ++k) sum = sum - a[F2(i, k, 3)] * a[F2(k, j, 3)];
      a[F2(i, j, 3)] = sum;
    }
    double aamax = 0;
    for (int i = j; i <= n; ++i) {
      double sum = a[F2(i, j, 3)];
      for (int k = 1; k <= j - 1; ++k) sum = sum - a[F2(i, k, 3)] * a[F2(k, j, 3)];
      a[F2(i, j, 3)] = sum;
      double dum = vv[i - 1] * std::fabs(sum);
      if (dum >= aamax) {
        imax = i;
        aamax = dum;
      }
    }
    if (j != imax) {
      for (int k = 1; k <= n; ++k) {
        double dum = a[F2(imax, k, 3)];
        a[F2(imax, k, 3)] = a[F2(j, k, 3)];
        a[F2(j, k, 3)] = dum;
      }
      d = -d;
      vv[imax - 1] = vv[j - 1];
    }
    indx[j - 1] = imax;
    if (a[F2(j, j, 3)] == 0.0) a[F2(j, j, 3)] = tiny;
    if (j != n) {
      double dum = 1 / a[F2(j, j, 3)];
      for (int i = j + 1; i <= n; ++i) a[F2(i, j, 3)] = a[F2(i, j, 3)] * dum;
    }
  }
}

void lubksb(const double* a, int n, const int* indx, double* b) {
  int ii = 0;
  for (int i = 1; i <= n; ++i) {
    int ll = indx[i - 1];
    double sum = b[ll - 1];
    b[ll - 1] = b[i - 1];
    if (ii != 0) {
      for (int j = ii; j <= i - 1; ++j) sum = sum - a[F2(i, j, 3)] * b[j - 1];
    } else if (sum != 0.0) {
      ii = i;
    }
    b[i - 1] = sum;
  }
  for (int i = n; i >= 1; --i) {
    double sum = b[i - 1];
    if (i < n)
      for (int j = i + 1; j <= n; ++j) sum = sum - a[F2(i, j, 3)] * b[j - 1];
    b[i - 1] = sum / a[F2(i, i, 3)];
  }
}

int xmatinv(const double* in, double* out) {
  double buf[9];
  int indx[3];
  double x;
  for (int i = 1; i <= 3; ++i) {
    for (int j = 1; j <= 3; ++j) {
      out[F2(i, j, 3)] = 0;
      buf[F2(i, j, 3)] = in[F2(i, j, 3)];
    }
    out[F2(i, i, 3)] = 1;
  }
  ludcmp(buf, 3, indx, x);
  if (x == 0.0) return 1;
  for (int j = 1; j <= 3; ++j) lubksb(buf, 3, indx, out + (j - 1) * 3);
  return 0;
}

double vlength(const double* v) {
  double x = 0;
  for (int i = 0; i < 3; ++i) x = x + v[i] * v[i];
  return std::sqrt(x);
}

int ndet(const int m[9]) {
  auto M = [&](int i, int j) { return m[F2(i, j, 3)]; };
  return M(1, 1) * (M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2)) - M(1, 2) * (M(2, 1) * M(3, 3) - M(2, 3) * M(3, 1)) +
         M(1, 3) * (M(2, 1) * M(3, 2) - M(2, 2) * M(3, 1));
}

// dlatmat2: point group of the lattice (force_constants.f90:1379-1545)
int dlatmat2(const double* cart, double eps, int& nmatrices, int matrices[48][9]) {
  const int nmax = 400;
  std::vector<double> dshort(nmax * 3, 0.0), vshort(3 * nmax * 3, 0.0);
  std::vector<int> ishort(3 * nmax * 3, 0);
  int nshort[3] = {0, 0, 0};
  double abc[9];
  for (int i = 1; i <= 3; ++i) abc[F2(i, i, 3)] = vlength(cart + (i - 1) * 3);
  for (int i = 2; i <= 3; ++i)
    for (int j = 1; j <= i - 1; ++j) {
      double v[3];
      for (int k = 0; k < 3; ++k) v[k] = cart[(i - 1) * 3 + k] - cart[(j - 1) * 3 + k];
      abc[F2(i, j, 3)] = vlength(v);
      abc[F2(j, i, 3)] = abc[F2(i, j, 3)];
    }
  int i = 0;
  bool foundone = true;
  double xmax = std::max(std::max(abc[F2(1, 1, 3)], abc[F2(2, 2, 3)]), abc[F2(3, 3, 3)]) + eps;
  while (foundone) {
    i = i + 1;
    foundone = false;
    for (int j1 = -i; j1 <= i; ++j1)
      for (int j2 = -i; j2 <= i; ++j2)
        for (int j3 = -i; j3 <= i; ++j3) {
          if (std::abs(j1) == i || std::abs(j2) == i || std::abs(j3) == i) {
            double v[3] = {0, 0, 0};
            for (int k = 1; k <= 3; ++k) {
              v[k - 1] = v[k - 1] + j1 * cart[F2(k, 1, 3)];
              v[k - 1] = v[k - 1] + j2 * cart[F2(k, 2, 3)];
              v[k - 1] = v[k - 1] + j3 * cart[F2(k, 3, 3)];
            }
            double d = vlength(v);
            if (d < xmax) foundone = true;
            for (int k = 1; k <= 3; ++k) {
              if (std::fabs(d - abc[F2(k, k, 3)]) < eps) {
                nshort[k - 1] = nshort[k - 1] + 1;
                if (nshort[k - 1] > nmax) return 1;
                int ns = nshort[k - 1];
                dshort[(ns - 1) + nmax * (k - 1)] = d;
                ishort[0 + 3 * ((ns - 1) + nmax * (k - 1))] = j1;
                ishort[1 + 3 * ((ns - 1) + nmax * (k - 1))] = j2;
                ishort[2 + 3 * ((ns - 1) + nmax * (k - 1))] = j3;
                vshort[0 + 3 * ((ns - 1) + nmax * (k - 1))] = v[0];
                vshort[1 + 3 * ((ns - 1) + nmax * (k - 1))] = v[1];
                vshort[2 + 3 * ((ns - 1) + nmax * (k - 1))] = v[2];
              }
            }
          }
        }
  }
  auto ISH = [&](int c, int n, int k) { return ishort[(c - 1) + 3 * ((n - 1) + nmax * (k - 1))]; };
  auto VSH = [&](int n, int k) { return &vshort[3 * ((n - 1) + nmax * (k - 1))]; };
  nmatrices = 1;
  int itrans[9];
  int ichoose[3];
  for (int i1 = 1; i1 <= nshort[0]; ++i1) {
    ichoose[0] = i1;
    for (int c = 1; c <= 3; ++c) itrans[F2(c, 1, 3)] = ISH(c, i1, 1);
    for (int i2 = 1; i2 <= nshort[1]; ++i2) {
      ichoose[1] = i2;
      for (int c = 1; c <= 3; ++c) itrans[F2(c, 2, 3)] = ISH(c, i2, 2);
      for (int i3 = 1; i3 <= nshort[2]; ++i3) {
        ichoose[2] = i3;
        for (int c = 1; c <= 3; ++c) itrans[F2(c, 3, 3)] = ISH(c, i3, 3);
        if (std::abs(ndet(itrans)) != 1) continue;
        bool bad = false;
        for (int ii = 2; ii <= 3 && !bad; ++ii)
          for (int jj = 1; jj <= ii - 1; ++jj) {
            double v[3];
            const double* a = VSH(ichoose[ii - 1], ii);
            const double* b = VSH(ichoose[jj - 1], jj);
            for (int k = 0; k < 3; ++k) v[k] = a[k] - b[k];
            double x = vlength(v);
            if (std::fabs(x - abc[F2(ii, jj, 3)]) > eps) {
              bad = true;
              break;
            }
          }
        if (bad) continue;
        if (itrans[F2(1, 1, 3)] + itrans[F2(2, 2, 3)] + itrans[F2(3, 3, 3)] == 3) {
          std::memcpy(matrices[0], itrans, sizeof itrans);
        } else {
          nmatrices = nmatrices + 1;
          if (nmatrices > 48) return 2;
          std::memcpy(matrices[nmatrices - 1], itrans, sizeof itrans);
        }
      }
    }
  }
  // close the set under multiplication
  std::vector<char> tried(48 * 48, 0);
  foundone = true;
  while (foundone) {
    foundone = false;
    int nm0 = nmatrices;
    for (int a = 1; a <= nm0; ++a) {
      int nm1 = nmatrices;
      for (int b = 1; b <= nm1; ++b) {
        if (tried[(a - 1) + 48 * (b - 1)]) continue;
        tried[(a - 1) + 48 * (b - 1)] = 1;
        int prod[9];
        for (int r = 1; r <= 3; ++r)
          for (int c = 1; c <= 3; ++c) {
            int s = 0;
            for (int k = 1; k <= 3; ++k) s += matrices[a - 1][F2(r, k, 3)] * matrices[b - 1][F2(k, c, 3)];
            prod[F2(r, c, 3)] = s;
          }
        int nm2 = nmatrices;
        for (int k = 1; k <= nm2; ++k) {
          bool same = true;
          for (int e = 0; e < 9; ++e)
            if (matrices[k - 1][e] != prod[e]) {
              same = false;
              break;
            }
          if (same) break;
          if (k == nm2) {
            foundone = true;
            nmatrices = nmatrices + 1;
            if (nmatrices > 48) return 2;
            std::memcpy(matrices[nmatrices - 1], prod, sizeof prod);
          }
        }
      }
    }
  }
  return 0;
}

}  // namespace

std::string read_inputs(State& S, const std::string& dir) {
  // ---------------------------------------------------------- latdyn.params
  {
    ListReader r;
    if (!r.open(dir + "/latdyn.params")) return "cannot open latdyn.params";
    auto t = r.read(4);
    for (int i = 0; i < 3; ++i) S.nc[i] = inum(t[i]);
    S.dos_bs_only = lnum(t[3]);
    t = r.read(3);
    for (int i = 0; i < 3; ++i) S.shft[i] = fnum(t[i]);
    t = r.read(3);
    for (int i = 0; i < 3; ++i) S.normald[i] = fnum(t[i]);
    t = r.read(2);
    S.wmesh = inum(t[0]);
    S.wmax = fnum(t[1]);
    t = r.read(2);
    S.width = fnum(t[0]);
    S.etaz = fnum(t[1]);
    t = r.read(1);
    S.verbose = lnum(t[0]);
    t = r.read(3);
    S.tmin = fnum(t[0]);
    S.tmax = fnum(t[1]);
    S.ntemp = inum(t[2]);
    t = r.read(1);
    S.job = inum(t[0]);
    t = r.read(1);
    S.ksub_size = inum(t[0]);
    r.read_line();  // v3path
    t = r.read(1);
    S.iso = inum(t[0]);
    t = r.read(1);
    S.classical = inum(t[0]);
    t = r.read(4);
    t = r.read(1);
    if (!r.ok) return "latdyn.params: " + r.err;
  }
  // ------------------------------------------------------- structure.params
  {
    ListReader r;
    if (!r.open(dir + "/structure.params")) return "cannot open structure.params";
    auto t = r.read(6);
    for (int i = 0; i < 6; ++i) S.latticeparameters[i] = fnum(t[i]);
    t = r.read(9);
    for (int i = 0; i < 9; ++i) S.primitivelattice[i] = fnum(t[i]);
    t = r.read(1);
    S.lattice_parameter = fnum(t[0]);
    for (int i = 0; i < 3; ++i) S.latticeparameters[i] = S.latticeparameters[i] * S.lattice_parameter;
    t = r.read(4);
    for (int i = 0; i < 4; ++i) S.include_fc[i] = inum(t[i]);
    r.read(1);
    r.read(1);
    r.read(1);
    t = r.read(1);
    S.natom_type = inum(t[0]);
    t = r.read(S.natom_type);
    S.mas.resize(S.natom_type);
    for (int i = 0; i < S.natom_type; ++i) S.mas[i] = fnum(t[i]);
    t = r.read(S.natom_type);
    S.atname.assign(t.begin(), t.end());
    t = r.read(1);
    S.natoms0 = inum(t[0]);
    for (int i = 0; i < 8; ++i) r.read(1);
    S.atom_type.assign(S.natoms0, 0);
    for (int i = 0; i < S.natoms0; ++i) {
      t = r.read(5);
      int label = inum(t[0]);
      if (label < 1 || label > S.natoms0) return "structure.params: bad atom label";
      S.atom_type[label - 1] = inum(t[1]);
    }
    if (!r.ok) return "structure.params: " + r.err;
    S.mass0.resize(S.natoms0);
    for (int i = 0; i < S.natoms0; ++i) S.mass0[i] = S.mas[S.atom_type[i] - 1];
  }
  // ------------------------------------------------------------ lat_fc.dat
  {
    ListReader r;
    if (!r.open(dir + "/lat_fc.dat")) return "cannot open lat_fc.dat";
    std::string line;
    do {
      line = r.read_line();
      if (!r.ok) return "lat_fc.dat: no '  Crystal data: transl' record";
    } while (line.substr(0, 22) != "  Crystal data: transl");
    auto t = r.read(3);
    for (int i = 0; i < 3; ++i) S.r1[i] = fnum(t[i]);
    t = r.read(3);
    for (int i = 0; i < 3; ++i) S.r2[i] = fnum(t[i]);
    t = r.read(3);
    for (int i = 0; i < 3; ++i) S.r3[i] = fnum(t[i]);
    auto cross = [](const double* a, const double* b, double* c) {
      c[0] = a[1] * b[2] - a[2] * b[1];
      c[1] = a[2] * b[0] - a[0] * b[2];
      c[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto dot = [](const double* a, const double* b) { return b[0] * a[0] + b[1] * a[1] + b[2] * a[2]; };
    // make_reciprocal_lattice_2pi (extratools.f90:209-228)
    double c23[3], c31[3], c12[3];
    cross(S.r2, S.r3, c23);
    cross(S.r3, S.r1, c31);
    cross(S.r1, S.r2, c12);
    double om = dot(S.r1, c23);
    for (int i = 0; i < 3; ++i) {
      S.g1[i] = 2 * S.K.pi * c23[i] / om;
      S.g2[i] = 2 * S.K.pi * c31[i] / om;
      S.g3[i] = 2 * S.K.pi * c12[i] / om;
    }
    set_k_dual(S);
    // calculate_volume (extratools.f90:177-186)
    S.volume_r = std::fabs(dot(S.r3, c12));
    double gc[3];
    cross(S.g1, S.g2, gc);
    S.volume_g = std::fabs(dot(S.g3, gc));
    r.read(1);
    t = r.read(1);
    if (inum(t[0]) != S.natoms0) return "lat_fc.dat: natoms0 incompatible with structure.params";
    for (int i = 1; i <= S.natoms0; ++i) {
      t = r.read(7);
      int tt = inum(t[0]), ttyp = inum(t[2]);
      double mss = fnum(t[6]);
      if (!(tt == i && ttyp == S.atom_type[i - 1] && S.mass0[i - 1] == mss))
        return "READ_LATTICE: structure.params and lat_fc.dat are not compatible";
    }
    r.read(1);
    t = r.read(4);
    for (int i = 0; i < 4; ++i) S.include_fc[i] = inum(t[i]);
    for (int i = 0; i < 8; ++i) r.read(1);
    r.read(1);
    r.read(4);  // ngroups
    r.read(1);
    t = r.read(4);
    for (int i = 0; i < 4; ++i) S.nterms[i] = inum(t[i]);
    r.read(1);
    r.read(1);
    r.read(1);
    t = r.read(2);
    int natoms2 = inum(t[1]);
    S.natoms = natoms2;
    S.atompos.assign(3 * natoms2, 0.0);
    S.iatomcell0.assign(natoms2, 0);
    S.iatomcell.assign(3 * natoms2, 0);
    for (int j = 0; j < natoms2; ++j) {
      t = r.read(8);
      if (!r.ok) return "End of lat_fc.dat file reached";
      int i = inum(t[0]);
      if (i < 1 || i > natoms2) return "lat_fc.dat: bad atom index";
      for (int k = 0; k < 3; ++k) S.atompos[F2(k + 1, i, 3)] = fnum(t[1 + k]);
      S.iatomcell0[i - 1] = inum(t[4]);
      for (int k = 0; k < 3; ++k) S.iatomcell[F2(k + 1, i, 3)] = inum(t[5 + k]);
    }
  }
  // ------------------------------------------- force_constants_init (subset)
  {
    const double* latp0 = S.latticeparameters;
    double latp[6];
    for (int i = 0; i < 6; ++i) latp[i] = latp0[i];
    double d2r = 4.0 * std::atan(1.0) / 180.0;
    for (int i = 3; i < 6; ++i) latp[i] = latp[i] * d2r;
    double conv_to_cart[9] = {0};
    conv_to_cart[F2(1, 1, 3)] = latp[0];
    conv_to_cart[F2(1, 2, 3)] = latp[1] * std::cos(latp[5]);
    conv_to_cart[F2(2, 2, 3)] = latp[1] * std::sin(latp[5]);
    conv_to_cart[F2(1, 3, 3)] = latp[2] * std::cos(latp[4]);
    conv_to_cart[F2(2, 3, 3)] = latp[2] * (std::cos(latp[3]) - std::cos(latp[5]) * std::cos(latp[4])) /
                                std::sin(latp[5]);
    conv_to_cart[F2(3, 3, 3)] = std::sqrt(latp[2] * latp[2] - conv_to_cart[F2(1, 3, 3)] * conv_to_cart[F2(1, 3, 3)] -
                                          conv_to_cart[F2(2, 3, 3)] * conv_to_cart[F2(2, 3, 3)]);
    {  // make_reciprocal_lattice_2pi of the conventional cell (force_constants.f90:100-104)
      const double* c1 = &conv_to_cart[0];
      const double* c2 = &conv_to_cart[3];
      const double* c3 = &conv_to_cart[6];
      double c23[3], c31[3], c12[3];
      auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
      };
      cross(c2, c3, c23);
      cross(c3, c1, c31);
      cross(c1, c2, c12);
      const double om = c1[0] * c23[0] + c1[1] * c23[1] + c1[2] * c23[2];
      for (int i = 0; i < 3; ++i) {
        S.g1conv[i] = 2 * S.K.pi * c23[i] / om;
        S.g2conv[i] = 2 * S.K.pi * c31[i] / om;
        S.g3conv[i] = 2 * S.K.pi * c12[i] / om;
      }
    }
    double prim_to_conv[9], prim_to_cart[9], cart_to_prim[9], conv_to_prim[9];
    std::memcpy(prim_to_conv, S.primitivelattice, sizeof prim_to_conv);
    xmatmlt3(conv_to_cart, prim_to_conv, prim_to_cart);
    if (xmatinv(prim_to_cart, cart_to_prim)) return "primitive_lattice is singular";
    if (xmatinv(prim_to_conv, conv_to_prim)) return "primitive_lattice is singular";
    int iop[48][9];
    if (dlatmat2(prim_to_cart, 1e-5, S.lattpgcount, iop)) return "dlatmat2 failed";
    for (int i = 0; i < S.lattpgcount; ++i) {
      double temp[9], tempi[9];
      for (int e = 0; e < 9; ++e) temp[e] = iop[i][e];
      xmatmlt3(temp, conv_to_prim, temp);
      xmatmlt3(prim_to_conv, temp, temp);
      if (xmatinv(temp, tempi)) return "op_kmatrix: singular operation";
      for (int j = 1; j <= 3; ++j)
        for (int k = 1; k <= 3; ++k) S.op_kmatrix[i][F2(k, j, 3)] = (double)std::lround(tempi[F2(j, k, 3)]);
    }
  }
  // ------------------------------------------------------------- fc2 / fc3
  {
    ListReader r;
    if (!r.open(dir + "/fc2.dat")) return "READ_FC234: file fc2.dat does not exist";
    r.read_line();
    int mx = 0;
    {
      ListReader c = r;
      while (!c.eof()) {
        c.read(1);
        ++mx;
      }
    }
    if (mx != S.nterms[1]) return "READ_FC2: number of lines inconsistent with lat_fc.dat";
    S.iatomterm_2.resize(2 * mx);
    S.ixyzterm_2.resize(2 * mx);
    S.fcs_2.resize(mx);
    for (int j = 0; j < mx; ++j) {
      auto t = r.read(7);
      S.iatomterm_2[0 + 2 * j] = inum(t[2]);
      S.ixyzterm_2[0 + 2 * j] = inum(t[3]);
      S.iatomterm_2[1 + 2 * j] = inum(t[4]);
      S.ixyzterm_2[1 + 2 * j] = inum(t[5]);
      S.fcs_2[j] = fnum(t[6]);
    }
  }
  if (S.include_fc[2] == 1) {
    ListReader r;
    if (!r.open(dir + "/fc3.dat")) return "READ_FC234: file fc3.dat does not exist";
    r.read_line();
    int mx = 0;
    {
      ListReader c = r;
      while (!c.eof()) {
        c.read(1);
        ++mx;
      }
    }
    if (mx != S.nterms[2]) return "READ_FC3: number of lines inconsistent with lat_fc.dat";
    S.iatomterm_3.resize(3 * mx);
    S.ixyzterm_3.resize(3 * mx);
    S.fcs_3.resize(mx);
    for (int j = 0; j < mx; ++j) {
      auto t = r.read(9);
      for (int c = 0; c < 3; ++c) {
        S.iatomterm_3[c + 3 * j] = inum(t[2 + 2 * c]);
        S.ixyzterm_3[c + 3 * j] = inum(t[3 + 2 * c]);
      }
      S.fcs_3[j] = fnum(t[8]);
    }
  }
  // ------------------------------------------------------- dielectric.params
  {
    ListReader r;
    if (r.open(dir + "/dielectric.params")) {
      auto t = r.read(1);
      S.born_flag = inum(t[0]);
      for (int i = 1; i <= 3; ++i) {
        t = r.read(3);
        for (int j = 1; j <= 3; ++j) S.epsil[F2(i, j, 3)] = fnum(t[j - 1]);
      }
      S.charge.assign(9 * S.natoms0, 0.0);
      for (int k = 1; k <= S.natoms0; ++k)
        for (int i = 1; i <= 3; ++i) {
          t = r.read(3);
          for (int j = 1; j <= 3; ++j) S.charge[F3(i, j, k, 3, 3)] = fnum(t[j - 1]);
        }
      if (!r.ok) return "dielectric.params: " + r.err;
    }
  }
  S.nkc = S.nc[0] * S.nc[1] * S.nc[2];
  S.ndyn = 3 * S.natoms0;
  return "";
}

}  // namespace orc
