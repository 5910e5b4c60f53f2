// Host side of libald: input readers, lattice point group, q-mesh, IBZ,
// star arms and tetrahedra.  Everything here runs once per context; the
// tables it builds are integer-indexed so the device never searches a
// mesh by floating-point comparison.
//
// Reference routines mirrored (file:line in THERMACOND/):
//   read_params rest.f90:2-76, read_input_fit rest.f90:78-149,
//   read_lattice rest.f90:152-289, read_fc234 rest.f90:303-443,
//   read_born rest.f90:3580-3601,
//   force_constants_init force_constants.f90:3-186 (point group, op_kmatrix),
//   dlatmat2 force_constants.f90:1379-1545,
//   make_kp_reg modules.f90:1721-1784, get_k_info rest.f90:3024-3058,
//   get_negatives rest.f90:3208-3260, getstar force_constants.f90:1748-1784,
//   get_weights modules.f90:2006-2160, kstarsinfbz1 sub.f90:5551-5590,
//   make_kp_reg_tet tetrahedron.f90:2-142.
#include <algorithm>
#include <array>
#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <numeric>
#include <string_view>
#include <thread>
#include <unordered_map>

#include "ald_internal.h"
#include "ald_pool.h"

namespace ald {

double PhysConst::const33() {
  return 1e30 * std::pow(hbar / uma, 1.5) / std::pow(std::sqrt(ee * 1e20 / uma), 1.5) * ee / h_plank / 100 /
         c_light;
}

namespace {

// ---------------------------------------------------------------- records
// Fortran list-directed input: a READ takes values from the next record
// on, spanning records when a list is longer than one line, and discards
// what is left of the last record.  Blank/comma separate values; '/' ends.
class Records {
 public:
  bool load(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char chunk[1 << 16];
    size_t n;
    while ((n = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf_.append(chunk, n);
    std::fclose(f);
    size_t b = 0;
    while (b < buf_.size()) {  // lines as getline gives them
      size_t e = buf_.find('\n', b);
      if (e == std::string::npos) e = buf_.size();
      rec_.push_back({b, e - b});
      b = e + 1;
    }
    return true;
  }
  bool next(size_t n, std::vector<std::string_view>& out) {
    out.clear();
    while (out.size() < n) {
      if (at_ >= rec_.size()) return false;
      split(record(at_++), out, n);
    }
    return true;
  }
  bool line(std::string& s) {
    if (at_ >= rec_.size()) return false;
    s.assign(record(at_++));
    return true;
  }
  // the records from the current one on that hold a value before any '/'
  std::vector<size_t> nonblank_records() const {
    std::vector<size_t> r;
    for (size_t i = at_; i < rec_.size(); ++i)
      for (char ch : record(i)) {
        if (ch == '/') break;
        if (!is_sep(ch)) {
          r.push_back(i);
          break;
        }
      }
    return r;
  }
  // the values of record i alone (at most cap)
  void values(size_t i, std::vector<std::string_view>& out, size_t cap) const {
    out.clear();
    split(record(i), out, cap);
  }

 private:
  std::string_view record(size_t i) const { return std::string_view(buf_.data() + rec_[i].first, rec_[i].second); }
  static bool is_sep(char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r'; }
  static void split(std::string_view l, std::vector<std::string_view>& out, size_t cap) {
    const char* p = l.data();
    const size_t n = l.size();
    size_t i = 0;
    while (i < n && out.size() < cap) {
      if (p[i] == '/') return;
      if (is_sep(p[i])) {
        ++i;
        continue;
      }
      size_t j = i;
      while (j < n && p[j] != '/' && !is_sep(p[j])) ++j;
      out.emplace_back(p + i, j - i);
      if (j < n && p[j] == '/') return;
      i = j;
    }
  }
  std::string buf_;
  std::vector<std::pair<size_t, size_t>> rec_;  // (offset, length) of each line in buf_
  size_t at_ = 0;
};

// a value as strtod / strtol read it (Fortran's D exponent read as E).
// std::from_chars (correctly rounded, as strtod is) takes the tokens it reads
// whole; anything else -- a leading '+', an out-of-range value, a token with
// trailing characters -- goes to strtod / strtol, so every token reads as
// strtod / strtol read it.
double dval(std::string_view s) {
  char b[64];
  if (s.size() >= sizeof b) {
    std::string t(s);
    for (char& c : t)
      if (c == 'd' || c == 'D') c = 'e';
    return std::strtod(t.c_str(), nullptr);
  }
  for (size_t i = 0; i < s.size(); ++i) b[i] = (s[i] == 'd' || s[i] == 'D') ? 'e' : s[i];
  b[s.size()] = 0;
  double v;
  const auto r = std::from_chars(b, b + s.size(), v);
  if (r.ec == std::errc() && r.ptr == b + s.size()) return v;
  return std::strtod(b, nullptr);
}
int ival(std::string_view s) {
  int v;
  const auto r = std::from_chars(s.data(), s.data() + s.size(), v);
  if (r.ec == std::errc() && r.ptr == s.data() + s.size()) return v;
  char b[64];
  if (s.size() >= sizeof b) return (int)std::strtol(std::string(s).c_str(), nullptr, 10);
  std::memcpy(b, s.data(), s.size());
  b[s.size()] = 0;
  return (int)std::strtol(b, nullptr, 10);
}

inline int cm(int i, int j) { return i + 3 * j; }  // 0-based column-major 3x3

void mat3mul(const double* a, const double* b, double* c) {  // c = a*b (column-major)
  double t[9];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += a[cm(i, k)] * b[cm(k, j)];
      t[cm(i, j)] = s;
    }
  std::memcpy(c, t, sizeof t);
}

bool mat3inv(const double* a, double* out) {
  double det = a[cm(0, 0)] * (a[cm(1, 1)] * a[cm(2, 2)] - a[cm(1, 2)] * a[cm(2, 1)]) -
               a[cm(0, 1)] * (a[cm(1, 0)] * a[cm(2, 2)] - a[cm(1, 2)] * a[cm(2, 0)]) +
               a[cm(0, 2)] * (a[cm(1, 0)] * a[cm(2, 1)] - a[cm(1, 1)] * a[cm(2, 0)]);
  if (std::fabs(det) < 1e-12) return false;
  double r[9];
  r[cm(0, 0)] = (a[cm(1, 1)] * a[cm(2, 2)] - a[cm(1, 2)] * a[cm(2, 1)]) / det;
  r[cm(0, 1)] = (a[cm(0, 2)] * a[cm(2, 1)] - a[cm(0, 1)] * a[cm(2, 2)]) / det;
  r[cm(0, 2)] = (a[cm(0, 1)] * a[cm(1, 2)] - a[cm(0, 2)] * a[cm(1, 1)]) / det;
  r[cm(1, 0)] = (a[cm(1, 2)] * a[cm(2, 0)] - a[cm(1, 0)] * a[cm(2, 2)]) / det;
  r[cm(1, 1)] = (a[cm(0, 0)] * a[cm(2, 2)] - a[cm(0, 2)] * a[cm(2, 0)]) / det;
  r[cm(1, 2)] = (a[cm(0, 2)] * a[cm(1, 0)] - a[cm(0, 0)] * a[cm(1, 2)]) / det;
  r[cm(2, 0)] = (a[cm(1, 0)] * a[cm(2, 1)] - a[cm(1, 1)] * a[cm(2, 0)]) / det;
  r[cm(2, 1)] = (a[cm(0, 1)] * a[cm(2, 0)] - a[cm(0, 0)] * a[cm(2, 1)]) / det;
  r[cm(2, 2)] = (a[cm(0, 0)] * a[cm(1, 1)] - a[cm(0, 1)] * a[cm(1, 0)]) / det;
  std::memcpy(out, r, sizeof r);
  return true;
}

double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Lattice point group in the order dlatmat2 enumerates it (the order sets
// which operation is attached to each star arm): integer matrices mapping
// the three basis vectors onto lattice vectors of equal length, found
// shell by shell, identity first, then closed under multiplication.
std::string lattice_point_group(const double* prim_to_cart, std::vector<std::array<int, 9>>& ops) {
  const double eps = 1e-5;
  double len[3], dif[3][3];
  const double* col[3] = {prim_to_cart, prim_to_cart + 3, prim_to_cart + 6};
  for (int i = 0; i < 3; ++i) len[i] = norm3(col[i]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v[3] = {col[i][0] - col[j][0], col[i][1] - col[j][1], col[i][2] - col[j][2]};
      dif[i][j] = norm3(v);
    }
  struct Cand {
    int n[3];
    double v[3];
  };
  std::vector<Cand> cand[3];
  double lmax = std::max(std::max(len[0], len[1]), len[2]) + eps;
  for (int shell = 1;; ++shell) {
    bool any_short = false;
    for (int a = -shell; a <= shell; ++a)
      for (int b = -shell; b <= shell; ++b)
        for (int c = -shell; c <= shell; ++c) {
          if (std::abs(a) != shell && std::abs(b) != shell && std::abs(c) != shell) continue;
          Cand k;
          k.n[0] = a;
          k.n[1] = b;
          k.n[2] = c;
          for (int x = 0; x < 3; ++x) k.v[x] = a * col[0][x] + b * col[1][x] + c * col[2][x];
          double d = norm3(k.v);
          if (d < lmax) any_short = true;
          for (int i = 0; i < 3; ++i)
            if (std::fabs(d - len[i]) < eps) {
              cand[i].push_back(k);
              if (cand[i].size() > 400) return "point group search: too many lattice vectors";
            }
        }
    if (!any_short) break;
  }
  ops.clear();
  std::array<int, 9> ident{};
  bool have_ident = false;
  std::vector<std::array<int, 9>> rest;
  for (auto& c0 : cand[0])
    for (auto& c1 : cand[1])
      for (auto& c2 : cand[2]) {
        std::array<int, 9> m;
        const Cand* cc[3] = {&c0, &c1, &c2};
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) m[cm(i, j)] = cc[j]->n[i];
        int det = m[cm(0, 0)] * (m[cm(1, 1)] * m[cm(2, 2)] - m[cm(1, 2)] * m[cm(2, 1)]) -
                  m[cm(0, 1)] * (m[cm(1, 0)] * m[cm(2, 2)] - m[cm(1, 2)] * m[cm(2, 0)]) +
                  m[cm(0, 2)] * (m[cm(1, 0)] * m[cm(2, 1)] - m[cm(1, 1)] * m[cm(2, 0)]);
        if (std::abs(det) != 1) continue;
        bool ok = true;
        for (int i = 1; i < 3 && ok; ++i)
          for (int j = 0; j < i; ++j) {
            double v[3] = {cc[i]->v[0] - cc[j]->v[0], cc[i]->v[1] - cc[j]->v[1], cc[i]->v[2] - cc[j]->v[2]};
            if (std::fabs(norm3(v) - dif[i][j]) > eps) {
              ok = false;
              break;
            }
          }
        if (!ok) continue;
        if (m[0] + m[4] + m[8] == 3) {
          ident = m;
          have_ident = true;
        } else {
          rest.push_back(m);
        }
      }
  if (!have_ident) return "point group search: identity not found";
  ops.push_back(ident);
  for (auto& m : rest) ops.push_back(m);
  if (ops.size() > 48) return "more than 48 point operations";
  // closure under products, visiting pairs in the reference's order
  std::vector<std::vector<char>> tried(48, std::vector<char>(48, 0));
  bool grew = true;
  while (grew) {
    grew = false;
    size_t na = ops.size();
    for (size_t a = 0; a < na; ++a) {
      size_t nb = ops.size();
      for (size_t b = 0; b < nb; ++b) {
        if (tried[a][b]) continue;
        tried[a][b] = 1;
        std::array<int, 9> p{};
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            int s = 0;
            for (int k = 0; k < 3; ++k) s += ops[a][cm(i, k)] * ops[b][cm(k, j)];
            p[cm(i, j)] = s;
          }
        if (std::find(ops.begin(), ops.end(), p) == ops.end()) {
          if (ops.size() == 48) return "more than 48 point operations";
          ops.push_back(p);
          grew = true;
        }
      }
    }
  }
  return "";
}

}  // namespace

// ======================================================================
std::string read_system(const std::string& dir, System& S) {
  std::vector<std::string_view> t;
  {  // ------------------------------------------------- latdyn.params
    Records R;
    if (!R.load(dir + "/latdyn.params")) return "cannot open latdyn.params";
    std::string dummy;
    bool ok = R.next(4, t);
    if (ok) {
      for (int i = 0; i < 3; ++i) S.nc[i] = ival(t[i]);
    }
    ok = ok && R.next(3, t);
    if (ok)
      for (int i = 0; i < 3; ++i) S.shft[i] = dval(t[i]);
    ok = ok && R.next(3, t);  // normald
    ok = ok && R.next(2, t);  // wmesh wmax
    ok = ok && R.next(2, t);
    if (ok) {
      S.width = dval(t[0]);
      S.etaz = dval(t[1]);
    }
    ok = ok && R.next(1, t);  // verbose
    ok = ok && R.next(3, t);
    if (ok) {
      S.tmin = dval(t[0]);
      S.tmax = dval(t[1]);
    }
    ok = ok && R.next(1, t);
    if (ok) S.job = ival(t[0]);
    ok = ok && R.next(1, t);  // ksub_size
    ok = ok && R.line(dummy);  // v3path, read with (a)
    ok = ok && R.next(1, t);
    if (ok) S.iso = ival(t[0]);
    ok = ok && R.next(1, t);
    if (ok) S.classical = ival(t[0]);
    ok = ok && R.next(4, t);
    ok = ok && R.next(1, t);
    if (!ok) return "latdyn.params: premature end of file";
  }
  {  // ---------------------------------------------- structure.params
    Records R;
    if (!R.load(dir + "/structure.params")) return "cannot open structure.params";
    bool ok = R.next(6, t);
    if (ok)
      for (int i = 0; i < 6; ++i) S.latp[i] = dval(t[i]);
    ok = ok && R.next(9, t);
    if (ok)
      for (int i = 0; i < 9; ++i) S.primlatt[i] = dval(t[i]);
    ok = ok && R.next(1, t);
    if (ok) {
      S.scale = dval(t[0]);
      for (int i = 0; i < 3; ++i) S.latp[i] *= S.scale;
    }
    ok = ok && R.next(4, t);
    for (int i = 0; i < 3 && ok; ++i) ok = R.next(1, t);
    int ntype = 0;
    ok = ok && R.next(1, t);
    if (ok) ntype = ival(t[0]);
    if (ok && (ntype < 1 || ntype > 100000)) return "structure.params: bad natom_type";
    ok = ok && R.next(ntype, t);
    if (ok)
      for (int i = 0; i < ntype; ++i) S.mas.push_back(dval(t[i]));
    ok = ok && R.next(ntype, t);
    if (ok)
      for (int i = 0; i < ntype; ++i) S.atname.emplace_back(t[i]);
    ok = ok && R.next(1, t);
    if (ok) S.nat0 = ival(t[0]);
    if (ok && (S.nat0 < 1 || S.nat0 > 4096)) return "structure.params: bad natoms0";
    for (int i = 0; i < 8 && ok; ++i) ok = R.next(1, t);
    S.atype.assign(S.nat0, 0);
    for (int i = 0; i < S.nat0 && ok; ++i) {
      ok = R.next(5, t);
      if (!ok) break;
      int lab = ival(t[0]);
      if (lab < 1 || lab > S.nat0) return "structure.params: atom label out of range";
      S.atype[lab - 1] = ival(t[1]);
    }
    if (!ok) return "structure.params: premature end of file";
    for (int i = 0; i < S.nat0; ++i) {
      if (S.atype[i] < 1 || S.atype[i] > ntype) return "structure.params: atom type out of range";
      S.mass0.push_back(S.mas[S.atype[i] - 1]);
    }
  }
  {  // ---------------------------------------------------- lat_fc.dat
    Records R;
    if (!R.load(dir + "/lat_fc.dat")) return "cannot open lat_fc.dat";
    std::string l;
    for (;;) {
      if (!R.line(l)) return "lat_fc.dat: no '  Crystal data: transl' record";
      if (l.compare(0, 22, "  Crystal data: transl") == 0) break;
    }
    for (int a = 0; a < 3; ++a) {
      if (!R.next(3, t)) return "lat_fc.dat: truncated lattice vectors";
      for (int x = 0; x < 3; ++x) S.r[a][x] = dval(t[x]);
    }
    auto cross = [](const double* u, const double* v, double* w) {
      w[0] = u[1] * v[2] - u[2] * v[1];
      w[1] = u[2] * v[0] - u[0] * v[2];
      w[2] = u[0] * v[1] - u[1] * v[0];
    };
    double c23[3], c31[3], c12[3];
    cross(S.r[1], S.r[2], c23);
    cross(S.r[2], S.r[0], c31);
    cross(S.r[0], S.r[1], c12);
    double om = S.r[0][0] * c23[0] + S.r[0][1] * c23[1] + S.r[0][2] * c23[2];
    for (int x = 0; x < 3; ++x) {
      S.g[0][x] = 2 * PhysConst::pi * c23[x] / om;
      S.g[1][x] = 2 * PhysConst::pi * c31[x] / om;
      S.g[2][x] = 2 * PhysConst::pi * c12[x] / om;
    }
    S.volume_r = std::fabs(c12[0] * S.r[2][0] + c12[1] * S.r[2][1] + c12[2] * S.r[2][2]);
    double gc[3];
    cross(S.g[0], S.g[1], gc);
    S.volume_g = std::fabs(gc[0] * S.g[2][0] + gc[1] * S.g[2][1] + gc[2] * S.g[2][2]);
    bool ok = R.next(1, t) && R.next(1, t);
    if (!ok) return "lat_fc.dat: truncated";
    if (ival(t[0]) != S.nat0) return "lat_fc.dat: natoms0 incompatible with structure.params";
    for (int i = 0; i < S.nat0; ++i) {
      if (!R.next(7, t)) return "lat_fc.dat: truncated atom list";
      if (ival(t[0]) != i + 1 || ival(t[2]) != S.atype[i] || dval(t[6]) != S.mass0[i])
        return "READ_LATTICE: structure.params and lat_fc.dat are not compatible";
    }
    ok = R.next(1, t) && R.next(4, t);
    if (ok)
      for (int i = 0; i < 4; ++i) S.include_fc[i] = ival(t[i]);
    for (int i = 0; i < 8 && ok; ++i) ok = R.next(1, t);
    ok = ok && R.next(1, t) && R.next(4, t) && R.next(1, t) && R.next(4, t);
    if (ok)
      for (int i = 0; i < 4; ++i) S.nterms[i] = ival(t[i]);
    ok = ok && R.next(1, t) && R.next(1, t) && R.next(1, t) && R.next(2, t);
    if (!ok) return "lat_fc.dat: truncated header";
    S.natoms = ival(t[1]);
    if (S.natoms < S.nat0 || S.natoms > 10000000) return "lat_fc.dat: bad atom count";
    S.atompos.assign(3 * S.natoms, 0.0);
    S.cell0.assign(S.natoms, 0);
    S.cell.assign(3 * S.natoms, 0);
    for (int n = 0; n < S.natoms; ++n) {
      if (!R.next(8, t)) return "End of lat_fc.dat file reached";
      int i = ival(t[0]);
      if (i < 1 || i > S.natoms) return "lat_fc.dat: atom index out of range";
      for (int x = 0; x < 3; ++x) S.atompos[3 * (i - 1) + x] = dval(t[1 + x]);
      S.cell0[i - 1] = ival(t[4]);
      for (int x = 0; x < 3; ++x) S.cell[3 * (i - 1) + x] = ival(t[5 + x]);
    }
    for (int n = 0; n < S.natoms; ++n)
      if (S.cell0[n] < 1 || S.cell0[n] > S.nat0) return "lat_fc.dat: iatomcell0 out of range";
  }
  // ------------------------------------------------------- fc2.dat / fc3.dat
  for (int rank = 2; rank <= 3; ++rank) {
    if (rank == 3 && S.include_fc[2] != 1) break;
    std::string fn = dir + (rank == 2 ? "/fc2.dat" : "/fc3.dat");
    Records R;
    if (!R.load(fn)) return "READ_FC234: file " + std::string(rank == 2 ? "fc2.dat" : "fc3.dat") + " does not exist";
    std::string hdr;
    R.line(hdr);
    const std::vector<size_t> lines = R.nonblank_records();
    const size_t mx = lines.size();
    if ((int)mx != S.nterms[rank - 1])
      return "READ_FC" + std::to_string(rank) + ": number of lines read inconsistent with lat_fc.dat";
    const int nv = 2 + 2 * rank + 1;
    auto& idx = rank == 2 ? S.t2 : S.t3;
    auto& val = rank == 2 ? S.f2 : S.f3;
    idx.resize(mx * 2 * rank);
    val.resize(mx);
    auto term = [&](size_t j, const std::vector<std::string_view>& v) {
      for (int c = 0; c < 2 * rank; ++c) idx[j * 2 * rank + c] = ival(v[2 + c]);
      val[j] = dval(v[nv - 1]);
      for (int c = 0; c < rank; ++c) {
        int at = idx[j * 2 * rank + 2 * c], xyz = idx[j * 2 * rank + 2 * c + 1];
        if (at < 1 || at > S.natoms || xyz < 1 || xyz > 3) return false;
      }
      return true;
    };
    // Each READ of a term takes at least one record and there are as many
    // nonblank records as terms, so in a file the reference accepts term j
    // is nonblank record j: the records are parsed on the worker pool.  A
    // record with fewer than nv values (a READ that would span records)
    // sends the file through the sequential reader, which fails where the
    // reference's READ does.
    std::atomic<bool> short_rec{false}, bad_index{false};
    const int nthr = (int)std::min<size_t>(pool_width(), mx / 256 + 1);
    run_parallel(nthr, [&](int w) {
      std::vector<std::string_view> v;
      for (size_t j = w; j < mx && !short_rec.load(std::memory_order_relaxed); j += nthr) {
        R.values(lines[j], v, nv);
        if ((int)v.size() < nv) short_rec = true;
        else if (!term(j, v)) bad_index = true;
      }
    });
    if (short_rec) {
      for (size_t j = 0; j < mx; ++j) {
        if (!R.next(nv, t)) return "fc file truncated";
        if (!term(j, t)) return "fc file: atom or xyz index out of range";
      }
    } else if (bad_index) {
      return "fc file: atom or xyz index out of range";
    }
  }
  {  // ------------------------------------------------ dielectric.params
    Records R;
    if (!R.load(dir + "/dielectric.params")) return "cannot open dielectric.params";
    if (!R.next(1, t)) return "dielectric.params: empty";
    S.born_flag = ival(t[0]);
    for (int i = 0; i < 3; ++i) {
      if (!R.next(3, t)) return "dielectric.params: truncated";
      for (int j = 0; j < 3; ++j) S.epsil[i + 3 * j] = dval(t[j]);
    }
    S.charge.assign(9 * S.nat0, 0.0);
    for (int k = 0; k < S.nat0; ++k)
      for (int i = 0; i < 3; ++i) {
        if (!R.next(3, t)) {
          if (S.born_flag != 0) return "dielectric.params: truncated Born charges";
          break;
        }
        for (int j = 0; j < 3; ++j) S.charge[9 * k + i + 3 * j] = dval(t[j]);
      }
  }
  {  // --------------------------------------------------- b200.params
    std::ifstream f(dir + "/b200.params");
    std::string key, v;
    while (f >> key >> v) {
      if (key == "delta") S.delta = (v == "gauss") ? ALD_DELTA_GAUSS : ALD_DELTA_TETRA;
      else if (key == "precision") S.precision = (v == "mixed") ? ALD_MIXED : ALD_FP64;
      else if (key == "cg_stop") S.cg_stop = (v == "residual") ? ALD_CG_RESIDUAL : ALD_CG_REFERENCE;
      else if (key == "cg_tol") S.cg_tol = dval(v);
      else if (key == "width_cm") S.width_cm = dval(v);
    }
  }
  if (S.nc[0] < 1 || S.nc[1] < 1 || S.nc[2] < 1) return "latdyn.params: bad mesh";
  return "";
}

// ======================================================================
// nearest integer by conversion (no libm call); a fraction of exactly .5
// rounds away from zero, which the tolerance tests below reject either way
static inline double round_near(double x) { return (double)(long long)(x + (x >= 0 ? 0.5 : -0.5)); }

std::string build_tables(const System& S, Tables& T) {
  const int N0 = S.nc[0], N1 = S.nc[1], N2 = S.nc[2];
  T.nkc = N0 * N1 * N2;
  T.b = 3 * S.nat0;
  T.shifted = (N0 % 2 == 0 && N1 % 2 == 0 && N2 % 2 == 0);
  // ---- conventional / primitive frames and the lattice point group
  double latp[6];
  std::memcpy(latp, S.latp, sizeof latp);
  double d2r = 4.0 * std::atan(1.0) / 180.0;
  for (int i = 3; i < 6; ++i) latp[i] *= d2r;
  double conv_to_cart[9] = {0};
  conv_to_cart[cm(0, 0)] = latp[0];
  conv_to_cart[cm(0, 1)] = latp[1] * std::cos(latp[5]);
  conv_to_cart[cm(1, 1)] = latp[1] * std::sin(latp[5]);
  conv_to_cart[cm(0, 2)] = latp[2] * std::cos(latp[4]);
  conv_to_cart[cm(1, 2)] = latp[2] * (std::cos(latp[3]) - std::cos(latp[5]) * std::cos(latp[4])) / std::sin(latp[5]);
  conv_to_cart[cm(2, 2)] = std::sqrt(latp[2] * latp[2] - conv_to_cart[cm(0, 2)] * conv_to_cart[cm(0, 2)] -
                                     conv_to_cart[cm(1, 2)] * conv_to_cart[cm(1, 2)]);
  {  // make_reciprocal_lattice_2pi of the conventional cell (force_constants.f90:100-104)
    const double* c1 = &conv_to_cart[0];
    const double* c2 = &conv_to_cart[3];
    const double* c3 = &conv_to_cart[6];
    const double* cc[3][2] = {{c2, c3}, {c3, c1}, {c1, c2}};
    double x[3][3];
    for (int v = 0; v < 3; ++v) {
      const double *u = cc[v][0], *w = cc[v][1];
      x[v][0] = u[1] * w[2] - u[2] * w[1];
      x[v][1] = u[2] * w[0] - u[0] * w[2];
      x[v][2] = u[0] * w[1] - u[1] * w[0];
    }
    const double om = c1[0] * x[0][0] + c1[1] * x[0][1] + c1[2] * x[0][2];
    for (int v = 0; v < 3; ++v)
      for (int i = 0; i < 3; ++i) T.gconv[v][i] = 2 * PhysConst::pi * x[v][i] / om;
  }
  double prim_to_cart[9], conv_to_prim[9];
  mat3mul(conv_to_cart, S.primlatt, prim_to_cart);
  if (!mat3inv(S.primlatt, conv_to_prim)) return "primitive_lattice is singular";
  std::vector<std::array<int, 9>> ops;
  std::string e = lattice_point_group(prim_to_cart, ops);
  if (!e.empty()) return e;
  T.npg = (int)ops.size();
  for (int o = 0; o < T.npg; ++o) {
    // k transformation in the conventional frame: ((P I P^-1)^-1)^T, entries rounded
    double m[9], t1[9], t2[9], inv[9];
    for (int i = 0; i < 9; ++i) m[i] = ops[o][i];
    mat3mul(m, conv_to_prim, t1);
    mat3mul(S.primlatt, t1, t2);
    if (!mat3inv(t2, inv)) return "singular point operation";
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) T.opk[o][cm(i, j)] = (double)std::lround(inv[cm(j, i)]);
  }
  // ---- the mesh of make_kp_reg: fractions are default-REAL quotients
  T.kpc32.assign(3 * (size_t)T.nkc, 0.0);
  for (int i = 0; i < N0; ++i)
    for (int j = 0; j < N1; ++j)
      for (int k = 0; k < N2; ++k) {
        size_t n = (size_t)k + (size_t)N2 * (j + (size_t)N1 * i);
        double f0 = (double)((float)i / (float)N0), f1 = (double)((float)j / (float)N1),
               f2 = (double)((float)k / (float)N2);
        for (int x = 0; x < 3; ++x) {
          double q = ((f0 * S.g[0][x] + f1 * S.g[1][x]) + f2 * S.g[2][x]);
          if (T.shifted) q += (-0.5) * ((S.g[0][x] + S.g[1][x]) + S.g[2][x]);
          T.kpc32[3 * n + x] = q;
        }
      }
  auto mesh_index = [&](int a, int b, int c) { return c + N2 * (b + N1 * a); };
  auto wrap = [](int v, int n) { return ((v % n) + n) % n; };
  // reduced k-coordinates of mesh point m are (m_a/N_a - s/2): keep twice-N integers
  // h_a = 2*m_a - s*N_a so that f_a = h_a / (2 N_a) exactly
  auto h_of = [&](int n, int* h) {
    int m[3] = {n / (N1 * N2), (n / N2) % N1, n % N2};
    for (int a = 0; a < 3; ++a) h[a] = 2 * m[a] - (T.shifted ? S.nc[a] : 0);
  };
  // point-group action on reduced k coordinates: Rk = G^-1 OPK G with G = [g1 g2 g3]
  double G[9], Ginv[9];
  for (int a = 0; a < 3; ++a)
    for (int x = 0; x < 3; ++x) G[cm(x, a)] = S.g[a][x];
  if (!mat3inv(G, Ginv)) return "singular reciprocal lattice";
  std::vector<std::array<double, 9>> rk(T.npg);  // reduced-frame rational action
  for (int o = 0; o < T.npg; ++o) {
    double t1[9], t2[9];
    mat3mul(T.opk[o], G, t1);
    mat3mul(Ginv, t1, t2);
    for (int i = 0; i < 9; ++i) rk[o][i] = t2[i];
  }
  // map reduced coordinates (h_a / 2N_a) of a rotated point back to a mesh
  // index; returns -1 when the point is not on the mesh, and reports
  // whether it lies inside the cell the mesh spans (exact match) or only a
  // reciprocal-lattice vector away (folded)
  auto locate = [&](const double* f, bool& in_cell) -> int {
    int m[3];
    in_cell = true;
    for (int a = 0; a < 3; ++a) {
      double x = f[a] * S.nc[a] + (T.shifted ? 0.5 * S.nc[a] : 0.0);
      double r = round_near(x);
      // x is in units of one mesh step; FP32 mesh fractions leave ~1e-6 noise
      if (std::fabs(r - x) > 1e-3) return -1;
      long ir = (long)r;
      if (ir < 0 || ir >= S.nc[a]) in_cell = false;
      m[a] = wrap((int)(ir % S.nc[a]), S.nc[a]);
    }
    return mesh_index(m[0], m[1], m[2]);
  };
  // getstar: arms of the star of a Cartesian k (duplicates removed with the
  // reference's test on v.primitivelattice differences)
  auto star = [&](const double* kc, std::vector<std::array<double, 3>>& arms, std::vector<int>& armop) {
    arms.clear();
    armop.clear();
    std::array<double, 3> key[48];  // at most 48 point operations
    int nkey = 0;
    // keys hashed by the bucket of their first fractional part (width 2^-16 >
    // 2e-6): a key within 1e-6 of fr[0] (mod 1) sits in the same or a
    // neighbouring bucket, so only the keys of those three buckets are compared
    constexpr int kBuckets = 1 << 16, kSlots = 128;
    int head[kSlots], nxt[48], kb[48];
    std::fill(head, head + kSlots, -1);
    auto bucket = [&](double f) { return std::min(kBuckets - 1, (int)(f * kBuckets)); };
    for (int o = 0; o < T.npg; ++o) {
      double v[3], v2[3];
      for (int a = 0; a < 3; ++a) {
        double s = 0;
        for (int b = 0; b < 3; ++b) s = s + T.opk[o][cm(a, b)] * kc[b];
        v[a] = s;
      }
      for (int a = 0; a < 3; ++a) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s = s + v[k] * S.primlatt[cm(k, a)];
        v2[a] = s;
      }
      // v2 - key within 1e-6 of integers in every component: compared on the
      // fractional parts, |fa - fb| <= 1e-6 or >= 1 - 1e-6
      double fr[3];
      for (int c = 0; c < 3; ++c) fr[c] = v2[c] - std::floor(v2[c]);
      const int bk = bucket(fr[0]);
      bool dup = false;
      for (int db = -1; db <= 1 && !dup; ++db) {
        const int bb = (bk + db + kBuckets) % kBuckets;  // the mod-1 wrap
        for (int q = head[bb % kSlots]; q >= 0 && !dup; q = nxt[q]) {
          if (kb[q] != bb) continue;
          const auto& kk = key[q];
          int c;
          for (c = 0; c < 3; ++c) {
            const double d = std::fabs(fr[c] - kk[c]);
            if (d > 1e-6 && d < 1 - 1e-6) break;
          }
          if (c == 3) dup = true;
        }
      }
      if (dup) continue;
      kb[nkey] = bk;
      nxt[nkey] = head[bk % kSlots];
      head[bk % kSlots] = nkey;
      key[nkey++] = {fr[0], fr[1], fr[2]};
      arms.push_back({v[0], v[1], v[2]});
      armop.push_back(o);
    }
  };
  auto reduced = [&](const double* kc, double* f) {
    for (int a = 0; a < 3; ++a) f[a] = Ginv[cm(a, 0)] * kc[0] + Ginv[cm(a, 1)] * kc[1] + Ginv[cm(a, 2)] * kc[2];
  };
  // ---- tetrahedra (make_kp_reg_tet): six per mesh cell, corner table, and
  // per mesh point its 24 incidences (tetrahedron corner (6n+l)*4+k at the
  // point) in increasing order.  Both depend on the mesh only: two workers
  // build them (tet_corner, tet_inc) while the others find the stars of the
  // mesh points.  A point is corner c of cell point - offset(c) for each of
  // the 8 corner numbers c (offset bits x, y, z = c & 1, c & 2, c & 4).
  static const int corner_of[6][4] = {{0, 1, 2, 5}, {1, 2, 3, 5}, {0, 2, 4, 5},
                                      {2, 3, 5, 7}, {2, 4, 5, 6}, {2, 5, 6, 7}};
  // corner slots 4l + k of the six tetrahedra at each corner number, ascending
  int slots[8][6], nslot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int l = 0; l < 6; ++l)
    for (int k = 0; k < 4; ++k) {
      const int c = corner_of[l][k];
      slots[c][nslot[c]++] = 4 * l + k;
    }
  auto up = [](int v, int n) { return v + 1 == n ? 0 : v + 1; };
  auto down = [](int v, int n) { return v == 0 ? n - 1 : v - 1; };
  auto build_tet_corner = [&]() {
    T.tet_corner.assign(24 * (size_t)T.nkc, 0);
    for (int n = 0; n < T.nkc; ++n) {
      const int m0 = n / (N1 * N2), m1 = (n / N2) % N1, m2 = n % N2;
      const int a[2] = {m0, up(m0, N0)}, b[2] = {m1, up(m1, N1)}, c2[2] = {m2, up(m2, N2)};
      int pt[8];
      for (int c = 0; c < 8; ++c) pt[c] = mesh_index(a[c & 1], b[(c >> 1) & 1], c2[c >> 2]);
      for (int l = 0; l < 6; ++l)
        for (int k = 0; k < 4; ++k) T.tet_corner[4 * (6 * (size_t)n + l) + k] = pt[corner_of[l][k]];
    }
  };
  // incidence (6n + l) * 4 + k = 24 n + slot: the runs of the 8 cells,
  // each ascending, concatenated in increasing cell order
  auto build_tet_inc = [&]() {
    T.tet_inc.assign(24 * (size_t)T.nkc, 0);
    for (int p = 0; p < T.nkc; ++p) {
      const int m0 = p / (N1 * N2), m1 = (p / N2) % N1, m2 = p % N2;
      const int a[2] = {m0, down(m0, N0)}, b[2] = {m1, down(m1, N1)}, c2[2] = {m2, down(m2, N2)};
      int cell[8], ord[8];
      for (int c = 0; c < 8; ++c) {
        cell[c] = mesh_index(a[c & 1], b[(c >> 1) & 1], c2[c >> 2]);
        ord[c] = c;
      }
      for (int i = 1; i < 8; ++i)
        for (int j = i; j > 0 && cell[ord[j - 1]] > cell[ord[j]]; --j) std::swap(ord[j - 1], ord[j]);
      int* v = &T.tet_inc[24 * (size_t)p];
      int nv = 0;
      bool dup = false;
      for (int i = 0; i < 8; ++i) {
        const int c = ord[i];
        dup |= i > 0 && cell[ord[i - 1]] == cell[c];
        for (int s2 = 0; s2 < nslot[c]; ++s2) v[nv++] = 24 * cell[c] + slots[c][s2];
      }
      if (dup) std::sort(v, v + nv);  // an edge of 1 or 2 points: one cell at several corners
    }
  };
  // ---- IBZ (get_weights): first mesh point of each exact (unfolded) orbit
  T.mapibz.assign(T.nkc, 0);
  T.mapinv.clear();
  std::vector<double> w;
  std::vector<std::array<double, 3>> arms;
  std::vector<int> armop;
  // The stars of all mesh points are independent: they are found on host
  // threads first, as per point the mesh index of each arm in star order
  // (-2: off the mesh or outside its cell, -1: end of the list); the pass
  // that assigns IBZ points is sequential, as in the reference.
  const int npg = T.npg;
  // getstar + locate for one mesh point, as star() and the reduced/locate
  // steps above, with each op's two products folded into one matrix per
  // frame: v2 = (primlatt^T opk) k for the duplicate test, f = (G^-1 opk) k
  // for the mesh index (reordered sums: the 1e-6 duplicate tolerance and the
  // 1e-3 mesh tolerance are far above their rounding).  out[c] is the mesh
  // index of the c-th distinct arm, -2 where it is off the mesh or outside
  // its cell; the list ends at -1, or at the first arm on a mesh point
  // before n (the point's own index).
  std::vector<std::array<double, 9>> opv2(npg), opf(npg);
  for (int o = 0; o < npg; ++o)
    for (int a = 0; a < 3; ++a)
      for (int b2 = 0; b2 < 3; ++b2) {
        double sv = 0, sf = 0;
        for (int k = 0; k < 3; ++k) {
          sv += S.primlatt[cm(k, a)] * T.opk[o][cm(k, b2)];
          sf += Ginv[cm(a, k)] * T.opk[o][cm(k, b2)];
        }
        opv2[o][3 * a + b2] = sv;
        opf[o][3 * a + b2] = sf;
      }
  auto mesh_star_cands = [&](const double* kc, int n, int* out) {
    constexpr int kBuckets = 1 << 16, kSlots = 128;
    double key[48][3];
    int head[kSlots], nxt[48], kb[48], nkey = 0;
    std::fill(head, head + kSlots, -1);
    for (int o = 0; o < npg; ++o) {
      const double* A = opv2[o].data();
      double fr[3];
      for (int a = 0; a < 3; ++a) {
        const double v2 = A[3 * a] * kc[0] + A[3 * a + 1] * kc[1] + A[3 * a + 2] * kc[2];
        fr[a] = v2 - std::floor(v2);
      }
      const int bk = std::min(kBuckets - 1, (int)(fr[0] * kBuckets));
      bool dup = false;
      for (int db = -1; db <= 1 && !dup; ++db) {
        const int bb = (bk + db + kBuckets) % kBuckets;
        for (int q = head[bb % kSlots]; q >= 0 && !dup; q = nxt[q]) {
          if (kb[q] != bb) continue;
          int c;
          for (c = 0; c < 3; ++c) {
            const double d = std::fabs(fr[c] - key[q][c]);
            if (d > 1e-6 && d < 1 - 1e-6) break;
          }
          if (c == 3) dup = true;
        }
      }
      if (dup) continue;
      kb[nkey] = bk;
      nxt[nkey] = head[bk % kSlots];
      head[bk % kSlots] = nkey;
      key[nkey][0] = fr[0];
      key[nkey][1] = fr[1];
      key[nkey][2] = fr[2];
      const double* B = opf[o].data();
      double f[3];
      for (int a = 0; a < 3; ++a) f[a] = B[3 * a] * kc[0] + B[3 * a + 1] * kc[1] + B[3 * a + 2] * kc[2];
      bool in_cell;
      const int idx = locate(f, in_cell);
      out[nkey++] = idx >= 0 && in_cell ? idx : -2;
      // the pass below takes the first arm on an earlier mesh point (every
      // earlier point is assigned by then): nothing after it is read
      if (idx >= 0 && in_cell && idx < n) return;
    }
  };
  // on the library's worker pool: task 0 and 1 build the tetrahedron tables,
  // tasks 2.. take stripes of mesh points (four per worker, handed out as
  // workers come free: an IBZ point costs all npg arms, the others a few)
  std::vector<int> cand((size_t)T.nkc * npg, -1);
  {
    const int nstripe = 4 * pool_width();
    run_parallel(nstripe + 2, [&](int task) {
      if (task == 0) return build_tet_corner();
      if (task == 1) return build_tet_inc();
      const int t = task - 2;
      for (int n = t; n < T.nkc; n += nstripe) mesh_star_cands(&T.kpc32[3 * (size_t)n], n, &cand[(size_t)n * npg]);
    });
  }
  for (int n = 0; n < T.nkc; ++n) {
    int found = -1;
    for (int c = 0; c < npg; ++c) {
      const int idx = cand[(size_t)n * npg + c];
      if (idx == -1) break;
      if (idx >= 0 && idx < n && T.mapibz[idx] > 0) {
        found = T.mapibz[idx];
        break;
      }
    }
    if (found > 0) {
      T.mapibz[n] = found;
      w[found - 1] += 1.0;
    } else {
      T.mapinv.push_back(n + 1);
      w.push_back(1.0);
      T.mapibz[n] = (int)T.mapinv.size();
    }
  }
  T.nibz = (int)T.mapinv.size();
  double sw = 0;
  for (double x : w) sw += x;
  T.wibz.resize(T.nibz);
  T.kibz.resize(3 * (size_t)T.nibz);
  for (int i = 0; i < T.nibz; ++i) {
    T.wibz[i] = w[i] / sw;
    for (int x = 0; x < 3; ++x) T.kibz[3 * i + x] = T.kpc32[3 * (size_t)(T.mapinv[i] - 1) + x];
  }
  // ---- get_negatives + subst_eivecs: e(q_pos) := conj(e(q_neg))
  for (int n = 0; n < T.nkc; ++n) {
    int h[3], m[3];
    h_of(n, h);
    for (int a = 0; a < 3; ++a) {
      int hm = -h[a] + (T.shifted ? S.nc[a] : 0);  // 2*m' for -q
      m[a] = wrap(hm / 2, S.nc[a]);
    }
    int mk = mesh_index(m[0], m[1], m[2]);
    if (mk < n) {  // n is in the negative list; its partner mk gets conj(e(n))
      T.neg_src.push_back(n);
      T.neg_dst.push_back(mk);
    }
  }
  // ---- star arms per IBZ point: mesh arms (kstarsinfbz1) and folded arms.
  // Per IBZ point (host threads): its arms as (index, op, in cell), or an
  // index of -1 when an arm is off the mesh; then concatenated in order.
  {
    std::vector<int> aq((size_t)T.nibz * npg, -1), ao((size_t)T.nibz * npg, 0), ain((size_t)T.nibz * npg, 0),
        na(T.nibz, 0);
    const int nthr = pool_width();
    run_parallel(nthr, [&](int t) {
      std::vector<std::array<double, 3>> ar;
      std::vector<int> op;
      for (int i = t; i < T.nibz; i += nthr) {
        star(&T.kibz[3 * (size_t)i], ar, op);
        na[i] = (int)ar.size();
        for (size_t c = 0; c < ar.size(); ++c) {
          double f[3];
          reduced(ar[c].data(), f);
          bool in_cell;
          aq[(size_t)i * npg + c] = locate(f, in_cell);
          ao[(size_t)i * npg + c] = op[c];
          ain[(size_t)i * npg + c] = in_cell ? 1 : 0;
        }
      }
    });
    T.arm_off.assign(1, 0);
    T.star_off.assign(1, 0);
    for (int i = 0; i < T.nibz; ++i) {
      for (int c = 0; c < na[i]; ++c) {
        const size_t k = (size_t)i * npg + c;
        if (aq[k] < 0) return "star arm is not a kpoint";
        if (ain[k]) {
          T.arm_q.push_back(aq[k]);
          T.arm_op.push_back(ao[k]);
        }
        T.star_q.push_back(aq[k]);
        T.star_op.push_back(ao[k]);
      }
      T.arm_off.push_back((int)T.arm_q.size());
      T.star_off.push_back((int)T.star_q.size());
    }
  }
  // ---- exact phases: q(m).R_j = 2 pi sum_a (m_a/N_a - s/2) n_ja
  long L = 1;
  for (int a = 0; a < 3; ++a) L = std::lcm(L, (long)S.nc[a]);
  if (T.shifted && L % 2) L *= 2;
  if (L > (1 << 20)) return "mesh too large for the phase table";
  T.L = (int)L;
  T.phase_coef.assign(4 * (size_t)S.natoms, 0);
  for (int j = 0; j < S.natoms; ++j) {
    int j0 = S.cell0[j] - 1;
    // check the lattice vector of lat_fc.dat against the positions
    for (int x = 0; x < 3; ++x) {
      double R = S.atompos[3 * j + x] - S.atompos[3 * j0 + x];
      double Rn = S.cell[3 * j] * S.r[0][x] + S.cell[3 * j + 1] * S.r[1][x] + S.cell[3 * j + 2] * S.r[2][x];
      if (std::fabs(R - Rn) > 1e-5 * (1 + std::fabs(R)))
        return "lat_fc.dat: atom " + std::to_string(j + 1) + " position is not its cell vector n1 n2 n3";
    }
    long s = 0;
    for (int a = 0; a < 3; ++a) {
      long c = (long)S.cell[3 * j + a] * (L / S.nc[a]);
      T.phase_coef[4 * j + a] = (int)(((c % L) + L) % L);
      s += S.cell[3 * j + a];
    }
    T.phase_coef[4 * j + 3] = T.shifted ? (int)((((s * (L / 2)) % L) + L) % L) : 0;
  }
  return "";
}

// ======================================================================
std::string build_fc3(const System& S, Fc3Blocks& F) {
  int nb = S.nat0;
  int nt = (int)S.f3.size();
  struct Key {
    int blk, j, k;
  };
  // map (i0, j, k) -> triple
  std::unordered_map<long long, int> where;
  std::vector<Key> keys;
  std::vector<std::array<double, 27>> vals;
  for (int t = 0; t < nt; ++t) {
    const int* id = &S.t3[6 * t];
    int i = id[0] - 1, j = id[2] - 1, k = id[4] - 1;
    if (S.cell0[i] != i + 1) continue;  // first index must be in the primitive cell
    int i0 = i, j0 = S.cell0[j] - 1, k0 = S.cell0[k] - 1;
    long long key = ((long long)i0 * S.natoms + j) * S.natoms + k;
    auto it = where.find(key);
    int tr;
    if (it == where.end()) {
      tr = (int)keys.size();
      where[key] = tr;
      keys.push_back({(i0 * nb + j0) * nb + k0, j, k});
      vals.push_back({});
      vals.back().fill(0.0);
    } else {
      tr = it->second;
    }
    double mi = S.mass0[i0], mj = S.mass0[j0], mk = S.mass0[k0];
    int comp = (id[1] - 1) * 9 + (id[3] - 1) * 3 + (id[5] - 1);
    vals[tr][comp] += S.f3[t] / std::sqrt(mi * mj * mk);
  }
  int nblk = nb * nb * nb;
  std::vector<int> order(keys.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return keys[a].blk < keys[b].blk; });
  F.ntrip = (int)keys.size();
  F.blk_off.assign(nblk + 1, 0);
  F.trip_j.resize(F.ntrip);
  F.trip_k.resize(F.ntrip);
  F.w.resize(27 * (size_t)F.ntrip);
  for (int n = 0; n < F.ntrip; ++n) {
    const Key& kk = keys[order[n]];
    F.blk_off[kk.blk + 1]++;
    F.trip_j[n] = kk.j;
    F.trip_k[n] = kk.k;
    for (int c = 0; c < 27; ++c) F.w[27 * (size_t)n + c] = vals[order[n]][c];
  }
  for (int b = 0; b < nblk; ++b) F.blk_off[b + 1] += F.blk_off[b];
  return "";
}

std::string build_v3_classes(const System& S, const Tables& T, const Fc3Blocks& F, V3Classes& C) {
  const int nb = S.nat0, L = T.L;
  struct Cls {
    int g, d[3];
    std::vector<int> members;
  };
  std::map<std::array<int, 4>, int> where;  // (g, d) -> class
  std::vector<Cls> cls;
  std::vector<int> owner_i0(F.ntrip);
  for (int blk = 0; blk < nb * nb * nb; ++blk)
    for (int t = F.blk_off[blk]; t < F.blk_off[blk + 1]; ++t) owner_i0[t] = blk / (nb * nb);
  for (int t = 0; t < F.ntrip; ++t) {
    const int j = F.trip_j[t], k = F.trip_k[t];
    const int j0 = S.cell0[j] - 1, k0 = S.cell0[k] - 1;
    std::array<int, 4> key = {j0 * nb + k0, S.cell[3 * j] - S.cell[3 * k], S.cell[3 * j + 1] - S.cell[3 * k + 1],
                              S.cell[3 * j + 2] - S.cell[3 * k + 2]};
    auto it = where.find(key);
    int c;
    if (it == where.end()) {
      c = (int)cls.size();
      where[key] = c;
      cls.push_back({key[0], {key[1], key[2], key[3]}, {}});
    } else {
      c = it->second;
    }
    cls[c].members.push_back(t);
  }
  // group order; within a group, first appearance order
  std::vector<int> order(cls.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cls[a].g < cls[b].g; });
  C.ncls = (int)cls.size();
  C.grp_off.assign(nb * nb + 1, 0);
  C.pc.assign(4 * (size_t)C.ncls, 0);
  C.trip_off.assign(1, 0);
  C.trip.clear();
  C.trip_i0.clear();
  C.trip_k.clear();
  for (int n = 0; n < C.ncls; ++n) {
    const Cls& c = cls[order[n]];
    C.grp_off[c.g + 1]++;
    // phase of q(m).(R_j - R_k): the difference of the two atoms' coefficients
    const int j = F.trip_j[c.members[0]], k = F.trip_k[c.members[0]];
    for (int a = 0; a < 4; ++a) {
      long v = (long)T.phase_coef[4 * j + a] - (long)T.phase_coef[4 * k + a];
      C.pc[4 * (size_t)n + a] = (int)(((v % L) + L) % L);
    }
    for (int t : c.members) {
      C.trip.push_back(t);
      C.trip_i0.push_back(owner_i0[t]);
      C.trip_k.push_back(F.trip_k[t]);
    }
    C.trip_off.push_back((int)C.trip.size());
  }
  for (int g = 0; g < nb * nb; ++g) C.grp_off[g + 1] += C.grp_off[g];
  return "";
}

std::string build_fc2(const System& S, Fc2Csr& F) {
  int b = 3 * S.nat0;
  int nt = (int)S.f2.size();
  std::vector<std::vector<int>> per(b * b);
  for (int t = 0; t < nt; ++t) {
    const int* id = &S.t2[4 * t];
    int i = id[0], al = id[1], j = id[2], be = id[3];
    if (i < 1 || i > S.nat0) continue;  // rows are primitive-cell atoms only
    int j0 = S.cell0[j - 1];
    int i3 = (al - 1) + 3 * (i - 1), j3 = (be - 1) + 3 * (j0 - 1);
    per[i3 * b + j3].push_back(t);
  }
  F.off.assign(b * b + 1, 0);
  for (int e = 0; e < b * b; ++e) F.off[e + 1] = F.off[e] + (int)per[e].size();
  F.atom.resize(F.off[b * b]);
  F.val.resize(F.off[b * b]);
  F.sqm.resize(F.off[b * b]);
  for (int e = 0; e < b * b; ++e) {
    int i0 = e / b / 3;
    for (size_t s = 0; s < per[e].size(); ++s) {
      int t = per[e][s];
      int j = S.t2[4 * t + 2] - 1;
      int j0 = S.cell0[j] - 1;
      F.atom[F.off[e] + s] = j;
      F.val[F.off[e] + s] = S.f2[t];
      F.sqm[F.off[e] + s] = std::sqrt(S.mass0[i0] * S.mass0[j0]);
    }
  }
  F.uatom = F.atom;
  std::sort(F.uatom.begin(), F.uatom.end());
  F.uatom.erase(std::unique(F.uatom.begin(), F.uatom.end()), F.uatom.end());
  F.uidx.resize(F.atom.size());
  for (size_t t = 0; t < F.atom.size(); ++t)
    F.uidx[t] = (int)(std::lower_bound(F.uatom.begin(), F.uatom.end(), F.atom[t]) - F.uatom.begin());
  return "";
}

// Natural isotopic compositions (isotope mass in amu, abundance in percent)
// with the values of the reference's cal_g table (sub.f90:3766-4693), for the
// elements covered here; others need ald_set_isotope_g.
namespace {
struct IsoLine {
  const char* element;
  double mass, percent;
};
const IsoLine kIsotopes[] = {
    {"Ar", 35.967546, 0.34},  {"Ar", 37.962732, 0.063},  {"Ar", 39.962383, 99.6},   {"C", 12.0, 98.9},
    {"C", 13.003355, 1.1},    {"Cl", 34.968853, 75.77},  {"Cl", 36.965903, 24.23},  {"Ge", 69.92425, 20.5},
    {"Ge", 71.92208, 27.4},   {"Ge", 72.923464, 7.8},    {"Ge", 73.921179, 36.5},   {"Ge", 75.921403, 7.8},
    {"Na", 22.98977, 100.0},  {"Si", 27.976928, 92.23},  {"Si", 28.976496, 4.67},   {"Si", 29.973772, 3.1},
};
}  // namespace

bool isotope_g(const std::string& element, double& g) {
  // mass variance: mbar = sum m f / 100, g = sum f (1 - m/mbar)^2 / 100
  double mbar = 0;
  int n = 0;
  for (const IsoLine& x : kIsotopes)
    if (element == x.element) {
      mbar = mbar + x.mass * x.percent;
      ++n;
    }
  if (n == 0) return false;
  mbar = mbar / 100;
  g = 0;
  for (const IsoLine& x : kIsotopes)
    if (element == x.element) g = g + x.percent * (1 - (x.mass / mbar)) * (1 - (x.mass / mbar));
  g = g / 100;
  return true;
}

std::string isotope_g_atoms(const System& S, std::vector<double>& g) {
  g.assign(S.nat0, 0.0);
  for (int i = 0; i < S.nat0; ++i) {
    const int t = S.atype[i];
    if (t < 1 || t > (int)S.atname.size()) return "isotope scattering: atom type without an element name";
    if (!isotope_g(S.atname[t - 1], g[i]))
      return "isotope scattering: no isotope data for element " + S.atname[t - 1] + " (ald_set_isotope_g)";
  }
  return "";
}

cudaError_t raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(m);
  size_t& cur = done[{func, dev}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

}  // namespace ald
