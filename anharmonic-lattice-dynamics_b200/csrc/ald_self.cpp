// The three-phonon self-energy of THERMACOND's job=2 block (kappa.f90:874-1040)
// through the C ABI: the band path of kpbs.params (make_kp_bs,
// modules.f90:1507-1652), eigenpairs at the path points and at every
// k3 = -q - k2 (the phonon kernel on point lists), function_self_w3/w4
// (rest.f90:4012-4240) on the device (ald_self.cu), and the files
// lw-selfenergy.dat / lw-selfenergy2.dat in the reference's list-directed
// layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ald_ctx.h"
#include "ald_fortran_io.h"

using namespace ald;
using namespace ald::capi;

namespace {

// make_kp_bs: kp (3*nkp) Cartesian, dk (nkp); units 0 = conventional reciprocal
// vectors, anything else primitive (the file's first record)
std::string make_kp_bs(const ald_ctx* c, const std::string& dir, std::vector<double>& kp, std::vector<double>& dk) {
  FILE* f = std::fopen((dir + "/kpbs.params").c_str(), "r");
  if (!f) return "MAKE_KP_BS: " + dir + "/kpbs.params does not exist";
  std::vector<std::string> lines;
  char buf[1024];
  while (std::fgets(buf, sizeof buf, f)) {
    for (char* p = buf; *p; ++p)
      if (*p == ',') *p = ' ';
    lines.emplace_back(buf);
  }
  std::fclose(f);
  int units = 0, nkdir = 0, ndir = 0;
  if (lines.size() < 3 || std::sscanf(lines[0].c_str(), "%d", &units) != 1 ||
      std::sscanf(lines[1].c_str(), "%d", &nkdir) != 1 || std::sscanf(lines[2].c_str(), "%d", &ndir) != 1)
    return "MAKE_KP_BS: kpbs.params must start with units, nkdir, ndir";
  if (nkdir < 1 || ndir < 1) return "MAKE_KP_BS: nkdir and ndir must be positive";
  if ((int)lines.size() < 4 + ndir) return "MAKE_KP_BS: kpbs.params lists fewer than ndir+1 points";
  std::vector<double> ext((size_t)3 * (ndir + 1));
  for (int i = 0; i <= ndir; ++i) {
    char name[256];
    if (std::sscanf(lines[3 + i].c_str(), "%255s %lf %lf %lf", name, &ext[3 * i], &ext[3 * i + 1],
                    &ext[3 * i + 2]) != 4)
      return "MAKE_KP_BS: bad point record: " + lines[3 + i];
  }
  const double* B[3];
  for (int v = 0; v < 3; ++v) B[v] = units == 0 ? c->T.gconv[v] : c->S.g[v];
  auto cart = [&](const double* e, double* out) {  // e1*b1 + e2*b2 + e3*b3
    for (int x = 0; x < 3; ++x) out[x] = e[0] * B[0][x] + e[1] * B[1][x] + e[2] * B[2][x];
  };
  kp.assign((size_t)3 * ndir * nkdir, 0.0);
  dk.assign((size_t)ndir * nkdir, 0.0);
  int nk = 0;
  for (int i = 0; i < ndir; ++i) {
    double ki[3], kf[3], q[3];
    cart(&ext[3 * i], ki);
    cart(&ext[3 * (i + 1)], kf);
    double lk = 0;
    for (int x = 0; x < 3; ++x) {
      q[x] = kf[x] - ki[x];
      lk = lk + q[x] * q[x];
    }
    lk = std::sqrt(lk);
    for (int j = 1; j <= nkdir; ++j) {
      ++nk;
      dk[nk - 1] = nk >= 2 ? (j >= 2 ? dk[nk - 2] + lk / (nkdir - 1 + 1e-8) : dk[nk - 2]) : 0.0;
      for (int x = 0; x < 3; ++x) kp[3 * (nk - 1) + x] = ki[x] + (j - 1) * q[x] / (nkdir - 1 + 1e-8);
    }
  }
  return "";
}

// eigenpairs at n points (d_pts: 3*n on the device): |lambda| sorted
// (get_frequencies' order) and the eigenvectors in that order
int points_eigen(ald_ctx* c, int n, const double* d_pts, double* d_w2, double* d_evec, double* d_w2all) {
  PhononArgs a;
  a.geo = c->geo;
  a.geo.nkc = n;
  a.kpc32 = d_pts;
  a.g = nullptr;
  a.fc2_off = c->fc2_off.p;
  a.fc2_atom = c->fc2_atom.p;
  a.fc2_val = c->fc2_val.p;
  a.fc2_sqm = c->fc2_sqm.p;
  a.fc2_uatom = c->fc2_uatom.p;
  a.fc2_uidx = c->fc2_uidx.p;
  a.nuniq = (int)c->F2.uatom.size();
  a.rr = c->rr.p;
  a.born_flag = c->S.born_flag;
  a.born = c->born.p;
  a.dq = (double)0.001f;
  a.ndisp = 1;
  a.w2_all = d_w2all;
  a.w2 = d_w2;
  a.evec = d_evec;
  a.err = c->err.p;
  ALD_CK(launch_phonons(a, c->stream));
  return ALD_OK;
}

// Self-energies of np points q (host, 3*np) for every band, target
// frequencies omega (np*b, [p*b + la]; NULL = omega0 of each mode),
// temperature temp in cm^-1.  out: np*b*4 (nself re, im, uself re, im);
// omega0 (optional): np*b.
int self_points(ald_ctx* c, int np, const double* q, const double* omega, double temp, int gauss,
                std::vector<double>& out, std::vector<double>* omega0) {
  if (c->S.include_fc[2] != 1) return fail(ALD_ERR_ARG, "fc3 terms are not included (include_fc(3) /= 1)");
  int r = ensure_phonons(c);
  if (r) return r;
  const int b = c->geo.b, nkc = c->T.nkc;
  if (b > 12) return fail(ALD_ERR_UNSUPPORTED, "self-energy: more than 12 bands is not supported by this build");
  const double cn = PhysConst::cnst();
  // path eigenpairs
  DevBuf<double> dq, wq, evq, wall;
  ALD_CKA(dq.alloc((size_t)3 * np));
  ALD_CKA(wq.alloc((size_t)np * b));
  ALD_CKA(evq.alloc((size_t)np * b * b * 2));
  ALD_CKA(wall.alloc((size_t)np * b));
  ALD_CK(cudaMemcpyAsync(dq.p, q, (size_t)3 * np * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  r = points_eigen(c, np, dq.p, wq.p, evq.p, wall.p);
  if (r) return r;
  std::vector<double> hw((size_t)np * b), om((size_t)np * b);
  ALD_CK(cudaMemcpyAsync(hw.data(), wq.p, hw.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ALD_CK(cudaStreamSynchronize(c->stream));
  r = check_err_flags(c);
  if (r) return r;
  for (size_t i = 0; i < hw.size(); ++i) om[i] = omega ? omega[i] : std::sqrt(std::fabs(hw[i])) * cn;
  if (omega0)
    for (size_t i = 0; i < hw.size(); ++i) (*omega0)[i] = std::sqrt(std::fabs(hw[i])) * cn;
  DevBuf<double> dom;
  ALD_CKA(dom.alloc(om.size()));
  ALD_CK(cudaMemcpyAsync(dom.p, om.data(), om.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  // the dual basis of g (check_inside_bz)
  SelfArgs s;
  {
    const double* g1 = c->S.g[0];
    const double* g2 = c->S.g[1];
    const double* g3 = c->S.g[2];
    const double* gg[3][2] = {{g2, g3}, {g3, g1}, {g1, g2}};
    double x[3][3];
    for (int v = 0; v < 3; ++v) {
      const double *u = gg[v][0], *w = gg[v][1];
      x[v][0] = u[1] * w[2] - u[2] * w[1];
      x[v][1] = u[2] * w[0] - u[0] * w[2];
      x[v][2] = u[0] * w[1] - u[1] * w[0];
    }
    const double o = x[0][0] * g1[0] + x[0][1] * g1[1] + x[0][2] * g1[2];
    for (int v = 0; v < 3; ++v)
      for (int i = 0; i < 3; ++i) s.gd[3 * v + i] = x[v][i] / o;
    for (int i = 0; i < 3; ++i) s.ghalf[i] = 0.5 * ((g1[i] + g2[i]) + g3[i]);
  }
  s.b = b;
  s.nkc = nkc;
  s.nat0 = c->S.nat0;
  s.kpc = c->kpc32.p;
  s.ev2 = c->evec.p;
  s.w2 = c->w2.p;
  s.ntrip = c->F3.ntrip;
  s.natoms = c->S.natoms;
  s.blk_off = c->blk_off.p;
  s.trip_j = c->trip_j.p;
  s.trip_k = c->trip_k.p;
  s.fc3w = c->fc3w.p;
  s.rr = c->rr.p;
  s.temp = temp;
  s.eta = c->S.etaz;
  s.etacut = gauss ? c->S.etaz * 6 : c->S.etaz * 3000;
  s.cnst = cn;
  s.const33 = PhysConst::const33();
  s.pi = PhysConst::pi;
  s.v3thr = (double)1e-7f;  // v3_threshold = 1E-7, a default-REAL literal (rest.f90:47)
  s.classical = c->S.classical;
  s.gauss = gauss;
  s.err = c->err.p;
  // path points in chunks: eigenpairs at np_chunk * nkc points k3 at a time
  const int chunk = std::max(1, std::min(np, (int)((size_t)262144 / (size_t)nkc)));
  s.np = chunk;
  DevBuf<double> k3, w3, ev3, w3all, part, dout;
  ALD_CKA(k3.alloc((size_t)3 * chunk * nkc));
  ALD_CKA(w3.alloc((size_t)chunk * nkc * b));
  ALD_CKA(ev3.alloc((size_t)chunk * nkc * b * b * 2));
  ALD_CKA(w3all.alloc((size_t)chunk * nkc * b));
  ALD_CKA(part.alloc(self_partial_doubles(s)));
  ALD_CKA(dout.alloc((size_t)np * b * 4));
  for (int p0 = 0; p0 < np; p0 += chunk) {
    const int n = std::min(chunk, np - p0);
    ALD_CK(launch_k3_points(n, nkc, dq.p + 3 * (size_t)p0, c->kpc32.p, k3.p, c->stream));
    r = points_eigen(c, n * nkc, k3.p, w3.p, ev3.p, w3all.p);
    if (r) return r;
    s.np = n;
    s.qp = dq.p + 3 * (size_t)p0;
    s.omega = dom.p + (size_t)p0 * b;
    s.evq = evq.p + (size_t)p0 * b * b * 2;
    s.wq = wq.p + (size_t)p0 * b;
    s.ev3 = ev3.p;
    s.w3 = w3.p;
    s.part = part.p;
    ALD_CK(launch_self(s, dout.p + (size_t)p0 * b * 4, c->stream));
  }
  out.resize((size_t)np * b * 4);
  ALD_CK(cudaMemcpyAsync(out.data(), dout.p, out.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ALD_CK(cudaStreamSynchronize(c->stream));
  return check_err_flags(c);
}

struct OutFile {
  FILE* f = nullptr;
  ~OutFile() {
    if (f) std::fclose(f);
  }
};

}  // namespace

extern "C" {

int ald_make_kp_bs(ald_ctx* c, const char* dir, int* nkp_bs, double* kp_bs, double* dk_bs, int cap) {
  if (!c || !dir || !nkp_bs) return fail(ALD_ERR_ARG, "null argument");
  std::vector<double> kp, dk;
  std::string e = make_kp_bs(c, dir, kp, dk);
  if (!e.empty()) return fail(ALD_ERR_IO, e);
  *nkp_bs = (int)dk.size();
  if (kp_bs && dk_bs) {
    if (cap < *nkp_bs) return fail(ALD_ERR_ARG, "kp_bs/dk_bs hold fewer than nkp_bs points");
    std::memcpy(kp_bs, kp.data(), kp.size() * sizeof(double));
    std::memcpy(dk_bs, dk.data(), dk.size() * sizeof(double));
  }
  return ALD_OK;
}

int ald_function_self_w(ald_ctx* c, int n, const double* q, const int* la, const double* omega, double temp,
                        int gauss, double* nself, double* uself) {
  if (!c || n <= 0 || !q || !la || !omega || !nself || !uself) return fail(ALD_ERR_ARG, "bad argument");
  const int b = c->geo.b;
  for (int j = 0; j < n; ++j)
    if (la[j] < 1 || la[j] > b) return fail(ALD_ERR_ARG, "la out of range 1..ndyn");
  ALD_CK(cudaSetDevice(c->device));
  std::vector<double> om((size_t)n * b);
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < b; ++l) om[(size_t)j * b + l] = omega[j];
  std::vector<double> out;
  int r = self_points(c, n, q, om.data(), temp, gauss, out, nullptr);
  if (r) return r;
  for (int j = 0; j < n; ++j) {
    const double* o = &out[((size_t)j * b + la[j] - 1) * 4];
    nself[2 * j] = o[0];
    nself[2 * j + 1] = o[1];
    uself[2 * j] = o[2];
    uself[2 * j + 1] = o[3];
  }
  return ALD_OK;
}

int ald_self_energy_bs(ald_ctx* c, const char* dir, double tempk, int gauss, int nkp_bs, double* omega0,
                       double* nself, double* uself, const char* out_dir) {
  if (!c || !dir || !omega0 || !nself || !uself) return fail(ALD_ERR_ARG, "null argument");
  ALD_CK(cudaSetDevice(c->device));
  std::vector<double> kp, dk;
  std::string e = make_kp_bs(c, dir, kp, dk);
  if (!e.empty()) return fail(ALD_ERR_IO, e);
  const int np = (int)dk.size(), b = c->geo.b;
  if (nkp_bs != np) return fail(ALD_ERR_ARG, "nkp_bs differs from the path of kpbs.params");
  const double temp = tempk * PhysConst::k_b / (100 * PhysConst::h_plank * PhysConst::c_light);
  std::vector<double> out, om0((size_t)np * b);
  int r = self_points(c, np, kp.data(), nullptr, temp, gauss, out, &om0);
  if (r) return r;
  for (int p = 0; p < np; ++p)
    for (int l = 0; l < b; ++l) {
      const size_t m = (size_t)p * b + l;
      omega0[l + (size_t)b * p] = om0[m];  // omega0(ndyn, nkp_bs)
      nself[2 * m] = out[4 * m];
      nself[2 * m + 1] = out[4 * m + 1];
      uself[2 * m] = out[4 * m + 2];
      uself[2 * m + 1] = out[4 * m + 3];
    }
  if (!out_dir) return ALD_OK;
  // lw-selfenergy.dat, lw-selfenergy2.dat (kappa.f90:1019-1031)
  std::string d = *out_dir ? out_dir : ".";
  if (d.back() != '/') d += '/';
  OutFile f1, f2;
  f1.f = std::fopen((d + "lw-selfenergy.dat").c_str(), "w");
  f2.f = std::fopen((d + "lw-selfenergy2.dat").c_str(), "w");
  if (!f1.f || !f2.f) return fail(ALD_ERR_IO, "cannot open lw-selfenergy files in " + d + ": " + std::strerror(errno));
  for (int p = 0; p < np; ++p) {
    fio::ListRecord rec2;
    rec2.r(tempk).r(dk[p]);
    std::vector<double> tse(b);
    for (int l = 0; l < b; ++l) {
      const size_t m = (size_t)p * b + l;
      const double ise = 2 * (out[4 * m + 1] + out[4 * m + 3]);  // 2*aimag(nself+uself)
      tse[l] = 1e10 / PhysConst::c_light / ise;
      fio::ListRecord rec;
      rec.r(tempk).i(l + 1).i(p + 1).r(kp[3 * p]).r(kp[3 * p + 1]).r(kp[3 * p + 2]).r(dk[p]).r(om0[m]);
      rec.r(ise / 2).r(ise).r(tse[l]).r(1 / tse[l]);
      std::fprintf(f1.f, "%s\n", rec.str().c_str());
    }
    for (int l = 0; l < b; ++l) rec2.r(om0[(size_t)p * b + l]);
    for (int l = 0; l < b; ++l) rec2.r(1 / tse[l]);
    std::fprintf(f2.f, "%s\n", rec2.str().c_str());
  }
  return ALD_OK;
}

}  // extern "C"
