// The output files of the reference's job=1 run, written the way its
// gfortran build writes them:
//
//   Qvalue.dat             Qandtau          THERMACOND/sub.f90:8198-8305 (rewrites the file
//                                           calculate_tauRTA_mpi2 opened, sub.f90:7998-8000)
//   tau_RTA.dat,           write_kappa      THERMACOND/sub.f90:1818-1916, after mode_kappa
//   kappa_RTA.dat                           (kappa.f90:559-560, 690-691)
//   tau_RTAandeff-cg.dat,  write_kappa      after mode_kappa_d (kappa.f90:713-714, 866)
//   kappa_direct-cg.dat
//
// Two kinds of records occur.  List-directed ones (`write(u,*)`): every
// item is preceded by one blank (the first one too), except a character
// item that follows another character item; an INTEGER is I11, a REAL(8)
// 17 significant digits in a 25-character field -- F20.(17-s) and five
// blanks when 0 <= s <= 17 (10^(s-1) <= |x| < 10^s after rounding; s = 1
// for zero), otherwise 1PE25.16 with a three-digit exponent
// ("-1.3169752846541651E-022").  Formatted ones use Iw, Fw.d, Ew.d and Gw.d
// with the Fortran rules: the optional leading zero of a number below one
// is dropped when the field is too narrow for it, a field still too narrow
// is filled with '*', Gw.d uses F(w-4).(d-s) and four blanks when 0 <= s <=
// d and Ew.d otherwise, a G edit of an INTEGER is Iw, and infinities and
// NaNs read "Infinity"/"Inf"/"NaN" right-justified.  Decimal rounding is
// the C library's (round to nearest on the exact binary value), as in
// gfortran's runtime.  Trailing X edits of an exhausted format write
// nothing.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ald_ctx.h"
#include "ald_fortran_io.h"

using namespace ald;
using namespace ald::capi;

namespace ald {
namespace fio {

namespace {

std::string pad_left(const std::string& s, int w) {
  if ((int)s.size() > w) return std::string(w, '*');
  return std::string(w - s.size(), ' ') + s;
}

// |x| rounded to nd significant digits: the digits and s with
// 10^(s-1) <= |x| < 10^s for the rounded value (0.d1d2... x 10^s)
void sig_digits(double ax, int nd, std::string& dig, int& s) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.*e", nd - 1, ax);
  dig.clear();
  const char* p = buf;
  for (; *p && *p != 'e'; ++p)
    if (*p >= '0' && *p <= '9') dig.push_back(*p);
  s = std::atoi(p + 1) + 1;
}

std::string infnan(int w, double x) {
  if (std::isnan(x)) return pad_left("NaN", w);
  const bool neg = std::signbit(x);
  const int room = w - (neg ? 1 : 0);
  std::string t = room >= 8 ? "Infinity" : "Inf";
  return pad_left((neg ? "-" : "") + t, w);
}

// sign + body into w, dropping the optional leading zero of "0." if needed
std::string fit(bool neg, std::string body, int w) {
  const int sign = neg ? 1 : 0;
  if ((int)body.size() + sign > w && body.size() > 1 && body[0] == '0' && body[1] == '.') body.erase(0, 1);
  return pad_left((neg ? "-" : "") + body, w);
}

}  // namespace

std::string edit_I(int w, long long v) { return pad_left(std::to_string(v), w); }

std::string edit_F(int w, int d, double x) {
  if (!std::isfinite(x)) return infnan(w, x);
  std::vector<char> buf(360 + d);
  std::snprintf(buf.data(), buf.size(), "%.*f", d, std::fabs(x));
  std::string body = buf.data();
  if (d == 0) body += ".";
  return fit(std::signbit(x), body, w);
}

std::string edit_E(int w, int d, double x) {
  if (!std::isfinite(x)) return infnan(w, x);
  std::string dig;
  int s = 0;
  if (x == 0.0) {
    dig.assign(d, '0');
  } else {
    sig_digits(std::fabs(x), d, dig, s);
  }
  const int ae = std::abs(s);
  char ex[16];
  if (ae <= 99)
    std::snprintf(ex, sizeof ex, "E%c%02d", s < 0 ? '-' : '+', ae);
  else
    std::snprintf(ex, sizeof ex, "%c%03d", s < 0 ? '-' : '+', ae);
  return fit(std::signbit(x), "0." + dig + ex, w);
}

std::string edit_G(int w, int d, double x) {
  if (!std::isfinite(x)) return infnan(w, x);
  int s = 1;
  if (x != 0.0) {
    std::string dig;
    sig_digits(std::fabs(x), d, dig, s);
  }
  if (s < 0 || s > d) return edit_E(w, d, x);
  return edit_F(w - 4, d - s, x) + "    ";
}

// one list-directed REAL(8) field (25 characters, without the separator)
std::string list_real(double x) {
  if (!std::isfinite(x)) return infnan(25, x);
  int s = 1;
  std::string dig;
  if (x != 0.0) sig_digits(std::fabs(x), 17, dig, s);
  if (s >= 0 && s <= 17) return edit_F(20, 17 - s, x) + "     ";
  // 1PE25.16E3
  const int e = s - 1, ae = std::abs(e);
  char ex[16];
  std::snprintf(ex, sizeof ex, "E%c%03d", e < 0 ? '-' : '+', ae);
  std::string body = dig.substr(0, 1) + "." + dig.substr(1) + ex;
  return pad_left((std::signbit(x) ? "-" : "") + body, 25);
}

std::string list_int(long long v) { return pad_left(std::to_string(v), 11); }


}  // namespace fio
}  // namespace ald

namespace {

using namespace ald::fio;

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

int open_out(File& F, const char* path) {
  F.f = std::fopen(path, "w");
  if (!F.f) return fail(ALD_ERR_IO, std::string("cannot open ") + path + " for writing: " + std::strerror(errno));
  return ALD_OK;
}

void line(File& F, const std::string& s) {
  std::fputs(s.c_str(), F.f);
  std::fputc('\n', F.f);
}

// frequency, dist (nkc, b) [q*b + l] and veloc [(q*b + l)*3 + x] on the host
int mode_tables(ald_ctx* c, double tempk, std::vector<double>& freq, std::vector<double>& dist,
                std::vector<double>& vel) {
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  const size_t n = (size_t)c->T.nkc * c->geo.b;
  freq.resize(n);
  dist.resize(n);
  vel.resize(3 * n);
  ALD_CK(cudaMemcpyAsync(freq.data(), c->freq.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ALD_CK(cudaMemcpyAsync(dist.data(), c->dist.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ALD_CK(cudaMemcpyAsync(vel.data(), c->vel.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ALD_CK(cudaStreamSynchronize(c->stream));
  return ALD_OK;
}

// tauinv_eff per mode on the device; F [(i*b + l)*3 + x]; out (nibz, b) column-major
int tau_eff_dev(ald_ctx* c, double tempk, const std::vector<double>& F, int averaged, double* out) {
  const int nibz = c->T.nibz, b = c->geo.b;
  DevBuf<double> dF, dt;
  ALD_CKA(dF.alloc(F.size()));
  ALD_CKA(dt.alloc((size_t)nibz * b));
  ALD_CK(cudaMemcpyAsync(dF.p, F.data(), F.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  KappaArgs k = kappa_args(c, tempk);
  ALD_CK(launch_tau_eff(k, dF.p, averaged, dt.p, c->stream));
  std::vector<double> h((size_t)nibz * b);
  ALD_CK(cudaMemcpyAsync(h.data(), dt.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  ALD_CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < nibz; ++i)
    for (int l = 0; l < b; ++l) out[i + (size_t)nibz * l] = h[(size_t)i * b + l];
  return ALD_OK;
}

// Qandtau (sub.f90:8244-8285): Qvalue.dat and the inverse lifetimes
int qandtau(ald_ctx* c, const std::vector<double>& dist, const double* Q, const double* QN, const double* QU,
            const char* path, double* tN, double* tU, double* tT) {
  const int nibz = c->T.nibz, b = c->geo.b;
  File F;
  if (path) {
    int r = open_out(F, path);
    if (r) return r;
    line(F, ListRecord().c("nk,la,Q").str());
  }
  const double cl = PhysConst::c_light;
  for (int ibz = 1; ibz <= nibz; ++ibz)
    for (int ii = 1; ii <= b; ++ii) {
      const size_t m = (size_t)(ibz - 1) + (size_t)nibz * (ii - 1);
      const double nb1 = dist[(size_t)(c->T.mapinv[ibz - 1] - 1) * b + (ii - 1)];
      if (path) line(F, ListRecord().i(ibz).i(ii).r(Q[m]).r(Q[m] / (nb1 * (nb1 + 1))).str());
      tN[m] = QN[m] / (nb1 * (nb1 + 1)) * cl * 100;
      tU[m] = QU[m] / (nb1 * (nb1 + 1)) * cl * 100;
      tT[m] = tN[m] + tU[m];
    }
  return ALD_OK;
}

// write_kappa (sub.f90:1818-1916)
int write_kappa(ald_ctx* c, double tempk, const std::vector<double>& freq, const std::vector<double>& dist,
                const std::vector<double>& vel, const double* kappa, double* tN, double* tU, const double* tT,
                const double* teff, const char* kappa_path, const char* tau_path) {
  const int nibz = c->T.nibz, b = c->geo.b;
  auto K = [&](int ii, int j, int jj) { return kappa[(ii - 1) + (size_t)b * ((j - 1) + 3 * (jj - 1))]; };
  if (kappa_path) {
    File F;
    int r = open_out(F, kappa_path);
    if (r) return r;
    line(F, ListRecord().c("la, kxx,kyy,kzz, kxy,kxz,kyz, k_RTA").str());
    double tot_kap = 0;
    for (int j = 1; j <= 3; ++j)
      for (int jj = 1; jj <= 3; ++jj)
        for (int ii = 1; ii <= b; ++ii)
          if (j == jj) tot_kap = tot_kap + K(ii, j, jj) / 3;
    for (int ii = 1; ii <= b; ++ii) {  // format (i2,99(1x,g11.4))
      std::string s = edit_I(2, ii);
      const double v[6] = {K(ii, 1, 1), K(ii, 2, 2), K(ii, 3, 3), K(ii, 1, 2), K(ii, 1, 3), K(ii, 2, 3)};
      for (double x : v) s += " " + edit_G(11, 4, x);
      line(F, s);
    }
    line(F, ListRecord().c(" ").str());
    line(F, ListRecord().c("tot_kap=").r(tot_kap).str());
    line(F, ListRecord().c(" ").str());
    std::string s = "   ";  // format 78: 2(3x,2(3(1x,f9.3),2x)) over three items
    for (int j = 1; j <= 3; ++j) {
      double sum = 0;
      for (int ii = 1; ii <= b; ++ii) sum = sum + K(ii, j, j);
      s += " " + edit_F(9, 3, sum);
    }
    line(F, s);
  }
  File T;
  if (tau_path) {
    int r = open_out(T, tau_path);
    if (r) return r;
    line(T, ListRecord()
                .c("tempk,i,kibz(:,i),ii,omega,nb0,1/tauinv_N(i,ii),1/tauinv_U(i,ii),1/tauinv_tot(i,ii),"
                   "1/tauinv_eff(i,ii),veloc(:,ii,mapinv(i))")
                .str());
  }
  for (int i = 1; i <= nibz; ++i)
    for (int ii = 1; ii <= b; ++ii) {
      const size_t m = (size_t)(i - 1) + (size_t)nibz * (ii - 1);
      const size_t q = (size_t)(c->T.mapinv[i - 1] - 1) * b + (ii - 1);
      if (tU[m] == 0) tU[m] = 1.0e10;  // the reference replaces zero rates in place
      if (tN[m] == 0) tN[m] = 1.0e10;
      if (!tau_path) continue;
      std::string s;  // format (99(1x,g14.8))
      auto g = [&](double x) { s += " " + edit_G(14, 8, x); };
      auto gi = [&](long long v) { s += " " + edit_I(14, v); };
      g(tempk);
      gi(i);
      for (int x = 0; x < 3; ++x) g(c->T.kibz[(size_t)(i - 1) * 3 + x]);
      gi(ii);
      g(freq[q]);
      g(dist[q]);
      g(1 / tN[m]);
      g(1 / tU[m]);
      g(1 / tT[m]);
      g(teff[m]);
      for (int x = 0; x < 3; ++x) g(vel[q * 3 + x]);
      line(T, s);
    }
  return ALD_OK;
}

std::string join(const char* dir, const char* name) {
  std::string d = dir && *dir ? dir : ".";
  if (d.back() != '/') d += '/';
  return d + name;
}

}  // namespace

extern "C" {

int ald_format_value(const char* edit, double value, char* out, int cap) {
  if (!edit || !out || cap <= 0) return -1;
  std::string s;
  int w = 0, d = 0;
  const char k = edit[0];
  if (std::strcmp(edit, "*") == 0) {
    s = list_real(value);
  } else if (std::strcmp(edit, "*I") == 0) {
    s = list_int((long long)value);
  } else if ((k == 'I') && std::sscanf(edit + 1, "%d", &w) == 1 && w > 0) {
    s = edit_I(w, (long long)value);
  } else if ((k == 'F' || k == 'E' || k == 'G') && std::sscanf(edit + 1, "%d.%d", &w, &d) == 2 && w > 0 &&
             d >= 0 && (k == 'F' || d > 0)) {
    s = k == 'F' ? edit_F(w, d, value) : k == 'E' ? edit_E(w, d, value) : edit_G(w, d, value);
  } else {
    return -1;
  }
  if ((int)s.size() + 1 > cap) return -1;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return (int)s.size();
}

int ald_tau_eff(ald_ctx* c, double tempk, const double* F, int solution, double* tauinv_eff) {
  if (!c || !F || !tauinv_eff) return fail(ALD_ERR_ARG, "null argument");
  if (solution != 0 && solution != 1) return fail(ALD_ERR_ARG, "solution must be 0 (F_RTA) or 1 (CG)");
  ALD_CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  const int nibz = c->T.nibz, b = c->geo.b;
  std::vector<double> h((size_t)nibz * b * 3);
  if (solution == 0) {  // FFF(nibz,ndyn,3) column-major
    for (int i = 0; i < nibz; ++i)
      for (int l = 0; l < b; ++l)
        for (int x = 0; x < 3; ++x) h[((size_t)i * b + l) * 3 + x] = F[i + (size_t)nibz * (l + (size_t)b * x)];
  } else {
    std::memcpy(h.data(), F, h.size() * sizeof(double));
  }
  return tau_eff_dev(c, tempk, h, solution, tauinv_eff);
}

int ald_qandtau(ald_ctx* c, double tempk, const double* Q, const double* QN, const double* QU,
                const char* qvalue_path, double* tauinv_N, double* tauinv_U, double* tauinv_tot) {
  if (!c || !Q || !QN || !QU || !tauinv_N || !tauinv_U || !tauinv_tot) return fail(ALD_ERR_ARG, "null argument");
  ALD_CK(cudaSetDevice(c->device));
  std::vector<double> freq, dist, vel;
  int r = mode_tables(c, tempk, freq, dist, vel);
  if (r) return r;
  return qandtau(c, dist, Q, QN, QU, qvalue_path, tauinv_N, tauinv_U, tauinv_tot);
}

int ald_write_kappa(ald_ctx* c, double tempk, const double* kappa, double* tauinv_N, double* tauinv_U,
                    const double* tauinv_tot, const double* tauinv_eff, const char* kappa_path,
                    const char* tau_path) {
  if (!c || !kappa || !tauinv_N || !tauinv_U || !tauinv_tot || !tauinv_eff)
    return fail(ALD_ERR_ARG, "null argument");
  ALD_CK(cudaSetDevice(c->device));
  std::vector<double> freq, dist, vel;
  int r = mode_tables(c, tempk, freq, dist, vel);
  if (r) return r;
  return write_kappa(c, tempk, freq, dist, vel, kappa, tauinv_N, tauinv_U, tauinv_tot, tauinv_eff, kappa_path,
                     tau_path);
}

int ald_write_job1_files(ald_ctx* c, const char* dir, double tempk, const double* Q, const double* QN,
                         const double* QU, const double* kappa_rta_modes, const double* kappa_cg_modes,
                         const double* x) {
  if (!c || !Q || !QN || !QU || !kappa_rta_modes || !kappa_cg_modes || !x) return fail(ALD_ERR_ARG, "null argument");
  ALD_CK(cudaSetDevice(c->device));
  std::vector<double> freq, dist, vel;
  int r = mode_tables(c, tempk, freq, dist, vel);
  if (r) return r;
  const int nibz = c->T.nibz, b = c->geo.b;
  const size_t nm = (size_t)nibz * b;
  // F_RTA (calculate_RTA_distributionfunction) on the device from Q
  std::vector<double> hq(nm), hF(nm * 3);
  for (int i = 0; i < nibz; ++i)
    for (int l = 0; l < b; ++l) hq[(size_t)i * b + l] = Q[i + (size_t)nibz * l];
  {
    DevBuf<double> dq, dF;
    ALD_CKA(dq.alloc(nm));
    ALD_CKA(dF.alloc(nm * 3));
    ALD_CK(cudaMemcpyAsync(dq.p, hq.data(), nm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    KappaArgs k = kappa_args(c, tempk);
    ALD_CK(launch_rta_F(k, dq.p, dF.p, c->stream));
    ALD_CK(cudaMemcpyAsync(hF.data(), dF.p, nm * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ALD_CK(cudaStreamSynchronize(c->stream));
  }
  // mode_kappa clears the whole tauinv_eff array before each mode's sum
  // (sub.f90:1337), so after it only the last mode, (nibz, ndyn), keeps its sum
  std::vector<double> rta(nm), teff(nm, 0.0), tN(nm), tU(nm), tT(nm);
  r = tau_eff_dev(c, tempk, hF, 0, rta.data());
  if (r) return r;
  teff[nm - 1] = rta[nm - 1];
  const std::string fq = join(dir, "Qvalue.dat"), ftr = join(dir, "tau_RTA.dat"), fkr = join(dir, "kappa_RTA.dat"),
                    fte = join(dir, "tau_RTAandeff-cg.dat"), fkd = join(dir, "kappa_direct-cg.dat");
  r = qandtau(c, dist, Q, QN, QU, fq.c_str(), tN.data(), tU.data(), tT.data());
  if (r) return r;
  r = write_kappa(c, tempk, freq, dist, vel, kappa_rta_modes, tN.data(), tU.data(), tT.data(), teff.data(),
                  fkr.c_str(), ftr.c_str());
  if (r) return r;
  // mode_kappa_d adds its sums to the array mode_kappa left (no reset, sub.f90:1471)
  std::vector<double> cg(nm), hx(x, x + nm * 3);
  r = tau_eff_dev(c, tempk, hx, 1, cg.data());
  if (r) return r;
  for (size_t m = 0; m < nm; ++m) teff[m] = teff[m] + cg[m];
  return write_kappa(c, tempk, freq, dist, vel, kappa_cg_modes, tN.data(), tU.data(), tT.data(), teff.data(),
                     fkd.c_str(), fte.c_str());
}

}  // extern "C"
