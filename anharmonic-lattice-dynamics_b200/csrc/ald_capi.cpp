// C ABI of libald (include/ald.h): context lifecycle, the per-stage entry
// points that stand in for THERMACOND's job=1 subroutines, and the fused
// device pipeline.  All compute runs in CUDA kernels on the context's
// stream; host code only parses inputs, builds index tables and moves
// buffers across the boundary.
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ald_internal.h"

using namespace ald;

#include "ald_ctx.h"


namespace ald {

namespace {
// every freed block is kept, whatever its size: a fresh context's first
// pipeline call allocates its small workspaces (Q, the CG vectors, kappa
// partials) next to the large ones, and a driver allocation there lands
// between kernel launches
constexpr size_t kCacheMin = 1, kCacheMax = (size_t)32 << 30;
struct DevCache {
  std::mutex m;
  std::map<std::pair<int, size_t>, std::vector<void*>> blocks;  // (device, bytes) -> free blocks
  std::map<int, size_t> held;                                   // bytes held per device
};
DevCache& dev_cache() {
  static DevCache* c = new DevCache;  // never destroyed: no CUDA calls in static destructors
  return *c;
}
void release_device(DevCache& c, int dev) {  // caller holds c.m
  for (auto it = c.blocks.begin(); it != c.blocks.end();) {
    if (it->first.first == dev) {
      for (void* p : it->second) cudaFree(p);
      it = c.blocks.erase(it);
    } else {
      ++it;
    }
  }
  c.held[dev] = 0;
}
}  // namespace

std::mutex& capture_mutex() {
  static std::mutex* m = new std::mutex;
  return *m;
}

cudaError_t dev_alloc(void** p, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  DevCache& c = dev_cache();
  if (bytes >= kCacheMin) {
    std::lock_guard<std::mutex> g(c.m);
    auto it = c.blocks.find({dev, bytes});
    if (it != c.blocks.end() && !it->second.empty()) {
      *p = it->second.back();
      it->second.pop_back();
      c.held[dev] -= bytes;
      return cudaSuccess;
    }
  }
  e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    {
      std::lock_guard<std::mutex> g(c.m);
      release_device(c, dev);
    }
    e = cudaMalloc(p, bytes);
  }
  return e;
}

void dev_free(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> cap(capture_mutex());
  cudaPointerAttributes at;
  if (bytes >= kCacheMin && cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeDevice) {
    const int dev = at.device;
    int cur = 0;
    cudaGetDevice(&cur);
    DevCache& c = dev_cache();
    std::lock_guard<std::mutex> g(c.m);
    bool keep = c.held[dev] + bytes <= kCacheMax;
    if (keep) {  // no queued work of this device may still use the block
      if (dev != cur) cudaSetDevice(dev);
      keep = cudaDeviceSynchronize() == cudaSuccess;
      if (dev != cur) cudaSetDevice(cur);
    }
    if (keep) {
      c.blocks[{dev, bytes}].push_back(p);
      c.held[dev] += bytes;
      return;
    }
  }
  cudaFree(p);
}

void dev_trim() {
  std::lock_guard<std::mutex> cap(capture_mutex());
  DevCache& c = dev_cache();
  std::lock_guard<std::mutex> g(c.m);
  int cur = 0;
  cudaGetDevice(&cur);
  std::vector<int> devs;
  for (auto& kv : c.held) devs.push_back(kv.first);
  for (int d : devs) {
    cudaSetDevice(d);
    release_device(c, d);
  }
  cudaSetDevice(cur);
}

namespace capi {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)
#define CKA(call)                                                                       \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e == cudaErrorMemoryAllocation) return fail(ALD_ERR_NOMEM, "device allocation failed: " #call); \
    if (_e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)

double g_h2d = 0;  // bytes uploaded by the create call in progress

// The context's tables go to the device as one block: staged back to back
// (256-byte aligned) in one host buffer, copied with one H2D copy into one
// device allocation (a size the device-memory cache keeps, so a context of
// the same shape reuses it), each table's DevBuf a view into the block.  One
// allocation and one copy instead of one of each per table: about forty
// small cudaMalloc calls and pageable copies per context otherwise.
class TableStager {
 public:
  template <class T>
  void add(DevBuf<T>& d, const std::vector<T>& h) {
    const size_t n = std::max<size_t>(h.size(), 1);
    off_ = (off_ + 255) / 256 * 256;
    host_.resize(off_ + n * sizeof(T), 0);
    if (!h.empty()) std::memcpy(host_.data() + off_, h.data(), h.size() * sizeof(T));
    views_.push_back({&d, off_, n, [](void* dv, char* q, size_t cnt) {
                        static_cast<DevBuf<T>*>(dv)->view_of(reinterpret_cast<T*>(q), cnt);
                      }});
    off_ += n * sizeof(T);
    bytes_ += (double)h.size() * sizeof(T);
  }
  // the block (whole MiB, at least one), the copy, then the views
  cudaError_t commit(DevBuf<char>& block, cudaStream_t s) {
    const size_t mib = (size_t)1 << 20;
    const size_t total = std::max(mib, (off_ + mib - 1) / mib * mib);
    cudaError_t e = block.alloc(total);
    if (e != cudaSuccess) return e;
    if (off_) e = cudaMemcpyAsync(block.p, host_.data(), off_, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    for (auto& v : views_) v.bind(v.buf, block.p + v.off, v.n);
    g_h2d += bytes_;
    return cudaSuccess;
  }

 private:
  struct View {
    void* buf;
    size_t off, n;
    void (*bind)(void*, char*, size_t);
  };
  std::vector<char> host_;
  std::vector<View> views_;
  size_t off_ = 0;
  double bytes_ = 0;
};

double temp_cm(double tempk) {
  return tempk * PhysConst::k_b / (100 * PhysConst::h_plank * PhysConst::c_light);
}

int check_err_flags(ald_ctx* c) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h) {
    CK(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
    if (h & 16) return fail(ALD_ERR_CUDA, "V3: a tensor-core wait timed out (MMA completion not observed)");
    if (h & 32) return fail(ALD_ERR_CUDA, "eigensolver: the QL iteration did not converge in 60 sweeps");
    if (h & 2) return fail(ALD_ERR_DEN_ZERO, "MATRIX_ELT: den=0 (an eigenvalue is exactly zero)");
    if (h & 1) return fail(ALD_ERR_NBE, "ERROR in N_BE: w=<0 or t=<0");
  }
  return ALD_OK;
}

int ensure_phonons(ald_ctx* c) {
  if (c->have_phonons) return ALD_OK;
  const int b = c->geo.b, nkc = c->geo.nkc;
  if (b > kHeevMaxBands)
    return fail(ALD_ERR_UNSUPPORTED, "eigensolver: more than 256 bands is not supported by this build");
  CKA(c->w2_all.alloc((size_t)nkc * 7 * b));
  CKA(c->w2.alloc((size_t)nkc * b));
  CKA(c->evec.alloc((size_t)nkc * b * b * 2));
  CKA(c->vel.alloc((size_t)nkc * b * 3));
  PhononArgs a;
  a.geo = c->geo;
  a.kpc32 = c->kpc32.p;
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
  a.dq = (double)0.001f;  // finitedif_vel: dq=0.001 is a default-REAL literal
  a.w2_all = c->w2_all.p;
  a.w2 = c->w2.p;
  a.evec = c->evec.p;
  a.err = c->err.p;
  // the shared-memory Jacobi up to 64 bands, else Householder + QL on global
  // workspace; ALD_EIGENSOLVER=householder selects the latter at any size
  const char* es = getenv("ALD_EIGENSOLVER");
  if (b > 64 || (es && std::string(es) == "householder")) {
    a.ndisp = 7;
    a.he_slots = heev_slots(nkc * a.ndisp);
    CKA(c->w_heev.alloc(heev_work_doubles(b, a.he_slots)));
    a.he_work = c->w_heev.p;
    CK(launch_heev(a, c->stream));
  } else {
    CK(launch_phonons(a, c->stream));
  }
  CK(launch_phonon_post(c->geo, c->w2_all.p, a.dq, PhysConst::cnst(), c->vel.p, c->stream));
  CK(launch_subst_eivecs(c->geo, c->neg_src.p, c->neg_dst.p, (int)c->T.neg_src.size(), c->evec.p, c->stream));
  c->have_phonons = true;
  ++c->phonon_epoch;
  c->dist_tempk = -1;
  return ALD_OK;
}

int ensure_dist(ald_ctx* c, double tempk) {
  if (c->dist_tempk == tempk) return ALD_OK;
  const size_t n = (size_t)c->geo.nkc * c->geo.b;
  CKA(c->freq.alloc(n));
  CKA(c->dist.alloc(n));
  CK(launch_freq_dist(c->geo, c->w2.p, PhysConst::cnst(), temp_cm(tempk), c->S.classical, c->freq.p, c->dist.p,
                      c->err.p, c->stream));
  int r = check_err_flags(c);
  if (r) return r;
  c->dist_tempk = tempk;
  return ALD_OK;
}

bool ksub_ok(ald_ctx* c, const int* k) { return k && k[0] >= 1 && k[1] >= k[0] && k[1] <= c->T.nibz; }

V3Args v3_args(ald_ctx* c, int first, int nrows, double* out) {
  V3Args a;
  a.geo = c->geo;
  a.n1_first = first;
  a.nrows = nrows;
  a.mapinv = c->mapinv.p;
  a.evec = c->evec.p;
  a.w2 = c->w2.p;
  a.ntrip = c->F3.ntrip;
  a.natoms = c->S.natoms;
  a.blk_off = c->blk_off.p;
  a.trip_j = c->trip_j.p;
  a.trip_k = c->trip_k.p;
  a.fc3w = c->fc3w.p;
  a.phase_coef = c->phase_coef.p;
  a.roots = c->roots.p;
  a.const33 = PhysConst::const33();
  a.v3sq = out;
  a.v3_layout = 0;
  a.err = c->err.p;
  a.ncls = c->VC.ncls;
  a.cls_grp_off = c->cls_grp_off.p;
  a.cls_pc = c->cls_pc.p;
  a.cls_trip_off = c->cls_trip_off.p;
  a.cls_trip = c->cls_trip.p;
  a.cls_trip_i0 = c->cls_trip_i0.p;
  a.cls_trip_k = c->cls_trip_k.p;
  a.hbuf = nullptr;
  return a;
}

// The mixed path's |V3|^2 near zero frequencies.  Where a mode of q1, q2 or
// q3 has |lambda| below 1e-9 of the largest (the acoustic modes at Gamma),
// the matrix element before its 1/sqrt|lambda1 lambda2 lambda3| scaling is a
// cancellation (translational invariance of the FC3 terms).  Split-FP16
// products leave it at about 1e-7 of its terms instead of the 1e-16 of FP64,
// and the scaling then blows that residue up by up to 1/sqrt|lambda|: on
// meshes where the reference's Gamma test (loop indices nc/2 + 1,
// sub.f90:7351-7356) misses Gamma, or at q1 = Gamma, those entries reached
// kappa.  Such pairs are formed again in FP64 with the dense GEMMs of
// ald_v3_dense.cu, over the chunk's output in its layout: every pair whose
// q2 or q3 is such a point (unless the delta zeroes every soft band there:
// at most 3 of them, at the point of the Gamma test), and for a row whose q1
// is one, every pair with its soft bands l1 (the leading ones: bands are
// ordered by |lambda|).  The
// linewidths of those soft modes are that residue in FP64 too, and through
// the collision matrix they reach kappa: their row is formed with the
// kernel the FP64 path uses for the cell (the direct form up to 12 bands),
// so that both paths carry the same residue there.
static int v3_soft_fp64(ald_ctx* c, const V3Args& a, int* nl) {
  const int b = c->geo.b, nkc = c->T.nkc;
  std::vector<double> w2((size_t)nkc * b);
  CK(cudaMemcpyAsync(w2.data(), c->w2.p, w2.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double mx = 0;
  for (double v : w2) mx = std::max(mx, std::fabs(v));
  const double thr = 1e-9 * mx;
  std::vector<int> nsoft(nkc, 0), soft;
  for (int q = 0; q < nkc; ++q) {
    for (int l = 0; l < b; ++l)
      if (std::fabs(w2[(size_t)q * b + l]) < thr) nsoft[q] = l + 1;
    if (nsoft[q]) soft.push_back(q);
  }
  if (soft.empty()) return ALD_OK;
  const int* nc = c->geo.nc;
  auto dec = [&](int q, int* m) {
    m[0] = q / (nc[1] * nc[2]);
    m[1] = (q / nc[2]) % nc[1];
    m[2] = q % nc[2];
  };
  std::vector<long long> all, part;
  std::vector<int> soft_rows;  // rows of a soft q1 formed by the direct FP64 kernel
  int nk1 = 0;
  for (int r = 0; r < a.nrows; ++r) {
    const int q1 = c->T.mapinv[a.n1_first + r] - 1;
    int m1[3];
    dec(q1, m1);
    for (int sp : soft) {
      int ms[3], m2[3];
      dec(sp, ms);
      // the delta zeroes bands l < 3 at the point with indices nc/2 (the
      // reference's Gamma test): there nothing of a soft mode reaches the sums
      if (ms[0] == nc[0] / 2 && ms[1] == nc[1] / 2 && ms[2] == nc[2] / 2 && nsoft[sp] <= 3) continue;
      all.push_back((long long)r * nkc + sp);  // q2 at the point
      for (int x = 0; x < 3; ++x) {            // q3 = -q1 - q2 at the point
        int v = (-m1[x] - ms[x] + (c->geo.shifted ? nc[x] / 2 : 0)) % nc[x];
        m2[x] = v < 0 ? v + nc[x] : v;
      }
      all.push_back((long long)r * nkc + m2[2] + nc[2] * (m2[1] + nc[1] * m2[0]));
    }
    if (nsoft[q1]) {
      nk1 = std::max(nk1, nsoft[q1]);
      if (v3_dense_supported(b))
        for (int q2 = 0; q2 < nkc; ++q2) part.push_back((long long)r * nkc + q2);
      else
        soft_rows.push_back(r);
    }
  }
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  const size_t nall = all.size(), npart = part.size();
  all.insert(all.end(), part.begin(), part.end());
  if (all.empty() && soft_rows.empty()) return ALD_OK;
  if (!all.empty()) {
    if (c->w_pairs.n < all.size()) CKA(c->w_pairs.alloc(all.size()));
    // pageable source: the copy has left the vector when the call returns
    CK(cudaMemcpyAsync(c->w_pairs.p, all.data(), all.size() * sizeof(long long), cudaMemcpyHostToDevice,
                       c->stream));
  }
  cudaError_t e = cudaSuccess;
  if (nall || npart) {  // the dense FP64 GEMMs over the pair lists
    V3Args f = a;
    const size_t hneed = v3_hbuf_bytes(b, c->VC.ncls, a.nrows, ALD_FP64);
    if (c->w_h64.n < hneed) CKA(c->w_h64.alloc(hneed));
    f.hbuf = c->w_h64.p;
    const size_t wb = v3_dense_work_bytes(b, (long long)std::max(nall, npart), (size_t)256 << 20);
    if (c->w_v3fix.n < wb) CKA(c->w_v3fix.alloc(wb));
    e = launch_v3_rows_f64(f, c->stream);
    *nl += 1;
    const long long per = (long long)(c->w_v3fix.n / (2 * (size_t)b * b * b * 16));
    f.pair_list = c->w_pairs.p;
    f.npairs_list = (long long)nall;
    if (nall && e == cudaSuccess) e = launch_v3_dense(f, c->w_v3fix.p, c->w_v3fix.n, c->stream);
    *nl += 3 * (int)(((long long)nall + per - 1) / per);
    if (npart && e == cudaSuccess) {
      f.pair_list = c->w_pairs.p + nall;
      f.npairs_list = (long long)npart;
      e = launch_v3_dense(f, c->w_v3fix.p, c->w_v3fix.n, c->stream, nk1);
      *nl += 3 * (int)(((long long)npart + per - 1) / per);
    }
  }
  if (!soft_rows.empty() && e == cudaSuccess) {
    const size_t rn = (size_t)nkc * b * b * b;
    if (c->w_v3fix.n < rn * sizeof(double)) CKA(c->w_v3fix.alloc(rn * sizeof(double)));
    for (int r : soft_rows) {
      V3Args g = a;
      g.n1_first = a.n1_first + r;
      g.nrows = 1;
      g.v3_layout = 0;
      g.v3sq = reinterpret_cast<double*>(c->w_v3fix.p);
      g.v3sq_f32 = nullptr;
      g.pair_list = nullptr;
      e = launch_v3_fp64(g, c->stream);
      if (e == cudaSuccess) e = launch_v3_copy_row(a, r, g.v3sq, nk1, c->stream);
      *nl += 2;
      if (e != cudaSuccess) break;
    }
  }
  if (e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string("V3 near zero frequencies: ") + cudaGetErrorString(e));
  return ALD_OK;
}

int run_v3(ald_ctx* c, const V3Args& a0, int* nlaunch) {
  int nl = 0;
  if (c->S.include_fc[2] != 1) return fail(ALD_ERR_ARG, "fc3 terms are not included (include_fc(3) /= 1)");
  if (c->geo.b > kHeevMaxBands)
    return fail(ALD_ERR_UNSUPPORTED, "V3: more than 256 bands is not supported by this build");
  const int prec = c->opt.precision;
  V3Args a = a0;
  cudaError_t e;
  if (prec == ALD_MIXED && v3_dense_tc_supported(c->geo.b)) {
    // more than 12 bands, mixed: split-FP16 tensor-core GEMMs per pair
    const size_t need = v3_hbuf_bytes(c->geo.b, c->VC.ncls, a.nrows, ALD_MIXED);
    if (c->w_h.n < need) CKA(c->w_h.alloc(need));
    a.hbuf = c->w_h.p;
    const long long npairs = (long long)a.nrows * c->geo.nkc;
    const long long P = v3_dense_tc_pairs(c->geo.b, npairs, c->tune_gemm_bytes ? c->tune_gemm_bytes : (size_t)2 << 30);
    const size_t wb = v3_dense_tc_work_bytes(c->geo.b, c->geo.nkc, a.nrows, P);
    // GEMM 1 never writes the padding of the T2 operand: it is zeroed when the
    // workspace is new or was last laid out for another (bands, pairs)
    bool zeroed = c->w_v3work.n >= wb && c->v3work_tc_b == c->geo.b && c->v3work_tc_p == P;
    if (c->w_v3work.n < wb) {
      CKA(c->w_v3work.alloc(wb));
      zeroed = false;
    }
    e = launch_v3_rows_f32(a, c->stream);
    if (e == cudaSuccess) e = launch_v3_dense_tc(a, c->w_v3work.p, P, zeroed, c->stream);
    c->v3work_tc_b = e == cudaSuccess ? c->geo.b : 0;
    c->v3work_tc_p = P;
    nl += 1 + v3_dense_tc_launches(npairs, P);
    if (e == cudaSuccess) {
      const int r = v3_soft_fp64(c, a, &nl);
      if (r) return r;
    }
  } else if (v3_dense_supported(c->geo.b)) {
    // more than 12 bands: batched GEMMs per pair (FP64)
    const size_t need = v3_hbuf_bytes(c->geo.b, c->VC.ncls, a.nrows, ALD_FP64);
    if (c->w_h.n < need) CKA(c->w_h.alloc(need));
    a.hbuf = c->w_h.p;
    const size_t wb = v3_dense_work_bytes(c->geo.b, (long long)a.nrows * c->geo.nkc, (size_t)2 << 30);
    if (c->w_v3work.n < wb) CKA(c->w_v3work.alloc(wb));
    c->v3work_tc_b = 0;  // the FP64 GEMMs overwrite the workspace
    e = launch_v3_rows_f64(a, c->stream);
    if (e == cudaSuccess) e = launch_v3_dense(a, c->w_v3work.p, c->w_v3work.n, c->stream);
    const long long per = (long long)(c->w_v3work.n / (2 * (size_t)c->geo.b * c->geo.b * c->geo.b * 16));
    nl += 1 + 3 * (int)(((long long)a.nrows * c->geo.nkc + per - 1) / per);
  } else if (prec == ALD_MIXED && v3_tc_supported(c->geo.b, c->VC.ncls)) {
    const size_t need = v3_hbuf_bytes(c->geo.b, c->VC.ncls, a.nrows, prec);
    if (c->w_h.n < need) CKA(c->w_h.alloc(need));
    a.hbuf = c->w_h.p;
    if (!c->ptiles_ok) {
      CKA(c->w_ptiles.alloc(v3_tc_ptile_bytes(c->geo.nkc, c->VC.ncls)));
      e = launch_v3_tc_ptiles(a, c->w_ptiles.p, c->stream);
      if (e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string("V3 phase tiles: ") + cudaGetErrorString(e));
      c->ptiles_ok = true;
      nl += 1;
    }
    const size_t bneed = v3_tc_btile_bytes(a.nrows, c->VC.ncls, c->geo.nkc);
    if (c->w_btiles.n < bneed) CKA(c->w_btiles.alloc(bneed));
    e = launch_v3_rows_f32(a, c->stream);
    if (e == cudaSuccess) e = launch_v3_tc(a, c->w_ptiles.p, c->w_btiles.p, c->stream, c->tune_v3_rpc, c->tune_v3_wg);
    nl += 4;  // class sums H, mode factors, B tiles, the MMA kernel
  } else if (v3_pair_supported(c->geo.b, prec)) {
    const size_t need = v3_hbuf_bytes(c->geo.b, c->VC.ncls, a.nrows, prec);
    if (c->w_h.n < need) CKA(c->w_h.alloc(need));
    a.hbuf = c->w_h.p;
    e = launch_v3_pair(a, prec, c->stream);
    nl += 2;
  } else if (prec == ALD_FP64 && a.v3_layout == 0) {
    e = launch_v3_fp64(a, c->stream);
    nl += 1;
  } else {
    return fail(ALD_ERR_UNSUPPORTED, "V3: the mixed-precision path and the slice-major layout support 3 or 6 bands");
  }
  if (e != cudaSuccess) return fail(ALD_ERR_CUDA, std::string("V3 launch: ") + cudaGetErrorString(e));
  if (nlaunch) *nlaunch += nl;
  return ALD_OK;
}

int ensure_giso(ald_ctx* c) {
  if (!c->giso_ok) {
    std::string e = isotope_g_atoms(c->S, c->giso);
    if (!e.empty()) return fail(ALD_ERR_UNSUPPORTED, e);
    c->giso_ok = true;
  }
  CKA(c->giso_d.alloc(c->giso.size()));
  CK(cudaMemcpyAsync(c->giso_d.p, c->giso.data(), c->giso.size() * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  return ALD_OK;
}

KappaArgs kappa_args(ald_ctx* c, double tempk) {
  KappaArgs k;
  k.geo = c->geo;
  k.nibz = c->T.nibz;
  k.mapinv = c->mapinv.p;
  k.freq = c->freq.p;
  k.dist = c->dist.p;
  k.vel = c->vel.p;
  k.w2 = c->w2.p;
  k.arm_off = c->arm_off.p;
  k.arm_q = c->arm_q.p;
  k.arm_op = c->arm_op.p;
  k.star_off = c->star_off.p;
  k.star_q = c->star_q.p;
  k.star_op = c->star_op.p;
  k.opk = c->opk.p;
  k.opk_inv = c->opk_inv.p;
  k.tempk = tempk;
  k.temp = temp_cm(tempk);
  k.const1 = PhysConst::h_plank * PhysConst::c_light * 100 * PhysConst::c_light /
             (c->T.nkc * c->S.volume_r / 1e30);
  k.const2 = PhysConst::k_b * (tempk * tempk) / (PhysConst::h_plank * PhysConst::c_light * 100) / PhysConst::c_light;
  k.classical = c->S.classical;
  k.arm_owner = c->arm_owner.p;
  k.narm = (int)c->T.arm_q.size();
  k.part = c->w_kpart.alloc(kappa_partial_doubles(c->geo.b, k.narm)) == cudaSuccess ? c->w_kpart.p : nullptr;
  k.zero_q_f = c->opt.precision != ALD_FP64;
  return k;
}

int delta_mode(ald_ctx* c) { return c->opt.delta; }
double gauss_width(ald_ctx* c) { return c->opt.width_cm > 0 ? c->opt.width_cm : c->S.width; }

// |V3|^2 rows per chunk within the byte budget
int rows_per_chunk(ald_ctx* c) {
  size_t per_row = (size_t)c->T.nkc * c->geo.b * c->geo.b * c->geo.b * sizeof(double);
  size_t budget = c->opt.chunk_bytes ? c->opt.chunk_bytes : (size_t)512 << 20;
  return (int)std::max<size_t>(1, std::min<size_t>(budget / per_row, (size_t)c->T.nibz));
}

}  // namespace capi
}  // namespace ald

using namespace ald::capi;

// =====================================================================
extern "C" {

void ald_default_options(ald_options* o) {
  std::memset(o, 0, sizeof *o);
  o->delta = ALD_DELTA_TETRA;
  o->precision = ALD_FP64;
  o->cg_stop = ALD_CG_REFERENCE;
  o->cg_max_iter = 100;
  o->cg_ndig = 2;
  o->cg_tol = 1e-8;
  o->width_cm = -1;
  o->device = 0;
  o->chunk_bytes = 0;
  o->deterministic = ALD_DET_AUTO;
}

const char* ald_last_error(void) { return g_err.c_str(); }

int ald_create_from_dir(const char* dir, const ald_options* opt, ald_ctx** out) {
  if (!dir || !out) return fail(ALD_ERR_ARG, "null argument");
  *out = nullptr;
  std::unique_ptr<ald_ctx> c(new ald_ctx());
  if (opt) c->opt = *opt;
  else ald_default_options(&c->opt);
  std::string e = read_system(dir, c->S);
  if (!e.empty()) return fail(ALD_ERR_IO, e);
  // b200.params knobs apply when the caller passes no options
  if (!opt) {
    if (c->S.delta >= 0) c->opt.delta = c->S.delta;
    if (c->S.precision >= 0) c->opt.precision = c->S.precision;
    if (c->S.cg_stop >= 0) c->opt.cg_stop = c->S.cg_stop;
    if (c->S.cg_tol > 0) c->opt.cg_tol = c->S.cg_tol;
    if (c->S.width_cm > 0) c->opt.width_cm = c->S.width_cm;
  }
  e = build_tables(c->S, c->T);
  if (!e.empty()) return fail(e.find("not a kpoint") != std::string::npos ? ALD_ERR_NOT_KPOINT : ALD_ERR_IO, e);
  if (c->S.include_fc[2] == 1) {
    e = build_fc3(c->S, c->F3);
    if (!e.empty()) return fail(ALD_ERR_IO, e);
    e = build_v3_classes(c->S, c->T, c->F3, c->VC);
    if (!e.empty()) return fail(ALD_ERR_IO, e);
  }
  e = build_fc2(c->S, c->F2);
  if (!e.empty()) return fail(ALD_ERR_IO, e);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ALD_ERR_CUDA, "no CUDA device");
  c->device = c->opt.device;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
  c->stream = c->own_stream;
  Geometry& g = c->geo;
  for (int a = 0; a < 3; ++a) g.nc[a] = c->S.nc[a];
  g.nkc = c->T.nkc;
  g.b = c->T.b;
  g.nat0 = c->S.nat0;
  g.shifted = c->T.shifted ? 1 : 0;
  g.L = c->T.L;
  {
    long long mx = (long long)c->T.L - 1;  // the largest phase sum of a mesh point
    for (int a = 0; a < 3; ++a) mx += (long long)(g.nc[a] - 1) * (c->T.L - 1);
    g.L32 = mx < (1LL << 31) ? 1 : 0;
  }
  cudaStream_t s = c->stream;
  g_h2d = 0;
  // tables
  TableStager st;
  st.add(c->kpc32, c->T.kpc32);
  std::vector<double> rr(3 * (size_t)c->S.natoms);
  for (int j = 0; j < c->S.natoms; ++j) {
    int j0 = c->S.cell0[j] - 1;
    for (int x = 0; x < 3; ++x) rr[3 * j + x] = c->S.atompos[3 * j + x] - c->S.atompos[3 * j0 + x];
  }
  st.add(c->rr, rr);
  st.add(c->fc2_off, c->F2.off);
  st.add(c->fc2_atom, c->F2.atom);
  st.add(c->fc2_val, c->F2.val);
  st.add(c->fc2_sqm, c->F2.sqm);
  st.add(c->fc2_uatom, c->F2.uatom);
  st.add(c->fc2_uidx, c->F2.uidx);
  {
    // epsil(9), charge(9*nat0), masses(nat0), eps_scale, rho2, om0
    std::vector<double> bo(9 + 10 * c->S.nat0 + 4, 0.0);
    std::memcpy(bo.data(), c->S.epsil, 9 * sizeof(double));
    std::copy(c->S.charge.begin(), c->S.charge.end(), bo.begin() + 9);
    std::copy(c->S.mass0.begin(), c->S.mass0.end(), bo.begin() + 9 + 9 * c->S.nat0);
    auto len = [](const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
    double gg = std::pow(len(c->S.g[0]) * len(c->S.g[1]) * len(c->S.g[2]), (double)0.33f);
    double rho = gg / 4.0;
    double* sc = bo.data() + 9 + 10 * c->S.nat0;
    sc[0] = 8.8541878176e-12 / 1e10 / PhysConst::ee;
    sc[1] = rho * rho;
    sc[2] = c->S.volume_r;
    st.add(c->born, bo);
  }
  if (c->S.include_fc[2] == 1) {
    st.add(c->blk_off, c->F3.blk_off);
    st.add(c->trip_j, c->F3.trip_j);
    st.add(c->trip_k, c->F3.trip_k);
    st.add(c->fc3w, c->F3.w);
    st.add(c->cls_grp_off, c->VC.grp_off);
    st.add(c->cls_pc, c->VC.pc);
    st.add(c->cls_trip_off, c->VC.trip_off);
    st.add(c->cls_trip, c->VC.trip);
    st.add(c->cls_trip_i0, c->VC.trip_i0);
    st.add(c->cls_trip_k, c->VC.trip_k);
  }
  {
    std::vector<double> rt(2 * (size_t)c->T.L);
    for (int t = 0; t < c->T.L; ++t) {
      double ang = 2.0 * PhysConst::pi * (double)t / (double)c->T.L;
      rt[2 * t] = std::cos(ang);
      rt[2 * t + 1] = std::sin(ang);
    }
    // exact values on the axes
    for (int t = 0; t < c->T.L; ++t) {
      if ((4L * t) % c->T.L == 0) {
        long k = (4L * t) / c->T.L;
        rt[2 * t] = k == 0 ? 1.0 : (k == 2 ? -1.0 : 0.0);
        rt[2 * t + 1] = k == 1 ? 1.0 : (k == 3 ? -1.0 : 0.0);
      }
    }
    st.add(c->roots, rt);
  }
  st.add(c->phase_coef, c->T.phase_coef);
  std::vector<int> mi(c->T.nibz);
  for (int i = 0; i < c->T.nibz; ++i) mi[i] = c->T.mapinv[i] - 1;
  st.add(c->mapinv, mi);
  st.add(c->neg_src, c->T.neg_src);
  st.add(c->neg_dst, c->T.neg_dst);
  st.add(c->arm_off, c->T.arm_off);
  st.add(c->arm_q, c->T.arm_q);
  st.add(c->arm_op, c->T.arm_op);
  st.add(c->star_off, c->T.star_off);
  st.add(c->star_q, c->T.star_q);
  st.add(c->star_op, c->T.star_op);
  st.add(c->tet_corner, c->T.tet_corner);
  st.add(c->tet_inc, c->T.tet_inc);
  {
    // update_mpi's rotation of F to every mesh point: the op of the point's
    // arm in kstarsinfbz1 of its IBZ point (every mesh point is such an arm
    // exactly once on the meshes the reference accepts)
    std::vector<int> m0(c->T.nkc), fop(c->T.nkc, -1);
    for (int q = 0; q < c->T.nkc; ++q) m0[q] = c->T.mapibz[q] - 1;
    for (int i = 0; i < c->T.nibz; ++i)
      for (int a = c->T.arm_off[i]; a < c->T.arm_off[i + 1]; ++a)
        if (fop[c->T.arm_q[a]] < 0 && m0[c->T.arm_q[a]] == i) fop[c->T.arm_q[a]] = c->T.arm_op[a];
    c->full_op_ok = std::all_of(fop.begin(), fop.end(), [](int v) { return v >= 0; });
    for (int& v : fop) v = std::max(v, 0);
    st.add(c->mapibz0, m0);
    st.add(c->full_op, fop);
    // mesh integers of every point, 4 ints each (the collision kernel's arm lookups)
    std::vector<int> mm(4 * (size_t)c->T.nkc, 0);
    const int N1 = c->S.nc[1], N2 = c->S.nc[2];
    for (int q = 0; q < c->T.nkc; ++q) {
      mm[4 * (size_t)q] = q / (N1 * N2);
      mm[4 * (size_t)q + 1] = (q / N2) % N1;
      mm[4 * (size_t)q + 2] = q % N2;
    }
    st.add(c->mesh_m, mm);
    std::vector<int> own(c->T.arm_q.size());
    for (int i = 0; i < c->T.nibz; ++i)
      for (int a = c->T.arm_off[i]; a < c->T.arm_off[i + 1]; ++a) own[a] = i;
    st.add(c->arm_owner, own);
  }
  {
    std::vector<double> op(48 * 9, 0.0), opi(48 * 9, 0.0);
    for (int o = 0; o < c->T.npg; ++o) {
      const double* m = c->T.opk[o];
      std::memcpy(&op[9 * o], m, 9 * sizeof(double));
      // exact inverse of an integer matrix with |det| = 1
      auto M = [&](int i, int j) { return m[i + 3 * j]; };
      double det = M(0, 0) * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) - M(0, 1) * (M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0)) +
                   M(0, 2) * (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0));
      double* r = &opi[9 * o];
      r[0 + 3 * 0] = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) / det;
      r[0 + 3 * 1] = (M(0, 2) * M(2, 1) - M(0, 1) * M(2, 2)) / det;
      r[0 + 3 * 2] = (M(0, 1) * M(1, 2) - M(0, 2) * M(1, 1)) / det;
      r[1 + 3 * 0] = (M(1, 2) * M(2, 0) - M(1, 0) * M(2, 2)) / det;
      r[1 + 3 * 1] = (M(0, 0) * M(2, 2) - M(0, 2) * M(2, 0)) / det;
      r[1 + 3 * 2] = (M(0, 2) * M(1, 0) - M(0, 0) * M(1, 2)) / det;
      r[2 + 3 * 0] = (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0)) / det;
      r[2 + 3 * 1] = (M(0, 1) * M(2, 0) - M(0, 0) * M(2, 1)) / det;
      r[2 + 3 * 2] = (M(0, 0) * M(1, 1) - M(0, 1) * M(1, 0)) / det;
    }
    st.add(c->opk, op);
    st.add(c->opk_inv, opi);
  }
  st.add(c->err, std::vector<int>(4, 0));  // the kernels' error flags, cleared
  CKA(st.commit(c->tables, s));
  CK(cudaStreamSynchronize(s));
  c->h2d_bytes = g_h2d;
  *out = c.release();
  return ALD_OK;
}

void ald_destroy(ald_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

int ald_set_stream(ald_ctx* c, void* stream) {
  if (!c) return fail(ALD_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return ALD_OK;
}

double ald_h2d_bytes(ald_ctx* c) { return c ? c->h2d_bytes : 0.0; }

void ald_release_cached_memory(void) { ald::dev_trim(); }

int ald_get_info(ald_ctx* c, ald_info* info) {
  if (!c || !info) return fail(ALD_ERR_ARG, "null argument");
  info->ndyn = c->geo.b;
  info->natoms0 = c->S.nat0;
  for (int a = 0; a < 3; ++a) info->nc[a] = c->S.nc[a];
  info->nkc = c->T.nkc;
  info->nibz = c->T.nibz;
  info->nterms2 = c->S.nterms[1];
  info->nterms3 = c->S.nterms[2];
  info->natoms = c->S.natoms;
  info->lattpgcount = c->T.npg;
  info->born_flag = c->S.born_flag;
  info->tempk = c->S.tmin;
  info->width_cm = c->S.width;
  info->volume_r = c->S.volume_r;
  return ALD_OK;
}

int ald_read_mesh(const char* dir, ald_info* info, double* kpc, int* mapibz, int* mapinv, double* kibz,
                  double* wibz) {
  if (!dir || !info) return fail(ALD_ERR_ARG, "null argument");
  System S;
  Tables T;
  std::string e = read_system(dir, S);
  if (!e.empty()) return fail(ALD_ERR_IO, e);
  e = build_tables(S, T);
  if (!e.empty()) return fail(e.find("not a kpoint") != std::string::npos ? ALD_ERR_NOT_KPOINT : ALD_ERR_IO, e);
  info->ndyn = T.b;
  info->natoms0 = S.nat0;
  for (int a = 0; a < 3; ++a) info->nc[a] = S.nc[a];
  info->nkc = T.nkc;
  info->nibz = T.nibz;
  info->nterms2 = S.nterms[1];
  info->nterms3 = S.nterms[2];
  info->natoms = S.natoms;
  info->lattpgcount = T.npg;
  info->born_flag = S.born_flag;
  info->tempk = S.tmin;
  info->width_cm = S.width;
  info->volume_r = S.volume_r;
  if (kpc) std::memcpy(kpc, T.kpc32.data(), T.kpc32.size() * sizeof(double));
  if (mapibz) std::memcpy(mapibz, T.mapibz.data(), T.mapibz.size() * sizeof(int));
  if (mapinv) std::memcpy(mapinv, T.mapinv.data(), T.mapinv.size() * sizeof(int));
  if (kibz) std::memcpy(kibz, T.kibz.data(), T.kibz.size() * sizeof(double));
  if (wibz) std::memcpy(wibz, T.wibz.data(), T.wibz.size() * sizeof(double));
  return ALD_OK;
}

int ald_get_mesh(ald_ctx* c, double* kpc, int* mapibz, int* mapinv, double* kibz, double* wibz) {
  if (!c) return fail(ALD_ERR_ARG, "null context");
  if (kpc) std::memcpy(kpc, c->T.kpc32.data(), c->T.kpc32.size() * sizeof(double));
  if (mapibz) std::memcpy(mapibz, c->T.mapibz.data(), c->T.mapibz.size() * sizeof(int));
  if (mapinv) std::memcpy(mapinv, c->T.mapinv.data(), c->T.mapinv.size() * sizeof(int));
  if (kibz) std::memcpy(kibz, c->T.kibz.data(), c->T.kibz.size() * sizeof(double));
  if (wibz) std::memcpy(wibz, c->T.wibz.data(), c->T.wibz.size() * sizeof(double));
  return ALD_OK;
}

int ald_get_frequencies(ald_ctx* c, double* eigenval, double* eigenvec, double* veloc) {
  if (!c) return fail(ALD_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  c->have_phonons = false;
  int r = ensure_phonons(c);
  if (r) return r;
  const size_t nkc = c->T.nkc, b = c->geo.b;
  if (eigenval) CK(cudaMemcpyAsync(eigenval, c->w2.p, nkc * b * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (eigenvec)
    CK(cudaMemcpyAsync(eigenvec, c->evec.p, nkc * b * b * 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (veloc) CK(cudaMemcpyAsync(veloc, c->vel.p, nkc * b * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_err_flags(c);
}

int ald_set_phonons(ald_ctx* c, const double* eigenval, const double* eigenvec, const double* veloc) {
  if (!c || !eigenval || !eigenvec || !veloc) return fail(ALD_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const size_t nkc = c->T.nkc, b = c->geo.b;
  CKA(c->w2.alloc(nkc * b));
  CKA(c->evec.alloc(nkc * b * b * 2));
  CKA(c->vel.alloc(nkc * b * 3));
  CK(cudaMemcpyAsync(c->w2.p, eigenval, nkc * b * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->evec.p, eigenvec, nkc * b * b * 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->vel.p, veloc, nkc * b * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_phonons = true;
  ++c->phonon_epoch;
  c->dist_tempk = -1;
  return ALD_OK;
}

int ald_calculate_w3_ibz_split_sq(ald_ctx* c, const int ksubset[2], double* v33s8) {
  if (!c || !v33s8) return fail(ALD_ERR_ARG, "null argument");
  if (!ksub_ok(c, ksubset)) return fail(ALD_ERR_ARG, "ksubset out of range");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  const int nr = ksubset[1] - ksubset[0] + 1;
  const size_t n = (size_t)nr * c->T.nkc * c->geo.b * c->geo.b * c->geo.b;
  DevBuf<double> v, f;
  CKA(v.alloc(n));
  CKA(f.alloc(n));
  r = run_v3(c, v3_args(c, ksubset[0] - 1, nr, v.p), nullptr);
  if (r) return r;
  CK(launch_to_fortran5(v.p, f.p, nr, c->T.nkc, c->geo.b, c->stream));
  CK(cudaMemcpyAsync(v33s8, f.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_err_flags(c);
}

int ald_calculate_fgr(ald_ctx* c, const int ksubset[2], const double* v33s8, double* P1smpi, double* P2smpi) {
  if (!c || !v33s8 || !P1smpi || !P2smpi) return fail(ALD_ERR_ARG, "null argument");
  if (!ksub_ok(c, ksubset)) return fail(ALD_ERR_ARG, "ksubset out of range");
  if (c->geo.b > kHeevMaxBands)
    return fail(ALD_ERR_UNSUPPORTED, "delta stage: more than 256 bands is not supported by this build");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, c->S.tmin);
  if (r) return r;
  const int nr = ksubset[1] - ksubset[0] + 1, b = c->geo.b, nkc = c->T.nkc;
  const size_t n = (size_t)nr * nkc * b * b * b;
  DevBuf<double> vf, v, p1, p2, R1, R2;
  DevBuf<char> scratch;
  CKA(vf.alloc(n));
  CKA(v.alloc(n));
  CKA(p1.alloc(n));
  CKA(p2.alloc(n));
  CKA(R1.alloc((size_t)nr * nkc * b * b));
  CKA(R2.alloc((size_t)nr * nkc * b * b));
  if (b <= kDeltaSmallBands) CKA(scratch.alloc(std::max<size_t>(256, combine_scratch_bytes(c->geo, nr, 0))));
  CK(cudaMemcpyAsync(vf.p, v33s8, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(vf.p, v.p, nr, nkc, b, c->stream));
  CombineArgs a;
  a.geo = c->geo;
  a.n1_first = ksubset[0] - 1;
  a.nrows = nr;
  a.mapinv = c->mapinv.p;
  a.v3sq = v.p;
  a.freq = c->freq.p;
  a.dist = c->dist.p;
  a.tet_corner = c->tet_corner.p;
  a.tet_inc = c->tet_inc.p;
  a.gauss = delta_mode(c) == ALD_DELTA_GAUSS;
  a.sigma = gauss_width(c);
  a.f32w = 0;  // the per-stage entry point keeps the reference's FP64 weights
  a.brange = nullptr;
  a.R1 = R1.p;
  a.R2 = R2.p;
  a.P1s = p1.p;
  a.P2s = p2.p;
  a.P1 = nullptr;
  a.P2 = nullptr;
  a.R1p = a.R2p = nullptr;
  a.v3_layout = 0;
  if (b > kDeltaSmallBands) {  // band-generic kernels: P1smpi/P2smpi only
    CK(cudaMemsetAsync(p1.p, 0, n * sizeof(double), c->stream));
    CK(cudaMemsetAsync(p2.p, 0, n * sizeof(double), c->stream));
    a.R1 = a.R2 = nullptr;
    CK(launch_delta_any(a, c->stream));
  } else {
    CK(launch_combine(a, scratch.p, c->stream));
  }
  CK(launch_to_fortran5(p1.p, vf.p, nr, nkc, b, c->stream));
  CK(cudaMemcpyAsync(P1smpi, vf.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(launch_to_fortran5(p2.p, vf.p, nr, nkc, b, c->stream));
  CK(cudaMemcpyAsync(P2smpi, vf.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_err_flags(c);
}

int ald_distribution(ald_ctx* c, double tempk, double* frequency, double* dist) {
  if (!c) return fail(ALD_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  const int nkc = c->T.nkc, b = c->geo.b;
  std::vector<double> f((size_t)nkc * b), d((size_t)nkc * b);
  CK(cudaMemcpyAsync(f.data(), c->freq.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(d.data(), c->dist.p, d.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < nkc; ++q)  // (nkc, ndyn) Fortran layout
    for (int l = 0; l < b; ++l) {
      if (frequency) frequency[q + (size_t)nkc * l] = f[(size_t)q * b + l];
      if (dist) dist[q + (size_t)nkc * l] = d[(size_t)q * b + l];
    }
  return ALD_OK;
}

int ald_calculate_tau_rta(ald_ctx* c, const int ksubset[2], double tempk, const double* P1smpi,
                          const double* P2smpi, double* Q, double* QN, double* QU, double* P1, double* P2) {
  if (!c || !P1smpi || !P2smpi || !Q || !QN || !QU) return fail(ALD_ERR_ARG, "null argument");
  if (!ksub_ok(c, ksubset)) return fail(ALD_ERR_ARG, "ksubset out of range");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  const int nr = ksubset[1] - ksubset[0] + 1, b = c->geo.b, nkc = c->T.nkc;
  const size_t n = (size_t)nr * nkc * b * b * b;
  DevBuf<double> tmp, s1, s2, o1, o2, q;
  CKA(tmp.alloc(n));
  CKA(s1.alloc(n));
  CKA(s2.alloc(n));
  if (P1) CKA(o1.alloc(n));
  if (P2) CKA(o2.alloc(n));
  CKA(q.alloc((size_t)3 * nr * b));
  CK(cudaMemcpyAsync(tmp.p, P1smpi, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(tmp.p, s1.p, nr, nkc, b, c->stream));
  CK(cudaMemcpyAsync(tmp.p, P2smpi, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(tmp.p, s2.p, nr, nkc, b, c->stream));
  CK(launch_tau(c->geo, ksubset[0] - 1, nr, c->mapinv.p, s1.p, s2.p, c->dist.p, q.p, q.p + nr * b,
                q.p + 2 * nr * b, o1.p, o2.p, c->stream));
  std::vector<double> hq((size_t)3 * nr * b);
  CK(cudaMemcpyAsync(hq.data(), q.p, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (P1) {
    CK(launch_to_fortran5(o1.p, tmp.p, nr, nkc, b, c->stream));
    CK(cudaMemcpyAsync(P1, tmp.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (P2) {
    CK(launch_to_fortran5(o2.p, tmp.p, nr, nkc, b, c->stream));
    CK(cudaMemcpyAsync(P2, tmp.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < nr; ++i)  // Q(nk1, ndyn)
    for (int l = 0; l < b; ++l) {
      Q[i + (size_t)nr * l] = hq[(size_t)i * b + l];
      QN[i + (size_t)nr * l] = hq[(size_t)nr * b + (size_t)i * b + l];
      QU[i + (size_t)nr * l] = hq[(size_t)2 * nr * b + (size_t)i * b + l];
    }
  return ALD_OK;
}

int ald_rta_kappa(ald_ctx* c, double tempk, const double* Q, double* FFF, double* kappa) {
  if (!c || !Q) return fail(ALD_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  const int nibz = c->T.nibz, b = c->geo.b;
  std::vector<double> hq((size_t)nibz * b);
  for (int i = 0; i < nibz; ++i)
    for (int l = 0; l < b; ++l) hq[(size_t)i * b + l] = Q[i + (size_t)nibz * l];
  DevBuf<double> dq, dF, dk;
  CKA(dq.alloc(hq.size()));
  CKA(dF.alloc(hq.size() * 3));
  CKA(dk.alloc((size_t)b * 9));
  CK(cudaMemcpyAsync(dq.p, hq.data(), hq.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  KappaArgs k = kappa_args(c, tempk);
  CK(launch_rta_F(k, dq.p, dF.p, c->stream));
  CK(launch_kappa(k, dF.p, 0, dk.p, c->err.p, c->stream));
  std::vector<double> hF(hq.size() * 3);
  CK(cudaMemcpyAsync(hF.data(), dF.p, hF.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (kappa) CK(cudaMemcpyAsync(kappa, dk.p, (size_t)b * 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (FFF)
    for (int i = 0; i < nibz; ++i)
      for (int l = 0; l < b; ++l)
        for (int x = 0; x < 3; ++x) FFF[i + (size_t)nibz * (l + (size_t)b * x)] = hF[((size_t)i * b + l) * 3 + x];
  return check_err_flags(c);
}

int ald_collision_matrix(ald_ctx* c, const int ksubset[2], const double* P1, const double* P2, double* CM) {
  if (!c || !P1 || !P2 || !CM) return fail(ALD_ERR_ARG, "null argument");
  if (!ksub_ok(c, ksubset)) return fail(ALD_ERR_ARG, "ksubset out of range");
  CK(cudaSetDevice(c->device));
  const int nr = ksubset[1] - ksubset[0] + 1, b = c->geo.b, nkc = c->T.nkc, nibz = c->T.nibz;
  const size_t n = (size_t)nr * nkc * b * b * b;
  DevBuf<double> tmp, p1, p2, R1, R2, Qd, cm, cmt;
  CKA(tmp.alloc(n));
  CKA(p1.alloc(n));
  CKA(p2.alloc(n));
  CKA(R1.alloc((size_t)nr * nkc * b * b));
  CKA(R2.alloc((size_t)nr * nkc * b * b));
  CKA(Qd.alloc((size_t)nr * b));
  const int rows = 3 * b * nr, cols = 3 * b * nibz;
  CKA(cm.alloc((size_t)rows * cols));
  CKA(cmt.alloc((size_t)rows * cols));
  CK(cudaMemcpyAsync(tmp.p, P1, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(tmp.p, p1.p, nr, nkc, b, c->stream));
  CK(cudaMemcpyAsync(tmp.p, P2, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(tmp.p, p2.p, nr, nkc, b, c->stream));
  CK(launch_collapse(c->geo, nr, p1.p, p2.p, R1.p, R2.p, Qd.p, c->stream));
  CK(launch_collision(c->geo, nibz, ksubset[0] - 1, nr, c->mapinv.p, c->arm_off.p, c->arm_q.p, c->arm_op.p,
                      c->opk.p, Qd.p, R1.p, R2.p, cm.p, (size_t)cols, 0, nullptr, c->mesh_m.p, c->stream));
  CK(launch_transpose(cm.p, cmt.p, rows, cols, c->stream));  // row-major -> Fortran column-major
  CK(cudaMemcpyAsync(CM, cmt.p, (size_t)rows * cols * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ALD_OK;
}

int ald_rhs(ald_ctx* c, double tempk, double* RHS) {
  if (!c || !RHS) return fail(ALD_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  size_t n = (size_t)c->T.nibz * c->geo.b * 3;
  DevBuf<double> d;
  CKA(d.alloc(n));
  KappaArgs k = kappa_args(c, tempk);
  CK(launch_rhs(k, d.p, c->stream));
  CK(cudaMemcpyAsync(RHS, d.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ALD_OK;
}

int ald_cg_quadratic(int n, const double* a, const double* b, double* vmin, double* funcmin, int max_iter,
                     int n_dig_accur, int* iters) {
  if (n <= 0 || !a || !b || !vmin) return fail(ALD_ERR_ARG, "bad argument");
  cudaStream_t s;
  CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SG {
    cudaStream_t s;
    ~SG() { cudaStreamDestroy(s); }
  } guard{s};
  DevBuf<double> A, At, db, dx;
  CKA(A.alloc((size_t)n * n));
  CKA(At.alloc((size_t)n * n));
  CKA(db.alloc(n));
  CKA(dx.alloc(n));
  CK(cudaMemcpyAsync(A.p, a, (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, s));
  // a(n,n) column-major == A^T row-major: transpose to row-major
  CK(launch_transpose(A.p, At.p, n, n, s));
  CK(cudaMemcpyAsync(db.p, b, n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dx.p, vmin, n * sizeof(double), cudaMemcpyHostToDevice, s));
  int it = 0;
  double err = 0, fm = 0;
  std::string msg;
  double tol = 1.0 / std::pow(10.0, 2 * n_dig_accur);
  CgWork work;
  int r = cg_device(n, At.p, db.p, dx.p, max_iter, ALD_CG_REFERENCE, tol, &it, &err, &fm, s, work, msg);
  if (r != ALD_OK && r != ALD_WARN_CG_MAXITER) return fail(r, msg);
  CK(cudaMemcpyAsync(vmin, dx.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (funcmin) *funcmin = fm;
  if (iters) *iters = it;
  return r;
}

int ald_weight_tet(int ntet, const double* w, double e, int fp32, double* c) {
  if (ntet < 0 || (ntet > 0 && (!w || !c))) return fail(ALD_ERR_ARG, "bad argument");
  if (ntet == 0) return ALD_OK;
  cudaStream_t s;
  CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct SG {
    cudaStream_t s;
    ~SG() { cudaStreamDestroy(s); }
  } guard{s};
  const size_t n = (size_t)4 * ntet;
  DevBuf<double> dw, dc;
  CKA(dw.alloc(n));
  CKA(dc.alloc(n));
  CK(cudaMemcpyAsync(dw.p, w, n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(launch_weight_tet(ntet, dw.p, e, fp32 ? 1 : 0, dc.p, s));
  CK(cudaMemcpyAsync(c, dc.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return ALD_OK;
}

int ald_set_isotope_g(ald_ctx* c, const double* g) {
  if (!c || !g) return fail(ALD_ERR_ARG, "null argument");
  c->giso.assign(g, g + c->S.nat0);
  c->giso_ok = true;
  return ALD_OK;
}

int ald_get_isotope_g(ald_ctx* c, double* g) {
  if (!c || !g) return fail(ALD_ERR_ARG, "null argument");
  if (!c->giso_ok) {
    std::string e = isotope_g_atoms(c->S, c->giso);
    if (!e.empty()) return fail(ALD_ERR_UNSUPPORTED, e);
    c->giso_ok = true;
  }
  std::memcpy(g, c->giso.data(), c->giso.size() * sizeof(double));
  return ALD_OK;
}

int ald_p_iso_split(ald_ctx* c, const int ksubset[2], double* Piso) {
  if (!c || !Piso) return fail(ALD_ERR_ARG, "null argument");
  if (!ksub_ok(c, ksubset)) return fail(ALD_ERR_ARG, "ksubset out of range");
  if (c->geo.b > 12) return fail(ALD_ERR_UNSUPPORTED, "isotope scattering: more than 12 bands");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  // frequencies only (cal_freq); the temperature of the occupations does not enter
  r = ensure_dist(c, c->dist_tempk > 0 ? c->dist_tempk : c->S.tmin);
  if (r) return r;
  r = ensure_giso(c);
  if (r) return r;
  const int nr = ksubset[1] - ksubset[0] + 1, b = c->geo.b;
  DevBuf<double> part, pd;
  CKA(part.alloc(piso_partial_doubles(c->geo, nr)));
  CKA(pd.alloc((size_t)nr * b));
  CK(launch_piso(c->geo, ksubset[0] - 1, nr, c->mapinv.p, c->freq.p, c->evec.p, c->tet_corner.p, c->giso_d.p, part.p,
                 pd.p, nullptr, nullptr, nullptr, c->stream));
  std::vector<double> h((size_t)nr * b);
  CK(cudaMemcpyAsync(h.data(), pd.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < nr; ++i)
    for (int l = 0; l < b; ++l) Piso[i + (size_t)nr * l] = h[(size_t)i * b + l];
  return check_err_flags(c);
}

int ald_collision_matrix_iso(ald_ctx* c, const double* P1, const double* P2, const double* Piso, double* CM) {
  if (!c || !P1 || !P2 || !Piso || !CM) return fail(ALD_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  const int b = c->geo.b, nkc = c->T.nkc, nibz = c->T.nibz, nr = nibz;
  const size_t n = (size_t)nr * nkc * b * b * b;
  DevBuf<double> tmp, p1, p2, R1, R2, Qd, pis, cm, cmt;
  CKA(tmp.alloc(n));
  CKA(p1.alloc(n));
  CKA(p2.alloc(n));
  CKA(R1.alloc((size_t)nr * nkc * b * b));
  CKA(R2.alloc((size_t)nr * nkc * b * b));
  CKA(Qd.alloc((size_t)nr * b));
  CKA(pis.alloc((size_t)nr * b));
  const int rows = 3 * b * nr, cols = 3 * b * nibz;
  CKA(cm.alloc((size_t)rows * cols));
  CKA(cmt.alloc((size_t)rows * cols));
  std::vector<double> hp((size_t)nr * b);
  for (int i = 0; i < nr; ++i)
    for (int l = 0; l < b; ++l) hp[(size_t)i * b + l] = Piso[i + (size_t)nr * l];
  CK(cudaMemcpyAsync(pis.p, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(tmp.p, P1, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(tmp.p, p1.p, nr, nkc, b, c->stream));
  CK(cudaMemcpyAsync(tmp.p, P2, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_from_fortran5(tmp.p, p2.p, nr, nkc, b, c->stream));
  CK(launch_collapse(c->geo, nr, p1.p, p2.p, R1.p, R2.p, Qd.p, c->stream));
  CK(launch_add((size_t)nr * b, Qd.p, pis.p, c->stream));  // the diagonal: -(sum(P1 + P2/2) + Piso)
  CK(launch_collision(c->geo, nibz, 0, nr, c->mapinv.p, c->arm_off.p, c->arm_q.p, c->arm_op.p, c->opk.p, Qd.p, R1.p,
                      R2.p, cm.p, (size_t)cols, 0, pis.p, c->mesh_m.p, c->stream));
  CK(launch_transpose(cm.p, cmt.p, rows, cols, c->stream));  // row-major -> Fortran column-major
  CK(cudaMemcpyAsync(CM, cmt.p, (size_t)rows * cols * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return ALD_OK;
}

int ald_update_mpi(ald_ctx* c, const int ksubset[2], const double* P1, const double* P2, const double* Qv,
                   const double* F_RTA, const double* FFF, double* F2mpi) {
  if (!c || !P1 || !P2 || !Qv || !F_RTA || !FFF || !F2mpi) return fail(ALD_ERR_ARG, "null argument");
  if (!ksub_ok(c, ksubset)) return fail(ALD_ERR_ARG, "ksubset out of range");
  if (!c->full_op_ok) return fail(ALD_ERR_UNSUPPORTED, "update_mpi: a mesh point is not a star arm of its IBZ point");
  if (c->geo.b > 16) return fail(ALD_ERR_UNSUPPORTED, "update_mpi: more than 16 bands is not supported");
  CK(cudaSetDevice(c->device));
  const int nr = ksubset[1] - ksubset[0] + 1, b = c->geo.b, nkc = c->T.nkc, nibz = c->T.nibz;
  const size_t n = (size_t)nr * nkc * b * b * b, nm = (size_t)nr * nkc * b * b, nf = (size_t)nibz * b * 3;
  DevBuf<double> tmp, s1, s2, R1, R2, R1p, R2p, Qd, q, frta, f, ff, out;
  CKA(tmp.alloc(n));
  CKA(s1.alloc(n));
  CKA(s2.alloc(n));
  CKA(R1.alloc(nm));
  CKA(R2.alloc(nm));
  CKA(R1p.alloc(nm));
  CKA(R2p.alloc(nm));
  CKA(Qd.alloc((size_t)nr * b));
  CKA(q.alloc((size_t)nibz * b));
  CKA(frta.alloc(nf));
  CKA(f.alloc(nf));
  CKA(ff.alloc((size_t)nkc * b * 3));
  CKA(out.alloc((size_t)nr * b * 3));
  DevBuf<double> part;
  CKA(part.alloc(update_part_doubles(c->geo, nr)));
  cudaStream_t s = c->stream;
  CK(cudaMemcpyAsync(tmp.p, P1, n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(launch_from_fortran5(tmp.p, s1.p, nr, nkc, b, s));
  CK(cudaMemcpyAsync(tmp.p, P2, n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(launch_from_fortran5(tmp.p, s2.p, nr, nkc, b, s));
  CK(launch_collapse(c->geo, nr, s1.p, s2.p, R1.p, R2.p, Qd.p, s));
  CK(launch_marginal_l2(c->geo, nr, s1.p, s2.p, R1p.p, R2p.p, s));
  // Q(nibz,ndyn), F_RTA and FFF (nibz,ndyn,3) to [n][l] and [n][l][xyz]
  std::vector<double> hq((size_t)nibz * b), hr(nf), hf(nf);
  for (int i = 0; i < nibz; ++i)
    for (int l = 0; l < b; ++l) {
      hq[(size_t)i * b + l] = Qv[i + (size_t)nibz * l];
      for (int x = 0; x < 3; ++x) {
        hr[((size_t)i * b + l) * 3 + x] = F_RTA[i + (size_t)nibz * (l + (size_t)b * x)];
        hf[((size_t)i * b + l) * 3 + x] = FFF[i + (size_t)nibz * (l + (size_t)b * x)];
      }
    }
  CK(cudaMemcpyAsync(q.p, hq.data(), hq.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(frta.p, hr.data(), nf * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(f.p, hf.data(), nf * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(launch_ffull(c->geo, c->mapibz0.p, c->full_op.p, c->opk.p, f.p, ff.p, s));
  CK(launch_update(c->geo, ksubset[0] - 1, nr, c->mapinv.p, R1.p, R1p.p, R2.p, R2p.p, ff.p, q.p, frta.p, f.p, 0.0,
                   out.p, part.p, s));
  std::vector<double> ho((size_t)nr * b * 3);
  CK(cudaMemcpyAsync(ho.data(), out.p, ho.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int i = 0; i < nr; ++i)
    for (int l = 0; l < b; ++l)
      for (int x = 0; x < 3; ++x) F2mpi[i + (size_t)nr * (l + (size_t)b * x)] = ho[((size_t)i * b + l) * 3 + x];
  return ALD_OK;
}

int ald_mode_kappa_d(ald_ctx* c, double tempk, const double* Fi_x, double* kappa) {
  if (!c || !Fi_x || !kappa) return fail(ALD_ERR_ARG, "null argument");
  CK(cudaSetDevice(c->device));
  int r = ensure_phonons(c);
  if (r) return r;
  r = ensure_dist(c, tempk);
  if (r) return r;
  const int b = c->geo.b;
  size_t n = (size_t)c->T.nibz * b * 3;
  DevBuf<double> dF, dk;
  CKA(dF.alloc(n));
  CKA(dk.alloc((size_t)b * 9));
  CK(cudaMemcpyAsync(dF.p, Fi_x, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  KappaArgs k = kappa_args(c, tempk);
  CK(launch_kappa(k, dF.p, 1, dk.p, c->err.p, c->stream));
  CK(cudaMemcpyAsync(kappa, dk.p, (size_t)b * 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_err_flags(c);
}

}  // extern "C"
