// The pipeline's autotuner: launch shapes chosen per workload shape by timing
// them, with an on-disk cache.  No counterpart in the reference, which has a
// single code path per routine.
//
// A shape is the device, the cell's band count, the q-mesh, the IBZ row count,
// the precision, the delta and the deterministic option.  For it the tuner
// times whole pipeline calls (ald_kappa_pipeline, device time of its stage
// events, the better of two calls so that allocations of a new workspace size
// stay outside) over a small candidate set, one knob at a time starting from
// the current choice:
//   1. the |V3|^2 chunk (IBZ rows per V3 and delta launch; 256 MiB .. 2 GiB,
//      within a quarter of the free device memory);
//   2. mixed path, 3 bands: the tensor-core V3's IBZ rows per CTA (phase-tile
//      reuse against grid size) and its epilogue warpgroups (2 or 3);
//   3. mixed path, 9 bands and up: the pair-batch workspace of the
//      tensor-core mode-product GEMMs (launch count against L2 reuse).
// The best choice stays on the context and goes into the cache file as one
// line "<shape> chunk_bytes=.. rpc=.. wg=.. gemm_bytes=.. ms=..", replaced
// in place when the shape is tuned again; a later call for the same shape
// reads it instead of timing.  Every knob changes launch shapes only: the
// per-pair and per-row arithmetic, and so the results, stay the same.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "ald_ctx.h"

using namespace ald::capi;

namespace {

struct Choice {
  size_t chunk_bytes = 0;
  int rpc = 0, wg = 0;
  size_t gemm_bytes = 0;
  double ms = 0;
};

std::mutex g_tune_mu;  // one tuner per process touches the cache file at a time

// the device's name and compute capability, looked up once per device
// (cudaGetDeviceProperties takes milliseconds)
std::string device_tag(int device) {
  static std::mutex mu;
  static std::map<int, std::string> tags;
  std::lock_guard<std::mutex> lk(mu);
  auto it = tags.find(device);
  if (it != tags.end()) return it->second;
  cudaDeviceProp p;
  std::string dev = "device";
  if (cudaGetDeviceProperties(&p, device) == cudaSuccess) {
    dev = p.name;
    dev += "-sm" + std::to_string(p.major) + std::to_string(p.minor);
  }
  for (char& ch : dev)
    if (ch == ' ' || ch == '\t') ch = '_';
  tags[device] = dev;
  return dev;
}

std::string shape_key(const ald_ctx* c) {
  const std::string dev = device_tag(c->device);
  std::ostringstream k;
  k << dev << "|b" << c->geo.b << "|mesh" << c->geo.nc[0] << "x" << c->geo.nc[1] << "x" << c->geo.nc[2] << "|nibz"
    << c->T.nibz << "|prec" << c->opt.precision << "|delta" << delta_mode(const_cast<ald_ctx*>(c)) << "|det"
    << c->opt.deterministic;
  return k.str();
}

bool cache_read(const std::string& path, const std::string& key, Choice& out) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  while (std::getline(f, line)) {
    const size_t sp = line.find(' ');
    if (sp == std::string::npos || line.compare(0, sp, key) != 0) continue;
    unsigned long long cb = 0, gb = 0;
    int rpc = 0, wg = 0;
    double ms = 0;
    if (std::sscanf(line.c_str() + sp, " chunk_bytes=%llu rpc=%d wg=%d gemm_bytes=%llu ms=%lf", &cb, &rpc, &wg, &gb,
                    &ms) == 5) {
      out.chunk_bytes = (size_t)cb;
      out.rpc = rpc;
      out.wg = wg;
      out.gemm_bytes = (size_t)gb;
      out.ms = ms;
      return true;
    }
  }
  return false;
}

bool cache_write(const std::string& path, const std::string& key, const Choice& ch) {
  std::vector<std::string> lines;
  {
    std::ifstream f(path);
    std::string line;
    while (f && std::getline(f, line))
      if (line.compare(0, key.size() + 1, key + " ") != 0 && !line.empty()) lines.push_back(line);
  }
  char buf[256];
  std::snprintf(buf, sizeof buf, " chunk_bytes=%llu rpc=%d wg=%d gemm_bytes=%llu ms=%.6f",
                (unsigned long long)ch.chunk_bytes, ch.rpc, ch.wg, (unsigned long long)ch.gemm_bytes, ch.ms);
  lines.push_back(key + buf);
  // a whole new file, then rename: readers see the old or the new file
  const std::string tmp = path + ".tmp" + std::to_string((long long)std::rand());
  {
    std::ofstream f(tmp);
    if (!f) return false;
    for (const auto& l : lines) f << l << "\n";
    if (!f) return false;
  }
  return std::rename(tmp.c_str(), path.c_str()) == 0;
}

void apply(ald_ctx* c, const Choice& ch) {
  c->opt.chunk_bytes = ch.chunk_bytes;
  c->tune_v3_rpc = ch.rpc;
  c->tune_v3_wg = ch.wg;
  c->tune_gemm_bytes = ch.gemm_bytes;
}

// device time of one pipeline call with choice ch (the better of two calls)
int time_choice(ald_ctx* c, const Choice& ch, double tempk, double& ms) {
  apply(c, ch);
  ms = 1e300;
  for (int rep = 0; rep < 2; ++rep) {
    c->v3c_epoch = 0;  // time V3 too, not the kept |V3|^2
    ald_kappa_result r;
    const int st = ald_kappa_pipeline(c, tempk, &r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    if (st != ALD_OK && st != ALD_WARN_CG_MAXITER) return st;
    ms = std::min(ms, r.stage_ms[9]);
  }
  return ALD_OK;
}

void fill(const Choice& ch, int from_cache, int ncand, ald_tuning* out) {
  if (!out) return;
  out->chunk_bytes = ch.chunk_bytes;
  out->v3_rows_per_cta = ch.rpc;
  out->v3_epilogue_wg = ch.wg;
  out->v3_gemm_bytes = ch.gemm_bytes;
  out->ms = ch.ms;
  out->from_cache = from_cache;
  out->candidates = ncand;
}

}  // namespace

extern "C" {

int ald_set_tuning(ald_ctx* c, const ald_tuning* t) {
  if (!c || !t) return fail(ALD_ERR_ARG, "null argument");
  if (t->v3_rows_per_cta < 0 || t->v3_rows_per_cta > 16 ||
      (t->v3_epilogue_wg != 0 && t->v3_epilogue_wg != 2 && t->v3_epilogue_wg != 3))
    return fail(ALD_ERR_ARG, "tuning out of range (rows per CTA 0..16, epilogue warpgroups 0, 2 or 3)");
  Choice ch;
  ch.chunk_bytes = t->chunk_bytes;
  ch.rpc = t->v3_rows_per_cta;
  ch.wg = t->v3_epilogue_wg;
  ch.gemm_bytes = t->v3_gemm_bytes;
  apply(c, ch);
  return ALD_OK;
}

int ald_autotune(ald_ctx* c, const char* cache_path, double budget_s, ald_tuning* out) {
  if (!c) return fail(ALD_ERR_ARG, "null context");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::string path = cache_path ? cache_path : "";
  if (path.empty()) {
    const char* e = std::getenv("ALD_TUNE_CACHE");
    if (e) path = e;
  }
  const std::string key = shape_key(c);
  Choice best;
  if (!path.empty() && cache_read(path, key, best)) {
    apply(c, best);
    fill(best, 1, 0, out);
    return ALD_OK;
  }
  ALD_CK(cudaSetDevice(c->device));
  const double tempk = c->S.tmin;
  if (budget_s <= 0) budget_s = 10.0;
  const auto t0 = std::chrono::steady_clock::now();
  auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
  best.chunk_bytes = c->opt.chunk_bytes;
  best.rpc = c->tune_v3_rpc;
  best.wg = c->tune_v3_wg;
  best.gemm_bytes = c->tune_gemm_bytes;
  int r = time_choice(c, best, tempk, best.ms);
  if (r) return r;
  int ncand = 1;
  auto trial = [&](Choice ch) -> int {
    if (elapsed() > budget_s) return ALD_OK;
    ++ncand;
    const int st = time_choice(c, ch, tempk, ch.ms);
    if (st == ALD_ERR_NOMEM) return ALD_OK;  // a candidate that does not fit is skipped
    if (st) return st;
    if (ch.ms < best.ms) best = ch;
    return ALD_OK;
  };
  // 1. the |V3|^2 chunk
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  for (size_t mb : {256, 1024, 2048}) {
    Choice ch = best;
    ch.chunk_bytes = mb << 20;
    if (ch.chunk_bytes == best.chunk_bytes || ch.chunk_bytes > fr / 4) continue;
    r = trial(ch);
    if (r) break;
  }
  // 2. 3-band tensor-core V3: rows per CTA x epilogue warpgroups
  if (!r && c->opt.precision == ALD_MIXED && v3_tc_supported(c->geo.b, c->VC.ncls)) {
    const Choice base = best;
    for (int rpc : {2, 4, 8, 16})
      for (int wg : {2, 3}) {
        Choice ch = base;
        ch.rpc = rpc;
        ch.wg = wg;
        if (!r) r = trial(ch);
      }
  }
  // 3. large cells: the GEMM pair-batch workspace
  if (!r && c->opt.precision == ALD_MIXED && v3_dense_tc_supported(c->geo.b)) {
    const Choice base = best;
    for (size_t mb : {512, 1024, 4096}) {
      Choice ch = base;
      ch.gemm_bytes = mb << 20;
      if (ch.gemm_bytes > fr / 4) continue;
      if (!r) r = trial(ch);
    }
  }
  apply(c, best);
  if (r) return r;
  if (!path.empty() && !cache_write(path, key, best))
    return fail(ALD_ERR_IO, "autotune: cannot write the cache file " + path);
  fill(best, 0, ncand, out);
  return ALD_OK;
}

}  // extern "C"
