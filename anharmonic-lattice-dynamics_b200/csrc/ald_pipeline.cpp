// ald_kappa_pipeline: the whole job=1 sequence of THERMACOND/kappa.f90:389-871
// on the device, without materialising any (nibz, nkc, ndyn^3) array:
//
//   phonons (get_frequencies + subst_eivecs)      unless injected
//   distribution                                   sub.f90:1955
//   for each chunk of IBZ rows:
//     |V3|^2                  calculate_w3_ibz_split_sq  sub.f90:1050
//     delta, Bose, band sums  calculate_FGR_mpi2 + calculate_tauRTA_mpi2
//   Q, Q_N, Q_U                                   (MPI_Allgatherv at kappa.f90:641 is a no-op here)
//   F_RTA, kappa_RTA          sub.f90:1238, 1292
//   collision matrix          CollisionMatrix_mpi sub.f90:3034 (kept row-major on the device)
//   RHS, CG, kappa            sub.f90:2618, cg.f90:19, sub.f90:1407
//
// Every stage is bracketed by CUDA events on the context's stream; the
// per-stage device times and kernel launch counts come back in the result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ald_ctx.h"

using namespace ald;
using namespace ald::capi;

namespace {

struct StageTimer {
  cudaStream_t s;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  cudaEvent_t open_ev = nullptr;
  int open_stage = -1;
  cudaError_t begin(int stage) {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return r;
    open_ev = e;
    open_stage = stage;
    return cudaEventRecord(e, s);
  }
  cudaError_t end() {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return r;
    r = cudaEventRecord(e, s);
    marks.push_back({open_stage, {open_ev, e}});
    open_ev = nullptr;
    return r;
  }
  void collect(double* ms) {
    for (auto& m : marks) {
      float t = 0;
      cudaEventElapsedTime(&t, m.second.first, m.second.second);
      ms[m.first] += t;
    }
  }
  ~StageTimer() {
    for (auto& m : marks) {
      cudaEventDestroy(m.second.first);
      cudaEventDestroy(m.second.second);
    }
    if (open_ev) cudaEventDestroy(open_ev);
  }
};

}  // namespace

// the job=3 iteration of kappa.f90:1390-1487 in place of the CG solve
struct IterSpec {
  int max_iter;
  double mix;
  double* F;  // optional out: FFF(nibz, ndyn, 3)
};

// the row split of the reference's MPI job (kappa.f90:418-428): nibz/nranks
// rows per rank, the last rank also takes the remainder; 0-based [rb, re)
static void shard_range(int nibz, int rank, int nranks, int& rb, int& re) {
  const int local = nibz / nranks;
  rb = rank * local;
  re = rank == nranks - 1 ? nibz : rb + local;
}

// one rank of a row-sharded job=1 (the reference's MPI decomposition): this
// rank computes V3, the delta, Q and the collision-matrix rows of its IBZ
// rows; Q and the CG matrix-vector products are exchanged through `gather`
struct ShardSpec {
  int rank, nranks;
  ald_allgather_fn gather;         // host buffers, or
  ald_allgather_dev_fn gather_dev; // device buffers, ordered on the context's stream
  void* user;
};

static int run_pipeline(ald_ctx* c, double tempk, ald_kappa_result* res, double* Qo, double* QNo, double* QUo,
                        double* kappa_rta_modes, double* kappa_cg_modes, double* xo, const IterSpec* it,
                        const ShardSpec* sh = nullptr) {
  if (!c || !res) return fail(ALD_ERR_ARG, "null argument");
  if (sh && (sh->nranks < 1 || sh->rank < 0 || sh->rank >= sh->nranks || (!sh->gather && !sh->gather_dev)))
    return fail(ALD_ERR_ARG, "sharded pipeline: bad rank, rank count or exchange function");
  if (sh && it) return fail(ALD_ERR_UNSUPPORTED, "the sharded pipeline runs job=1 only");
  if (it && !c->full_op_ok) return fail(ALD_ERR_UNSUPPORTED, "update_mpi: a mesh point is not a star arm of its IBZ point");
  // job=3 with iso=1 has no defined result to reproduce: kappa_full deallocates
  // Piso (kappa.f90:1252) before update_iso reads it (sub.f90:2598)
  if (it && c->S.iso == 1)
    return fail(ALD_ERR_UNSUPPORTED,
                "job=3 with iso=1: the reference frees Piso (kappa.f90:1252) before update_iso reads it "
                "(sub.f90:2598), so there is no defined result to reproduce");
  if (c->S.include_fc[2] != 1) return fail(ALD_ERR_ARG, "fc3 terms are not included (include_fc(3) /= 1)");
  if (c->geo.b > kHeevMaxBands)
    return fail(ALD_ERR_UNSUPPORTED, "pipeline: more than 256 bands is not supported by this build");
  if (it && c->geo.b > kDeltaSmallBands)
    return fail(ALD_ERR_UNSUPPORTED, "job=3: more than 16 bands is not supported by this build");
  ALD_CK(cudaSetDevice(c->device));
  std::memset(res, 0, sizeof *res);
  cudaStream_t s = c->stream;
  StageTimer tm;
  tm.s = s;
  const int b = c->geo.b, nkc = c->T.nkc, nibz = c->T.nibz;
  cudaEvent_t t0, t1;
  ALD_CK(cudaEventCreate(&t0));
  ALD_CK(cudaEventCreate(&t1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evg{t0, t1};
  ALD_CK(cudaEventRecord(t0, s));
  // ---- 0: phonons and occupations
  ALD_CK(tm.begin(0));
  bool had = c->have_phonons;
  int r = ensure_phonons(c);
  if (r) return r;
  if (!had) res->launches[0] += 3;
  if (c->dist_tempk != tempk) res->launches[0] += 1;
  r = ensure_dist(c, tempk);
  if (r) return r;
  ALD_CK(tm.end());
  // this rank's IBZ rows [rb, re) (all rows unless sharded)
  int rb = 0, re = nibz;
  if (sh) shard_range(nibz, sh->rank, sh->nranks, rb, re);
  const int nloc = re - rb;
  // exchange of per-row blocks of `unit` values through the caller's
  // all-gather, staged in host memory
  auto gather_rows = [&](const double* mine, double* all, size_t unit) -> int {
    std::vector<long long> counts(sh->nranks);
    for (int k2 = 0; k2 < sh->nranks; ++k2) {
      int a0, a1;
      shard_range(nibz, k2, sh->nranks, a0, a1);
      counts[k2] = (long long)(a1 - a0) * (long long)unit;
    }
    if (sh->gather_dev)  // device buffers: no staging, ordered on the stream
      return sh->gather_dev(sh->user, mine, (long long)nloc * (long long)unit, all, counts.data(), sh->nranks,
                            (void*)s) != 0
                 ? ALD_ERR_ARG
                 : ALD_OK;
    std::vector<double> hm((size_t)nloc * unit), ha((size_t)nibz * unit);
    if (!hm.empty() && cudaMemcpyAsync(hm.data(), mine, hm.size() * sizeof(double), cudaMemcpyDeviceToHost, s))
      return ALD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return ALD_ERR_CUDA;
    if (sh->gather(sh->user, hm.data(), (long long)hm.size(), ha.data(), counts.data(), sh->nranks) != 0)
      return ALD_ERR_ARG;
    if (cudaMemcpyAsync(all, ha.data(), ha.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return ALD_ERR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? ALD_OK : ALD_ERR_CUDA;
  };
  // ---- 1, 2: V3 and delta/Bose/band sums, chunk by chunk (this rank's rows)
  const size_t rsz = (size_t)std::max(nloc, 1) * nkc * b * b;
  DevBuf<double>& R1 = c->w_R1;
  DevBuf<double>& R2 = c->w_R2;
  DevBuf<double>& Q = c->w_Q;
  DevBuf<double>& v3 = c->w_v3;
  DevBuf<char>& escratch = c->w_scratch;
  ALD_CKA(R1.alloc(rsz));
  ALD_CKA(R2.alloc(rsz));
  if (it) {  // update_mpi also needs the band marginals over l2
    ALD_CKA(c->w_R1p.alloc(rsz));
    ALD_CKA(c->w_R2p.alloc(rsz));
  }
  ALD_CKA(Q.alloc((size_t)3 * nibz * b));
  const int gauss = delta_mode(c) == ALD_DELTA_GAUSS;
  // tetrahedron: weights straight into R1/R2 (no corner-energy/weight arrays)
  // the delta kernels read |V3|^2 slice by slice (coalesced over q2): the
  // class-form V3 kernels write that layout; the large-cell tensor-core V3
  // writes runs of l1 instead (layout 2)
  const int v3_layout = v3_pipeline_layout(b, c->opt.precision);
  const bool mixed = c->opt.precision != ALD_FP64;
  const bool fused = !gauss && v3_layout != 2 && delta_fused_supported(c->geo);
  // deterministic option: the fused delta in two passes with fixed-point sums
  // (the same bits on every run); its per-entry largest terms need a buffer
  // of the chunk's R1/R2 (and R1p/R2p) size
  const bool det = fused && (c->opt.deterministic > 0 ||
                             (c->opt.deterministic == ALD_DET_AUTO && c->opt.precision == ALD_FP64));
  // more than 16 bands, or layout 2: the band-generic delta kernels, straight into R1/R2
  const bool any = !fused && (b > kDeltaSmallBands || v3_layout == 2);
  // the mixed pipeline hands |V3|^2 to the delta in FP32 where the delta
  // reads it so: the large-cell tensor-core V3 (layout 2), and the class-form
  // V3 of 3 and 6 bands into the fused tetrahedron delta.  Half the bytes,
  // twice the rows per chunk.
  const bool v3f = v3_layout == 2 || (mixed && fused && v3_layout == 1 && (b == 3 || b == 6));
  const int K = v3f ? std::min(nibz, 2 * rows_per_chunk(c)) : rows_per_chunk(c);
  const size_t v3n = (size_t)K * nkc * b * b * b;
  ALD_CKA(v3.alloc(v3f ? (v3n + 1) / 2 : v3n));
  const size_t rchunk = (size_t)K * nkc * b * b;  // entries of one chunk's R1
  if (det) ALD_CKA(c->w_rmax.alloc((it ? 4 : 2) * rchunk));
  if (!fused && !any) ALD_CKA(escratch.alloc(std::max<size_t>(256, combine_scratch_bytes(c->geo, K, gauss))));
  ALD_CKA(c->w_brange.alloc((size_t)2 * b));
  ALD_CK(launch_band_range(c->geo, c->freq.p, c->w_brange.p, s));
  res->launches[0] += 1;  // band ranges of the occupations, outside the timed delta stage
  // one chunk holds every row: |V3|^2 kept from an earlier call with the same
  // eigenpairs and rows is reused (a run over several temperatures forms it once)
  const bool one_chunk = re - rb <= K;
  const bool v3_kept = one_chunk && c->v3c_epoch != 0 && c->v3c_epoch == c->phonon_epoch && c->v3c_rb == rb &&
                       c->v3c_re == re && c->v3c_layout == v3_layout && c->v3c_f32 == v3f && c->v3c_ptr == v3.p &&
                       c->v3c_n == v3.n;
  c->v3c_epoch = 0;
  for (int r0 = rb; r0 < re; r0 += K) {
    int nr = std::min(K, re - r0);
    ALD_CK(tm.begin(1));
    if (!v3_kept) {
      V3Args va = v3_args(c, r0, nr, v3.p);
      va.v3_layout = v3_layout;
      if (v3f) va.v3sq_f32 = reinterpret_cast<float*>(v3.p);
      r = run_v3(c, va, &res->launches[1]);
      if (r) return r;
    }
    ALD_CK(tm.end());
    if (one_chunk) {
      c->v3c_epoch = c->phonon_epoch;
      c->v3c_rb = rb;
      c->v3c_re = re;
      c->v3c_layout = v3_layout;
      c->v3c_f32 = v3f;
      c->v3c_ptr = v3.p;
      c->v3c_n = v3.n;
    }
    CombineArgs a;
    a.geo = c->geo;
    a.n1_first = r0;
    a.nrows = nr;
    a.mapinv = c->mapinv.p;
    a.v3sq = v3.p;
    a.v3_layout = v3_layout;
    a.v3sq_f32 = v3f ? reinterpret_cast<const float*>(v3.p) : nullptr;
    a.freq = c->freq.p;
    a.dist = c->dist.p;
    a.tet_corner = c->tet_corner.p;
    a.tet_inc = c->tet_inc.p;
    a.gauss = gauss;
    a.sigma = gauss_width(c);
    a.f32w = c->opt.precision != ALD_FP64;  // mixed: FP32 delta weights
    a.brange = c->w_brange.p;
    a.R1 = R1.p + (size_t)(r0 - rb) * nkc * b * b;
    a.R2 = R2.p + (size_t)(r0 - rb) * nkc * b * b;
    a.P1s = a.P2s = a.P1 = a.P2 = nullptr;
    a.R1p = it ? c->w_R1p.p + (size_t)r0 * nkc * b * b : nullptr;
    a.R2p = it ? c->w_R2p.p + (size_t)r0 * nkc * b * b : nullptr;
    // the sums that the delta kernels add into start at zero; the zeroing
    // runs outside the delta stage, so that stage times the kernel alone
    const size_t rbytes = (size_t)nr * nkc * b * b * sizeof(double);
    if (it) {
      ALD_CK(cudaMemsetAsync(a.R1p, 0, rbytes, s));
      ALD_CK(cudaMemsetAsync(a.R2p, 0, rbytes, s));
    }
    if (det) {
      unsigned long long* M = reinterpret_cast<unsigned long long*>(c->w_rmax.p);
      a.M1 = M;
      a.M2 = M + rchunk;
      a.M1p = it ? M + 2 * rchunk : nullptr;
      a.M2p = it ? M + 3 * rchunk : nullptr;
      ALD_CK(cudaMemsetAsync(M, 0, (it ? 4 : 2) * rchunk * sizeof(unsigned long long), s));
    }
    if (fused || (any && !gauss)) {
      ALD_CK(cudaMemsetAsync(a.R1, 0, rbytes, s));
      ALD_CK(cudaMemsetAsync(a.R2, 0, rbytes, s));
    }
    ALD_CK(tm.begin(2));
    if (det) {
      const size_t n = (size_t)nr * nkc * b * b;
      ALD_CK(launch_delta_fused(a, s, 1));
      ALD_CK(launch_delta_fused(a, s, 2));
      ALD_CK(launch_delta_finalize(a.R1, a.M1, n, b, s));
      ALD_CK(launch_delta_finalize(a.R2, a.M2, n, b, s));
      res->launches[2] += 4;
      if (it) {
        ALD_CK(launch_delta_finalize(a.R1p, a.M1p, n, b, s));
        ALD_CK(launch_delta_finalize(a.R2p, a.M2p, n, b, s));
        res->launches[2] += 2;
      }
    } else if (fused) {
      ALD_CK(launch_delta_fused(a, s));
      res->launches[2] += 1;
    } else if (any) {
      ALD_CK(launch_delta_any(a, s));
      res->launches[2] += 1;
    } else {
      ALD_CK(launch_combine(a, escratch.p, s));
      res->launches[2] += gauss ? 1 : 3;
    }
    ALD_CK(tm.end());
  }
  // ---- 3: Q, Q_N, Q_U from the band sums
  double* dQ = Q.p;
  double* dQN = Q.p + (size_t)nibz * b;
  double* dQU = Q.p + (size_t)2 * nibz * b;
  ALD_CK(tm.begin(3));
  if (nloc > 0) ALD_CK(launch_q_from_r(c->geo, rb, nloc, c->mapinv.p, R1.p, R2.p, dQ, dQN, dQU, nibz, s));
  res->launches[3] += 1;
  // iso=1: isotope scattering (P_iso_split), Q, Q_N, Q_U += Piso as in
  // calculate_tauRTA_iso (sub.f90:8311-8549)
  const bool iso = c->S.iso == 1;
  if (iso) {
    r = ensure_giso(c);
    if (r) return r;
    ALD_CKA(c->w_piso.alloc((size_t)std::max(nloc, 1) * b));
    ALD_CKA(c->w_piso_part.alloc(piso_partial_doubles(c->geo, std::max(nloc, 1))));
    if (nloc > 0)
      ALD_CK(launch_piso(c->geo, rb, nloc, c->mapinv.p, c->freq.p, c->evec.p, c->tet_corner.p, c->giso_d.p,
                         c->w_piso_part.p, c->w_piso.p, dQ + (size_t)rb * b, dQN + (size_t)rb * b,
                         dQU + (size_t)rb * b, s));
    res->launches[3] += 2;
  }
  if (sh) {  // every rank needs Q of every row (MPI_Allgatherv, kappa.f90:641-643)
    for (double* q : {dQ, dQN, dQU}) {
      r = gather_rows(q + (size_t)rb * b, q, (size_t)b);
      if (r) return fail(r, "sharded pipeline: the exchange of Q failed");
    }
  }
  ALD_CK(tm.end());
  // ---- 4: RTA
  KappaArgs k = kappa_args(c, tempk);
  const size_t N = (size_t)3 * b * nibz;
  DevBuf<double>& F = c->w_F;
  DevBuf<double>& x = c->w_x;
  DevBuf<double>& rhs = c->w_rhs;
  DevBuf<double>& kr = c->w_kr;
  DevBuf<double>& kc = c->w_kc;
  DevBuf<double>& cm = c->w_cm;
  ALD_CKA(F.alloc(N));
  ALD_CKA(x.alloc(N));
  ALD_CKA(rhs.alloc(N));
  ALD_CKA(kr.alloc((size_t)9 * b));
  ALD_CKA(kc.alloc((size_t)9 * b));
  ALD_CK(tm.begin(4));
  ALD_CK(launch_rta_F(k, dQ, F.p, s));
  ALD_CK(launch_kappa(k, F.p, 0, kr.p, c->err.p, s));
  res->launches[4] += 2;
  ALD_CK(tm.end());
  if (it) {
    // ---- 7: FFF += mix (update_mpi(FFF) - FFF), kappa = mode_kappa(FFF), until
    // sqrt(sum((kappa_new - kappa_old)^2) / (ndyn*9)) < 1e-4 (kappa.f90:1390-1487)
    DevBuf<double>& Ff = c->w_Ff;
    DevBuf<double>& Frta = c->w_Frta;
    ALD_CKA(Ff.alloc((size_t)nkc * b * 3));
    ALD_CKA(Frta.alloc(N));
    ALD_CKA(c->w_part.alloc(update_part_doubles(c->geo, nibz)));
    ALD_CK(cudaMemcpyAsync(Frta.p, F.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ALD_CK(tm.begin(7));
    std::vector<double> kold((size_t)9 * b), knew((size_t)9 * b);
    ALD_CK(cudaMemcpyAsync(kold.data(), kr.p, kold.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    ALD_CK(cudaStreamSynchronize(s));
    int iters = 0;
    double normk = 0;
    bool conv = false;
    for (int i = 1; i <= it->max_iter; ++i) {
      ALD_CK(launch_ffull(c->geo, c->mapibz0.p, c->full_op.p, c->opk.p, F.p, Ff.p, s));
      ALD_CK(launch_update(c->geo, 0, nibz, c->mapinv.p, R1.p, c->w_R1p.p, R2.p, c->w_R2p.p, Ff.p, dQ, Frta.p, F.p,
                           it->mix, F.p, c->w_part.p, s));
      ALD_CK(launch_kappa(k, F.p, 0, kc.p, c->err.p, s));
      res->launches[7] += 3;
      ALD_CK(cudaMemcpyAsync(knew.data(), kc.p, knew.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      ALD_CK(cudaStreamSynchronize(s));
      double e = 0;
      for (int j = 0; j < 9 * b; ++j) e = e + (knew[j] - kold[j]) * (knew[j] - kold[j]) / (b * 3 * 3);
      iters = i;
      normk = std::sqrt(e);
      if (normk < 0.0001) {
        conv = true;
        break;
      }
      kold = knew;
    }
    ALD_CK(tm.end());
    ALD_CK(cudaEventRecord(t1, s));
    std::vector<double> hkr((size_t)9 * b), hF;
    ALD_CK(cudaMemcpyAsync(hkr.data(), kr.p, hkr.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    double d2h = 2.0 * hkr.size() * sizeof(double) * (1 + iters);
    std::vector<double> hq;
    if (Qo || QNo || QUo) {
      hq.resize((size_t)3 * nibz * b);
      ALD_CK(cudaMemcpyAsync(hq.data(), Q.p, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      d2h += hq.size() * sizeof(double);
    }
    if (it->F) {
      hF.resize(N);
      ALD_CK(cudaMemcpyAsync(hF.data(), F.p, N * sizeof(double), cudaMemcpyDeviceToHost, s));
      d2h += N * sizeof(double);
    }
    ALD_CK(cudaStreamSynchronize(s));
    r = check_err_flags(c);
    if (r) return r;
    tm.collect(res->stage_ms);
    float total = 0;
    cudaEventElapsedTime(&total, t0, t1);
    res->stage_ms[9] = total;
    for (int i = 0; i < 9; ++i) res->launches[9] += res->launches[i];
    for (int e = 0; e < 9; ++e) {
      double sr = 0, sc = 0;
      for (int l = 0; l < b; ++l) {
        sr += hkr[l + (size_t)b * e];
        sc += knew[l + (size_t)b * e];
      }
      res->kappa_rta[e] = sr;
      res->kappa_cg[e] = sc;
    }
    if (kappa_rta_modes) std::memcpy(kappa_rta_modes, hkr.data(), hkr.size() * sizeof(double));
    if (kappa_cg_modes) std::memcpy(kappa_cg_modes, knew.data(), knew.size() * sizeof(double));
    for (int i = 0; i < nibz; ++i)
      for (int l = 0; l < b; ++l) {
        if (Qo) Qo[i + (size_t)nibz * l] = hq[(size_t)i * b + l];
        if (QNo) QNo[i + (size_t)nibz * l] = hq[(size_t)nibz * b + (size_t)i * b + l];
        if (QUo) QUo[i + (size_t)nibz * l] = hq[(size_t)2 * nibz * b + (size_t)i * b + l];
        if (it->F)
          for (int x = 0; x < 3; ++x) it->F[i + (size_t)nibz * (l + (size_t)b * x)] = hF[((size_t)i * b + l) * 3 + x];
      }
    res->cg_iters = iters;
    res->status_cg = conv ? ALD_OK : ALD_WARN_CG_MAXITER;
    res->cg_err = normk;
    res->triplet_bands = (double)nibz * nkc * (double)b * b * b;
    res->d2h_bytes = d2h;
    return ALD_OK;
  }
  // ---- 5: collision matrix (row-major, all IBZ rows; rows padded to 16
  // bytes).  The mixed-precision pipeline stores it in FP32: CG streams it
  // once per iteration, and the products are still summed in FP64.
  const int cm_f32 = c->opt.precision != ALD_FP64;
  const size_t ld = cm_f32 ? (N + 3) / 4 * 4 : (N + 1) / 2 * 2;
  const size_t Nloc = (size_t)3 * b * nloc;  // this rank's rows of the matrix
  const size_t cm_bytes = std::max<size_t>(Nloc, 1) * ld * (cm_f32 ? sizeof(float) : sizeof(double));
  ALD_CKA(cm.alloc((cm_bytes + sizeof(double) - 1) / sizeof(double)));
  ALD_CK(tm.begin(5));
  if (nloc > 0)
    ALD_CK(launch_collision(c->geo, nibz, rb, nloc, c->mapinv.p, c->arm_off.p, c->arm_q.p, c->arm_op.p, c->opk.p,
                            dQ + (size_t)rb * b, R1.p, R2.p, cm.p, ld, cm_f32, iso ? c->w_piso.p : nullptr,
                            c->mesh_m.p, s));
  res->launches[5] += 1;
  ALD_CK(tm.end());
  // ---- 6: RHS and the initial guess x0 = F_RTA (kappa.f90:835-843)
  ALD_CK(tm.begin(6));
  ALD_CK(launch_rhs(k, rhs.p, s));
  ALD_CK(cudaMemcpyAsync(x.p, F.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  res->launches[6] += 1;
  ALD_CK(tm.end());
  // ---- 7: cg_quadratic(nibz*ndyn*3, CM, RHS, x, fm, 100, 2) (kappa.f90:846)
  int iters = 0;
  double cg_err = 0, fm = 0;
  std::string msg;
  double tol = c->opt.cg_stop == ALD_CG_REFERENCE ? 1.0 / std::pow(10.0, 2 * c->opt.cg_ndig) : c->opt.cg_tol;
  ALD_CK(tm.begin(7));
  int rc;
  if (sh) {
    const CgAllGather gather = [&](const double* mine, size_t, double* all) {
      return gather_rows(mine, all, (size_t)3 * b);
    };
    rc = cg_device_rows((int)N, 3 * b * rb, (int)Nloc, ld, cm.p, cm_f32, rhs.p, x.p, c->opt.cg_max_iter,
                        c->opt.cg_stop, tol, gather, &iters, &cg_err, &fm, s, c->cg, msg);
    res->launches[7] += 4 + 4 * iters;
  } else {
    rc = cg_device_ld((int)N, ld, cm.p, cm_f32, rhs.p, x.p, c->opt.cg_max_iter, c->opt.cg_stop, tol, &iters, &cg_err,
                      &fm, s, c->cg, msg);
    res->launches[7] += 4 + 3 * cg_launched_iterations(iters, c->opt.cg_max_iter);
  }
  if (rc != ALD_OK && rc != ALD_WARN_CG_MAXITER) return fail(rc, msg);
  ALD_CK(tm.end());
  // ---- 8: mode_kappa_d
  ALD_CK(tm.begin(8));
  ALD_CK(launch_kappa(k, x.p, 1, kc.p, c->err.p, s));
  res->launches[8] += 1;
  ALD_CK(tm.end());
  ALD_CK(cudaEventRecord(t1, s));
  // ---- results to the host
  std::vector<double> hkr((size_t)9 * b), hkc((size_t)9 * b);
  ALD_CK(cudaMemcpyAsync(hkr.data(), kr.p, hkr.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  ALD_CK(cudaMemcpyAsync(hkc.data(), kc.p, hkc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  double d2h = 2.0 * hkr.size() * sizeof(double);
  std::vector<double> hq;
  if (Qo || QNo || QUo) {
    hq.resize((size_t)3 * nibz * b);
    ALD_CK(cudaMemcpyAsync(hq.data(), Q.p, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    d2h += hq.size() * sizeof(double);
  }
  if (xo) {
    ALD_CK(cudaMemcpyAsync(xo, x.p, N * sizeof(double), cudaMemcpyDeviceToHost, s));
    d2h += N * sizeof(double);
  }
  ALD_CK(cudaStreamSynchronize(s));
  r = check_err_flags(c);
  if (r) return r;
  tm.collect(res->stage_ms);
  float total = 0;
  cudaEventElapsedTime(&total, t0, t1);
  res->stage_ms[9] = total;
  for (int i = 0; i < 9; ++i) res->launches[9] += res->launches[i];
  for (int e = 0; e < 9; ++e) {
    double sr = 0, sc = 0;
    for (int l = 0; l < b; ++l) {
      sr += hkr[l + (size_t)b * e];
      sc += hkc[l + (size_t)b * e];
    }
    res->kappa_rta[e] = sr;
    res->kappa_cg[e] = sc;
  }
  if (kappa_rta_modes) std::memcpy(kappa_rta_modes, hkr.data(), hkr.size() * sizeof(double));
  if (kappa_cg_modes) std::memcpy(kappa_cg_modes, hkc.data(), hkc.size() * sizeof(double));
  for (int i = 0; i < nibz; ++i)
    for (int l = 0; l < b; ++l) {
      if (Qo) Qo[i + (size_t)nibz * l] = hq[(size_t)i * b + l];
      if (QNo) QNo[i + (size_t)nibz * l] = hq[(size_t)nibz * b + (size_t)i * b + l];
      if (QUo) QUo[i + (size_t)nibz * l] = hq[(size_t)2 * nibz * b + (size_t)i * b + l];
    }
  res->cg_iters = iters;
  res->status_cg = rc;
  res->cg_err = cg_err;
  res->triplet_bands = (double)nibz * nkc * (double)b * b * b;
  res->d2h_bytes = d2h;
  return ALD_OK;
}

extern "C" int ald_kappa_pipeline(ald_ctx* c, double tempk, ald_kappa_result* res, double* Qo, double* QNo,
                                  double* QUo, double* kappa_rta_modes, double* kappa_cg_modes, double* xo) {
  return run_pipeline(c, tempk, res, Qo, QNo, QUo, kappa_rta_modes, kappa_cg_modes, xo, nullptr);
}

// the pipeline workspaces of a context (their blocks go to the library's
// device-memory cache, where the next structure of the same sizes finds them)
static void release_pipeline_workspaces(ald_ctx* c) {
  c->v3c_epoch = 0;  // the kept |V3|^2 goes with its buffer
  for (DevBuf<double>* b : {&c->w_R1, &c->w_R2, &c->w_v3, &c->w_cm, &c->w_R1p, &c->w_R2p, &c->w_heev, &c->w_rmax})
    b->free();
  c->w_h.free();
  c->w_h64.free();
  c->w_v3fix.free();
  c->w_pairs.free();
  c->w_v3work.free();
  c->v3work_tc_b = 0;
  c->w_btiles.free();
  c->w_scratch.free();
}

// An upper estimate of the device bytes one pipeline call on c allocates
// beyond the context's tables: R1/R2, |V3|^2 of one chunk, the collision
// matrix, the fixed-point sums of the deterministic delta, and for large
// cells the V3 GEMM workspace (2 GiB at most) and the Householder
// eigensolver's slots.  The batched entry point admits structures by it.
static size_t pipeline_bytes_estimate(const ald_ctx* c) {
  const size_t nibz = c->T.nibz, nkc = c->T.nkc, b = c->geo.b;
  const size_t rsz = nibz * nkc * b * b * sizeof(double);
  const size_t per_row = nkc * b * b * b * sizeof(double);
  const size_t budget = c->opt.chunk_bytes ? c->opt.chunk_bytes : (size_t)512 << 20;
  const size_t k = std::max<size_t>(1, std::min<size_t>(budget / per_row, nibz));
  const size_t N = 3 * b * nibz;
  size_t s = 2 * rsz + k * per_row + N * N * sizeof(double);
  s += 2 * (k * nkc * b * b) * sizeof(unsigned long long);  // deterministic delta
  if (b > 12) s += c->tune_gemm_bytes ? c->tune_gemm_bytes : (size_t)2 << 30;
  if (b > 64) s += heev_work_doubles((int)b, heev_slots((int)nkc * 7)) * sizeof(double);
  return s + ((size_t)256 << 20);
}

extern "C" int ald_release_workspaces(ald_ctx* c) {
  if (!c) return fail(ALD_ERR_ARG, "null context");
  ALD_CK(cudaSetDevice(c->device));
  release_pipeline_workspaces(c);
  return ALD_OK;
}

extern "C" int ald_kappa_batched(int n, ald_ctx* const* ctx, const double* tempk, ald_kappa_result* res,
                                 int* status) {
  if (n <= 0 || !ctx || !tempk || !res) return fail(ALD_ERR_ARG, "bad argument");
  for (int i = 0; i < n; ++i) {
    if (!ctx[i]) return fail(ALD_ERR_ARG, "null context");
    for (int j = 0; j < i; ++j)
      if (ctx[j] == ctx[i]) return fail(ALD_ERR_ARG, "a context appears twice in the batch");
  }
  // A pool of host threads, each issuing one structure at a time on that
  // structure's own stream, so that structures overlap on the device; the
  // largest (nibz nkc b^3) go first.  Admission is memory-aware: a structure
  // starts only while the pipeline workspaces of the structures in flight on
  // its device, plus its own (pipeline_bytes_estimate), stay within 85 % of
  // the device memory free when the batch began; one structure always runs.
  // When the batch is larger than what runs at once, a structure's pipeline
  // workspaces return to the library's device-memory cache after its run.
  const int pool = std::min(n, 8);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  auto work = [&](int i) {
    const ald_ctx* c = ctx[i];
    return (double)c->T.nibz * c->T.nkc * (double)c->geo.b * c->geo.b * c->geo.b;
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  std::vector<size_t> est(n);
  std::map<int, size_t> budget, inflight;
  size_t total_est = 0;
  for (int i = 0; i < n; ++i) {
    est[i] = pipeline_bytes_estimate(ctx[i]);
    total_est += est[i];
    const int dev = ctx[i]->device;
    if (!budget.count(dev)) {
      size_t fr = 0, tot = 0;
      cudaSetDevice(dev);
      budget[dev] = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? fr / 100 * 85 : (size_t)-1;
      inflight[dev] = 0;
    }
  }
  bool release_after = n > pool;
  for (auto& kv : budget)
    if (total_est > kv.second) release_after = n > 1;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<int> st(n, ALD_OK);
  std::vector<std::string> msg(n);
  int next = 0;
  std::vector<std::thread> th;
  th.reserve(pool);
  for (int t = 0; t < pool; ++t)
    th.emplace_back([&] {
      for (;;) {
        int i;
        {
          std::unique_lock<std::mutex> lk(mu);
          if (next >= n) break;
          const int dev = ctx[order[next]]->device;
          // the next structure in order, once it fits (or nothing else runs)
          cv.wait(lk, [&] {
            return next >= n || inflight[ctx[order[next]]->device] == 0 ||
                   inflight[ctx[order[next]]->device] + est[order[next]] <= budget[ctx[order[next]]->device];
          });
          (void)dev;
          if (next >= n) break;
          i = order[next++];
          inflight[ctx[i]->device] += est[i];
        }
        st[i] = run_pipeline(ctx[i], tempk[i], &res[i], nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                             nullptr);
        if (st[i] != ALD_OK) msg[i] = ald_last_error();
        if (release_after) {
          cudaSetDevice(ctx[i]->device);
          release_pipeline_workspaces(ctx[i]);
        }
        {
          std::lock_guard<std::mutex> lk(mu);
          inflight[ctx[i]->device] -= est[i];
        }
        cv.notify_all();
      }
    });
  for (auto& t : th) t.join();
  int first = ALD_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = st[i];
    if (first == ALD_OK && st[i] != ALD_OK) {
      first = st[i];
      fail(first, "structure " + std::to_string(i) + ": " + msg[i]);
    }
  }
  return first;
}

extern "C" int ald_shard_rows(const ald_ctx* c, int rank, int nranks, int ksubset[2]) {
  if (!c || !ksubset || nranks < 1 || rank < 0 || rank >= nranks) return fail(ALD_ERR_ARG, "bad rank or rank count");
  int rb, re;
  shard_range(c->T.nibz, rank, nranks, rb, re);
  ksubset[0] = rb + 1;
  ksubset[1] = re;
  return ALD_OK;
}

extern "C" int ald_kappa_pipeline_sharded(ald_ctx* c, double tempk, int rank, int nranks, ald_allgather_fn gather,
                                          void* user, ald_kappa_result* res, double* Qo, double* QNo, double* QUo,
                                          double* kappa_rta_modes, double* kappa_cg_modes, double* xo) {
  ShardSpec sh{rank, nranks, gather, nullptr, user};
  return run_pipeline(c, tempk, res, Qo, QNo, QUo, kappa_rta_modes, kappa_cg_modes, xo, nullptr, &sh);
}

extern "C" int ald_kappa_pipeline_sharded_dev(ald_ctx* c, double tempk, int rank, int nranks,
                                              ald_allgather_dev_fn gather, void* user, ald_kappa_result* res,
                                              double* Qo, double* QNo, double* QUo, double* kappa_rta_modes,
                                              double* kappa_cg_modes, double* xo) {
  if (!gather) return fail(ALD_ERR_ARG, "sharded pipeline: no exchange function");
  ShardSpec sh{rank, nranks, nullptr, gather, user};
  return run_pipeline(c, tempk, res, Qo, QNo, QUo, kappa_rta_modes, kappa_cg_modes, xo, nullptr, &sh);
}

extern "C" int ald_kappa_iterative(ald_ctx* c, double tempk, int max_iter, double update_mix, ald_kappa_result* res,
                                   double* Qo, double* kappa_rta_modes, double* kappa_iter_modes, double* FFF) {
  if (max_iter < 0 || !(update_mix > 0)) return fail(ALD_ERR_ARG, "max_iter < 0 or update_mix <= 0");
  IterSpec it{max_iter, update_mix, FFF};
  return run_pipeline(c, tempk, res, Qo, nullptr, nullptr, kappa_rta_modes, kappa_iter_modes, nullptr, &it);
}
