// |V3|^2 for 3-band cells with the phase-class sums on the tensor cores:
// the ALD_MIXED path (tcgen05, kind::f16, FP32 accumulation in TMEM).
//
// The class form of V3 (ald_v3_pair.cu) spends most of its work, for one
// atom per cell, in
//   A[q2][l1 be ga] = sum_c P_c(q2) H[c][be ga][l1],
// a complex GEMM of M = q2, K = ncls phase classes (79 for the LJ argon
// crystal), N = 27.  Here one CTA takes one IBZ row and 128 consecutive q2
// (one TMEM lane each) and runs it in real form
//   [Ar | Ai] = [Pr | Pi] x [[Hr, Hi], [-Hi, Hr]],  K' = 2 ncls (to 16), N' = 54 (to 64).
// Every FP32 operand x is split into FP16 hi + lo (hi = fp16(x), lo =
// fp16(x - hi)); the product is hi.hi + hi.lo + lo.hi, three MMAs per K step
// into one FP32 accumulator (relative error about 2^-22 of |P||H|).  Each H
// column pair is scaled by a power of two so that FP16 keeps its range.
// Then every thread (= one q2) reads its 64 accumulator columns from TMEM
// and does the two eigenvector mode products with e(q2), e(q3) in FP32, the
// (const33/den)^2 scaling and |V|^2 in FP64, and the slice-major store.
//
// Operand layout in shared memory: the UMMA canonical K-major layout
// without swizzle -- 8x8 FP16 core matrices of 8 rows x 16 bytes, rows
// contiguous inside a core matrix (SBO = 128 bytes between 8-row groups) and
// the two 8-element K halves of one MMA ROWS*16 bytes apart (LBO).
//
// The phase tiles (A) depend on q2 only and are built once per context; the
// B operands (H of one row, split and scaled) once per row by
// v3_btile_kernel.  Both reach shared memory by bulk copies; B streams
// through two buffers so the next row's copy overlaps this row's MMAs.
//
// Every wait of the CTA (the bulk-copy and MMA-completion mbarriers) is
// bounded: on timeout the CTA sets bit 16 of the error flag, waits (bounded)
// for its copies and MMAs in flight, frees its TMEM and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kTM = 128;      // q2 per CTA = TMEM lanes = threads
constexpr int kNC = 27;       // complex outputs (l1, be, ga) for 3 bands
constexpr int kNP = 64;       // real outputs padded to a valid N
constexpr int kMaxKp = 208;   // K' bound (ncls <= 104): A + 2 B buffers fit 227 KB
constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}
// mesh index of q3 = -q1-q2 with the wrap done by compares (|m| < nc)
__device__ __forceinline__ int idx_q3_fast(const Geometry& g, const int* m1, const int* m2) {
  int m3[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int n = g.nc[a];
    int v = -m1[a] - m2[a] + (g.shifted ? n / 2 : 0);
    v += v < 0 ? n : 0;
    v += v < 0 ? n : 0;
    v -= v >= n ? n : 0;
    m3[a] = v;
  }
  return m3[2] + g.nc[2] * (m3[1] + g.nc[1] * m3[0]);
}
__device__ __forceinline__ int phase_index(const int* pc, const int* m, int L, int L32) {
  if (L32) {  // the sum fits in 32 bits: a 32-bit remainder
    const unsigned t = (unsigned)(m[0] * pc[0] + m[1] * pc[1] + m[2] * pc[2] + pc[3]);
    return (int)(t % (unsigned)L);
  }
  long long t = (long long)m[0] * pc[0] + (long long)m[1] * pc[1] + (long long)m[2] * pc[2] + pc[3];
  return (int)(t % L);
}

// canonical K-major, no swizzle: element (r, k) of a ROWS x K' operand, in halves
__device__ __forceinline__ int kmaj(int r, int k, int rows) { return ((k >> 3) * rows + r) * 8 + (k & 7); }

__device__ __forceinline__ void split_store(__half* hi, __half* lo, int i, float x) {
  const __half h = __float2half_rn(x);
  hi[i] = h;
  lo[i] = __float2half_rn(x - __half2float(h));
}

// UMMA shared-memory descriptor: start, LBO, SBO in 16-byte units, version 1
// (Blackwell), base offset 0, legacy LBO mode, layout SWIZZLE_NONE
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16: D F32, A and B F16, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;  // disable-output-lane mask: every lane written
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// The A operand (phases P_c(q2), split FP16 hi/lo in the canonical layout)
// depends on q2 and the class only, not on the IBZ row: built once per
// context for every 128-q2 tile, [tile][hi|lo][kmaj].
__global__ void v3_ptile_kernel(Geometry g, int ncls, int kp, const int* cls_pc, const double* roots_d,
                                __half* Pt) {
  const int tile = blockIdx.x, r = threadIdx.x;
  const int q2 = min(tile * kTM + r, g.nkc - 1);
  int m2[3];
  decompose(g, q2, m2);
  const double2* roots = reinterpret_cast<const double2*>(roots_d);
  __half* hi = Pt + (size_t)tile * 2 * kTM * kp;
  __half* lo = hi + (size_t)kTM * kp;
  for (int k = 0; k < kp; ++k) {
    float v = 0.f;
    if (k < 2 * ncls) {
      const int c = k < ncls ? k : k - ncls;
      const double2 p = roots[phase_index(cls_pc + 4 * c, m2, g.L, g.L32)];
      v = (float)(k < ncls ? p.x : p.y);
    }
    split_store(hi, lo, kmaj(r, k, kTM), v);
  }
}

// Per-launch scratch of the tensor-core V3, carved from one buffer:
//   bt     [row][hi|lo][kmaj]     B operands (2 kNP kp halves per row)
//   isc    [row][32]              inverse column scales (27 used)
//   rq     [row]                  int4 {q1, m1[0..2]}
//   rt     [row][4]               const33^2/8 / sqrt|l(q1)| per band (3 used)
//   tq     [q][3]                 1/sqrt|l(q)| of every mesh mode
//   evf    [q][9]                 e(q) as float2, [l][i]
struct TcScratch {
  __half* bt;
  float* isc;
  int4* rq;
  double* rt;
  double* tq;
  float2* evf;
};
__host__ __device__ inline size_t tc_align(size_t x) { return (x + 255) & ~(size_t)255; }
inline TcScratch tc_carve(void* base, int nrows, int kp, int nkc, size_t* total) {
  char* p = static_cast<char*>(base);
  size_t o = 0;
  TcScratch t;
  t.bt = reinterpret_cast<__half*>(p + o);
  o = tc_align(o + (size_t)nrows * 2 * kNP * kp * sizeof(__half));
  t.isc = reinterpret_cast<float*>(p + o);
  o = tc_align(o + (size_t)nrows * 32 * sizeof(float));
  t.rq = reinterpret_cast<int4*>(p + o);
  o = tc_align(o + (size_t)nrows * sizeof(int4));
  t.rt = reinterpret_cast<double*>(p + o);
  o = tc_align(o + (size_t)nrows * 4 * sizeof(double));
  t.tq = reinterpret_cast<double*>(p + o);
  o = tc_align(o + (size_t)nkc * 3 * sizeof(double));
  t.evf = reinterpret_cast<float2*>(p + o);
  o = tc_align(o + (size_t)nkc * 9 * sizeof(float2));
  if (total) *total = o;
  return t;
}

// per mesh mode: 1/sqrt|lambda| and the eigenvectors in FP32
__global__ void v3_tc_modes_kernel(V3Args a, TcScratch t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.geo.nkc) return;
  const double2* ev = reinterpret_cast<const double2*>(a.evec);
#pragma unroll
  for (int l = 0; l < 3; ++l) t.tq[(size_t)q * 3 + l] = 1.0 / sqrt(fabs(a.w2[(size_t)q * 3 + l]));
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const double2 x = ev[(size_t)q * 9 + i];
    t.evf[(size_t)q * 9 + i] = make_float2((float)x.x, (float)x.y);
  }
}

// The B operand of every IBZ row of the chunk (H in real form, split FP16,
// canonical layout), built once per row: [row][hi|lo][kmaj], and the
// inverses of the 27 column scales (powers of two with max |H| * scale in
// [0.5, 1)).
__global__ void v3_btile_kernel(V3Args a, int kp, TcScratch t) {
  __shared__ float s_scale[kNC];
  const int row = blockIdx.x, tid = threadIdx.x, ncls = a.ncls;
  __half* Bt = t.bt;
  float* inv_scales = t.isc;
  if (tid == 0) {
    const int q1 = a.mapinv[a.n1_first + row];
    int m1[3];
    decompose(a.geo, q1, m1);
    t.rq[row] = make_int4(q1, m1[0], m1[1], m1[2]);
    const double c33 = a.const33 * a.const33 / 8;
    for (int l = 0; l < 3; ++l) t.rt[(size_t)row * 4 + l] = c33 / sqrt(fabs(a.w2[(size_t)q1 * 3 + l]));
    t.rt[(size_t)row * 4 + 3] = 0.0;
  }
  const float2* H = static_cast<const float2*>(a.hbuf) + (size_t)row * ncls * 9 * 3;
  if (tid < kNC) {
    const int l1 = tid / 9, bg = tid % 9;
    float mx = 0.f;
    for (int c = 0; c < ncls; ++c) {
      const float2 h = H[((size_t)c * 9 + bg) * 3 + l1];
      mx = fmaxf(mx, fmaxf(fabsf(h.x), fabsf(h.y)));
    }
    int e = 0;
    if (mx > 0.f) frexpf(mx, &e);
    s_scale[tid] = ldexpf(1.f, -e);
    inv_scales[(size_t)row * 32 + tid] = ldexpf(1.f, e);
  }
  __syncthreads();
  __half* hi = Bt + (size_t)row * 2 * kNP * kp;
  __half* lo = hi + (size_t)kNP * kp;
  for (int i = tid; i < kNP * kp; i += blockDim.x) {
    const int n = i / kp, k = i % kp;
    float v = 0.f;
    const int col = n >> 1;
    if (col < kNC && k < 2 * ncls) {
      const int l1 = col / 9, bg = col % 9, c = k < ncls ? k : k - ncls;
      const float2 h = H[((size_t)c * 9 + bg) * 3 + l1];
      const float sc = s_scale[col];
      if ((n & 1) == 0) v = k < ncls ? h.x * sc : -h.y * sc;  // Ar = Pr Hr - Pi Hi
      else v = k < ncls ? h.y * sc : h.x * sc;                // Ai = Pr Hi + Pi Hr
    }
    split_store(hi, lo, kmaj(n, k, kNP), v);
  }
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < kWaitLimit; ++it)
    if (mbar_try(bar, parity)) return true;
  return false;
}

// bounded wait that also gives up once another warp has raised the CTA's
// failure flag
__device__ __forceinline__ bool mbar_wait_or_fail(uint32_t bar, uint32_t parity, const volatile int* fail) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63u) == 63u && *fail) return false;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(bar) : "memory");
  const char* p = static_cast<const char*>(src);
  for (uint32_t off = 0; off < bytes; off += 32768u) {
    const uint32_t n = bytes - off < 32768u ? bytes - off : 32768u;
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst + off),
                 "l"(p + off), "r"(n), "r"(bar)
                 : "memory");
  }
}

// NE epilogue warpgroups = NE TMEM accumulators of 64 columns, + one producer warp
template <int NE>
struct TcShape {
  static constexpr int threads = 128 * NE + 32;
  static constexpr int tmem_cols = NE <= 2 ? 128 : 256;  // a power of two >= 64 NE
};

// One CTA: one 128-q2 tile and up to `rpc` IBZ rows, warp-specialised.
// * Producer warp (one lane): copies the phase tile once and the B tiles of
//   the rows through two buffers, issues the 3 (kp/16) MMAs of a row into
//   accumulator (row % NE) once that accumulator has been drained, commits.
// * Epilogue warpgroup w takes the rows with (row - r0) % NE == w: thread =
//   TMEM lane = q2; it loads its 64 accumulator columns, releases the
//   accumulator, then does the mode products with e(q2), e(q3), the scaling
//   and the stores, while the producer already runs the next rows' MMAs.
template <int NE>
__global__ void __launch_bounds__(TcShape<NE>::threads, 1)
    v3_tc3_kernel(V3Args a, int kp, const __half* Pt, TcScratch ts, int rpc) {
  constexpr int kTmemAlloc = TcShape<NE>::tmem_cols;
  const __half* Bt = ts.bt;
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar_a, s_bar_b[2], s_full[NE], s_empty[NE];
  __shared__ volatile int s_fail;
  const Geometry& g = a.geo;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, tile = blockIdx.x;
  const int r0 = blockIdx.y * rpc, n = min(rpc, a.nrows - r0);
  const uint32_t a_sh = (uint32_t)__cvta_generic_to_shared(smraw);
  const uint32_t b_sh = a_sh + (uint32_t)(2 * kTM * kp * sizeof(__half));
  const uint32_t bbytes = (uint32_t)(2 * kNP * kp * sizeof(__half));
  const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(&s_bar_a);
  const uint32_t bar_b0 = (uint32_t)__cvta_generic_to_shared(&s_bar_b[0]);
  const uint32_t bar_b1 = (uint32_t)__cvta_generic_to_shared(&s_bar_b[1]);
  // accumulator k's barriers at full0 + 8k, empty0 + 8k
  const uint32_t full0 = (uint32_t)__cvta_generic_to_shared(&s_full[0]);
  const uint32_t empty0 = (uint32_t)__cvta_generic_to_shared(&s_empty[0]);

  if (warp == 0) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_tmem);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTmemAlloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_b0));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_b1));
    for (int k = 0; k < NE; ++k) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8 * k));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty0 + 8 * k), "r"(kTM));
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  if (warp == 4 * NE) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int bq0 = -1, bq1 = -1, pend_acc = -1, pend_par = 0;  // copies and MMAs in flight
      bulk_g2s(a_sh, Pt + (size_t)tile * 2 * kTM * kp, (uint32_t)(2 * kTM * kp * sizeof(__half)), bar_a);
      bulk_g2s(b_sh, Bt + (size_t)r0 * 2 * kNP * kp, bbytes, bar_b0);
      bq0 = 0;
      if (n > 1) {
        bulk_g2s(b_sh + bbytes, Bt + (size_t)(r0 + 1) * 2 * kNP * kp, bbytes, bar_b1);
        bq1 = 0;
      }
      bool ok = mbar_wait_or_fail(bar_a, 0, &s_fail);
      const uint32_t idesc = instr_desc(kTM, kNP);
      const uint32_t aH = a_sh, aL = a_sh + (uint32_t)(kTM * kp * sizeof(__half));
      for (int it = 0; ok && it < n; ++it) {
        const int buf = it & 1, acc = it % NE, use = it / NE;
        ok = mbar_wait_or_fail(buf ? bar_b1 : bar_b0, (uint32_t)((it >> 1) & 1), &s_fail);
        if (!ok) break;
        if (buf) bq1 = -1;
        else bq0 = -1;
        if (use >= 1) {  // accumulator acc drained by the epilogue of row it - NE
          ok = mbar_wait_or_fail(empty0 + 8 * acc, (uint32_t)((use - 1) & 1), &s_fail);
          if (!ok) break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t bH = b_sh + (uint32_t)buf * bbytes, bL = bH + (uint32_t)(kNP * kp * sizeof(__half));
        const uint32_t dt = tmem + (uint32_t)(acc * kNP);
        for (int st = 0; st < kp / 16; ++st) {
          // K step st covers K chunks 2st, 2st+1: ROWS*16 bytes per chunk
          const uint32_t oa = (uint32_t)(2 * st * kTM * 16), ob = (uint32_t)(2 * st * kNP * 16);
          const uint64_t dAh = smem_desc(aH + oa, kTM * 16, 128), dAl = smem_desc(aL + oa, kTM * 16, 128);
          const uint64_t dBh = smem_desc(bH + ob, kNP * 16, 128), dBl = smem_desc(bL + ob, kNP * 16, 128);
          mma_f16(dt, dAh, dBh, idesc, st > 0 ? 1u : 0u);
          mma_f16(dt, dAh, dBl, idesc, 1u);
          mma_f16(dt, dAl, dBh, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         full0 + 8 * acc)
                     : "memory");
        pend_acc = acc;
        pend_par = use & 1;
        // B buffer of row it - 1 is free once that row's MMAs completed:
        // refill it with row it + 1
        if (it >= 1 && it + 1 < n) {
          const int pb = buf ^ 1;
          ok = mbar_wait_or_fail(full0 + 8 * ((it - 1) % NE), (uint32_t)(((it - 1) / NE) & 1), &s_fail);
          if (!ok) break;
          bulk_g2s(b_sh + (uint32_t)pb * bbytes, Bt + (size_t)(r0 + it + 1) * 2 * kNP * kp, bbytes,
                   pb ? bar_b1 : bar_b0);
          if (pb) bq1 = ((it + 1) >> 1) & 1;
          else bq0 = ((it + 1) >> 1) & 1;
        }
      }
      if (!ok) s_fail = 1;
      // wait (bounded) for whatever is still in flight before the TMEM and
      // the CTA go; on the normal path these have completed already
      mbar_wait_bounded(bar_a, 0);
      if (bq0 >= 0) mbar_wait_bounded(bar_b0, (uint32_t)bq0);
      if (bq1 >= 0) mbar_wait_bounded(bar_b1, (uint32_t)bq1);
      if (pend_acc >= 0) mbar_wait_bounded(full0 + 8 * pend_acc, (uint32_t)pend_par);
    }
  } else {
    // ---------------- epilogue ----------------
    const int wg = warp >> 2, lt = tid & (kTM - 1);
    const int qg = tile * kTM + lt;
    const int q2 = min(qg, g.nkc - 1);
    int m2[3];
    decompose(g, q2, m2);
    float2 e2[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) e2[i] = ts.evf[(size_t)q2 * 9 + i];  // e[q][l][i]
    double t2[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) t2[l] = ts.tq[(size_t)q2 * 3 + l];
    const size_t nk = g.nkc;
    const uint32_t full = full0 + 8 * wg, empty = empty0 + 8 * wg;
    const uint32_t taddr = tmem + (uint32_t)(wg * kNP) + ((uint32_t)(32 * (warp & 3)) << 16);
    for (int it = wg; it < n; it += NE) {
      const int row = r0 + it;
      // row-dependent data before the wait: q3, e(q3), the mode factors
      const int4 ri = ts.rq[row];
      const int m1[3] = {ri.y, ri.z, ri.w};
      const int q3 = idx_q3_fast(g, m1, m2);
      float2 e3[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) e3[i] = ts.evf[(size_t)q3 * 9 + i];
      double t23[9], t1[3];
#pragma unroll
      for (int l = 0; l < 3; ++l) t1[l] = ts.rt[(size_t)row * 4 + l];
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        const double t3 = ts.tq[(size_t)q3 * 3 + l];
#pragma unroll
        for (int l2 = 0; l2 < 3; ++l2) t23[l2 * 3 + l] = t2[l2] * t3;
      }
      const float* isc = ts.isc + (size_t)row * 32;
      const bool w = mbar_wait_or_fail(full, (uint32_t)((it / NE) & 1), &s_fail);
      if (!__all_sync(0xffffffffu, w)) {  // warp-uniform exit
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t d[kNP];
#pragma unroll
      for (int c8 = 0; c8 < kNP / 8; ++c8)
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(d[8 * c8 + 0]), "=r"(d[8 * c8 + 1]), "=r"(d[8 * c8 + 2]), "=r"(d[8 * c8 + 3]), "=r"(d[8 * c8 + 4]),
              "=r"(d[8 * c8 + 5]), "=r"(d[8 * c8 + 6]), "=r"(d[8 * c8 + 7])
            : "r"(taddr + 8 * c8));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(empty) : "memory");
      if (qg < g.nkc) {
#pragma unroll
        for (int l1 = 0; l1 < 3; ++l1) {
          // A[l1][b][c] and T[l2][c] = sum_b A[l1][b][c] e2[b][l2]   (e2[b][l2] at e2[l2*3 + b])
          float2 A[9];
#pragma unroll
          for (int j = 0; j < 9; ++j) {
            const float inv = __ldg(isc + l1 * 9 + j);
            A[j] = make_float2(__uint_as_float(d[2 * (l1 * 9 + j)]) * inv,
                               __uint_as_float(d[2 * (l1 * 9 + j) + 1]) * inv);
          }
          float2 T[3][3];
#pragma unroll
          for (int l2 = 0; l2 < 3; ++l2)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              float2 sm = make_float2(0.f, 0.f);
#pragma unroll
              for (int bb = 0; bb < 3; ++bb) {
                const float2 x = A[bb * 3 + c], y = e2[l2 * 3 + bb];
                sm.x = fmaf(x.x, y.x, fmaf(-x.y, y.y, sm.x));
                sm.y = fmaf(x.x, y.y, fmaf(x.y, y.x, sm.y));
              }
              T[l2][c] = sm;
            }
#pragma unroll
          for (int l2 = 0; l2 < 3; ++l2)
#pragma unroll
            for (int l3 = 0; l3 < 3; ++l3) {
              float2 sm = make_float2(0.f, 0.f);
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                const float2 x = T[l2][c], y = e3[l3 * 3 + c];
                sm.x = fmaf(x.x, y.x, fmaf(-x.y, y.y, sm.x));
                sm.y = fmaf(x.x, y.y, fmaf(x.y, y.x, sm.y));
              }
              const double sc = t1[l1] * t23[l2 * 3 + l3];
              double v = 0.0;
              if (sc < 1.0 / 0.0) v = (double)fmaf(sm.x, sm.x, sm.y * sm.y) * sc;
              else atomicOr(a.err, 2);  // matrix_elt_simplified: den = 0
              const size_t o = a.v3_layout == 1 ? ((size_t)row * 27 + l2 * 9 + l3 * 3 + l1) * nk + qg
                                                 : ((size_t)row * nk + qg) * 27 + l1 * 9 + l2 * 3 + l3;
              if (a.v3sq_f32) a.v3sq_f32[o] = (float)v;  // the mixed pipeline's FP32 |V3|^2
              else a.v3sq[o] = v;
            }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (tid == 0 && s_fail) atomicOr(a.err, 16);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemAlloc));
}

}  // namespace

bool v3_tc_supported(int b, int ncls) { return b == 3 && ncls >= 1 && 2 * ncls <= kMaxKp; }

size_t v3_tc_ptile_bytes(int nkc, int ncls) {
  const int kp = (2 * ncls + 15) / 16 * 16;
  return (size_t)((nkc + kTM - 1) / kTM) * 2 * kTM * kp * sizeof(__half);
}

cudaError_t launch_v3_tc_ptiles(const V3Args& a, void* ptiles, cudaStream_t s) {
  if (!v3_tc_supported(a.geo.b, a.ncls)) return cudaErrorInvalidValue;
  const int kp = (2 * a.ncls + 15) / 16 * 16;
  v3_ptile_kernel<<<(a.geo.nkc + kTM - 1) / kTM, kTM, 0, s>>>(a.geo, a.ncls, kp, a.cls_pc, a.roots,
                                                              static_cast<__half*>(ptiles));
  return cudaGetLastError();
}

size_t v3_tc_btile_bytes(int nrows, int ncls, int nkc) {
  const int kp = (2 * ncls + 15) / 16 * 16;
  size_t total = 0;
  tc_carve(nullptr, nrows, kp, nkc, &total);
  return total;
}

cudaError_t launch_v3_tc(const V3Args& a, const void* ptiles, void* btiles, cudaStream_t s, int rows_per_cta,
                         int epilogue_wg) {
  if (!v3_tc_supported(a.geo.b, a.ncls)) return cudaErrorInvalidValue;
  const int kp = (2 * a.ncls + 15) / 16 * 16;
  const TcScratch ts = tc_carve(btiles, a.nrows, kp, a.geo.nkc, nullptr);
  v3_tc_modes_kernel<<<(a.geo.nkc + 127) / 128, 128, 0, s>>>(a, ts);
  v3_btile_kernel<<<a.nrows, 256, 0, s>>>(a, kp, ts);
  const size_t smem = (size_t)(2 * kTM + 4 * kNP) * kp * sizeof(__half);
  // epilogue warpgroups: 2 unless the caller (the autotuner) or ALD_V3_TC_WG=3 selects three
  static const int ne_env = [] {
    const char* v = getenv("ALD_V3_TC_WG");
    return v && atoi(v) == 3 ? 3 : 2;
  }();
  const int ne = epilogue_wg == 2 || epilogue_wg == 3 ? epilogue_wg : ne_env;
  cudaError_t e = raise_smem_limit(ne == 3 ? (const void*)v3_tc3_kernel<3> : (const void*)v3_tc3_kernel<2>, smem);
  if (e != cudaSuccess) return e;
  const int ntiles = (a.geo.nkc + kTM - 1) / kTM;
  // rows per CTA: reuse the phase tile over several rows while the grid still fills the GPU twice
  int rpc = 16;
  while (rpc > 1 && (long)ntiles * ((a.nrows + rpc - 1) / rpc) < 2 * 148) rpc /= 2;
  if (rows_per_cta >= 1 && rows_per_cta <= 16) rpc = rows_per_cta;
  dim3 grid(ntiles, (a.nrows + rpc - 1) / rpc);
  if (ne == 3)
    v3_tc3_kernel<3><<<grid, TcShape<3>::threads, smem, s>>>(a, kp, static_cast<const __half*>(ptiles), ts, rpc);
  else
    v3_tc3_kernel<2><<<grid, TcShape<2>::threads, smem, s>>>(a, kp, static_cast<const __half*>(ptiles), ts, rpc);
  return cudaGetLastError();
}

}  // namespace ald
