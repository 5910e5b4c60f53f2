// |V3|^2 for cells of more than 6 bands, mixed precision: the two
// eigenvector mode products of every (q1, q2) pair as split-FP16 tcgen05
// GEMMs with FP32 accumulation in TMEM (the ALD_MIXED path).
//
// Replaces calculate_w3_ibz_split_sq + matrix_elt_simplified
// (THERMACOND/sub.f90:1050-1233, 5888-6011) for large cells.  The FP64 form
// (ald_v3_dense.cu) computes per pair
//   T1[jb][l1][kc] = sum_{c in group (j0,k0)} P_c(q2) H[c][be ga][l1]
//   T2 = T1 x e(q2) over jb,   V = T2 x e(q3) over kc,   |V|^2 (const33/den)^2.
// Here both GEMMs run on the tensor cores in real block form
//   [Cr | Ci] = [Ar | Ai] x [[Br, Bi], [-Bi, Br]]
// (M = b^2 rows, K' = 2 Kh, N' = 2 Nh with Kh, Nh = b rounded up to 16).
// Every operand x is scaled by a power of two and split into FP16 hi + lo
// (hi = fp16(x), lo = fp16(x - hi)); each K step issues hi.hi + hi.lo +
// lo.hi (relative error about 2^-22 of |A||B|).  Scales: the eigenvector
// blocks by 2^13 (|e| <= 1); T1 by 2^(13 - e1) where 2^e1 bounds
// sum_c |H| of the row; T2 by a further 2^-ceil(log2 sqrt b) (Cauchy-Schwarz:
// |T2| <= sqrt(b) max|T1| for unit eigenvectors).  The scaled operands stay
// below 2^14, inside FP16's range, and the scales cancel exactly.
//
// Operands sit in global memory in the UMMA canonical K-major layout without
// swizzle, cut into chunks of 32 K' so that each chunk is one contiguous
// block: per pair A is [M tile][chunk][hi|lo][128 x 32] (16 KB per block),
// per mesh point B is [chunk][hi|lo][N' x 32].  One CTA computes one
// 128 x N' tile of one pair: a producer warp streams (A, B) chunks through a
// ring of shared-memory stages with bulk copies, one thread issues the MMAs
// (N = the CTA's columns, one MMA into the Re and one into the Im accumulator per K
// step and split term), and four epilogue
// warps read the accumulator: GEMM 1 writes T2, scaled and split, as GEMM 2's
// A operand; GEMM 2 forms |V|^2 in FP64 and stores the chunk's layout.
//
// Every wait is bounded: on timeout the CTA sets bit 16 of the error flag,
// waits (bounded) for its copies and MMAs in flight, frees its TMEM and
// returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kTM = 128;   // rows per tile = TMEM lanes
constexpr int kBK = 32;    // K' per chunk
constexpr int kEpWarps = 4;
constexpr int kThreads = 64 + 32 * kEpWarps;  // producer, MMA, epilogue warps
constexpr unsigned kWaitLimit = 1u << 24;
constexpr int kSplitE = 13;  // operands scaled below 2^14

// Output columns: Nh = b rounded up to 16 (to 32 above 128 bands), in the
// real block form N' = 2 Nh (Re | Im).  Each CTA takes a contiguous range of
// `ncol` = Nh / nsplit columns of both parts (nsplit = 2 above 128 bands), as
// two accumulators of ncol TMEM columns (Re, Im), so that the TMEM (at most
// 256 columns) and the shared-memory stages of two CTAs fit one SM: one
// CTA's epilogue then overlaps the other's MMAs.
struct DenseTcShape {
  int b, kh, nh, kp, np, nchunk, mtiles, nsplit, ncol, tmem_cols, stages;
  size_t a_block_halves;  // one (M tile, chunk) block: hi + lo
  size_t a_pair_halves;   // one pair's A operand
  size_t b_chunk_halves;  // one chunk of B (global, all N' rows): hi + lo
  size_t bq_halves;       // one mesh point's B operand
  size_t b_stage_bytes;   // one chunk of a CTA's B rows in shared memory
  size_t stage_bytes, smem;
};

__host__ __device__ inline DenseTcShape dense_tc_shape(int b) {
  DenseTcShape s;
  s.b = b;
  s.kh = (b + 15) / 16 * 16;
  s.nsplit = b > 128 ? 2 : 1;
  s.nh = s.nsplit == 2 ? (b + 31) / 32 * 32 : (b + 15) / 16 * 16;
  s.ncol = s.nh / s.nsplit;
  s.kp = 2 * s.kh;
  s.np = 2 * s.nh;
  s.nchunk = s.kp / kBK;
  s.mtiles = (b * b + kTM - 1) / kTM;
  int tc = 32;
  while (tc < 2 * s.ncol) tc *= 2;
  s.tmem_cols = tc;
  s.a_block_halves = (size_t)2 * kTM * kBK;
  s.a_pair_halves = (size_t)s.mtiles * s.nchunk * s.a_block_halves;
  s.b_chunk_halves = (size_t)2 * s.np * kBK;
  s.bq_halves = (size_t)s.nchunk * s.b_chunk_halves;
  s.b_stage_bytes = (size_t)2 * (2 * s.ncol) * kBK * sizeof(__half);
  s.stage_bytes = s.a_block_halves * sizeof(__half) + s.b_stage_bytes;
  int st = (int)((size_t)104 * 1024 / s.stage_bytes);  // two CTAs per SM
  s.stages = st > 4 ? 4 : st;
  s.smem = (size_t)s.stages * s.stage_bytes;
  return s;
}

// the device buffers of one launch
struct DenseTc {
  __half* a1;    // [pair][A operand] of GEMM 1 (T1)
  __half* a2;    // [pair][A operand] of GEMM 2 (T2); padding stays zero
  __half* bq;    // [q][B operand]: e(q) in real block form
  int* rexp;     // per row of the chunk: e1 (sum_c |H| <= 2^e1)
  double* tq;    // [q][l]: 1/sqrt|lambda| of every mesh mode (+inf where lambda = 0)
  DenseTcShape sh;
};

__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}
__device__ __forceinline__ int wrapm(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}
__device__ __forceinline__ int idx_q3(const Geometry& g, const int* m1, const int* m2) {
  int m3[3];
  for (int a = 0; a < 3; ++a) m3[a] = wrapm(-m1[a] - m2[a] + (g.shifted ? g.nc[a] / 2 : 0), g.nc[a]);
  return m3[2] + g.nc[2] * (m3[1] + g.nc[1] * m3[0]);
}
__device__ __forceinline__ int phase_index(const int* pc, const int* m, int L, int L32) {
  if (L32) {
    const unsigned t = (unsigned)(m[0] * pc[0] + m[1] * pc[1] + m[2] * pc[2] + pc[3]);
    return (int)(t % (unsigned)L);
  }
  long long t = (long long)m[0] * pc[0] + (long long)m[1] * pc[1] + (long long)m[2] * pc[2] + pc[3];
  return (int)(t % L);
}
struct PairIdx {
  int row, q1, q2, q3;
};
__device__ __forceinline__ PairIdx pair_idx(const V3Args& a, long long pair) {
  PairIdx p;
  const int nkc = a.geo.nkc;
  p.row = (int)(pair / nkc);
  p.q2 = (int)(pair % nkc);
  p.q1 = a.mapinv[a.n1_first + p.row];
  int m1[3], m2[3];
  decompose(a.geo, p.q1, m1);
  decompose(a.geo, p.q2, m2);
  p.q3 = idx_q3(a.geo, m1, m2);
  return p;
}

// half offset of A element (m, k') inside one pair's operand
__device__ __forceinline__ size_t a_off(const DenseTcShape& s, int m, int k) {
  const int mt = m / kTM, r = m % kTM, ch = k / kBK, kl = k % kBK;
  return ((size_t)mt * s.nchunk + ch) * s.a_block_halves + (size_t)((kl >> 3) * kTM + r) * 8 + (kl & 7);
}
// half offset (hi part; lo follows at + 128*32) of the 8-element K group kg of row m
__device__ __forceinline__ size_t a_group_off(const DenseTcShape& s, int m, int kg) {
  return a_off(s, m, kg * 8);
}

__device__ __forceinline__ void split8(const float* x, __half* hi, __half* lo) {
  __align__(16) __half h[8], l[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    h[i] = __float2half_rn(x[i]);
    l[i] = __float2half_rn(x[i] - __half2float(h[i]));
  }
  *reinterpret_cast<uint4*>(hi) = *reinterpret_cast<const uint4*>(h);
  *reinterpret_cast<uint4*>(lo) = *reinterpret_cast<const uint4*>(l);
}

// ---------------------------------------------------------------- operands
// B operand of every mesh point: B'[k'][n'] of [[Br, Bi], [-Bi, Br]] with
// B[jb][n] = e(q)[n][jb], scaled by 2^13; thread = (n', K group of 8)
__global__ void v3tc_bq_kernel(V3Args a, DenseTc t) {
  const DenseTcShape& s = t.sh;
  const int q = blockIdx.x, b = a.geo.b;
  const double2* ev = reinterpret_cast<const double2*>(a.evec) + (size_t)q * b * b;
  __half* base = t.bq + (size_t)q * s.bq_halves;
  const int ng = s.kp / 8;
  const float sc = ldexpf(1.f, kSplitE);
  for (int e = threadIdx.x; e < s.np * ng; e += blockDim.x) {
    const int n = e % s.np, kg = e / s.np;
    const bool nr = n < s.nh;
    const int col = nr ? n : n - s.nh;
    float x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = kg * 8 + i;
      const bool kr = k < s.kh;
      const int jb = kr ? k : k - s.kh;
      float v = 0.f;
      if (jb < b && col < b) {
        const double2 z = ev[(size_t)col * b + jb];
        v = (float)(kr ? (nr ? z.x : z.y) : (nr ? -z.y : z.x)) * sc;
      }
      x[i] = v;
    }
    const int ch = kg * 8 / kBK, kl = kg * 8 % kBK;
    __half* hi = base + (size_t)ch * s.b_chunk_halves + (size_t)((kl >> 3) * s.np + n) * 8;
    split8(x, hi, hi + (size_t)s.np * kBK);
  }
}

// per row: e1 with sum_{c in group} |H[c][be ga][l1]| <= 2^e1 for every
// group, be ga and l1 (a bound of |T1|); atomicMax on the positive float bits
__global__ void v3tc_rowbound_kernel(V3Args a, unsigned* bound) {
  const int row = blockIdx.y, b = a.geo.b, nat0 = a.geo.nat0;
  const float2* H = static_cast<const float2*>(a.hbuf) + (size_t)row * a.ncls * 9 * b;
  const long long n = (long long)nat0 * nat0 * 9 * b;
  float mx = 0.f;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int l1 = (int)(e % b), bg = (int)((e / b) % 9), grp = (int)(e / (9LL * b));
    float sm = 0.f;
    for (int c = a.cls_grp_off[grp]; c < a.cls_grp_off[grp + 1]; ++c) {
      const float2 h = H[((size_t)c * 9 + bg) * b + l1];
      sm += fabsf(h.x) + fabsf(h.y);
    }
    mx = fmaxf(mx, sm);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0.f) atomicMax(bound + row, __float_as_uint(mx));
}

__global__ void v3tc_modes_kernel(V3Args a, double* tq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.geo.nkc * a.geo.b) return;
  const double w = fabs(a.w2[i]);
  tq[i] = w != 0.0 ? 1.0 / sqrt(w) : 1.0 / 0.0;
}

__global__ void v3tc_rowexp_kernel(int nrows, const unsigned* bound, int* rexp) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  int e = 0;
  const float mx = __uint_as_float(bound[r]);
  if (mx > 0.f) frexpf(mx, &e);  // mx < 2^e
  rexp[r] = e;
}

// A operand of GEMM 1 for the batch's pairs: rows m = l1 b + kc, K' = (Re |
// Im) jb; a thread per (row of the tile, K group of 8 jb)
__global__ void __launch_bounds__(256) v3tc_t1_kernel(V3Args a, DenseTc t, long long pair0, int table_ph) {
  extern __shared__ float2 s_ph[];  // P_c(q2) of every class
  const DenseTcShape& s = t.sh;
  const Geometry& g = a.geo;
  const int b = g.b, nat0 = g.nat0, mt = blockIdx.x, p = blockIdx.y;
  const PairIdx pi = pair_idx(a, pair0 + p);
  int m2[3];
  decompose(g, pi.q2, m2);
  const double2* roots = reinterpret_cast<const double2*>(a.roots);
  // the classes' phases in shared memory when they fit (table_ph), else
  // read from the roots table where used
  if (table_ph)
    for (int c = threadIdx.x; c < a.ncls; c += blockDim.x) {
      const double2 r = roots[phase_index(a.cls_pc + 4 * c, m2, g.L, g.L32)];
      s_ph[c] = make_float2((float)r.x, (float)r.y);
    }
  __syncthreads();
  const float2* H = static_cast<const float2*>(a.hbuf) + (size_t)pi.row * a.ncls * 9 * b;
  const float sc = ldexpf(1.f, kSplitE - t.rexp[pi.row]);
  __half* A = t.a1 + (size_t)p * s.a_pair_halves;
  const int ng = s.kh / 8;
  for (int e = threadIdx.x; e < kTM * ng; e += blockDim.x) {
    const int r = e % kTM, kg = e / kTM, m = mt * kTM + r;
    float xr[8], xi[8];
    const bool live = m < b * b;
    const int l1 = live ? m / b : 0, kc = live ? m % b : 0, k0 = kc / 3, ga = kc % 3;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int jb = kg * 8 + i;
      float2 acc = make_float2(0.f, 0.f);
      if (live && jb < b) {
        const int grp = (jb / 3) * nat0 + k0, be = jb % 3;
        for (int c = a.cls_grp_off[grp]; c < a.cls_grp_off[grp + 1]; ++c) {
          float2 ph;
          if (table_ph) {
            ph = s_ph[c];
          } else {
            const double2 r = roots[phase_index(a.cls_pc + 4 * c, m2, g.L, g.L32)];
            ph = make_float2((float)r.x, (float)r.y);
          }
          const float2 h = H[((size_t)c * 9 + be * 3 + ga) * b + l1];
          acc.x = fmaf(ph.x, h.x, fmaf(-ph.y, h.y, acc.x));
          acc.y = fmaf(ph.x, h.y, fmaf(ph.y, h.x, acc.y));
        }
      }
      xr[i] = acc.x * sc;
      xi[i] = acc.y * sc;
    }
    __half* hr = A + a_group_off(s, m, kg);
    split8(xr, hr, hr + (size_t)kTM * kBK);
    __half* him = A + a_group_off(s, m, s.kh / 8 + kg);
    split8(xi, him, him + (size_t)kTM * kBK);
  }
}

// ---------------------------------------------------------------- tcgen05
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// kind::f16 instruction descriptor: D F32, A and B F16, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
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
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < kWaitLimit; ++it)
    if (mbar_try(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ bool mbar_wait_or_fail(uint32_t bar, uint32_t parity, const volatile int* fail) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63u) == 63u && *fail) return false;
  }
  return false;
}
// the epilogue warps wait through the whole main loop: they back off between
// polls so that the producer and MMA threads keep the issue slots
__device__ __forceinline__ bool mbar_wait_idle(uint32_t bar, uint32_t parity, const volatile int* fail) {
  for (unsigned it = 0; it < kWaitLimit / 64; ++it) {
    if (mbar_try(bar, parity)) return true;
    if (*fail) return false;
    __nanosleep(256);
  }
  return false;
}
__device__ __forceinline__ void expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(bar) : "memory");
}
// bulk copy global -> shared in pieces of at most 32 KB, completing on bar
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  const char* p = static_cast<const char*>(src);
  for (uint32_t off = 0; off < bytes; off += 32768u) {
    const uint32_t n = bytes - off < 32768u ? bytes - off : 32768u;
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst + off),
                 "l"(p + off), "r"(n), "r"(bar)
                 : "memory");
  }
}

// 16 accumulator columns at ta and 16 at tb (this warp's 32 lanes), one wait
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float* va, float* vb) {
  uint32_t d[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%33];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]), "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]), "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
      : "r"(ta), "r"(tb)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(d[i]);
    vb[i] = __uint_as_float(d[16 + i]);
  }
}

// |V3|^2 element offset in the chunk's layout
__device__ __forceinline__ size_t v3_out_off(int layout, int row, int q2, int l1, int l2, int l3, int b, size_t nkc) {
  const size_t b3 = (size_t)b * b * b;
  if (layout == 2) return (((size_t)row * b + l2) * b + l3) * nkc * b + (size_t)q2 * b + l1;  // [row][l2][l3][q2][l1]
  if (layout == 1) return (size_t)row * nkc * b3 + (((size_t)l2 * b + l3) * b + l1) * nkc + q2;  // [row][l2][l3][l1][q2]
  return ((size_t)row * nkc + q2) * b3 + ((size_t)l1 * b + l2) * b + l3;  // [row][q2][l1][l2][l3]
}

// One CTA = one 128-row tile of one pair.  KIND 1: A = T1, B = e(q2),
// epilogue -> T2 as GEMM 2's A.  KIND 2: A = T2, B = e(q3), epilogue |V3|^2.
template <int KIND>
__global__ void __launch_bounds__(kThreads, 2) v3tc_gemm_kernel(V3Args a, DenseTc t, long long pair0) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_full[4], s_empty[4], s_accf;
  __shared__ volatile int s_fail;
  const DenseTcShape& s = t.sh;
  const Geometry& g = a.geo;
  const int b = g.b, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int mt = blockIdx.x / s.nsplit, split = blockIdx.x % s.nsplit, p = blockIdx.y, S = s.stages;
  const PairIdx pi = pair_idx(a, pair0 + p);
  const uint32_t sm0 = (uint32_t)__cvta_generic_to_shared(smraw);
  const uint32_t full0 = (uint32_t)__cvta_generic_to_shared(&s_full[0]);
  const uint32_t empty0 = (uint32_t)__cvta_generic_to_shared(&s_empty[0]);
  const uint32_t accf = (uint32_t)__cvta_generic_to_shared(&s_accf);
  if (warp == 1) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_tmem);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(s.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int k = 0; k < S; ++k) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8 * k));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0 + 8 * k));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(accf));
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t a_bytes = (uint32_t)(s.a_block_halves * sizeof(__half));
  const uint32_t b_bytes = (uint32_t)s.b_stage_bytes;
  const int nh0 = split * s.ncol;  // this CTA's first output column of each part
  const __half* Asrc = (KIND == 1 ? t.a1 : t.a2) + (size_t)p * s.a_pair_halves + (size_t)mt * s.nchunk * s.a_block_halves;
  const __half* Bsrc = t.bq + (size_t)(KIND == 1 ? pi.q2 : pi.q3) * s.bq_halves;

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      bool ok = true;
      int issued = 0;
      for (int c = 0; c < s.nchunk; ++c) {
        const int st = c % S;
        if (c >= S) {
          ok = mbar_wait_or_fail(empty0 + 8 * st, (uint32_t)((c / S - 1) & 1), &s_fail);
          if (!ok) break;
        }
        const uint32_t dst = sm0 + (uint32_t)(st * s.stage_bytes);
        expect_tx(full0 + 8 * st, a_bytes + b_bytes);
        bulk_copy(dst, Asrc + (size_t)c * s.a_block_halves, a_bytes, full0 + 8 * st);
        // B: per hi/lo and K group, this CTA's Re rows then its Im rows
        const uint32_t piece = (uint32_t)(s.ncol * 16);
        for (int hl = 0; hl < 2; ++hl)
          for (int kg = 0; kg < kBK / 8; ++kg) {
            const __half* src = Bsrc + (size_t)c * s.b_chunk_halves + (size_t)hl * s.np * kBK + (size_t)kg * s.np * 8;
            const uint32_t d = dst + a_bytes + (uint32_t)((hl * (kBK / 8) + kg) * 2) * piece;
            bulk_copy(d, src + (size_t)nh0 * 8, piece, full0 + 8 * st);
            bulk_copy(d + piece, src + (size_t)(s.nh + nh0) * 8, piece, full0 + 8 * st);
          }
        issued = c + 1;
      }
      if (!ok) s_fail = 1;
      // the last copies of each stage have landed before the CTA leaves
      for (int c = issued - S < 0 ? 0 : issued - S; c < issued; ++c)
        mbar_wait_bounded(full0 + 8 * (c % S), (uint32_t)((c / S) & 1));
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      bool ok = true;
      int done = 0;
      const uint32_t idesc = instr_desc(kTM, s.ncol);
      const uint32_t brows = (uint32_t)(2 * s.ncol);  // B rows of one K group in shared memory
      for (int c = 0; c < s.nchunk; ++c) {
        const int st = c % S;
        ok = mbar_wait_or_fail(full0 + 8 * st, (uint32_t)((c / S) & 1), &s_fail);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t aH = sm0 + (uint32_t)(st * s.stage_bytes), aL = aH + (uint32_t)(kTM * kBK * 2);
        const uint32_t bH = aH + a_bytes, bL = bH + (uint32_t)(brows * kBK * 2);
        for (int ks = 0; ks < kBK / 16; ++ks) {
          const uint32_t oa = (uint32_t)(2 * ks * kTM * 16), ob = (uint32_t)(2 * ks * brows * 16);
          const uint64_t dAh = smem_desc(aH + oa, kTM * 16, 128), dAl = smem_desc(aL + oa, kTM * 16, 128);
          for (int h = 0; h < 2; ++h) {  // accumulator 0: the Re columns, 1: the Im columns
            const uint32_t on = (uint32_t)(h * s.ncol * 16);
            const uint64_t dBh = smem_desc(bH + ob + on, brows * 16, 128);
            const uint64_t dBl = smem_desc(bL + ob + on, brows * 16, 128);
            const uint32_t dt = tmem + (uint32_t)(h * s.ncol);
            mma_f16(dt, dAh, dBh, idesc, (c > 0 || ks > 0) ? 1u : 0u);
            mma_f16(dt, dAh, dBl, idesc, 1u);
            mma_f16(dt, dAl, dBh, idesc, 1u);
          }
        }
        // the stage is free once these MMAs have read it
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         empty0 + 8 * st)
                     : "memory");
        done = c + 1;
      }
      if (ok) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(accf)
                     : "memory");
      } else {
        s_fail = 1;
        if (done > 0) mbar_wait_bounded(empty0 + 8 * ((done - 1) % S), (uint32_t)(((done - 1) / S) & 1));
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int quad = warp & 3, r = quad * 32 + lane, m = mt * kTM + r;
    const uint32_t taddr = tmem + ((uint32_t)(32 * quad) << 16);
    const bool w = mbar_wait_idle(accf, 0u, &s_fail);
    if (__all_sync(0xffffffffu, w)) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const bool live = m < b * b;
      const int e1 = t.rexp[pi.row];
      const int et = (int)ceilf(0.5f * log2f((float)b));  // 2^et >= sqrt(b)
      if (KIND == 1) {
        // T2 = acc / (2^(13-e1) 2^13), written scaled by 2^(13-e1-et)
        const float f = ldexpf(1.f, -et - kSplitE);
        const int l1 = live ? m / b : 0, kc = live ? m % b : 0;
        __half* A2 = t.a2 + (size_t)p * s.a_pair_halves;
        // b a multiple of 8: every aligned group of 8 rows is 8 consecutive kc
        // of one l1, i.e. one 16-byte K group of an A2 row.  The warp stages
        // its 32 x 8 values in shared memory (the stages are free once the
        // MMAs completed) and each lane stores one group of one column.
        float* scr = reinterpret_cast<float*>(smraw) + (warp - 2) * 32 * 9;
        const int grp = lane >> 3, gi = lane & 7;
        const int mg = mt * kTM + quad * 32 + 8 * grp;
        for (int cg = 0; cg < s.ncol / 16; ++cg) {
          float vr[16], vi[16];
          tmem_ld16x2(taddr + (uint32_t)(16 * cg), taddr + (uint32_t)(s.ncol + 16 * cg), vr, vi);
          if ((b & 7) == 0) {
#pragma unroll
            for (int q8 = 0; q8 < 2; ++q8)
#pragma unroll
              for (int part = 0; part < 2; ++part) {
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 8; ++j) scr[lane * 9 + j] = (part ? vi[8 * q8 + j] : vr[8 * q8 + j]) * f;
                __syncwarp();
                float x[8];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) x[jj] = scr[(8 * grp + jj) * 9 + gi];
                const int l2 = nh0 + 16 * cg + 8 * q8 + gi;
                if (mg < b * b && l2 < b) {
                  const int m2 = l2 * b + mg / b, kc0 = mg % b;
                  __half* dst = A2 + a_off(s, m2, (part ? s.kh : 0) + kc0);
                  split8(x, dst, dst + (size_t)kTM * kBK);
                }
              }
          } else if (live) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int l2 = nh0 + 16 * cg + j;
              if (l2 >= b) break;
              const int m2 = l2 * b + l1;
              const float xr = vr[j] * f, xi = vi[j] * f;
              const __half hr = __float2half_rn(xr), hi_ = __float2half_rn(xi);
              const size_t o_r = a_off(s, m2, kc), o_i = a_off(s, m2, s.kh + kc);
              A2[o_r] = hr;
              A2[o_r + (size_t)kTM * kBK] = __float2half_rn(xr - __half2float(hr));
              A2[o_i] = hi_;
              A2[o_i + (size_t)kTM * kBK] = __float2half_rn(xi - __half2float(hi_));
            }
          }
        }
      } else {
        // V = acc / (2^(13-e1-et) 2^13), |V|^2 in FP32, then the FP64 factor
        // const33^2 / (8 sqrt|l1 l2 l3|) from the per-mode 1/sqrt|l|
        const float u = ldexpf(1.f, e1 + et - 2 * kSplitE);
        const int l2 = live ? m / b : 0, l1 = live ? m % b : 0;
        const double c12 = live ? a.const33 * a.const33 / 8 * t.tq[(size_t)pi.q1 * b + l1] * t.tq[(size_t)pi.q2 * b + l2]
                                : 0.0;
        const double* t3 = t.tq + (size_t)pi.q3 * b;
        const size_t nkc = g.nkc;
        for (int cg = 0; cg < s.ncol / 16; ++cg) {
          float vr[16], vi[16];
          tmem_ld16x2(taddr + (uint32_t)(16 * cg), taddr + (uint32_t)(s.ncol + 16 * cg), vr, vi);
          if (!live) continue;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int l3 = nh0 + 16 * cg + j;
            if (l3 >= b) break;
            const double sc = c12 * t3[l3];
            double v = 0.0;
            if (sc < 1.0 / 0.0) {
              const float re = vr[j] * u, im = vi[j] * u;
              v = (double)fmaf(re, re, im * im) * sc;
            } else {
              atomicOr(a.err, 2);  // matrix_elt_simplified: den = 0
            }
            const size_t o = v3_out_off(a.v3_layout, pi.row, pi.q2, l1, l2, l3, b, nkc);
            if (a.v3sq_f32) a.v3sq_f32[o] = (float)v;
            else a.v3sq[o] = v;
          }
        }
      }
    } else {
      s_fail = 1;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (tid == 0 && s_fail) atomicOr(a.err, 16);
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(s.tmem_cols));
}

}  // namespace

bool v3_dense_tc_supported(int b) {
  // every cell but the 3- and 6-band ones, which have their own kernels
  if (b < 7 || b > kHeevMaxBands) return false;
  const DenseTcShape s = dense_tc_shape(b);
  return s.stages >= 2 && s.tmem_cols <= 256 && s.ncol % 16 == 0;
}

int v3_pipeline_layout(int b, int precision) {
  if (precision == ALD_MIXED && v3_dense_tc_supported(b)) return 2;
  if (b == 3 || b == 6 || b > 12) return 1;
  return 0;
}

long long v3_dense_tc_pairs(int b, long long npairs, size_t budget) {
  const DenseTcShape s = dense_tc_shape(b);
  const size_t per = 2 * s.a_pair_halves * sizeof(__half);
  return std::max<long long>(1, std::min<long long>({npairs, (long long)(budget / per), 65535LL}));
}

size_t v3_dense_tc_work_bytes(int b, int nkc, int nrows, long long pairs) {
  const DenseTcShape s = dense_tc_shape(b);
  return (size_t)pairs * 2 * s.a_pair_halves * sizeof(__half) + (size_t)nkc * s.bq_halves * sizeof(__half) +
         (size_t)nkc * b * sizeof(double) + (size_t)nrows * 2 * sizeof(int) + 512;
}

int v3_dense_tc_launches(long long npairs, long long pairs) { return 4 + 3 * (int)((npairs + pairs - 1) / pairs); }

cudaError_t launch_v3_dense_tc(const V3Args& a, void* work, long long P, bool a2_zeroed, cudaStream_t s) {
  const int b = a.geo.b;
  if (!v3_dense_tc_supported(b) || !a.hbuf || P < 1 || P > 65535) return cudaErrorInvalidValue;
  const DenseTcShape sh = dense_tc_shape(b);
  const long long npairs = (long long)a.nrows * a.geo.nkc;
  char* w = static_cast<char*>(work);
  DenseTc t;
  t.sh = sh;
  t.a1 = reinterpret_cast<__half*>(w);
  t.a2 = t.a1 + (size_t)P * sh.a_pair_halves;
  t.bq = t.a2 + (size_t)P * sh.a_pair_halves;
  t.tq = reinterpret_cast<double*>(t.bq + (size_t)a.geo.nkc * sh.bq_halves);
  unsigned* bound = reinterpret_cast<unsigned*>(t.tq + (size_t)a.geo.nkc * b);
  t.rexp = reinterpret_cast<int*>(bound + a.nrows);
  cudaError_t e;
  if (!a2_zeroed) {  // GEMM 1's epilogue never writes the padding of A2
    e = cudaMemsetAsync(t.a2, 0, (size_t)P * sh.a_pair_halves * sizeof(__half), s);
    if (e != cudaSuccess) return e;
  }
  e = cudaMemsetAsync(bound, 0, (size_t)a.nrows * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  v3tc_bq_kernel<<<a.geo.nkc, 256, 0, s>>>(a, t);
  v3tc_modes_kernel<<<(a.geo.nkc * b + 255) / 256, 256, 0, s>>>(a, t.tq);
  v3tc_rowbound_kernel<<<dim3(64, a.nrows), 256, 0, s>>>(a, bound);
  v3tc_rowexp_kernel<<<(a.nrows + 127) / 128, 128, 0, s>>>(a.nrows, bound, t.rexp);
  // phase table of every class in shared memory up to 96 KB (12 288 classes)
  const int table_ph = (size_t)a.ncls * sizeof(float2) <= 96 * 1024;
  const size_t t1_smem = table_ph ? (size_t)std::max(a.ncls, 1) * sizeof(float2) : 0;
  if (t1_smem > 48 * 1024) {
    e = raise_smem_limit((const void*)v3tc_t1_kernel, t1_smem);
    if (e != cudaSuccess) return e;
  }
  e = raise_smem_limit((const void*)v3tc_gemm_kernel<1>, t.sh.smem);
  if (e != cudaSuccess) return e;
  e = raise_smem_limit((const void*)v3tc_gemm_kernel<2>, t.sh.smem);
  if (e != cudaSuccess) return e;
  for (long long p0 = 0; p0 < npairs; p0 += P) {
    const int np = (int)std::min<long long>(P, npairs - p0);
    v3tc_t1_kernel<<<dim3(sh.mtiles, np), 256, t1_smem, s>>>(a, t, p0, table_ph);
    const dim3 gg(sh.mtiles * sh.nsplit, np);  // the column halves of one tile are neighbours
    v3tc_gemm_kernel<1><<<gg, kThreads, t.sh.smem, s>>>(a, t, p0);
    v3tc_gemm_kernel<2><<<gg, kThreads, t.sh.smem, s>>>(a, t, p0);
  }
  return cudaGetLastError();
}

}  // namespace ald
