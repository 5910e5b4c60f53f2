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
// The single wait of the CTA (the MMA-completion mbarrier) is bounded: on
// timeout the CTA sets bit 4 of the error flag, waits (bounded) once more,
// frees its TMEM and returns without storing.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kTM = 128;      // q2 per CTA = TMEM lanes = threads
constexpr int kNC = 27;       // complex outputs (l1, be, ga) for 3 bands
constexpr int kNP = 64;       // real outputs padded to a valid N
constexpr int kTmemCols = 64; // FP32 accumulator columns
constexpr int kMaxKp = 256;   // K' bound (ncls <= 128)
constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ int wrapm(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}
__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}
__device__ __forceinline__ int idx_q3(const Geometry& g, const int* m1, const int* m2) {
  int m3[3];
  for (int a = 0; a < 3; ++a) m3[a] = wrapm(-m1[a] - m2[a] + (g.shifted ? g.nc[a] / 2 : 0), g.nc[a]);
  return m3[2] + g.nc[2] * (m3[1] + g.nc[1] * m3[0]);
}
__device__ __forceinline__ int phase_index(const int* pc, const int* m, int L) {
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

__global__ void __launch_bounds__(kTM, 1) v3_tc3_kernel(V3Args a, int kp) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ float s_scale[kNC];
  __shared__ int s_ok;
  const Geometry& g = a.geo;
  const int tid = threadIdx.x, warp = tid >> 5, row = blockIdx.y;
  const int ncls = a.ncls;
  __half* Ahi = reinterpret_cast<__half*>(smraw);
  __half* Alo = Ahi + kTM * kp;
  __half* Bhi = Alo + kTM * kp;
  __half* Blo = Bhi + kNP * kp;

  // TMEM: 64 columns, allocated by warp 0
  if (warp == 0) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_tmem);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&s_bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_ok = 1;
  }

  const int q1 = a.mapinv[a.n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  const int q2 = min((int)(blockIdx.x * kTM) + tid, g.nkc - 1);
  int m2[3];
  decompose(g, q2, m2);
  const int q3 = idx_q3(g, m1, m2);

  // H of this row: column scales (a power of two >= max |H| of the column)
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
    s_scale[tid] = ldexpf(1.f, -e);  // mx * scale in [0.5, 1)
  }
  __syncthreads();
  // B operand (N' x K'): n' = 2 col + {0: real, 1: imaginary}
  for (int i = tid; i < kNP * kp; i += kTM) {
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
    split_store(Bhi, Blo, kmaj(n, k, kNP), v);
  }
  // A operand (M x K'): row = q2, [Pr | Pi] of every class
  const double2* roots = reinterpret_cast<const double2*>(a.roots);
  for (int k = 0; k < kp; ++k) {  // thread tid fills row tid (its own q2)
    float v = 0.f;
    if (k < 2 * ncls) {
      const int c = k < ncls ? k : k - ncls;
      const double2 p = roots[phase_index(a.cls_pc + 4 * c, m2, g.L)];
      v = (float)(k < ncls ? p.x : p.y);
    }
    split_store(Ahi, Alo, kmaj(tid, k, kTM), v);
  }
  // make the generic-proxy stores visible to the tensor core, then issue
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&s_bar);
  if (tid == 0) {
    const uint32_t idesc = instr_desc(kTM, kNP);
    const uint32_t aH = (uint32_t)__cvta_generic_to_shared(Ahi), aL = (uint32_t)__cvta_generic_to_shared(Alo);
    const uint32_t bH = (uint32_t)__cvta_generic_to_shared(Bhi), bL = (uint32_t)__cvta_generic_to_shared(Blo);
    for (int s = 0; s < kp / 16; ++s) {
      // K step s covers K chunks 2s, 2s+1: start ROWS*16 bytes per chunk
      const uint32_t oa = (uint32_t)(2 * s * kTM * 16), ob = (uint32_t)(2 * s * kNP * 16);
      const uint64_t dAh = smem_desc(aH + oa, kTM * 16, 128), dAl = smem_desc(aL + oa, kTM * 16, 128);
      const uint64_t dBh = smem_desc(bH + ob, kNP * 16, 128), dBl = smem_desc(bL + ob, kNP * 16, 128);
      mma_f16(tmem, dAh, dBh, idesc, s > 0 ? 1u : 0u);
      mma_f16(tmem, dAh, dBl, idesc, 1u);
      mma_f16(tmem, dAl, dBh, idesc, 1u);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
  }
  // bounded wait for the MMAs
  bool done = false;
  for (unsigned it = 0; it < kWaitLimit && !done; ++it) done = mbar_try(bar, 0);
  if (!done) s_ok = 0;  // benign race: every writer stores 0
  __syncthreads();
  const bool ok = s_ok != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok) {
    if (tid == 0) atomicOr(a.err, 16);
    for (unsigned it = 0; it < kWaitLimit && !done; ++it) done = mbar_try(bar, 0);
  } else {
    // this thread's accumulator row: TMEM lane 32*warp + lane
    uint32_t d[kNP];
    const uint32_t base = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
    for (int c8 = 0; c8 < kNP / 8; ++c8)
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(d[8 * c8 + 0]), "=r"(d[8 * c8 + 1]), "=r"(d[8 * c8 + 2]), "=r"(d[8 * c8 + 3]), "=r"(d[8 * c8 + 4]),
            "=r"(d[8 * c8 + 5]), "=r"(d[8 * c8 + 6]), "=r"(d[8 * c8 + 7])
          : "r"(base + 8 * c8));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    float2 A[kNC];
#pragma unroll
    for (int c = 0; c < kNC; ++c) {
      const float inv = 1.f / s_scale[c];
      A[c] = make_float2(__uint_as_float(d[2 * c]) * inv, __uint_as_float(d[2 * c + 1]) * inv);
    }
    // mode products with e(q2), e(q3): V[l1][l2][l3] = sum_{b,c} A[l1][b][c] e2[b][l2] e3[c][l3]
    const double2* ev = reinterpret_cast<const double2*>(a.evec);
    float2 e2[9], e3[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const double2 x = ev[(size_t)q2 * 9 + i], y = ev[(size_t)q3 * 9 + i];  // e[q][l][i]
      e2[i] = make_float2((float)x.x, (float)x.y);
      e3[i] = make_float2((float)y.x, (float)y.y);
    }
    const int qg = blockIdx.x * kTM + tid;
    if (qg < g.nkc) {
      const double c33 = a.const33 * a.const33 / 8;
      double t2[3], t3[3];
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        t2[l] = 1.0 / sqrt(fabs(a.w2[(size_t)q2 * 3 + l]));
        t3[l] = 1.0 / sqrt(fabs(a.w2[(size_t)q3 * 3 + l]));
      }
      const size_t nk = g.nkc;
#pragma unroll
      for (int l1 = 0; l1 < 3; ++l1) {
        const double c1 = c33 / sqrt(fabs(a.w2[(size_t)q1 * 3 + l1]));
        // T[l2][c] = sum_b A[l1][b][c] e2[b][l2]   (e2[b][l2] at e2[l2*3 + b])
        float2 T[3][3];
#pragma unroll
        for (int l2 = 0; l2 < 3; ++l2)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) {
              const float2 x = A[l1 * 9 + bb * 3 + c], y = e2[l2 * 3 + bb];
              s.x = fmaf(x.x, y.x, fmaf(-x.y, y.y, s.x));
              s.y = fmaf(x.x, y.y, fmaf(x.y, y.x, s.y));
            }
            T[l2][c] = s;
          }
#pragma unroll
        for (int l2 = 0; l2 < 3; ++l2)
#pragma unroll
          for (int l3 = 0; l3 < 3; ++l3) {
            float2 s = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const float2 x = T[l2][c], y = e3[l3 * 3 + c];
              s.x = fmaf(x.x, y.x, fmaf(-x.y, y.y, s.x));
              s.y = fmaf(x.x, y.y, fmaf(x.y, y.x, s.y));
            }
            const double sc = c1 * t2[l2] * t3[l3];
            double v = 0.0;
            if (sc < 1.0 / 0.0) v = ((double)s.x * s.x + (double)s.y * s.y) * sc;
            else atomicOr(a.err, 2);  // matrix_elt_simplified: den = 0
            double* out = a.v3_layout == 1 ? a.v3sq + (((size_t)row * 27 + l2 * 9 + l3 * 3 + l1) * nk + qg)
                                           : a.v3sq + ((size_t)row * nk + qg) * 27 + l1 * 9 + l2 * 3 + l3;
            *out = v;
          }
      }
    }
  }
  // free TMEM after every warp's loads
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

bool v3_tc_supported(int b, int ncls) { return b == 3 && ncls >= 1 && 2 * ncls <= kMaxKp; }

cudaError_t launch_v3_tc(const V3Args& a, cudaStream_t s) {
  if (!v3_tc_supported(a.geo.b, a.ncls)) return cudaErrorInvalidValue;
  const int kp = (2 * a.ncls + 15) / 16 * 16;
  const size_t smem = (size_t)(kTM + kNP) * kp * 2 * sizeof(__half);
  cudaError_t e = cudaFuncSetAttribute(v3_tc3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.geo.nkc + kTM - 1) / kTM, a.nrows);
  v3_tc3_kernel<<<grid, kTM, smem, s>>>(a, kp);
  return cudaGetLastError();
}

}  // namespace ald
