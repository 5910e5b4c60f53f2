// |V3|^2 for cells of more than 12 bands: the class sums and the two
// eigenvector mode products as batched dense complex GEMMs (FP64 path).
//
// Replaces calculate_w3_ibz_split_sq + matrix_elt_simplified
// (THERMACOND/sub.f90:1050-1233, 5888-6011) and cal_eiqr2 (sub.f90:6015)
// for large cells.  With the phase classes of ald_v3_pair.cu (row stage
// H[c][be ga][l1], one per IBZ row), a pair (q1, q2) needs
//   T1[jb][l1][kc] = sum_{c in group (j0,k0)} P_c(q2) H[c][be ga][l1]
//                    (jb = 3 j0 + be, kc = 3 k0 + ga)
//   T2[l2][l1][kc] = sum_jb T1[jb][l1][kc] e2[jb][l2]        GEMM 1
//   V[l1][l2][l3]  = sum_kc T2[l2][l1][kc] e3[kc][l3]        GEMM 2
// and |V|^2 (const33 / sqrt(8 sqrt|l1 l2 l3|))^2.  GEMM 1 has M = b^2 rows
// (l1, kc), N = b (l2), K = b (jb); GEMM 2 M = b^2 rows (l2, l1), N = b
// (l3), K = b (kc): 8 b^4 real flops each per pair, the 24 b^4 of the
// dense contraction with the class sums.  A batch of pairs (consecutive in
// (row, q2)) keeps T1 and T2 in a workspace; GEMM 2's epilogue forms |V|^2
// and writes the chunk's |V3|^2 layout.  Eigenvectors are not conjugated,
// as in the reference.  Sums are reordered: agreement to FP64 rounding.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

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

// the pair's row (local to the chunk), q1, q2 and q3
struct PairIdx {
  int row, q1, q2, q3;
};
__device__ __forceinline__ PairIdx pair_idx(const V3Args& a, long long pair) {
  PairIdx p;
  const int nkc = a.geo.nkc;
  if (a.pair_list) pair = a.pair_list[pair];
  p.row = (int)(pair / nkc);
  p.q2 = (int)(pair % nkc);
  p.q1 = a.mapinv[a.n1_first + p.row];
  int m1[3], m2[3];
  decompose(a.geo, p.q1, m1);
  decompose(a.geo, p.q2, m2);
  p.q3 = idx_q3(a.geo, m1, m2);
  return p;
}

// T1 of the batch's pairs: CTA (pair, jb), threads over (l1, kc)
constexpr int kT1Threads = 256;
__global__ void __launch_bounds__(kT1Threads) v3_t1_kernel(V3Args a, long long pair0, double2* T1, int table_ph,
                                                             int nk1) {
  extern __shared__ double2 s_ph[];  // P_c(q2) of every class
  const Geometry& g = a.geo;
  const int b = g.b, nat0 = g.nat0;
  const int p = blockIdx.x, jb = blockIdx.y, j0 = jb / 3, be = jb % 3;
  const PairIdx pi = pair_idx(a, pair0 + p);
  int m2[3];
  decompose(g, pi.q2, m2);
  const double2* roots = reinterpret_cast<const double2*>(a.roots);
  // the classes' phases in shared memory when they fit (table_ph), else
  // read from the roots table where used
  if (table_ph)
    for (int c = threadIdx.x; c < a.ncls; c += blockDim.x) s_ph[c] = roots[phase_index(a.cls_pc + 4 * c, m2, g.L, g.L32)];
  __syncthreads();
  const double2* H = static_cast<const double2*>(a.hbuf) + (size_t)pi.row * a.ncls * 9 * b;
  double2* out = T1 + ((size_t)p * b + jb) * b * b;
  for (int e = threadIdx.x; e < nk1 * b; e += blockDim.x) {  // bands l1 < nk1
    const int l1 = e / b, kc = e % b, k0 = kc / 3, ga = kc % 3;
    const int grp = j0 * nat0 + k0;
    double2 acc = make_double2(0.0, 0.0);
    for (int c = a.cls_grp_off[grp]; c < a.cls_grp_off[grp + 1]; ++c) {
      const double2 ph = table_ph ? s_ph[c] : roots[phase_index(a.cls_pc + 4 * c, m2, g.L, g.L32)];
      const double2 h = H[((size_t)c * 9 + be * 3 + ga) * b + l1];
      acc.x = fma(ph.x, h.x, fma(-ph.y, h.y, acc.x));
      acc.y = fma(ph.x, h.y, fma(ph.y, h.x, acc.y));
    }
    out[e] = acc;  // T1[p][jb][l1][kc]
  }
}

// Batched complex GEMM, FP64: C(m, n) = sum_k A(m, k) B(k, n) for every pair
// of the batch.  64 x 64 tile per CTA, K steps of 8, 256 threads with 4 x 4
// outputs each (rows ty + 16 i, columns tx + 16 j).
//   kind 1 (GEMM 1): A(m = l1 b + kc, k = jb) = T1[p][k][m]   (m contiguous)
//                    B(k, n = l2) = e(q2)[n][k],  C -> T2[p][n][m]
//   kind 2 (GEMM 2): A(m = l2 b + l1, k = kc) = T2[p][m][k]   (k contiguous)
//                    B(k, n = l3) = e(q3)[n][k],  epilogue |V|^2 -> v3sq
// With l1 < nk1 only (nk1 < b): GEMM 1 has the first nk1 b rows; GEMM 2 the
// rows m' = l2 nk1 + l1 (A row l2 b + l1).
constexpr int kGM = 64, kGN = 64, kGK = 8, kGThreads = 256;

template <int KIND>
__global__ void __launch_bounds__(kGThreads) v3_zgemm_kernel(V3Args a, long long pair0, const double2* Ain,
                                                             double2* Cout, int nk1) {
  __shared__ double2 As[kGK][kGM + 1];
  __shared__ double2 Bs[kGK][kGN + 1];
  const Geometry& g = a.geo;
  const int b = g.b, b2 = b * b;
  const int M = nk1 * b, N = b, K = b;
  // A row of GEMM row m (GEMM 2 with a band subset: m = l2 nk1 + l1)
  auto arow = [&](int m) { return KIND == 2 && nk1 < b ? (m / nk1) * b + m % nk1 : m; };
  const int p = blockIdx.z;
  const PairIdx pi = pair_idx(a, pair0 + p);
  const int m0 = blockIdx.x * kGM, n0 = blockIdx.y * kGN;
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const double2* A = Ain + (size_t)p * b2 * b;
  const double2* B = reinterpret_cast<const double2*>(a.evec) + (size_t)(KIND == 1 ? pi.q2 : pi.q3) * b2;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < K; k0 += kGK) {
    // A tile: 64 x 8 = 512 elements, two per thread
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = tid + r * kGThreads;
      int mi, ki;
      if (KIND == 1) {  // m contiguous
        mi = e % kGM;
        ki = e / kGM;
      } else {  // k contiguous
        ki = e % kGK;
        mi = e / kGK;
      }
      const int m = m0 + mi, k = k0 + ki;
      double2 v = make_double2(0.0, 0.0);
      if (m < M && k < K) v = KIND == 1 ? A[(size_t)k * b2 + m] : A[(size_t)arow(m) * b + k];
      As[ki][mi] = v;
    }
    // B tile: 8 x 64, k contiguous in e(q)[n][k]
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = tid + r * kGThreads;
      const int ki = e % kGK, ni = e / kGK;
      const int n = n0 + ni, k = k0 + ki;
      Bs[ki][ni] = (n < N && k < K) ? B[(size_t)n * b + k] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(av[i].x, bv[j].x, fma(-av[i].y, bv[j].y, acc[i][j].x));
          acc[i][j].y = fma(av[i].x, bv[j].y, fma(av[i].y, bv[j].x, acc[i][j].y));
        }
    }
    __syncthreads();
  }
  if (KIND == 1) {
    double2* C = Cout + (size_t)p * b2 * b;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
        if (m < M && n < N) C[(size_t)n * b2 + m] = acc[i][j];  // T2[p][l2][l1][kc]
      }
  } else {
    const double* w2 = a.w2;
    const size_t nkc = g.nkc;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int m = m0 + ty + 16 * i, l3 = n0 + tx + 16 * j;
        if (m >= M || l3 >= N) continue;
        const int l2 = m / nk1, l1 = m % nk1;
        const double den = sqrt(8 * sqrt(fabs(w2[(size_t)pi.q1 * b + l1] * w2[(size_t)pi.q2 * b + l2] *
                                              w2[(size_t)pi.q3 * b + l3])));
        double v = 0.0;
        if (den != 0.0) {
          const double re = acc[i][j].x / den * a.const33, im = acc[i][j].y / den * a.const33;
          v = re * re + im * im;
        } else {
          atomicOr(a.err, 2);
        }
        const size_t b3 = (size_t)b2 * b;
        size_t o;
        if (a.v3_layout == 2)  // [row][l2][l3][q2][l1]
          o = (((size_t)pi.row * b + l2) * b + l3) * nkc * b + (size_t)pi.q2 * b + l1;
        else if (a.v3_layout == 1)  // [row][l2][l3][l1][q2]
          o = (size_t)pi.row * nkc * b3 + (((size_t)l2 * b + l3) * b + l1) * nkc + pi.q2;
        else  // [row][q2][l1][l2][l3]
          o = ((size_t)pi.row * nkc + pi.q2) * b3 + ((size_t)l1 * b + l2) * b + l3;
        if (a.v3sq_f32) a.v3sq_f32[o] = (float)v;
        else a.v3sq[o] = v;
      }
  }
}

// |V3|^2 of one row in the reference's order, [q2][l1][l2][l3] FP64, into
// row `row` of a chunk in its layout and precision, bands l1 < nk1 only
__global__ void v3_copy_row_kernel(V3Args a, int row, const double* __restrict__ src, int nk1) {
  const int b = a.geo.b, nkc = a.geo.nkc;
  const long long n = (long long)nkc * nk1 * b * b;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int l3 = (int)(i % b), l2 = (int)((i / b) % b), l1 = (int)((i / ((long long)b * b)) % nk1);
    const int q2 = (int)(i / ((long long)b * b * nk1));
    const double v = src[(((size_t)q2 * b + l1) * b + l2) * b + l3];
    const size_t b3 = (size_t)b * b * b;
    size_t o;
    if (a.v3_layout == 2) o = (((size_t)row * b + l2) * b + l3) * nkc * b + (size_t)q2 * b + l1;
    else if (a.v3_layout == 1) o = (size_t)row * nkc * b3 + (((size_t)l2 * b + l3) * b + l1) * nkc + q2;
    else o = ((size_t)row * nkc + q2) * b3 + ((size_t)l1 * b + l2) * b + l3;
    if (a.v3sq_f32) a.v3sq_f32[o] = (float)v;
    else a.v3sq[o] = v;
  }
}

}  // namespace

bool v3_dense_supported(int b) { return b > 12 && b <= kHeevMaxBands; }

size_t v3_dense_work_bytes(int b, long long npairs, size_t budget) {
  const size_t per = 2 * (size_t)b * b * b * sizeof(double2);
  const long long p = std::max<long long>(1, std::min<long long>({npairs, (long long)(budget / per), 65535LL}));
  return (size_t)p * per;
}

cudaError_t launch_v3_dense(const V3Args& a, void* work, size_t work_bytes, cudaStream_t s, int l1_keep) {
  const int b = a.geo.b;
  // any band count as the FP64 near-zero-mode pass of the mixed path (a pair list)
  if (!a.hbuf || b > kHeevMaxBands || (!a.pair_list && !v3_dense_supported(b))) return cudaErrorInvalidValue;
  const int nk1 = l1_keep > 0 && l1_keep < b ? l1_keep : b;
  const size_t b3 = (size_t)b * b * b;
  const long long npairs = a.pair_list ? a.npairs_list : (long long)a.nrows * a.geo.nkc;
  // pairs per batch: as many as the workspace holds, at most 65535 (grid z)
  const long long P =
      std::min<long long>(65535, std::max<long long>(1, (long long)(work_bytes / (2 * b3 * sizeof(double2)))));
  double2* T1 = static_cast<double2*>(work);
  double2* T2 = T1 + (size_t)P * b3;
  // phase table of every class in shared memory up to 96 KB (6 144 classes)
  const int table_ph = (size_t)a.ncls * sizeof(double2) <= 96 * 1024;
  const size_t t1_smem = table_ph ? (size_t)std::max(a.ncls, 1) * sizeof(double2) : 0;
  if (t1_smem > 48 * 1024) {
    cudaError_t e = raise_smem_limit((const void*)v3_t1_kernel, t1_smem);
    if (e != cudaSuccess) return e;
  }
  for (long long p0 = 0; p0 < npairs; p0 += P) {
    const int np = (int)std::min<long long>(P, npairs - p0);
    v3_t1_kernel<<<dim3(np, b), kT1Threads, t1_smem, s>>>(a, p0, T1, table_ph, nk1);
    const dim3 gg((nk1 * b + kGM - 1) / kGM, (b + kGN - 1) / kGN, np);
    v3_zgemm_kernel<1><<<gg, kGThreads, 0, s>>>(a, p0, T1, T2, nk1);
    v3_zgemm_kernel<2><<<gg, kGThreads, 0, s>>>(a, p0, T2, nullptr, nk1);
  }
  return cudaGetLastError();
}

cudaError_t launch_v3_copy_row(const V3Args& a, int row, const double* src, int l1_keep, cudaStream_t s) {
  const int b = a.geo.b;
  const int nk1 = l1_keep > 0 && l1_keep < b ? l1_keep : b;
  const long long n = (long long)a.geo.nkc * nk1 * b * b;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
  v3_copy_row_kernel<<<blocks, 256, 0, s>>>(a, row, src, nk1);
  return cudaGetLastError();
}

}  // namespace ald
