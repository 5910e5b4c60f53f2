// |V3|^2 by phase classes: the pair kernel (3 and 6 bands).
//
// Replaces calculate_w3_ibz_split_sq + matrix_elt_simplified
// (THERMACOND/sub.f90:1050-1233, 5888-6011) and cal_eiqr2 (sub.f90:6015)
// for small cells.  The reference sums nterms3 complex terms per band triplet;
// with q3 = -q1-q2 folded on the mesh the phase of an FC3 atom triple
// (i0, j, k) factors as
//     exp(i q2.R_j) exp(i q3.R_k) = exp(i q2.(R_j - R_k)) * exp(-i q1.R_k)
// (exact on mesh integers: q.R reduced mod L), so the sum is reorganised:
//   row stage   H[c][be ga][l1] = sum_{triples t in class c} exp(-i q1.R_k)
//                 sum_al W_t[al be ga] e1[i0 al][l1]
//               for every class c of triples sharing (j0, k0, R_j - R_k);
//               H depends on the IBZ row only.
//   pair stage  A[l1][j0 be][k0 ga] = sum_{c in group (j0,k0)} P_c(q2) H[c][be ga][l1]
//               with P_c(q2) = exp(i q2.(R_j - R_k)), a tile of q2 per CTA;
//               T[l1][l2][c']   = sum_b' A[l1][b'][c'] e2[b'][l2]   (e(q2))
//               V[l1][l2][l3]   = sum_c' T[l1][l2][c'] e3[c'][l3]   (e(q3))
//               |V|^2 (const33 / sqrt(8 sqrt|l1 l2 l3|))^2, the scale formed from
//               per-mode factors 1/sqrt|l| (reordered against the reference).
// Eigenvectors are not conjugated, as in the reference.  The sums are
// reordered against the reference, so results agree to FP64 rounding.
//
// precision ALD_FP64 runs every stage in double.  ALD_MIXED runs the class
// sums and both mode products in float (FP32 accumulation) from double
// inputs, and keeps den and |V|^2 in double.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

template <class T>
struct Cx;
template <>
struct Cx<double> {
  using t = double2;
};
template <>
struct Cx<float> {
  using t = float2;
};

template <class C>
__device__ __forceinline__ void cmac(C& acc, const C& a, const C& b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

template <class C>
__device__ __forceinline__ C cvt(const double2& v);
template <>
__device__ __forceinline__ double2 cvt<double2>(const double2& v) {
  return v;
}
template <>
__device__ __forceinline__ float2 cvt<float2>(const double2& v) {
  return make_float2((float)v.x, (float)v.y);
}

__device__ __forceinline__ int wrapm(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}
__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}
// mesh index of q3 = -q1-q2
__device__ __forceinline__ int idx_q3(const Geometry& g, const int* m1, const int* m2) {
  int m3[3];
  for (int a = 0; a < 3; ++a) m3[a] = wrapm(-m1[a] - m2[a] + (g.shifted ? g.nc[a] / 2 : 0), g.nc[a]);
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

// ---------------------------------------------------------------- row stage
template <class C>
__global__ void v3_row_kernel(V3Args a) {
  const Geometry& g = a.geo;
  const int b = g.b, b2 = b * b, row = blockIdx.y;
  const int q1 = a.mapinv[a.n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  const int n = a.ncls * 9 * b;
  C* H = static_cast<C*>(a.hbuf) + (size_t)row * n;
  const double2* roots = reinterpret_cast<const double2*>(a.roots);
  const double2* e1 = reinterpret_cast<const double2*>(a.evec) + (size_t)q1 * b2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int l1 = e % b, bg = (e / b) % 9, c = e / (9 * b);
    double2 acc = make_double2(0.0, 0.0);
    for (int s = a.cls_trip_off[c]; s < a.cls_trip_off[c + 1]; ++s) {
      const int t = a.cls_trip[s], i0 = a.cls_trip_i0[s], k = a.cls_trip_k[s];
      int ph = phase_index(a.phase_coef + 4 * k, m1, g.L, g.L32);
      const double2 r = roots[ph == 0 ? 0 : g.L - ph];  // exp(-i q1.R_k)
      double2 x = make_double2(0.0, 0.0);
      for (int al = 0; al < 3; ++al) {
        const double w = a.fc3w[27 * (size_t)t + al * 9 + bg];
        const double2 v = e1[l1 * b + 3 * i0 + al];
        x.x = fma(w, v.x, x.x);
        x.y = fma(w, v.y, x.y);
      }
      cmac(acc, r, x);
    }
    H[e] = cvt<C>(acc);  // H[row][c][be ga][l1]
  }
}

// ---------------------------------------------------------------- pair stage
// One CTA: one IBZ row, QT consecutive q2.  Shared memory (complex units):
//   At[QT][AP]  the class sums A, then T in place (odd pitch: no bank conflicts
//               when lanes walk q)
//   E2[QT][EP], E3[QT][EP]  e(q2), e(q3) as [l][i]
//   P[QT][PP]   P_c(q2)
// Tasks: class sums (q, j0 be, k0 ga) -> B values of l1 each;
// mode product 2 (q, c', l1 block) -> (B/S) x B accumulators;
// mode product 3 (q, l1, l2 block) -> (B/S) x B accumulators and |V|^2.
template <class T, int B, int QT, int S, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 3 : 2) v3_pair_kernel(V3Args a) {
  using C = typename Cx<T>::t;
  constexpr int NAT = B / 3, B2 = B * B, B3 = B2 * B, NG = NAT * NAT;
  constexpr int AP = B3 | 1, EP = B2 | 1, BS = B / S;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const Geometry& g = a.geo;
  const int tid = threadIdx.x, row = blockIdx.y;
  const int PP = a.ncls | 1;
  C* At = sm;
  C* E2 = At + QT * AP;
  C* E3 = E2 + QT * EP;
  C* P = E3 + QT * EP;
  __shared__ int s_q2[QT], s_q3[QT];
  // 1/sqrt|lambda| of the tile's q2 and q3 modes: (const33/den)^2 with
  // den = sqrt(8 sqrt|l1 l2 l3|) is const33^2/8 * t1 t2 t3
  __shared__ double s_t2[QT * B], s_t3[QT * B];

  const int q1 = a.mapinv[a.n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  const int qbase = blockIdx.x * QT;
  if (tid < QT) {
    const int q2 = min(qbase + tid, g.nkc - 1);
    int m2[3];
    decompose(g, q2, m2);
    s_q2[tid] = q2;
    s_q3[tid] = idx_q3(g, m1, m2);
  }
  __syncthreads();
  for (int i = tid; i < QT * B; i += NT) {
    const int q = i / B, l = i % B;
    s_t2[i] = 1.0 / sqrt(fabs(a.w2[(size_t)s_q2[q] * B + l]));
    s_t3[i] = 1.0 / sqrt(fabs(a.w2[(size_t)s_q3[q] * B + l]));
  }
  const double2* ev = reinterpret_cast<const double2*>(a.evec);
  for (int i = tid; i < QT * B2; i += NT) {
    const int q = i / B2, e = i % B2;
    E2[q * EP + e] = cvt<C>(ev[(size_t)s_q2[q] * B2 + e]);
    E3[q * EP + e] = cvt<C>(ev[(size_t)s_q3[q] * B2 + e]);
  }
  const double2* roots = reinterpret_cast<const double2*>(a.roots);
  for (int i = tid; i < QT * a.ncls; i += NT) {
    const int q = i % QT, c = i / QT;
    int m2[3];
    decompose(g, s_q2[q], m2);
    P[q * PP + c] = cvt<C>(roots[phase_index(a.cls_pc + 4 * c, m2, g.L, g.L32)]);
  }
  __syncthreads();

  // class sums: A[q][l1][j0 be][k0 ga]; in FP32 a thread per (column, q and
  // q + QT/2), so that each H value it loads serves two pairs (FP64: one q,
  // the registers of two would spill)
  const C* H = static_cast<const C*>(a.hbuf) + (size_t)row * a.ncls * 9 * B;
  constexpr int QB = sizeof(T) == 4 ? 2 : 1, QH = QT / QB;
  for (int task = tid; task < QH * NG * 9; task += NT) {
    const int q = task % QH, col = task / QH;
    const int grp = col / 9, bg = col % 9;
    const int j0 = grp / NAT, k0 = grp % NAT, be = bg / 3, ga = bg % 3;
    C acc[QB][B];
#pragma unroll
    for (int k = 0; k < QB; ++k)
#pragma unroll
      for (int l = 0; l < B; ++l) acc[k][l] = C{0, 0};
    const int c0 = a.cls_grp_off[grp], c1 = a.cls_grp_off[grp + 1];
    for (int c = c0; c < c1; ++c) {
      C p[QB];
#pragma unroll
      for (int k = 0; k < QB; ++k) p[k] = P[(q + k * QH) * PP + c];
      const C* h = H + ((size_t)c * 9 + bg) * B;
#pragma unroll
      for (int l = 0; l < B; ++l) {
        const C hv = h[l];
#pragma unroll
        for (int k = 0; k < QB; ++k) cmac(acc[k][l], p[k], hv);
      }
    }
    C* dst = At + q * AP + (3 * j0 + be) * B + 3 * k0 + ga;
#pragma unroll
    for (int k = 0; k < QB; ++k)
#pragma unroll
      for (int l = 0; l < B; ++l) dst[k * QH * AP + l * B2] = acc[k][l];
  }
  __syncthreads();

  // mode product 2, in place: T[q][l1][l2][c'] = sum_b' A[q][l1][b'][c'] e2[b'][l2]
  for (int task = tid; task < QT * B * S; task += NT) {
    const int q = task % QT, r = task / QT;
    const int cp = r % B, l1b = (r / B) * BS;
    C acc[BS][B];
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int l = 0; l < B; ++l) acc[i][l] = C{0, 0};
    C* Aq = At + q * AP + cp;
    const C* e2 = E2 + q * EP;
#pragma unroll
    for (int bp = 0; bp < B; ++bp) {
      C av[BS], evv[B];
#pragma unroll
      for (int i = 0; i < BS; ++i) av[i] = Aq[(l1b + i) * B2 + bp * B];
#pragma unroll
      for (int l = 0; l < B; ++l) evv[l] = e2[l * B + bp];
#pragma unroll
      for (int i = 0; i < BS; ++i)
#pragma unroll
        for (int l = 0; l < B; ++l) cmac(acc[i][l], av[i], evv[l]);
    }
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int l = 0; l < B; ++l) Aq[(l1b + i) * B2 + l * B] = acc[i][l];
  }
  __syncthreads();

  // mode product 3 and |V3|^2: V[q][l1][l2][l3] = sum_c' T[q][l1][l2][c'] e3[c'][l3]
  const double* w2 = a.w2;
  for (int task = tid; task < QT * B * S; task += NT) {
    const int q = task % QT, r = task / QT;
    const int l1 = r % B, l2b = (r / B) * BS;
    const int q2 = qbase + q;
    C acc[BS][B];
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int l = 0; l < B; ++l) acc[i][l] = C{0, 0};
    const C* Tq = At + q * AP + l1 * B2 + l2b * B;
    const C* e3 = E3 + q * EP;
#pragma unroll
    for (int cp = 0; cp < B; ++cp) {
      C tv[BS], evv[B];
#pragma unroll
      for (int i = 0; i < BS; ++i) tv[i] = Tq[i * B + cp];
#pragma unroll
      for (int l = 0; l < B; ++l) evv[l] = e3[l * B + cp];
#pragma unroll
      for (int i = 0; i < BS; ++i)
#pragma unroll
        for (int l = 0; l < B; ++l) cmac(acc[i][l], tv[i], evv[l]);
    }
    if (q2 < g.nkc) {
      const double c1 = a.const33 * a.const33 / 8 / sqrt(fabs(w2[(size_t)q1 * B + l1]));
      // layout 0: [row][q2][l1][l2][l3]; layout 1: [row][l2][l3][l1][q2]
      const size_t nk = g.nkc;
      // FP64, or FP32 (a.v3sq_f32: the mixed pipeline) at the same index
      const size_t o = a.v3_layout == 1 ? ((size_t)row * B3 + l2b * B2 + l1) * nk + q2
                                        : ((size_t)row * nk + q2) * B3 + l1 * B2 + l2b * B;
      const size_t st_l2 = a.v3_layout == 1 ? (size_t)B2 * nk : B, st_l3 = a.v3_layout == 1 ? (size_t)B * nk : 1;
#pragma unroll
      for (int i = 0; i < BS; ++i) {
        const double c12 = c1 * s_t2[q * B + l2b + i];
#pragma unroll
        for (int l = 0; l < B; ++l) {
          const double sc = c12 * s_t3[q * B + l];  // (const33/den)^2; inf where den = 0
          const double re = (double)acc[i][l].x, im = (double)acc[i][l].y;
          double v = 0.0;
          if (sc < 1.0 / 0.0) {
            v = (re * re + im * im) * sc;
          } else {
            atomicOr(a.err, 2);  // matrix_elt_simplified: den = 0
          }
          if (a.v3sq_f32) a.v3sq_f32[o + i * st_l2 + l * st_l3] = (float)v;
          else a.v3sq[o + i * st_l2 + l * st_l3] = v;
        }
      }
    }
  }
}

struct PairCfg {
  int qt, nt;
};

template <class T, int B, int QT, int S, int NT>
cudaError_t launch_pair_t(const V3Args& a, cudaStream_t s) {
  using C = typename Cx<T>::t;
  constexpr int B2 = B * B, B3 = B2 * B;
  const size_t smem = ((size_t)QT * ((B3 | 1) + 2 * (B2 | 1) + (a.ncls | 1))) * sizeof(C);
  if (smem > 220 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = raise_smem_limit((const void*)v3_pair_kernel<T, B, QT, S, NT>, smem);
  if (e != cudaSuccess) return e;
  // row stage
  const int n = a.ncls * 9 * B;
  dim3 rg((n + 255) / 256, a.nrows);
  v3_row_kernel<C><<<rg, 256, 0, s>>>(a);
  // pair stage
  dim3 grid((a.geo.nkc + QT - 1) / QT, a.nrows);
  v3_pair_kernel<T, B, QT, S, NT><<<grid, NT, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_v3_rows_f32(const V3Args& a, cudaStream_t s) {
  const int n = a.ncls * 9 * a.geo.b;
  dim3 rg((n + 255) / 256, a.nrows);
  v3_row_kernel<float2><<<rg, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_v3_rows_f64(const V3Args& a, cudaStream_t s) {
  const int n = a.ncls * 9 * a.geo.b;
  dim3 rg((n + 255) / 256, a.nrows);
  v3_row_kernel<double2><<<rg, 256, 0, s>>>(a);
  return cudaGetLastError();
}

bool v3_pair_supported(int b, int precision) {
  (void)precision;
  return b == 3 || b == 6;
}

size_t v3_hbuf_bytes(int b, int ncls, int nrows, int precision) {
  const size_t cplx = precision != ALD_FP64 ? sizeof(float2) : sizeof(double2);
  return (size_t)nrows * ncls * 9 * b * cplx;
}

cudaError_t launch_v3_pair(const V3Args& a, int precision, cudaStream_t s) {
  const int b = a.geo.b;
  if (precision != ALD_FP64) {
    if (b == 3) return launch_pair_t<float, 3, 32, 3, 288>(a, s);
    if (b == 6) return launch_pair_t<float, 6, 16, 3, 288>(a, s);
  } else {
    if (b == 3) return launch_pair_t<double, 3, 32, 3, 288>(a, s);
    if (b == 6) return launch_pair_t<double, 6, 16, 3, 288>(a, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ald
