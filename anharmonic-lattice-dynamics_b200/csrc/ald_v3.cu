// |V3|^2 on the device, FP64 path.
//
// Replaces calculate_w3_ibz_split_sq + matrix_elt_simplified
// (THERMACOND/sub.f90:1050-1233, 5888-6011) and cal_eiqr2 (sub.f90:6015).
// The reference evaluates, for every (q1 lambda1, q2 lambda2, lambda3),
//   xx = sum_t fcs_3(t)/sqrt(mi mj mk) eiqr2(q2,j) eiqr2(q3,k) e1 e2 e3
// i.e. nterms3 complex terms per band triplet.  Here the sum is split:
//   1. Fourier sum  Phi(q2)[a,b,c] = sum_{triples (i0,j,k)} W[a,b,c] P(j,k)
//      with P = exp(i q2.R_j + i q3.R_k) read from a table of L-th roots of
//      unity: q.R is reduced mod L on mesh integers (exact phases);
//   2. three mode products with e(q1), e(q2), e(q3) (no conjugation);
//   3. |.|^2 * (const33 / sqrt(8 sqrt|l1 l2 l3|))^2.
// One CTA handles one IBZ row and a tile of consecutive q2; the b^3 tensor
// and the eigenvector tiles stay in shared memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ int wrapm(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// mesh index of -q1-q2 (get_k_info on q3 = -q2-q1)
__device__ __forceinline__ int idx_mq1mq2(const Geometry& g, const int* m1, const int* m2, int* m3) {
  for (int a = 0; a < 3; ++a) {
    int v = -m1[a] - m2[a] + (g.shifted ? g.nc[a] / 2 : 0);
    m3[a] = wrapm(v, g.nc[a]);
  }
  return m3[2] + g.nc[2] * (m3[1] + g.nc[1] * m3[0]);
}

__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}

__device__ __forceinline__ int phase_index(const int* pc, const int* m, int L, int L32) {
  if (L32) {  // the sum fits in 32 bits: a 32-bit remainder
    const unsigned t = (unsigned)(m[0] * pc[0] + m[1] * pc[1] + m[2] * pc[2] + pc[3]);
    return (int)(t % (unsigned)L);
  }
  long long t = (long long)m[0] * pc[0] + (long long)m[1] * pc[1] + (long long)m[2] * pc[2] + pc[3];
  return (int)(t % L);
}

// dynamic shared memory per pair: e2, e3 (b*b), phi, tmp (b^3), P (ntrip), t2/t3 (natoms ints)
__global__ void __launch_bounds__(kBlock) v3_fp64_kernel(V3Args a, int ppb, int ntrip, int natoms) {
  extern __shared__ double2 sm[];
  const Geometry& g = a.geo;
  const int b = g.b, b2 = b * b, b3 = b2 * b;
  const int nt = kBlock / ppb;              // threads per pair
  const int slot = threadIdx.x / nt, lt = threadIdx.x % nt;
  const int row = blockIdx.y;
  const int n1 = a.n1_first + row;
  const int q1 = a.mapinv[n1];
  int q2 = blockIdx.x * ppb + slot;
  const bool live = q2 < g.nkc;
  if (!live) q2 = g.nkc - 1;

  const size_t per_pair = 2 * (size_t)b2 + 2 * (size_t)b3 + ntrip;
  double2* e1 = sm;
  double2* base = sm + b2 + slot * per_pair;
  double2* e2 = base;
  double2* e3 = e2 + b2;
  double2* phi = e3 + b2;
  double2* tmp = phi + b3;
  double2* P = tmp + b3;
  int* tix = reinterpret_cast<int*>(sm + b2 + ppb * per_pair) + slot * 2 * natoms;
  const double2* roots = reinterpret_cast<const double2*>(a.roots);
  const double2* ev = reinterpret_cast<const double2*>(a.evec);

  int m1[3], m2[3], m3[3];
  decompose(g, q1, m1);
  decompose(g, q2, m2);
  const int q3 = idx_mq1mq2(g, m1, m2, m3);

  for (int e = threadIdx.x; e < b2; e += blockDim.x) e1[e] = ev[(size_t)q1 * b2 + e];
  for (int e = lt; e < b2; e += nt) {
    e2[e] = ev[(size_t)q2 * b2 + e];
    e3[e] = ev[(size_t)q3 * b2 + e];
  }
  for (int j = lt; j < natoms; j += nt) {
    tix[j] = phase_index(a.phase_coef + 4 * j, m2, g.L, g.L32);
    tix[natoms + j] = phase_index(a.phase_coef + 4 * j, m3, g.L, g.L32);
  }
  __syncthreads();
  for (int t = lt; t < ntrip; t += nt) {
    int s = tix[a.trip_j[t]] + tix[natoms + a.trip_k[t]];
    if (s >= g.L) s -= g.L;
    P[t] = roots[s];
  }
  __syncthreads();
  // Fourier sum: output channel (a,b,c) with a = 3*i0+al, b = 3*j0+be, c = 3*k0+ga
  const int nat0 = g.nat0;
  for (int o = lt; o < b3; o += nt) {
    int ca = o / b2, cb = (o / b) % b, cc = o % b;
    int i0 = ca / 3, j0 = cb / 3, k0 = cc / 3;
    int comp = (ca % 3) * 9 + (cb % 3) * 3 + (cc % 3);
    int blk = (i0 * nat0 + j0) * nat0 + k0;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = a.blk_off[blk]; t < a.blk_off[blk + 1]; ++t) {
      double w = a.fc3w[27 * (size_t)t + comp];
      double2 p = P[t];
      acc.x = fma(w, p.x, acc.x);
      acc.y = fma(w, p.y, acc.y);
    }
    phi[o] = acc;
  }
  __syncthreads();
  // mode product 1: tmp[l1][b][c] = sum_a e1[a][l1] phi[a][b][c]   (e1[a][l1] at e1[l1*b + a])
  for (int o = lt; o < b3; o += nt) {
    int l1 = o / b2, bc = o % b2;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < b; ++k) {
      double2 e = e1[l1 * b + k], f = phi[k * b2 + bc];
      acc.x = fma(e.x, f.x, fma(-e.y, f.y, acc.x));
      acc.y = fma(e.x, f.y, fma(e.y, f.x, acc.y));
    }
    tmp[o] = acc;
  }
  __syncthreads();
  // mode product 2: phi[l1][l2][c] = sum_b e2[b][l2] tmp[l1][b][c]
  for (int o = lt; o < b3; o += nt) {
    int l1 = o / b2, l2 = (o / b) % b, c = o % b;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < b; ++k) {
      double2 e = e2[l2 * b + k], f = tmp[l1 * b2 + k * b + c];
      acc.x = fma(e.x, f.x, fma(-e.y, f.y, acc.x));
      acc.y = fma(e.x, f.y, fma(e.y, f.x, acc.y));
    }
    phi[o] = acc;
  }
  __syncthreads();
  // mode product 3 and |V3|^2
  const double* w2 = a.w2;
  for (int o = lt; o < b3; o += nt) {
    int l1 = o / b2, l2 = (o / b) % b, l3 = o % b;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < b; ++k) {
      double2 e = e3[l3 * b + k], f = phi[l1 * b2 + l2 * b + k];
      acc.x = fma(e.x, f.x, fma(-e.y, f.y, acc.x));
      acc.y = fma(e.x, f.y, fma(e.y, f.x, acc.y));
    }
    double den = sqrt(8 * sqrt(fabs(w2[(size_t)q1 * b + l1] * w2[(size_t)q2 * b + l2] * w2[(size_t)q3 * b + l3])));
    double v = 0.0;
    if (den != 0.0) {
      double re = acc.x / den * a.const33, im = acc.y / den * a.const33;
      v = re * re + im * im;
    } else if (live) {
      atomicOr(a.err, 2);
    }
    if (live) a.v3sq[((size_t)row * g.nkc + q2) * b3 + o] = v;
  }
}

}  // namespace

cudaError_t launch_v3_fp64(const V3Args& a, cudaStream_t s) {
  const int ntrip = a.ntrip, natoms = a.natoms;
  const int b = a.geo.b;
  const int b2 = b * b, b3 = b2 * b;
  int nt = std::min(kBlock, ((b3 + 31) / 32) * 32);
  int ppb = std::max(1, kBlock / nt);
  while (kBlock % ppb) --ppb;
  size_t per_pair = 2 * (size_t)b2 + 2 * (size_t)b3 + ntrip;
  size_t sm = (b2 + ppb * per_pair) * sizeof(double2) + (size_t)ppb * 2 * natoms * sizeof(int);
  if (sm > 200 * 1024) return cudaErrorInvalidValue;
  if (sm > 48 * 1024) {
    cudaError_t e = raise_smem_limit((const void*)v3_fp64_kernel, sm);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((a.geo.nkc + ppb - 1) / ppb, a.nrows);
  v3_fp64_kernel<<<grid, kBlock, sm, s>>>(a, ppb, ntrip, natoms);
  return cudaGetLastError();
}


}  // namespace ald
