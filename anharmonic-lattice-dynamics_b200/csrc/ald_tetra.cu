// Energy-conserving delta, Bose weighting and band sums.
//
// Replaces, fused:
//   calculate_FGR_mpi2     THERMACOND/sub.f90:7199-7499 (P1smpi, P2smpi)
//   weight_tet / SSORT     THERMACOND/tetrahedron.f90:188-384, 716-738
//   calculate_tauRTA_mpi2  THERMACOND/sub.f90:7953-8194 (P1, P2, Q, Q_N, Q_U)
// and produces R1/R2(q1,q,l1,l2) = sum_l3 P1/P2, the only part of P1/P2
// that CollisionMatrix_mpi (sub.f90:3034) reads, so the (nibz,nkc,b^3)
// arrays of the reference are never stored.
//
// For one IBZ row q1 and bands (l2, l3) -- a "slice" -- the reference gives
// every mesh point w the corner energy
//   process 1: E(w) = -omega(w,l2) + omega(q1+w,l3)   (coalescence)
//   process 2: E(w) =  omega(w,l2) + omega(q1-w,l3)   (decay)
// runs weight_tet(omega1(l1)) over the 6*nkc tetrahedra and adds c/6 * F(w)
// into P(w) at the four corners.  Only tetrahedra whose energy range
// contains omega1 carry weight.  Since omega1(l1) is ascending in l1, the
// bands with weight on a tetrahedron form one contiguous range.  So:
//   1. tet_energy_kernel   E(w) for every slice, as default REAL;
//   2. delta_tet_kernel    a CTA sorts a block of tetrahedra once, queues
//                          the (tetrahedron, l1) pairs with weight in shared
//                          memory, then processes the queue densely: four
//                          corner weights per pair, accumulated into
//                          W(slice, w, l1) with FP64 atomics;
//   3. delta_point_kernel  per mesh point: P = W * |V3|^2 * (2pi)^2/nkc,
//                          Bose factors, sum over l3 in registers -> R1, R2.
// The corner weights reproduce weight_tet's mixed FP32/FP64 arithmetic bit
// for bit (ald_tet.h; this file is compiled with -fmad=false).  The sum of
// the corner contributions into W(w, l1) runs in atomic order, so P1smpi
// agrees with the reference to FP64 rounding, not bitwise.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"
#include "ald_tet.h"

namespace ald {

namespace {

constexpr int kTets = 1024;     // tetrahedra per CTA of delta_tet_kernel
constexpr int kTetThreads = 256;
constexpr int kPointBlock = 128;
constexpr int kMaxBandsTet = 16;  // queue entries pack l1 into 4 bits

__device__ __forceinline__ int wrapm(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}
__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}
__device__ __forceinline__ int compose(const Geometry& g, const int* m) { return m[2] + g.nc[2] * (m[1] + g.nc[1] * m[0]); }
// q1 + w (sign=+1) or q1 - w (sign=-1) on the mesh; `inside` is get_k_info's flag
__device__ __forceinline__ int pm_index(const Geometry& g, const int* m1, const int* mw, int sign, int& inside) {
  int m[3];
  inside = 1;
  for (int a = 0; a < 3; ++a) {
    int v = m1[a] + sign * mw[a] + (g.shifted ? -sign * (g.nc[a] / 2) : 0);
    if (v < 0 || v >= g.nc[a]) inside = 0;
    m[a] = wrapm(v, g.nc[a]);
  }
  return compose(g, m);
}
__device__ __forceinline__ int neg_index(const Geometry& g, const int* mw) {
  int m[3];
  for (int a = 0; a < 3; ++a) m[a] = wrapm(-mw[a], g.nc[a]);
  return compose(g, m);
}
// the reference's acoustic-at-Gamma test: loop indices equal NC/2+1 (sub.f90:7351)
__device__ __forceinline__ bool at_gamma_index(const Geometry& g, const int* m) {
  return m[0] == g.nc[0] / 2 && m[1] == g.nc[1] / 2 && m[2] == g.nc[2] / 2;
}
__device__ __forceinline__ double delta_g(double x, double w) {  // extratools.f90:239
  return exp(-x * x / 2.0 / w / w) / sqrt(2 * PhysConst::pi) / w;
}

// make_kp_reg_tet (tetrahedron.f90:2-142): tetrahedron t = 6*cube + l; cube
// corners pt1..pt8 at offsets (0,0,0) (1,0,0) (0,1,0) (1,1,0) (0,0,1) (1,0,1)
// (0,1,1) (1,1,1); tetrahedra use (1,2,3,6) (2,3,4,6) (1,3,5,6) (3,4,6,8)
// (3,5,6,7) (3,6,7,8)
__constant__ int c_off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                                {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
__constant__ int c_tet[6][4] = {{0, 1, 2, 5}, {1, 2, 3, 5}, {0, 2, 4, 5}, {2, 3, 5, 7}, {2, 4, 5, 6}, {2, 5, 6, 7}};

__device__ __forceinline__ void tet_corners(const Geometry& g, int t, int* c) {
  int m[3];
  decompose(g, t / 6, m);
  const int l = t % 6;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int* o = c_off[c_tet[l][k]];
    int mm[3] = {m[0] + o[0], m[1] + o[1], m[2] + o[2]};
    if (mm[0] == g.nc[0]) mm[0] = 0;
    if (mm[1] == g.nc[1]) mm[1] = 0;
    if (mm[2] == g.nc[2]) mm[2] = 0;
    c[k] = compose(g, mm);
  }
}

// ---------------------------------------------------------------------------
// E[slice][w], slice = ((row*b + l2)*b + l3)*2 + process
__global__ void tet_energy_kernel(Geometry g, int n1_first, int nrows, const int* mapinv, const double* freq,
                                  float* E) {
  const int b = g.b, nkc = g.nkc;
  size_t total = (size_t)nrows * b * b * 2 * nkc;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    int w = (int)(e % nkc);
    size_t t = e / nkc;
    int proc = (int)(t % 2);
    t /= 2;
    int l3 = (int)(t % b);
    t /= b;
    int l2 = (int)(t % b);
    int row = (int)(t / b);
    int q1 = mapinv[n1_first + row];
    int m1[3], mw[3], ins;
    decompose(g, q1, m1);
    decompose(g, w, mw);
    int q3 = pm_index(g, m1, mw, proc == 0 ? 1 : -1, ins);
    double en = proc == 0 ? -freq[(size_t)w * b + l2] + freq[(size_t)q3 * b + l3]
                          : freq[(size_t)w * b + l2] + freq[(size_t)q3 * b + l3];
    E[e] = (float)en;
  }
}

// weight_tet over a block of tetrahedra of one slice; W[slice][w][l1] += c/6
__global__ void __launch_bounds__(kTetThreads) delta_tet_kernel(Geometry g, int n1_first, const int* mapinv,
                                                                const double* freq, const float* __restrict__ E,
                                                                double* W) {
  __shared__ double s_om[kMaxBandsTet];
  __shared__ unsigned short s_queue[kTets * kMaxBandsTet];
  __shared__ int s_qn;
  const int b = g.b, nkc = g.nkc, tid = threadIdx.x, lane = tid & 31;
  const int slice = blockIdx.y;
  const int row = slice / (2 * b * b);
  const int q1 = mapinv[n1_first + row];
  if (tid < b) s_om[tid] = freq[(size_t)q1 * b + tid];
  if (tid == 0) s_qn = 0;
  __syncthreads();
  const float* Es = E + (size_t)slice * nkc;
  double* Ws = W + (size_t)slice * nkc * b;
  const int ntet = 6 * nkc, t0 = blockIdx.x * kTets;
  // phase 1: sort every tetrahedron once and queue (tetrahedron, l1) pairs with weight
  for (int k = 0; k < kTets / kTetThreads; ++k) {
    const int tl = k * kTetThreads + tid, t = t0 + tl;
    int lo = 0, hi = 0;
    if (t < ntet) {
      int c[4];
      tet_corners(g, t, c);
      TetSorted ts = tet_sort(__ldg(Es + c[0]), __ldg(Es + c[1]), __ldg(Es + c[2]), __ldg(Es + c[3]));
      const double E1 = ts.e1, E4 = ts.e4;
      lo = b;
      for (int l = 0; l < b; ++l) {
        double e = s_om[l];
        if (!(e < E1 || e > E4)) {
          lo = min(lo, l);
          hi = l + 1;
        }
      }
    }
    int cnt = hi > lo ? hi - lo : 0;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    int base = 0;
    if (lane == 31) base = atomicAdd(&s_qn, incl);
    base = __shfl_sync(0xffffffffu, base, 31);
    int pos = base + incl - cnt;
    for (int l = lo; l < hi; ++l) s_queue[pos++] = (unsigned short)((tl << 4) | l);
  }
  __syncthreads();
  // phase 2: the queued pairs, four corner weights each
  const int n = s_qn;
  for (int i = tid; i < n; i += kTetThreads) {
    const unsigned v = s_queue[i];
    const int t = t0 + (int)(v >> 4), l = (int)(v & 15u);
    int c[4];
    tet_corners(g, t, c);
    float en[4] = {__ldg(Es + c[0]), __ldg(Es + c[1]), __ldg(Es + c[2]), __ldg(Es + c[3])};
    TetSorted ts = tet_sort(en[0], en[1], en[2], en[3]);
    double cp[4];
    if (!tet_weights4(ts, s_om[l], cp)) continue;
    for (int k = 0; k < 4; ++k) {
      const double cw = cp[tet_pos(en, k)];
      if (cw != 0.0) atomicAdd(Ws + (size_t)c[k] * b + l, cw / 6.0);
    }
  }
}

// per mesh point: P = F * W, Bose factors, sums over l3
template <int B>
__global__ void __launch_bounds__(kPointBlock) delta_point_kernel(CombineArgs a, const double* __restrict__ W) {
  __shared__ double s_om1[B], s_nb1[B];
  const Geometry& g = a.geo;
  const int b = g.b, nkc = g.nkc, b2 = b * b, b3 = b2 * b;
  const int row = blockIdx.z, l2 = blockIdx.y, tid = threadIdx.x;
  const int q1 = a.mapinv[a.n1_first + row];
  if (tid < B) {
    s_om1[tid] = tid < b ? a.freq[(size_t)q1 * b + tid] : 0.0;
    s_nb1[tid] = tid < b ? a.dist[(size_t)q1 * b + tid] : 0.0;
  }
  __syncthreads();
  const int w = blockIdx.x * blockDim.x + tid;
  if (w >= nkc) return;
  int m1[3], mw[3];
  decompose(g, q1, m1);
  decompose(g, w, mw);
  int ins1, ins2;
  const int q3p = pm_index(g, m1, mw, 1, ins1);   // q1 + w
  const int q3m = pm_index(g, m1, mw, -1, ins2);  // q1 - w
  const int wneg = neg_index(g, mw);
  int m3p[3], m3m[3];
  decompose(g, q3p, m3p);
  decompose(g, q3m, m3m);
  const bool w_gamma = at_gamma_index(g, mw);
  const bool p_gamma = at_gamma_index(g, m3p), m_gamma = at_gamma_index(g, m3m);
  const double fnorm = (2 * PhysConst::pi) * (2 * PhysConst::pi) / nkc;
  const double n2 = a.dist[(size_t)w * b + l2];
  const double* v3 = a.v3sq + (size_t)row * nkc * b3;
  double R1[B], R2[B];
#pragma unroll
  for (int l = 0; l < B; ++l) R1[l] = R2[l] = 0.0;
  for (int l3 = 0; l3 < b; ++l3) {
#pragma unroll
    for (int proc = 0; proc < 2; ++proc) {
      const int q3 = proc == 0 ? q3p : q3m;
      const size_t slice = (((size_t)row * b + l2) * b + l3) * 2 + proc;
      const bool zero = (l2 < 3 && w_gamma) || (l3 < 3 && (proc == 0 ? p_gamma : m_gamma));
      const int src = proc == 0 ? w : wneg;
      const double n3 = a.dist[(size_t)q3 * b + l3];
      const double w2 = a.freq[(size_t)w * b + l2], w3 = a.freq[(size_t)q3 * b + l3];
      double* Ps = proc == 0 ? a.P1s : a.P2s;
      double* Pb = proc == 0 ? a.P1 : a.P2;
#pragma unroll
      for (int l = 0; l < B; ++l) {
        if (l >= b) continue;
        double wl;
        if (a.gauss) wl = delta_g(proc == 0 ? s_om1[l] + w2 - w3 : s_om1[l] - w2 - w3, a.sigma);
        else wl = W[(slice * nkc + w) * b + l];
        double ps = 0.0;
        if (wl != 0.0 && !zero) ps = wl * (v3[(size_t)src * b3 + (l * b + l2) * b + l3] * fnorm);
        const double nb1 = s_nb1[l];
        const double Fb = proc == 0 ? nb1 * n2 * (n3 + 1) : nb1 * (n2 + 1) * (n3 + 1);
        const double p = ps * Fb;
        if (proc == 0) R1[l] += p;
        else R2[l] += p;
        if (Ps || Pb) {
          size_t o5 = (((size_t)row * nkc + w) * b + l) * b2 + l2 * b + l3;
          if (Ps) Ps[o5] = ps;
          if (Pb) Pb[o5] = p;
        }
      }
    }
  }
#pragma unroll
  for (int l = 0; l < B; ++l) {
    if (l >= b) continue;
    size_t ri = (((size_t)row * nkc + w) * b + l) * b + l2;
    a.R1[ri] = R1[l];
    a.R2[ri] = R2[l];
  }
}

// Q, Q_N, Q_U from the band sums: Q = sum_{w,l2} R1 + R2/2, split by the
// normal/umklapp flag of q1+w (process 1) and q1-w (process 2)
__global__ void q_from_r_kernel(Geometry g, int n1_first, const int* mapinv, const double* R1, const double* R2,
                                double* Q, double* QN, double* QU) {
  __shared__ double red[3][32];
  const int b = g.b, nkc = g.nkc;
  const int row = blockIdx.x, l1 = blockIdx.y;
  const int q1 = mapinv[n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  double s = 0, sn = 0, su = 0;
  for (int w = threadIdx.x; w < nkc; w += blockDim.x) {
    int mw[3], i1, i2;
    decompose(g, w, mw);
    pm_index(g, m1, mw, 1, i1);
    pm_index(g, m1, mw, -1, i2);
    double r1 = 0, r2 = 0;
    const size_t base = (((size_t)row * nkc + w) * b + l1) * b;
    for (int l2 = 0; l2 < b; ++l2) {
      r1 += R1[base + l2];
      r2 += R2[base + l2];
    }
    s += r1 + 0.5 * r2;
    sn += (i1 ? r1 : 0.0) + (i2 ? 0.5 * r2 : 0.0);
    su += (i1 ? 0.0 : r1) + (i2 ? 0.0 : 0.5 * r2);
  }
  double v[3] = {s, sn, su};
  for (int k = 0; k < 3; ++k) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[threadIdx.x][i];
    double* out = threadIdx.x == 0 ? Q : (threadIdx.x == 1 ? QN : QU);
    out[(size_t)(n1_first + row) * b + l1] = t;
  }
}

}  // namespace

size_t combine_scratch_bytes(const Geometry& geo, int nrows, int gauss) {
  if (gauss) return 0;
  size_t nslice = (size_t)nrows * geo.b * geo.b * 2;
  size_t ebytes = (nslice * geo.nkc * sizeof(float) + 255) / 256 * 256;
  return ebytes + nslice * geo.nkc * geo.b * sizeof(double);
}

cudaError_t launch_combine(const CombineArgs& a, void* scratch, cudaStream_t s) {
  const Geometry& g = a.geo;
  if (g.b > kMaxBandsTet) return cudaErrorInvalidValue;
  const double* W = nullptr;
  if (!a.gauss) {
    size_t nslice = (size_t)a.nrows * g.b * g.b * 2;
    float* E = static_cast<float*>(scratch);
    size_t ebytes = (nslice * g.nkc * sizeof(float) + 255) / 256 * 256;
    double* Wd = reinterpret_cast<double*>(static_cast<char*>(scratch) + ebytes);
    size_t total = nslice * g.nkc;
    int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 64);
    tet_energy_kernel<<<blocks, 256, 0, s>>>(g, a.n1_first, a.nrows, a.mapinv, a.freq, E);
    cudaError_t e = cudaMemsetAsync(Wd, 0, nslice * g.nkc * g.b * sizeof(double), s);
    if (e != cudaSuccess) return e;
    dim3 tg((6 * g.nkc + kTets - 1) / kTets, (unsigned)nslice);
    delta_tet_kernel<<<tg, kTetThreads, 0, s>>>(g, a.n1_first, a.mapinv, a.freq, E, Wd);
    W = Wd;
  }
  dim3 grid((g.nkc + kPointBlock - 1) / kPointBlock, g.b, a.nrows);
  if (g.b <= 3)
    delta_point_kernel<3><<<grid, kPointBlock, 0, s>>>(a, W);
  else if (g.b <= 6)
    delta_point_kernel<6><<<grid, kPointBlock, 0, s>>>(a, W);
  else if (g.b <= 12)
    delta_point_kernel<12><<<grid, kPointBlock, 0, s>>>(a, W);
  else if (g.b <= 16)
    delta_point_kernel<16><<<grid, kPointBlock, 0, s>>>(a, W);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_q_from_r(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* R1,
                            const double* R2, double* Q, double* QN, double* QU, int nibz, cudaStream_t s) {
  (void)nibz;
  dim3 grid(nrows, geo.b);
  q_from_r_kernel<<<grid, 256, 0, s>>>(geo, n1_first, mapinv, R1, R2, Q, QN, QU);
  return cudaGetLastError();
}

}  // namespace ald
