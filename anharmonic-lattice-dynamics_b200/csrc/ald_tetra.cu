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
#include <type_traits>

#include "ald_internal.h"
#include "ald_tet.h"

namespace ald {

namespace {

constexpr int kTets = 1024;     // tetrahedra per CTA of delta_tet_kernel
constexpr int kTetThreads = 256;
constexpr int kPointBlock = 128;
constexpr int kMaxBandsTet = 16;  // queue entries pack l1 into 4 bits

__device__ __forceinline__ void decompose(const Geometry& g, int n, int* m) {
  m[0] = n / (g.nc[1] * g.nc[2]);
  m[1] = (n / g.nc[2]) % g.nc[1];
  m[2] = n % g.nc[2];
}
__device__ __forceinline__ int compose(const Geometry& g, const int* m) { return m[2] + g.nc[2] * (m[1] + g.nc[1] * m[0]); }
// v mod n for v in [-n, 2n), by compares
__device__ __forceinline__ int wrap2(int v, int n) {
  v += v < 0 ? n : 0;
  return v >= n ? v - n : v;
}
// q1 + w (sign=+1) or q1 - w (sign=-1) on the mesh, and its mesh integers m;
// `inside` is get_k_info's flag.  m1 + -mw -+ nc/2 lies in [-nc, 2nc).
__device__ __forceinline__ int pm_index_m(const Geometry& g, const int* m1, const int* mw, int sign, int& inside,
                                          int* m) {
  inside = 1;
  for (int a = 0; a < 3; ++a) {
    int v = m1[a] + sign * mw[a] + (g.shifted ? -sign * (g.nc[a] / 2) : 0);
    if (v < 0 || v >= g.nc[a]) inside = 0;
    m[a] = wrap2(v, g.nc[a]);
  }
  return compose(g, m);
}
__device__ __forceinline__ int pm_index(const Geometry& g, const int* m1, const int* mw, int sign, int& inside) {
  int m[3];
  return pm_index_m(g, m1, mw, sign, inside, m);
}
__device__ __forceinline__ int neg_index(const Geometry& g, const int* mw) {
  int m[3];
  for (int a = 0; a < 3; ++a) m[a] = wrap2(-mw[a], g.nc[a]);
  return compose(g, m);
}
// the reference's acoustic-at-Gamma test: loop indices equal NC/2+1 (sub.f90:7351)
__device__ __forceinline__ bool at_gamma_index(const Geometry& g, const int* m) {
  return m[0] == g.nc[0] / 2 && m[1] == g.nc[1] / 2 && m[2] == g.nc[2] / 2;
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

// per mesh point: P = F * W, Bose factors, sums over l3.  Two thread maps:
//   TILE: a CTA takes kPointBlock / b consecutive mesh points w of one IBZ
//         row and all b bands l2 (thread = (w, l2), l2 fastest), so the loads
//         of omega, n at (w, l2) and the R1/R2 tile [w][l1][l2] it writes
//         (staged in shared memory) are contiguous;
//   else: a CTA takes kPointBlock consecutive w of one row and one l2
//         (blockIdx.z), so the |V3|^2 loads of a warp are one run of q2.
// Measured on B200: TILE for the FP64 Gaussian (exp-bound), the other map
// for the FP32 one (load-latency bound).
// The Gaussian is delta_g of extratools.f90:239, exp(-x^2/2/w/w)/sqrt(2 pi)/w,
// with the constant factors formed once (FP64 rounding, not bitwise), and
// skipped where exp underflows to zero.
template <int B, bool F32W, bool TILE>
__global__ void __launch_bounds__(kPointBlock) delta_point_kernel(CombineArgs a, const double* __restrict__ W) {
  __shared__ double s_om1[B], s_nb1[B];
  __shared__ double s_r[2][TILE ? kPointBlock * B : 1];  // R1, R2 tiles: [w local][l1][l2]
  const Geometry& g = a.geo;
  const int b = g.b, nkc = g.nkc, b2 = b * b, b3 = b2 * b;
  const int row = blockIdx.y, tid = threadIdx.x;
  const int nw = TILE ? kPointBlock / b : kPointBlock;  // mesh points per CTA
  const int wl = TILE ? tid / b : tid, l2 = TILE ? tid % b : (int)blockIdx.z;
  const int w0 = blockIdx.x * nw;
  const int w = w0 + wl;
  const bool ok = wl < nw && w < nkc;
  const int q1 = a.mapinv[a.n1_first + row];
  if (tid < B) {
    s_om1[tid] = tid < b ? a.freq[(size_t)q1 * b + tid] : 0.0;
    s_nb1[tid] = tid < b ? a.dist[(size_t)q1 * b + tid] : 0.0;
  }
  __syncthreads();
  double R1[B], R2[B];
#pragma unroll
  for (int l = 0; l < B; ++l) R1[l] = R2[l] = 0.0;
  if (ok) {
    int m1[3], mw[3];
    decompose(g, q1, m1);
    decompose(g, w, mw);
    int ins1, ins2;
    int m3p[3], m3m[3];
    const int q3p = pm_index_m(g, m1, mw, 1, ins1, m3p);   // q1 + w
    const int q3m = pm_index_m(g, m1, mw, -1, ins2, m3m);  // q1 - w
    const int wneg = neg_index(g, mw);
    const bool w_gamma = at_gamma_index(g, mw);
    const bool p_gamma = at_gamma_index(g, m3p), m_gamma = at_gamma_index(g, m3m);
    const double fnorm = (2 * PhysConst::pi) * (2 * PhysConst::pi) / nkc;
    const double n2 = a.dist[(size_t)w * b + l2];
    const double w2 = a.freq[(size_t)w * b + l2];
    const double* v3 = a.v3sq + (size_t)row * nkc * b3;
    // |V3|^2 strides of (q, l1, l2, l3) in the chunk's layout
    const size_t sq = a.v3_layout == 1 ? 1 : (size_t)b3, s1 = a.v3_layout == 1 ? (size_t)nkc : (size_t)b2;
    const size_t s2 = a.v3_layout == 1 ? (size_t)b2 * nkc : (size_t)b, s3 = a.v3_layout == 1 ? (size_t)b * nkc : 1;
    // Gaussian factors: FP64 (exp underflows to 0 beyond 746) and FP32 (beyond 104)
    const double gc1 = 0.5 / (a.sigma * a.sigma), gc2 = 1.0 / (sqrt(2 * PhysConst::pi) * a.sigma);
    const float fc1 = (float)gc1, fc2 = (float)gc2;
    for (int l3 = 0; l3 < b; ++l3) {
#pragma unroll
      for (int proc = 0; proc < 2; ++proc) {
        const int q3 = proc == 0 ? q3p : q3m;
        const size_t slice = (((size_t)row * b + l2) * b + l3) * 2 + proc;
        const bool zero = (l2 < 3 && w_gamma) || (l3 < 3 && (proc == 0 ? p_gamma : m_gamma));
        const int src = proc == 0 ? w : wneg;
        const double n3 = a.dist[(size_t)q3 * b + l3];
        const double w3 = a.freq[(size_t)q3 * b + l3];
        double* Ps = proc == 0 ? a.P1s : a.P2s;
        double* Pb = proc == 0 ? a.P1 : a.P2;
#pragma unroll
        for (int l = 0; l < B; ++l) {
          if (l >= b) continue;
          double wl_ = 0.0;
          if (a.gauss) {
            const double x = proc == 0 ? s_om1[l] + w2 - w3 : s_om1[l] - w2 - w3;
            if constexpr (F32W) {
              const float xf = (float)x, arg = xf * xf * fc1;
              if (arg < 104.0f) wl_ = (double)(expf(-arg) * fc2);
            } else {
              const double arg = x * x * gc1;
              if (arg < 746.0) wl_ = exp(-arg) * gc2;
            }
          } else {
            wl_ = W[(slice * nkc + w) * b + l];
          }
          double ps = 0.0;
          if (wl_ != 0.0 && !zero) ps = wl_ * (v3[(size_t)src * sq + l * s1 + l2 * s2 + l3 * s3] * fnorm);
          const double nb1 = s_nb1[l];
          const double Fb = proc == 0 ? nb1 * n2 * (n3 + 1) : nb1 * (n2 + 1) * (n3 + 1);
          const double p = ps * Fb;
          if (proc == 0) R1[l] += p;
          else R2[l] += p;
          double* Rpm = proc == 0 ? a.R1p : a.R2p;
          if (Rpm && p != 0.0) atomicAdd(Rpm + (((size_t)row * nkc + w) * b + l) * b + l3, p);
          if (Ps || Pb) {
            size_t o5 = (((size_t)row * nkc + w) * b + l) * b2 + l2 * b + l3;
            if (Ps) Ps[o5] = ps;
            if (Pb) Pb[o5] = p;
          }
        }
      }
    }
  }
  if constexpr (!TILE) {
    if (ok) {
#pragma unroll
      for (int l = 0; l < B; ++l) {
        if (l >= b) continue;
        const size_t ri = (((size_t)row * nkc + w) * b + l) * b + l2;
        a.R1[ri] = R1[l];
        a.R2[ri] = R2[l];
      }
    }
    return;
  }
  if (wl < nw) {
#pragma unroll
    for (int l = 0; l < B; ++l) {
      if (l >= b) continue;
      s_r[0][(wl * b + l) * b + l2] = R1[l];
      s_r[1][(wl * b + l) * b + l2] = R2[l];
    }
  }
  __syncthreads();
  // the tile is one contiguous run of R1/R2: rows w0 .. w0 + nv - 1
  const int nv = min(nw, nkc - w0);
  const size_t base = ((size_t)row * nkc + w0) * b2;
  for (int i = tid; i < nv * b2; i += blockDim.x) {
    a.R1[base + i] = s_r[0][i];
    a.R2[base + i] = s_r[1][i];
  }
}

// The FP32 Gaussian of the mixed pipeline with both processes per thread:
// a thread takes mesh point q and band l2 and reads each |V3|^2(q) once for
// process 1 at w = q (q3 = q1 + q) and for process 2 at w = -q, whose q3 =
// q1 - w is the same point and whose |V3|^2 source is q again.  It writes
// R1 at w = q and R2 at w = -q (the map q -> -q is a permutation of the
// mesh).  P1s/P2s/P1/P2 are not produced (pipeline only).
template <int B>
__global__ void __launch_bounds__(kPointBlock) delta_point_pair_kernel(CombineArgs a) {
  __shared__ double s_om1[B], s_nb1[B];
  const Geometry& g = a.geo;
  const int b = g.b, nkc = g.nkc, b2 = b * b, b3 = b2 * b;
  const int row = blockIdx.y, l2 = blockIdx.z, tid = threadIdx.x;
  const int q1 = a.mapinv[a.n1_first + row];
  if (tid < B) {
    s_om1[tid] = tid < b ? a.freq[(size_t)q1 * b + tid] : 0.0;
    s_nb1[tid] = tid < b ? a.dist[(size_t)q1 * b + tid] : 0.0;
  }
  __syncthreads();
  const int q = blockIdx.x * blockDim.x + tid;
  if (q >= nkc) return;  // no barrier below
  int m1[3], mq[3], m3[3], mn[3];
  decompose(g, q1, m1);
  decompose(g, q, mq);
  int ins;
  const int q3 = pm_index_m(g, m1, mq, 1, ins, m3);  // q1 + q = q1 - (-q)
  for (int x = 0; x < 3; ++x) mn[x] = wrap2(-mq[x], g.nc[x]);
  const int wn = compose(g, mn);  // -q
  const bool gq = at_gamma_index(g, mq), gn = at_gamma_index(g, mn), g3 = at_gamma_index(g, m3);
  const double fnorm = (2 * PhysConst::pi) * (2 * PhysConst::pi) / nkc;
  const double n2a = a.dist[(size_t)q * b + l2], w2a = a.freq[(size_t)q * b + l2];
  const double n2b = a.dist[(size_t)wn * b + l2], w2b = a.freq[(size_t)wn * b + l2];
  const double* v3 = a.v3sq + (size_t)row * nkc * b3;
  const size_t sq = a.v3_layout == 1 ? 1 : (size_t)b3, s1 = a.v3_layout == 1 ? (size_t)nkc : (size_t)b2;
  const size_t s2 = a.v3_layout == 1 ? (size_t)b2 * nkc : (size_t)b, s3 = a.v3_layout == 1 ? (size_t)b * nkc : 1;
  const float fc1 = (float)(0.5 / (a.sigma * a.sigma)), fc2 = (float)(1.0 / (sqrt(2 * PhysConst::pi) * a.sigma));
  double R1[B], R2[B];
#pragma unroll
  for (int l = 0; l < B; ++l) R1[l] = R2[l] = 0.0;
  for (int l3 = 0; l3 < b; ++l3) {
    const double n3 = a.dist[(size_t)q3 * b + l3], w3 = a.freq[(size_t)q3 * b + l3];
    const bool zero1 = (l2 < 3 && gq) || (l3 < 3 && g3);
    const bool zero2 = (l2 < 3 && gn) || (l3 < 3 && g3);
#pragma unroll
    for (int l = 0; l < B; ++l) {
      if (l >= b) continue;
      const double v = v3[(size_t)q * sq + l * s1 + l2 * s2 + l3 * s3] * fnorm;
      const double nb1 = s_nb1[l];
      {  // process 1 at w = q
        const float xf = (float)(s_om1[l] + w2a - w3), arg = xf * xf * fc1;
        if (arg < 104.0f && !zero1) {
          const double p = ((double)(expf(-arg) * fc2) * v) * (nb1 * n2a * (n3 + 1));
          R1[l] += p;
          if (a.R1p && p != 0.0) atomicAdd(a.R1p + (((size_t)row * nkc + q) * b + l) * b + l3, p);
        }
      }
      {  // process 2 at w = -q
        const float xf = (float)(s_om1[l] - w2b - w3), arg = xf * xf * fc1;
        if (arg < 104.0f && !zero2) {
          const double p = ((double)(expf(-arg) * fc2) * v) * (nb1 * (n2b + 1) * (n3 + 1));
          R2[l] += p;
          if (a.R2p && p != 0.0) atomicAdd(a.R2p + (((size_t)row * nkc + wn) * b + l) * b + l3, p);
        }
      }
    }
  }
#pragma unroll
  for (int l = 0; l < B; ++l) {
    if (l >= b) continue;
    a.R1[(((size_t)row * nkc + q) * b + l) * b + l2] = R1[l];
    a.R2[(((size_t)row * nkc + wn) * b + l) * b + l2] = R2[l];
  }
}

// Q, Q_N, Q_U from the band sums: Q = sum_{w,l2} R1 + R2/2, split by the
// normal/umklapp flag of q1+w (process 1) and q1-w (process 2)
__global__ void __launch_bounds__(256) q_from_r_kernel(Geometry g, int n1_first, const int* mapinv,
                                                       const double* R1, const double* R2, double* Q, double* QN,
                                                       double* QU) {
  // one CTA per IBZ row; thread = (w slot, l1) with l1 fastest and a block
  // size that is a multiple of b, so each thread keeps one l1 and a warp
  // reads consecutive (w, l1) rows of b doubles: coalesced
  __shared__ double red[3][256];
  const int b = g.b, nkc = g.nkc;
  const int row = blockIdx.x, tid = threadIdx.x;
  const int nslot = blockDim.x / b, l1 = tid % b, slot = tid / b;
  const int q1 = mapinv[n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  double s = 0, sn = 0, su = 0;
  for (int w = slot; w < nkc; w += nslot) {
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
  red[0][tid] = s;
  red[1][tid] = sn;
  red[2][tid] = su;
  __syncthreads();
  if (tid < 3 * b) {  // thread (k, l1): the slots of one l1 in order
    const int k = tid / b, l = tid % b;
    double t = 0;
    for (int i = 0; i < nslot; ++i) t += red[k][i * b + l];
    double* out = k == 0 ? Q : (k == 1 ? QN : QU);
    out[(size_t)(n1_first + row) * b + l] = t;
  }
}

// ---------------------------------------------------------------------------
// Fused tetrahedron delta for the pipeline: the weights of every
// (tetrahedron, l1) pair go straight into R1/R2 -- no corner-energy or weight
// array in HBM.  A CTA owns one IBZ row, one process and one band l2, and a
// block of mesh cells: plane i, rows j0 .. j0+R-1, all k (thread = cell).  The
// corners of those cells form a window of 2 x (R+1) x N2 mesh points.
// Once per CTA the window's indices and flags are staged in shared memory;
// then per l3 (one slice of the reference's loops):
//   1. per window point: E = -+omega(w,l2) + omega(q1+-w,l3) as default REAL,
//      G = n2 (n3+1) [process 1] or (n2+1)(n3+1) [process 2], G = 0 where the
//      reference zeroes acoustic modes at Gamma (sub.f90:7351-7356, 7412-7417);
//   2. per cell: min/max of its 8 corner energies; cells whose range holds
//      no band energy omega1(l1) are skipped, else its 6 tetrahedra are
//      sorted once and each one whose range may hold an omega1(l1) is stored
//      as a record (the window point at each sorted position; the energies
//      are read back from the window) with its (record, l1) pairs queued;
//   3. per queued pair: weight_tet's four corner weights c (bitwise, ald_tet.h)
//      and R(row, w, l1, l2) += c/6 (2pi)^2/nkc |V3|^2 n1 G for each corner
//      (FP64 atomics in L2; FP64 atomics on shared memory would be CAS loops).
//      |V3|^2(src(w), l1, l2, l3) is gathered where needed; in the slice-major
//      layout the corners of one tetrahedron share sectors.
// MODE 0: the sums run in atomic order (FP64 rounding, not bitwise, against
// the reference's P1/P2 summed over l3).  MODE 1 and 2 (the deterministic
// option) run the kernel twice: first each entry's largest term (its FP64
// bits, atomicMax: every term is >= 0 and the bit order of nonnegative
// doubles is their numeric order), then every term as a 64-bit integer,
// round(term * 2^(62 - e)) with 2^e >= kDetTerms(b) x the largest term, added
// with integer atomics: integer sums do not depend on their order.  At most
// kDetTerms(b) = 24 b terms reach an entry (24 tetrahedron corners at a
// point, b slices l3 -- or b bands l2 for the marginals), so the sum stays
// below 2^63 and each rounding is at most 2^-63 x 24 b of the entry.
// launch_delta_finalize turns the integers back into doubles.
// corners of make_kp_reg_tet's six tetrahedra (c = o0 + 2 o1 + 4 o2), 3 bits
// each, tetrahedra 0..4 in one word; tetrahedron 5 is (2, 5, 6, 7)
constexpr unsigned long long kTetCornerCode =
    (0ull | 1ull << 3 | 2ull << 6 | 5ull << 9) | (1ull | 2ull << 3 | 3ull << 6 | 5ull << 9) << 12 |
    (0ull | 2ull << 3 | 4ull << 6 | 5ull << 9) << 24 | (2ull | 3ull << 3 | 5ull << 6 | 7ull << 9) << 36 |
    (2ull | 4ull << 3 | 5ull << 6 | 6ull << 9) << 48;
constexpr unsigned kTet5Code = 2u | 5u << 3 | 6u << 6 | 7u << 9;
__device__ __forceinline__ unsigned tet_code(int t) {
  return t < 5 ? (unsigned)(kTetCornerCode >> (12 * t)) & 0xfffu : kTet5Code;
}

constexpr int kFusedThreads = 128;

__host__ __device__ constexpr int kDetTerms(int b) { return 24 * b; }
// exponent e of the fixed-point scale of an entry whose largest term has the
// bits m: 2^e >= kDetTerms(b) * largest term
__device__ __forceinline__ int det_exponent(unsigned long long m, int b) {
  int e;
  frexp(__longlong_as_double((long long)m) * (double)kDetTerms(b), &e);
  return e;
}
__device__ __forceinline__ unsigned long long det_fixed(double v, unsigned long long m, int b) {
  return (unsigned long long)llrint(ldexp(v, 62 - det_exponent(m, b)));
}

struct FusedShape {
  int R, nbj, NW, maxrec;
  size_t smem;
};

__host__ __device__ inline FusedShape fused_shape(const Geometry& g) {
  FusedShape f;
  const int N1 = g.nc[1], N2 = g.nc[2];
  f.R = kFusedThreads / N2;
  if (f.R < 1) f.R = 1;
  if (f.R > N1) f.R = N1;
  f.nbj = (N1 + f.R - 1) / f.R;
  f.NW = 2 * (f.R + 1) * N2;
  f.maxrec = 6 * f.R * N2;
  const size_t nw2 = (size_t)(f.NW + (f.NW & 1));
  // doubles: G; ushort4 records; ints: w, src, q3; floats: E; bytes: flags; ushorts: queue
  // doubles: G, omega(w, l2), n(w, l2); ushort4 records; ints: w, src, q3;
  // floats: E; bytes: flags; ushorts: queue
  f.smem = nw2 * 8 * 3 + (size_t)f.maxrec * 8 + (size_t)f.NW * 3 * 4 + (size_t)f.NW * 4 + (size_t)((f.NW + 3) & ~3) +
           (size_t)f.maxrec * g.b * 2;
  return f;
}

template <int B, bool F32W, class VT, int MODE>
__device__ __forceinline__ void delta_fused_body(const CombineArgs& a, const VT* __restrict__ v3sq) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double s_om[B], s_nb1[B];
  __shared__ int s_nrec, s_nq;
  __shared__ unsigned short s_lp[kFusedThreads][8];              // window point of each cell corner
  __shared__ unsigned char s_hit[kFusedThreads / 32][32];      // the warp's cells that passed, by lane
  const Geometry& g = a.geo;
  const FusedShape F = fused_shape(g);
  const int R = F.R, NW = F.NW, maxrec = F.maxrec;
  const int N0 = g.nc[0], N1 = g.nc[1], N2 = g.nc[2], nkc = g.nkc, b = g.b;
  const int tid = threadIdx.x, lane = tid & 31;
  const int row = blockIdx.y, proc = blockIdx.z % 2, l2 = blockIdx.z / 2;
  const int pi = blockIdx.x / F.nbj, j0 = (blockIdx.x % F.nbj) * R;
  // shared layout
  const int nw2 = NW + (NW & 1);
  double* s_G = reinterpret_cast<double*>(smraw);
  double* s_fw = s_G + nw2;  // omega(w, l2) and n(w, l2): the same for every slice
  double* s_n2 = s_fw + nw2;
  ushort4* s_recp = reinterpret_cast<ushort4*>(s_n2 + nw2);
  int* s_w = reinterpret_cast<int*>(s_recp + maxrec);
  int* s_src = s_w + NW;
  int* s_q3 = s_src + NW;
  float* s_E = reinterpret_cast<float*>(s_q3 + NW);
  unsigned char* s_fl = reinterpret_cast<unsigned char*>(s_E + NW);
  unsigned short* s_queue = reinterpret_cast<unsigned short*>(s_fl + ((NW + 3) & ~3));

  const int q1 = a.mapinv[a.n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  if (tid < b) {
    s_om[tid] = a.freq[(size_t)q1 * b + tid];
    s_nb1[tid] = a.dist[(size_t)q1 * b + tid];
  }
  // conservative FP32 bounds of omega1 for the range tests (unused bands never count)
  float omlo[B], omhi[B];
#pragma unroll
  for (int l1 = 0; l1 < B; ++l1) {
    const double om = l1 < b ? a.freq[(size_t)q1 * b + l1] : 0.0;
    omlo[l1] = l1 < b ? __double2float_rd(om) : 3.4e38f;
    omhi[l1] = l1 < b ? __double2float_ru(om) : 3.4e38f;
  }
  // window points: global index, q3 = q1 +- w, source of |V3|^2, Gamma flags,
  // omega and n of band l2
  for (int p = tid; p < NW; p += blockDim.x) {
    const int k = p % N2, t = p / N2, dj = t % (R + 1), di = t / (R + 1);
    int mw[3] = {(pi + di) % N0, (j0 + dj) % N1, k};
    const int w = compose(g, mw);
    int ins;
    int m3[3];
    const int q3 = pm_index_m(g, m1, mw, proc == 0 ? 1 : -1, ins, m3);
    s_w[p] = w;
    s_q3[p] = q3;
    s_src[p] = proc == 0 ? w : neg_index(g, mw);
    s_fl[p] = (unsigned char)((at_gamma_index(g, mw) ? 1 : 0) | (at_gamma_index(g, m3) ? 2 : 0));
    s_fw[p] = a.freq[(size_t)w * b + l2];
    s_n2[p] = a.dist[(size_t)w * b + l2];
  }
  // (2pi)^2/nkc and the 1/6 of the corner weights in one factor
  const double fnorm6 = (2 * PhysConst::pi) * (2 * PhysConst::pi) / nkc / 6.0;
  double* Rp = proc == 0 ? a.R1 : a.R2;
  double* Rpp = proc == 0 ? a.R1p : a.R2p;  // band marginal over l2 (optional)
  unsigned long long* Mp = proc == 0 ? a.M1 : a.M2;  // largest terms (MODE 1, 2)
  unsigned long long* Mpp = proc == 0 ? a.M1p : a.M2p;
  // |V3|^2 strides of (q, l1, l2, l3) in the chunk's layout
  size_t sq, s1, s2, s3;
  if (a.v3_layout == 1) {
    sq = 1;
    s1 = nkc;
    s3 = (size_t)b * nkc;
    s2 = (size_t)b * b * nkc;
  } else {
    s3 = 1;
    s2 = b;
    s1 = (size_t)b * b;
    sq = (size_t)b * b * b;
  }
  const VT* v3row = v3sq + (size_t)row * nkc * b * b * b;
  // this thread's cell and its corners in the window
  const int cdj = tid / N2, ck = tid % N2;
  const bool cell_ok = tid < R * N2 && j0 + cdj < N1;
  int lp[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int o0 = c & 1, o1 = (c >> 1) & 1, o2 = (c >> 2) & 1;  // c_off order
    const int kk = ck + o2 == N2 ? 0 : ck + o2;
    lp[c] = cell_ok ? (o0 * (R + 1) + cdj + o1) * N2 + kk : 0;
    s_lp[tid][c] = (unsigned short)lp[c];
  }
  // The energies of slice l3, -+omega(w,l2) + omega(q3,l3), lie within the
  // bands' ranges over the mesh; when that range misses every omega1 of the
  // row (with a margin far above the FP32 rounding of E) no tetrahedron of the
  // slice has weight and the slice is skipped (the same for every thread).
  unsigned live = 0xffffffffu;
  if (a.brange) {
    __syncthreads();  // s_om
    double o1min = s_om[0], o1max = s_om[0];
    for (int l = 1; l < b; ++l) {
      o1min = fmin(o1min, s_om[l]);
      o1max = fmax(o1max, s_om[l]);
    }
    for (int l3 = 0; l3 < b; ++l3) {
      const double lo2 = a.brange[l2], hi2 = a.brange[b + l2], lo3 = a.brange[l3], hi3 = a.brange[b + l3];
      const double emin = proc == 0 ? lo3 - hi2 : lo2 + lo3, emax = proc == 0 ? hi3 - lo2 : hi2 + hi3;
      const double tol = 1e-5 * (fabs(hi2) + fabs(hi3)) + 1e-10;
      if (emax + tol < o1min || emin - tol > o1max) live &= ~(1u << l3);
    }
  }
  for (int l3 = 0; l3 < b; ++l3) {
    if (!((live >> l3) & 1u)) continue;
    __syncthreads();  // window staged / previous slice done
    if (tid == 0) {
      s_nrec = 0;
      s_nq = 0;
    }
    for (int p = tid; p < NW; p += blockDim.x) {
      const int q3 = s_q3[p];
      const double fw = s_fw[p], f3 = a.freq[(size_t)q3 * b + l3];
      s_E[p] = (float)(proc == 0 ? -fw + f3 : fw + f3);
      const double n2 = s_n2[p], n3 = a.dist[(size_t)q3 * b + l3];
      const bool zero = (l2 < 3 && (s_fl[p] & 1)) || (l3 < 3 && (s_fl[p] & 2));
      s_G[p] = zero ? 0.0 : (proc == 0 ? n2 * (n3 + 1) : (n2 + 1) * (n3 + 1));
    }
    __syncthreads();
    // phase 1: cells -> tetrahedron records and (record, l1) pairs
    // (make_kp_reg_tet's six tetrahedra of a cell, as corner numbers, tet_code).
    // Bands lo .. hi-1 may carry weight on a tetrahedron with energies in
    // [mn, mx]: omega1 is ascending, so lo and hi are counts; the exact test
    // is tet_weights4's in phase 2.
    float ec[8];
    float emin = 3.4e38f, emax = -3.4e38f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      ec[c] = s_E[lp[c]];
      emin = fminf(emin, ec[c]);
      emax = fmaxf(emax, ec[c]);
    }
    int clo = 0, chi = 0;
#pragma unroll
    for (int l1 = 0; l1 < B; ++l1) {
      clo += omhi[l1] < emin;
      chi += omlo[l1] <= emax;
    }
    const bool any = cell_ok && chi > clo;
    if constexpr (F32W) {
      // mixed: the six tetrahedra of every cell of a warp that has a cell in
      // range (measured faster here than the compacted form below)
      constexpr int kTetOf[6][4] = {{0, 1, 2, 5}, {1, 2, 3, 5}, {0, 2, 4, 5}, {2, 3, 5, 7}, {2, 4, 5, 6}, {2, 5, 6, 7}};
      if (__any_sync(0xffffffffu, any)) {
        // band range of each tetrahedron, then one warp scan of the packed
        // (queue entries << 16 | records) counts of the six, and one slot
        // reservation per warp for both lists
        int tlo[6], tcnt[6];
        int nrec = 0, nq = 0;
  #pragma unroll
        for (int l = 0; l < 6; ++l) {
          const float e0 = ec[kTetOf[l][0]], e1 = ec[kTetOf[l][1]], e2 = ec[kTetOf[l][2]], e3 = ec[kTetOf[l][3]];
          const float mn = fminf(fminf(e0, e1), fminf(e2, e3));
          const float mx = fmaxf(fmaxf(e0, e1), fmaxf(e2, e3));
          int lo = 0, hi = 0;
  #pragma unroll
          for (int l1 = 0; l1 < B; ++l1) {
            lo += omhi[l1] < mn;
            hi += omlo[l1] <= mx;
          }
          const int cnt = any && hi > lo ? hi - lo : 0;
          tlo[l] = lo;
          tcnt[l] = cnt;
          nrec += cnt > 0;
          nq += cnt;
        }
        const int packed = (nq << 16) | nrec;  // nrec <= 6 * 32 and nq <= 6 * 16 * 32 per warp
        int incl = packed;
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        int rbase = 0, qbase = 0;
        if (lane == 31 && incl != 0) {
          rbase = atomicAdd(&s_nrec, incl & 0xffff);
          qbase = atomicAdd(&s_nq, incl >> 16);
        }
        rbase = __shfl_sync(0xffffffffu, rbase, 31);
        qbase = __shfl_sync(0xffffffffu, qbase, 31);
        int rec = rbase + (incl & 0xffff) - nrec;
        int q = qbase + (incl >> 16) - nq;
  #pragma unroll
        for (int l = 0; l < 6; ++l) {
          if (tcnt[l] == 0) continue;
          float en[4];
  #pragma unroll
          for (int k = 0; k < 4; ++k) en[k] = ec[kTetOf[l][k]];
          // corner at each sorted position (tet_pos is a permutation of 0..3)
          const int ps0 = tet_pos(en, 0), ps1 = tet_pos(en, 1), ps2 = tet_pos(en, 2);
          const int c0 = lp[kTetOf[l][0]], c1 = lp[kTetOf[l][1]], c2 = lp[kTetOf[l][2]], c3 = lp[kTetOf[l][3]];
          auto at = [&](int p) { return (unsigned short)(ps0 == p ? c0 : ps1 == p ? c1 : ps2 == p ? c2 : c3); };
          s_recp[rec] = make_ushort4(at(0), at(1), at(2), at(3));
          for (int l1 = tlo[l]; l1 < tlo[l] + tcnt[l]; ++l1) s_queue[q++] = (unsigned short)((rec << 4) | l1);
          ++rec;
        }
      }
    } else {
      // the six tetrahedra of the warp's cells that passed, compacted over the
      // lanes: item = (hit cell, tetrahedron); then one packed warp scan of the
      // (queue entries << 16 | records) counts and one slot reservation per
      // warp for both lists, per round of 32 items
      const unsigned hit = __ballot_sync(0xffffffffu, any);
      if (hit) {
        const int warp = tid >> 5;
        if (any) s_hit[warp][__popc(hit & ((1u << lane) - 1u))] = (unsigned char)lane;
        __syncwarp();
        const int nitem = 6 * __popc(hit);
        for (int it0 = 0; it0 < nitem; it0 += 32) {
          const int item = it0 + lane;
          int cnt = 0, lo = 0;
          float en[4];
          int cpt[4];
          if (item < nitem) {
            const int h = item / 6, t = item - 6 * h;
            const int cell = (warp << 5) + s_hit[warp][h];
            const unsigned code = tet_code(t);
  #pragma unroll
            for (int k = 0; k < 4; ++k) {
              cpt[k] = s_lp[cell][(code >> (3 * k)) & 7u];
              en[k] = s_E[cpt[k]];
            }
            const float mn = fminf(fminf(en[0], en[1]), fminf(en[2], en[3]));
            const float mx = fmaxf(fmaxf(en[0], en[1]), fmaxf(en[2], en[3]));
            int hi = 0;
  #pragma unroll
            for (int l1 = 0; l1 < B; ++l1) {
              lo += omhi[l1] < mn;
              hi += omlo[l1] <= mx;
            }
            cnt = hi > lo ? hi - lo : 0;
          }
          const int packed = (cnt << 16) | (cnt > 0 ? 1 : 0);  // <= 32 records, <= 32*16 entries
          int incl = packed;
  #pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
          }
          int rbase = 0, qbase = 0;
          if (lane == 31 && incl != 0) {
            rbase = atomicAdd(&s_nrec, incl & 0xffff);
            qbase = atomicAdd(&s_nq, incl >> 16);
          }
          rbase = __shfl_sync(0xffffffffu, rbase, 31);
          qbase = __shfl_sync(0xffffffffu, qbase, 31);
          if (cnt > 0) {
            const int rec = rbase + (incl & 0xffff) - 1;
            int q = qbase + (incl >> 16) - cnt;
            // corner at each sorted position (tet_pos is a permutation of 0..3)
            const int ps0 = tet_pos(en, 0), ps1 = tet_pos(en, 1), ps2 = tet_pos(en, 2);
            auto at = [&](int p) {
              return (unsigned short)(ps0 == p ? cpt[0] : ps1 == p ? cpt[1] : ps2 == p ? cpt[2] : cpt[3]);
            };
            s_recp[rec] = make_ushort4(at(0), at(1), at(2), at(3));
            for (int l1 = lo; l1 < lo + cnt; ++l1) s_queue[q++] = (unsigned short)((rec << 4) | l1);
          }
        }
      }
    }
    __syncthreads();
    // phase 2: corner weights of the queued pairs into R
    const int nq = s_nq;
    for (int i = tid; i < nq; i += blockDim.x) {
      const unsigned v = s_queue[i];
      const int rec = (int)(v >> 4), l1 = (int)(v & 15u);
      const ushort4 pp = s_recp[rec];
      // sorted positions 0..3 hold the highest .. lowest corner
      const TetSorted ts = tet_sort(s_E[pp.w], s_E[pp.z], s_E[pp.y], s_E[pp.x]);
      double cp[4];
      if constexpr (F32W) {
        float cf[4];
        if (!tet_weights4_f32(ts, s_om[l1], cf)) continue;
#pragma unroll
        for (int k = 0; k < 4; ++k) cp[k] = cf[k];
      } else {
        if (!tet_weights4(ts, s_om[l1], cp)) continue;
      }
      const int pos_pt[4] = {pp.x, pp.y, pp.z, pp.w};
      const double nb1 = s_nb1[l1];
      const size_t o = (size_t)row * nkc * b * b + l1 * b + l2, op = (size_t)row * nkc * b * b + l1 * b + l3;
      const VT* vs = v3row + l2 * s2 + l3 * s3 + l1 * s1;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int p = pos_pt[k];
        const double G = s_G[p];
        if (cp[k] == 0.0 || G == 0.0) continue;
        const double val = cp[k] * ((double)__ldg(vs + (size_t)s_src[p] * sq) * fnorm6) * (nb1 * G);
        const size_t w = (size_t)s_w[p] * b * b;
        if constexpr (MODE == 0) {
          atomicAdd(Rp + o + w, val);
          if (Rpp) atomicAdd(Rpp + op + w, val);
        } else if constexpr (MODE == 1) {
          const unsigned long long bits = (unsigned long long)__double_as_longlong(val);
          atomicMax(Mp + o + w, bits);
          if (Rpp) atomicMax(Mpp + op + w, bits);
        } else {
          atomicAdd(reinterpret_cast<unsigned long long*>(Rp + o + w), det_fixed(val, Mp[o + w], b));
          if (Rpp) atomicAdd(reinterpret_cast<unsigned long long*>(Rpp + op + w), det_fixed(val, Mpp[op + w], b));
        }
      }
    }
  }
}

// the kernels: the mixed one with the compiler's own register choice (55-62
// registers at 6 bands, measured fastest), the FP64 one held to 64 registers
// (8 CTAs per SM; measured fastest for it)
template <int B, class VT, int MODE>
__global__ void __launch_bounds__(kFusedThreads) delta_fused_mixed_kernel(CombineArgs a, const VT* __restrict__ v3sq) {
  delta_fused_body<B, true, VT, MODE>(a, v3sq);
}
template <int B, int MODE>
__global__ void __launch_bounds__(kFusedThreads, 8) delta_fused_fp64_kernel(CombineArgs a,
                                                                            const double* __restrict__ v3sq) {
  delta_fused_body<B, false, double, MODE>(a, v3sq);
}

// the fixed-point sums of the deterministic passes back to FP64, in place
__global__ void delta_finalize_kernel(double* R, const unsigned long long* __restrict__ M, size_t n, int b) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long m = M[i];
    const unsigned long long acc = reinterpret_cast<const unsigned long long*>(R)[i];
    R[i] = m == 0 ? 0.0 : ldexp((double)acc, det_exponent(m, b) - 62);
  }
}

// ---------------------------------------------------------------------------
// Any number of bands (the large cells): the delta straight from the slice
// energies, no per-band register arrays.
//
// Tetrahedron: a thread per (slice, tetrahedron); its four corner energies
// E = -+omega(w,l2) + omega(q1+-w,l3) as default REAL, one sort, the bands
// l1 whose omega1 lies in [E_min, E_max] by binary search (omega1 ascending),
// and for each one weight_tet's corner weights c (bitwise, ald_tet.h) added
// at the four corners w:
//   P1s/P2s(row, w, l1, l2, l3) += c/6 |V3|^2(src(w)) (2pi)^2/nkc        (if given)
//   R(row, w, l1, l2)           += that * n1 G(w)                       (if given)
// with G and the Gamma-acoustic zeros of the fused kernel.  FP64 atomics:
// the sums agree with the reference to FP64 rounding, not bitwise.
template <bool F32W, class VT>
__global__ void __launch_bounds__(256) delta_tet_any_kernel(CombineArgs a, const VT* __restrict__ v3sq) {
  extern __shared__ double s_any[];  // omega1[b], n1[b]
  const Geometry& g = a.geo;
  const int b = g.b, nkc = g.nkc, b2 = b * b;
  const int slice = blockIdx.x;  // x: up to 2^31 - 1 slices; y: blocks of tetrahedra
  const int proc = slice & 1, l3 = (slice >> 1) % b, l2 = (slice / (2 * b)) % b, row = slice / (2 * b2);
  const int q1 = a.mapinv[a.n1_first + row];
  double* s_om = s_any;
  double* s_nb = s_any + b;
  for (int l = threadIdx.x; l < b; l += blockDim.x) {
    s_om[l] = a.freq[(size_t)q1 * b + l];
    s_nb[l] = a.dist[(size_t)q1 * b + l];
  }
  __syncthreads();
  const int t = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= 6 * nkc) return;
  int m1[3];
  decompose(g, q1, m1);
  int c[4], src[4];
  float en[4];
  double G[4];
  tet_corners(g, t, c);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int mw[3], m3[3], ins;
    decompose(g, c[k], mw);
    const int q3 = pm_index_m(g, m1, mw, proc == 0 ? 1 : -1, ins, m3);
    const double fw = a.freq[(size_t)c[k] * b + l2], f3 = a.freq[(size_t)q3 * b + l3];
    en[k] = (float)(proc == 0 ? -fw + f3 : fw + f3);
    const bool zero = (l2 < 3 && at_gamma_index(g, mw)) || (l3 < 3 && at_gamma_index(g, m3));
    const double n2 = a.dist[(size_t)c[k] * b + l2], n3 = a.dist[(size_t)q3 * b + l3];
    G[k] = zero ? -1.0 : (proc == 0 ? n2 * (n3 + 1) : (n2 + 1) * (n3 + 1));
    src[k] = proc == 0 ? c[k] : neg_index(g, mw);
  }
  const TetSorted ts = tet_sort(en[0], en[1], en[2], en[3]);
  const double E1 = ts.e1, E4 = ts.e4;
  // first band with omega1 >= E1, first band with omega1 > E4
  int lo = 0, hi = b;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (s_om[mid] < E1) lo = mid + 1;
    else hi = mid;
  }
  int lo2 = lo, hi2 = b;
  while (lo2 < hi2) {
    const int mid = (lo2 + hi2) >> 1;
    if (s_om[mid] > E4) hi2 = mid;
    else lo2 = mid + 1;
  }
  const int lend = lo2;
  const double fnorm = (2 * PhysConst::pi) * (2 * PhysConst::pi) / nkc;
  size_t sq, s1, s2, s3;
  if (a.v3_layout == 1) {  // [l2][l3][l1][q]
    sq = 1;
    s1 = nkc;
    s3 = (size_t)b * nkc;
    s2 = (size_t)b2 * nkc;
  } else if (a.v3_layout == 2) {  // [l2][l3][q][l1]
    s1 = 1;
    sq = b;
    s3 = (size_t)b * nkc;
    s2 = (size_t)b2 * nkc;
  } else {  // [q][l1][l2][l3]
    s3 = 1;
    s2 = b;
    s1 = (size_t)b2;
    sq = (size_t)b2 * b;
  }
  const VT* v3 = v3sq + (size_t)row * nkc * b2 * b + l2 * s2 + l3 * s3;
  double* Ps = proc == 0 ? a.P1s : a.P2s;
  double* Rp = proc == 0 ? a.R1 : a.R2;
  double* Rpp = proc == 0 ? a.R1p : a.R2p;
  int pos[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) pos[k] = tet_pos(en, k);
  for (int l1 = lo; l1 < lend; ++l1) {
    double cp[4];
    if constexpr (F32W) {
      float cf[4];
      if (!tet_weights4_f32(ts, s_om[l1], cf)) continue;
#pragma unroll
      for (int k = 0; k < 4; ++k) cp[k] = cf[k];
    } else {
      if (!tet_weights4(ts, s_om[l1], cp)) continue;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double cw = cp[pos[k]];
      if (cw == 0.0 || G[k] < 0.0) continue;
      const double ps = (cw / 6.0) * ((double)__ldg(v3 + (size_t)src[k] * sq + l1 * s1) * fnorm);
      const size_t w = (size_t)row * nkc + c[k];
      if (Ps) atomicAdd(Ps + (w * b + l1) * b2 + l2 * b + l3, ps);
      if (Rp) {
        const double p = ps * (s_nb[l1] * G[k]);
        atomicAdd(Rp + (w * b + l1) * b + l2, p);
        if (Rpp) atomicAdd(Rpp + (w * b + l1) * b + l3, p);
      }
    }
  }
}

// Gaussian: a thread per (row, w, l1, l2), w fastest; the sums over l3 of
// both processes (R1, R2 at w) in registers, P1s/P2s written when given.
// The Gaussian is delta_g of extratools.f90:239 as in delta_point_kernel.
template <bool F32W, class VT>
__global__ void __launch_bounds__(128) delta_gauss_any_kernel(CombineArgs a, const VT* __restrict__ v3sq) {
  const Geometry& g = a.geo;
  const int b = g.b, nkc = g.nkc, b2 = b * b, b3 = b2 * b;
  // x: (l1, l2, w), w fastest for layouts 0/1 (|V3|^2 runs of q2), l1
  // fastest for layout 2 (runs of l1); y: row
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  int w, l1, l2;
  if (a.v3_layout == 2) {
    l1 = (int)(gid % b);
    w = (int)((gid / b) % nkc);
    l2 = (int)(gid / ((long long)b * nkc));
  } else {
    w = (int)(gid % nkc);
    const long long l12 = gid / nkc;
    l1 = (int)(l12 / b);
    l2 = (int)(l12 % b);
  }
  if (l2 >= b || l1 >= b) return;
  const int q1 = a.mapinv[a.n1_first + row];
  int m1[3], mw[3], m3p[3], m3m[3], ins1, ins2;
  decompose(g, q1, m1);
  decompose(g, w, mw);
  const int q3p = pm_index_m(g, m1, mw, 1, ins1, m3p);
  const int q3m = pm_index_m(g, m1, mw, -1, ins2, m3m);
  const int wneg = neg_index(g, mw);
  const bool w_gamma = at_gamma_index(g, mw), p_gamma = at_gamma_index(g, m3p), m_gamma = at_gamma_index(g, m3m);
  const double fnorm = (2 * PhysConst::pi) * (2 * PhysConst::pi) / nkc;
  const double om1 = a.freq[(size_t)q1 * b + l1], nb1 = a.dist[(size_t)q1 * b + l1];
  const double n2 = a.dist[(size_t)w * b + l2], w2 = a.freq[(size_t)w * b + l2];
  const VT* v3 = v3sq + (size_t)row * nkc * b3;
  const int L = a.v3_layout;
  const size_t sq = L == 1 ? 1 : (L == 2 ? (size_t)b : (size_t)b3);
  const size_t s1 = L == 1 ? (size_t)nkc : (L == 2 ? 1 : (size_t)b2);
  const size_t s2 = L == 0 ? (size_t)b : (size_t)b2 * nkc, s3 = L == 0 ? 1 : (size_t)b * nkc;
  const double gc1 = 0.5 / (a.sigma * a.sigma), gc2 = 1.0 / (sqrt(2 * PhysConst::pi) * a.sigma);
  const float fc1 = (float)gc1, fc2 = (float)gc2;
  double R[2] = {0.0, 0.0};
  for (int l3 = 0; l3 < b; ++l3) {
#pragma unroll
    for (int proc = 0; proc < 2; ++proc) {
      const int q3 = proc == 0 ? q3p : q3m;
      const bool zero = (l2 < 3 && w_gamma) || (l3 < 3 && (proc == 0 ? p_gamma : m_gamma));
      const int src = proc == 0 ? w : wneg;
      const double n3 = a.dist[(size_t)q3 * b + l3], w3 = a.freq[(size_t)q3 * b + l3];
      const double x = proc == 0 ? om1 + w2 - w3 : om1 - w2 - w3;
      double wl = 0.0;
      if constexpr (F32W) {
        const float xf = (float)x, arg = xf * xf * fc1;
        if (arg < 104.0f) wl = (double)(expf(-arg) * fc2);
      } else {
        const double arg = x * x * gc1;
        if (arg < 746.0) wl = exp(-arg) * gc2;
      }
      double ps = 0.0;
      if (wl != 0.0 && !zero) ps = wl * ((double)v3[(size_t)src * sq + l1 * s1 + l2 * s2 + l3 * s3] * fnorm);
      const double p = ps * (proc == 0 ? nb1 * n2 * (n3 + 1) : nb1 * (n2 + 1) * (n3 + 1));
      R[proc] += p;
      double* Rpm = proc == 0 ? a.R1p : a.R2p;
      if (Rpm && p != 0.0) atomicAdd(Rpm + (((size_t)row * nkc + w) * b + l1) * b + l3, p);
      double* Ps = proc == 0 ? a.P1s : a.P2s;
      if (Ps) Ps[(((size_t)row * nkc + w) * b + l1) * b2 + l2 * b + l3] = ps;
    }
  }
  const size_t ri = (((size_t)row * nkc + w) * b + l1) * b + l2;
  if (a.R1) a.R1[ri] = R[0];
  if (a.R2) a.R2[ri] = R[1];
}

// Q, Q_N, Q_U of any number of bands: a CTA per (row, l1), threads over w
__global__ void __launch_bounds__(256) q_from_r_any_kernel(Geometry g, int n1_first, const int* mapinv,
                                                           const double* R1, const double* R2, double* Q,
                                                           double* QN, double* QU) {
  __shared__ double red[3][256];
  const int b = g.b, nkc = g.nkc, row = blockIdx.x, l1 = blockIdx.y, tid = threadIdx.x;
  const int q1 = mapinv[n1_first + row];
  int m1[3];
  decompose(g, q1, m1);
  double s = 0, sn = 0, su = 0;
  for (int w = tid; w < nkc; w += blockDim.x) {
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
  red[0][tid] = s;
  red[1][tid] = sn;
  red[2][tid] = su;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {  // fixed tree: deterministic
    if (tid < o)
      for (int k = 0; k < 3; ++k) red[k][tid] += red[k][tid + o];
    __syncthreads();
  }
  if (tid == 0) {
    const size_t o = (size_t)(n1_first + row) * b + l1;
    Q[o] = red[0][0];
    QN[o] = red[1][0];
    QU[o] = red[2][0];
  }
}

// weight_tet over a list of tetrahedra at one energy e, one thread each:
// w[4 t + k] corner energies, c[4 t + k] corner weights (0 outside the
// tetrahedron's energy range).  fp32 = 0: the FP64 form the FP64 pipeline
// uses (bit for bit the reference's arithmetic); 1: the FP32 form of the
// mixed pipeline.
__global__ void __launch_bounds__(256) weight_tet_kernel(int ntet, const double* __restrict__ w, double e, int fp32,
                                                         double* __restrict__ c) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
    float en[4];
    for (int k = 0; k < 4; ++k) en[k] = (float)w[4 * (size_t)t + k];
    const TetSorted ts = tet_sort(en[0], en[1], en[2], en[3]);
    double cp[4] = {0.0, 0.0, 0.0, 0.0};
    if (fp32) {
      float cf[4];
      if (tet_weights4_f32(ts, e, cf))
        for (int k = 0; k < 4; ++k) cp[k] = (double)cf[k];
    } else if (!tet_weights4(ts, e, cp)) {
      cp[0] = cp[1] = cp[2] = cp[3] = 0.0;
    }
    for (int k = 0; k < 4; ++k) c[4 * (size_t)t + k] = cp[tet_pos(en, k)];
  }
}

}  // namespace

cudaError_t launch_weight_tet(int ntet, const double* w, double e, int fp32, double* c, cudaStream_t s) {
  if (ntet <= 0) return cudaSuccess;
  const int blocks = std::min((ntet + 255) / 256, 148 * 8);
  weight_tet_kernel<<<blocks, 256, 0, s>>>(ntet, w, e, fp32, c);
  return cudaGetLastError();
}

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
  const int nw = kPointBlock / g.b;
  dim3 grid_tile((g.nkc + nw - 1) / nw, a.nrows), grid_row((g.nkc + kPointBlock - 1) / kPointBlock, a.nrows, g.b);
  // FP32 weights only for the Gaussian (the tetrahedron weights W are FP64 here)
  const bool fw = a.f32w && a.gauss;
  const bool pair = fw && !a.P1s && !a.P2s && !a.P1 && !a.P2;
#define ALD_POINT(BB)                                                               \
  if (pair)                                                                         \
    delta_point_pair_kernel<BB><<<grid_row, kPointBlock, 0, s>>>(a);                \
  else if (fw)                                                                      \
    delta_point_kernel<BB, true, false><<<grid_row, kPointBlock, 0, s>>>(a, W);     \
  else                                                                              \
    delta_point_kernel<BB, false, true><<<grid_tile, kPointBlock, 0, s>>>(a, W);
  if (g.b <= 3) {
    ALD_POINT(3)
  } else if (g.b <= 6) {
    ALD_POINT(6)
  } else if (g.b <= 12) {
    ALD_POINT(12)
  } else if (g.b <= 16) {
    ALD_POINT(16)
  } else {
    return cudaErrorInvalidValue;
  }
#undef ALD_POINT
  return cudaGetLastError();
}

bool delta_fused_supported(const Geometry& g) {
  return g.b <= kMaxBandsTet && g.nc[2] <= kFusedThreads && fused_shape(g).smem <= 200 * 1024;
}

#define ALD_COMMA ,
template <int MODE>
static cudaError_t launch_delta_fused_mode(const CombineArgs& a, cudaStream_t s) {
  const Geometry& g = a.geo;
  const FusedShape f = fused_shape(g);
  dim3 grid(g.nc[0] * f.nbj, a.nrows, 2 * g.b);
  cudaError_t e;
#define ALD_FUSED2(KERNEL, PTR)                                                          \
  {                                                                                      \
    e = raise_smem_limit((const void*)KERNEL, f.smem);                                   \
    if (e != cudaSuccess) return e;                                                      \
    KERNEL<<<grid, kFusedThreads, f.smem, s>>>(a, PTR);                                  \
  }
  // FP32 |V3|^2 only comes with the FP32 weights of the mixed pipeline
#define ALD_FUSED(BB)                                                                  \
  if (a.v3sq_f32) {                                                                    \
    ALD_FUSED2(delta_fused_mixed_kernel<BB ALD_COMMA float ALD_COMMA MODE>, a.v3sq_f32) \
  } else if (a.f32w) {                                                                 \
    ALD_FUSED2(delta_fused_mixed_kernel<BB ALD_COMMA double ALD_COMMA MODE>, a.v3sq)    \
  } else {                                                                             \
    ALD_FUSED2(delta_fused_fp64_kernel<BB ALD_COMMA MODE>, a.v3sq)                      \
  }
  if (a.v3sq_f32 && !a.f32w) return cudaErrorInvalidValue;
  if (g.b <= 3) {
    ALD_FUSED(3)
  } else if (g.b <= 6) {
    ALD_FUSED(6)
  } else if (g.b <= 12) {
    ALD_FUSED(12)
  } else {
    ALD_FUSED(16)
  }
#undef ALD_FUSED
#undef ALD_FUSED2
  return cudaGetLastError();
}
#undef ALD_COMMA

cudaError_t launch_delta_fused(const CombineArgs& a, cudaStream_t s, int mode) {
  if (!delta_fused_supported(a.geo)) return cudaErrorInvalidValue;
  if (mode == 0) return launch_delta_fused_mode<0>(a, s);
  if (!a.M1 || !a.M2 || (a.R1p && !a.M1p) || (a.R2p && !a.M2p)) return cudaErrorInvalidValue;
  if (mode == 1) return launch_delta_fused_mode<1>(a, s);
  if (mode == 2) return launch_delta_fused_mode<2>(a, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_delta_finalize(double* R, const unsigned long long* M, size_t n, int b, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  delta_finalize_kernel<<<blocks, 256, 0, s>>>(R, M, n, b);
  return cudaGetLastError();
}

cudaError_t launch_delta_any(const CombineArgs& a, cudaStream_t s) {
  const Geometry& g = a.geo;
  if (g.b > 256) return cudaErrorInvalidValue;
  if (a.gauss) {
    const long long nx = ((long long)g.nkc * g.b * g.b + 127) / 128;
    if (nx > 2147483647LL || a.nrows > 65535) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)nx, a.nrows);
    if (a.v3sq_f32) {
      if (a.f32w) delta_gauss_any_kernel<true, float><<<grid, 128, 0, s>>>(a, a.v3sq_f32);
      else delta_gauss_any_kernel<false, float><<<grid, 128, 0, s>>>(a, a.v3sq_f32);
    } else {
      if (a.f32w) delta_gauss_any_kernel<true, double><<<grid, 128, 0, s>>>(a, a.v3sq);
      else delta_gauss_any_kernel<false, double><<<grid, 128, 0, s>>>(a, a.v3sq);
    }
  } else {
    const long long nslice = (long long)a.nrows * g.b * g.b * 2;
    if (nslice > 2147483647LL) return cudaErrorInvalidValue;
    if ((6LL * g.nkc + 255) / 256 > 65535) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)nslice, (6 * g.nkc + 255) / 256);
    const size_t smem = 2 * (size_t)g.b * sizeof(double);
    if (a.v3sq_f32) {
      if (a.f32w) delta_tet_any_kernel<true, float><<<grid, 256, smem, s>>>(a, a.v3sq_f32);
      else delta_tet_any_kernel<false, float><<<grid, 256, smem, s>>>(a, a.v3sq_f32);
    } else {
      if (a.f32w) delta_tet_any_kernel<true, double><<<grid, 256, smem, s>>>(a, a.v3sq);
      else delta_tet_any_kernel<false, double><<<grid, 256, smem, s>>>(a, a.v3sq);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_q_from_r(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* R1,
                            const double* R2, double* Q, double* QN, double* QU, int nibz, cudaStream_t s) {
  (void)nibz;
  if (3 * geo.b > 256) {
    q_from_r_any_kernel<<<dim3(nrows, geo.b), 256, 0, s>>>(geo, n1_first, mapinv, R1, R2, Q, QN, QU);
    return cudaGetLastError();
  }
  q_from_r_kernel<<<nrows, 256 / geo.b * geo.b, 0, s>>>(geo, n1_first, mapinv, R1, R2, Q, QN, QU);
  return cudaGetLastError();
}

}  // namespace ald
