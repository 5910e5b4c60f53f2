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
// Structure.  For one IBZ row q1 and bands (l2, l3) the reference gives
// every mesh point w the corner energies
//   process 1: E(w) = -omega(w,l2) + omega(q1+w,l3)   (coalescence)
//   process 2: E(w) =  omega(w,l2) + omega(q1-w,l3)   (decay)
// evaluates weight_tet(omega1) on the 6*nkc tetrahedra and adds c/6 * F(w)
// into P(w) for each of the four corners.  Here each thread owns one mesh
// point w and gathers the 24 (tetrahedron, corner) incidences of w; all
// their corners lie in the 3x3x3 neighbourhood of w, whose 27 energies the
// thread holds in registers (the incidence table is a compile-time
// constant).  P = F * sum(c/6) is formed only where a weight is nonzero,
// then Bose-weighted and summed over l3 in registers.
//
// The corner weights reproduce weight_tet's mixed FP32/FP64 arithmetic
// (ald_tet.h); this file is compiled with -fmad=false.
#include <cuda_runtime.h>

#include "ald_internal.h"
#include "ald_tet.h"

namespace ald {

namespace {

constexpr int kBlock = 128;

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

// ---------------------------------------------------------------------------
// The 24 incidences of a mesh point.  Cube corners (make_kp_reg_tet):
// pt1..pt8 at offsets (0,0,0) (1,0,0) (0,1,0) (1,1,0) (0,0,1) (1,0,1) (0,1,1)
// (1,1,1); tetrahedra l=1..6 use corners (1,2,3,6) (2,3,4,6) (1,3,5,6)
// (3,4,6,8) (3,5,6,7) (3,6,7,8).  A point w is corner p of the cube based at
// w - off(p).  Each incidence stores its four corners as indices of the
// 3x3x3 neighbourhood of w (nb = (dx+1)*9 + (dy+1)*3 + (dz+1)) in the
// tetrahedron's corner order, and which of the four is w.
struct Incidence {
  int nb[4];
  int slot;
};

struct IncTable {
  Incidence inc[24];
};

constexpr int kOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
constexpr int kTet[6][4] = {{0, 1, 2, 5}, {1, 2, 3, 5}, {0, 2, 4, 5}, {2, 3, 5, 7}, {2, 4, 5, 6}, {2, 5, 6, 7}};

__host__ __device__ constexpr IncTable make_table() {
  IncTable t{};
  int n = 0;
  for (int p = 0; p < 8; ++p)
    for (int l = 0; l < 6; ++l)
      for (int k = 0; k < 4; ++k)
        if (kTet[l][k] == p) {
          for (int c = 0; c < 4; ++c) {
            int q = kTet[l][c];
            int dx = kOff[q][0] - kOff[p][0], dy = kOff[q][1] - kOff[p][1], dz = kOff[q][2] - kOff[p][2];
            t.inc[n].nb[c] = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
          }
          t.inc[n].slot = k;
          ++n;
        }
  return t;
}

// ---------------------------------------------------------------------------
// corner energies E[row][l2][l3][proc][w] as default REAL (weight_tet's en)
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

__constant__ int c_inc[24][5];  // four neighbourhood indices + the slot of w

template <int B>
__global__ void __launch_bounds__(kBlock) delta_gather_kernel(CombineArgs a, const float* __restrict__ E) {
  __shared__ double s_om1[B], s_nb1[B];
  __shared__ float s_en[27 * kBlock];  // s_en[k * kBlock + tid]: energies of the 3x3x3 neighbourhood
  __shared__ int s_nbr[27 * kBlock];
  __shared__ double s_W[B * kBlock];   // per-thread sum_inc c/6 for each lambda1
  const Geometry& g = a.geo;
  const int b = g.b, nkc = g.nkc, b2 = b * b, b3 = b2 * b;
  const int row = blockIdx.z, l2 = blockIdx.y, tid = threadIdx.x;
  const int n1 = a.n1_first + row;
  const int q1 = a.mapinv[n1];
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
  double emin = 1e300, emax = -1e300;
  for (int l = 0; l < b; ++l) {
    emin = fmin(emin, s_om1[l]);
    emax = fmax(emax, s_om1[l]);
  }
  for (int k = 0; k < 27; ++k) {
    int dx = k / 9 - 1, dy = (k / 3) % 3 - 1, dz = k % 3 - 1;
    int m[3] = {wrapm(mw[0] + dx, g.nc[0]), wrapm(mw[1] + dy, g.nc[1]), wrapm(mw[2] + dz, g.nc[2])};
    s_nbr[k * kBlock + tid] = compose(g, m);
  }
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
    for (int proc = 0; proc < 2; ++proc) {
      double* W = s_W + tid;  // W[l * kBlock]
      for (int l = 0; l < b; ++l) W[l * kBlock] = 0.0;
      const int q3 = proc == 0 ? q3p : q3m;
      if (!a.gauss) {
        const float* Ep = E + ((((size_t)row * b + l2) * b + l3) * 2 + proc) * nkc;
        for (int k = 0; k < 27; ++k) s_en[k * kBlock + tid] = __ldg(Ep + s_nbr[k * kBlock + tid]);
        for (int i = 0; i < 24; ++i) {
          float c4[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) c4[c] = s_en[c_inc[i][c] * kBlock + tid];
          TetSorted ts = tet_sort(c4[0], c4[1], c4[2], c4[3]);
          if (emax < (double)ts.e1 || emin > (double)ts.e4) continue;
          int pos = tet_pos(c4, c_inc[i][4]);
#pragma unroll 1
          for (int l = 0; l < b; ++l) {
            double c = tet_weight(ts, pos, s_om1[l]);
            if (c != 0.0) W[l * kBlock] += c / 6.0;
          }
        }
      } else {
        double w2 = a.freq[(size_t)w * b + l2], w3 = a.freq[(size_t)q3 * b + l3];
        for (int l = 0; l < b; ++l)
          W[l * kBlock] = delta_g(proc == 0 ? s_om1[l] + w2 - w3 : s_om1[l] - w2 - w3, a.sigma);
      }
      const bool zero = (l2 < 3 && w_gamma) || (l3 < 3 && (proc == 0 ? p_gamma : m_gamma));
      const int src = proc == 0 ? w : wneg;
      const double n3 = a.dist[(size_t)q3 * b + l3];
      double* Ps = proc == 0 ? a.P1s : a.P2s;
      double* Pb = proc == 0 ? a.P1 : a.P2;
#pragma unroll
      for (int l = 0; l < B; ++l) {
        if (l >= b) continue;
        double ps = 0.0;
        const double wl = W[l * kBlock];
        if (wl != 0.0 && !zero) ps = wl * (v3[(size_t)src * b3 + (l * b + l2) * b + l3] * fnorm);
        double nb1 = s_nb1[l];
        double Fb = proc == 0 ? nb1 * n2 * (n3 + 1) : nb1 * (n2 + 1) * (n3 + 1);
        double p = ps * Fb;
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
                                double* Q, double* QN, double* QU, int nibz) {
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
    double n = (i1 ? r1 : 0.0) + (i2 ? 0.5 * r2 : 0.0);
    sn += n;
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
  return gauss ? 0 : (size_t)nrows * geo.b * geo.b * 2 * geo.nkc * sizeof(float);
}

cudaError_t launch_combine(const CombineArgs& a, float* scratch, cudaStream_t s) {
  const Geometry& g = a.geo;
  static bool table_set = false;
  if (!table_set) {
    constexpr IncTable T = make_table();
    int h[24][5];
    for (int i = 0; i < 24; ++i) {
      for (int c = 0; c < 4; ++c) h[i][c] = T.inc[i].nb[c];
      h[i][4] = T.inc[i].slot;
    }
    cudaError_t e = cudaMemcpyToSymbol(c_inc, h, sizeof h);
    if (e != cudaSuccess) return e;
    table_set = true;
  }
  if (!a.gauss) {
    size_t total = (size_t)a.nrows * g.b * g.b * 2 * g.nkc;
    int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 64);
    tet_energy_kernel<<<blocks, 256, 0, s>>>(g, a.n1_first, a.nrows, a.mapinv, a.freq, scratch);
  }
  dim3 grid((g.nkc + kBlock - 1) / kBlock, g.b, a.nrows);
  if (g.b <= 3)
    delta_gather_kernel<3><<<grid, kBlock, 0, s>>>(a, scratch);
  else if (g.b <= 6)
    delta_gather_kernel<6><<<grid, kBlock, 0, s>>>(a, scratch);
  else if (g.b <= 12)
    delta_gather_kernel<12><<<grid, kBlock, 0, s>>>(a, scratch);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_q_from_r(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* R1,
                            const double* R2, double* Q, double* QN, double* QU, int nibz, cudaStream_t s) {
  dim3 grid(nrows, geo.b);
  q_from_r_kernel<<<grid, 256, 0, s>>>(geo, n1_first, mapinv, R1, R2, Q, QN, QU, nibz);
  return cudaGetLastError();
}

}  // namespace ald
