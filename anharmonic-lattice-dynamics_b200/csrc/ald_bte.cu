// Boltzmann-equation stage on the device.
//
//   calculate_RTA_distributionfunction  THERMACOND/sub.f90:1238-1289
//   mode_kappa / mode_kappa_d           THERMACOND/sub.f90:1292-1401, 1407-1530
//   veloc_avergeIBZ_invsyFBZ            THERMACOND/sub.f90:5479-5537
//   cal_RHS_IBZ                         THERMACOND/sub.f90:2618-2691
//   CollisionMatrix_mpi                 THERMACOND/sub.f90:3034-3210
//   cg_quadratic                        THERMACOND/cg.f90:19-61
//
// Vectors indexed like the reference's DirectSolution / RHS:
// s = 3*((ibz)*ndyn + l) + xyz (0-based).  The collision matrix is kept
// row-major on the device (row s1 contiguous) so that the CG matrix-vector
// product reads each row with coalesced loads; HBM bandwidth bounds it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "ald_internal.h"

namespace ald {

namespace {

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
// mesh index of q1 + w (sign=+1) or q1 - w (sign=-1); `inside` is get_k_info's flag
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

__device__ __forceinline__ double nbe_dev(double w, double t, int m, int* err) {
  if (t <= 0 || w <= 0) {
    atomicOr(err, 1);
    return 0.0;
  }
  double z = w / t;
  if (m == 0) {
    if (z > 60) return 0.0;
    if (z < (double)0.0010f) return 1 / (z * (1 + z / 2 * (1 + z / 3)));
    return 1 / (exp(z) - 1);
  }
  return 1 / z;
}

// syop_f's product (column-major 3x3), rounded as the Fortran rounds it (no
// fused multiply-add), so that near-cancelling components come out the same
__device__ __forceinline__ void opmul(const double* op, const double* v, double* out) {
  for (int i = 0; i < 3; ++i) {
    double x = 0;
    for (int j = 0; j < 3; ++j) x = __dadd_rn(x, __dmul_rn(op[i + 3 * j], v[j]));
    out[i] = x;
  }
}

__global__ void rta_F_kernel(KappaArgs a, const double* Q, double* F) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int b = a.geo.b;
  if (idx >= a.nibz * b) return;
  int i = idx / b, l = idx % b;
  int n0 = a.mapinv[i];
  double omega = a.freq[(size_t)n0 * b + l], nb = a.dist[(size_t)n0 * b + l];
  const double c = PhysConst::c_light, h = PhysConst::h_plank, kb = PhysConst::k_b;
  for (int x = 0; x < 3; ++x) {
    double v = a.vel[((size_t)n0 * b + l) * 3 + x];
    // zero_q_f: a mode without scattering (Q = 0 exactly) gets F = 0 instead
    // of a division by zero (the mixed path, where the FP32 weights of the
    // acoustic modes at Gamma can vanish; those carry no heat, omega v = 0)
    F[(size_t)idx * 3 + x] =
        a.zero_q_f && Q[idx] == 0.0
            ? 0.0
            : -((((((c * v) * h) * ((omega * c) * 100)) * nb) * (nb + 1)) / (kb * (a.tempk * a.tempk)) /
                ((Q[idx] * c) * 100));
  }
}

__global__ void rhs_kernel(KappaArgs a, double* rhs) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int b = a.geo.b;
  if (idx >= a.nibz * b) return;
  int i = idx / b, l = idx % b;
  int n0 = a.mapinv[i];
  double omega = a.freq[(size_t)n0 * b + l], nb0 = a.dist[(size_t)n0 * b + l];
  const double c = PhysConst::c_light, h = PhysConst::h_plank, kb = PhysConst::k_b;
  for (int x = 0; x < 3; ++x) {
    double v = a.vel[((size_t)n0 * b + l) * 3 + x];
    rhs[(size_t)idx * 3 + x] =
        ((((((c * v) * h) * ((omega * c) * 100)) * nb0) * (nb0 + 1)) / (kb * (a.tempk * a.tempk))) / (c * 100);
  }
}

// one CTA per band l; threads over IBZ points; 9 sums reduced in the block
// kappa per band: a thread per (arm of an IBZ point, band), a CTA per
// (block of kKapThreads arms, band); per-CTA partial sums of the 9
// components, added in CTA order by kappa_final_kernel
constexpr int kKapThreads = 128;

// velocity of IBZ mode (i, l): veloc at mapinv(i) (mode_kappa), or the star
// average with inverse operations (veloc_avergeIBZ_invsyFBZ, sub.f90:5479)
__device__ __forceinline__ void mode_velocity(const KappaArgs& a, int i, int l, int averaged, double vv[3]) {
  const int b = a.geo.b;
  if (averaged) {
    int s0 = a.star_off[i], s1 = a.star_off[i + 1];
    double narms = (double)(s1 - s0);
    double va[3] = {0, 0, 0};
    for (int t = s0; t < s1; ++t) {
      const double* vq = a.vel + ((size_t)a.star_q[t] * b + l) * 3;
      double vin[3] = {vq[0], vq[1], vq[2]}, vr[3];
      opmul(a.opk_inv + 9 * a.star_op[t], vin, vr);
      for (int x = 0; x < 3; ++x) va[x] = va[x] + (vr[x] / narms);
    }
    for (int x = 0; x < 3; ++x) vv[x] = va[x];
  } else {
    const double* vq = a.vel + ((size_t)a.mapinv[i] * b + l) * 3;
    vv[0] = vq[0];
    vv[1] = vq[1];
    vv[2] = vq[2];
  }
}

__global__ void __launch_bounds__(kKapThreads) kappa_arm_kernel(KappaArgs a, const double* F, int averaged,
                                                                int narm, int* err) {
  __shared__ double red[9][kKapThreads / 32];
  const int b = a.geo.b, l = blockIdx.y;
  const int s = blockIdx.x * kKapThreads + threadIdx.x;
  double acc[9];
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  if (s < narm) {
    const int i = a.arm_owner[s];
    double f[3] = {F[((size_t)i * b + l) * 3], F[((size_t)i * b + l) * 3 + 1], F[((size_t)i * b + l) * 3 + 2]};
    double vv[3];
    mode_velocity(a, i, l, averaged, vv);
    const double* op = a.opk + 9 * a.arm_op[s];
    double F12[3], velocc[3];
    opmul(op, f, F12);
    opmul(op, vv, velocc);
    int n0 = a.arm_q[s];
    double omega = sqrt(a.w2[(size_t)n0 * b + l]) * PhysConst::cnst();
    double nb0 = nbe_dev(omega, a.temp, a.classical, err);
    for (int j = 0; j < 3; ++j)
      for (int jj = 0; jj < 3; ++jj)
        acc[j + 3 * jj] -= ((((a.const1 * omega) * velocc[j]) * nb0) * (nb0 + 1)) * F12[jj];
  }
  for (int k = 0; k < 9; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double t = 0;
    for (int w = 0; w < kKapThreads / 32; ++w) t += red[threadIdx.x][w];
    a.part[((size_t)l * gridDim.x + blockIdx.x) * 9 + threadIdx.x] = t;
  }
}

__global__ void kappa_final_kernel(int b, int nblk, const double* part, double* kappa_modes) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 9 * b) return;
  const int l = t / 9, k = t % 9;
  double s = 0;
  for (int q = 0; q < nblk; ++q) s += part[((size_t)l * nblk + q) * 9 + k];
  const int j = k % 3, jj = k / 3;
  kappa_modes[l + b * (j + 3 * jj)] = s;  // kappa(ndyn,3,3) column-major
}

// tauinv_eff(i, l): a thread per IBZ mode, its star arms in table order.
//   mode_kappa   (averaged = 0, sub.f90:1360-1365): per arm and j,
//     -= const2 F12(j)/omega/0.01 where velocc(j) == 0, else
//     -= const2 F12(j)/omega/velocc(j)/(3 narms);
//   mode_kappa_d (averaged = 1, sub.f90:1497): per arm, three times (the j
//     loop around it), -= const2 (F12.velocc)/omega/(velocc.velocc)/(3 narms).
// F12 and velocc are F and the velocity rotated onto the arm (syop_f).
__global__ void tau_eff_kernel(KappaArgs a, const double* F, int averaged, double* tinv) {
  const int b = a.geo.b;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.nibz * b) return;
  const int i = idx / b, l = idx % b;
  const double f[3] = {F[(size_t)idx * 3], F[(size_t)idx * 3 + 1], F[(size_t)idx * 3 + 2]};
  double vv[3];
  mode_velocity(a, i, l, averaged, vv);
  const int s0 = a.arm_off[i], s1 = a.arm_off[i + 1];
  const double narms3 = (double)(s1 - s0) * 3.0;
  double t = 0.0;
  for (int s = s0; s < s1; ++s) {
    const double* op = a.opk + 9 * a.arm_op[s];
    double F12[3], velocc[3];
    opmul(op, f, F12);
    opmul(op, vv, velocc);
    const double omega = sqrt(a.w2[(size_t)a.arm_q[s] * b + l]) * PhysConst::cnst();
    if (averaged) {
      const double fv = __dadd_rn(__dadd_rn(__dmul_rn(F12[0], velocc[0]), __dmul_rn(F12[1], velocc[1])),
                                  __dmul_rn(F12[2], velocc[2]));
      const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(velocc[0], velocc[0]), __dmul_rn(velocc[1], velocc[1])),
                                  __dmul_rn(velocc[2], velocc[2]));
      const double term = (((a.const2 * fv) / omega) / v2) / narms3;
      for (int j = 0; j < 3; ++j) t = t - term;
    } else {
      for (int j = 0; j < 3; ++j) {
        if (velocc[j] == 0.0)
          t = t - ((a.const2 * F12[j]) / omega) / 0.01;
        else
          t = t - (((a.const2 * F12[j]) / omega) / velocc[j]) / narms3;
      }
    }
  }
  tinv[idx] = t;
}

// collision matrix: thread per (n1, n2, l1, l2), l2 fastest, so that the b*b
// band block of R(q1, arm, ., .) read for one arm is contiguous across the
// threads of a warp (one IBZ row n1 per blockIdx.y).  T = double, or float
// for the mixed-precision pipeline (sums in double, stored rounded).  With
// piso (iso=1) the arms off the diagonal take CollisionMatrix_iso's form
// (sub.f90:3387-3570): C = -R1(arm) + R1(q1+arm) + R2(arm) + Piso(n1,l1).
template <class T>
__global__ void collision_kernel(Geometry g, int nibz, int n1_first, const int* mapinv, const int* arm_off,
                                 const int* arm_q, const int* arm_op, const double* opk, const double* Q,
                                 const double* R1, const double* R2, T* CM, size_t ld, const double* piso,
                                 const int4* __restrict__ mesh_m) {
  const int b = g.b, b2 = b * b, nkc = g.nkc;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nibz * b2) return;
  const int n2 = t / b2, l1 = (t / b) % b, l2 = t % b;
  const int nl = blockIdx.y;  // IBZ row local to the range
  const int n1 = n1_first + nl;
  const int q1 = mapinv[n1];
  int m1[3];
  decompose(g, q1, m1);
  const size_t base = (size_t)nl * nkc;  // R arrays are local to the row range
  double blk[9];
  for (int k = 0; k < 9; ++k) blk[k] = 0.0;
  for (int s = arm_off[n2]; s < arm_off[n2 + 1]; ++s) {
    int n0 = arm_q[s];
    double C;
    if (n0 == q1 && l1 == l2) {
      C = -Q[(size_t)nl * b + l1];
    } else {
      // the arm's mesh integers from the table; m1 - m0 + sh and m0 - m1 + sh
      // lie in (-nc, 3nc/2), so two compares wrap them
      const int4 mm = __ldg(mesh_m + n0);
      const int m0[3] = {mm.x, mm.y, mm.z};
      int mp1[3], mp2[3];
      for (int a = 0; a < 3; ++a) {
        const int n = g.nc[a], sh = g.shifted ? n / 2 : 0;
        int v1 = m1[a] - m0[a] + sh, v2 = m0[a] - m1[a] + sh;
        v1 += v1 < 0 ? n : 0;
        v1 -= v1 >= n ? n : 0;
        v2 += v2 < 0 ? n : 0;
        v2 -= v2 >= n ? n : 0;
        mp1[a] = v1;  // q1 - arm
        mp2[a] = v2;  // arm - q1
      }
      int nk3_p1 = compose(g, mp1), nk3_p2 = compose(g, mp2);
      const int bl = l1 * b + l2;
      if (piso) {
        int ins;
        const int nqp = pm_index(g, m1, m0, 1, ins);  // q1 + arm
        C = -R1[(base + n0) * b2 + bl] + R1[(base + nqp) * b2 + bl] + R2[(base + n0) * b2 + bl];
        C = C + piso[(size_t)nl * b + l1];
      } else {
        C = -R1[(base + n0) * b2 + bl] + R1[(base + nk3_p2) * b2 + bl] + 0.5 * R2[(base + n0) * b2 + bl] +
            0.5 * R2[(base + nk3_p1) * b2 + bl];
      }
    }
    const double* op = opk + 9 * arm_op[s];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) blk[i + 3 * j] = blk[i + 3 * j] + (C * op[i + 3 * j]);
  }
  const size_t r0 = 3 * ((size_t)nl * b + l1), c0 = 3 * ((size_t)n2 * b + l2);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) CM[(r0 + i) * ld + c0 + j] = (T)blk[i + 3 * j];
}

// ------------------------------------------------- iterative BTE (job=3)
// F over the whole mesh: Ff[q][l][:] = op_kmatrix(op(q)) F[ibz(q)][l][:]
// (syop_f, sub.f90:2117), op(q) the op of q's arm in kstarsinfbz1 of its
// IBZ point -- what update_mpi's kvecop and get_kvecopn2 pick
__global__ void ffull_kernel(Geometry g, const int* mapibz, const int* full_op, const double* opk, const double* F,
                             double* Ff) {
  const int b = g.b;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.nkc * b) return;
  const int q = e / b, l = e % b;
  const double* f = F + ((size_t)mapibz[q] * b + l) * 3;
  double in[3] = {f[0], f[1], f[2]}, out[3];
  opmul(opk + 9 * full_op[q], in, out);
  double* o = Ff + ((size_t)q * b + l) * 3;
  o[0] = out[0];
  o[1] = out[1];
  o[2] = out[2];
}

// update_mpi, pass 1: a CTA covers one IBZ row and one of kUpdSlices ranges
// of q2.  Its threads walk the row's R1/R1p/R2/R2p blocks element by element
// (coalesced); the block size is a multiple of b*b, so each thread keeps one
// (l1, l) pair and three accumulators.  Per-CTA sums in a fixed order go to
// part[row][slice][l1][xyz].
constexpr int kUpdSlices = 8;

__global__ void update_partial_kernel(Geometry g, int n1_first, const int* mapinv, const double* R1, const double* R1p,
                                      const double* R2, const double* R2p, const double* Ff, double* part) {
  __shared__ double red[256][3];
  const int b = g.b, b2 = b * b, nkc = g.nkc;
  const int nl = blockIdx.y, sl = blockIdx.x;
  const int q1 = mapinv[n1_first + nl];
  int m1[3];
  decompose(g, q1, m1);
  const int t = threadIdx.x, l = t % b;  // l1 = (t / b) % b
  const size_t e0 = (size_t)(sl * nkc / kUpdSlices) * b2, e1 = (size_t)((sl + 1) * nkc / kUpdSlices) * b2;
  const size_t rb = (size_t)nl * nkc * b2;
  double a0 = 0, a1 = 0, a2 = 0;
  for (size_t e = e0 + t; e < e1; e += blockDim.x) {
    const int q = (int)(e / b2);
    int mq[3], ins;
    decompose(g, q, mq);
    const int qp = pm_index(g, m1, mq, 1, ins), qm = pm_index(g, m1, mq, -1, ins);
    const double c1 = R1[rb + e], c1p = R1p[rb + e], c2 = R2[rb + e], c2p = R2p[rb + e];
    const double* fq = Ff + ((size_t)q * b + l) * 3;
    const double* fp = Ff + ((size_t)qp * b + l) * 3;
    const double* fm = Ff + ((size_t)qm * b + l) * 3;
    a0 += c1p * fp[0] - c1 * fq[0] + 0.5 * (c2 * fq[0] + c2p * fm[0]);
    a1 += c1p * fp[1] - c1 * fq[1] + 0.5 * (c2 * fq[1] + c2p * fm[1]);
    a2 += c1p * fp[2] - c1 * fq[2] + 0.5 * (c2 * fq[2] + c2p * fm[2]);
  }
  red[t][0] = a0;
  red[t][1] = a1;
  red[t][2] = a2;
  __syncthreads();
  if (t < 3 * b) {
    const int L1 = t / 3, x = t % 3;
    double A = 0;
    for (int u = 0; u < (int)blockDim.x; ++u)
      if ((u / b) % b == L1) A += red[u][x];
    part[(((size_t)nl * kUpdSlices + sl) * b + L1) * 3 + x] = A;
  }
}

// update_mpi, pass 2: F2 = F_RTA + A/Q, optionally mixed into F
__global__ void update_final_kernel(Geometry g, int n1_first, int nrows, const double* part, const double* Q,
                                    const double* F_RTA, const double* F, double mix, double* Fout) {
  const int b = g.b;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nrows * b * 3) return;
  const int nl = e / (3 * b), l1 = (e / 3) % b, x = e % 3, n1 = n1_first + nl;
  double A = 0;
  for (int sl = 0; sl < kUpdSlices; ++sl) A += part[(((size_t)nl * kUpdSlices + sl) * b + l1) * 3 + x];
  const size_t fi = ((size_t)n1 * b + l1) * 3 + x;
  const double f2 = F_RTA[fi] + A / Q[(size_t)n1 * b + l1];
  Fout[((size_t)nl * b + l1) * 3 + x] = mix > 0 ? F[fi] + mix * (f2 - F[fi]) : f2;
}

// ---------------------------------------------------------------- CG
constexpr int kGemvWarps = 8;
constexpr int kVecThreads = 1024;

struct CgDev {
  double num, den, err;
  int done, iters;
  double bnorm;
};

// y = A x for a row-major A of nrows x n (leading dimension ld) of double or
// float, x and y double; partial[blk] = the block's sum of y*x (and partial_g[blk]
// that of g*x).  A block takes
// kGemvRows rows; its warps split the columns, so each x vector a warp
// loads serves all the rows, and small matrices still give n/kGemvRows
// blocks.  With vec (rows 16-byte aligned) A is read as 16-byte vectors,
// else element-wise.  The products are summed in double.
constexpr int kGemvRows = 4;

template <class T>
struct Vec16;
template <>
struct Vec16<double> {
  using t = double2;
  static constexpr int w = 2;
  __device__ static double at(const double2& v, int i) { return i == 0 ? v.x : v.y; }
};
template <>
struct Vec16<float> {
  using t = float4;
  static constexpr int w = 4;
  __device__ static double at(const float4& v, int i) {
    return (double)(i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w);
  }
};

template <class T>
__global__ void __launch_bounds__(kGemvWarps * 32) gemv_kernel(int nrows, int n, size_t ld, int vec,
                                                               const T* __restrict__ A,
                                                               const double* __restrict__ x, double* __restrict__ y,
                                                               double* partial, const double* g, double* partial_g,
                                                               const CgDev* st) {
  if (st && st->done) return;
  using V = typename Vec16<T>::t;
  constexpr int W = Vec16<T>::w;
  __shared__ double red[kGemvWarps][kGemvRows];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * kGemvRows;
  const T* Ar[kGemvRows];
#pragma unroll
  for (int r = 0; r < kGemvRows; ++r) Ar[r] = A + (size_t)min(row0 + r, nrows - 1) * ld;  // rows past nrows: discarded
  double acc[kGemvRows];
#pragma unroll
  for (int r = 0; r < kGemvRows; ++r) acc[r] = 0.0;
  // this warp's slice of the vectors [v0, v1), then of the scalar tail
  const int nv = vec ? n / W : 0;
  const int per = (nv + kGemvWarps - 1) / kGemvWarps;
  const int v0 = warp * per, v1 = min(nv, v0 + per);
  const double2* x2 = reinterpret_cast<const double2*>(x);
#pragma unroll 2
  for (int v = v0 + lane; v < v1; v += 32) {
    double xv[W];
#pragma unroll
    for (int h = 0; h < W / 2; ++h) {
      const double2 t2 = __ldg(x2 + (size_t)v * (W / 2) + h);
      xv[2 * h] = t2.x;
      xv[2 * h + 1] = t2.y;
    }
    V av[kGemvRows];
#pragma unroll
    for (int r = 0; r < kGemvRows; ++r) av[r] = __ldg(reinterpret_cast<const V*>(Ar[r]) + v);
#pragma unroll
    for (int r = 0; r < kGemvRows; ++r)
#pragma unroll
      for (int i = 0; i < W; ++i) acc[r] = fma(Vec16<T>::at(av[r], i), xv[i], acc[r]);
  }
  for (int j = nv * W + warp * 32 + lane; j < n; j += 32 * kGemvWarps) {
    const double xj = x[j];
#pragma unroll
    for (int r = 0; r < kGemvRows; ++r) acc[r] = fma((double)Ar[r][j], xj, acc[r]);
  }
#pragma unroll
  for (int r = 0; r < kGemvRows; ++r) {
    double v = acc[r];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][r] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double dot = 0.0, gdot = 0.0;
    for (int r = 0; r < kGemvRows && row0 + r < nrows; ++r) {
      double t = 0.0;
      for (int w = 0; w < kGemvWarps; ++w) t += red[w][r];
      y[row0 + r] = t;
      dot += t * x[row0 + r];
      if (g) gdot += g[row0 + r] * x[row0 + r];
    }
    if (partial) partial[blockIdx.x] = dot;
    if (partial_g) partial_g[blockIdx.x] = gdot;
  }
}

__device__ double vblock_sum(double v) {
  __shared__ double red[kVecThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) red[0] = t;
  }
  __syncthreads();
  double r = red[0];
  __syncthreads();
  return r;
}

// grad = A x - b ; conj = -grad  (y holds A x)
__global__ void cg_init_kernel(int n, const double* y, const double* b, double* grad, double* conj, CgDev* st) {
  double bb = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double gr = y[i] - b[i];
    grad[i] = gr;
    conj[i] = -gr;
    bb += b[i] * b[i];
  }
  bb = vblock_sum(bb);
  if (threadIdx.x == 0) {
    st->done = 0;
    st->iters = 0;
    st->err = 9999;
    st->bnorm = sqrt(bb);
  }
}

// One CG iteration after aux = A conj (cg.f90:37-55) in two grid-wide
// kernels of kCgBlocks CTAs.  Every CTA reduces the same per-block partials
// in the same order, so all of them hold the same alpha (and later beta).
constexpr int kCgThreads = 256;
constexpr int kCgBlocksMax = 64;

// alpha = (grad . conj) / (conj . A conj); x -= alpha conj; grad -= alpha aux;
// per-CTA partial sums of x.x, conj.conj, grad_new.grad_new, grad_old.grad_old
__global__ void __launch_bounds__(kCgThreads) cg_update_kernel(int n, const double* aux, const double* pden,
                                                              const double* pnum, int nparts, double* grad,
                                                              const double* conj, double* v0, double* x,
                                                              double* p4, CgDev* st) {
  if (st->done) return;
  double num = 0, den = 0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    num += pnum[i];
    den += pden[i];
  }
  num = vblock_sum(num);
  den = vblock_sum(den);
  const double alpha = num / den;
  double v2 = 0, cc = 0, gg = 0, g2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double gi = grad[i];
    v0[i] = gi;
    double ci = conj[i];
    double xi = x[i] - alpha * ci;
    x[i] = xi;
    double gn = gi - alpha * aux[i];
    grad[i] = gn;
    v2 += xi * xi;
    cc += ci * ci;
    gg += gn * gn;
    g2 += gi * gi;
  }
  v2 = vblock_sum(v2);
  cc = vblock_sum(cc);
  gg = vblock_sum(gg);
  g2 = vblock_sum(g2);
  if (threadIdx.x == 0) {
    p4[0 * kCgBlocksMax + blockIdx.x] = v2;
    p4[1 * kCgBlocksMax + blockIdx.x] = cc;
    p4[2 * kCgBlocksMax + blockIdx.x] = gg;
    p4[3 * kCgBlocksMax + blockIdx.x] = g2;
    if (blockIdx.x == 0) {
      st->num = num;
      st->den = den;
    }
  }
}

// the stop rule; unless it fires, conj = -grad + beta conj with beta = gg/g2
__global__ void __launch_bounds__(kCgThreads) cg_dir_kernel(int n, const double* p4, const double* grad,
                                                           double* conj, CgDev* st, int mode, double tol) {
  if (st->done) return;
  __shared__ double s4[4];
  if (threadIdx.x < 4) {
    double t = 0;
    for (int k = 0; k < (int)gridDim.x; ++k) t += p4[threadIdx.x * kCgBlocksMax + k];
    s4[threadIdx.x] = t;
  }
  __syncthreads();
  const double v2 = s4[0], cc = s4[1], gg = s4[2], g2 = s4[3];
  const double num = st->num, den = st->den;
  double err = mode == ALD_CG_REFERENCE ? (num * num / den / den) * cc / v2 : sqrt(gg) / st->bnorm;
  bool stop = err < tol;
  if (!stop) {
    double beta = gg / g2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      conj[i] = -grad[i] + beta * conj[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iters += 1;
    st->err = err;
    if (stop) st->done = 1;
  }
}

// per-CTA partial sums of aux.conj (den) and grad.conj (num) over full
// vectors, the row-sharded CG's stand-in for the gemv partials
__global__ void __launch_bounds__(256) cg_dots_kernel(int n, const double* aux, const double* conj,
                                                      const double* grad, double* pden, double* pnum,
                                                      const CgDev* st) {
  if (st->done) return;
  __shared__ double red[2][8];
  double d = 0, g = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double c = conj[i];
    d += aux[i] * c;
    g += grad[i] * c;
  }
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_down_sync(0xffffffffu, d, o);
    g += __shfl_down_sync(0xffffffffu, g, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = d;
    red[1][threadIdx.x >> 5] = g;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    pden[blockIdx.x] = a;
    pnum[blockIdx.x] = b;
  }
}

__global__ void cg_fmin_kernel(int n, const double* x, const double* Ax, const double* b, double* out) {
  double s1 = 0, s2 = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s1 += x[i] * Ax[i];
    s2 += x[i] * b[i];
  }
  s1 = vblock_sum(s1);
  s2 = vblock_sum(s2);
  if (threadIdx.x == 0) *out = 0.5 * s1 - s2;
}

}  // namespace

cudaError_t launch_rta_F(const KappaArgs& a, const double* Q, double* FFF, cudaStream_t s) {
  int n = a.nibz * a.geo.b;
  rta_F_kernel<<<(n + 255) / 256, 256, 0, s>>>(a, Q, FFF);
  return cudaGetLastError();
}

size_t kappa_partial_doubles(int b, int narm) {
  return (size_t)b * std::max(1, (narm + kKapThreads - 1) / kKapThreads) * 9;
}

cudaError_t launch_kappa(const KappaArgs& a, const double* F, int averaged, double* kappa_modes, int* err,
                         cudaStream_t s) {
  if (!a.part) return cudaErrorMemoryAllocation;
  const int narm = a.narm;
  const int nblk = std::max(1, (narm + kKapThreads - 1) / kKapThreads);
  kappa_arm_kernel<<<dim3(nblk, a.geo.b), kKapThreads, 0, s>>>(a, F, averaged, narm, err);
  kappa_final_kernel<<<(9 * a.geo.b + 127) / 128, 128, 0, s>>>(a.geo.b, nblk, a.part, kappa_modes);
  return cudaGetLastError();
}

cudaError_t launch_tau_eff(const KappaArgs& a, const double* F, int averaged, double* tauinv_eff,
                           cudaStream_t s) {
  const int n = a.nibz * a.geo.b;
  tau_eff_kernel<<<(n + 127) / 128, 128, 0, s>>>(a, F, averaged, tauinv_eff);
  return cudaGetLastError();
}

cudaError_t launch_ffull(const Geometry& geo, const int* mapibz, const int* full_op, const double* opk,
                         const double* F, double* Ff, cudaStream_t s) {
  const int n = geo.nkc * geo.b;
  ffull_kernel<<<(n + 255) / 256, 256, 0, s>>>(geo, mapibz, full_op, opk, F, Ff);
  return cudaGetLastError();
}

size_t update_part_doubles(const Geometry& geo, int nrows) { return (size_t)nrows * kUpdSlices * geo.b * 3; }

cudaError_t launch_update(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* R1,
                          const double* R1p, const double* R2, const double* R2p, const double* Ff, const double* Q,
                          const double* F_RTA, const double* F, double mix, double* Fout, double* part,
                          cudaStream_t s) {
  const int b2 = geo.b * geo.b;
  if (b2 > 256) return cudaErrorInvalidValue;
  const int threads = b2 * (256 / b2);
  dim3 grid(kUpdSlices, nrows);
  update_partial_kernel<<<grid, threads, 0, s>>>(geo, n1_first, mapinv, R1, R1p, R2, R2p, Ff, part);
  const int n = nrows * geo.b * 3;
  update_final_kernel<<<(n + 255) / 256, 256, 0, s>>>(geo, n1_first, nrows, part, Q, F_RTA, F, mix, Fout);
  return cudaGetLastError();
}

cudaError_t launch_rhs(const KappaArgs& a, double* rhs, cudaStream_t s) {
  int n = a.nibz * a.geo.b;
  rhs_kernel<<<(n + 255) / 256, 256, 0, s>>>(a, rhs);
  return cudaGetLastError();
}

cudaError_t launch_collision(const Geometry& geo, int nibz, int n1_first, int nrows, const int* mapinv,
                             const int* arm_off, const int* arm_q, const int* arm_op, const double* opk,
                             const double* Q, const double* R1, const double* R2, void* CM, size_t ld, int cm_f32,
                             const double* piso, const int* mesh_m, cudaStream_t s) {
  const int nt = nibz * geo.b * geo.b;
  const int4* mm = reinterpret_cast<const int4*>(mesh_m);
  dim3 grid((nt + 127) / 128, nrows);
  if (cm_f32)
    collision_kernel<float><<<grid, 128, 0, s>>>(geo, nibz, n1_first, mapinv, arm_off, arm_q, arm_op, opk, Q, R1, R2,
                                                 static_cast<float*>(CM), ld, piso, mm);
  else
    collision_kernel<double><<<grid, 128, 0, s>>>(geo, nibz, n1_first, mapinv, arm_off, arm_q, arm_op, opk, Q, R1,
                                                  R2, static_cast<double*>(CM), ld, piso, mm);
  return cudaGetLastError();
}

// Conjugate gradients of cg_quadratic on a device matrix.  The iterations
// run as CUDA graphs of kCgChunk iterations each (captured once per problem);
// a device flag turns the rest of a chunk into no-ops once the stop rule
// fires, and the host reads that flag between chunks, so a solve that stops
// after k iterations launches at most k + kCgChunk - 1 of them.
constexpr int kCgChunk = 8;

template <class T>
static cudaError_t capture_cg(int iters, int n, size_t ld, int vec, int nblk, const T* dA, double* dx, CgWork& w, CgDev* st,
                              int mode, double tol, cudaStream_t s, cudaGraphExec_t* out) {
  cudaGraph_t graph = nullptr;
  const int nb = std::min(kCgBlocksMax, (n + kCgThreads - 1) / kCgThreads);
  std::lock_guard<std::mutex> cap(capture_mutex());
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  for (int it = 0; it < iters; ++it) {
    gemv_kernel<T><<<nblk, kGemvWarps * 32, 0, s>>>(n, n, ld, vec, dA, w.conj.p, w.aux.p, w.partial.p, w.grad.p,
                                                     w.pnum.p, st);
    cg_update_kernel<<<nb, kCgThreads, 0, s>>>(n, w.aux.p, w.partial.p, w.pnum.p, nblk, w.grad.p, w.conj.p, w.v0.p,
                                               dx, w.p4.p, st);
    cg_dir_kernel<<<nb, kCgThreads, 0, s>>>(n, w.p4.p, w.grad.p, w.conj.p, st, mode, tol);
  }
  e = cudaStreamEndCapture(s, &graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  return e;
}

template <class T>
static int cg_device_t(int n, size_t ld, const T* dA, const double* db, double* dx, int max_iter, int mode,
                       double tol, int* iters, double* err_out, double* funcmin, cudaStream_t s, CgWork& w,
                       std::string& msg) {
  const int nblk = (n + kGemvRows - 1) / kGemvRows;
  if (ld < (size_t)n) {
    msg = "cg: leading dimension below n";
    return ALD_ERR_ARG;
  }
  const int vec = ((uintptr_t)dA & 15u) == 0 && (ld * sizeof(T)) % 16 == 0;  // rows 16-byte aligned
  if (w.grad.alloc(n) || w.conj.alloc(n) || w.aux.alloc(n) || w.v0.alloc(n) || w.partial.alloc(nblk) ||
      w.pnum.alloc(nblk) || w.p4.alloc(4 * kCgBlocksMax) ||
      w.fmin.alloc(1) || w.st.alloc(sizeof(CgDev)) ||
      (!w.h_done && cudaHostAlloc((void**)&w.h_done, sizeof(int), cudaHostAllocDefault) != cudaSuccess)) {
    msg = "cg: allocation failed";
    return ALD_ERR_NOMEM;
  }
  CgDev* st = reinterpret_cast<CgDev*>(w.st.p);
  gemv_kernel<T><<<nblk, kGemvWarps * 32, 0, s>>>(n, n, ld, vec, dA, dx, w.aux.p, nullptr, nullptr, nullptr,
                                                   nullptr);
  cg_init_kernel<<<1, kVecThreads, 0, s>>>(n, w.aux.p, db, w.grad.p, w.conj.p, st);
  cudaError_t e = cudaSuccess;
  const bool same = w.exec && w.n == n && w.max_iter == max_iter && w.mode == mode && w.tol == tol && w.A == (const void*)dA && w.ld == ld &&
                    w.b == db && w.x == dx;
  const int chunk = max_iter <= 0 ? 1 : (max_iter < kCgChunk ? max_iter : kCgChunk);
  const int tail = max_iter > 0 ? max_iter % chunk : 0;
  if (!same && max_iter > 0) {
    if (w.exec) cudaGraphExecDestroy(w.exec);
    if (w.exec_tail) cudaGraphExecDestroy(w.exec_tail);
    w.exec = w.exec_tail = nullptr;
    e = capture_cg<T>(chunk, n, ld, vec, nblk, dA, dx, w, st, mode, tol, s, &w.exec);
    if (e == cudaSuccess && tail)
      e = capture_cg<T>(tail, n, ld, vec, nblk, dA, dx, w, st, mode, tol, s, &w.exec_tail);
    if (e == cudaSuccess) {
      w.n = n;
      w.max_iter = max_iter;
      w.mode = mode;
      w.tol = tol;
      w.A = dA;
      w.ld = ld;
      w.b = db;
      w.x = dx;
    }
  }
  for (int done = 0; e == cudaSuccess && done < max_iter;) {
    const bool full = max_iter - done >= chunk;
    e = cudaGraphLaunch(full ? w.exec : w.exec_tail, s);
    done += full ? chunk : tail;
    if (e == cudaSuccess && done < max_iter) {
      e = cudaMemcpyAsync(w.h_done, &st->done, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e == cudaSuccess && *w.h_done) break;
    }
  }
  if (e != cudaSuccess) {
    msg = std::string("cg: ") + cudaGetErrorString(e);
    return ALD_ERR_CUDA;
  }
  gemv_kernel<T><<<nblk, kGemvWarps * 32, 0, s>>>(n, n, ld, vec, dA, dx, w.aux.p, nullptr, nullptr, nullptr,
                                                   nullptr);
  cg_fmin_kernel<<<1, kVecThreads, 0, s>>>(n, dx, w.aux.p, db, w.fmin.p);
  CgDev h;
  e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(funcmin, w.fmin.p, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    msg = std::string("cg: ") + cudaGetErrorString(e);
    return ALD_ERR_CUDA;
  }
  *iters = h.iters;
  *err_out = h.err;
  return h.done ? ALD_OK : ALD_WARN_CG_MAXITER;
}

int cg_device(int n, const double* dA, const double* db, double* dx, int max_iter, int mode, double tol, int* iters,
              double* err_out, double* funcmin, cudaStream_t s, CgWork& w, std::string& msg) {
  return cg_device_t<double>(n, (size_t)n, dA, db, dx, max_iter, mode, tol, iters, err_out, funcmin, s, w, msg);
}

// Row-sharded cg_quadratic: this rank holds rows [row0, row0 + nrows) of A
// (row-major, leading dimension ld); x, b and the CG vectors are full and
// replicated.  Per iteration: the local rows of A conj, the all-gather of
// that product (the caller's exchange), then the same update kernels as
// cg_device on every rank, so every rank takes the same steps and stops at
// the same iteration.  No graphs: the exchange runs on the host.
template <class T>
static int cg_rows_t(int n, int row0, int nrows, size_t ld, const T* dA, const double* db, double* dx, int max_iter,
                     int mode, double tol, const CgAllGather& gather, int* iters, double* err_out, double* funcmin,
                     cudaStream_t s, CgWork& w, std::string& msg) {
  const int nblk = (nrows + kGemvRows - 1) / kGemvRows;
  const int nb = std::min(kCgBlocksMax, (n + kCgThreads - 1) / kCgThreads);
  if (w.grad.alloc(n) || w.conj.alloc(n) || w.aux.alloc(n) || w.v0.alloc(n) || w.partial.alloc(nb) ||
      w.pnum.alloc(nb) || w.p4.alloc(4 * kCgBlocksMax) || w.fmin.alloc(1) || w.st.alloc(sizeof(CgDev)) ||
      w.yloc.alloc(std::max(nrows, 1))) {
    msg = "cg: allocation failed";
    return ALD_ERR_NOMEM;
  }
  const int vec = ((uintptr_t)dA & 15u) == 0 && (ld * sizeof(T)) % 16 == 0;
  CgDev* st = reinterpret_cast<CgDev*>(w.st.p);
  auto product = [&](const double* v, const CgDev* stp) -> int {  // aux = A v, all rows
    if (nrows > 0)
      gemv_kernel<T><<<nblk, kGemvWarps * 32, 0, s>>>(nrows, n, ld, vec, dA, v, w.yloc.p, nullptr, nullptr, nullptr,
                                                       stp);
    if (cudaGetLastError() != cudaSuccess) return ALD_ERR_CUDA;
    return gather(w.yloc.p, (size_t)nrows, w.aux.p);
  };
  int r = product(dx, nullptr);
  if (r) {
    msg = "cg: the exchange of A x failed";
    return r;
  }
  cg_init_kernel<<<1, kVecThreads, 0, s>>>(n, w.aux.p, db, w.grad.p, w.conj.p, st);
  CgDev h{};
  for (int it = 0; it < max_iter; ++it) {
    r = product(w.conj.p, nullptr);
    if (r) {
      msg = "cg: the exchange of A conj failed";
      return r;
    }
    cg_dots_kernel<<<nb, 256, 0, s>>>(n, w.aux.p, w.conj.p, w.grad.p, w.partial.p, w.pnum.p, st);
    cg_update_kernel<<<nb, kCgThreads, 0, s>>>(n, w.aux.p, w.partial.p, w.pnum.p, nb, w.grad.p, w.conj.p, w.v0.p, dx,
                                               w.p4.p, st);
    cg_dir_kernel<<<nb, kCgThreads, 0, s>>>(n, w.p4.p, w.grad.p, w.conj.p, st, mode, tol);
    cudaError_t e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      msg = std::string("cg: ") + cudaGetErrorString(e);
      return ALD_ERR_CUDA;
    }
    if (h.done) break;
  }
  r = product(dx, nullptr);
  if (r) {
    msg = "cg: the exchange of A x failed";
    return r;
  }
  cg_fmin_kernel<<<1, kVecThreads, 0, s>>>(n, dx, w.aux.p, db, w.fmin.p);
  cudaError_t e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(funcmin, w.fmin.p, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    msg = std::string("cg: ") + cudaGetErrorString(e);
    return ALD_ERR_CUDA;
  }
  *iters = h.iters;
  *err_out = h.err;
  return h.done ? ALD_OK : ALD_WARN_CG_MAXITER;
}

int cg_device_rows(int n, int row0, int nrows, size_t ld, const void* dA, int a_f32, const double* db, double* dx,
                   int max_iter, int mode, double tol, const CgAllGather& gather, int* iters, double* err_out,
                   double* funcmin, cudaStream_t s, CgWork& w, std::string& msg) {
  (void)row0;
  if (a_f32)
    return cg_rows_t<float>(n, row0, nrows, ld, static_cast<const float*>(dA), db, dx, max_iter, mode, tol, gather,
                            iters, err_out, funcmin, s, w, msg);
  return cg_rows_t<double>(n, row0, nrows, ld, static_cast<const double*>(dA), db, dx, max_iter, mode, tol, gather,
                           iters, err_out, funcmin, s, w, msg);
}

int cg_launched_iterations(int iters, int max_iter) {
  if (max_iter <= 0) return 0;
  const int chunk = max_iter < kCgChunk ? max_iter : kCgChunk;
  const int full = max_iter / chunk, tail = max_iter % chunk;
  const int nfull = std::min(full, (iters + chunk - 1) / chunk);
  int n = nfull * chunk;
  if (nfull == full && tail && iters > full * chunk) n += tail;
  return std::max(n, std::min(iters, max_iter));
}

int cg_device_ld(int n, size_t ld, const void* dA, int a_f32, const double* db, double* dx, int max_iter, int mode,
                 double tol, int* iters, double* err_out, double* funcmin, cudaStream_t s, CgWork& w,
                 std::string& msg) {
  if (a_f32)
    return cg_device_t<float>(n, ld, static_cast<const float*>(dA), db, dx, max_iter, mode, tol, iters, err_out,
                              funcmin, s, w, msg);
  return cg_device_t<double>(n, ld, static_cast<const double*>(dA), db, dx, max_iter, mode, tol, iters, err_out,
                             funcmin, s, w, msg);
}

}  // namespace ald
