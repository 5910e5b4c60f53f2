// Phonon stage on the device: dynamical matrix, Hermitian eigensolver,
// finite-difference group velocities and e(-q) = conj e(q).
//
//   set_dynamical_matrix  THERMACOND/rest.f90:445-556
//   nonanal               THERMACOND/rest.f90:3517-3578
//   diagonalize / ZHEEV   THERMACOND/rest.f90:558-598, zhegv.f:213
//   get_freq              THERMACOND/rest.f90:4319-4445
//   finitedif_vel         THERMACOND/rest.f90:2587-2630
//   get_frequencies       THERMACOND/rest.f90:2230-2398
//   subst_eivecs          THERMACOND/rest.f90:3262-3293
//   distribution / nbe    THERMACOND/sub.f90:1955-1980, extratools.f90:257-285
//
// One CTA owns one matrix (a mesh point or one of its six +-dq
// neighbours) in shared memory: the FC2 sum, the reference's
// hermitisation, the dipole term, then a parallel cyclic (round-robin)
// complex Jacobi in FP64.  Eigenvalues are exact to FP64 rounding; inside
// exactly degenerate subspaces the basis is arbitrary, as it is for ZHEEV.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kThreads = 128;
constexpr int kMaxSweeps = 40;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    red[0] = s;
  }
  __syncthreads();
  s = red[0];
  __syncthreads();
  return s;
}

// round-robin pairing: round r, slot k of n2 (even) indices
__device__ __forceinline__ void rr_pair(int r, int k, int n2, int& p, int& q) {
  auto pos = [&](int i) { return i == 0 ? 0 : ((i - 1 + r) % (n2 - 1)) + 1; };
  int a = pos(k), b = pos(n2 - 1 - k);
  p = min(a, b);
  q = max(a, b);
}

__global__ void __launch_bounds__(kThreads) phonon_kernel(PhononArgs a) {
  extern __shared__ double2 smem[];
  __shared__ double red[kThreads / 32];
  __shared__ double4 rot[64];      // c, s, wx, wy per pair
  __shared__ double2 newdiag[64];  // (app', aqq')
  __shared__ int active[64];
  __shared__ int perm[64];
  __shared__ double lam[64];
  __shared__ int conv;

  const int b = a.geo.b;
  const int bb = b * b;
  const int pt = blockIdx.x / a.ndisp, d = blockIdx.x % a.ndisp;
  double2* A = smem;        // row-major b x b
  double2* V = smem + bb;   // eigenvectors (columns), only for d == 0

  double q[3] = {a.kpc32[3 * pt], a.kpc32[3 * pt + 1], a.kpc32[3 * pt + 2]};
  if (d > 0) {
    int ax = (d - 1) / 2;
    q[ax] = (d & 1) ? q[ax] + a.dq : q[ax] - a.dq;
  }
  // ---------------------------------------------------------- FC2 sum
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int t = a.fc2_off[e]; t < a.fc2_off[e + 1]; ++t) {
      const double* rr = a.rr + 3 * a.fc2_atom[t];
      double x = q[0] * rr[0] + q[1] * rr[1] + q[2] * rr[2];
      double sn, cs;
      sincos(x, &sn, &cs);
      double f = a.fc2_val[t], sq = a.fc2_sqm[t];
      acc.x += (f * cs) / sq;
      acc.y += (f * sn) / sq;
    }
    A[e] = acc;
  }
  __syncthreads();
  // ------------------------------------------ hermitisation (rest.f90:513-544)
  // diagonal: imaginary part dropped only when it is large; off-diagonal
  // pairs averaged for columns up to ndim-1 (the last column is left as is)
  for (int t = threadIdx.x; t < b; t += blockDim.x) {
    double2 v = A[t * b + t];
    if (fabs(v.y) > 9e-4 * fabs(v.x)) A[t * b + t] = make_double2(v.x, 0.0);
  }
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    int t = e / b, j = e % b;
    if (j > t && j <= b - 2) {
      double2 u = A[t * b + j], l = A[j * b + t];
      double mi = (u.y - l.y) / 2, mj = (u.x + l.x) / 2;
      A[t * b + j] = make_double2(mj, mi);
      A[j * b + t] = make_double2(mj, -mi);
    }
  }
  __syncthreads();
  double sim = 0, sre = 0;
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    sim += fabs(A[e].y);
    sre += fabs(A[e].x);
  }
  sim = block_sum(sim, red) / bb;
  sre = block_sum(sre, red) / bb;
  if (sim < sre * 1e-10)
    for (int e = threadIdx.x; e < bb; e += blockDim.x) A[e].y = 0.0;
  __syncthreads();
  // --------------------------------------------------- dipole term (nonanal)
  if (a.born_flag != 0) {
    int nat0 = a.geo.nat0;
    const double* eps = a.born;
    const double* chg = a.born + 9;
    const double* mass = a.born + 9 + 9 * nat0;
    const double* sc = a.born + 9 + 10 * nat0;  // eps_scale, rho2, om0
    double kh[3] = {q[0], q[1], q[2]};
    if (q[0] == 0.0 && q[1] == 0.0 && q[2] == 0.0) kh[0] = kh[1] = kh[2] = 1.0e-10;
    double qeq = (kh[0] * (eps[0] * kh[0] + eps[3] * kh[1] + eps[6] * kh[2]) +
                  kh[1] * (eps[1] * kh[0] + eps[4] * kh[1] + eps[7] * kh[2]) +
                  kh[2] * (eps[2] * kh[0] + eps[5] * kh[1] + eps[8] * kh[2]));
    double q2 = kh[0] * kh[0] + kh[1] * kh[1] + kh[2] * kh[2];
    double ex = exp(-q2 / sc[1]);
    for (int e = threadIdx.x; e < bb; e += blockDim.x) {
      int r = e / b, c = e % b;
      int na = r / 3, i = r % 3, nb = c / 3, j = c % 3;
      const double* za = chg + 9 * na;
      const double* zb = chg + 9 * nb;
      double zag = kh[0] * za[0 + 3 * i] + kh[1] * za[1 + 3 * i] + kh[2] * za[2 + 3 * i];
      double zbg = kh[0] * zb[0 + 3 * j] + kh[1] * zb[1 + 3 * j] + kh[2] * zb[2 + 3 * j];
      A[e].x += zag * zbg / (qeq * sc[0]) / sc[2] / sqrt(mass[na] * mass[nb]) * ex;
    }
    __syncthreads();
  }
  // --------------------- Hermitian matrix of the upper triangle (ZHEEV 'U')
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    int i = e / b, j = e % b;
    if (i == j) A[e].y = 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    int i = e / b, j = e % b;
    if (i > j) A[e] = cconj(A[j * b + i]);
  }
  if (d == 0)
    for (int e = threadIdx.x; e < bb; e += blockDim.x) V[e] = make_double2((e / b) == (e % b) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  // ------------------------------------------------ parallel cyclic Jacobi
  const int n2 = b + (b & 1);
  const int npair = n2 / 2;
  for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
    double off = 0, dia = 0;
    for (int e = threadIdx.x; e < bb; e += blockDim.x) {
      double m2 = A[e].x * A[e].x + A[e].y * A[e].y;
      if (e / b == e % b) dia += m2;
      else off += m2;
    }
    off = block_sum(off, red);
    dia = block_sum(dia, red);
    if (threadIdx.x == 0) conv = (off == 0.0 || off <= 1e-32 * dia);
    __syncthreads();
    if (conv) break;
    for (int r = 0; r < n2 - 1; ++r) {
      for (int k = threadIdx.x; k < npair; k += blockDim.x) {
        int p, qq;
        rr_pair(r, k, n2, p, qq);
        int act = 0;
        double4 R = make_double4(1, 0, 1, 0);
        double2 nd = make_double2(0, 0);
        if (qq < b) {
          double app = A[p * b + p].x, aqq = A[qq * b + qq].x;
          double2 apq = A[p * b + qq];
          double mag = hypot(apq.x, apq.y);
          if (mag > 0.0 && mag > 1e-300) {
            double wx = apq.x / mag, wy = apq.y / mag;
            double th = (aqq - app) / (2 * mag);
            double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1));
            double c = 1 / sqrt(t * t + 1), s = t * c;
            R = make_double4(c, s, wx, wy);
            nd = make_double2(app - t * mag, aqq + t * mag);
            act = 1;
          }
        }
        perm[2 * k] = p;
        perm[2 * k + 1] = qq;
        rot[k] = R;
        newdiag[k] = nd;
        active[k] = act;
      }
      __syncthreads();
      // columns: A <- A J, V <- V J
      for (int e = threadIdx.x; e < npair * b; e += blockDim.x) {
        int k = e / b, i = e % b;
        if (!active[k]) continue;
        int p = perm[2 * k], qq = perm[2 * k + 1];
        double4 R = rot[k];
        double2 wb = make_double2(R.z, -R.w);  // conj(w)
        double2 aip = A[i * b + p], aiq = A[i * b + qq];
        double2 t1 = cmul(wb, aiq);
        A[i * b + p] = make_double2(R.x * aip.x - R.y * t1.x, R.x * aip.y - R.y * t1.y);
        A[i * b + qq] = make_double2(R.y * aip.x + R.x * t1.x, R.y * aip.y + R.x * t1.y);
        if (d == 0) {
          double2 vip = V[i * b + p], viq = V[i * b + qq];
          double2 t2 = cmul(wb, viq);
          V[i * b + p] = make_double2(R.x * vip.x - R.y * t2.x, R.x * vip.y - R.y * t2.y);
          V[i * b + qq] = make_double2(R.y * vip.x + R.x * t2.x, R.y * vip.y + R.x * t2.y);
        }
      }
      __syncthreads();
      // rows: A <- J^H A
      for (int e = threadIdx.x; e < npair * b; e += blockDim.x) {
        int k = e / b, j = e % b;
        if (!active[k]) continue;
        int p = perm[2 * k], qq = perm[2 * k + 1];
        double4 R = rot[k];
        double2 w = make_double2(R.z, R.w);
        double2 apj = A[p * b + j], aqj = A[qq * b + j];
        double2 t1 = cmul(w, aqj);
        A[p * b + j] = make_double2(R.x * apj.x - R.y * t1.x, R.x * apj.y - R.y * t1.y);
        A[qq * b + j] = make_double2(R.y * apj.x + R.x * t1.x, R.y * apj.y + R.x * t1.y);
      }
      __syncthreads();
      for (int k = threadIdx.x; k < npair; k += blockDim.x) {
        if (!active[k]) continue;
        int p = perm[2 * k], qq = perm[2 * k + 1];
        A[p * b + p] = make_double2(newdiag[k].x, 0.0);
        A[qq * b + qq] = make_double2(newdiag[k].y, 0.0);
        A[p * b + qq] = make_double2(0.0, 0.0);
        A[qq * b + p] = make_double2(0.0, 0.0);
      }
      __syncthreads();
    }
  }
  // ---------------------------------------------------------- ordering
  // get_freq: ascending signed eigenvalues (ZHEEV order, then `sort`),
  // eival = |lambda|; get_frequencies then sorts the |lambda| once more and
  // permutes the eigenvectors (velocities keep the first order).
  __shared__ int ord[64], ord2[64];
  __shared__ double lab[64];
  if (threadIdx.x == 0) {
    for (int i = 0; i < b; ++i) {
      lam[i] = A[i * b + i].x;
      ord[i] = i;
    }
    for (int i = 0; i < b; ++i)  // exchange sort of extratools.f90:154-175
      for (int j = i + 1; j < b; ++j)
        if (lam[ord[i]] > lam[ord[j]]) {
          int t = ord[i];
          ord[i] = ord[j];
          ord[j] = t;
        }
    for (int i = 0; i < b; ++i) {
      lab[i] = fabs(lam[ord[i]]);
      ord2[i] = i;
    }
    for (int i = 0; i < b; ++i)
      for (int j = i + 1; j < b; ++j)
        if (lab[ord2[i]] > lab[ord2[j]]) {
          int t = ord2[i];
          ord2[i] = ord2[j];
          ord2[j] = t;
        }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < b; i += blockDim.x) a.w2_all[((size_t)pt * a.ndisp + d) * b + i] = lab[i];
  if (d == 0) {
    // eigenvector of final band l: column ord[ord2[l]]; pure-imaginary fix
    for (int l = threadIdx.x >> 5; l < b; l += blockDim.x >> 5) {
      int col = ord[ord2[l]];
      double sre2 = 0;
      for (int c = threadIdx.x & 31; c < b; c += 32) sre2 += fabs(V[c * b + col].x);
      for (int o = 16; o > 0; o >>= 1) sre2 += __shfl_xor_sync(0xffffffffu, sre2, o);
      bool rot90 = sre2 < 1e-3;
      for (int c = threadIdx.x & 31; c < b; c += 32) {
        double2 v = V[c * b + col];
        if (rot90) v = make_double2(-v.y, v.x);
        size_t o = (((size_t)pt * b + l) * b + c) * 2;
        a.evec[o] = v.x;
        a.evec[o + 1] = v.y;
      }
    }
    for (int l = threadIdx.x; l < b; l += blockDim.x) a.w2[(size_t)pt * b + l] = lab[ord2[l]];
  }
}

// ------------------------------------------------------------------
// Small cells (b <= 12): G matrices per warp (32/G lanes each: G = 4 up to 4
// bands, 2 up to 8, else 1), kPhWarps warps per CTA, synchronised with
// __syncwarp only.  Every lane runs the same sequence of __syncwarp and
// shuffle calls: a matrix that has converged (or a slot past the last
// matrix) just stops doing work.  The same arithmetic as phonon_kernel
// element by element (FC2 sum in the file's term order, hermitisation,
// dipole term, cyclic Jacobi rounds, sorts); the q.R phase of every distinct
// FC2 atom is evaluated once per matrix instead of once per matrix element,
// and the sweep's off-diagonal and diagonal norms are sums over the matrix's
// lanes.  Each term keeps the reference's (f cos)/sqrt(m m) rounding: the
// acoustic modes at Gamma are rounding residues of these sums, and a sum
// rounded differently can reach exactly zero.
constexpr int kPhWarps = 4;
constexpr int kPhBMax = 12;

template <int LPM>
__device__ __forceinline__ double group_sum(double v) {  // over the LPM aligned lanes of a matrix
  for (int o = LPM / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int G>
__global__ void __launch_bounds__(kPhWarps * 32) phonon_warp_kernel(PhononArgs a, int nmat) {
  constexpr int LPM = 32 / G;  // lanes per matrix
  constexpr int NS = kPhWarps * G;  // matrix slots per CTA
  extern __shared__ double2 smem[];
  __shared__ double4 s_rot[NS][kPhBMax / 2];
  __shared__ double2 s_nd[NS][kPhBMax / 2];
  __shared__ int s_act[NS][kPhBMax / 2];
  __shared__ int s_perm[NS][kPhBMax];
  __shared__ double s_lam[NS][kPhBMax], s_lab[NS][kPhBMax];
  __shared__ int s_ord[NS][kPhBMax], s_ord2[NS][kPhBMax];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sg = lane / LPM, sl = lane % LPM, slot = warp * G + sg;
  const int m0 = (blockIdx.x * kPhWarps + warp) * G;
  if (m0 >= nmat) return;  // the whole warp; nothing below synchronises the CTA
  const int m = m0 + sg;
  const bool valid = m < nmat;  // a slot past the last matrix repeats the last one and writes nothing
  const int mc = valid ? m : nmat - 1;
  const int b = a.geo.b, bb = b * b;
  const int pt = mc / a.ndisp, d = mc % a.ndisp;
  double2* A = smem + (size_t)slot * (2 * bb + a.nuniq);
  double2* V = A + bb;
  double2* ph = V + bb;
  double4* rot = s_rot[slot];
  double2* newdiag = s_nd[slot];
  int* active = s_act[slot];
  int* perm = s_perm[slot];

  double q[3] = {a.kpc32[3 * pt], a.kpc32[3 * pt + 1], a.kpc32[3 * pt + 2]};
  if (d > 0) {
    int ax = (d - 1) / 2;
    q[ax] = (d & 1) ? q[ax] + a.dq : q[ax] - a.dq;
  }
  // ------------------------------------------- phases, then the FC2 sum
  for (int u = sl; u < a.nuniq; u += LPM) {
    const double* rr = a.rr + 3 * a.fc2_uatom[u];
    double x = q[0] * rr[0] + q[1] * rr[1] + q[2] * rr[2];
    double sn, cs;
    sincos(x, &sn, &cs);
    ph[u] = make_double2(cs, sn);
  }
  __syncwarp();
  for (int e = sl; e < bb; e += LPM) {
    double2 acc = make_double2(0.0, 0.0);
    for (int t = a.fc2_off[e]; t < a.fc2_off[e + 1]; ++t) {
      const double2 p = ph[a.fc2_uidx[t]];
      double f = a.fc2_val[t], sq = a.fc2_sqm[t];
      acc.x += (f * p.x) / sq;
      acc.y += (f * p.y) / sq;
    }
    A[e] = acc;
  }
  __syncwarp();
  // ------------------------------------------ hermitisation (rest.f90:513-544)
  for (int t = sl; t < b; t += LPM) {
    double2 v = A[t * b + t];
    if (fabs(v.y) > 9e-4 * fabs(v.x)) A[t * b + t] = make_double2(v.x, 0.0);
  }
  __syncwarp();
  for (int e = sl; e < bb; e += LPM) {
    int t = e / b, j = e % b;
    if (j > t && j <= b - 2) {
      double2 u = A[t * b + j], l = A[j * b + t];
      double mi = (u.y - l.y) / 2, mj = (u.x + l.x) / 2;
      A[t * b + j] = make_double2(mj, mi);
      A[j * b + t] = make_double2(mj, -mi);
    }
  }
  __syncwarp();
  double sim = 0, sre = 0;
  for (int e = sl; e < bb; e += LPM) {
    sim += fabs(A[e].y);
    sre += fabs(A[e].x);
  }
  sim = group_sum<LPM>(sim) / bb;
  sre = group_sum<LPM>(sre) / bb;
  if (sim < sre * 1e-10)
    for (int e = sl; e < bb; e += LPM) A[e].y = 0.0;
  __syncwarp();
  // --------------------------------------------------- dipole term (nonanal)
  if (a.born_flag != 0) {
    int nat0 = a.geo.nat0;
    const double* eps = a.born;
    const double* chg = a.born + 9;
    const double* mass = a.born + 9 + 9 * nat0;
    const double* sc = a.born + 9 + 10 * nat0;  // eps_scale, rho2, om0
    double kh[3] = {q[0], q[1], q[2]};
    if (q[0] == 0.0 && q[1] == 0.0 && q[2] == 0.0) kh[0] = kh[1] = kh[2] = 1.0e-10;
    double qeq = (kh[0] * (eps[0] * kh[0] + eps[3] * kh[1] + eps[6] * kh[2]) +
                  kh[1] * (eps[1] * kh[0] + eps[4] * kh[1] + eps[7] * kh[2]) +
                  kh[2] * (eps[2] * kh[0] + eps[5] * kh[1] + eps[8] * kh[2]));
    double q2 = kh[0] * kh[0] + kh[1] * kh[1] + kh[2] * kh[2];
    double ex = exp(-q2 / sc[1]);
    for (int e = sl; e < bb; e += LPM) {
      int r = e / b, c = e % b;
      int na = r / 3, i = r % 3, nb = c / 3, j = c % 3;
      const double* za = chg + 9 * na;
      const double* zb = chg + 9 * nb;
      double zag = kh[0] * za[0 + 3 * i] + kh[1] * za[1 + 3 * i] + kh[2] * za[2 + 3 * i];
      double zbg = kh[0] * zb[0 + 3 * j] + kh[1] * zb[1 + 3 * j] + kh[2] * zb[2 + 3 * j];
      A[e].x += zag * zbg / (qeq * sc[0]) / sc[2] / sqrt(mass[na] * mass[nb]) * ex;
    }
    __syncwarp();
  }
  // --------------------- Hermitian matrix of the upper triangle (ZHEEV 'U')
  for (int e = sl; e < bb; e += LPM)
    if (e / b == e % b) A[e].y = 0.0;
  __syncwarp();
  for (int e = sl; e < bb; e += LPM) {
    int i = e / b, j = e % b;
    if (i > j) A[e] = cconj(A[j * b + i]);
  }
  if (d == 0)
    for (int e = sl; e < bb; e += LPM) V[e] = make_double2((e / b) == (e % b) ? 1.0 : 0.0, 0.0);
  __syncwarp();
  // ------------------------------------------------ parallel cyclic Jacobi
  const int n2 = b + (b & 1);
  const int npair = n2 / 2;
  bool conv = false;  // uniform over the matrix's lanes
  for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
    double off = 0, dia = 0;
    for (int e = sl; e < bb; e += LPM) {
      double m2 = A[e].x * A[e].x + A[e].y * A[e].y;
      if (e / b == e % b) dia += m2;
      else off += m2;
    }
    off = group_sum<LPM>(off);
    dia = group_sum<LPM>(dia);
    if (!conv && (off == 0.0 || off <= 1e-32 * dia)) conv = true;
    if (__all_sync(0xffffffffu, conv)) break;  // warp-uniform
    for (int r = 0; r < n2 - 1; ++r) {
      if (!conv && sl < npair) {
        const int k = sl;
        int p, qq;
        rr_pair(r, k, n2, p, qq);
        int act = 0;
        double4 R = make_double4(1, 0, 1, 0);
        double2 nd = make_double2(0, 0);
        if (qq < b) {
          double app = A[p * b + p].x, aqq = A[qq * b + qq].x;
          double2 apq = A[p * b + qq];
          double mag = hypot(apq.x, apq.y);
          if (mag > 0.0 && mag > 1e-300) {
            double wx = apq.x / mag, wy = apq.y / mag;
            double th = (aqq - app) / (2 * mag);
            double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1));
            double c = 1 / sqrt(t * t + 1), s = t * c;
            R = make_double4(c, s, wx, wy);
            nd = make_double2(app - t * mag, aqq + t * mag);
            act = 1;
          }
        }
        perm[2 * k] = p;
        perm[2 * k + 1] = qq;
        rot[k] = R;
        newdiag[k] = nd;
        active[k] = act;
      }
      __syncwarp();
      // columns: A <- A J, V <- V J
      if (!conv)
        for (int e = sl; e < npair * b; e += LPM) {
          int k = e / b, i = e % b;
          if (!active[k]) continue;
          int p = perm[2 * k], qq = perm[2 * k + 1];
          double4 R = rot[k];
          double2 wb = make_double2(R.z, -R.w);  // conj(w)
          double2 aip = A[i * b + p], aiq = A[i * b + qq];
          double2 t1 = cmul(wb, aiq);
          A[i * b + p] = make_double2(R.x * aip.x - R.y * t1.x, R.x * aip.y - R.y * t1.y);
          A[i * b + qq] = make_double2(R.y * aip.x + R.x * t1.x, R.y * aip.y + R.x * t1.y);
          if (d == 0) {
            double2 vip = V[i * b + p], viq = V[i * b + qq];
            double2 t2 = cmul(wb, viq);
            V[i * b + p] = make_double2(R.x * vip.x - R.y * t2.x, R.x * vip.y - R.y * t2.y);
            V[i * b + qq] = make_double2(R.y * vip.x + R.x * t2.x, R.y * vip.y + R.x * t2.y);
          }
        }
      __syncwarp();
      // rows: A <- J^H A
      if (!conv)
        for (int e = sl; e < npair * b; e += LPM) {
          int k = e / b, j = e % b;
          if (!active[k]) continue;
          int p = perm[2 * k], qq = perm[2 * k + 1];
          double4 R = rot[k];
          double2 w = make_double2(R.z, R.w);
          double2 apj = A[p * b + j], aqj = A[qq * b + j];
          double2 t1 = cmul(w, aqj);
          A[p * b + j] = make_double2(R.x * apj.x - R.y * t1.x, R.x * apj.y - R.y * t1.y);
          A[qq * b + j] = make_double2(R.y * apj.x + R.x * t1.x, R.y * apj.y + R.x * t1.y);
        }
      __syncwarp();
      if (!conv && sl < npair && active[sl]) {
        const int k = sl;
        int p = perm[2 * k], qq = perm[2 * k + 1];
        A[p * b + p] = make_double2(newdiag[k].x, 0.0);
        A[qq * b + qq] = make_double2(newdiag[k].y, 0.0);
        A[p * b + qq] = make_double2(0.0, 0.0);
        A[qq * b + p] = make_double2(0.0, 0.0);
      }
      __syncwarp();
    }
  }
  // ---------------------------------------------------------- ordering
  double* lam = s_lam[slot];
  double* lab = s_lab[slot];
  int* ord = s_ord[slot];
  int* ord2 = s_ord2[slot];
  if (sl == 0) {
    for (int i = 0; i < b; ++i) {
      lam[i] = A[i * b + i].x;
      ord[i] = i;
    }
    for (int i = 0; i < b; ++i)  // exchange sort of extratools.f90:154-175
      for (int j = i + 1; j < b; ++j)
        if (lam[ord[i]] > lam[ord[j]]) {
          int t = ord[i];
          ord[i] = ord[j];
          ord[j] = t;
        }
    for (int i = 0; i < b; ++i) {
      lab[i] = fabs(lam[ord[i]]);
      ord2[i] = i;
    }
    for (int i = 0; i < b; ++i)
      for (int j = i + 1; j < b; ++j)
        if (lab[ord2[i]] > lab[ord2[j]]) {
          int t = ord2[i];
          ord2[i] = ord2[j];
          ord2[j] = t;
        }
  }
  __syncwarp();
  if (valid)
    for (int i = sl; i < b; i += LPM) a.w2_all[((size_t)pt * a.ndisp + d) * b + i] = lab[i];
  for (int l = 0; l < b; ++l) {  // every lane: the sums below shuffle over the matrix's lanes
    int col = ord[ord2[l]];
    double sre2 = 0;
    if (d == 0)
      for (int c = sl; c < b; c += LPM) sre2 += fabs(V[c * b + col].x);
    sre2 = group_sum<LPM>(sre2);
    bool rot90 = sre2 < 1e-3;
    if (valid && d == 0)
      for (int c = sl; c < b; c += LPM) {
        double2 v = V[c * b + col];
        if (rot90) v = make_double2(-v.y, v.x);
        size_t o = (((size_t)pt * b + l) * b + c) * 2;
        a.evec[o] = v.x;
        a.evec[o + 1] = v.y;
      }
  }
  if (valid && d == 0)
    for (int l = sl; l < b; l += LPM) a.w2[(size_t)pt * b + l] = lab[ord2[l]];
}

// finite differences use the get_freq order (before the second sort)
__global__ void phonon_post_kernel(Geometry geo, const double* w2_all, double dq, double cnst, double* vel) {
  int b = geo.b;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= geo.nkc * b) return;
  int pt = idx / b, l = idx % b;
  const double* W = w2_all + (size_t)pt * 7 * b;
  // evl0 of finitedif_vel: |lambda| in get_freq order
  double w0 = W[l];
  const double pi = PhysConst::pi;
  for (int i = 0; i < 3; ++i) {
    double wp = W[(1 + 2 * i) * b + l], wm = W[(2 + 2 * i) * b + l];
    vel[(size_t)idx * 3 + i] = (wp - wm) / 2 / dq / 2 / sqrt(w0) * cnst * 1e-8 * 2 * pi;
  }
}

__global__ void subst_kernel(int b, const int* src, const int* dst, int n, double* evec) {
  size_t bb2 = (size_t)b * b;
  size_t total = (size_t)n * bb2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    size_t k = e / bb2, r = e % bb2;
    const double* s = evec + ((size_t)src[k] * bb2 + r) * 2;
    double* t = evec + ((size_t)dst[k] * bb2 + r) * 2;
    t[0] = s[0];
    t[1] = -s[1];
  }
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

__global__ void freq_dist_kernel(Geometry geo, const double* w2, double cnst, double temp, int classical,
                                 double* freq, double* dist, int* err) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= geo.nkc * geo.b) return;
  double f = sqrt(w2[idx]) * cnst;
  freq[idx] = f;
  dist[idx] = nbe_dev(f, temp, classical, err);
}

}  // namespace

cudaError_t launch_phonons(const PhononArgs& a, cudaStream_t s) {
  int b = a.geo.b;
  const int G = b <= 4 ? 4 : (b <= 8 ? 2 : 1);  // matrices per warp
  const size_t smw = (size_t)kPhWarps * G * (2 * (size_t)b * b + a.nuniq) * sizeof(double2);
  if (b <= kPhBMax && smw <= 160 * 1024) {
    const int nmat = a.geo.nkc * a.ndisp;
    const int per_cta = kPhWarps * G;
    cudaError_t e = cudaSuccess;
#define ALD_PHW(GG)                                                                                            \
  if (smw > 48 * 1024)                                                                                         \
    e = raise_smem_limit((const void*)phonon_warp_kernel<GG>, smw);                                            \
  if (e != cudaSuccess) return e;                                                                              \
  phonon_warp_kernel<GG><<<(nmat + per_cta - 1) / per_cta, kPhWarps * 32, smw, s>>>(a, nmat);
    if (G == 4) {
      ALD_PHW(4)
    } else if (G == 2) {
      ALD_PHW(2)
    } else {
      ALD_PHW(1)
    }
#undef ALD_PHW
    return cudaGetLastError();
  }
  size_t sm = 2 * (size_t)b * b * sizeof(double2);
  if (b > 64) return cudaErrorInvalidValue;
  if (sm > 48 * 1024) {
    cudaError_t e = raise_smem_limit((const void*)phonon_kernel, sm);
    if (e != cudaSuccess) return e;
  }
  phonon_kernel<<<a.geo.nkc * a.ndisp, kThreads, sm, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_phonon_post(const Geometry& geo, const double* w2_all, double dq, double cnst, double* vel,
                               cudaStream_t s) {
  int n = geo.nkc * geo.b;
  phonon_post_kernel<<<(n + 255) / 256, 256, 0, s>>>(geo, w2_all, dq, cnst, vel);
  return cudaGetLastError();
}

cudaError_t launch_subst_eivecs(const Geometry& geo, const int* src, const int* dst, int n, double* evec,
                                cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  size_t total = (size_t)n * geo.b * geo.b;
  int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
  subst_kernel<<<blocks, 256, 0, s>>>(geo.b, src, dst, n, evec);
  return cudaGetLastError();
}

cudaError_t launch_freq_dist(const Geometry& geo, const double* w2, double cnst, double temp, int classical,
                             double* freq, double* dist, int* err, cudaStream_t s) {
  int n = geo.nkc * geo.b;
  freq_dist_kernel<<<(n + 255) / 256, 256, 0, s>>>(geo, w2, cnst, temp, classical, freq, dist, err);
  return cudaGetLastError();
}

}  // namespace ald
