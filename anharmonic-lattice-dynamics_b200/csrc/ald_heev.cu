// Hermitian eigensolver for large cells (more than 64 bands, up to 256):
// Householder tridiagonalisation, implicit QL with Wilkinson shifts and the
// back-transformation, in FP64, one CTA per matrix.
//
// Replaces, for one mesh point or one of its six +-dq neighbours:
//   set_dynamical_matrix  THERMACOND/rest.f90:445-556 (+ nonanal rest.f90:3517-3578)
//   diagonalize / ZHEEV   THERMACOND/rest.f90:558-598, zhegv.f:213
//   get_freq              THERMACOND/rest.f90:4319-4445 (the two sorts, the x i fix)
// ZHEEV itself reduces to a real tridiagonal matrix by Householder
// reflections and runs implicit QL/QR on it; this kernel does the same steps
// (Golub & Van Loan, "Matrix Computations", 8.3; the implicit QL sweep of
// Bowdler, Martin, Reinsch & Wilkinson, Numer. Math. 11 (1968) 293), so
// eigenvalues agree to FP64 rounding and eigenvectors up to a phase (a basis
// inside exactly degenerate subspaces).
//
// The matrix does not fit in shared memory (192 bands: 590 KB), so each
// resident CTA owns a workspace slot in global memory (L2-resident):
//   A  b*b complex, row-major: D(q), then the Householder vectors in the
//      columns below the diagonal
//   Z  b*b real, column-major: eigenvectors of the tridiagonal matrix
//   V  b*b complex, [component][vector]: the back-transformed eigenvectors
// A persistent grid loops over the matrices.  The six +-dq matrices of a
// point need eigenvalues only: no Z, no V.
//
// Work per matrix: tridiagonalisation (4/3) b^3 complex multiply-adds, each
// step a warp-per-row matrix-vector product and a rank-2 update of the
// trailing block; QL: the rotations of a sweep are formed by one thread
// (a serial recurrence) and applied to the rows of Z by all threads; the
// back-transformation b^3 complex multiply-adds, one eigenvector per thread.
// The QL loop is bounded: 60 sweeps per eigenvalue, after which bit 5 of the
// error flag is set.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kHeThreads = 256;
constexpr int kHeMaxB = 256;
constexpr int kQlMaxIter = 60;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ double he_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
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

// D(q) of one matrix into A (row-major, full Hermitian from the upper
// triangle): the FC2 sum in the file's term order, the hermitisation of
// rest.f90:513-544, the real-part-only rule, the dipole term and ZHEEV's 'U'
// triangle -- the steps of the shared-memory Jacobi kernel, on global memory
__device__ void he_dynmat(const PhononArgs& a, const double* q, double2* A, double* red) {
  const int b = a.geo.b, bb = b * b;
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int t = a.fc2_off[e]; t < a.fc2_off[e + 1]; ++t) {
      const double* rr = a.rr + 3 * a.fc2_atom[t];
      const double x = q[0] * rr[0] + q[1] * rr[1] + q[2] * rr[2];
      double sn, cs;
      sincos(x, &sn, &cs);
      const double f = a.fc2_val[t], sq = a.fc2_sqm[t];
      acc.x += (f * cs) / sq;
      acc.y += (f * sn) / sq;
    }
    A[e] = acc;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < b; t += blockDim.x) {
    const double2 v = A[t * b + t];
    if (fabs(v.y) > 9e-4 * fabs(v.x)) A[t * b + t] = make_double2(v.x, 0.0);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    const int t = e / b, j = e % b;
    if (j > t && j <= b - 2) {
      const double2 u = A[t * b + j], l = A[j * b + t];
      const double mi = (u.y - l.y) / 2, mj = (u.x + l.x) / 2;
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
  sim = he_block_sum(sim, red) / bb;
  sre = he_block_sum(sre, red) / bb;
  if (sim < sre * 1e-10)
    for (int e = threadIdx.x; e < bb; e += blockDim.x) A[e].y = 0.0;
  __syncthreads();
  if (a.born_flag != 0) {
    const int nat0 = a.geo.nat0;
    const double* eps = a.born;
    const double* chg = a.born + 9;
    const double* mass = a.born + 9 + 9 * nat0;
    const double* sc = a.born + 9 + 10 * nat0;  // eps_scale, rho2, om0
    double kh[3] = {q[0], q[1], q[2]};
    if (q[0] == 0.0 && q[1] == 0.0 && q[2] == 0.0) kh[0] = kh[1] = kh[2] = 1.0e-10;
    const double qeq = (kh[0] * (eps[0] * kh[0] + eps[3] * kh[1] + eps[6] * kh[2]) +
                        kh[1] * (eps[1] * kh[0] + eps[4] * kh[1] + eps[7] * kh[2]) +
                        kh[2] * (eps[2] * kh[0] + eps[5] * kh[1] + eps[8] * kh[2]));
    const double q2 = kh[0] * kh[0] + kh[1] * kh[1] + kh[2] * kh[2];
    const double ex = exp(-q2 / sc[1]);
    for (int e = threadIdx.x; e < bb; e += blockDim.x) {
      const int r = e / b, c = e % b;
      const int na = r / 3, i = r % 3, nb = c / 3, j = c % 3;
      const double* za = chg + 9 * na;
      const double* zb = chg + 9 * nb;
      const double zag = kh[0] * za[0 + 3 * i] + kh[1] * za[1 + 3 * i] + kh[2] * za[2 + 3 * i];
      const double zbg = kh[0] * zb[0 + 3 * j] + kh[1] * zb[1 + 3 * j] + kh[2] * zb[2 + 3 * j];
      A[e].x += zag * zbg / (qeq * sc[0]) / sc[2] / sqrt(mass[na] * mass[nb]) * ex;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < b; i += blockDim.x) A[i * b + i].y = 0.0;
  __syncthreads();
  for (int e = threadIdx.x; e < bb; e += blockDim.x) {
    const int i = e / b, j = e % b;
    if (i > j) A[e] = cconj(A[j * b + i]);
  }
  __syncthreads();
}

struct HeShared {
  double2 v[kHeMaxB];      // Householder vector of the current step
  double2 p[kHeMaxB];      // A v, then w
  double2 dl[kHeMaxB];     // diagonal phases of the real tridiagonal form
  double d[kHeMaxB], e[kHeMaxB], tau[kHeMaxB];
  double rc[kHeMaxB], rs[kHeMaxB];  // rotations of one QL sweep
  double lab[kHeMaxB];
  int ord[kHeMaxB], ord2[kHeMaxB];
  double red[kHeThreads / 32];
  double2 kred[kHeThreads / 32];
  int cmd, lo, hi;
};

__host__ __device__ inline size_t heev_slot_doubles(int b) {
  const size_t bb = (size_t)b * b;
  return 5 * bb + (bb & 1);
}

__global__ void __launch_bounds__(kHeThreads) heev_kernel(PhononArgs a, int nmat) {
  __shared__ HeShared S;
  const int b = a.geo.b, bb = b * b;
  const int tid = threadIdx.x, nth = blockDim.x, warp = tid >> 5, lane = tid & 31, nwarp = nth >> 5;
  // slot layout (doubles): A at 0, V at 2 bb, Z at 4 bb; the stride keeps
  // every slot 16-byte aligned
  double* slot = a.he_work + (size_t)blockIdx.x * heev_slot_doubles(b);
  double2* A = reinterpret_cast<double2*>(slot);
  double2* V = A + bb;
  double* Z = slot + (size_t)4 * bb;
  for (int mat = blockIdx.x; mat < nmat; mat += gridDim.x) {
    const int pt = mat / a.ndisp, dsp = mat % a.ndisp;
    const bool vecs = dsp == 0;
    double q[3] = {a.kpc32[3 * pt], a.kpc32[3 * pt + 1], a.kpc32[3 * pt + 2]};
    if (dsp > 0) {
      const int ax = (dsp - 1) / 2;
      q[ax] = (dsp & 1) ? q[ax] + a.dq : q[ax] - a.dq;
    }
    he_dynmat(a, q, A, S.red);
    // ------------------------------------------------ tridiagonalisation
    // step k: x = A[k+1.., k]; H = I - tau v v^H with v = x + ph |x| e1,
    // ph = x0/|x0|, tau = 1/(|x| (|x| + |x0|)), so H x = -ph |x| e1 and the
    // subdiagonal entry becomes eps_k = -ph |x|.  A22 <- H A22 H through
    // p = tau A22 v, w = p - (tau/2)(v^H p) v, A22 -= v w^H + w v^H.
    for (int k = 0; k + 2 < b; ++k) {
      const int m = b - k - 1;  // length of x
      double xs = 0;
      for (int i = 2 + tid; i <= m; i += nth) {
        const double2 x = A[(size_t)(k + i) * b + k];
        xs += x.x * x.x + x.y * x.y;
      }
      xs = he_block_sum(xs, S.red);
      const double2 alpha = A[(size_t)(k + 1) * b + k];
      const double an = hypot(alpha.x, alpha.y);
      if (xs == 0.0) {  // nothing below the subdiagonal: no reflection, eps_k = alpha
        if (tid == 0) {
          S.tau[k] = 0.0;
          S.dl[k] = alpha;
        }
        __syncthreads();
        continue;
      }
      const double nrm = sqrt(an * an + xs);
      const double2 ph = an > 0.0 ? make_double2(alpha.x / an, alpha.y / an) : make_double2(1.0, 0.0);
      const double tau = 1.0 / (nrm * (nrm + an));
      for (int i = tid; i < m; i += nth) {
        double2 v = A[(size_t)(k + 1 + i) * b + k];
        if (i == 0) v = make_double2(ph.x * (an + nrm), ph.y * (an + nrm));
        S.v[i] = v;
        A[(size_t)(k + 1 + i) * b + k] = v;  // kept for the back-transformation
      }
      if (tid == 0) {
        S.tau[k] = tau;
        S.dl[k] = make_double2(-ph.x * nrm, -ph.y * nrm);  // eps_k, turned into a phase below
      }
      __syncthreads();
      // p = tau A22 v: one warp per row, lanes over the columns
      for (int i = warp; i < m; i += nwarp) {
        const double2* Ar = A + (size_t)(k + 1 + i) * b + (k + 1);
        double2 s = make_double2(0.0, 0.0);
        for (int j = lane; j < m; j += 32) {
          const double2 x = Ar[j], v = S.v[j];
          s.x = fma(x.x, v.x, fma(-x.y, v.y, s.x));
          s.y = fma(x.x, v.y, fma(x.y, v.x, s.y));
        }
        for (int o = 16; o > 0; o >>= 1) {
          s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
          s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
        }
        if (lane == 0) S.p[i] = make_double2(tau * s.x, tau * s.y);
      }
      __syncthreads();
      // K = (tau/2) v^H p
      double2 kk = make_double2(0.0, 0.0);
      for (int i = tid; i < m; i += nth) {
        const double2 v = S.v[i], p = S.p[i];
        kk.x += v.x * p.x + v.y * p.y;
        kk.y += v.x * p.y - v.y * p.x;
      }
      for (int o = 16; o > 0; o >>= 1) {
        kk.x += __shfl_xor_sync(0xffffffffu, kk.x, o);
        kk.y += __shfl_xor_sync(0xffffffffu, kk.y, o);
      }
      if (lane == 0) S.kred[warp] = kk;
      __syncthreads();
      kk = make_double2(0.0, 0.0);
      for (int w = 0; w < nwarp; ++w) {
        kk.x += S.kred[w].x;
        kk.y += S.kred[w].y;
      }
      kk.x *= 0.5 * tau;
      kk.y *= 0.5 * tau;
      __syncthreads();
      for (int i = tid; i < m; i += nth) {
        const double2 p = S.p[i], v = S.v[i], kv = cmul(kk, v);
        S.p[i] = make_double2(p.x - kv.x, p.y - kv.y);  // w
      }
      __syncthreads();
      // A22 -= v w^H + w v^H
      for (size_t e = tid; e < (size_t)m * m; e += nth) {
        const int i = (int)(e / m), j = (int)(e % m);
        const double2 vi = S.v[i], wi = S.p[i], vj = S.v[j], wj = S.p[j];
        const double2 t1 = cmul(vi, cconj(wj)), t2 = cmul(wi, cconj(vj));
        double2* x = A + (size_t)(k + 1 + i) * b + (k + 1 + j);
        const double2 o = *x;
        *x = make_double2(o.x - t1.x - t2.x, o.y - t1.y - t2.y);
      }
      __syncthreads();
    }
    // tridiagonal: d = Re diag, eps_{b-2} = A[b-1][b-2]; phases delta with
    // delta_0 = 1, delta_{k+1} = delta_k eps_k/|eps_k| make e_k = |eps_k| real
    if (tid == 0) {
      if (b >= 2) {
        S.dl[b - 2] = A[(size_t)(b - 1) * b + (b - 2)];
        S.tau[b - 2] = 0.0;
      }
      for (int i = 0; i < b; ++i) S.d[i] = A[(size_t)i * b + i].x;
      double2 del = make_double2(1.0, 0.0);
      for (int k = 0; k + 1 < b; ++k) {
        const double2 ep = S.dl[k];
        const double me = hypot(ep.x, ep.y);
        S.e[k] = me;
        S.dl[k] = del;  // delta_k
        if (me > 0.0) del = cmul(del, make_double2(ep.x / me, ep.y / me));
      }
      S.dl[b - 1] = del;
      S.e[b - 1] = 0.0;
      S.cmd = 0;
    }
    if (vecs)
      for (size_t e = tid; e < (size_t)bb; e += nth) Z[e] = (e / b == e % b) ? 1.0 : 0.0;
    __syncthreads();
    // ---------------------------------------------------------- implicit QL
    // thread 0 forms the rotations of one sweep (e[i] couples i and i+1);
    // every thread then applies them, in order, to its rows of Z
    int ql_l = 0, ql_iter = 0;
    for (;;) {
      if (tid == 0) {
        int cmd = 1;  // done
        while (ql_l < b) {
          int m = ql_l;
          for (; m < b - 1; ++m) {
            const double dd = fabs(S.d[m]) + fabs(S.d[m + 1]);
            if (fabs(S.e[m]) + dd == dd) break;
          }
          if (m == ql_l) {
            ++ql_l;
            ql_iter = 0;
            continue;
          }
          if (++ql_iter > kQlMaxIter) {
            atomicOr(a.err, 32);
            cmd = 2;
            break;
          }
          const int l = ql_l;
          double g = (S.d[l + 1] - S.d[l]) / (2.0 * S.e[l]);
          double r = hypot(g, 1.0);
          g = S.d[m] - S.d[l] + S.e[l] / (g + (g >= 0 ? fabs(r) : -fabs(r)));
          double s = 1.0, c = 1.0, p = 0.0;
          int i = m - 1;
          bool under = false;
          for (; i >= l; --i) {
            const double f = s * S.e[i], bq = c * S.e[i];
            r = hypot(f, g);
            S.e[i + 1] = r;
            if (r == 0.0) {  // underflow: deflate and sweep again
              S.d[i + 1] -= p;
              S.e[m] = 0.0;
              under = true;
              break;
            }
            s = f / r;
            c = g / r;
            g = S.d[i + 1] - p;
            r = (S.d[i] - g) * s + 2.0 * c * bq;
            p = s * r;
            S.d[i + 1] = g + p;
            g = c * r - bq;
            S.rc[i] = c;
            S.rs[i] = s;
          }
          if (!under) {
            S.d[l] -= p;
            S.e[l] = g;
            S.e[m] = 0.0;
          }
          S.hi = m - 1;
          S.lo = under ? i + 1 : l;
          cmd = 0;
          break;
        }
        S.cmd = cmd;
      }
      __syncthreads();
      const int cmd = S.cmd;
      if (cmd != 0) break;
      if (vecs) {
        const int hi = S.hi, lo = S.lo;
        for (int rr = tid; rr < b; rr += nth)
          for (int i = hi; i >= lo; --i) {
            const double c = S.rc[i], s = S.rs[i];
            const double f = Z[(size_t)(i + 1) * b + rr], z = Z[(size_t)i * b + rr];
            Z[(size_t)(i + 1) * b + rr] = s * z + c * f;
            Z[(size_t)i * b + rr] = c * z - s * f;
          }
      }
      __syncthreads();
    }
    // ---------------------------------------------------------- ordering
    // get_freq: ascending signed eigenvalues (exchange sort of
    // extratools.f90:154-175), eival = |lambda|; get_frequencies sorts the
    // |lambda| once more (velocities keep the first order)
    if (tid == 0) {
      for (int i = 0; i < b; ++i) S.ord[i] = i;
      for (int i = 0; i < b; ++i)
        for (int j = i + 1; j < b; ++j)
          if (S.d[S.ord[i]] > S.d[S.ord[j]]) {
            const int t = S.ord[i];
            S.ord[i] = S.ord[j];
            S.ord[j] = t;
          }
      for (int i = 0; i < b; ++i) {
        S.lab[i] = fabs(S.d[S.ord[i]]);
        S.ord2[i] = i;
      }
      for (int i = 0; i < b; ++i)
        for (int j = i + 1; j < b; ++j)
          if (S.lab[S.ord2[i]] > S.lab[S.ord2[j]]) {
            const int t = S.ord2[i];
            S.ord2[i] = S.ord2[j];
            S.ord2[j] = t;
          }
    }
    __syncthreads();
    for (int i = tid; i < b; i += nth) a.w2_all[((size_t)pt * a.ndisp + dsp) * b + i] = S.lab[i];
    if (vecs) {
      // ---------------------------------------- back-transformation V = Q D Z
      // thread j owns eigenvector j: V[r][j] = delta_r Z[r][j], then the
      // reflections H_k for k = b-3 .. 0 on components k+1..
      for (int j = tid; j < b; j += nth)
        for (int rr = 0; rr < b; ++rr) {
          const double z = Z[(size_t)j * b + rr];
          const double2 dl = S.dl[rr];
          V[(size_t)rr * b + j] = make_double2(dl.x * z, dl.y * z);
        }
      __syncthreads();
      for (int k = b - 3; k >= 0; --k) {
        const double tau = S.tau[k];
        if (tau == 0.0) continue;  // uniform: S.tau is shared
        const int m = b - k - 1;
        for (int i = tid; i < m; i += nth) S.v[i] = A[(size_t)(k + 1 + i) * b + k];
        __syncthreads();
        for (int j = tid; j < b; j += nth) {
          double2 s = make_double2(0.0, 0.0);
          for (int i = 0; i < m; ++i) {  // v^H y
            const double2 v = S.v[i], y = V[(size_t)(k + 1 + i) * b + j];
            s.x += v.x * y.x + v.y * y.y;
            s.y += v.x * y.y - v.y * y.x;
          }
          s.x *= tau;
          s.y *= tau;
          for (int i = 0; i < m; ++i) {
            const double2 t = cmul(S.v[i], s);
            double2* y = V + (size_t)(k + 1 + i) * b + j;
            const double2 o = *y;
            *y = make_double2(o.x - t.x, o.y - t.y);
          }
        }
        __syncthreads();
      }
      // eigenvector of final band l: column ord[ord2[l]]; pure-imaginary fix
      for (int l = warp; l < b; l += nwarp) {
        const int col = S.ord[S.ord2[l]];
        double sre2 = 0;
        for (int c = lane; c < b; c += 32) sre2 += fabs(V[(size_t)c * b + col].x);
        for (int o = 16; o > 0; o >>= 1) sre2 += __shfl_xor_sync(0xffffffffu, sre2, o);
        const bool rot90 = sre2 < 1e-3;
        for (int c = lane; c < b; c += 32) {
          double2 v = V[(size_t)c * b + col];
          if (rot90) v = make_double2(-v.y, v.x);
          const size_t o = (((size_t)pt * b + l) * b + c) * 2;
          a.evec[o] = v.x;
          a.evec[o + 1] = v.y;
        }
      }
      for (int l = tid; l < b; l += nth) a.w2[(size_t)pt * b + l] = S.lab[S.ord2[l]];
    }
    __syncthreads();  // the slot is reused by the next matrix
  }
}

}  // namespace

size_t heev_work_doubles(int b, int slots) { return (size_t)slots * heev_slot_doubles(b); }

int heev_slots(int nmat) { return std::max(1, std::min(nmat, 148 * 4)); }

cudaError_t launch_heev(const PhononArgs& a, cudaStream_t s) {
  const int b = a.geo.b;
  if (b < 1 || b > kHeMaxB || !a.he_work) return cudaErrorInvalidValue;
  const int nmat = a.geo.nkc * a.ndisp;
  heev_kernel<<<std::min(heev_slots(nmat), a.he_slots), kHeThreads, 0, s>>>(a, nmat);
  return cudaGetLastError();
}

}  // namespace ald
