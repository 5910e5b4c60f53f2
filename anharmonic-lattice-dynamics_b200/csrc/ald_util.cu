// Layout conversions at the C-ABI boundary and the stand-alone forms of
// calculate_tauRTA_mpi2 (THERMACOND/sub.f90:7953-8194) and of the P1/P2
// band sums that CollisionMatrix_mpi (sub.f90:3034-3210) reads, used when a
// caller drives the stages one by one with its own P1smpi/P2smpi arrays.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

__global__ void to_fortran5_kernel(const double* src, double* dst, int nr, int nkc, int b) {
  size_t b3 = (size_t)b * b * b;
  size_t total = (size_t)nr * nkc * b3;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    // e enumerates the Fortran array: r fastest, then q, l1, l2, l3
    size_t r = e % nr, t = e / nr;
    size_t q = t % nkc;
    t /= nkc;
    size_t l1 = t % b, l2 = (t / b) % b, l3 = t / ((size_t)b * b);
    dst[e] = src[(r * nkc + q) * b3 + (l1 * b + l2) * b + l3];
  }
}

__global__ void from_fortran5_kernel(const double* src, double* dst, int nr, int nkc, int b) {
  size_t b3 = (size_t)b * b * b;
  size_t total = (size_t)nr * nkc * b3;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    size_t r = e % nr, t = e / nr;
    size_t q = t % nkc;
    t /= nkc;
    size_t l1 = t % b, l2 = (t / b) % b, l3 = t / ((size_t)b * b);
    dst[(r * nkc + q) * b3 + (l1 * b + l2) * b + l3] = src[e];
  }
}

__global__ void transpose_kernel(const double* src, double* dst, int rows, int cols) {
  __shared__ double tile[32][33];
  int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 32 + threadIdx.y;
  for (int k = 0; k < 32; k += 8)
    if (x < cols && y + k < rows) tile[threadIdx.y + k][threadIdx.x] = src[(size_t)(y + k) * cols + x];
  __syncthreads();
  x = blockIdx.y * 32 + threadIdx.x;
  y = blockIdx.x * 32 + threadIdx.y;
  for (int k = 0; k < 32; k += 8)
    if (x < rows && y + k < cols) dst[(size_t)(y + k) * rows + x] = tile[threadIdx.x][threadIdx.y + k];
}

__device__ __forceinline__ int wrapm(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

__device__ double bsum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
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

// one CTA per (row, l1); threads over q
__global__ void tau_kernel(Geometry g, int n1_first, const int* mapinv, const double* P1s, const double* P2s,
                           const double* dist, double* Q, double* QN, double* QU, double* P1, double* P2) {
  __shared__ double red[32];
  const int b = g.b, nkc = g.nkc, b2 = b * b;
  const int row = blockIdx.x, l1 = blockIdx.y;
  const int q1 = mapinv[n1_first + row];
  int m1[3] = {q1 / (g.nc[1] * g.nc[2]), (q1 / g.nc[2]) % g.nc[1], q1 % g.nc[2]};
  double n1b = dist[(size_t)q1 * b + l1];
  double q = 0, qn = 0, qu = 0;
  for (int w = threadIdx.x; w < nkc; w += blockDim.x) {
    int mw[3] = {w / (g.nc[1] * g.nc[2]), (w / g.nc[2]) % g.nc[1], w % g.nc[2]};
    int ma[3], mb[3], ina = 1, inb = 1;
    for (int a = 0; a < 3; ++a) {
      int sh = g.shifted ? g.nc[a] / 2 : 0;
      int va = m1[a] + mw[a] - sh, vb = m1[a] - mw[a] + sh;
      if (va < 0 || va >= g.nc[a]) ina = 0;
      if (vb < 0 || vb >= g.nc[a]) inb = 0;
      ma[a] = wrapm(va, g.nc[a]);
      mb[a] = wrapm(vb, g.nc[a]);
    }
    int qa = ma[2] + g.nc[2] * (ma[1] + g.nc[1] * ma[0]);
    int qb = mb[2] + g.nc[2] * (mb[1] + g.nc[1] * mb[0]);
    for (int l2 = 0; l2 < b; ++l2) {
      double n2 = dist[(size_t)w * b + l2];
      for (int l3 = 0; l3 < b; ++l3) {
        size_t o = (((size_t)row * nkc + w) * b + l1) * b2 + l2 * b + l3;
        double p1 = P1s[o] * (n1b * n2 * (dist[(size_t)qa * b + l3] + 1));
        double p2 = P2s[o] * (n1b * (n2 + 1) * (dist[(size_t)qb * b + l3] + 1));
        if (P1) P1[o] = p1;
        if (P2) P2[o] = p2;
        q += p1 + 0.5 * p2;
        if (ina) qn += p1;
        else qu += p1;
        if (inb) qn += 0.5 * p2;
        else qu += 0.5 * p2;
      }
    }
  }
  q = bsum(q, red);
  qn = bsum(qn, red);
  qu = bsum(qu, red);
  if (threadIdx.x == 0) {
    Q[(size_t)row * b + l1] = q;
    QN[(size_t)row * b + l1] = qn;
    QU[(size_t)row * b + l1] = qu;
  }
}

// R[row][q][l1][l2] = sum_l3 P[row][q][l1][l2][l3]; Qd[row][l1] via a second pass
__global__ void collapse_kernel(int nrows, int nkc, int b, const double* P1, const double* P2, double* R1,
                                double* R2) {
  size_t total = (size_t)nrows * nkc * b * b;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    double s1 = 0, s2 = 0;
    for (int l3 = 0; l3 < b; ++l3) {
      s1 += P1[e * b + l3];
      s2 += P2[e * b + l3];
    }
    R1[e] = s1;
    R2[e] = s2;
  }
}

__global__ void qdiag_kernel(int nkc, int b, const double* R1, const double* R2, double* Qd) {
  __shared__ double red[32];
  int row = blockIdx.x, l1 = blockIdx.y;
  double s = 0;
  for (int w = threadIdx.x; w < nkc; w += blockDim.x)
    for (int l2 = 0; l2 < b; ++l2) {
      size_t o = (((size_t)row * nkc + w) * b + l1) * b + l2;
      s += R1[o] + 0.5 * R2[o];
    }
  s = bsum(s, red);
  if (threadIdx.x == 0) Qd[(size_t)row * b + l1] = s;
}

int grid_for(size_t total) { return (int)std::min<size_t>((total + 255) / 256, 148 * 32); }

// Rp[row][q][l1][l3] = sum_l2 P[row][q][l1][l2][l3] (the other band marginal)
__global__ void marginal_l2_kernel(int nrows, int nkc, int b, const double* P1, const double* P2, double* R1p,
                                   double* R2p) {
  const size_t total = (size_t)nrows * nkc * b * b;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t rq = e / ((size_t)b * b);
    const int l1 = (int)((e / b) % b), l3 = (int)(e % b);
    double s1 = 0, s2 = 0;
    for (int l2 = 0; l2 < b; ++l2) {
      const size_t o = ((rq * b + l1) * b + l2) * b + l3;
      s1 += P1[o];
      s2 += P2[o];
    }
    R1p[e] = s1;
    R2p[e] = s2;
  }
}

}  // namespace

// per band over the mesh: brange[l] = min omega, brange[b + l] = max omega
__global__ void band_range_kernel(int nkc, int b, const double* freq, double* brange) {
  __shared__ double smin[8], smax[8];
  const int l = blockIdx.x;
  double mn = 1e300, mx = -1e300;
  for (int q = threadIdx.x; q < nkc; q += blockDim.x) {
    const double f = freq[(size_t)q * b + l];
    mn = fmin(mn, f);
    mx = fmax(mx, f);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    smin[threadIdx.x >> 5] = mn;
    smax[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      mn = fmin(mn, smin[w]);
      mx = fmax(mx, smax[w]);
    }
    brange[l] = fmin(mn, smin[0]);
    brange[b + l] = fmax(mx, smax[0]);
  }
}

cudaError_t launch_band_range(const Geometry& geo, const double* freq, double* brange, cudaStream_t s) {
  band_range_kernel<<<geo.b, 256, 0, s>>>(geo.nkc, geo.b, freq, brange);
  return cudaGetLastError();
}

cudaError_t launch_marginal_l2(const Geometry& geo, int nrows, const double* P1, const double* P2, double* R1p,
                               double* R2p, cudaStream_t s) {
  const size_t total = (size_t)nrows * geo.nkc * geo.b * geo.b;
  marginal_l2_kernel<<<grid_for(total), 256, 0, s>>>(nrows, geo.nkc, geo.b, P1, P2, R1p, R2p);
  return cudaGetLastError();
}

cudaError_t launch_to_fortran5(const double* src, double* dst, int nr, int nkc, int b, cudaStream_t s) {
  size_t total = (size_t)nr * nkc * b * b * b;
  to_fortran5_kernel<<<grid_for(total), 256, 0, s>>>(src, dst, nr, nkc, b);
  return cudaGetLastError();
}
cudaError_t launch_from_fortran5(const double* src, double* dst, int nr, int nkc, int b, cudaStream_t s) {
  size_t total = (size_t)nr * nkc * b * b * b;
  from_fortran5_kernel<<<grid_for(total), 256, 0, s>>>(src, dst, nr, nkc, b);
  return cudaGetLastError();
}
cudaError_t launch_transpose(const double* src, double* dst, int rows, int cols, cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_kernel<<<grid, block, 0, s>>>(src, dst, rows, cols);
  return cudaGetLastError();
}
cudaError_t launch_tau(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* P1s,
                       const double* P2s, const double* dist, double* Q, double* QN, double* QU, double* P1,
                       double* P2, cudaStream_t s) {
  dim3 grid(nrows, geo.b);
  tau_kernel<<<grid, 256, 0, s>>>(geo, n1_first, mapinv, P1s, P2s, dist, Q, QN, QU, P1, P2);
  return cudaGetLastError();
}
cudaError_t launch_collapse(const Geometry& geo, int nrows, const double* P1, const double* P2, double* R1,
                            double* R2, double* Qd, cudaStream_t s) {
  size_t total = (size_t)nrows * geo.nkc * geo.b * geo.b;
  collapse_kernel<<<grid_for(total), 256, 0, s>>>(nrows, geo.nkc, geo.b, P1, P2, R1, R2);
  dim3 grid(nrows, geo.b);
  qdiag_kernel<<<grid, 256, 0, s>>>(geo.nkc, geo.b, R1, R2, Qd);
  return cudaGetLastError();
}

}  // namespace ald
