// Isotope scattering (iso=1 in latdyn.params) on the device.
//
//   P_iso_split           THERMACOND/sub.f90:4825-4961
//   calculate_tauRTA_iso  THERMACOND/sub.f90:8311-8549 (Q, Q_N, Q_U each + Piso)
//
// Piso(n1, l1) = omega1^2 pi/2 sum_l2 sum_tet sum_corner gs(w, l1, l2) c/6,
//   gs = sum_ai g(ai) |e_ai(q1,l1)^H e_ai(w,l2)|^2,
// c the corner weights of weight_tet at omega1 on the corner energies
// frequency(w, l2) (the reference's n2 loop runs nkc times over a body that
// does not use n2, then divides by nkc: folded here).  The weights are the
// bitwise restatement of ald_tet.h, so this file is compiled with
// -fmad=false like ald_tetra.cu.  One thread per tetrahedron, a CTA per
// (tile of tetrahedra, IBZ row, l2); per-CTA partial sums reduced in a fixed
// order by piso_final_kernel.
#include <cuda_runtime.h>

#include "ald_internal.h"
#include "ald_tet.h"

namespace ald {

namespace {

constexpr int kIsoThreads = 256;

template <int B>
__global__ void __launch_bounds__(kIsoThreads) piso_kernel(Geometry g, int n1_first, const int* mapinv,
                                                           const double* freq, const double* evec,
                                                           const int* tet_corner, const double* giso,
                                                           double* partial) {
  __shared__ double s_om[B];
  __shared__ double2 s_e1[B * B];  // e(q1) as [l1][component]
  __shared__ double s_g[B / 3];
  __shared__ double s_red[kIsoThreads / 32][B];
  const int b = g.b, nat0 = b / 3, row = blockIdx.y, l2 = blockIdx.z, tid = threadIdx.x;
  const int q1 = mapinv[n1_first + row];
  const double2* ev = reinterpret_cast<const double2*>(evec);
  for (int i = tid; i < b * b; i += blockDim.x) s_e1[i] = ev[(size_t)q1 * b * b + i];
  if (tid < b) s_om[tid] = freq[(size_t)q1 * b + tid];
  if (tid < nat0) s_g[tid] = giso[tid];
  __syncthreads();
  double acc[B];
#pragma unroll
  for (int l = 0; l < B; ++l) acc[l] = 0.0;
  const int t = blockIdx.x * blockDim.x + tid;
  if (t < 6 * g.nkc) {
    int w[4];
    float en[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      w[k] = tet_corner[4 * (size_t)t + k];
      en[k] = (float)freq[(size_t)w[k] * b + l2];  // tet%p%w, default REAL
    }
    const TetSorted ts = tet_sort(en[0], en[1], en[2], en[3]);
    int pos[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) pos[k] = tet_pos(en, k);
#pragma unroll
    for (int l1 = 0; l1 < B; ++l1) {
      if (l1 >= b) continue;
      double cp[4];
      if (!tet_weights4(ts, s_om[l1], cp)) continue;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double c = cp[pos[k]];
        if (c == 0.0) continue;
        const double2* e2 = ev + ((size_t)w[k] * b + l2) * b;
        double gs = 0.0;
        for (int ai = 0; ai < nat0; ++ai) {
          double dr = 0.0, di = 0.0;  // e1^H e2 over the atom's three components
          for (int x = 0; x < 3; ++x) {
            const double2 a = s_e1[l1 * b + 3 * ai + x], z = e2[3 * ai + x];
            dr += a.x * z.x + a.y * z.y;
            di += a.x * z.y - a.y * z.x;
          }
          gs = gs + s_g[ai] * (dr * dr + di * di);
        }
        acc[l1] = acc[l1] + gs * c / 6.0;
      }
    }
  }
  // fixed-order block sums of the b values
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int l = 0; l < B; ++l) {
    double v = acc[l];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s_red[warp][l] = v;
  }
  __syncthreads();
  if (tid < b) {
    double s = 0.0;
    for (int i = 0; i < kIsoThreads / 32; ++i) s += s_red[i][tid];
    partial[(((size_t)row * b + l2) * gridDim.x + blockIdx.x) * b + tid] = s;
  }
}

__global__ void piso_final_kernel(Geometry g, int n1_first, int nrows, const int* mapinv, const double* freq,
                                  const double* partial, int nblk, double* Piso, double* Q, double* QN,
                                  double* QU) {
  const int b = g.b;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nrows * b) return;
  const int row = idx / b, l1 = idx % b;
  double s = 0.0;
  for (int l2 = 0; l2 < b; ++l2)
    for (int k = 0; k < nblk; ++k) s += partial[(((size_t)row * b + l2) * nblk + k) * b + l1];
  const double om1 = freq[(size_t)mapinv[n1_first + row] * b + l1];
  const double p = s * om1 * om1 * PhysConst::pi / 2;
  Piso[idx] = p;
  if (Q) {
    Q[idx] += p;
    QN[idx] += p;
    QU[idx] += p;
  }
}

__global__ void add_kernel(size_t n, double* y, const double* x) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

}  // namespace

size_t piso_partial_doubles(const Geometry& geo, int nrows) {
  const int nblk = (6 * geo.nkc + kIsoThreads - 1) / kIsoThreads;
  return (size_t)nrows * geo.b * nblk * geo.b;
}

cudaError_t launch_piso(const Geometry& geo, int n1_first, int nrows, const int* mapinv, const double* freq,
                        const double* evec, const int* tet_corner, const double* giso, double* partial,
                        double* Piso, double* Q, double* QN, double* QU, cudaStream_t s) {
  const int nblk = (6 * geo.nkc + kIsoThreads - 1) / kIsoThreads;
  dim3 grid(nblk, nrows, geo.b);
  if (geo.b <= 3)
    piso_kernel<3><<<grid, kIsoThreads, 0, s>>>(geo, n1_first, mapinv, freq, evec, tet_corner, giso, partial);
  else if (geo.b <= 6)
    piso_kernel<6><<<grid, kIsoThreads, 0, s>>>(geo, n1_first, mapinv, freq, evec, tet_corner, giso, partial);
  else if (geo.b <= 12)
    piso_kernel<12><<<grid, kIsoThreads, 0, s>>>(geo, n1_first, mapinv, freq, evec, tet_corner, giso, partial);
  else
    return cudaErrorInvalidValue;
  const int n = nrows * geo.b;
  piso_final_kernel<<<(n + 255) / 256, 256, 0, s>>>(geo, n1_first, nrows, mapinv, freq, partial, nblk, Piso, Q, QN,
                                                    QU);
  return cudaGetLastError();
}

cudaError_t launch_add(size_t n, double* y, const double* x, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, y, x);
  return cudaGetLastError();
}

}  // namespace ald
