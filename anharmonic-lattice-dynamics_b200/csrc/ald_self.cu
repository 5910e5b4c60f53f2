// Three-phonon self-energy at arbitrary q on the device (THERMACOND job=2).
//
//   function_self_w3  THERMACOND/rest.f90:4012-4124  (Lorentzian, four terms, real + imaginary)
//   function_self_w4  THERMACOND/rest.f90:4126-4240  (Gaussian, three terms, imaginary only)
//   matrix_elt_full   THERMACOND/rest.f90:3664-3719
//   check_inside_bz   THERMACOND/extratools.f90:325-341, get_direct_components :561-592
//
// For a path point q, a mode la with target frequency omega and every mesh
// point k2 (k3 = -q - k2), the reference sums over l2, l3
//   |w33(q la, k2 l2, k3 l3)|^2 * self(omega, om2, om3)
// into the normal or umklapp part by check_inside_bz(k3).  Here one CTA owns
// a path point and a tile of consecutive k2; for each (q, k2) pair:
//   1. the phases exp(i (k2.R_j + k3.R_k)) per FC3 atom triple, from the
//      per-atom dot products (sum(v*w) order, no fused multiply-add);
//   2. the Fourier sum Phi[a,b,c] = sum_triples W[a,b,c] P (b^3 complex);
//   3. three mode products with e(q) (every la), e(k2), e(k3), no conjugation;
//   4. per (la, l2, l3): den, the v3_threshold cut, |w33|^2 and self, whose
//      parts are rounded to REAL(4) because CMPLX(x, y) without KIND is
//      default COMPLEX in the reference;
//   5. per-la sums over (l2, l3) and the CTA's pairs in a fixed order, as
//      per-CTA partials; self_final_kernel adds them in tile order and applies
//      the /nkc * pi of the reference.
// The eigenpairs at k3 come from the phonon kernel run on the list of k3
// points (ndisp = 1).  Compiled with -fmad=false: the arithmetic of the
// self terms follows the reference's operation order.
#include <cuda_runtime.h>

#include <algorithm>

#include "ald_internal.h"

namespace ald {

namespace {

constexpr int kSelfBlock = 256;

__device__ __forceinline__ double nbe_self(double w, double t, int m, int* err) {  // nbe, extratools.f90:257
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

__device__ __forceinline__ double dot_a(const double* v, const double* w) {  // sum(v*w)
  return __dadd_rn(__dadd_rn(__dmul_rn(v[0], w[0]), __dmul_rn(v[1], w[1])), __dmul_rn(v[2], w[2]));
}

__global__ void k3_points_kernel(int np, int nkc, const double* qp, const double* kpc, double* k3) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)np * nkc) return;
  const int p = (int)(i / nkc), k = (int)(i % nkc);
  for (int c = 0; c < 3; ++c) k3[3 * i + c] = -qp[3 * p + c] - kpc[3 * k + c];
}

// dynamic shared memory: e1 (b*b, shared) + per pair: e2, e3 (b*b), phi, tmp
// (b^3), con (2 b^3: N and U parts as double2), P (ntrip), d2/d3 (2 natoms doubles)
__global__ void __launch_bounds__(kSelfBlock) self_kernel(SelfArgs a, int ppb) {
  extern __shared__ double2 sm[];
  const int b = a.b, b2 = b * b, b3 = b2 * b, nkc = a.nkc;
  const int nt = kSelfBlock / ppb;
  const int slot = threadIdx.x / nt, lt = threadIdx.x % nt;
  const int p = blockIdx.y;
  int k2 = blockIdx.x * ppb + slot;
  const bool live = k2 < nkc;
  if (!live) k2 = nkc - 1;
  const size_t per_pair = 2 * (size_t)b2 + 4 * (size_t)b3 + a.ntrip + a.natoms;
  double2* e1 = sm;
  double2* base = sm + b2 + slot * per_pair;
  double2* e2 = base;
  double2* e3 = e2 + b2;
  double2* phi = e3 + b2;
  double2* tmp = phi + b3;
  double2* conN = tmp + b3;
  double2* conU = conN + b3;
  double2* P = conU + b3;
  double* d23 = reinterpret_cast<double*>(P + a.ntrip);  // d2 [natoms], d3 [natoms]
  const double2* evq = reinterpret_cast<const double2*>(a.evq) + (size_t)p * b2;
  const double2* ev2 = reinterpret_cast<const double2*>(a.ev2) + (size_t)k2 * b2;
  const size_t pk = (size_t)p * nkc + k2;
  const double2* ev3 = reinterpret_cast<const double2*>(a.ev3) + pk * b2;

  double q[3], kk2[3], k3[3];
  for (int c = 0; c < 3; ++c) {
    q[c] = a.qp[3 * p + c];
    kk2[c] = a.kpc[3 * k2 + c];
    k3[c] = -q[c] - kk2[c];
  }
  for (int e = threadIdx.x; e < b2; e += blockDim.x) e1[e] = evq[e];
  for (int e = lt; e < b2; e += nt) {
    e2[e] = ev2[e];
    e3[e] = ev3[e];
  }
  for (int j = lt; j < a.natoms; j += nt) {
    d23[j] = dot_a(kk2, a.rr + 3 * j);
    d23[a.natoms + j] = dot_a(k3, a.rr + 3 * j);
  }
  __syncthreads();
  for (int t = lt; t < a.ntrip; t += nt) {
    double sn, cs;
    sincos(__dadd_rn(d23[a.trip_j[t]], d23[a.natoms + a.trip_k[t]]), &sn, &cs);
    P[t] = make_double2(cs, sn);
  }
  __syncthreads();
  // Fourier sum: channel (a,b,c) = (3*i0+al, 3*j0+be, 3*k0+ga)
  const int nat0 = a.nat0;
  for (int o = lt; o < b3; o += nt) {
    int ca = o / b2, cb = (o / b) % b, cc = o % b;
    int blk = ((ca / 3) * nat0 + cb / 3) * nat0 + cc / 3;
    int comp = (ca % 3) * 9 + (cb % 3) * 3 + (cc % 3);
    double2 acc = make_double2(0.0, 0.0);
    for (int t = a.blk_off[blk]; t < a.blk_off[blk + 1]; ++t) {
      double w = a.fc3w[27 * (size_t)t + comp];
      double2 ph = P[t];
      acc.x += w * ph.x;
      acc.y += w * ph.y;
    }
    phi[o] = acc;
  }
  __syncthreads();
  // tmp[la][b][c] = sum_a e1[la][a] phi[a][b][c]
  for (int o = lt; o < b3; o += nt) {
    int l1 = o / b2, bc = o % b2;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < b; ++k) {
      double2 e = e1[l1 * b + k], f = phi[k * b2 + bc];
      acc.x += e.x * f.x - e.y * f.y;
      acc.y += e.x * f.y + e.y * f.x;
    }
    tmp[o] = acc;
  }
  __syncthreads();
  // phi[la][l2][c] = sum_b e2[l2][b] tmp[la][b][c]
  for (int o = lt; o < b3; o += nt) {
    int l1 = o / b2, l2 = (o / b) % b, c = o % b;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < b; ++k) {
      double2 e = e2[l2 * b + k], f = tmp[l1 * b2 + k * b + c];
      acc.x += e.x * f.x - e.y * f.y;
      acc.y += e.x * f.y + e.y * f.x;
    }
    phi[o] = acc;
  }
  __syncthreads();
  // inside flag of k3 (check_inside_bz)
  int inside = 1;
  {
    double q2[3];
    for (int c = 0; c < 3; ++c) q2[c] = k3[c] + a.ghalf[c];
    for (int r = 0; r < 3; ++r) {
      const double x = dot_a(q2, a.gd + 3 * r) + 5e-10;
      if (x < 0 || x >= 1) inside = 0;
    }
  }
  const double cn = a.cnst, eta = a.eta, pi = a.pi;
  for (int o = lt; o < b3; o += nt) {
    int l1 = o / b2, l2 = (o / b) % b, l3 = o % b;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < b; ++k) {
      double2 e = e3[l3 * b + k], f = phi[l1 * b2 + l2 * b + k];
      acc.x += e.x * f.x - e.y * f.y;
      acc.y += e.x * f.y + e.y * f.x;
    }
    double2 cN = make_double2(0.0, 0.0), cU = make_double2(0.0, 0.0);
    const double omq = sqrt(fabs(a.wq[(size_t)p * b + l1])) * cn;
    const double om2 = sqrt(fabs(a.w2[(size_t)k2 * b + l2])) * cn;
    const double om3 = sqrt(fabs(a.w3[pk * b + l3])) * cn;
    const double omega = a.omega[(size_t)p * b + l1];
    const double den = sqrt(8 * omq * om2 * om3 / (cn * cn * cn));
    if (den == 0.0) {
      if (live) atomicOr(a.err, 2);
    } else if (live) {
      const double re = acc.x / den * a.const33, im = acc.y / den * a.const33;
      if (!(hypot(re, im) < a.v3thr)) {
        const double term = __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
        const double nb2 = nbe_self(om2, a.temp, a.classical, a.err);
        const double nb3 = nbe_self(om3, a.temp, a.classical, a.err);
        double ires = 0, rres = 0, arg;
        if (!a.gauss) {
          arg = (omega - om3) - om2;
          if (fabs(arg) < a.etacut) {
            ires = (nb3 + nb2 + 1) * (eta / (arg * arg + eta * eta) / pi);
            rres = (nb3 + nb2 + 1) * arg / (arg * arg + eta * eta);
          }
          arg = (omega + om3) + om2;
          if (fabs(arg) < a.etacut) {
            ires = ires - (nb3 + nb2 + 1) * (eta / (arg * arg + eta * eta) / pi);
            rres = rres - (nb3 + nb2 + 1) * arg / (arg * arg + eta * eta);
          }
          arg = (omega - om3) + om2;
          if (fabs(arg) < a.etacut) {
            ires = ires + (nb2 - nb3) * (eta / (arg * arg + eta * eta) / pi);
            rres = rres + (nb2 - nb3) * arg / (arg * arg + eta * eta);
          }
          arg = (omega - om2) + om3;
          if (fabs(arg) < a.etacut) {
            ires = ires + (nb3 - nb2) * (eta / (arg * arg + eta * eta) / pi);
            rres = rres + (nb3 - nb2) * arg / (arg * arg + eta * eta);
          }
        } else {
          const double g0 = sqrt(2 * pi);
          arg = (omega - om3) - om2;
          if (fabs(arg) < a.etacut) ires = (nb3 + nb2 + 1) * (exp(-arg * arg / 2.0 / eta / eta) / g0 / eta);
          arg = (omega - om3) + om2;
          if (fabs(arg) < a.etacut) ires = ires + (nb2 - nb3) * (exp(-arg * arg / 2.0 / eta / eta) / g0 / eta);
          arg = (omega - om2) + om3;
          if (fabs(arg) < a.etacut) ires = ires + (nb3 - nb2) * (exp(-arg * arg / 2.0 / eta / eta) / g0 / eta);
        }
        const double sre = (double)__double2float_rn(rres), sim = (double)__double2float_rn(ires * pi);
        const double2 c = make_double2(term * sre, term * sim);
        if (inside == 1)
          cN = c;
        else
          cU = c;
      }
    }
    conN[o] = cN;
    conU[o] = cU;
  }
  __syncthreads();
  // per-la sums over (l2, l3), then over the CTA's pairs in slot order
  double* red = reinterpret_cast<double*>(tmp);  // reuse: per pair 4*b doubles fit in b^3 double2
  for (int r = lt; r < 4 * b; r += nt) {
    const int l1 = r / 4, part = r % 4;
    const double2* con = (part < 2) ? conN : conU;
    double s = 0;
    for (int u = 0; u < b2; ++u) {
      const double2 v = con[l1 * b2 + u];
      s += (part & 1) ? v.y : v.x;
    }
    red[r] = live ? s : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < 4 * b; r += blockDim.x) {
    double s = 0;
    for (int sl = 0; sl < ppb; ++sl) s += reinterpret_cast<const double*>(sm + b2 + sl * per_pair + 2 * b2 + b3)[r];
    a.part[((size_t)p * gridDim.x + blockIdx.x) * 4 * b + r] = s;
  }
}

__global__ void self_final_kernel(int np, int b, int nblk, int nkc, double pi, const double* part, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // (p, la, part)
  if (i >= np * b * 4) return;
  const int p = i / (4 * b), r = i % (4 * b);
  double s = 0;
  for (int k = 0; k < nblk; ++k) s += part[((size_t)p * nblk + k) * 4 * b + r];
  out[i] = s / (double)nkc * pi;  // nself/nkc*pi, uself/nkc*pi
}

}  // namespace

size_t self_smem_bytes(const SelfArgs& a, int* ppb_out) {
  const int b = a.b, b2 = b * b, b3 = b2 * b;
  // 3 bands: a warp per pair (8 pairs per CTA); 4 to 6 bands: 64 threads per
  // pair, 4 pairs per CTA (the stages between barriers are short; one pair per
  // CTA left the CTA waiting at them)
  int nt = b3 <= 32 ? 32 : b <= 6 ? 64 : std::min(kSelfBlock, ((b3 + 31) / 32) * 32);
  int ppb = std::max(1, kSelfBlock / nt);
  while (kSelfBlock % ppb) --ppb;
  const size_t per_pair = 2 * (size_t)b2 + 4 * (size_t)b3 + a.ntrip + a.natoms;
  size_t sm = (b2 + ppb * per_pair) * sizeof(double2);
  while (ppb > 1 && sm > 200 * 1024) {
    ppb /= 2;
    sm = (b2 + ppb * per_pair) * sizeof(double2);
  }
  if (ppb_out) *ppb_out = ppb;
  return sm;
}

size_t self_partial_doubles(const SelfArgs& a) {
  int ppb = 1;
  self_smem_bytes(a, &ppb);
  return (size_t)a.np * ((a.nkc + ppb - 1) / ppb) * 4 * a.b;
}

cudaError_t launch_k3_points(int np, int nkc, const double* qp, const double* kpc, double* k3, cudaStream_t s) {
  const size_t n = (size_t)np * nkc;
  k3_points_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(np, nkc, qp, kpc, k3);
  return cudaGetLastError();
}

cudaError_t launch_self(const SelfArgs& a, double* out, cudaStream_t s) {
  int ppb = 1;
  const size_t sm = self_smem_bytes(a, &ppb);
  if (sm > 200 * 1024) return cudaErrorInvalidValue;
  if (sm > 48 * 1024) {
    cudaError_t e = raise_smem_limit((const void*)self_kernel, sm);
    if (e != cudaSuccess) return e;
  }
  const int nblk = (a.nkc + ppb - 1) / ppb;
  self_kernel<<<dim3(nblk, a.np), kSelfBlock, sm, s>>>(a, ppb);
  const int n = a.np * a.b * 4;
  self_final_kernel<<<(n + 127) / 128, 128, 0, s>>>(a.np, a.b, nblk, a.nkc, a.pi, a.part, out);
  return cudaGetLastError();
}

}  // namespace ald
