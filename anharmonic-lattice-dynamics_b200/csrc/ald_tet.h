// Tetrahedron corner weights of THERMACOND's weight_tet
// (THERMACOND/tetrahedron.f90:188-384), for host and device.
//
// weight_tet sorts the four corner energies (SSORT, descending, values as
// default REAL), maps sorted positions back to corners with a tie rule, and
// evaluates the linear-tetrahedron delta weights in mixed FP32/FP64: the
// energies and their differences are REAL, every term that involves the
// REAL(8) energy e is promoted to double, and the c/b temporaries of the
// middle branch are REAL.  Callers compile this with FMA contraction off
// (-fmad=false / -ffp-contract=off) so each operation rounds like the
// reference's.
//
// Tie rule: among equal corner energies the corner with the smaller index
// takes the earlier (higher) sorted position, which is what the uns
// bookkeeping of tetrahedron.f90:227-290 produces; hence
//   pos(corner) = #{m : E_m > E_corner} + #{m < corner : E_m == E_corner}
// with pos 0 the highest and 3 the lowest energy.
#pragma once

#ifdef __CUDACC__
#define ALD_TET_HD __host__ __device__ __forceinline__
#else
#define ALD_TET_HD inline
#include <cmath>
#endif

namespace ald {

struct TetSorted {
  float e1, e2, e3, e4;              // ascending: e1 lowest
  float e21, e31, e41, e32, e42, e43;
};

// |x| < small1 = 1e-10 is compared in double in the reference; for a float x
// that is |x| <= the largest float below 1e-10 (0x1.b7cdfcp-34), the same test
// without conversions.  Then x = +-(float)small2, small2 = 1e-10.
ALD_TET_HD void tet_fix_small(float& x) {
  constexpr float kBelowSmall1 = 0x1.b7cdfcp-34f;
  if (fabsf(x) <= kBelowSmall1) {
    if (x > 0.0f) x = (float)1e-10;
    else if (x < 0.0f) x = (float)(-1e-10);
  }
}

ALD_TET_HD float fmax4(float a, float b) { return a > b ? a : b; }
ALD_TET_HD float fmin4(float a, float b) { return a < b ? a : b; }

// sorted energies of one tetrahedron (corner order irrelevant for the values)
ALD_TET_HD TetSorted tet_sort(float a, float b, float c, float d) {
  // sorting network, ascending
  float t;
  if (a > b) { t = a; a = b; b = t; }
  if (c > d) { t = c; c = d; d = t; }
  if (a > c) { t = a; a = c; c = t; }
  if (b > d) { t = b; b = d; d = t; }
  if (b > c) { t = b; b = c; c = t; }
  TetSorted s;
  s.e1 = a;
  s.e2 = b;
  s.e3 = c;
  s.e4 = d;
  s.e21 = s.e2 - s.e1;
  s.e31 = s.e3 - s.e1;
  s.e41 = s.e4 - s.e1;
  s.e32 = s.e3 - s.e2;
  s.e42 = s.e4 - s.e2;
  s.e43 = s.e4 - s.e3;
  tet_fix_small(s.e21);
  tet_fix_small(s.e31);
  tet_fix_small(s.e41);
  tet_fix_small(s.e42);
  tet_fix_small(s.e43);
  return s;
}

// sorted position (0 highest ... 3 lowest) of corner `slot` among en[0..3]
ALD_TET_HD int tet_pos(const float* en, int slot) {
  float x = en[slot];
  int p = 0;
  for (int m = 0; m < 4; ++m) p += (en[m] > x) || (m < slot && en[m] == x);
  return p;
}

// weight c of the corner at sorted position `pos` for energy e
ALD_TET_HD double tet_weight(const TetSorted& t, int pos, double e) {
  const double E1 = t.e1, E2 = t.e2, E3 = t.e3, E4 = t.e4;
  if (e < E1 || e > E4) return 0.0;
  const float e21 = t.e21, e31 = t.e31, e41 = t.e41, e32 = t.e32, e42 = t.e42, e43 = t.e43;
  if (E1 <= e && e <= E2) {
    double x = e - E1;
    double x3 = x * (x * x);
    switch (pos) {
      case 3:
        return ((E2 - e) / (double)e21 + (E3 - e) / (double)e31 + (E4 - e) / (double)e41) * (x * x) /
               (double)((e41 * e31) * e21);
      case 2: return x3 / (double)(((e21 * e21) * e31) * e41);
      case 1: return x3 / (double)((e21 * (e31 * e31)) * e41);
      default: return x3 / (double)((e21 * e31) * (e41 * e41));
    }
  }
  if (E2 <= e && e <= E3) {
    float ca, cb, ba, bb;
    switch (pos) {
      case 3:
        ca = (float)((E3 - e) / (double)(e31 * e31));
        cb = (float)((E4 - e) / (double)(e41 * e41));
        ba = (float)((E3 - e) * (e - E2) / (double)(e42 * e32) + (E4 - e) * (e - E1) / (double)(e41 * e42) +
                     (E3 - e) * (e - E1) / (double)(e32 * e41));
        bb = (float)((E4 - e) * (e - E1) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e32) +
                     (E3 - e) * (e - E1) / (double)(e31 * e32));
        break;
      case 2:
        ca = (float)((E3 - e) / (double)(e32 * e32));
        cb = (float)((E4 - e) / (double)(e42 * e42));
        ba = (float)((E3 - e) * (e - E2) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e41) +
                     (E3 - e) * (e - E1) / (double)(e31 * e41));
        bb = (float)((E3 - e) * (e - E2) / (double)(e32 * e31) + (E4 - e) * (e - E1) / (double)(e41 * e31) +
                     (E4 - e) * (e - E2) / (double)(e32 * e41));
        break;
      case 1:
        ca = (float)((e - E2) / (double)(e32 * e32));
        cb = (float)((e - E1) / (double)(e31 * e31));
        ba = (float)((E3 - e) * (e - E2) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e41) +
                     (E3 - e) * (e - E1) / (double)(e31 * e41));
        bb = (float)((E3 - e) * (e - E2) / (double)(e42 * e32) + (E4 - e) * (e - E1) / (double)(e41 * e42) +
                     (E3 - e) * (e - E1) / (double)(e32 * e41));
        break;
      default:
        ca = (float)((e - E2) / (double)(e42 * e42));
        cb = (float)((e - E1) / (double)(e41 * e41));
        ba = (float)((E3 - e) * (e - E2) / (double)(e32 * e31) + (E4 - e) * (e - E1) / (double)(e41 * e31) +
                     (E4 - e) * (e - E2) / (double)(e32 * e41));
        bb = (float)((E4 - e) * (e - E1) / (double)(e42 * e31) + (E4 - e) * (e - E2) / (double)(e42 * e32) +
                     (E3 - e) * (e - E1) / (double)(e31 * e32));
        break;
    }
    return (double)(0.5f * (ca * ba + cb * bb));
  }
  double x = E4 - e;
  double x3 = x * (x * x);
  switch (pos) {
    case 3: return x3 / (double)(((e41 * e41) * e42) * e43);
    case 2: return x3 / (double)((e41 * (e42 * e42)) * e43);
    case 1: return x3 / (double)((e41 * e42) * (e43 * e43));
    default:
      return ((e - E3) / (double)e43 + (e - E2) / (double)e42 + (e - E1) / (double)e41) * (x * x) /
             (double)((e41 * e42) * e43);
  }
}

// The energy regime of e for a sorted tetrahedron, in weight_tet's test
// order: 0 outside [E1, E4] (all weights zero), 1 E1 <= e <= E2, 2 E2 <= e <= E3,
// 3 E3 < e <= E4.
ALD_TET_HD int tet_regime(const TetSorted& t, double e) {
  const double E1 = t.e1, E2 = t.e2, E3 = t.e3, E4 = t.e4;
  if (e < E1 || e > E4) return 0;
  if (E1 <= e && e <= E2) return 1;
  if (E2 <= e && e <= E3) return 2;
  return 3;
}

// all four weights of one regime: c[pos] for sorted positions 0 (highest) ..
// 3 (lowest); the same expressions as tet_weight.
ALD_TET_HD void tet_weights_low(const TetSorted& t, double e, double* c) {
  const double E1 = t.e1, E2 = t.e2, E3 = t.e3, E4 = t.e4;
  const float e21 = t.e21, e31 = t.e31, e41 = t.e41;
  double x = e - E1;
  double x3 = x * (x * x);
  c[3] = ((E2 - e) / (double)e21 + (E3 - e) / (double)e31 + (E4 - e) / (double)e41) * (x * x) /
         (double)((e41 * e31) * e21);
  c[2] = x3 / (double)(((e21 * e21) * e31) * e41);
  c[1] = x3 / (double)((e21 * (e31 * e31)) * e41);
  c[0] = x3 / (double)((e21 * e31) * (e41 * e41));
}

ALD_TET_HD void tet_weights_mid(const TetSorted& t, double e, double* c) {
  const double E1 = t.e1, E2 = t.e2, E3 = t.e3, E4 = t.e4;
  const float e31 = t.e31, e41 = t.e41, e32 = t.e32, e42 = t.e42;
  const double a3 = E3 - e, a4 = E4 - e, b1 = e - E1, b2 = e - E2;
  float c11 = (float)(a3 / (double)(e31 * e31));
  float c12 = (float)(a4 / (double)(e41 * e41));
  float c21 = (float)(a3 / (double)(e32 * e32));
  float c22 = (float)(a4 / (double)(e42 * e42));
  float c31 = (float)(b2 / (double)(e32 * e32));
  float c32 = (float)(b1 / (double)(e31 * e31));
  float c41 = (float)(b2 / (double)(e42 * e42));
  float c42 = (float)(b1 / (double)(e41 * e41));
  float b11 = (float)(a3 * b2 / (double)(e42 * e32) + a4 * b1 / (double)(e41 * e42) + a3 * b1 / (double)(e32 * e41));
  float b12 = (float)(a4 * b1 / (double)(e42 * e31) + a4 * b2 / (double)(e42 * e32) + a3 * b1 / (double)(e31 * e32));
  float b21 = (float)(a3 * b2 / (double)(e42 * e31) + a4 * b2 / (double)(e42 * e41) + a3 * b1 / (double)(e31 * e41));
  float b22 = (float)(a3 * b2 / (double)(e32 * e31) + a4 * b1 / (double)(e41 * e31) + a4 * b2 / (double)(e32 * e41));
  float b31 = b21;  // identical expressions in the reference
  float b32 = b11;
  float b41 = b22;
  float b42 = b12;
  c[3] = (double)(0.5f * (c11 * b11 + c12 * b12));
  c[2] = (double)(0.5f * (c21 * b21 + c22 * b22));
  c[1] = (double)(0.5f * (c31 * b31 + c32 * b32));
  c[0] = (double)(0.5f * (c41 * b41 + c42 * b42));
}

ALD_TET_HD void tet_weights_high(const TetSorted& t, double e, double* c) {
  const double E1 = t.e1, E2 = t.e2, E3 = t.e3, E4 = t.e4;
  const float e41 = t.e41, e42 = t.e42, e43 = t.e43;
  double x = E4 - e;
  double x3 = x * (x * x);
  c[3] = x3 / (double)(((e41 * e41) * e42) * e43);
  c[2] = x3 / (double)((e41 * (e42 * e42)) * e43);
  c[1] = x3 / (double)((e41 * e42) * (e43 * e43));
  c[0] = ((e - E3) / (double)e43 + (e - E2) / (double)e42 + (e - E1) / (double)e41) * (x * x) /
         (double)((e41 * e42) * e43);
}

ALD_TET_HD void tet_weights_in(const TetSorted& t, int regime, double e, double* c) {
  if (regime == 1) tet_weights_low(t, e, c);
  else if (regime == 2) tet_weights_mid(t, e, c);
  else tet_weights_high(t, e, c);
}

// all four weights at once; false when e lies outside [E1, E4] (all zero)
ALD_TET_HD bool tet_weights4(const TetSorted& t, double e, double* c) {
  const int r = tet_regime(t, e);
  if (r == 0) return false;
  tet_weights_in(t, r, e, c);
  return true;
}

#ifdef __CUDACC__
// The same four weights in FP32 for the mixed-precision pipeline: the regime
// test and the four distances e - E_i are taken in double (e is the FP64
// omega1, so the cancellation stays exact) and rounded once; every quotient
// becomes a product with one reciprocal per sorted difference.  Not bitwise
// against weight_tet: relative errors of a few FP32 ulps per weight.
__device__ __forceinline__ float tet_rcp(float x) { return __fdividef(1.0f, x); }

__device__ __forceinline__ bool tet_weights4_f32(const TetSorted& t, double e, float* c) {
  const int r = tet_regime(t, e);
  if (r == 0) return false;
  const float d1 = (float)(e - (double)t.e1), d2 = (float)(e - (double)t.e2);
  const float d3 = (float)(e - (double)t.e3), d4 = (float)(e - (double)t.e4);  // d4 <= 0
  if (r == 1) {
    const float r21 = tet_rcp(t.e21), r31 = tet_rcp(t.e31), r41 = tet_rcp(t.e41);
    const float x = d1, base = x * x * (r21 * r31 * r41), xb = x * base;
    c[3] = (-d2 * r21 - d3 * r31 - d4 * r41) * base;
    c[2] = xb * r21;
    c[1] = xb * r31;
    c[0] = xb * r41;
  } else if (r == 2) {
    const float r31 = tet_rcp(t.e31), r41 = tet_rcp(t.e41), r32 = tet_rcp(t.e32), r42 = tet_rcp(t.e42);
    const float a3 = -d3, a4 = -d4, b1 = d1, b2 = d2;
    const float c11 = a3 * r31 * r31, c12 = a4 * r41 * r41, c21 = a3 * r32 * r32, c22 = a4 * r42 * r42;
    const float c31 = b2 * r32 * r32, c32 = b1 * r31 * r31, c41 = b2 * r42 * r42, c42 = b1 * r41 * r41;
    const float a3b2 = a3 * b2, a4b1 = a4 * b1, a3b1 = a3 * b1, a4b2 = a4 * b2;
    const float b11 = a3b2 * (r42 * r32) + a4b1 * (r41 * r42) + a3b1 * (r32 * r41);
    const float b12 = a4b1 * (r42 * r31) + a4b2 * (r42 * r32) + a3b1 * (r31 * r32);
    const float b21 = a3b2 * (r42 * r31) + a4b2 * (r42 * r41) + a3b1 * (r31 * r41);
    const float b22 = a3b2 * (r32 * r31) + a4b1 * (r41 * r31) + a4b2 * (r32 * r41);
    c[3] = 0.5f * (c11 * b11 + c12 * b12);
    c[2] = 0.5f * (c21 * b21 + c22 * b22);
    c[1] = 0.5f * (c31 * b21 + c32 * b11);
    c[0] = 0.5f * (c41 * b22 + c42 * b12);
  } else {
    const float r41 = tet_rcp(t.e41), r42 = tet_rcp(t.e42), r43 = tet_rcp(t.e43);
    const float x = -d4, base = x * x * (r41 * r42 * r43), xb = x * base;
    c[3] = xb * r41;
    c[2] = xb * r42;
    c[1] = xb * r43;
    c[0] = (d3 * r43 + d2 * r42 + d1 * r41) * base;
  }
  return true;
}
#endif

}  // namespace ald
