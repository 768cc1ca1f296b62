// Spectral contraction with the discrete Green operator for strains of an
// isotropic reference medium (shear modulus g, Poisson ratio nu), applied on
// the fly to each half-spectrum coefficient of a Mandel strain field.
//
// The continuous operator (janus/material/elastic/linear/isotropic.pyx:158-
// 182, 227-290) is applied without forming its Mandel matrix:
//   Gamma(k):tau = [ (k (x) v + v (x) k) / |k|^2
//                    - (k.v) k (x) k / ((1 - nu) |k|^4) ] / (2 g),  v = tau k,
// which is the same tensor as the reference's closed form
// (tests/test_greenop.py:21-35) contracted with a symmetric tau, at a third
// of the arithmetic.  Gamma(0) = 0 (isotropic.pyx:164-170, 235-257).
//
// Discretisations (janus/green.pyx):
//  * truncated (TruncatedGreenOperator2D/3D.c_set_frequency, 434-445,
//    507-523): k_i = 2 pi/(h n_i) * (b_i - n_i if 2 b_i > n_i else b_i);
//  * filtered (FilteredGreenOperator2D/3D.c_set_frequency, 609-670, 732-910):
//    sum over the 2^d aliases k_i in {s_i (b_i - n_i), s_i b_i} of
//    prod_i cos^2(h k_i / 4) * Gamma(k).
// The per-axis k values and cos^2 weights are tabulated on the host in
// double precision, exactly as the reference evaluates them.
#pragma once

#include "jb_device.cuh"

namespace jb {

template <typename T> struct GreenTables {
  // truncated: kt[d][b]; filtered: kn/kp/wn/wp[d][b] (b < n_d)
  const T* kt[3];
  const T* kn[3];
  const T* kp[3];
  const T* wn[3];
  const T* wp[3];
  T inv2g;  // 1 / (2 g)
  T c1;     // 1 / (1 - nu)
  int variant;  // 0 truncated, 1 filtered
};

// acc += w * Gamma(k) : t  (3D, Mandel, real and imaginary parts)
template <typename T, typename C>
__device__ __forceinline__ void gamma3_acc(T k0, T k1, T k2, T w, const C* t, C* acc,
                                           T inv2g, T c1) {
  const T kk = k0 * k0 + k1 * k1 + k2 * k2;
  if (kk == T(0)) return;
  const T q = T(1) / kk;
  const T al = q * inv2g * w;
  const T u = T(0.70710678118654752440084436210485);
  const T s2 = T(1.4142135623730950488016887242097);
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    const T t0 = part ? t[0].y : t[0].x;
    const T t1 = part ? t[1].y : t[1].x;
    const T t2 = part ? t[2].y : t[2].x;
    const T t3 = part ? t[3].y : t[3].x;
    const T t4 = part ? t[4].y : t[4].x;
    const T t5 = part ? t[5].y : t[5].x;
    const T v0 = t0 * k0 + u * (t5 * k1 + t4 * k2);
    const T v1 = t1 * k1 + u * (t5 * k0 + t3 * k2);
    const T v2 = t2 * k2 + u * (t4 * k0 + t3 * k1);
    const T kv = k0 * v0 + k1 * v1 + k2 * v2;
    const T be = kv * q * c1 * al;
    const T o0 = T(2) * k0 * v0 * al - k0 * k0 * be;
    const T o1 = T(2) * k1 * v1 * al - k1 * k1 * be;
    const T o2 = T(2) * k2 * v2 * al - k2 * k2 * be;
    const T o3 = s2 * ((k1 * v2 + k2 * v1) * al - k1 * k2 * be);
    const T o4 = s2 * ((k2 * v0 + k0 * v2) * al - k2 * k0 * be);
    const T o5 = s2 * ((k0 * v1 + k1 * v0) * al - k0 * k1 * be);
    if (part == 0) {
      acc[0].x += o0; acc[1].x += o1; acc[2].x += o2;
      acc[3].x += o3; acc[4].x += o4; acc[5].x += o5;
    } else {
      acc[0].y += o0; acc[1].y += o1; acc[2].y += o2;
      acc[3].y += o3; acc[4].y += o4; acc[5].y += o5;
    }
  }
}

// acc += w * Gamma(k) : t  (2D plane strain, Mandel (xx, yy, sqrt2 xy))
template <typename T, typename C>
__device__ __forceinline__ void gamma2_acc(T k0, T k1, T w, const C* t, C* acc, T inv2g,
                                           T c1) {
  const T kk = k0 * k0 + k1 * k1;
  if (kk == T(0)) return;
  const T q = T(1) / kk;
  const T al = q * inv2g * w;
  const T u = T(0.70710678118654752440084436210485);
  const T s2 = T(1.4142135623730950488016887242097);
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    const T t0 = part ? t[0].y : t[0].x;
    const T t1 = part ? t[1].y : t[1].x;
    const T t2 = part ? t[2].y : t[2].x;
    const T v0 = t0 * k0 + u * t2 * k1;
    const T v1 = t1 * k1 + u * t2 * k0;
    const T kv = k0 * v0 + k1 * v1;
    const T be = kv * q * c1 * al;
    const T o0 = T(2) * k0 * v0 * al - k0 * k0 * be;
    const T o1 = T(2) * k1 * v1 * al - k1 * k1 * be;
    const T o2 = s2 * ((k0 * v1 + k1 * v0) * al - k0 * k1 * be);
    if (part == 0) {
      acc[0].x += o0; acc[1].x += o1; acc[2].x += o2;
    } else {
      acc[0].y += o0; acc[1].y += o1; acc[2].y += o2;
    }
  }
}

// eta = Gamma_discrete(b) : tau for one half-spectrum index b (b[d] < n_d).
// tau and eta may alias.
template <int DIM, typename T, typename C>
__device__ __forceinline__ void green_contract(const GreenTables<T>& g, const int* b,
                                               C* tau_eta) {
  constexpr int S = DIM == 2 ? 3 : 6;
  C t[S], acc[S];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    t[i] = tau_eta[i];
    acc[i] = mkc(T(0), T(0));
  }
  if (g.variant == 0) {
    if (DIM == 2)
      gamma2_acc(g.kt[0][b[0]], g.kt[1][b[1]], T(1), t, acc, g.inv2g, g.c1);
    else
      gamma3_acc(g.kt[0][b[0]], g.kt[1][b[1]], g.kt[2][b[2]], T(1), t, acc, g.inv2g, g.c1);
  } else {
    if (DIM == 2) {
      const T kn0 = g.kn[0][b[0]], kp0 = g.kp[0][b[0]], wn0 = g.wn[0][b[0]], wp0 = g.wp[0][b[0]];
      const T kn1 = g.kn[1][b[1]], kp1 = g.kp[1][b[1]], wn1 = g.wn[1][b[1]], wp1 = g.wp[1][b[1]];
      gamma2_acc(kn0, kn1, wn0 * wn1, t, acc, g.inv2g, g.c1);
      gamma2_acc(kn0, kp1, wn0 * wp1, t, acc, g.inv2g, g.c1);
      gamma2_acc(kp0, kn1, wp0 * wn1, t, acc, g.inv2g, g.c1);
      gamma2_acc(kp0, kp1, wp0 * wp1, t, acc, g.inv2g, g.c1);
    } else {
      const T kn0 = g.kn[0][b[0]], kp0 = g.kp[0][b[0]], wn0 = g.wn[0][b[0]], wp0 = g.wp[0][b[0]];
      const T kn1 = g.kn[1][b[1]], kp1 = g.kp[1][b[1]], wn1 = g.wn[1][b[1]], wp1 = g.wp[1][b[1]];
      const T kn2 = g.kn[2][b[2]], kp2 = g.kp[2][b[2]], wn2 = g.wn[2][b[2]], wp2 = g.wp[2][b[2]];
      gamma3_acc(kn0, kn1, kn2, wn0 * wn1 * wn2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kn0, kn1, kp2, wn0 * wn1 * wp2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kn0, kp1, kn2, wn0 * wp1 * wn2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kn0, kp1, kp2, wn0 * wp1 * wp2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kp0, kn1, kn2, wp0 * wn1 * wn2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kp0, kn1, kp2, wp0 * wn1 * wp2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kp0, kp1, kn2, wp0 * wp1 * wn2, t, acc, g.inv2g, g.c1);
      gamma3_acc(kp0, kp1, kp2, wp0 * wp1 * wp2, t, acc, g.inv2g, g.c1);
    }
  }
#pragma unroll
  for (int i = 0; i < S; ++i) tau_eta[i] = acc[i];
}

}  // namespace jb
