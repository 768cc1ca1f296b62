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

// correctly rounded reciprocals (same result as 1/x, cheaper than a division)
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }

template <typename T> struct GreenTables {
  // truncated: kt[d][b]; filtered: kn/kp/wn/wp[d][b] (b < n_d)
  const T* kt[3];
  const T* kn[3];
  const T* kp[3];
  const T* wn[3];
  const T* wp[3];
  T inv2g;  // 1 / (2 g)
  T c1;     // 1 / (1 - nu)
  int variant;  // 0 truncated, 1 filtered, 2 finite differences (Willot)
};

// Gamma(k) depends on k / |k| only.  In FP32 the rank-4 terms form k^4 and
// 1/|k|^4, which underflow / overflow for tiny k (the finite-difference
// wave-vector has components ~1e-17 where two cosines vanish): scale k by
// its largest component first.  FP64 keeps the reference's arithmetic.
template <typename T>
__device__ __forceinline__ void scale_k(T& k0, T& k1, T& k2) {
  if constexpr (sizeof(T) == 4) {
    const T m = fmaxf(fabsf(k0), fmaxf(fabsf(k1), fabsf(k2)));
    if (m > T(0)) {
      const T inv = T(1) / m;
      k0 *= inv;
      k1 *= inv;
      k2 *= inv;
    }
  }
}

// acc += w * Gamma(k) : t  (3D, Mandel, real and imaginary parts)
template <typename T, typename C>
__device__ __forceinline__ void gamma3_acc(T k0, T k1, T k2, T w, const C* t, C* acc,
                                           T inv2g, T c1) {
  scale_k(k0, k1, k2);
  const T kk = k0 * k0 + k1 * k1 + k2 * k2;
  if (kk == T(0)) return;
  const T q = rcp_rn(kk);
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
  T kz = T(0);
  scale_k(k0, k1, kz);
  const T kk = k0 * k0 + k1 * k1;
  if (kk == T(0)) return;
  const T q = rcp_rn(kk);
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

// Filtered operator as accumulated tensors.  With q_a = 1/|k_a|^2,
// alpha_a = w_a q_a / (2g) and beta_a = alpha_a q_a / (1 - nu),
//   sum_a w_a Gamma(k_a):t = M t + t M - N:t,
//   M = sum_a alpha_a k_a (x) k_a,  N = sum_a beta_a k_a (x) k_a (x) k_a (x) k_a,
// so the 2^d aliases cost one symmetric rank-2 and one fully symmetric
// rank-4 accumulation each, and the contraction is done once per part.
// FP64 computes the 2^d reciprocals with one division (batched inversion:
// prefix products, one reciprocal, back substitution).
template <typename T, int NA>
__device__ __forceinline__ void batch_reciprocal(T* x) {
  if constexpr (sizeof(T) == 8) {
    T pre[NA];
    pre[0] = x[0];
#pragma unroll
    for (int i = 1; i < NA; ++i) pre[i] = pre[i - 1] * x[i];
    T inv = rcp_rn(pre[NA - 1]);
#pragma unroll
    for (int i = NA - 1; i > 0; --i) {
      const T xi = x[i];
      x[i] = inv * pre[i - 1];
      inv *= xi;
    }
    x[0] = inv;
  } else {
#pragma unroll
    for (int i = 0; i < NA; ++i) x[i] = rcp_rn(x[i]);
  }
}

// kx/wx, ky/wy, kz/wz: the two aliases (b - n, b) of each axis and their
// cos^2 weights
template <typename T, typename C>
__device__ __forceinline__ void green_filtered3(const T* kx, const T* wx, const T* ky,
                                                const T* wy, const T* kz, const T* wz, T inv2g,
                                                T c1, C* te) {
  T q[8];
  bool zero[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const T k0 = kx[a >> 2], k1 = ky[(a >> 1) & 1], k2 = kz[a & 1];
    const T kk = k0 * k0 + k1 * k1 + k2 * k2;
    zero[a] = kk == T(0);
    q[a] = zero[a] ? T(1) : kk;
  }
  batch_reciprocal<T, 8>(q);
  // M: m00 m11 m22 m12 m20 m01; N: fully symmetric quartic moments
  T m00 = 0, m11 = 0, m22 = 0, m12 = 0, m20 = 0, m01 = 0;
  T n400 = 0, n040 = 0, n004 = 0, n220 = 0, n202 = 0, n022 = 0, n310 = 0, n301 = 0, n130 = 0,
    n031 = 0, n103 = 0, n013 = 0, n211 = 0, n121 = 0, n112 = 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    if (zero[a]) continue;
    const T k0 = kx[a >> 2], k1 = ky[(a >> 1) & 1], k2 = kz[a & 1];
    const T w = wx[a >> 2] * wy[(a >> 1) & 1] * wz[a & 1];
    const T al = w * q[a] * inv2g;
    const T be = al * q[a] * c1;
    const T p00 = k0 * k0, p11 = k1 * k1, p22 = k2 * k2;
    const T p12 = k1 * k2, p20 = k2 * k0, p01 = k0 * k1;
    m00 += al * p00; m11 += al * p11; m22 += al * p22;
    m12 += al * p12; m20 += al * p20; m01 += al * p01;
    const T b00 = be * p00, b11 = be * p11, b22 = be * p22;
    n400 += b00 * p00; n040 += b11 * p11; n004 += b22 * p22;
    n220 += b00 * p11; n202 += b00 * p22; n022 += b11 * p22;
    n310 += b00 * p01; n301 += b00 * p20; n130 += b11 * p01;
    n031 += b11 * p12; n103 += b22 * p20; n013 += b22 * p12;
    n211 += b00 * p12; n121 += b11 * p20; n112 += b22 * p01;
  }
  const T u = T(0.70710678118654752440084436210485);
  const T s2 = T(1.4142135623730950488016887242097);
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    const T t00 = part ? te[0].y : te[0].x;
    const T t11 = part ? te[1].y : te[1].x;
    const T t22 = part ? te[2].y : te[2].x;
    const T t12 = u * (part ? te[3].y : te[3].x);
    const T t20 = u * (part ? te[4].y : te[4].x);
    const T t01 = u * (part ? te[5].y : te[5].x);
    const T S00 = n400 * t00 + n220 * t11 + n202 * t22 + T(2) * (n211 * t12 + n301 * t20 + n310 * t01);
    const T S11 = n220 * t00 + n040 * t11 + n022 * t22 + T(2) * (n031 * t12 + n121 * t20 + n130 * t01);
    const T S22 = n202 * t00 + n022 * t11 + n004 * t22 + T(2) * (n013 * t12 + n103 * t20 + n112 * t01);
    const T S12 = n211 * t00 + n031 * t11 + n013 * t22 + T(2) * (n022 * t12 + n112 * t20 + n121 * t01);
    const T S20 = n301 * t00 + n121 * t11 + n103 * t22 + T(2) * (n112 * t12 + n202 * t20 + n211 * t01);
    const T S01 = n310 * t00 + n130 * t11 + n112 * t22 + T(2) * (n121 * t12 + n211 * t20 + n220 * t01);
    const T P00 = T(2) * (m00 * t00 + m01 * t01 + m20 * t20);
    const T P11 = T(2) * (m01 * t01 + m11 * t11 + m12 * t12);
    const T P22 = T(2) * (m20 * t20 + m12 * t12 + m22 * t22);
    const T P12 = (m11 + m22) * t12 + m12 * (t11 + t22) + m01 * t20 + m20 * t01;
    const T P20 = (m22 + m00) * t20 + m20 * (t22 + t00) + m12 * t01 + m01 * t12;
    const T P01 = (m00 + m11) * t01 + m01 * (t00 + t11) + m20 * t12 + m12 * t20;
    const T o0 = P00 - S00, o1 = P11 - S11, o2 = P22 - S22;
    const T o3 = s2 * (P12 - S12), o4 = s2 * (P20 - S20), o5 = s2 * (P01 - S01);
    if (part == 0) {
      te[0].x = o0; te[1].x = o1; te[2].x = o2; te[3].x = o3; te[4].x = o4; te[5].x = o5;
    } else {
      te[0].y = o0; te[1].y = o1; te[2].y = o2; te[3].y = o3; te[4].y = o4; te[5].y = o5;
    }
  }
}

template <typename T, typename C>
__device__ __forceinline__ void green_filtered2(const T* kx, const T* wx, const T* ky,
                                                const T* wy, T inv2g, T c1, C* te) {
  T q[4];
  bool zero[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const T k0 = kx[a >> 1], k1 = ky[a & 1];
    const T kk = k0 * k0 + k1 * k1;
    zero[a] = kk == T(0);
    q[a] = zero[a] ? T(1) : kk;
  }
  batch_reciprocal<T, 4>(q);
  T m00 = 0, m11 = 0, m01 = 0, n40 = 0, n31 = 0, n22 = 0, n13 = 0, n04 = 0;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    if (zero[a]) continue;
    const T k0 = kx[a >> 1], k1 = ky[a & 1];
    const T w = wx[a >> 1] * wy[a & 1];
    const T al = w * q[a] * inv2g;
    const T be = al * q[a] * c1;
    const T p00 = k0 * k0, p11 = k1 * k1, p01 = k0 * k1;
    m00 += al * p00; m11 += al * p11; m01 += al * p01;
    const T b00 = be * p00, b11 = be * p11;
    n40 += b00 * p00; n31 += b00 * p01; n22 += b00 * p11; n13 += b11 * p01; n04 += b11 * p11;
  }
  const T u = T(0.70710678118654752440084436210485);
  const T s2 = T(1.4142135623730950488016887242097);
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    const T t00 = part ? te[0].y : te[0].x;
    const T t11 = part ? te[1].y : te[1].x;
    const T t01 = u * (part ? te[2].y : te[2].x);
    const T S00 = n40 * t00 + n22 * t11 + T(2) * n31 * t01;
    const T S11 = n22 * t00 + n04 * t11 + T(2) * n13 * t01;
    const T S01 = n31 * t00 + n13 * t11 + T(2) * n22 * t01;
    const T P00 = T(2) * (m00 * t00 + m01 * t01);
    const T P11 = T(2) * (m01 * t01 + m11 * t11);
    const T P01 = (m00 + m11) * t01 + m01 * (t00 + t11);
    const T o0 = P00 - S00, o1 = P11 - S11, o2 = s2 * (P01 - S01);
    if (part == 0) {
      te[0].x = o0; te[1].x = o1; te[2].x = o2;
    } else {
      te[0].y = o0; te[1].y = o1; te[2].y = o2;
    }
  }
}

// ---------------------------------------------------------------------------
// Tabulated form: per half-spectrum coefficient the tensors M (sym. rank 2)
// and N (fully sym. rank 4) of  Gamma_discrete:t = M t + t M - N:t  (with the
// 1/(2g) and 1/(1-nu) factors folded in).  Truncated = one alias, filtered =
// the 2^d-alias sums.  3D: 21 reals [m00 m11 m22 m12 m20 m01 | n400 n040 n004
// n220 n202 n022 n310 n301 n130 n031 n103 n013 n211 n121 n112]; 2D: 8 reals
// [m00 m11 m01 | n40 n31 n22 n13 n04].
// ---------------------------------------------------------------------------
template <int DIM> struct MnSize;
template <> struct MnSize<2> { static constexpr int value = 8; };
template <> struct MnSize<3> { static constexpr int value = 21; };

template <typename T>
__device__ __forceinline__ void mn_accumulate3(T k0, T k1, T k2, T al, T be, T* mn) {
  const T p00 = k0 * k0, p11 = k1 * k1, p22 = k2 * k2;
  const T p12 = k1 * k2, p20 = k2 * k0, p01 = k0 * k1;
  mn[0] += al * p00; mn[1] += al * p11; mn[2] += al * p22;
  mn[3] += al * p12; mn[4] += al * p20; mn[5] += al * p01;
  const T b00 = be * p00, b11 = be * p11, b22 = be * p22;
  mn[6] += b00 * p00; mn[7] += b11 * p11; mn[8] += b22 * p22;
  mn[9] += b00 * p11; mn[10] += b00 * p22; mn[11] += b11 * p22;
  mn[12] += b00 * p01; mn[13] += b00 * p20; mn[14] += b11 * p01;
  mn[15] += b11 * p12; mn[16] += b22 * p20; mn[17] += b22 * p12;
  mn[18] += b00 * p12; mn[19] += b11 * p20; mn[20] += b22 * p01;
}

template <typename T>
__device__ __forceinline__ void mn_accumulate2(T k0, T k1, T al, T be, T* mn) {
  const T p00 = k0 * k0, p11 = k1 * k1, p01 = k0 * k1;
  mn[0] += al * p00; mn[1] += al * p11; mn[2] += al * p01;
  const T b00 = be * p00, b11 = be * p11;
  mn[3] += b00 * p00; mn[4] += b00 * p01; mn[5] += b00 * p11; mn[6] += b11 * p01;
  mn[7] += b11 * p11;
}

// finite-difference wave-vector from per-axis (sin, cos) of phi = pi b / n
// (green.pyx:983-989, 1001-1016): k_i = sin(phi_i) prod_{j != i} cos(phi_j),
// products left to right as in the reference
template <int DIM, typename T>
__device__ __forceinline__ void willot_k(const T* a0, const T* a1, const T* a2, T& k0, T& k1,
                                         T& k2) {
  if (DIM == 2) {
    k0 = a0[0] * a1[1];
    k1 = a0[1] * a1[0];
    k2 = T(0);
  } else {
    k0 = a0[0] * a1[1] * a2[1];
    k1 = a0[1] * a1[0] * a2[1];
    k2 = a0[1] * a1[1] * a2[0];
  }
}

// M/N of one coefficient from its per-axis values (AxisK: truncated k in
// v[0]; filtered k-, k+, w-, w+; finite differences sin, cos)
template <int DIM, typename T>
__device__ __forceinline__ void mn_build(int variant, const T* a0, const T* a1, const T* a2,
                                         T inv2g, T c1, T* mn) {
  constexpr int NT = MnSize<DIM>::value;
#pragma unroll
  for (int i = 0; i < NT; ++i) mn[i] = T(0);
  constexpr int NA = DIM == 3 ? 8 : 4;
  const int na = variant == 1 ? NA : 1;
  for (int a = 0; a < na; ++a) {
    T k0, k1, k2 = T(0), w;
    if (variant == 0) {
      k0 = a0[0];
      k1 = a1[0];
      if (DIM == 3) k2 = a2[0];
      w = T(1);
    } else if (variant == 2) {
      willot_k<DIM, T>(a0, a1, a2, k0, k1, k2);
      w = T(1);
    } else if (DIM == 3) {
      const int s0 = a >> 2, s1 = (a >> 1) & 1, s2 = a & 1;
      k0 = a0[s0];
      k1 = a1[s1];
      k2 = a2[s2];
      w = a0[2 + s0] * a1[2 + s1] * a2[2 + s2];
    } else {
      const int s0 = a >> 1, s1 = a & 1;
      k0 = a0[s0];
      k1 = a1[s1];
      w = a0[2 + s0] * a1[2 + s1];
    }
    scale_k(k0, k1, k2);
    const T kk = k0 * k0 + k1 * k1 + k2 * k2;
    if (kk == T(0)) continue;
    const T q = rcp_rn(kk);
    const T al = w * q * inv2g;
    const T be = al * q * c1;
    if (DIM == 3)
      mn_accumulate3(k0, k1, k2, al, be, mn);
    else
      mn_accumulate2(k0, k1, al, be, mn);
  }
}

// ---------------------------------------------------------------------------
// Tabulated operator: the symmetric Mandel matrix G of the discrete operator
// at one coefficient (o = G t for the real and the imaginary part), upper
// triangle stored diagonal first:
//   3D (21): G00 G11 G22 G33 G44 G55 | G01 G02 G03 G04 G05 G12 G13 G14 G15
//            G23 G24 G25 G34 G35 G45
//   2D (6):  G00 G11 G22 | G01 G02 G12
// The reference applies the filtered operator as this matrix too
// (green.pyx:954-973, 687-694).  Column J is the M/N contraction of the
// Mandel unit vector e_J, so the table carries the same sums as the M/N form.
// ---------------------------------------------------------------------------
template <int DIM> struct GSize;
template <> struct GSize<2> { static constexpr int value = 6; };
template <> struct GSize<3> { static constexpr int value = 21; };

// o = (M t + t M - N:t) for one real Mandel vector t
template <int DIM, typename T>
__device__ __forceinline__ void mn_apply_real(const T* mn, const T* t, T* o) {
  const T u = T(0.70710678118654752440084436210485);
  const T s2 = T(1.4142135623730950488016887242097);
  if (DIM == 3) {
    const T m00 = mn[0], m11 = mn[1], m22 = mn[2], m12 = mn[3], m20 = mn[4], m01 = mn[5];
    const T n400 = mn[6], n040 = mn[7], n004 = mn[8], n220 = mn[9], n202 = mn[10],
            n022 = mn[11], n310 = mn[12], n301 = mn[13], n130 = mn[14], n031 = mn[15],
            n103 = mn[16], n013 = mn[17], n211 = mn[18], n121 = mn[19], n112 = mn[20];
    const T t00 = t[0], t11 = t[1], t22 = t[2];
    const T t12 = u * t[3], t20 = u * t[4], t01 = u * t[5];
    const T S00 = n400 * t00 + n220 * t11 + n202 * t22 + T(2) * (n211 * t12 + n301 * t20 + n310 * t01);
    const T S11 = n220 * t00 + n040 * t11 + n022 * t22 + T(2) * (n031 * t12 + n121 * t20 + n130 * t01);
    const T S22 = n202 * t00 + n022 * t11 + n004 * t22 + T(2) * (n013 * t12 + n103 * t20 + n112 * t01);
    const T S12 = n211 * t00 + n031 * t11 + n013 * t22 + T(2) * (n022 * t12 + n112 * t20 + n121 * t01);
    const T S20 = n301 * t00 + n121 * t11 + n103 * t22 + T(2) * (n112 * t12 + n202 * t20 + n211 * t01);
    const T S01 = n310 * t00 + n130 * t11 + n112 * t22 + T(2) * (n121 * t12 + n211 * t20 + n220 * t01);
    const T P00 = T(2) * (m00 * t00 + m01 * t01 + m20 * t20);
    const T P11 = T(2) * (m01 * t01 + m11 * t11 + m12 * t12);
    const T P22 = T(2) * (m20 * t20 + m12 * t12 + m22 * t22);
    const T P12 = (m11 + m22) * t12 + m12 * (t11 + t22) + m01 * t20 + m20 * t01;
    const T P20 = (m22 + m00) * t20 + m20 * (t22 + t00) + m12 * t01 + m01 * t12;
    const T P01 = (m00 + m11) * t01 + m01 * (t00 + t11) + m20 * t12 + m12 * t20;
    o[0] = P00 - S00;
    o[1] = P11 - S11;
    o[2] = P22 - S22;
    o[3] = s2 * (P12 - S12);
    o[4] = s2 * (P20 - S20);
    o[5] = s2 * (P01 - S01);
  } else {
    const T m00 = mn[0], m11 = mn[1], m01 = mn[2];
    const T n40 = mn[3], n31 = mn[4], n22 = mn[5], n13 = mn[6], n04 = mn[7];
    const T t00 = t[0], t11 = t[1], t01 = u * t[2];
    const T S00 = n40 * t00 + n22 * t11 + T(2) * n31 * t01;
    const T S11 = n22 * t00 + n04 * t11 + T(2) * n13 * t01;
    const T S01 = n31 * t00 + n13 * t11 + T(2) * n22 * t01;
    const T P00 = T(2) * (m00 * t00 + m01 * t01);
    const T P11 = T(2) * (m01 * t01 + m11 * t11);
    const T P01 = (m00 + m11) * t01 + m01 * (t00 + t11);
    o[0] = P00 - S00;
    o[1] = P11 - S11;
    o[2] = s2 * (P01 - S01);
  }
}

// G from the M/N tensors of one coefficient (column J = contraction of e_J;
// the upper triangle is kept)
template <int DIM, typename T>
__device__ __forceinline__ void mn_to_g(const T* mn, T* g) {
  constexpr int S = DIM == 3 ? 6 : 3;
  T col[S][S];
#pragma unroll
  for (int j = 0; j < S; ++j) {
    T e[S];
#pragma unroll
    for (int i = 0; i < S; ++i) e[i] = i == j ? T(1) : T(0);
    mn_apply_real<DIM, T>(mn, e, col[j]);
  }
  int q = 0;
#pragma unroll
  for (int i = 0; i < S; ++i) g[q++] = col[i][i];
#pragma unroll
  for (int i = 0; i < S; ++i)
#pragma unroll
    for (int j = i + 1; j < S; ++j) g[q++] = col[j][i];
}

// o = G t for one real Mandel vector (G in the table order above)
template <int DIM, typename T>
__device__ __forceinline__ void g_apply_real(const T* g, const T* t, T* o) {
  if (DIM == 3) {
    o[0] = g[0] * t[0] + g[6] * t[1] + g[7] * t[2] + g[8] * t[3] + g[9] * t[4] + g[10] * t[5];
    o[1] = g[6] * t[0] + g[1] * t[1] + g[11] * t[2] + g[12] * t[3] + g[13] * t[4] + g[14] * t[5];
    o[2] = g[7] * t[0] + g[11] * t[1] + g[2] * t[2] + g[15] * t[3] + g[16] * t[4] + g[17] * t[5];
    o[3] = g[8] * t[0] + g[12] * t[1] + g[15] * t[2] + g[3] * t[3] + g[18] * t[4] + g[19] * t[5];
    o[4] = g[9] * t[0] + g[13] * t[1] + g[16] * t[2] + g[18] * t[3] + g[4] * t[4] + g[20] * t[5];
    o[5] = g[10] * t[0] + g[14] * t[1] + g[17] * t[2] + g[19] * t[3] + g[20] * t[4] + g[5] * t[5];
  } else {
    o[0] = g[0] * t[0] + g[3] * t[1] + g[4] * t[2];
    o[1] = g[3] * t[0] + g[1] * t[1] + g[5] * t[2];
    o[2] = g[4] * t[0] + g[5] * t[1] + g[2] * t[2];
  }
}

// te <- G te (real and imaginary parts)
template <int DIM, typename T, typename C>
__device__ __forceinline__ void g_apply(const T* g, C* te) {
  constexpr int S = DIM == 3 ? 6 : 3;
  T re[S], im[S], ore[S], oim[S];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    re[i] = te[i].x;
    im[i] = te[i].y;
  }
  g_apply_real<DIM, T>(g, re, ore);
  g_apply_real<DIM, T>(g, im, oim);
#pragma unroll
  for (int i = 0; i < S; ++i) te[i] = mkc(ore[i], oim[i]);
}

// Per-axis values of one index b_d: truncated k (slot 0) or the filtered
// aliases (k-, k+, w-, w+).
template <typename T> struct AxisK {
  T v[4];
};

template <typename T>
__device__ __forceinline__ AxisK<T> axis_values(const GreenTables<T>& g, int d, int bd) {
  AxisK<T> r;
  if (g.variant == 0) {
    r.v[0] = g.kt[d][bd];
    r.v[1] = r.v[2] = r.v[3] = T(0);
  } else if (g.variant == 2) {
    r.v[0] = g.kn[d][bd];  // sin(phi)
    r.v[1] = g.kp[d][bd];  // cos(phi)
    r.v[2] = r.v[3] = T(0);
  } else {
    r.v[0] = g.kn[d][bd];
    r.v[1] = g.kp[d][bd];
    r.v[2] = g.wn[d][bd];
    r.v[3] = g.wp[d][bd];
  }
  return r;
}

// eta = Gamma_discrete : tau for one half-spectrum coefficient whose per-axis
// values are given (a1 unused in 2D).  tau and eta alias.
template <int DIM, typename T, typename C>
__device__ __forceinline__ void green_contract_k(int variant, const AxisK<T>& a0,
                                                 const AxisK<T>& a1, const AxisK<T>& a2,
                                                 T inv2g, T c1, C* te) {
  constexpr int S = DIM == 2 ? 3 : 6;
  C t[S];
#pragma unroll
  for (int i = 0; i < S; ++i) t[i] = te[i];
  if (variant == 0 || variant == 2) {
    C acc[S];
#pragma unroll
    for (int i = 0; i < S; ++i) acc[i] = mkc(T(0), T(0));
    T k0 = a0.v[0], k1 = a1.v[0], k2 = a2.v[0];
    if (variant == 2) willot_k<DIM, T>(a0.v, a1.v, a2.v, k0, k1, k2);
    if (DIM == 2)
      gamma2_acc(k0, k1, T(1), t, acc, inv2g, c1);
    else
      gamma3_acc(k0, k1, k2, T(1), t, acc, inv2g, c1);
#pragma unroll
    for (int i = 0; i < S; ++i) te[i] = acc[i];
  } else {
    const T kx[2] = {a0.v[0], a0.v[1]}, wx[2] = {a0.v[2], a0.v[3]};
    const T ky[2] = {a1.v[0], a1.v[1]}, wy[2] = {a1.v[2], a1.v[3]};
    if (DIM == 2) {
      green_filtered2<T>(kx, wx, ky, wy, inv2g, c1, t);
    } else {
      const T kz[2] = {a2.v[0], a2.v[1]}, wz[2] = {a2.v[2], a2.v[3]};
      green_filtered3<T>(kx, wx, ky, wy, kz, wz, inv2g, c1, t);
    }
#pragma unroll
    for (int i = 0; i < S; ++i) te[i] = t[i];
  }
}

// eta = Gamma_discrete(b) : tau for one half-spectrum index b (b[d] < n_d),
// reading the per-axis tables from global memory.  tau and eta may alias.
template <int DIM, typename T, typename C>
__device__ __forceinline__ void green_contract(const GreenTables<T>& g, const int* b,
                                               C* tau_eta) {
  const AxisK<T> a0 = axis_values(g, 0, b[0]);
  const AxisK<T> a1 = axis_values(g, 1, b[1]);
  const AxisK<T> a2 = DIM == 3 ? axis_values(g, 2, b[2]) : a1;
  green_contract_k<DIM, T>(g.variant, a0, a1, a2, g.inv2g, g.c1, tau_eta);
}

}  // namespace jb
