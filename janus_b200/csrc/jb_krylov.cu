// Vector kernels of the BiCGSTAB inner solver of the mixed-precision scheme:
// batched over load cases (fields [L][nel] back to back, one set of scalars
// per load case, all scalars kept on the device so that an iteration needs no
// host round trip).  Dot products accumulate in FP64 with per-block partial
// sums reduced in a fixed order (deterministic).
//
// BiCGSTAB (van der Vorst 1992), per load case, for A x = b from x = 0:
//   r = b, rh = b, rho = alpha = omega = 1, rho1 = rh.r, v = p = 0
//   repeat: beta = (rho1/rho)(alpha/omega); p = r + beta (p - omega v)
//           v = A p; alpha = rho1/(rh.v); rho = rho1; s = r - alpha v
//           t = A s; omega = (t.s)/(t.t); x += alpha p + omega s
//           r = s - omega t; rho1 = rh.r
// A load case whose denominators vanish or stop being finite (breakdown or
// exact convergence) is frozen: its x and r are left as they are.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "jb_kernels.h"

namespace jb {
namespace {

constexpr int kKrThreads = 256;

// four consecutive elements per access (16 bytes FP32, 2 x 16 bytes FP64)
template <typename T> struct V4;
template <> struct V4<float> {
  using type = float4;
};
template <> struct V4<double> {
  using type = double4;
};

__device__ __forceinline__ double kr_block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

__device__ __forceinline__ bool kr_finite(double v) { return isfinite(v); }

// vector accesses apply when every field of the load case starts on a
// 16-byte (FP32) / 32-byte (FP64) boundary; the tail runs scalar
template <typename T>
__device__ __forceinline__ bool kr_vec4(int64_t nel, const T* a, const T* b, const T* c) {
  const uintptr_t m = (uintptr_t)(4 * sizeof(T) - 1);
  return nel >= 4 && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                       reinterpret_cast<uintptr_t>(c)) & m) == 0;
}

// partials[(l * 2 + q) * nb + b] of a.b (q = 0) and c.d (q = 1, if c)
template <typename T>
__global__ void __launch_bounds__(kKrThreads)
    kr_dot_kernel(int64_t nel, const T* __restrict__ a, const T* __restrict__ b,
                  const T* __restrict__ c, const T* __restrict__ d, double* partials) {
  __shared__ double red[kKrThreads / 32];
  const int l = blockIdx.y, nb = gridDim.x;
  const int64_t off = (int64_t)l * nel;
  double s0 = 0.0, s1 = 0.0;
  const int64_t stride = (int64_t)nb * blockDim.x;
  int64_t i0 = 0;
  if (kr_vec4(nel, a + off, b + off, c ? c + off : a + off) &&
      kr_vec4(nel, d ? d + off : a + off, a + off, a + off)) {
    using V = typename V4<T>::type;
    const V* a4 = reinterpret_cast<const V*>(a + off);
    const V* b4 = reinterpret_cast<const V*>(b + off);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel / 4; i += stride) {
      const V x = a4[i], y = b4[i];
      s0 += (double)x.x * (double)y.x + (double)x.y * (double)y.y + (double)x.z * (double)y.z +
            (double)x.w * (double)y.w;
      if (c) {
        const V u = reinterpret_cast<const V*>(c + off)[i];
        const V w = reinterpret_cast<const V*>(d + off)[i];
        s1 += (double)u.x * (double)w.x + (double)u.y * (double)w.y + (double)u.z * (double)w.z +
              (double)u.w * (double)w.w;
      }
    }
    i0 = nel / 4 * 4;
  }
  for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel; i += stride) {
    s0 += (double)a[off + i] * (double)b[off + i];
    if (c) s1 += (double)c[off + i] * (double)d[off + i];
  }
  s0 = kr_block_sum(s0, red);
  if (threadIdx.x == 0) partials[((int64_t)l * 2) * nb + blockIdx.x] = s0;
  if (c) {
    s1 = kr_block_sum(s1, red);
    if (threadIdx.x == 0) partials[((int64_t)l * 2 + 1) * nb + blockIdx.x] = s1;
  }
}

// sum of the nb partials of dot q of load case blockIdx.x (fixed order)
__device__ double kr_reduce(const double* partials, int nb, int q, double* red) {
  const int l = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partials[((int64_t)l * 2 + q) * nb + b];
  return kr_block_sum(s, red);
}

// stage 0: rho1 = rh.r after init; 1: alpha; 2: omega; 3: rho1 after x/r
__global__ void __launch_bounds__(kKrThreads)
    kr_scalar_kernel(int stage, const double* partials, int nb, KrylovState* st) {
  __shared__ double red[kKrThreads / 32];
  KrylovState& k = st[blockIdx.x];
  const double s0 = kr_reduce(partials, nb, 0, red);
  const double s1 = stage == 2 ? kr_reduce(partials, nb, 1, red) : 0.0;
  if (threadIdx.x != 0) return;
  if (stage == 0) {
    k.rho = k.alpha = k.omega = 1.0;
    k.rho1 = s0;
    k.active = (s0 != 0.0 && kr_finite(s0)) ? 1 : 0;
  } else if (stage == 1) {
    if (k.active && s0 != 0.0 && kr_finite(k.rho1 / s0)) {
      k.alpha = k.rho1 / s0;
      k.rho = k.rho1;
    } else {
      k.active = 0;
    }
  } else if (stage == 2) {
    // s1 = t.t, s0 = t.s
    if (k.active) {
      if (s1 != 0.0 && kr_finite(s0 / s1)) {
        k.omega = s0 / s1;
      } else {
        k.omega = 0.0;  // t = 0: s solves it; finish with x += alpha p, r = s
        k.active = 2;   // last update, then frozen
      }
    }
  } else {
    if (k.active == 2 || k.omega == 0.0 || s0 == 0.0 || !kr_finite(s0)) {
      k.active = 0;
    } else if (k.active) {
      k.rho1 = s0;
    }
  }
}

// p = r + beta (p - omega v)
template <typename T>
__global__ void kr_update_p_kernel(int64_t nel, const T* __restrict__ r, const T* __restrict__ v,
                                   T* __restrict__ p, const KrylovState* st) {
  const int l = blockIdx.y;
  const KrylovState k = st[l];
  if (k.active != 1) return;
  const double beta = (k.rho1 / k.rho) * (k.alpha / k.omega);
  const T b = (T)beta, om = (T)k.omega;
  const int64_t off = (int64_t)l * nel;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i0 = 0;
  if (kr_vec4(nel, r + off, v + off, p + off)) {
    using V = typename V4<T>::type;
    const V* r4 = reinterpret_cast<const V*>(r + off);
    const V* v4 = reinterpret_cast<const V*>(v + off);
    V* p4 = reinterpret_cast<V*>(p + off);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel / 4; i += stride) {
      const V rr = r4[i], vv = v4[i];
      V pp = p4[i];
      pp.x = rr.x + b * (pp.x - om * vv.x);
      pp.y = rr.y + b * (pp.y - om * vv.y);
      pp.z = rr.z + b * (pp.z - om * vv.z);
      pp.w = rr.w + b * (pp.w - om * vv.w);
      p4[i] = pp;
    }
    i0 = nel / 4 * 4;
  }
  for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel; i += stride)
    p[off + i] = r[off + i] + b * (p[off + i] - om * v[off + i]);
}

// s = r - alpha v
template <typename T>
__global__ void kr_update_s_kernel(int64_t nel, const T* __restrict__ r, const T* __restrict__ v,
                                   T* __restrict__ s, const KrylovState* st) {
  const int l = blockIdx.y;
  const KrylovState k = st[l];
  if (k.active != 1) return;
  const T a = (T)k.alpha;
  const int64_t off = (int64_t)l * nel;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i0 = 0;
  if (kr_vec4(nel, r + off, v + off, s + off)) {
    using V = typename V4<T>::type;
    const V* r4 = reinterpret_cast<const V*>(r + off);
    const V* v4 = reinterpret_cast<const V*>(v + off);
    V* s4 = reinterpret_cast<V*>(s + off);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel / 4; i += stride) {
      const V rr = r4[i], vv = v4[i];
      V o;
      o.x = rr.x - a * vv.x;
      o.y = rr.y - a * vv.y;
      o.z = rr.z - a * vv.z;
      o.w = rr.w - a * vv.w;
      s4[i] = o;
    }
    i0 = nel / 4 * 4;
  }
  for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel; i += stride)
    s[off + i] = r[off + i] - a * v[off + i];
}

// x += alpha p + omega s; r = s - omega t; partials of rh.r
template <typename T>
__global__ void __launch_bounds__(kKrThreads)
    kr_update_xr_kernel(int64_t nel, T* __restrict__ x, const T* __restrict__ p,
                        const T* __restrict__ s, const T* __restrict__ t, T* __restrict__ r,
                        const T* __restrict__ rh, const KrylovState* st, double* partials) {
  __shared__ double red[kKrThreads / 32];
  const int l = blockIdx.y, nb = gridDim.x;
  const KrylovState k = st[l];
  const int64_t off = (int64_t)l * nel;
  double acc = 0.0;
  if (k.active != 0) {
    const T a = (T)k.alpha, om = (T)k.omega;
    const int64_t stride = (int64_t)nb * blockDim.x;
    int64_t i0 = 0;
    if (kr_vec4(nel, x + off, p + off, s + off) && kr_vec4(nel, t + off, r + off, rh + off)) {
      using V = typename V4<T>::type;
      V* x4 = reinterpret_cast<V*>(x + off);
      V* r4 = reinterpret_cast<V*>(r + off);
      const V* p4 = reinterpret_cast<const V*>(p + off);
      const V* s4 = reinterpret_cast<const V*>(s + off);
      const V* t4 = reinterpret_cast<const V*>(t + off);
      const V* h4 = reinterpret_cast<const V*>(rh + off);
      for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel / 4;
           i += stride) {
        V xx = x4[i];
        const V pp = p4[i], ss = s4[i], tt = t4[i], hh = h4[i];
        xx.x += a * pp.x + om * ss.x;
        xx.y += a * pp.y + om * ss.y;
        xx.z += a * pp.z + om * ss.z;
        xx.w += a * pp.w + om * ss.w;
        x4[i] = xx;
        V rn;
        rn.x = ss.x - om * tt.x;
        rn.y = ss.y - om * tt.y;
        rn.z = ss.z - om * tt.z;
        rn.w = ss.w - om * tt.w;
        r4[i] = rn;
        acc += (double)hh.x * (double)rn.x + (double)hh.y * (double)rn.y +
               (double)hh.z * (double)rn.z + (double)hh.w * (double)rn.w;
      }
      i0 = nel / 4 * 4;
    }
    for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel; i += stride) {
      x[off + i] += a * p[off + i] + om * s[off + i];
      const T rn = s[off + i] - om * t[off + i];
      r[off + i] = rn;
      acc += (double)rh[off + i] * (double)rn;
    }
  }
  acc = kr_block_sum(acc, red);
  if (threadIdx.x == 0) partials[((int64_t)l * 2) * nb + blockIdx.x] = acc;
}

// ---------------------------------------------------------------------------
// GMRES(m) vector kernels (FP64).  Basis vector i of load case l starts at
// V + i * vs + l * nel; up to kGmChunk basis vectors are streamed per launch
// next to the vector w they are combined with.
// ---------------------------------------------------------------------------
constexpr int kGmChunk = 8;

// partials[(l * kGmChunk + i) * nb + b] = block b's share of w . V_{j0+i},
// i < CNT; VEC: two consecutive elements per access (every field 16-byte
// aligned and nel even)
template <int CNT, bool VEC>
__global__ void __launch_bounds__(kKrThreads)
    gm_dots_kernel(int64_t nel, const double* __restrict__ w, const double* __restrict__ V,
                   int64_t vs, int j0, double* partials) {
  __shared__ double red[kKrThreads / 32];
  const int l = blockIdx.y, nb = gridDim.x;
  const int64_t off = (int64_t)l * nel;
  const double* wl = w + off;
  const double* vb = V + (int64_t)j0 * vs + off;
  double acc[CNT];
#pragma unroll
  for (int i = 0; i < CNT; ++i) acc[i] = 0.0;
  const int64_t stride = (int64_t)nb * blockDim.x;
  const int64_t e0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if constexpr (VEC) {
    const double2* w2 = reinterpret_cast<const double2*>(wl);
    for (int64_t e = e0; e < nel / 2; e += stride) {
      const double2 x = w2[e];
#pragma unroll
      for (int i = 0; i < CNT; ++i) {
        const double2 v = reinterpret_cast<const double2*>(vb + (int64_t)i * vs)[e];
        acc[i] += x.x * v.x + x.y * v.y;
      }
    }
  } else {
    for (int64_t e = e0; e < nel; e += stride) {
      const double x = wl[e];
#pragma unroll
      for (int i = 0; i < CNT; ++i) acc[i] += x * vb[(int64_t)i * vs + e];
    }
  }
#pragma unroll
  for (int i = 0; i < CNT; ++i) {
    const double t = kr_block_sum(acc[i], red);
    if (threadIdx.x == 0) partials[((int64_t)l * kGmChunk + i) * nb + blockIdx.x] = t;
  }
}

// out[l * ldo + o0 + i] = sum_b partials[(l * kGmChunk + i) * nb + b], fixed order
__global__ void __launch_bounds__(kKrThreads)
    gm_reduce_kernel(const double* partials, int nb, double* out, int ldo, int o0) {
  __shared__ double red[kKrThreads / 32];
  const int i = blockIdx.x, l = blockIdx.y;
  double t = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    t += partials[((int64_t)l * kGmChunk + i) * nb + b];
  t = kr_block_sum(t, red);
  if (threadIdx.x == 0) out[(int64_t)l * ldo + o0 + i] = t;
}

// w += sign * sum_{i < CNT} coef[l * ldc + c0 + i] V_{j0+i}; with partials,
// also block b's share of |w|^2 after the update at partials[l * kGmChunk * nb + b]
template <int CNT, bool VEC>
__global__ void __launch_bounds__(kKrThreads)
    gm_axpys_kernel(int64_t nel, double* __restrict__ w, const double* __restrict__ V,
                    int64_t vs, int j0, const double* __restrict__ coef, int ldc, int c0,
                    double sign, double* partials) {
  __shared__ double red[kKrThreads / 32];
  const int l = blockIdx.y;
  const int64_t off = (int64_t)l * nel;
  double* wl = w + off;
  const double* vb = V + (int64_t)j0 * vs + off;
  double a[CNT];
#pragma unroll
  for (int i = 0; i < CNT; ++i) a[i] = sign * coef[(int64_t)l * ldc + c0 + i];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t e0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double nn = 0.0;
  if constexpr (VEC) {
    double2* w2 = reinterpret_cast<double2*>(wl);
    for (int64_t e = e0; e < nel / 2; e += stride) {
      double2 x = w2[e];
#pragma unroll
      for (int i = 0; i < CNT; ++i) {
        const double2 v = reinterpret_cast<const double2*>(vb + (int64_t)i * vs)[e];
        x.x += a[i] * v.x;
        x.y += a[i] * v.y;
      }
      w2[e] = x;
      nn += x.x * x.x + x.y * x.y;
    }
  } else {
    for (int64_t e = e0; e < nel; e += stride) {
      double x = wl[e];
#pragma unroll
      for (int i = 0; i < CNT; ++i) x += a[i] * vb[(int64_t)i * vs + e];
      wl[e] = x;
      nn += x * x;
    }
  }
  if (partials) {  // uniform over the grid
    nn = kr_block_sum(nn, red);
    if (threadIdx.x == 0) partials[(int64_t)l * kGmChunk * gridDim.x + blockIdx.x] = nn;
  }
}

// w /= sqrt(sq[l]); a vector of zero or non-finite norm becomes 0 (the
// Arnoldi process of that load case has broken down or converged)
__global__ void __launch_bounds__(kKrThreads)
    gm_scale_kernel(int64_t nel, double* __restrict__ w, const double* __restrict__ sq) {
  const int l = blockIdx.y;
  const double n = sqrt(sq[l]);
  const double f = (n > 0.0 && isfinite(1.0 / n)) ? 1.0 / n : 0.0;
  double* wl = w + (int64_t)l * nel;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t e0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t done = 0;
  if (kr_vec4(nel, wl, wl, wl)) {  // 32-byte accesses
    double4* w4 = reinterpret_cast<double4*>(wl);
    for (int64_t e = e0; e < nel / 4; e += stride) {
      double4 x = w4[e];
      x.x *= f;
      x.y *= f;
      x.z *= f;
      x.w *= f;
      w4[e] = x;
    }
    done = nel / 4 * 4;
  }
  for (int64_t e = done + e0; e < nel; e += stride) wl[e] *= f;
}

// r = E_l - ax (the residual of the macroscopic load; r may alias ax),
// element-wise over the load case's nvox * C values: consecutive threads
// take consecutive elements (component = element mod C)
template <int C>
__global__ void __launch_bounds__(kKrThreads)
    gm_resid_kernel(int64_t nvox, const double* __restrict__ E, const double* ax, double* r) {
  const int l = blockIdx.y;
  const int64_t nel = nvox * C, off = (int64_t)l * nel;
  double e[C];
#pragma unroll
  for (int c = 0; c < C; ++c) e[c] = E[l * C + c];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nel; i += stride) {
    const int c = (int)(i % C);
    double ev = e[0];
#pragma unroll
    for (int q = 1; q < C; ++q)
      if (c == q) ev = e[q];
    r[off + i] = ev - ax[off + i];
  }
}

int kr_blocks(int64_t nel, int L) {
  int64_t b = (nel + kKrThreads * 4 - 1) / (kKrThreads * 4);
  const int64_t cap = (148 * 8 + L - 1) / L;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

int krylov_blocks(int64_t nel, int L) { return kr_blocks(nel, L); }

int gmres_chunk() { return kGmChunk; }

namespace {

// every field of the call starts on a 16-byte boundary and holds an even
// number of elements
bool gm_vec2(int64_t nel, int64_t vs, const void* a, const void* b) {
  return nel % 2 == 0 && vs % 2 == 0 &&
         ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
}

template <int CNT>
void gm_dots_go(bool vec, dim3 grid, cudaStream_t st, int64_t nel, const double* w,
                const double* V, int64_t vs, int j0, double* partials) {
  if (vec)
    gm_dots_kernel<CNT, true><<<grid, kKrThreads, 0, st>>>(nel, w, V, vs, j0, partials);
  else
    gm_dots_kernel<CNT, false><<<grid, kKrThreads, 0, st>>>(nel, w, V, vs, j0, partials);
}

template <int CNT>
void gm_axpys_go(bool vec, dim3 grid, cudaStream_t st, int64_t nel, double* w, const double* V,
                 int64_t vs, int j0, const double* coef, int ldc, int c0, double sign,
                 double* partials) {
  if (vec)
    gm_axpys_kernel<CNT, true><<<grid, kKrThreads, 0, st>>>(nel, w, V, vs, j0, coef, ldc, c0,
                                                            sign, partials);
  else
    gm_axpys_kernel<CNT, false><<<grid, kKrThreads, 0, st>>>(nel, w, V, vs, j0, coef, ldc, c0,
                                                             sign, partials);
}

}  // namespace

cudaError_t launch_gmres_dots(int64_t nel, int L, const double* w, const double* V, int64_t vs,
                              int j0, int cnt, double* partials, double* out, int ldo, int o0,
                              cudaStream_t st) {
  if (cnt < 1 || cnt > kGmChunk) return cudaErrorInvalidValue;
  const int nb = kr_blocks(nel, L);
  const dim3 grid((unsigned)nb, (unsigned)L);
  const bool vec = gm_vec2(nel, vs, w, V + (int64_t)j0 * vs);
  switch (cnt) {
    case 1: gm_dots_go<1>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    case 2: gm_dots_go<2>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    case 3: gm_dots_go<3>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    case 4: gm_dots_go<4>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    case 5: gm_dots_go<5>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    case 6: gm_dots_go<6>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    case 7: gm_dots_go<7>(vec, grid, st, nel, w, V, vs, j0, partials); break;
    default: gm_dots_go<8>(vec, grid, st, nel, w, V, vs, j0, partials); break;
  }
  gm_reduce_kernel<<<dim3((unsigned)cnt, (unsigned)L), kKrThreads, 0, st>>>(partials, nb, out,
                                                                             ldo, o0);
  return cudaGetLastError();
}

cudaError_t launch_gmres_axpys(int64_t nel, int L, double* w, const double* V, int64_t vs, int j0,
                               int cnt, const double* coef, int ldc, int c0, double sign,
                               double* partials, double* sq, cudaStream_t st) {
  if (cnt < 1 || cnt > kGmChunk) return cudaErrorInvalidValue;
  if ((partials == nullptr) != (sq == nullptr)) return cudaErrorInvalidValue;
  const int nb = kr_blocks(nel, L);
  const dim3 grid((unsigned)nb, (unsigned)L);
  const bool vec = gm_vec2(nel, vs, w, V + (int64_t)j0 * vs);
  switch (cnt) {
    case 1: gm_axpys_go<1>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    case 2: gm_axpys_go<2>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    case 3: gm_axpys_go<3>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    case 4: gm_axpys_go<4>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    case 5: gm_axpys_go<5>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    case 6: gm_axpys_go<6>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    case 7: gm_axpys_go<7>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
    default: gm_axpys_go<8>(vec, grid, st, nel, w, V, vs, j0, coef, ldc, c0, sign, partials); break;
  }
  if (sq)
    gm_reduce_kernel<<<dim3(1u, (unsigned)L), kKrThreads, 0, st>>>(partials, nb, sq, 1, 0);
  return cudaGetLastError();
}

cudaError_t launch_gmres_scale(int64_t nel, int L, double* w, const double* sq, cudaStream_t st) {
  gm_scale_kernel<<<dim3((unsigned)kr_blocks(nel, L), (unsigned)L), kKrThreads, 0, st>>>(nel, w,
                                                                                         sq);
  return cudaGetLastError();
}

cudaError_t launch_gmres_resid(int64_t nvox, int C, int L, const double* E, const double* ax,
                               double* r, cudaStream_t st) {
  const dim3 grid((unsigned)kr_blocks(nvox * C, L), (unsigned)L);
  if (C == 3)
    gm_resid_kernel<3><<<grid, kKrThreads, 0, st>>>(nvox, E, ax, r);
  else if (C == 6)
    gm_resid_kernel<6><<<grid, kKrThreads, 0, st>>>(nvox, E, ax, r);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_krylov_dot(int dtype, int64_t nel, int L, const void* a, const void* b,
                              const void* c, const void* d, double* partials, cudaStream_t st) {
  const dim3 grid((unsigned)kr_blocks(nel, L), (unsigned)L);
  if (dtype == F64)
    kr_dot_kernel<double><<<grid, kKrThreads, 0, st>>>(
        nel, static_cast<const double*>(a), static_cast<const double*>(b),
        static_cast<const double*>(c), static_cast<const double*>(d), partials);
  else
    kr_dot_kernel<float><<<grid, kKrThreads, 0, st>>>(
        nel, static_cast<const float*>(a), static_cast<const float*>(b),
        static_cast<const float*>(c), static_cast<const float*>(d), partials);
  return cudaGetLastError();
}

cudaError_t launch_krylov_scalars(int stage, int64_t nel, int L, const double* partials,
                                  KrylovState* state, cudaStream_t st) {
  kr_scalar_kernel<<<L, kKrThreads, 0, st>>>(stage, partials, kr_blocks(nel, L), state);
  return cudaGetLastError();
}

cudaError_t launch_krylov_update(int dtype, int which, int64_t nel, int L, void* x, const void* p,
                                 const void* s, const void* t, void* r, const void* rh,
                                 const KrylovState* state, double* partials, cudaStream_t st) {
  const dim3 grid((unsigned)kr_blocks(nel, L), (unsigned)L);
  if (dtype == F64) {
    using T = double;
    if (which == 0)
      kr_update_p_kernel<T><<<grid, kKrThreads, 0, st>>>(nel, static_cast<const T*>(r),
                                                         static_cast<const T*>(t),
                                                         static_cast<T*>(x), state);
    else if (which == 1)
      kr_update_s_kernel<T><<<grid, kKrThreads, 0, st>>>(nel, static_cast<const T*>(r),
                                                         static_cast<const T*>(t),
                                                         static_cast<T*>(x), state);
    else
      kr_update_xr_kernel<T><<<grid, kKrThreads, 0, st>>>(
          nel, static_cast<T*>(x), static_cast<const T*>(p), static_cast<const T*>(s),
          static_cast<const T*>(t), static_cast<T*>(r), static_cast<const T*>(rh), state,
          partials);
  } else {
    using T = float;
    if (which == 0)
      kr_update_p_kernel<T><<<grid, kKrThreads, 0, st>>>(nel, static_cast<const T*>(r),
                                                         static_cast<const T*>(t),
                                                         static_cast<T*>(x), state);
    else if (which == 1)
      kr_update_s_kernel<T><<<grid, kKrThreads, 0, st>>>(nel, static_cast<const T*>(r),
                                                         static_cast<const T*>(t),
                                                         static_cast<T*>(x), state);
    else
      kr_update_xr_kernel<T><<<grid, kKrThreads, 0, st>>>(
          nel, static_cast<T*>(x), static_cast<const T*>(p), static_cast<const T*>(s),
          static_cast<const T*>(t), static_cast<T*>(r), static_cast<const T*>(rh), state,
          partials);
  }
  return cudaGetLastError();
}

}  // namespace jb
