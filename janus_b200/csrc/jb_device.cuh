// Device building blocks of the janus_b200 Lippmann-Schwinger path (sm_100a).
//
//  * complex arithmetic on double2 / float2;
//  * small DFT kernels (radix 2, 3, 4, 5, 8) held in registers;
//  * one Stockham autosort stage over a shared-memory tile of W independent
//    columns (element (row e, column c) at tile[e * W + c]); a full transform
//    is a sequence of stages, ping-ponging between two tiles.
//
// The Stockham stage follows the textbook formulation: for butterfly j of a
// radix-R stage with Ns = product of the radices already applied,
//   v[r]  = x[j + r n/R] * w_n^(k r n/(Ns R)),  k = j mod Ns,
//   V     = DFT_R(v),
//   y[(j - k) R + k + r Ns] = V[r].
// The twiddles come from a per-axis table tw[t] = exp(-2 pi i t / n) that
// the host computes in long double and rounds once.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace jb {

template <typename T> struct cx_of;
template <> struct cx_of<double> { using type = double2; };
template <> struct cx_of<float> { using type = float2; };
template <typename T> using cx = typename cx_of<T>::type;

__device__ __forceinline__ double2 mkc(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ float2 mkc(float r, float i) { return make_float2(r, i); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mkc(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mkc(a.x, -a.y); }
// a * (DIR * i):  DIR = -1 -> a * (-i) = (a.y, -a.x);  DIR = +1 -> (-a.y, a.x)
template <int DIR, typename C> __device__ __forceinline__ C mul_i(C a) {
  return DIR < 0 ? mkc(a.y, -a.x) : mkc(-a.y, a.x);
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(a.x) s) { return mkc(a.x * s, a.y * s); }

// twiddle w_n^t for direction DIR (-1 forward: tw[t]; +1 inverse: conj)
template <int DIR, typename C> __device__ __forceinline__ C twid(const C* tw, int t) {
  C w = tw[t];
  return DIR < 0 ? w : mkc(w.x, -w.y);
}

// ---------------------------------------------------------------------------
// small DFTs, V[q] = sum_r v[r] exp(DIR 2 pi i r q / R)
// ---------------------------------------------------------------------------
template <int R, int DIR, typename C> struct Dft;

template <int DIR, typename C> struct Dft<2, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR, typename C> struct Dft<4, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    C s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
    C s1 = cadd(v[1], v[3]), d1 = mul_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(s0, s1);
    v[2] = csub(s0, s1);
    v[1] = cadd(d0, d1);
    v[3] = csub(d0, d1);
  }
};

template <int DIR, typename C> struct Dft<3, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = decltype(v[0].x);
    const T s3 = T(0.86602540378443864676372317075294);
    C t1 = cadd(v[1], v[2]);
    C t2 = mkc(v[0].x - T(0.5) * t1.x, v[0].y - T(0.5) * t1.y);
    C t3 = cscale(mul_i<DIR>(csub(v[1], v[2])), s3);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

template <int DIR, typename C> struct Dft<5, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = decltype(v[0].x);
    const T c1 = T(0.30901699437494742410229341718282);
    const T c2 = T(-0.80901699437494742410229341718282);
    const T s1 = T(0.95105651629515357211643933337938);
    const T s2 = T(0.58778525229247312916870595463907);
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C t1 = mkc(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    C t2 = mkc(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    C u1 = mul_i<DIR>(mkc(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    C u2 = mul_i<DIR>(mkc(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = cadd(v[0], cadd(a1, a2));
    v[1] = cadd(t1, u1);
    v[4] = csub(t1, u1);
    v[2] = cadd(t2, u2);
    v[3] = csub(t2, u2);
  }
};

// 6 = 2 x 3 and 12 = 4 x 3 by the prime-factor (Good-Thomas) mapping, which
// needs no twiddles for coprime factors P, Q: input n = (Q p + P q) mod PQ,
// a Q-point DFT over q for each p, a P-point DFT over p for each output
// residue, output k = the CRT index with k = k1 mod P, k = k2 mod Q.
template <int P, int Q, int DIR, typename C>
__device__ __forceinline__ void dft_pfa(C* v, const int (&kmap)[P][Q]) {
  C a[P][Q];
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int q = 0; q < Q; ++q) a[p][q] = v[(Q * p + P * q) % (P * Q)];
    Dft<Q, DIR, C>::run(a[p]);
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    C g[P];
#pragma unroll
    for (int p = 0; p < P; ++p) g[p] = a[p][q];
    Dft<P, DIR, C>::run(g);
#pragma unroll
    for (int p = 0; p < P; ++p) v[kmap[p][q]] = g[p];
  }
}

template <int DIR, typename C> struct Dft<6, DIR, C> {
  // k = (3 k1 + 4 k2) mod 6
  __device__ __forceinline__ static void run(C* v) {
    constexpr int km[2][3] = {{0, 4, 2}, {3, 1, 5}};
    dft_pfa<2, 3, DIR>(v, km);
  }
};

template <int DIR, typename C> struct Dft<12, DIR, C> {
  // k = (9 k1 + 4 k2) mod 12
  __device__ __forceinline__ static void run(C* v) {
    constexpr int km[4][3] = {{0, 4, 8}, {9, 1, 5}, {6, 10, 2}, {3, 7, 11}};
    dft_pfa<4, 3, DIR>(v, km);
  }
};

template <int DIR, typename C> struct Dft<8, DIR, C> {
  __device__ __forceinline__ static void run(C* v) {
    using T = decltype(v[0].x);
    const T h = T(0.70710678118654752440084436210485);
    C a[4], b[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      a[j] = cadd(v[j], v[j + 4]);
      b[j] = csub(v[j], v[j + 4]);
    }
    // b[j] *= w8^(DIR j)
    // w8^DIR = (1 + DIR i)/sqrt2, w8^(2 DIR) = DIR i, w8^(3 DIR) = (-1 + DIR i)/sqrt2
    b[1] = mkc(h * (b[1].x - DIR * b[1].y), h * (b[1].y + DIR * b[1].x));
    b[2] = mul_i<DIR>(b[2]);
    b[3] = mkc(h * (-b[3].x - DIR * b[3].y), h * (-b[3].y + DIR * b[3].x));
    Dft<4, DIR, C>::run(a);
    Dft<4, DIR, C>::run(b);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      v[2 * q] = a[q];
      v[2 * q + 1] = b[q];
    }
  }
};

template <int DIR, typename C> struct Dft<16, DIR, C> {
  // 16 = 4 x 4: DFT4 over stride-4 groups, twiddles w16^(j q), DFT4 across
  __device__ __forceinline__ static void run(C* v) {
    using T = decltype(v[0].x);
    const T c1 = T(0.92387953251128675612818318939679);  // cos(pi/8)
    const T s1 = T(0.38268343236508977172845998403040);  // sin(pi/8)
    const T h = T(0.70710678118654752440084436210485);
    C a[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      C g[4] = {v[j], v[j + 4], v[j + 8], v[j + 12]};
      Dft<4, DIR, C>::run(g);
#pragma unroll
      for (int q = 0; q < 4; ++q) a[j][q] = g[q];
    }
    // w16^(DIR m) = cos(m pi/8) + DIR i sin(m pi/8), m = j q
    auto rot = [&](C x, T c, T s) { return mkc(x.x * c - DIR * x.y * s, x.y * c + DIR * x.x * s); };
    a[1][1] = rot(a[1][1], c1, s1);
    a[1][2] = rot(a[1][2], h, h);
    a[1][3] = rot(a[1][3], s1, c1);
    a[2][1] = rot(a[2][1], h, h);
    a[2][2] = mul_i<DIR>(a[2][2]);
    a[2][3] = rot(a[2][3], -h, h);
    a[3][1] = rot(a[3][1], s1, c1);
    a[3][2] = rot(a[3][2], -h, h);
    a[3][3] = rot(a[3][3], -c1, -s1);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      C g[4] = {a[0][q], a[1][q], a[2][q], a[3][q]};
      Dft<4, DIR, C>::run(g);
#pragma unroll
      for (int p = 0; p < 4; ++p) v[q + 4 * p] = g[p];
    }
  }
};

// ---------------------------------------------------------------------------
// one Stockham stage over a W-column tile
// ---------------------------------------------------------------------------
//
// Thread mapping: a block of T*W threads; thread t works on column
// t % W and on the butterflies j = t / W, t / W + T, ... of every stage, so
// the inner loops need no integer division.  k = j mod Ns uses a
// multiply-high by the host-computed ceil(2^32 / Ns), exact for j < 2^16.

struct AxisPlan {
  int n;
  int nf;
  int fac[24];
  int tstep[24];          // n / (Ns_f * R_f): twiddle index step of stage f
  unsigned nsmagic[24];   // ceil(2^32 / Ns_f) (0 when Ns_f == 1)
};

struct Lane {
  int col;  // column of the tile
  int j0;   // first butterfly
  int T;    // butterfly stride (threads per column)
};

__device__ __forceinline__ Lane make_lane(int W) {
  Lane l;
  l.T = blockDim.x / W;
  l.col = threadIdx.x % W;
  l.j0 = threadIdx.x / W;
  if (l.j0 >= l.T) l.j0 = 1 << 30;  // surplus threads take no butterflies
  return l;
}

template <int R, int DIR, typename C>
__device__ __forceinline__ void stage_fixed(const C* __restrict__ x, C* __restrict__ y,
                                            const C* __restrict__ tw, int n, int Ns,
                                            unsigned magic, int tstep, int W, Lane ln) {
  const int nr = n / R;
  for (int j = ln.j0; j < nr; j += ln.T) {
    const int q = Ns == 1 ? j : (int)__umulhi((unsigned)j, magic);
    const int k = j - q * Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = x[(j + r * nr) * W + ln.col];
    if (k != 0) {
      const int kt = k * tstep;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<DIR>(tw, kt * r));
    }
    Dft<R, DIR, C>::run(v);
    const int base = q * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) y[(base + r * Ns) * W + ln.col] = v[r];
  }
}

// any radix (used for prime factors above 5): direct O(R^2) butterfly that
// reads its inputs from the tile for every output
template <int DIR, typename C>
__device__ __forceinline__ void stage_generic(const C* __restrict__ x, C* __restrict__ y,
                                              const C* __restrict__ tw, int n, int Ns,
                                              unsigned magic, int tstep, int W, int R,
                                              Lane ln) {
  using T = decltype(x[0].x);
  const int nr = n / R;
  for (int j = ln.j0; j < nr; j += ln.T) {
    const int q0 = Ns == 1 ? j : (int)__umulhi((unsigned)j, magic);
    const int k = j - q0 * Ns;
    const int base = q0 * Ns * R + k;
    for (int q = 0; q < R; ++q) {
      C acc = mkc(T(0), T(0));
      for (int r = 0; r < R; ++r) {
        C v = x[(j + r * nr) * W + ln.col];
        if (k != 0 && r != 0) v = cmul(v, twid<DIR>(tw, k * r * tstep));
        const int t = ((r * q) % R) * nr;  // w_R^(rq) = w_n^((rq mod R) n/R)
        acc = cadd(acc, cmul(v, twid<DIR>(tw, t)));
      }
      y[(base + q * Ns) * W + ln.col] = acc;
    }
  }
}

// Full 1D transform of all W columns of tile `a` (length n), using `b` as the
// ping-pong partner.  Returns the tile that holds the result.  All threads of
// the block must call it; it synchronises between stages.
template <int DIR, typename C>
__device__ C* fft_tile(C* a, C* b, const C* tw, const AxisPlan& p, int W, Lane ln) {
  int Ns = 1;
  C* x = a;
  C* y = b;
  for (int f = 0; f < p.nf; ++f) {
    const int R = p.fac[f];
    const unsigned mg = p.nsmagic[f];
    const int ts = p.tstep[f];
    switch (R) {
      case 2: stage_fixed<2, DIR>(x, y, tw, p.n, Ns, mg, ts, W, ln); break;
      case 3: stage_fixed<3, DIR>(x, y, tw, p.n, Ns, mg, ts, W, ln); break;
      case 4: stage_fixed<4, DIR>(x, y, tw, p.n, Ns, mg, ts, W, ln); break;
      case 5: stage_fixed<5, DIR>(x, y, tw, p.n, Ns, mg, ts, W, ln); break;
      case 8: stage_fixed<8, DIR>(x, y, tw, p.n, Ns, mg, ts, W, ln); break;
      default: stage_generic<DIR>(x, y, tw, p.n, Ns, mg, ts, W, R, ln); break;
    }
    __syncthreads();
    Ns *= R;
    C* t = x;
    x = y;
    y = t;
  }
  return x;
}

}  // namespace jb
