// Axis-0 Green pass (sm_100a): each column of the half spectrum
// [L][n0][F][C] (complex, F coefficients of C Mandel components per row) goes
// through the forward transform along axis 0, every coefficient is contracted
// with the discrete Green operator, and the column is transformed back: the
// work of janus/green.pyx:356-390 (DiscreteGreenOperator3D.c_apply, axis-0
// part) and 185-216 (2D).  One HBM round trip per value; the result is
// unnormalised (the c2r pass scales by 1/N, as
// janus/fft/serial/_serial_fft.pyx:121-150 does).
//
// n0 = 32 ... 256: five-phase tiles.  n0 = N1 N2 is split as n = j + N2 m,
// k = k1 + N1 k2:
//   X[k1 + N1 k2] = sum_j w_N2^(j k2) [w_n0^(j k1) sum_m x[j + N2 m] w_N1^(m k1)].
// A tile is one load case, 6 NG columns (NG 6-column groups: one 3D
// coefficient or two 2D ones each) and all n0 rows, in shared memory as
// S[k1][j][c].
//   P1 (lane per column c and j): the N1 values x[j + N2 m] from global
//      memory, the N1-point transform in registers, the twiddles
//      w_n0^(j k1), to S[k1][j][c].
//   2a (lane per k1 and c): the N2-point transform over j in registers, in
//      place (j becomes k2).
//   2b (lane per k1, k2 and group): the group's components at
//      b0 = k1 + N1 k2 contracted with the operator (a symmetric Mandel
//      matrix from the table, or on the fly), in place.
//   2c: the inverse of 2a; P3: the conjugate twiddles, the inverse of P1's
//      transform and the store to global memory.
// Every transform is a compile-time sequence in one lane's registers (no
// shuffles); the phases hand values over through shared memory, four
// barriers per tile.  P3 reads exactly the positions its own lane's P1 of
// the next tile writes, so no barrier separates them.  The lanes use at most
// 85 registers in FP64 (128 where both transforms hold 16 values), so that
// three CTAs of 256 threads share an SM, and 51 in FP32 (five CTAs).
//
// n0 = 192, 384, 512, 768, 1024: seven-phase tiles, the same scheme with the
// N2-point transform split once more (N1 8 8 with N1 = 3, 6, 8, 12, 16): P1
// (6 and 12 points by the prime-factor mappings 2 x 3 and 4 x 3), then an
// 8-point transform over the high part of j with its twiddles, an 8-point
// transform over the low part, the contraction, and the mirror images; the
// middle phases loop over more jobs than the block has lanes.
//
// No waits besides the block barriers.
#include <cuda_runtime.h>
#include <stdint.h>

#include "jb_green.cuh"
#include "jb_kernels.h"

namespace jb {
namespace {

// ---- shared by the tile kinds ----

template <typename T> struct Axis0Args {
  const cx<T>* in;
  cx<T>* out;
  const cx<T>* tw;   // exp(-2 pi i t / n0), t < n0
  int64_t inner;     // complex columns per row (F * C)
  int64_t pitch;     // complex elements between rows
  int64_t ncoef;     // F
  int64_t m_last;    // 3D: coefficient f = b1 * m_last + b2
  int L;
  GreenTables<T> gt;
  const T* tab;      // symmetric Mandel matrices [f][c][b0], or nullptr: on the fly
};

// the value, re-read each time: lane indices derived from it are recomputed
// in each phase instead of being hoisted out of the tile loop and held in
// registers throughout
__device__ __forceinline__ int opaque(int x) {
  int r;
  asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(x));
  return r;
}

// the Green contraction of coefficient f at row b0 on the fly (te: its C
// components), for the single-alias operators (truncated, finite
// differences); the table form is in contract_row
template <typename T, int DIM>
__device__ __forceinline__ void contract_fly(const Axis0Args<T>& a, int64_t f, int b0,
                                             cx<T>* te) {
  constexpr int S = DIM == 3 ? 6 : 3;
  int b1, b2;
  if (DIM == 3) {
    b1 = (int)(f / a.m_last);
    b2 = (int)(f - (int64_t)b1 * a.m_last);
  } else {
    b1 = (int)f;
    b2 = 0;
  }
  const AxisK<T> a0 = axis_values(a.gt, 0, b0);
  const AxisK<T> a1 = axis_values(a.gt, 1, b1);
  const AxisK<T> a2 = DIM == 3 ? axis_values(a.gt, 2, b2) : a1;
  T k0 = a0.v[0], k1 = a1.v[0], k2 = a2.v[0];
  if (a.gt.variant == 2) willot_k<DIM, T>(a0.v, a1.v, a2.v, k0, k1, k2);
  cx<T> t[S], acc[S];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    t[i] = te[i];
    acc[i] = mkc(T(0), T(0));
  }
  if (DIM == 2)
    gamma2_acc(k0, k1, T(1), t, acc, a.gt.inv2g, a.gt.c1);
  else
    gamma3_acc(k0, k1, k2, T(1), t, acc, a.gt.inv2g, a.gt.c1);
#pragma unroll
  for (int i = 0; i < S; ++i) te[i] = acc[i];
}

// index of entry (i, j) of a symmetric S x S matrix stored as its diagonal
// then the upper triangle row by row (the layout g_apply reads)
template <int S> __device__ __forceinline__ constexpr int gidx(int i, int j) {
  const int lo = i < j ? i : j, hi = i < j ? j : i;
  return lo == hi ? lo : S + lo * (S - 1) - lo * (lo - 1) / 2 + (hi - lo - 1);
}

// dst = G te for the coefficients of one 6-column group at row b0, written
// component by component (only te and the operator values stay live); a
// coefficient past the end is copied unchanged
template <typename T, int DIM, bool TAB, typename C>
__device__ __forceinline__ void contract_row(const Axis0Args<T>& a, int64_t fbase, int b0,
                                             int n0, C* te, C* dst) {
  constexpr int S = DIM == 3 ? 6 : 3;
#pragma unroll
  for (int h = 0; h < 6 / S; ++h) {
    const int64_t f = fbase + h;
    C* t = te + h * S;
    if constexpr (TAB) {
      if (f < a.ncoef) {
        constexpr int NT = GSize<DIM>::value;
        const T* g = a.tab + (size_t)f * NT * n0 + b0;
        T gv[NT];
#pragma unroll
        for (int k = 0; k < NT; ++k) gv[k] = __ldg(g + (size_t)k * n0);
#pragma unroll
        for (int i = 0; i < S; ++i) {
          T re = T(0), im = T(0);
#pragma unroll
          for (int j = 0; j < S; ++j) {
            re = fma(gv[gidx<S>(i, j)], t[j].x, re);
            im = fma(gv[gidx<S>(i, j)], t[j].y, im);
          }
          dst[h * S + i] = mkc(re, im);
        }
      } else {
#pragma unroll
        for (int i = 0; i < S; ++i) dst[h * S + i] = t[i];
      }
    } else {
      if (f < a.ncoef) contract_fly<T, DIM>(a, f, b0, t);
#pragma unroll
      for (int i = 0; i < S; ++i) dst[h * S + i] = t[i];
    }
  }
}

int g_sm_count = 0;

// persistent grid: the resident CTAs of every SM, at most one per tile
template <typename KFn>
int persistent_grid(KFn k, int threads, size_t smem, int64_t tiles) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        g_sm_count <= 0)
      g_sm_count = 148;
  }
  const int64_t g = (int64_t)per_sm * g_sm_count;
  return (int)(tiles < g ? tiles : g);
}

// ---- five-phase tiles (n0 = 32 ... 256) ----

// Five-phase tile of one load case, 6 NG columns and all n0 = N1 N2 rows
// (n = j + N2 m, k = k1 + N1 k2), in shared memory as S[k1][j][c] with row
// (j) stride PJ = 6 NG and k1 stride PK = N2 PJ + pad: the pad (1 for FP64,
// 2 for FP32 tiles of two groups, 1 otherwise) was found by an exhaustive
// search of the bank conflicts of every phase's access pattern, all
// conflict-free except one 2-way phase in FP32.  A copy of the n0 axis
// twiddles follows the tile.
template <int N0> struct R8Shape;
template <> struct R8Shape<32> { static constexpr int N1 = 8, N2 = 4, NG = 4; };
template <> struct R8Shape<64> { static constexpr int N1 = 8, N2 = 8, NG = 2; };
template <> struct R8Shape<128> { static constexpr int N1 = 8, N2 = 16, NG = 2; };
template <> struct R8Shape<256> { static constexpr int N1 = 16, N2 = 16, NG = 1; };

template <typename T, int DIM, int N0> struct R8Tile {
  static constexpr int N1 = R8Shape<N0>::N1, N2 = R8Shape<N0>::N2, NG = R8Shape<N0>::NG;
  static constexpr int C = DIM == 3 ? 6 : 3;
  static constexpr int WC = 6 * NG;        // columns
  static constexpr int P1 = WC * N2;       // phase-1/3 lanes (c, j)
  static constexpr int P2A = N1 * WC;      // phase-2a/2c lanes (k1, c)
  static constexpr int P2B = N1 * N2 * NG; // contraction lanes (k1, k2, group)
  static constexpr int THREADS = P1 > P2A ? (P1 > P2B ? P1 : P2B) : (P2A > P2B ? P2A : P2B);
  static constexpr int PJ = WC;
  static constexpr int PK = N2 * PJ + (sizeof(T) == 8 || NG != 2 ? 1 : 2);
  static constexpr size_t SMEM = ((size_t)N1 * PK + N0) * sizeof(cx<T>);
  // resident CTAs asked of the register allocator: 24 warps per SM in FP64
  // (at most 85 registers; 16 warps and 128 registers where both transform
  // phases hold 16 values), 40 in FP32 (51 registers; 32 where both hold 16).
  // Measured at 128^3 x 6: FP32 Green pass 0.206 ms at 32 warps, 0.195 at
  // 40, 0.202 at 48.
  static constexpr int MINB =
      (sizeof(T) == 8 ? (N1 == 16 && N2 == 16 ? 16 : 24) : (N1 == 16 && N2 == 16 ? 32 : 40)) *
      32 / THREADS;
};

template <typename T, int DIM, int N0, bool TAB>
__global__ void __launch_bounds__(R8Tile<T, DIM, N0>::THREADS, R8Tile<T, DIM, N0>::MINB)
    green_axis0_r8_kernel(Axis0Args<T> a) {
  using C = cx<T>;
  using K = R8Tile<T, DIM, N0>;
  constexpr int N1 = K::N1, N2 = K::N2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* S = reinterpret_cast<C*>(smem_raw);
  // the axis twiddles, copied once per CTA: P1 and P3 read them from shared
  // memory (measured 0.364 -> 0.352 ms FP64, 0.196 -> 0.191 ms FP32 against
  // reading them through L1 at 128^3 x 6)
  C* TW = S + (size_t)N1 * K::PK;
  const int tid = threadIdx.x;
  for (int i = tid; i < N0; i += blockDim.x) TW[i] = a.tw[i];
  __syncthreads();
  const int LP = a.L;
  const int64_t total = (a.inner + K::WC - 1) / K::WC * LP;
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    const int64_t chunk = t / LP;
    const int lg = (int)(t - chunk * LP);
    const int64_t col0 = chunk * K::WC;
    // P1: lane (c, j): N1-point transform over m, twiddles w_n0^(j k1)
    if (tid < K::P1) {
      const int tq = opaque(tid);
      const int c = tq % K::WC, j = tq / K::WC;
      const bool ok = col0 + c < a.inner;
      C v[N1];
      const int64_t pitch = a.pitch;
      const C* src = a.in + ((int64_t)lg * N0 + j) * pitch + col0 + c;
#pragma unroll
      for (int m = 0; m < N1; ++m) v[m] = ok ? src[(int64_t)m * N2 * pitch] : mkc(T(0), T(0));
      Dft<N1, -1, C>::run(v);
      asm volatile("" ::: "memory");
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], TW[j * k1]);
      C* s = S + j * K::PJ + c;
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) s[k1 * K::PK] = v[k1];
    }
    __syncthreads();
    // 2a: lane (k1, c): N2-point transform over j
    if (tid < K::P2A) {
      const int tq = opaque(tid);
      C* s = S + (tq % N1) * K::PK + tq / N1;
      C w[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) w[j] = s[j * K::PJ];
      Dft<N2, -1, C>::run(w);
#pragma unroll
      for (int j = 0; j < N2; ++j) s[j * K::PJ] = w[j];
    }
    __syncthreads();
    // 2b: lane (k1, k2, g2): the contraction at b0 = k1 + N1 k2
    if (tid < K::P2B) {
      const int tq = opaque(tid);
      const int k1 = tq % N1, k2 = (tq / N1) % N2, g2 = tq / (N1 * N2);
      C* s = S + k1 * K::PK + k2 * K::PJ + g2 * 6;
      C y[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) y[q] = s[q];
      contract_row<T, DIM, TAB>(a, (col0 + g2 * 6) / K::C, k1 + N1 * k2, N0, y, s);
    }
    __syncthreads();
    // 2c: inverse over k2
    if (tid < K::P2A) {
      const int tq = opaque(tid);
      C* s = S + (tq % N1) * K::PK + tq / N1;
      C w[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) w[j] = s[j * K::PJ];
      Dft<N2, +1, C>::run(w);
#pragma unroll
      for (int j = 0; j < N2; ++j) s[j * K::PJ] = w[j];
    }
    __syncthreads();
    // P3: conj twiddles, inverse over k1, store (the next tile's P1 writes
    // only the positions this lane reads here: no barrier)
    if (tid < K::P1) {
      const int tq = opaque(tid);
      const int c = tq % K::WC, j = tq / K::WC;
      C v[N1];
      const C* s = S + j * K::PJ + c;
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) v[k1] = s[k1 * K::PK];
      asm volatile("" ::: "memory");
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmulc(v[k1], TW[j * k1]);
      Dft<N1, +1, C>::run(v);
      if (col0 + c < a.inner) {
        const int64_t pitch = a.pitch;
        C* dst = a.out + ((int64_t)lg * N0 + j) * pitch + col0 + c;
#pragma unroll
        for (int m = 0; m < N1; ++m) __stcs(dst + (int64_t)m * N2 * pitch, v[m]);
      }
    }
  }
}

template <typename T, int DIM, int N0, bool TAB>
cudaError_t axis0_r8_go(const Axis0Args<T>& a, cudaStream_t st) {
  using K = R8Tile<T, DIM, N0>;
  auto k = &green_axis0_r8_kernel<T, DIM, N0, TAB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)K::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int64_t tiles = (a.inner + K::WC - 1) / K::WC * a.L;
  k<<<persistent_grid(k, K::THREADS, K::SMEM, tiles), K::THREADS, K::SMEM, st>>>(a);
  return cudaGetLastError();
}

// ---- seven-phase tiles (n0 = 192, 384, 512, 768, 1024) ----

// n0 = N1 A B: n = j + M m (M = A B), k = k1 + N1 k2; the M-point transform
// over j = ja + A jb is split again, k2 = kb + B ka:
//   sum_j w_M^(j k2) z_j = sum_ja w_A^(ja ka) [w_M^(ja kb) sum_jb w_B^(jb kb) z_(ja + A jb)].
// A tile is one load case x 6 columns x n0 rows in shared memory as
// S[k1][p][c] (p = ja + A jb, then ja + A kb, then ka + A kb).  P1 (lane per
// column and j): N1-point transform over m and the twiddles w_n0^(j k1);
// 2a (job per k1, ja, column): B-point transform over jb and the twiddles
// w_M^(ja kb); 2a' (job per k1, kb, column): A-point transform over ja; 2b
// (job per k1, kb, ka): the contraction at b0 = k1 + N1 (kb + B ka); then
// the mirror images.  The middle phases have more jobs than the block has
// lanes and loop over them.  k1 stride padded by one value: every phase is
// free of bank conflicts in FP64 (searched on the CPU, like the five-phase
// tiles).
template <int N0> struct R16Shape;
template <> struct R16Shape<512> { static constexpr int N1 = 8, A = 8, B = 8; };
template <> struct R16Shape<1024> { static constexpr int N1 = 16, A = 8, B = 8; };
// 192, 384, 768 = 3, 6, 12 times 64: a 3-point first phase, or a 6- or
// 12-point one (2 x 3, 4 x 3 prime-factor transforms)
template <> struct R16Shape<192> { static constexpr int N1 = 3, A = 8, B = 8; };
template <> struct R16Shape<384> { static constexpr int N1 = 6, A = 8, B = 8; };
template <> struct R16Shape<768> { static constexpr int N1 = 12, A = 8, B = 8; };

template <typename T, int DIM, int N0> struct R16Tile {
  static constexpr int N1 = R16Shape<N0>::N1, A = R16Shape<N0>::A, B = R16Shape<N0>::B;
  static constexpr int M = A * B;
  static constexpr int C = DIM == 3 ? 6 : 3;
  static constexpr int WC = 6;
  static constexpr int THREADS = WC * M;  // P1 lanes (c, j)
  static constexpr int J2A = N1 * A * WC;
  static constexpr int J2A_ = N1 * B * WC;
  static constexpr int J2B = N1 * M;
  static constexpr int PJ = WC;
  static constexpr int PK = M * PJ + 1;
  static constexpr size_t SMEM = (size_t)N1 * PK * sizeof(cx<T>);
  // 24 warps per SM in FP64 (at most 85 registers: the 1024-point tile
  // spills about 200 bytes there and still measured faster than at 12 warps
  // without spills); in FP32 24, and 36 for the 1024-point tile (56
  // registers, no spills: 1024^2 x 3 Green pass 0.0481 -> 0.0451 ms, while
  // the 768-point tile measured 0.0310 -> 0.0350 ms at that cap)
  static constexpr int MINB =
      (sizeof(T) == 8 ? 24 : (N0 == 1024 ? 36 : 24)) * 32 / THREADS;
};

template <typename T, int DIM, int N0, bool TAB>
__global__ void __launch_bounds__(R16Tile<T, DIM, N0>::THREADS, R16Tile<T, DIM, N0>::MINB)
    green_axis0_r16_kernel(Axis0Args<T> a) {
  using C = cx<T>;
  using K = R16Tile<T, DIM, N0>;
  constexpr int N1 = K::N1, A = K::A, B = K::B, M = K::M;
  constexpr int TS = N0 / M;  // w_M = w_n0^TS
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* S = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  const int LP = a.L;
  const int64_t total = (a.inner + K::WC - 1) / K::WC * LP;
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    const int64_t chunk = t / LP;
    const int lg = (int)(t - chunk * LP);
    const int64_t col0 = chunk * K::WC;
    // P1: lane (c, j): N1-point transform over m, twiddles w_n0^(j k1)
    {
      const int tq = opaque(tid);
      const int c = tq % K::WC, j = tq / K::WC;
      const bool ok = col0 + c < a.inner;
      C v[N1];
      const int64_t pitch = a.pitch;
      const C* src = a.in + ((int64_t)lg * N0 + j) * pitch + col0 + c;
#pragma unroll
      for (int m = 0; m < N1; ++m) v[m] = ok ? src[(int64_t)m * M * pitch] : mkc(T(0), T(0));
      Dft<N1, -1, C>::run(v);
      asm volatile("" ::: "memory");
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], a.tw[j * k1]);
      C* s = S + j * K::PJ + c;
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) s[k1 * K::PK] = v[k1];
    }
    __syncthreads();
    // 2a: job (k1, ja, c): B-point transform over jb, twiddles w_M^(ja kb)
    for (int job = opaque(tid); job < K::J2A; job += K::THREADS) {
      const int k1 = job % N1, ja = (job / N1) % A, c = job / (N1 * A);
      C* s = S + k1 * K::PK + ja * K::PJ + c;
      C w[B];
#pragma unroll
      for (int jb = 0; jb < B; ++jb) w[jb] = s[A * jb * K::PJ];
      Dft<B, -1, C>::run(w);
      asm volatile("" ::: "memory");
#pragma unroll
      for (int kb = 1; kb < B; ++kb) w[kb] = cmul(w[kb], a.tw[TS * ja * kb]);
#pragma unroll
      for (int kb = 0; kb < B; ++kb) s[A * kb * K::PJ] = w[kb];
    }
    __syncthreads();
    // 2a': job (k1, kb, c): A-point transform over ja
    for (int job = opaque(tid); job < K::J2A_; job += K::THREADS) {
      const int k1 = job % N1, kb = (job / N1) % B, c = job / (N1 * B);
      C* s = S + k1 * K::PK + A * kb * K::PJ + c;
      C w[A];
#pragma unroll
      for (int ja = 0; ja < A; ++ja) w[ja] = s[ja * K::PJ];
      Dft<A, -1, C>::run(w);
#pragma unroll
      for (int ka = 0; ka < A; ++ka) s[ka * K::PJ] = w[ka];
    }
    __syncthreads();
    // 2b: job (k1, kb, ka): the contraction at b0 = k1 + N1 (kb + B ka)
    for (int job = opaque(tid); job < K::J2B; job += K::THREADS) {
      const int k1 = job % N1, kb = (job / N1) % B, ka = job / (N1 * B);
      C* s = S + k1 * K::PK + (ka + A * kb) * K::PJ;
      C y[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) y[q] = s[q];
      contract_row<T, DIM, TAB>(a, col0 / K::C, k1 + N1 * (kb + B * ka), N0, y, s);
    }
    __syncthreads();
    // 2c': inverse over ka
    for (int job = opaque(tid); job < K::J2A_; job += K::THREADS) {
      const int k1 = job % N1, kb = (job / N1) % B, c = job / (N1 * B);
      C* s = S + k1 * K::PK + A * kb * K::PJ + c;
      C w[A];
#pragma unroll
      for (int ja = 0; ja < A; ++ja) w[ja] = s[ja * K::PJ];
      Dft<A, +1, C>::run(w);
#pragma unroll
      for (int ja = 0; ja < A; ++ja) s[ja * K::PJ] = w[ja];
    }
    __syncthreads();
    // 2c: conjugate twiddles, inverse over kb
    for (int job = opaque(tid); job < K::J2A; job += K::THREADS) {
      const int k1 = job % N1, ja = (job / N1) % A, c = job / (N1 * A);
      C* s = S + k1 * K::PK + ja * K::PJ + c;
      C w[B];
#pragma unroll
      for (int kb = 0; kb < B; ++kb) w[kb] = s[A * kb * K::PJ];
      asm volatile("" ::: "memory");
#pragma unroll
      for (int kb = 1; kb < B; ++kb) w[kb] = cmulc(w[kb], a.tw[TS * ja * kb]);
      Dft<B, +1, C>::run(w);
#pragma unroll
      for (int jb = 0; jb < B; ++jb) s[A * jb * K::PJ] = w[jb];
    }
    __syncthreads();
    // P3: conjugate twiddles, inverse over k1, store (no barrier before the
    // next tile's P1: it writes only the positions this lane reads here)
    {
      const int tq = opaque(tid);
      const int c = tq % K::WC, j = tq / K::WC;
      C v[N1];
      const C* s = S + j * K::PJ + c;
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) v[k1] = s[k1 * K::PK];
      asm volatile("" ::: "memory");
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmulc(v[k1], a.tw[j * k1]);
      Dft<N1, +1, C>::run(v);
      if (col0 + c < a.inner) {
        const int64_t pitch = a.pitch;
        C* dst = a.out + ((int64_t)lg * N0 + j) * pitch + col0 + c;
#pragma unroll
        for (int m = 0; m < N1; ++m) __stcs(dst + (int64_t)m * M * pitch, v[m]);
      }
    }
  }
}

template <typename T, int DIM, int N0, bool TAB>
cudaError_t axis0_r16_go(const Axis0Args<T>& a, cudaStream_t st) {
  using K = R16Tile<T, DIM, N0>;
  auto k = &green_axis0_r16_kernel<T, DIM, N0, TAB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)K::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int64_t tiles = (a.inner + K::WC - 1) / K::WC * a.L;
  k<<<persistent_grid(k, K::THREADS, K::SMEM, tiles), K::THREADS, K::SMEM, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int DIM, bool TAB>
cudaError_t axis0_n(const Axis0Args<T>& a, int n0, cudaStream_t st) {
  switch (n0) {
    case 32: return axis0_r8_go<T, DIM, 32, TAB>(a, st);
    case 64: return axis0_r8_go<T, DIM, 64, TAB>(a, st);
    case 128: return axis0_r8_go<T, DIM, 128, TAB>(a, st);
    case 256: return axis0_r8_go<T, DIM, 256, TAB>(a, st);
    case 192: return axis0_r16_go<T, DIM, 192, TAB>(a, st);
    case 384: return axis0_r16_go<T, DIM, 384, TAB>(a, st);
    case 512: return axis0_r16_go<T, DIM, 512, TAB>(a, st);
    case 768: return axis0_r16_go<T, DIM, 768, TAB>(a, st);
    default: return axis0_r16_go<T, DIM, 1024, TAB>(a, st);
  }
}

template <typename T, bool TAB>
cudaError_t axis0_dim(const Axis0Args<T>& a, int n0, int dim, cudaStream_t st) {
  return dim == 3 ? axis0_n<T, 3, TAB>(a, n0, st) : axis0_n<T, 2, TAB>(a, n0, st);
}

template <typename T>
cudaError_t axis0_t(const AxisData& ax0, int64_t L, int64_t inner, int64_t pitch,
                    const void* in, void* out, int C, int dim, const GreenDeviceTables& gt,
                    int64_t m_last, cudaStream_t st) {
  const int n0 = ax0.plan.n;
  if (!green_axis0_regs_supported(n0, C, dim)) return cudaErrorNotSupported;
  if (L < 1 || L > 65535 || inner < 1 || (inner % C) != 0 || pitch < inner)
    return cudaErrorInvalidValue;
  const size_t cs = sizeof(cx<T>);
  auto al = [](const void* p, size_t b) { return (reinterpret_cast<uintptr_t>(p) % b) == 0; };
  if (!al(in, cs) || !al(out, cs) || !ax0.tw) return cudaErrorInvalidValue;
  Axis0Args<T> a{};
  a.in = static_cast<const cx<T>*>(in);
  a.out = static_cast<cx<T>*>(out);
  a.tw = static_cast<const cx<T>*>(ax0.tw);
  a.inner = inner;
  a.pitch = pitch;
  a.ncoef = inner / C;
  a.m_last = m_last;
  a.L = (int)L;
  GreenTables<T> t{};
  for (int d = 0; d < 3; ++d) {
    t.kt[d] = static_cast<const T*>(gt.kt[d]);
    t.kn[d] = static_cast<const T*>(gt.kn[d]);
    t.kp[d] = static_cast<const T*>(gt.kp[d]);
    t.wn[d] = static_cast<const T*>(gt.wn[d]);
    t.wp[d] = static_cast<const T*>(gt.wp[d]);
  }
  t.inv2g = static_cast<T>(gt.inv2g);
  t.c1 = static_cast<T>(gt.c1);
  t.variant = gt.variant;
  a.gt = t;
  a.tab = static_cast<const T*>(gt.mn);
  if (a.tab != nullptr) return axis0_dim<T, true>(a, n0, dim, st);
  // on the fly: the single-alias operators only (the filtered operator's
  // 2^d aliases per coefficient are left to the table)
  if (gt.variant == FILTERED) return cudaErrorNotSupported;
  return axis0_dim<T, false>(a, n0, dim, st);
}

}  // namespace

bool green_axis0_regs_supported(int n0, int C, int dim) {
  return (n0 == 32 || n0 == 64 || n0 == 128 || n0 == 192 || n0 == 256 || n0 == 384 ||
          n0 == 512 || n0 == 768 || n0 == 1024) &&
         ((dim == 3 && C == 6) || (dim == 2 && C == 3));
}

cudaError_t launch_green_axis0_regs(int dtype, const AxisData& ax0, int64_t L, int64_t inner,
                                  int64_t pitch, const void* in, void* out, int C, int dim,
                                  const GreenDeviceTables& gt, int64_t m_last,
                                  cudaStream_t st) {
  return dtype == F64 ? axis0_t<double>(ax0, L, inner, pitch, in, out, C, dim, gt, m_last, st)
                      : axis0_t<float>(ax0, L, inner, pitch, in, out, C, dim, gt, m_last, st);
}

}  // namespace jb
