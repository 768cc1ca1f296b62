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
// 85 registers (128 where both transforms hold 16 values), so that three
// CTAs of 256 threads share an SM.
//
// n0 = 512, 1024: lane-split tiles.  n0 = 4 NL, n = j + 4 m, k = k1 + NL k2;
// phase 1: the S = NL/16 lanes of a (column, j) slice each load 16 values
// (m = a + S b), transform them in registers, apply w_NL^(a e) and finish
// the NL-point transform across the S lanes by shuffles (radix-2 steps and a
// bit-reversal exchange); phase 2: one lane per (k1, group) applies the
// twiddles w_n0^(j k1), the 4-point transform over j, the contraction at the
// four rows b0 = k1 + NL k2, and the inverse; phase 3 mirrors phase 1.  The
// next tile's rows are prefetched into L2 while a tile is transformed.
//
// No waits besides the block barriers.
#include <cuda_runtime.h>
#include <stdint.h>

#include "jb_green.cuh"
#include "jb_kernels.h"

namespace jb {
namespace {

// ---- shared by both tile kinds ----

template <typename T> struct Axis0Args {
  const cx<T>* in;
  cx<T>* out;
  const cx<T>* tw;   // exp(-2 pi i t / n0), t < n0
  int64_t inner;     // complex columns per row (F * C)
  int64_t pitch;     // complex elements between rows
  int64_t ncoef;     // F
  int64_t m_last;    // 3D: coefficient f = b1 * m_last + b2
  int L;
  int prefetch;      // rows 16-byte aligned (lane-split tiles: L2 prefetch)
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

// the Green contraction of coefficient f at row b0 (te: its C components):
// through the table (TAB), or on the fly for the single-alias operators
// (truncated, finite differences)
template <typename T, int DIM, bool TAB>
__device__ __forceinline__ void contract(const Axis0Args<T>& a, int64_t f, int b0, int n0,
                                         cx<T>* te) {
  if constexpr (TAB) {
    constexpr int NT = GSize<DIM>::value;
    const T* g = a.tab + (size_t)f * NT * n0 + b0;
    T gv[NT];
#pragma unroll
    for (int c = 0; c < NT; ++c) gv[c] = __ldg(g + (size_t)c * n0);
    g_apply<DIM, T>(gv, te);
  } else {
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
      if (f < a.ncoef) contract<T, DIM, false>(a, f, b0, n0, t);
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
// conflict-free except one 2-way phase in FP32.
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
  static constexpr size_t SMEM = (size_t)N1 * PK * sizeof(cx<T>);
  // resident CTAs asked of the register allocator: 24 warps per SM in FP64
  // (at most 85 registers; 16 warps and 128 registers where both transform
  // phases hold 16 values), 32 in FP32 (64 registers)
  static constexpr int MINB =
      (sizeof(T) == 8 ? (N1 == 16 && N2 == 16 ? 16 : 24) : 32) * 32 / THREADS;
};

template <typename T, int DIM, int N0, bool TAB>
__global__ void __launch_bounds__(R8Tile<T, DIM, N0>::THREADS, R8Tile<T, DIM, N0>::MINB)
    green_axis0_r8_kernel(Axis0Args<T> a) {
  using C = cx<T>;
  using K = R8Tile<T, DIM, N0>;
  constexpr int N1 = K::N1, N2 = K::N2;
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
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], a.tw[j * k1]);
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
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmulc(v[k1], a.tw[j * k1]);
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

// ---- lane-split tiles (n0 = 512, 1024) ----

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// lanes per column slice of the lane-split tiles: NL = 16 S is split over S
// consecutive lanes of a warp, 16 values each, m = a + S b for lane a
template <int NL> struct LaneSplit {
  static_assert(NL >= 64 && NL % 16 == 0, "lane-split tiles: NL = 16 S, S >= 4");
  static constexpr int SPL = NL / 16;
  static constexpr int V = 16;
};

// row (relative to j) of value i of lane a (n = j + 4 m)
template <int NL> __device__ __forceinline__ int lane_row(int i, int a) {
  return 4 * (a + LaneSplit<NL>::SPL * i);
}

template <int S> __device__ __forceinline__ int bit_reverse(int x) {
  int r = 0;
#pragma unroll
  for (int m = 1; m < S; m <<= 1) {
    r = (r << 1) | (x & 1);
    x >>= 1;
  }
  return r;
}

// S-point DFT across the S lanes of a slice (S = 4, 8, 16) for each of the
// 16 values: lane a holds V_a[e]; on return lane d holds
// sum_a w_S^(DIR a d) V_a[e].  Radix-2 decimation in frequency over the lane
// index (the lower lane of a pair keeps u + o, the upper (o - u) w_2h^q,
// q = a mod h, both as fma(sg, u, o) times a twiddle that is exactly 1 on the
// lower lane), then a bit-reversal permutation of the lanes.  tw: the axis
// table exp(-2 pi i t / n0), n0 = 64 S.
template <int S, int DIR, typename C>
__device__ __forceinline__ void cross_lane_dft(C* v, int a, const C* tw) {
  using T = decltype(v[0].x);
  constexpr int N0 = 64 * S;
#pragma unroll
  for (int h = S / 2; h >= 1; h >>= 1) {
    const bool upper = (a & h) != 0;
    asm volatile("" ::: "memory");  // one stage's twiddle live at a time
    const C wt = tw[(a % h) * (N0 / (2 * h))];
    const C w = upper ? (DIR > 0 ? cconj(wt) : wt) : mkc(T(1), T(0));
    const T sg = upper ? T(-1) : T(1);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const C u = v[e];
      const C o = mkc(__shfl_xor_sync(0xffffffffu, u.x, h), __shfl_xor_sync(0xffffffffu, u.y, h));
      v[e] = cmul(mkc(fma(sg, u.x, o.x), fma(sg, u.y, o.y)), w);
    }
  }
  const int src = ((threadIdx.x & 31) & ~(S - 1)) | bit_reverse<S>(a);
#pragma unroll
  for (int e = 0; e < 16; ++e)
    v[e] = mkc(__shfl_sync(0xffffffffu, v[e].x, src), __shfl_sync(0xffffffffu, v[e].y, src));
}

// forward transform over m of a column slice: on entry v[i] holds row
// j + 4 m(i, a); on return v[i] = Y[k1] at k1 = i + 16 a
template <int NL, typename C>
__device__ __forceinline__ void lane_fwd(C* v, int a, const C* tw) {
  constexpr int S = LaneSplit<NL>::SPL;
  Dft<16, -1, C>::run(v);
  // V_a[e] = w_NL^(a e) U_a[e], w_NL = w_n0^4; the twiddles are read here,
  // not ahead of the transform, where they would only hold registers
  asm volatile("" ::: "memory");
#pragma unroll
  for (int e = 1; e < 16; ++e) v[e] = cmul(v[e], tw[4 * a * e]);
  cross_lane_dft<S, -1>(v, a, tw);
}

// inverse: v[i] = V[k1] at k1 = i + 16 a -> v[i] = x at row j + 4 m(i, a)
template <int NL, typename C>
__device__ __forceinline__ void lane_inv(C* v, int a, const C* tw) {
  constexpr int S = LaneSplit<NL>::SPL;
  cross_lane_dft<S, +1>(v, a, tw);
  asm volatile("" ::: "memory");
#pragma unroll
  for (int e = 1; e < 16; ++e) v[e] = cmulc(v[e], tw[4 * a * e]);
  Dft<16, +1, C>::run(v);
}

// lane-split tile geometry for n0 = 4 NL (one load case, one 6-column group)
template <typename T, int DIM, int NL> struct R4Tile {
  static constexpr int C = DIM == 3 ? 6 : 3;
  static constexpr int LT = 1;                    // load cases per tile
  static constexpr int NG = 1;                    // 6-column groups per tile
  static constexpr int WC = 6 * NG;               // columns per tile
  static constexpr int SPL = LaneSplit<NL>::SPL;
  static constexpr int P1 = LT * WC * 4 * SPL;    // phase-1/3 threads
  static constexpr int P2 = LT * NL * NG;         // phase-2 threads
  static constexpr int THREADS = P1 > P2 ? P1 : P2;
  static constexpr int P = 4 * WC + 1;            // k1 stride (odd)
  // shared-memory phases: 8 lanes of 16 bytes (FP64), 16 of 8 bytes (FP32)
  static constexpr int LMOD = sizeof(T) == 8 ? 8 : 16;
  // block d of 16 values (lane d of a split slice) sits d OSTEP further on,
  // so that the lanes of a slice write disjoint banks
  static constexpr int OSTEP = SPL >= LMOD ? 1 : LMOD / SPL;
  static constexpr int LS = NL * P + SPL * OSTEP;
  static constexpr size_t SMEM = (size_t)LT * LS * sizeof(cx<T>);
  // resident CTAs asked of the register allocator
  static constexpr int MINB = THREADS > 256 ? 1 : (sizeof(T) == 8 ? 2 : 3);
};

// offset of value k1 in a (load case, j, column) slice
template <typename K> __device__ __forceinline__ int k1_off(int k1) {
  return k1 * K::P + (k1 >> 4) * K::OSTEP;
}

template <typename T, int DIM, int NL, bool TAB>
__global__ void __launch_bounds__(R4Tile<T, DIM, NL>::THREADS, R4Tile<T, DIM, NL>::MINB)
    green_axis0_r4_kernel(Axis0Args<T> a) {
  using C = cx<T>;
  using K = R4Tile<T, DIM, NL>;
  constexpr int N0 = 4 * NL;
  constexpr int NV = LaneSplit<NL>::V;  // 16
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* S = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  // phase-1/3 lane: lane a1 of a split slice, column c, load case l1, j1
  const bool p1 = tid < K::P1;
  const int a1 = tid % K::SPL;
  const int s1 = tid / K::SPL;
  const int c = s1 % K::WC;
  const int l1 = (s1 / K::WC) % K::LT;
  const int j1 = s1 / (K::WC * K::LT);
  // phase-2 lane: load case l2, k1, group g2
  const bool p2 = tid < K::P2;
  const int l2 = tid % K::LT;
  const int k1 = (tid / K::LT) % NL;
  const int g2 = tid / (K::LT * NL);
  const int64_t nchunk = (a.inner + K::WC - 1) / K::WC;
  const int LP = (a.L + K::LT - 1) / K::LT;
  const int64_t total = nchunk * LP;
  const int64_t lstride = (int64_t)N0 * a.pitch;
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    const int64_t chunk = t / LP;
    const int lp = (int)(t - chunk * LP);
    const int64_t col0 = chunk * K::WC;
    // the next tile's rows head for L2 while this one is transformed
    if (a.prefetch) {
      const int64_t tn = t + gridDim.x;
      if (tn < total) {
        const int64_t cn = tn / LP;
        const int lpn = (int)(tn - cn * LP);
        const int64_t cols = min((int64_t)K::WC, a.inner - cn * K::WC);
        const uint32_t bytes = (uint32_t)(cols * sizeof(C)) & ~15u;
        for (int q = tid; q < K::LT * N0; q += blockDim.x) {
          const int l = lpn * K::LT + q / N0;
          if (l < a.L && bytes > 0)
            prefetch_l2(a.in + l * lstride + (int64_t)(q % N0) * a.pitch + cn * K::WC, bytes);
        }
      }
    }
    // phase 1: load the slice's rows, transform over m.  The row pitch is
    // re-read opaquely each tile so that the row offsets are not hoisted out
    // of the tile loop (they would stay live through phase 2)
    int64_t pitch;
    asm volatile("mov.b64 %0, %1;" : "=l"(pitch) : "l"(a.pitch));
    C v[NV];
    const int64_t col = col0 + c;
    const int lg1 = lp * K::LT + l1;
    const bool ok1 = p1 && col < a.inner && lg1 < a.L;
    if (p1) {
      const C* src = a.in + lg1 * lstride + (int64_t)j1 * pitch + col;
#pragma unroll
      for (int i = 0; i < NV; ++i)
        v[i] = ok1 ? src[(int64_t)lane_row<NL>(i, a1) * pitch] : mkc(T(0), T(0));
      lane_fwd<NL>(v, a1, a.tw);
    }
    // (no barrier: phase 3 of the previous tile read these positions in
    // this same lane)
    if (p1) {
      C* s = S + l1 * K::LS + j1 * K::WC + c;
#pragma unroll
      for (int i = 0; i < NV; ++i) s[k1_off<K>(i + NV * a1)] = v[i];
    }
    __syncthreads();
    // phase 2: twiddles, 4-point transform, Green contraction, and back
    const int lg2 = lp * K::LT + l2;
    if (p2 && lg2 < a.L) {
      C* s = S + l2 * K::LS + k1_off<K>(k1) + g2 * 6;
      C x[4][6];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 6; ++q) x[j][q] = s[j * K::WC + q];
      // w_n0^(j k1), j = 1..3 (read each tile: nothing stays live across phases)
      const C tw1 = a.tw[k1], tw2 = a.tw[2 * k1], tw3 = a.tw[3 * k1];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        C g4[4] = {x[0][q], cmul(x[1][q], tw1), cmul(x[2][q], tw2), cmul(x[3][q], tw3)};
        Dft<4, -1, C>::run(g4);
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k][q] = g4[k];
      }
      // coefficients of the group (3D: one; 2D: two of three components)
      const int64_t fbase = (col0 + g2 * 6) / K::C;
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) {
        const int b0 = k1 + NL * k2;
#pragma unroll
        for (int h = 0; h < 6 / K::C; ++h) {
          const int64_t f = fbase + h;
          if (f < a.ncoef) contract<T, DIM, TAB>(a, f, b0, N0, &x[k2][h * K::C]);
        }
        // one row's operator values live at a time
        asm volatile("" ::: "memory");
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        C g4[4] = {x[0][q], x[1][q], x[2][q], x[3][q]};
        Dft<4, +1, C>::run(g4);
        x[0][q] = g4[0];
        x[1][q] = cmulc(g4[1], tw1);
        x[2][q] = cmulc(g4[2], tw2);
        x[3][q] = cmulc(g4[3], tw3);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 6; ++q) s[j * K::WC + q] = x[j][q];
    }
    __syncthreads();
    // phase 3: read the slice back, inverse transform over k1, store
    if (p1) {
      const C* s = S + l1 * K::LS + j1 * K::WC + c;
#pragma unroll
      for (int i = 0; i < NV; ++i) v[i] = s[k1_off<K>(i + NV * a1)];
      lane_inv<NL>(v, a1, a.tw);
      if (ok1) {
        int64_t pitch3;
        asm volatile("mov.b64 %0, %1;" : "=l"(pitch3) : "l"(a.pitch));
        C* dst = a.out + lg1 * lstride + (int64_t)j1 * pitch3 + col;
#pragma unroll
        for (int i = 0; i < NV; ++i) __stcs(dst + (int64_t)lane_row<NL>(i, a1) * pitch3, v[i]);
      }
    }
  }
}

template <typename T, int DIM, int NL, bool TAB>
cudaError_t axis0_r4_go(const Axis0Args<T>& a, cudaStream_t st) {
  using K = R4Tile<T, DIM, NL>;
  auto k = &green_axis0_r4_kernel<T, DIM, NL, TAB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)K::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int64_t tiles = (a.inner + K::WC - 1) / K::WC * ((a.L + K::LT - 1) / K::LT);
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
    case 512: return axis0_r4_go<T, DIM, 128, TAB>(a, st);
    default: return axis0_r4_go<T, DIM, 256, TAB>(a, st);
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
  if (!green_axis0_r4_supported(n0, C, dim)) return cudaErrorNotSupported;
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
  a.prefetch = al(in, 16) && (pitch * cs) % 16 == 0;
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

bool green_axis0_r4_supported(int n0, int C, int dim) {
  return (n0 == 32 || n0 == 64 || n0 == 128 || n0 == 256 || n0 == 512 || n0 == 1024) &&
         ((dim == 3 && C == 6) || (dim == 2 && C == 3));
}

cudaError_t launch_green_axis0_r4(int dtype, const AxisData& ax0, int64_t L, int64_t inner,
                                  int64_t pitch, const void* in, void* out, int C, int dim,
                                  const GreenDeviceTables& gt, int64_t m_last,
                                  cudaStream_t st) {
  return dtype == F64 ? axis0_t<double>(ax0, L, inner, pitch, in, out, C, dim, gt, m_last, st)
                      : axis0_t<float>(ax0, L, inner, pitch, in, out, C, dim, gt, m_last, st);
}

}  // namespace jb
