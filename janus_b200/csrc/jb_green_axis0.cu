// Axis-0 Green pass with a register-resident middle stage (sm_100a).
//
// The pass takes each column of the half spectrum [L][n0][F][C] (complex,
// F coefficients of C Mandel components per row) through the forward
// transform along axis 0, contracts every coefficient with the discrete
// Green operator, and transforms back: the work of janus/green.pyx:356-390
// (DiscreteGreenOperator3D.c_apply, axis-0 part) and 185-216 (2D).
//
// n0 = 4 NL is split as n = j + 4 m (j < 4, m < NL), k = k1 + NL k2:
//   X[k1 + NL k2] = sum_j w4^(j k2) w_n0^(j k1) sum_m x[j + 4 m] w_NL^(m k1).
// Phase 1: the lanes of a (load case, column, j) slice load its NL values of
//          the column straight from global memory into registers and compute
//          the NL-point transform over m in registers: one lane for NL <= 16;
//          for NL = 16 S, S lanes (m = a + S b), each a 16-point transform
//          of its rows, a twiddle, then an S-point transform across the
//          lanes by shuffles (S = 2: one radix-2 step with compile-time
//          twiddles; S = 4..16: radix-2 steps and a bit-reversal exchange);
//          then the NL results go to shared memory.
// Phase 2: one thread per (load case, k1, group of 6 columns: one 3D
//          coefficient or two 2D ones) reads its 4 x 6 values, applies the
//          twiddles w_n0^(j k1) and the 4-point transform over j, contracts
//          the Green operator at the 4 rows b0 = k1 + NL k2 in registers,
//          transforms back and writes the 4 x 6 values in place.
// Phase 3: the phase-1 lanes read their values, transform back and store
//          the column to global memory.
// Each spectral value therefore crosses shared memory twice each way and is
// read and written once in HBM.  Up to n0 = 256 a tile holds two load cases
// of the same coefficients, so the two lanes of a phase-2 pair read the same
// table entries in one broadcast.  The next tile's rows are prefetched into L2
// while the current tile is transformed.  There are no waits besides the
// block barriers.  The result is unnormalised (the c2r pass scales by 1/N,
// as janus/fft/serial/_serial_fft.pyx:121-150 does).
#include <cuda_runtime.h>
#include <stdint.h>

#include "jb_green.cuh"
#include "jb_kernels.h"

namespace jb {
namespace {

// cos(pi e / 16), e = 0..8 (correctly rounded to double)
__host__ __device__ constexpr double cospi16(int e) {
  return e == 0   ? 1.0
         : e == 1 ? 0.98078528040323044912618223613424
         : e == 2 ? 0.92387953251128675612818318939679
         : e == 3 ? 0.83146961230254523707878837761791
         : e == 4 ? 0.70710678118654752440084436210485
         : e == 5 ? 0.55557023301960222474283081394853
         : e == 6 ? 0.38268343236508977172845998403040
         : e == 7 ? 0.19509032201612826784828486847702
                  : 0.0;
}
// forward twiddle w32^e = exp(-2 pi i e / 32) = (cos(pi e/16), -sin(pi e/16)), e < 16
template <typename T> __device__ __forceinline__ constexpr T w32_re(int e) {
  return e <= 8 ? T(cospi16(e)) : T(-cospi16(16 - e));
}
template <typename T> __device__ __forceinline__ constexpr T w32_im(int e) {
  return e <= 8 ? T(-cospi16(8 - e)) : T(-cospi16(e - 8));
}

// multiply by w32^e (DIR -1) or its conjugate (DIR +1) where `on` (the odd
// lane of a pair), by 1 elsewhere: a per-lane selection instead of a
// divergent branch
template <int DIR, int E, typename C> __device__ __forceinline__ C rot32_if(C a, bool on) {
  using T = decltype(a.x);
  if constexpr (E == 0) {
    return a;
  } else {
    const T c = on ? w32_re<T>(E) : T(1);
    const T s = on ? (DIR < 0 ? w32_im<T>(E) : -w32_im<T>(E)) : T(0);
    return mkc(a.x * c - a.y * s, a.y * c + a.x * s);
  }
}

template <typename C> __device__ __forceinline__ C shfl_xor1(C v) {
  return mkc(__shfl_xor_sync(0xffffffffu, v.x, 1), __shfl_xor_sync(0xffffffffu, v.y, 1));
}

// lanes per column slice and values a lane holds: NL <= 16 is held by one
// lane; NL = 16 S (S = 2, 4, 8, 16) is split over S consecutive lanes of a
// warp, 16 values each, m = a + S b for lane a
template <int NL> struct LaneSplit {
  static constexpr int SPL = NL <= 16 ? 1 : NL / 16;
  static constexpr int V = NL / SPL;
};

// row (relative to j) of value i of lane a (n = j + 4 m)
template <int NL> __device__ __forceinline__ int lane_row(int i, int a) {
  return 4 * (a + LaneSplit<NL>::SPL * i);
}

template <int E, typename C> struct PairLoop {
  // forward: v[e] = U_a[e] -> Y[e + 16 a], with Y[e] = U0 + w32^e U1 and
  // Y[e + 16] = U0 - w32^e U1
  __device__ __forceinline__ static void fwd(C* v, bool odd) {
    const C u = rot32_if<-1, E>(v[E], odd);
    const C o = shfl_xor1(u);
    v[E] = odd ? csub(o, u) : cadd(u, o);
    PairLoop<E + 1, C>::fwd(v, odd);
  }
  // inverse: v[e] = V[e + 16 a] -> lane 0: V[e] + V[e + 16], lane 1:
  // conj(w32^e) (V[e] - V[e + 16])
  __device__ __forceinline__ static void inv(C* v, bool odd) {
    const C u = v[E];
    const C o = shfl_xor1(u);
    v[E] = odd ? rot32_if<+1, E>(csub(o, u), true) : cadd(u, o);
    PairLoop<E + 1, C>::inv(v, odd);
  }
};
template <typename C> struct PairLoop<16, C> {
  __device__ __forceinline__ static void fwd(C*, bool) {}
  __device__ __forceinline__ static void inv(C*, bool) {}
};

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
// q = a mod h), then a bit-reversal permutation of the lanes.  tw: the
// axis table exp(-2 pi i t / n0), n0 = 64 S.
template <int S, int DIR, typename C>
__device__ __forceinline__ void cross_lane_dft(C* v, int a, const C* tw) {
  constexpr int N0 = 64 * S;
#pragma unroll
  for (int h = S / 2; h >= 1; h >>= 1) {
    const bool upper = (a & h) != 0;
    C w = tw[(a % h) * (N0 / (2 * h))];
    if (DIR > 0) w = cconj(w);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const C u = v[e];
      const C o = mkc(__shfl_xor_sync(0xffffffffu, u.x, h), __shfl_xor_sync(0xffffffffu, u.y, h));
      v[e] = upper ? cmul(csub(o, u), w) : cadd(u, o);
    }
  }
  const int src = ((threadIdx.x & 31) & ~(S - 1)) | bit_reverse<S>(a);
#pragma unroll
  for (int e = 0; e < 16; ++e)
    v[e] = mkc(__shfl_sync(0xffffffffu, v[e].x, src), __shfl_sync(0xffffffffu, v[e].y, src));
}

// forward transform over m of a column slice: on entry v[i] holds row
// j + 4 m(i, a); on return v[i] = Y[k1] at k1 = i + V a
template <int NL, typename C>
__device__ __forceinline__ void lane_fwd(C* v, int a, const C* tw) {
  constexpr int S = LaneSplit<NL>::SPL;
  if constexpr (S == 1) {
    Dft<NL, -1, C>::run(v);
  } else if constexpr (S == 2) {
    Dft<16, -1, C>::run(v);
    PairLoop<0, C>::fwd(v, a != 0);
  } else {
    Dft<16, -1, C>::run(v);
    // V_a[e] = w_NL^(a e) U_a[e], w_NL = w_n0^4
#pragma unroll
    for (int e = 1; e < 16; ++e) v[e] = cmul(v[e], tw[4 * a * e]);
    cross_lane_dft<S, -1>(v, a, tw);
  }
}

// inverse: v[i] = V[k1] at k1 = i + V a -> v[i] = x at row j + 4 m(i, a)
template <int NL, typename C>
__device__ __forceinline__ void lane_inv(C* v, int a, const C* tw) {
  constexpr int S = LaneSplit<NL>::SPL;
  if constexpr (S == 1) {
    Dft<NL, +1, C>::run(v);
  } else if constexpr (S == 2) {
    PairLoop<0, C>::inv(v, a != 0);
    Dft<16, +1, C>::run(v);
  } else {
    cross_lane_dft<S, +1>(v, a, tw);
#pragma unroll
    for (int e = 1; e < 16; ++e) v[e] = cmulc(v[e], tw[4 * a * e]);
    Dft<16, +1, C>::run(v);
  }
}

// tile geometry for n0 = 4 NL (3D: C = 6, a 6-column group is one
// coefficient; 2D: C = 3, two coefficients)
template <typename T, int DIM, int NL> struct R4Tile {
  static constexpr int C = DIM == 3 ? 6 : 3;
  static constexpr int LT = NL <= 64 ? 2 : 1;     // load cases per tile
  static constexpr int NG = NL <= 64 ? 128 / (LT * NL) : 1;  // 6-column groups per tile
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
  static constexpr int OSTEP = SPL == 1 ? 0 : (SPL >= LMOD ? 1 : LMOD / SPL);
  // load-case stride: past the last value, and LMOD/2 mod LMOD, so that the
  // two load cases of a phase-2 lane pair fall in disjoint banks
  static constexpr int LS0 = NL * P + SPL * OSTEP;
  static constexpr int LS = LS0 + ((LMOD / 2 - LS0 % LMOD) + LMOD) % LMOD;
  static constexpr size_t SMEM = (size_t)LT * LS * sizeof(cx<T>);
  // resident CTAs asked of the register allocator
  static constexpr int MINB = THREADS > 256 ? 1 : (sizeof(T) == 8 ? 2 : 3);
};

// offset of value k1 in a (load case, j, column) slice
template <typename K> __device__ __forceinline__ int k1_off(int k1) {
  return k1 * K::P + (k1 >> 4) * K::OSTEP;
}

template <typename T> struct Axis0Args {
  const cx<T>* in;
  cx<T>* out;
  const cx<T>* tw;   // exp(-2 pi i t / n0), t < n0
  int64_t inner;     // complex columns per row (F * C)
  int64_t pitch;     // complex elements between rows
  int64_t ncoef;     // F
  int64_t m_last;    // 3D: coefficient f = b1 * m_last + b2
  int L;
  int prefetch;      // rows 16-byte aligned: prefetch the next tile into L2
  GreenTables<T> gt;
  const T* tab;      // symmetric Mandel matrices [f][c][b0], or nullptr: on the fly
};

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
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

template <typename T, int DIM, int NL, bool TAB>
__global__ void __launch_bounds__(R4Tile<T, DIM, NL>::THREADS, R4Tile<T, DIM, NL>::MINB)
    green_axis0_r4_kernel(Axis0Args<T> a) {
  using C = cx<T>;
  using K = R4Tile<T, DIM, NL>;
  constexpr int N0 = 4 * NL;
  constexpr int NV = LaneSplit<NL>::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* S = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  // phase-1/3 lane: half a of a pair (pair split), column c, load case l1, j1
  const bool p1 = tid < K::P1;
  const int a1 = tid % K::SPL;
  const int s1 = tid / K::SPL;
  const int c = s1 % K::WC;
  const int l1 = (s1 / K::WC) % K::LT;
  const int j1 = s1 / (K::WC * K::LT);
  // phase-2 lane: load case l2 (fastest, so pairs share table loads), k1, group g2
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
    __syncthreads();  // the previous tile's phase 3 has read S
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

int g_sm_count = 0;

template <typename T, int DIM, int NL, bool TAB>
cudaError_t axis0_go(const Axis0Args<T>& a, cudaStream_t st) {
  using K = R4Tile<T, DIM, NL>;
  auto k = &green_axis0_r4_kernel<T, DIM, NL, TAB>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)K::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, K::THREADS, K::SMEM) !=
          cudaSuccess ||
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
  const int64_t tiles = (a.inner + K::WC - 1) / K::WC * ((a.L + K::LT - 1) / K::LT);
  const int64_t g = (int64_t)per_sm * g_sm_count;
  const int grid = (int)(tiles < g ? tiles : g);
  k<<<grid, K::THREADS, K::SMEM, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int DIM, bool TAB>
cudaError_t axis0_n(const Axis0Args<T>& a, int n0, cudaStream_t st) {
  switch (n0) {
    case 32: return axis0_go<T, DIM, 8, TAB>(a, st);
    case 64: return axis0_go<T, DIM, 16, TAB>(a, st);
    case 128: return axis0_go<T, DIM, 32, TAB>(a, st);
    case 256: return axis0_go<T, DIM, 64, TAB>(a, st);
    case 512: return axis0_go<T, DIM, 128, TAB>(a, st);
    default: return axis0_go<T, DIM, 256, TAB>(a, st);
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
