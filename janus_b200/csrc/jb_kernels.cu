// Pass kernels of the janus_b200 Lippmann-Schwinger path (sm_100a).
//
// A Green-operator application y = F^-1[Gamma-hat F[x]] on an n0 x n1 (x n2)
// grid of s-component Mandel fields is a sequence of shared-memory passes,
// each reading and writing every spectral value once:
//   2D: rows_r2c (axis 1) | cols mode 2 (axis 0: fwd, Gamma, inv) | rows_c2r
//   3D: rows_r2c (axis 2) | cols fwd (axis 1) | cols mode 2 (axis 0)
//       | cols inv (axis 1) | rows_c2r
// The local operator (C - C0):eps is fused into rows_r2c and the solver
// update eps = E - y/N with its FP64 residual partials into rows_c2r.
//
// Spectral layout in HBM: complex [L][n0][(n1)][m][s], m = n_last/2 + 1,
// Mandel component fastest (so one spectral coefficient's s components are
// one contiguous 48-byte (3D) / 24-byte (2D) group in FP64 complex).
#include <cudaTypedefs.h>

#include <type_traits>

#include <cstdlib>
#include <mutex>
#include <unordered_map>

#include "jb_async.cuh"
#include "jb_fft_ct.cuh"
#include "jb_green.cuh"
#include "jb_kernels.h"

namespace jb {

namespace {

constexpr int kThreads = 256;
constexpr size_t kSmemCap = 227 * 1024;
constexpr size_t kSmemBudget = 96 * 1024;
constexpr int kTabStage = 512;  // phase tables up to this size are staged in smem

template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T sub_rn(T a, T b);
template <> __device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// FourthRankIsotropicTensor2D/3D.c_apply (janus/operators.pyx:317-324,
// 354-365) with the reference's operation order and no contraction into
// FMA, so the result is bitwise that of the reference for the same inputs.
// In place: p[0..s-1] <- (tr J' + dev I) : p.
template <typename T>
__device__ __forceinline__ void iso_apply(T* p, T tr, T dev, int dim) {
  if (dim == 2) {
    const T x0 = p[0], x1 = p[1], x2 = p[2];
    const T aux = mul_rn(tr, add_rn(x0, x1));
    p[0] = add_rn(aux, mul_rn(dev, x0));
    p[1] = add_rn(aux, mul_rn(dev, x1));
    p[2] = mul_rn(dev, x2);
  } else {
    const T x0 = p[0], x1 = p[1], x2 = p[2];
    const T aux = mul_rn(tr, add_rn(add_rn(x0, x1), x2));
    p[0] = add_rn(aux, mul_rn(dev, x0));
    p[1] = add_rn(aux, mul_rn(dev, x1));
    p[2] = add_rn(aux, mul_rn(dev, x2));
    p[3] = mul_rn(dev, p[3]);
    p[4] = mul_rn(dev, p[4]);
    p[5] = mul_rn(dev, p[5]);
  }
}

// y = M x for one voxel, M row-major s x s: y_i = (((0 + m_i0 x_0) + m_i1 x_1)
// + ...) without FMA contraction, the order of LinearOperator.c_apply and of
// FourthRankCubicTensor2D.c_apply (janus/operators.pyx:209-214, 435-441)
template <typename T>
__device__ __forceinline__ void mat_apply(T* p, const T* m, int C) {
  T x[6];
  for (int c = 0; c < C; ++c) x[c] = p[c];
  for (int i = 0; i < C; ++i) {
    T y = mul_rn(m[i * C], x[0]);
    for (int j = 1; j < C; ++j) y = add_rn(y, mul_rn(m[i * C + j], x[j]));
    p[i] = y;
  }
}

// the local operator of entry ph: isotropic (tr, dev) or a full matrix
template <typename T>
__device__ __forceinline__ void local_apply(T* p, const T* tab, int ph, int kind, int dim) {
  const int C = dim == 2 ? 3 : 6;
  if (kind == 0)
    iso_apply<T>(p, tab[2 * ph], tab[2 * ph + 1], dim);
  else
    mat_apply<T>(p, tab + (size_t)ph * C * C, C);
}

// reals per table entry of a local operator
__host__ __device__ __forceinline__ int local_entry(int kind, int dim) {
  return kind == 0 ? 2 : (dim == 2 ? 9 : 36);
}

// phase id of voxel v: uint8 or int32 map; index_bytes 0 = one table entry
// per voxel (stiffness fields)
__device__ __forceinline__ int load_phase(const void* phase, int ib, int64_t v) {
  if (ib == 0) return static_cast<int>(v);
  return ib == 1 ? static_cast<int>(static_cast<const uint8_t*>(phase)[v])
                 : static_cast<const int32_t*>(phase)[v];
}

// deterministic block sum (fixed shuffle tree + fixed warp order)
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) s += red[w];
  }
  return s;
}

// threads of a tile kernel: those of its compile-time FFT tile, else kThreads
template <int NCT, int WCT> constexpr int tile_max_threads() {
  if constexpr (NCT > 0)
    return ct_threads<NCT, WCT>();
  else
    return kThreads;
}

// resident CTAs per SM asked of the register allocator for the row kernels'
// compile-time tiles of up to 192 threads (FP64: 4, at most 80 registers;
// FP32: 6), so that registers never bound their occupancy below shared memory
template <typename T, int NCT, int WCT> constexpr int rows_min_blocks() {
  if constexpr (NCT > 0) {
    if (ct_threads<NCT, WCT>() <= 192) return sizeof(T) == 8 ? 4 : 6;
  }
  return 1;
}

template <typename T> struct RowsArgs {
  const T* x;
  cx<T>* out;
  const cx<T>* cin;
  T* y;
  const cx<T>* tw;
  AxisPlan plan;
  RealGeom g;
  int R, W, m;
  int64_t sp;  // spectral row pitch in complex elements (m * C, or one more)
  int L;       // load cases (persistent kernels)
  int contig;  // real side rows are contiguous [rows][n][C]
  int64_t cstride_l;
  const void* phase;
  int index_bytes;
  const T* table;
  int nphase;  // table entries (staged in shared memory when <= kTabStage reals / 2)
  int kind;    // local operator entries: 0 (tr, dev), 1 s x s matrices
  int dim;
  const double* E;
  double* partials;
  const T* rhs;   // kEpiRhs: right-hand side field
  float* rout;    // kEpiResid: FP32 residual field
  T scale;
};

__device__ __forceinline__ int64_t geom_off(const RealGeom& g, int64_t row, int e, int c) {
  return (row / g.n1r) * g.s0 + (row % g.n1r) * g.s1 + e * g.es + c * g.cs;
}

template <typename P> __device__ __forceinline__ P* align16_ptr(void* p) {
  return reinterpret_cast<P*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
}

// two-element vectors for 16-byte (FP64) / 8-byte (FP32) shared-memory access
template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// padding (reals) after each row of a raw real chunk staged in shared memory
// by the compile-time row kernels: 32 bytes shift consecutive rows by 8
// banks, so a warp mapping (row fastest, voxel next) reads and writes the
// chunk and the FFT tile without bank conflicts.  A tile (n + 2) x W complex
// holds R rows of n*CC reals plus 2*CC reals of slack per row, so FP32 with
// CC = 3 takes 16 bytes.
template <typename T, int CC> constexpr int row_pad() {
  return (2 * CC * (int)sizeof(T) >= 32 ? 32 : 16) / (int)sizeof(T);
}

// the CC components of one voxel between shared memory and registers
// (vector accesses when CC is even)
template <typename T, int CC>
__device__ __forceinline__ void load_voxel(const T* __restrict__ src, T (&v)[CC]) {
  if constexpr (CC % 2 == 0) {
    using V = typename Vec2<T>::type;
#pragma unroll
    for (int j = 0; j < CC / 2; ++j) {
      const V w = reinterpret_cast<const V*>(src)[j];
      v[2 * j] = w.x;
      v[2 * j + 1] = w.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < CC; ++c) v[c] = src[c];
  }
}

template <typename T, int CC>
__device__ __forceinline__ void store_voxel(T* __restrict__ dst, const T (&v)[CC]) {
  if constexpr (CC % 2 == 0) {
    using V = typename Vec2<T>::type;
#pragma unroll
    for (int j = 0; j < CC / 2; ++j) {
      V w;
      w.x = v[2 * j];
      w.y = v[2 * j + 1];
      reinterpret_cast<V*>(dst)[j] = w;
    }
  } else {
#pragma unroll
    for (int c = 0; c < CC; ++c) dst[c] = v[c];
  }
}

// every thread waits (bounded) on the tile barrier; false if any timed out
__device__ __forceinline__ bool tile_wait(uint64_t* bar, int* fail_flag) {
  if (!mbar_wait(bar, 0)) atomicOr(fail_flag, 1);
  __syncthreads();
  return *fail_flag == 0;
}

// r2c along the contiguous axis of CC-component real rows, optionally with
// the local operator (C - C0):eps fused on the way in.
// Shared memory: twiddles | tile A | tile B, tiles (n+2) x W complex.
//  1. the R-row input chunk (contiguous) lands in B by bulk copies, with the
//     tile's phase ids (uint8 / int32 maps) and the twiddles on the same
//     barrier (per-thread loads of those at every CTA's start measured 6-9%
//     slower at 128^3 x 6);
//  2. B -> A transposes it so tile rows are the transform axis (real view:
//     row e holds the R*CC reals of voxel e of each row), applying the local
//     operator per voxel;
//  3. Stockham FFT of the W complex columns (real columns paired as re/im);
//  4. split into the two half spectra, staged as [rr][k][c] and written out
//     by one bulk copy.
template <typename T, int CC, bool LOCAL, int NCT = 0, int WCT = 0>
__global__ void __launch_bounds__(tile_max_threads<NCT, WCT>(), rows_min_blocks<T, NCT, WCT>())
    rows_r2c_kernel(RowsArgs<T> a) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int fail_flag;
  const int n = NCT > 0 ? NCT : a.plan.n;
  const int W = WCT > 0 ? WCT : a.W;
  const int R = WCT > 0 ? 2 * WCT / CC : a.R;
  const int m = n / 2 + 1;
  C* tw = reinterpret_cast<C*>(smem);
  C* A = align16_ptr<C>(tw + n);
  // spectral row pitch: six-component rows are never padded (m * 6 complex
  // is even), so theirs is a compile-time constant; + R complex in the
  // staging buffers when rows are padded (one element a row)
  const int64_t sp = CC == 6 ? (int64_t)(n / 2 + 1) * 6 : a.sp;
  const int padr = (CC != 6 && sp > (int64_t)(n / 2 + 1) * CC) ? R : 0;
  C* B = align16_ptr<C>(A + (size_t)(n + 2) * W + padr);
  T* Ar = reinterpret_cast<T*>(A);
  T* Br = reinterpret_cast<T*>(B);
  const int ldr = 2 * W;
  const int l = blockIdx.y;
  const int64_t row0 = (int64_t)blockIdx.x * R;
  const int rows_here = (int)min((int64_t)R, a.g.rows - row0);
  constexpr int kC = CC;
  const int RC = R * kC;
  // raw chunk rows in B, ldb reals apart (padded for the compile-time tiles)
  const int ldb = n * kC + (NCT > 0 ? row_pad<T, kC>() : 0);
  const T* xl = a.x + l * a.g.ls;
  const T* chunk = xl + row0 * n * kC;
  const uint32_t bytes = (uint32_t)(rows_here * n * kC * sizeof(T));
  const uint32_t rbytes = (uint32_t)(n * kC * sizeof(T));
  const bool bulk = a.contig && aligned16(chunk) && (rbytes % 16 == 0) && aligned16(Br);
  // phase ids (uint8 or int32 maps) and the twiddles travel with the rows
  int* phs = reinterpret_cast<int*>(B + (size_t)(n + 2) * W + padr);
  const int ib = LOCAL ? a.index_bytes : 0;
  const unsigned char* phsrc =
      ib > 0 ? static_cast<const unsigned char*>(a.phase) + row0 * n * ib : nullptr;
  const uint32_t phbytes = (uint32_t)(rows_here * n * ib);
  const bool bulk_ph =
      bulk && (ib == 1 || ib == 4) && aligned16(phsrc) && phbytes % 16 == 0;
  const bool ph8 = bulk_ph && ib == 1;
  const uint32_t twbytes = (uint32_t)(n * sizeof(C));
  const bool bulk_tw = bulk && aligned16(a.tw) && twbytes % 16 == 0;
  if (threadIdx.x == 0) {
    fail_flag = 0;
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (bulk) {
    if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&bar, bytes + (bulk_ph ? phbytes : 0u) + (bulk_tw ? twbytes : 0u));
      if (NCT > 0) {
        for (int rr = 0; rr < rows_here; ++rr)
          bulk_load(Br + (size_t)rr * ldb, chunk + (size_t)rr * n * kC, rbytes, &bar);
      } else {
        bulk_load(Br, chunk, bytes, &bar);
      }
      if (bulk_ph) bulk_load(phs, phsrc, phbytes, &bar);
      if (bulk_tw) bulk_load(tw, a.tw, twbytes, &bar);
    }
  } else {
    for (int rr = 0; rr < rows_here; ++rr)
      for (int e = threadIdx.x; e < n; e += blockDim.x)
#pragma unroll
        for (int c = 0; c < kC; ++c)
          Br[rr * ldb + e * kC + c] = xl[geom_off(a.g, row0 + rr, e, c)];
  }
  if (!bulk_tw)
    for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = a.tw[i];
  // local operator: the (tr, dev) table (and the phase ids when they could
  // not come by bulk copy) go to shared memory while the copies are in flight
  T* tabs = align16_ptr<T>(phs + (size_t)R * n);
  const T* tab = a.table;
  auto phase_at = [&](int i) {
    return ph8 ? (int)reinterpret_cast<const uint8_t*>(phs)[i] : phs[i];
  };
  if constexpr (LOCAL) {
    if (!bulk_ph)
      for (int i = threadIdx.x; i < rows_here * n; i += blockDim.x)
        phs[i] = load_phase(a.phase, a.index_bytes, row0 * n + i);
    const int tabn = a.nphase * local_entry(a.kind, a.dim);
    if (tabn <= 2 * kTabStage) {
      for (int i = threadIdx.x; i < tabn; i += blockDim.x) tabs[i] = a.table[i];
      tab = tabs;
    }
  }
  if (bulk) {
    if (!tile_wait(&bar, &fail_flag)) return;
  } else {
    __syncthreads();
  }
  if constexpr (NCT > 0) {
    // voxel v = (e, rr) with the row fastest (R a compile-time constant)
    for (int v = threadIdx.x; v < R * n; v += blockDim.x) {
      const int rr = v % R, e = v / R;
      T x[kC];
      if (rr < rows_here) {
        load_voxel<T, kC>(Br + rr * ldb + e * kC, x);
        if constexpr (LOCAL) local_apply<T>(x, tab, phase_at(rr * n + e), a.kind, kC == 3 ? 2 : 3);
      } else {
#pragma unroll
        for (int c = 0; c < kC; ++c) x[c] = T(0);
      }
      store_voxel<T, kC>(Ar + e * ldr + rr * kC, x);
    }
  } else {
    for (int rr = 0; rr < R; ++rr)
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        T v[kC];
        if (rr < rows_here) {
#pragma unroll
          for (int c = 0; c < kC; ++c) v[c] = Br[rr * ldb + e * kC + c];
          if constexpr (LOCAL) local_apply<T>(v, tab, phase_at(rr * n + e), a.kind, kC == 3 ? 2 : 3);
        } else {
#pragma unroll
          for (int c = 0; c < kC; ++c) v[c] = T(0);
        }
#pragma unroll
        for (int c = 0; c < kC; ++c) Ar[e * ldr + rr * kC + c] = v[c];
      }
  }
  if (ldr > RC)
    for (int e = threadIdx.x; e < n; e += blockDim.x)
      for (int j = RC; j < ldr; ++j) Ar[e * ldr + j] = T(0);
  __syncthreads();
  const Lane ln = make_lane(W);
  C* Z;
  if constexpr (NCT > 0)
    Z = fft_ct<NCT, WCT, -1>(A, B, tw);
  else
    Z = fft_tile<-1>(A, B, tw, a.plan, W, ln);
  C* S = (Z == A) ? B : A;
  {
    const int col = ln.col;
    const int ra = 2 * col, rb = 2 * col + 1;
    const int rra = ra / kC, ca = ra - rra * kC;
    const int rrb = rb / kC, cb = rb - rrb * kC;
    for (int k = ln.j0; k < m; k += ln.T) {
      const C P = Z[k * W + col];
      const C Q = cconj(Z[(k == 0 ? 0 : n - k) * W + col]);
      if (ra < RC && rra < rows_here)
        S[(int64_t)rra * sp + k * kC + ca] = mkc(T(0.5) * (P.x + Q.x), T(0.5) * (P.y + Q.y));
      if (rb < RC && rrb < rows_here)
        S[(int64_t)rrb * sp + k * kC + cb] = mkc(T(0.5) * (P.y - Q.y), T(-0.5) * (P.x - Q.x));
    }
  }
  fence_async_shared();
  __syncthreads();
  C* dst = a.out + l * a.cstride_l + row0 * sp;
  const uint32_t obytes = (uint32_t)(rows_here * sp * sizeof(C));
  if (aligned16(dst) && obytes % 16 == 0) {
    if (threadIdx.x == 0) {
      bulk_store(dst, S, obytes);
      bulk_commit();
      bulk_wait_read();
    }
  } else {
    const int cnt = (int)(rows_here * sp);
    for (int idx = threadIdx.x; idx < cnt; idx += blockDim.x) dst[idx] = S[idx];
  }
}

// c2r along the contiguous axis; the spectral chunk (and, for the solver
// epilogues, one real side field) arrive by bulk copies; the output chunk
// leaves by one bulk copy.  Epilogues (y = scale * c2r(spectrum)):
//   kEpiPlain : out = y
//   kEpiUpdate: eps <- E - y in place, partials += (new - old)^2
//   kEpiResid : r = (E - y) - eps written as FP32 to `rout` (eps unchanged),
//               partials += r^2 (the basic scheme's increment, FP64)
//   kEpiRhs   : d <- rhs - y in place (rhs a field of the same type)
enum { kEpiPlain = 0, kEpiUpdate = 1, kEpiResid = 2, kEpiRhs = 3 };

template <typename T, int CC, int EPI, int NCT = 0, int WCT = 0>
__global__ void __launch_bounds__(tile_max_threads<NCT, WCT>(), rows_min_blocks<T, NCT, WCT>())
    rows_c2r_kernel(RowsArgs<T> a) {
  using C = cx<T>;
  using OT = typename std::conditional<EPI == kEpiResid, float, T>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int fail_flag;
  __shared__ double red[tile_max_threads<NCT, WCT>() / 32];
  constexpr int kC = CC;
  constexpr bool kSide = EPI != kEpiPlain;
  const int n = NCT > 0 ? NCT : a.plan.n;
  const int W = WCT > 0 ? WCT : a.W;
  const int R = WCT > 0 ? 2 * WCT / CC : a.R;
  C* tw = reinterpret_cast<C*>(smem);
  C* A = align16_ptr<C>(tw + n);
  // spectral row pitch (compile-time for six components, see rows_r2c)
  const int64_t sp = CC == 6 ? (int64_t)(n / 2 + 1) * 6 : a.sp;
  const int padr = (CC != 6 && sp > (int64_t)(n / 2 + 1) * CC) ? R : 0;
  C* B = align16_ptr<C>(A + (size_t)(n + 2) * W + padr);
  T* Eo = align16_ptr<T>(B + (size_t)(n + 2) * W + padr);  // [R][n][CC] side-field staging
  const int ldr = 2 * W;
  const int l = blockIdx.y;
  const int64_t row0 = (int64_t)blockIdx.x * R;
  const int rows_here = (int)min((int64_t)R, a.g.rows - row0);
  const int RC = R * kC;
  const C* src = a.cin + l * a.cstride_l + row0 * sp;
  const uint32_t sbytes = (uint32_t)(rows_here * sp * sizeof(C));
  // side field: old eps (update, resid) or the right-hand side (rhs)
  const T* sidel = (EPI == kEpiRhs ? a.rhs : a.y) + l * a.g.ls;
  const T* sidechunk = sidel + row0 * n * kC;
  OT* outl = (EPI == kEpiResid ? reinterpret_cast<OT*>(a.rout) : reinterpret_cast<OT*>(a.y)) +
             l * a.g.ls;
  OT* outchunk = outl + row0 * n * kC;
  const uint32_t ebytes = (uint32_t)(rows_here * n * kC * sizeof(T));
  const uint32_t obytes = (uint32_t)(rows_here * n * kC * sizeof(OT));
  const uint32_t erow = (uint32_t)(n * kC * sizeof(T)), orow = (uint32_t)(n * kC * sizeof(OT));
  // side field and output staged [rr][e][c] with rows ldE / ldO reals apart
  // (padded for the compile-time tiles, one bulk copy per row)
  const int ldE = n * kC + (NCT > 0 ? row_pad<T, kC>() : 0);
  const int ldO = n * kC + (NCT > 0 ? row_pad<OT, kC>() : 0);
  const bool bulk_s = aligned16(src) && sbytes % 16 == 0;
  const bool bulk_e = kSide && a.contig && aligned16(sidechunk) && erow % 16 == 0;
  const bool bulk_o = a.contig && aligned16(outchunk) && orow % 16 == 0;
  if (threadIdx.x == 0) {
    fail_flag = 0;
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && (bulk_s || bulk_e)) {
    mbar_arrive_expect_tx(&bar, (bulk_s ? sbytes : 0u) + (bulk_e ? ebytes : 0u));
    if (bulk_s) bulk_load(B, src, sbytes, &bar);
    if (bulk_e) {
      if (NCT > 0) {
        for (int rr = 0; rr < rows_here; ++rr)
          bulk_load(Eo + (size_t)rr * ldE, sidechunk + (size_t)rr * n * kC, erow, &bar);
      } else {
        bulk_load(Eo, sidechunk, ebytes, &bar);
      }
    }
  }
  if (!bulk_s) {
    const int cnt = (int)(rows_here * sp);
    for (int idx = threadIdx.x; idx < cnt; idx += blockDim.x) B[idx] = src[idx];
  }
  if (kSide && !bulk_e) {
    for (int rr = 0; rr < rows_here; ++rr)
      for (int e = threadIdx.x; e < n; e += blockDim.x)
#pragma unroll
        for (int c = 0; c < kC; ++c)
          Eo[rr * ldE + e * kC + c] = sidel[geom_off(a.g, row0 + rr, e, c)];
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = a.tw[i];
  if (bulk_s || bulk_e) {
    if (!tile_wait(&bar, &fail_flag)) return;
  } else {
    __syncthreads();
  }
  const Lane ln = make_lane(W);
  {
    const int col = ln.col;
    const int ra = 2 * col, rb = 2 * col + 1;
    const int rra = ra / kC, ca = ra - rra * kC;
    const int rrb = rb / kC, cb = rb - rrb * kC;
    const bool va = ra < RC && rra < rows_here, vb = rb < RC && rrb < rows_here;
    for (int k = ln.j0; k < n; k += ln.T) {
      const bool mirror = 2 * k > n;
      const int kk = mirror ? n - k : k;
      C Av = mkc(T(0), T(0)), Bv = mkc(T(0), T(0));
      if (va) Av = B[(int64_t)rra * sp + kk * kC + ca];
      if (vb) Bv = B[(int64_t)rrb * sp + kk * kC + cb];
      if (kk == 0 || 2 * kk == n) {
        Av.y = T(0);
        Bv.y = T(0);
      }
      A[k * W + col] = mirror ? mkc(Av.x + Bv.y, Bv.x - Av.y) : mkc(Av.x - Bv.y, Av.y + Bv.x);
    }
  }
  __syncthreads();
  C* Z;
  if constexpr (NCT > 0)
    Z = fft_ct<NCT, WCT, +1>(A, B, tw);
  else
    Z = fft_tile<+1>(A, B, tw, a.plan, W, ln);
  const T* Zr = reinterpret_cast<const T*>(Z);
  // output staging [rr][e][c]: in place over the side field, or the free tile
  OT* O = (EPI == kEpiUpdate || EPI == kEpiRhs) ? reinterpret_cast<OT*>(Eo)
                                                : reinterpret_cast<OT*>(Z == A ? B : A);
  double acc = 0.0;
  T Ev[kC];
#pragma unroll
  for (int c = 0; c < kC; ++c)
    Ev[c] = (EPI == kEpiUpdate || EPI == kEpiResid) ? static_cast<T>(a.E[l * kC + c]) : T(0);
  // one voxel: y = tile values, side = staged side field -> output values
  auto epilogue = [&](const T (&y)[kC], const T (&side)[kC], OT (&out)[kC]) {
#pragma unroll
    for (int c = 0; c < kC; ++c) {
      if (EPI == kEpiUpdate) {
        const T nv = sub_rn(Ev[c], mul_rn(a.scale, y[c]));
        out[c] = nv;
        const double d = static_cast<double>(nv) - static_cast<double>(side[c]);
        acc += d * d;
      } else if (EPI == kEpiResid) {
        const T nv = sub_rn(Ev[c], mul_rn(a.scale, y[c]));
        const double d = static_cast<double>(nv) - static_cast<double>(side[c]);
        out[c] = static_cast<OT>(d);
        acc += d * d;
      } else if (EPI == kEpiRhs) {
        out[c] = static_cast<OT>(sub_rn(side[c], mul_rn(a.scale, y[c])));
      } else {
        out[c] = static_cast<OT>(mul_rn(a.scale, y[c]));
      }
    }
  };
  if constexpr (NCT > 0) {
    // voxel v = (e, rr) with the row fastest (R a compile-time constant)
    for (int v = threadIdx.x; v < R * n; v += blockDim.x) {
      const int rr = v % R, e = v / R;
      if (rr >= rows_here) continue;
      T y[kC], side[kC];
      OT out[kC];
      load_voxel<T, kC>(Zr + e * ldr + rr * kC, y);
      if constexpr (kSide) {
        load_voxel<T, kC>(Eo + rr * ldE + e * kC, side);
      } else {
#pragma unroll
        for (int c = 0; c < kC; ++c) side[c] = T(0);
      }
      epilogue(y, side, out);
      store_voxel<OT, kC>(O + rr * ldO + e * kC, out);
    }
  } else {
    for (int rr = 0; rr < rows_here; ++rr)
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        T y[kC], side[kC];
        OT out[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) {
          y[c] = Zr[e * ldr + rr * kC + c];
          side[c] = kSide ? Eo[rr * ldE + e * kC + c] : T(0);
        }
        epilogue(y, side, out);
#pragma unroll
        for (int c = 0; c < kC; ++c) O[rr * ldO + e * kC + c] = out[c];
      }
  }
  fence_async_shared();
  __syncthreads();
  if (bulk_o) {
    if (threadIdx.x == 0) {
      if (NCT > 0) {
        for (int rr = 0; rr < rows_here; ++rr)
          bulk_store(outchunk + (size_t)rr * n * kC, O + (size_t)rr * ldO, orow);
      } else {
        bulk_store(outchunk, O, obytes);
      }
      bulk_commit();
      bulk_wait_read();
    }
  } else {
    for (int rr = 0; rr < rows_here; ++rr)
      for (int e = threadIdx.x; e < n; e += blockDim.x)
#pragma unroll
        for (int c = 0; c < kC; ++c)
          outl[geom_off(a.g, row0 + rr, e, c)] = O[rr * ldO + e * kC + c];
  }
  if (EPI == kEpiUpdate || EPI == kEpiResid) {
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) a.partials[(int64_t)l * gridDim.x + blockIdx.x] = s;
  }
}

template <typename T> struct ColsArgs {
  const cx<T>* in;
  cx<T>* out;
  const cx<T>* tw;
  AxisPlan plan;
  int64_t inner;  // columns transformed
  int64_t pitch;  // complex elements between consecutive rows (>= inner)
  int64_t outer;
  int W, C;
  int64_t m_last;
  GreenTables<T> gt;
  const T* mn;  // MODE 2: operator table (symmetric Mandel matrices), or nullptr: on the fly
  int nbuf;     // tensor-TMA kernel: rotating input tiles (2 or 3)
};

// complex transform along a strided axis of [outer][n][inner]: a tile of n
// rows x W consecutive columns, loaded and stored by one bulk copy per row
// (issued by warp 0).  MODE 0/1: forward/inverse; MODE 2: forward, Green
// contraction of each spectral coefficient (axis 0 index = tile row), inverse.
template <typename T, int MODE, int DIM>
__global__ void __launch_bounds__(kThreads) cols_kernel(ColsArgs<T> a) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int fail_flag;
  const int n = a.plan.n, W = a.W;
  C* tw = reinterpret_cast<C*>(smem);
  C* A = align16_ptr<C>(tw + n);
  C* B = align16_ptr<C>(A + (size_t)n * W);
  const int64_t c0 = (int64_t)blockIdx.x * W;
  const int Wc = (int)min((int64_t)W, a.inner - c0);
  const int64_t o = blockIdx.y;
  const C* src = a.in + o * n * a.pitch + c0;
  C* dst = a.out + o * n * a.pitch + c0;
  const uint32_t rowbytes = (uint32_t)(Wc * sizeof(C));
  const bool bulk = aligned16(src) && aligned16(dst) && ((a.pitch * sizeof(C)) % 16 == 0) &&
                    (rowbytes % 16 == 0) && ((W * sizeof(C)) % 16 == 0);
  if (threadIdx.x == 0) {
    fail_flag = 0;
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (bulk) {
    if (threadIdx.x < 32) {
      if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, rowbytes * (uint32_t)n);
      __syncwarp();
      for (int e = threadIdx.x; e < n; e += 32)
        bulk_load(A + (size_t)e * W, src + (int64_t)e * a.pitch, rowbytes, &bar);
    }
    if (Wc < W)
      for (int idx = threadIdx.x; idx < n * (W - Wc); idx += blockDim.x) {
        const int e = idx / (W - Wc);
        A[e * W + Wc + (idx - e * (W - Wc))] = mkc(T(0), T(0));
      }
  } else {
    for (int idx = threadIdx.x; idx < n * W; idx += blockDim.x) {
      const int e = idx / W;
      const int col = idx - e * W;
      A[idx] = col < Wc ? src[(int64_t)e * a.pitch + col] : mkc(T(0), T(0));
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = a.tw[i];
  if (bulk) {
    if (!tile_wait(&bar, &fail_flag)) return;
  } else {
    __syncthreads();
  }
  const Lane ln = make_lane(W);
  C* Z;
  if (MODE == 1)
    Z = fft_tile<+1>(A, B, tw, a.plan, W, ln);
  else
    Z = fft_tile<-1>(A, B, tw, a.plan, W, ln);
  if (MODE == 2) {
    const int Cc = a.C;
    const int Wf = W / Cc;
    const int nthr = (blockDim.x / Wf) * Wf;
    if ((int)threadIdx.x < nthr) {
      const int fl = threadIdx.x % Wf;
      const int e0 = threadIdx.x / Wf;
      const int est = nthr / Wf;
      const int col0 = fl * Cc;
      if (col0 < Wc) {
        const int64_t f = (c0 + col0) / Cc;
        int b[3];
        if (DIM == 3) {
          b[1] = (int)(f / a.m_last);
          b[2] = (int)(f % a.m_last);
        } else {
          b[1] = (int)f;
          b[2] = 0;
        }
        for (int e = e0; e < n; e += est) {
          b[0] = e;
          green_contract<DIM, T>(a.gt, b, Z + e * W + col0);
        }
      }
    }
    __syncthreads();
    C* other = (Z == A) ? B : A;
    Z = fft_tile<+1>(Z, other, tw, a.plan, W, ln);
  }
  if (bulk) {
    fence_async_shared();
    __syncthreads();
    if (threadIdx.x < 32) {
      for (int e = threadIdx.x; e < n; e += 32)
        bulk_store(dst + (int64_t)e * a.pitch, Z + (size_t)e * W, rowbytes);
      bulk_commit();
      bulk_wait_read();
    }
  } else {
    for (int idx = threadIdx.x; idx < n * W; idx += blockDim.x) {
      const int e = idx / W;
      const int col = idx - e * W;
      if (col < Wc) dst[(int64_t)e * a.pitch + col] = Z[idx];
    }
  }
}

// ===========================================================================
// Persistent, software-pipelined forms of the three pass kernels.
//
// A grid of (SM count x resident CTAs) walks the tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ...  Each CTA keeps two input buffers: while it
// computes tile i, the bulk load of tile i+1 is in flight into the other
// buffer and the bulk store of tile i-1 drains, so HBM traffic overlaps the
// shared-memory FFT.  Before a buffer is reloaded the storing thread(s) wait
// until their earlier bulk stores have finished reading shared memory.
// These kernels are used when every tile satisfies the bulk-copy alignment
// rules (checked on the host); otherwise the one-tile-per-CTA kernels above
// run.
// ===========================================================================

template <typename P> __device__ __forceinline__ P* align128_ptr(void* p) {
  return reinterpret_cast<P*>((reinterpret_cast<uintptr_t>(p) + 127) & ~uintptr_t(127));
}

// Column pass with tensor TMA: the tile (n rows x W complex columns of
// [outer][n][inner]) is one 3D box of the tensor map (split into boxes of at
// most 256 rows), loaded into one of two input buffers while the previous
// tile is computed, and stored back as boxes from shared memory.  Columns
// past `inner` in the last chunk are zero-filled by the load and skipped by
// the store.  Persistent grid; thread 0 issues all copies.
// resident CTAs per SM the Green pass asks the register allocator for
// (register pressure, not shared memory, bounded its occupancy)
template <typename T, int MODE, int NCT> constexpr int cols_min_blocks() {
  return (MODE == 2 && NCT > 0) ? (sizeof(T) == 8 ? 2 : 4) : 1;
}

template <typename T, int MODE, int DIM, int NCT, int WCT, bool INPL>
__device__ __forceinline__ void cols_tma_body(const CUtensorMap& tin, const CUtensorMap& tout,
                                              const ColsArgs<T>& a, int nbox) {
  using C = cx<T>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[3];
  __shared__ int fail_flag;
  const int n = NCT > 0 ? NCT : a.plan.n;
  const int W = WCT > 0 ? WCT : a.W;
  const int nbuf = a.nbuf;
  const size_t tile = (size_t)n * W;
  C* tw = reinterpret_cast<C*>(smem);
  // input tiles rotate so that the tile a load overwrites was stored an
  // iteration earlier with three of them: its store has drained by then
  C* const In0 = align128_ptr<C>(tw + n);
  const size_t tstride = (tile * sizeof(C) + 127) / 128 * 128;  // bytes between input tiles
  auto in_tile = [&](int b) {
    return reinterpret_cast<C*>(reinterpret_cast<unsigned char*>(In0) + b * tstride);
  };
  // ping-pong partner of the transforms (none when they run in place)
  C* Wk = INPL ? nullptr : in_tile(nbuf);
  AxisK<T>* ax0 = align128_ptr<AxisK<T>>(INPL ? in_tile(nbuf) : Wk + tile);  // MODE 2: axis-0 values
  const int64_t ntx = (a.inner + W - 1) / W;
  const int64_t total = ntx * a.outer;
  if (threadIdx.x == 0) {
    fail_flag = 0;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    fence_mbar_init();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = a.tw[i];
  if (MODE == 2 && a.mn == nullptr)
    for (int i = threadIdx.x; i < n; i += blockDim.x) ax0[i] = axis_values(a.gt, 0, i);
  __syncthreads();
  // tile t -> (o, chunk); the Green pass walks the load cases of a chunk
  // consecutively so they share its table slice in L2
  auto tile_of = [&](int64_t t, int64_t& o, int64_t& chunk) {
    if (MODE == 2) {
      chunk = t / a.outer;
      o = t - chunk * a.outer;
    } else {
      o = t / ntx;
      chunk = t - o * ntx;
    }
  };
  auto issue_load = [&](int64_t t, C* dst, uint64_t* b) {
    int64_t o, chunk;
    tile_of(t, o, chunk);
    const int x = (int)(2 * chunk * W);
    mbar_arrive_expect_tx(b, (uint32_t)(tile * sizeof(C)));
    for (int yb = 0; yb < n; yb += nbox) tma_load_3d(dst + (size_t)yb * W, &tin, x, yb, (int)o, b);
  };
  int64_t t = blockIdx.x;
  if (t < total && threadIdx.x == 0) issue_load(t, In0, &bar[0]);
  const Lane ln = make_lane(W);
  bool stored_wk = false;  // the last store read the partner tile Wk
  for (int i = 0, buf = 0, use = 0; t < total; ++i, t += gridDim.x) {
    int64_t o, chunk;
    tile_of(t, o, chunk);
    const int64_t c0 = chunk * W;
    const int Wc = (int)min((int64_t)W, a.inner - c0);
    C* in = in_tile(buf);
    if (!mbar_wait(&bar[buf], use & 1)) atomicOr(&fail_flag, 1);
    // the store that read the next buffer: the previous tile's with two
    // buffers, the one before it with three (at most one group pending);
    // all of them when the last store read Wk, which this tile rewrites
    if (threadIdx.x == 0) {
      if (nbuf > 2 && !stored_wk)
        bulk_wait_read_1();
      else
        bulk_wait_read();
    }
    __syncthreads();
    if (fail_flag) return;
    const int64_t tn = t + gridDim.x;
    const int nb = buf + 1 == nbuf ? 0 : buf + 1;
    if (threadIdx.x == 0 && tn < total) issue_load(tn, in_tile(nb), &bar[nb]);
    use += nb == 0;
    buf = nb;
    if (MODE == 2 && a.mn != nullptr) {
      // the tile's table slice ([f][c][e], consecutive coefficients
      // adjacent) heads for L1 while the forward transform runs
      constexpr int NT = GSize<DIM>::value;
      const int nf = (Wc + a.C - 1) / a.C;
      const char* base = reinterpret_cast<const char*>(a.mn + (size_t)(c0 / a.C) * n * NT);
      const int lines = (int)(((size_t)nf * n * NT * sizeof(T) + 127) / 128);
      for (int q = threadIdx.x; q < lines; q += blockDim.x) prefetch_l1(base + (size_t)q * 128);
    }
    C* Z;
    if constexpr (INPL) {
      if (MODE == 1)
        fft_ct_inplace<NCT, WCT, +1>(in, tw);
      else
        fft_ct_inplace<NCT, WCT, -1>(in, tw);
      Z = in;
    } else if constexpr (NCT > 0) {
      if (MODE == 1)
        Z = fft_ct<NCT, WCT, +1>(in, Wk, tw);
      else
        Z = fft_ct<NCT, WCT, -1>(in, Wk, tw);
    } else {
      if (MODE == 1)
        Z = fft_tile<+1>(in, Wk, tw, a.plan, W, ln);
      else
        Z = fft_tile<-1>(in, Wk, tw, a.plan, W, ln);
    }
    if (MODE == 2) {
      const int Cc = a.C;
      const int Wf = W / Cc;
      const int nthr = (blockDim.x / Wf) * Wf;
      if ((int)threadIdx.x < nthr) {
        const int fl = threadIdx.x % Wf;
        const int e0 = threadIdx.x / Wf;
        const int est = nthr / Wf;
        const int col0 = fl * Cc;
        if (col0 < Wc) {
          const int64_t f = (c0 + col0) / Cc;
          int b1, b2;
          if (DIM == 3) {
            b1 = (int)(f / a.m_last);
            b2 = (int)(f % a.m_last);
          } else {
            b1 = (int)f;
            b2 = 0;
          }
          if (a.mn != nullptr) {
            constexpr int NT = GSize<DIM>::value;
            const T* tab = a.mn + (size_t)f * n * NT;
            for (int e = e0; e < n; e += est) {
              T g[NT];
#pragma unroll
              for (int c = 0; c < NT; ++c) g[c] = __ldg(tab + (size_t)c * n + e);
              g_apply<DIM, T>(g, Z + e * W + col0);
            }
          } else {
            const AxisK<T> a1 = axis_values(a.gt, 1, b1);
            const AxisK<T> a2 = DIM == 3 ? axis_values(a.gt, 2, b2) : a1;
            for (int e = e0; e < n; e += est)
              green_contract_k<DIM, T>(a.gt.variant, ax0[e], a1, a2, a.gt.inv2g, a.gt.c1,
                                       Z + e * W + col0);
          }
        }
      }
      __syncthreads();
      C* other = (Z == in) ? Wk : in;
      if constexpr (INPL)
        fft_ct_inplace<NCT, WCT, +1>(Z, tw);
      else if constexpr (NCT > 0)
        Z = fft_ct<NCT, WCT, +1>(Z, other, tw);
      else
        Z = fft_tile<+1>(Z, other, tw, a.plan, W, ln);
    }
    fence_async_shared();
    __syncthreads();
    stored_wk = !INPL && Z == Wk;
    if (threadIdx.x == 0) {
      const int x = (int)(2 * c0);
      for (int yb = 0; yb < n; yb += nbox) tma_store_3d(&tout, x, yb, (int)o, Z + (size_t)yb * W);
      bulk_commit();
    }
  }
  if (threadIdx.x == 0) bulk_wait_read();
}

template <typename T, int MODE, int DIM, int NCT = 0, int WCT = 0>
__global__ void __launch_bounds__(tile_max_threads<NCT, WCT>(), cols_min_blocks<T, MODE, NCT>())
    cols_tma_kernel(const __grid_constant__ CUtensorMap tin,
                    const __grid_constant__ CUtensorMap tout, ColsArgs<T> a, int nbox) {
  cols_tma_body<T, MODE, DIM, NCT, WCT, false>(tin, tout, a, nbox);
}

// Green tiles transformed in place (no partner tile): twice the columns in
// the same shared memory, every thread busy in the largest-radix stage
template <typename T, int DIM, int NCT, int WCT>
__global__ void __launch_bounds__(ct_threads_inplace<NCT, WCT>(), cols_min_blocks<T, 2, NCT>())
    cols_tma_inplace_kernel(const __grid_constant__ CUtensorMap tin,
                            const __grid_constant__ CUtensorMap tout, ColsArgs<T> a, int nbox) {
  cols_tma_body<T, 2, DIM, NCT, WCT, true>(tin, tout, a, nbox);
}

// y[l][v] = local(v) : x[l][v]; load case l = blockIdx.y; a voxel's CC
// components move as two-element vectors when CC is even
template <typename T, int CC>
__global__ void local_kernel(LocalDesc loc, const T* table, int64_t nvox, const T* x, T* y) {
  const int64_t off = (int64_t)blockIdx.y * nvox * CC;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int ph = load_phase(loc.phase, loc.index_bytes, v);
    T p[CC];
    load_voxel<T, CC>(x + off + v * CC, p);
    local_apply<T>(p, table, ph, loc.kind, loc.dim);
    store_voxel<T, CC>(y + off + v * CC, p);
  }
}

template <typename T>
__global__ void local_sum_kernel(LocalDesc loc, const T* table, int C, int64_t nvox,
                                 const T* eps, double* partials) {
  __shared__ double red[kThreads / 32];
  const int l = blockIdx.y;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const T* el = eps + (int64_t)l * nvox * C;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int ph = load_phase(loc.phase, loc.index_bytes, v);
    T p[6];
    for (int c = 0; c < C; ++c) p[c] = el[v * C + c];
    local_apply<T>(p, table, ph, loc.kind, loc.dim);
    for (int c = 0; c < C; ++c) acc[c] += static_cast<double>(p[c]);
  }
  for (int c = 0; c < C; ++c) {
    const double s = block_sum(acc[c], red);
    if (threadIdx.x == 0) partials[((int64_t)l * C + c) * gridDim.x + blockIdx.x] = s;
  }
}

// out[v] = scale * sum_j (tr z_j tr e_j / dim, z_j . e_j - tr z_j tr e_j / dim):
// the isotropic-projector contractions of strain and adjoint strain
template <typename T>
__global__ void local_gradient_kernel(int dim, int64_t nvox, int L, const T* __restrict__ eps,
                                      const T* __restrict__ zeta, double scale,
                                      double* __restrict__ out) {
  const int C = dim == 2 ? 3 : 6;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    double sj = 0.0, sk = 0.0;
    for (int l = 0; l < L; ++l) {
      const T* e = eps + ((int64_t)l * nvox + v) * C;
      const T* z = zeta + ((int64_t)l * nvox + v) * C;
      double tre = 0.0, trz = 0.0, dot = 0.0;
      for (int c = 0; c < C; ++c) {
        const double ec = static_cast<double>(e[c]), zc = static_cast<double>(z[c]);
        dot += zc * ec;
        if (c < dim) {
          tre += ec;
          trz += zc;
        }
      }
      const double j = tre * trz / dim;
      sj += j;
      sk += dot - j;
    }
    out[2 * v] = scale * sj;
    out[2 * v + 1] = scale * sk;
  }
}

template <typename T>
__global__ void block_linear_kernel(int64_t nvox, int L, int osz, int isz, const T* a,
                                    const T* x, T* y, int transpose) {
  const int64_t total = (int64_t)L * nvox;
  const int ni = transpose ? osz : isz;  // length of x per voxel
  const int no = transpose ? isz : osz;  // length of y per voxel
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = i % nvox;
    const T* av = a + v * osz * isz;
    const T* xv = x + i * ni;
    T xl[8];
    for (int j = 0; j < ni; ++j) xl[j] = xv[j];
    T* yv = y + i * no;
    for (int r = 0; r < no; ++r) {
      T s = T(0);
      for (int j = 0; j < ni; ++j)
        s = add_rn(s, mul_rn(transpose ? av[j * isz + r] : av[r * isz + j], xl[j]));
      yv[r] = s;
    }
  }
}

template <typename T, int DIM>
__global__ void green_by_freq_kernel(GreenTables<T> gt, int64_t count, const int* b,
                                     const cx<T>* tau, cx<T>* eta) {
  constexpr int S = DIM == 2 ? 3 : 6;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    cx<T> t[S];
    for (int c = 0; c < S; ++c) t[c] = tau[i * S + c];
    int bb[3] = {b[i * DIM], b[i * DIM + 1], DIM == 3 ? b[i * DIM + 2] : 0};
    green_contract<DIM, T>(gt, bb, t);
    for (int c = 0; c < S; ++c) eta[i * S + c] = t[c];
  }
}

__global__ void axpy_f64_kernel(int64_t n, const double* __restrict__ d,
                                double* __restrict__ y) {
  const int64_t n2 = n / 2;
  const double2* d2 = reinterpret_cast<const double2*>(d);
  double2* y2 = reinterpret_cast<double2*>(y);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = d2[i];
    double2 a = y2[i];
    a.x += v.x;
    a.y += v.y;
    y2[i] = a;
  }
  for (int64_t i = 2 * n2 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] += d[i];
}

__global__ void axpy_f32_to_f64_kernel(int64_t n, const float* __restrict__ d,
                                       double* __restrict__ y) {
  const int64_t n4 = n / 4;
  const float4* d4 = reinterpret_cast<const float4*>(d);
  double2* y2 = reinterpret_cast<double2*>(y);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 v = d4[i];
    double2 a = y2[2 * i], b = y2[2 * i + 1];
    a.x += v.x;
    a.y += v.y;
    b.x += v.z;
    b.y += v.w;
    y2[2 * i] = a;
    y2[2 * i + 1] = b;
  }
  for (int64_t i = 4 * n4 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] += d[i];
}


template <typename T, int DIM>
__global__ void green_table_kernel(GreenTables<T> gt, int64_t n0, int64_t n1, int64_t m_last,
                                   T* out) {
  constexpr int NM = MnSize<DIM>::value;
  constexpr int NT = GSize<DIM>::value;
  const int64_t f12n = DIM == 3 ? n1 * m_last : m_last;
  const int64_t total = f12n * n0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = i / n0;
    const int b0 = (int)(i - f * n0);
    int b1, b2 = 0;
    if (DIM == 3) {
      b1 = (int)(f / m_last);
      b2 = (int)(f - (int64_t)b1 * m_last);
    } else {
      b1 = (int)f;
    }
    const AxisK<T> a0 = axis_values(gt, 0, b0);
    const AxisK<T> a1 = axis_values(gt, 1, b1);
    const AxisK<T> a2 = DIM == 3 ? axis_values(gt, 2, b2) : a1;
    T mn[NM], g[NT];
    mn_build<DIM, T>(gt.variant, a0.v, a1.v, a2.v, gt.inv2g, gt.c1, mn);
    mn_to_g<DIM, T>(mn, g);
#pragma unroll
    for (int c = 0; c < NT; ++c) out[(f * NT + c) * n0 + b0] = g[c];
  }
}

template <typename T>
__global__ void fill_macro_kernel(int C, int L, int64_t nvox, const double* E, T* eps) {
  const int64_t total = (int64_t)L * nvox * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int l = (int)(i / (nvox * C));
    eps[i] = static_cast<T>(E[l * C + c]);
  }
}

__global__ void reduce_rows_kernel(const double* partials, int nb, double* out, double factor,
                                   const double* factors, int take_sqrt) {
  __shared__ double red[kThreads / 32];
  const int l = blockIdx.x;
  double acc = 0.0;
  // fixed assignment of partials to threads, fixed tree: deterministic
  for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += partials[(int64_t)l * nb + i];
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) {
    const double f = factors ? factor * factors[l] : factor;
    out[l] = take_sqrt ? sqrt(s) * f : s * f;
  }
}

// long contiguous rows (n = 384, 512, 768, 1024) of 2D fields
#include "jb_rows_long.cuh"

std::mutex g_attr_mu;
std::unordered_map<const void*, size_t> g_attr;

// Opt the kernel in to `bytes` of dynamic shared memory (static + dynamic
// must stay within the 227 KB per-block limit).
cudaError_t ensure_smem(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  auto it = g_attr.find(fn);
  if (it != g_attr.end() && it->second >= bytes) return cudaSuccess;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  const size_t cap = kSmemCap - fa.sharedSizeBytes;
  if (bytes > cap) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
  if (e != cudaSuccess) {
    cudaGetLastError();  // do not leave the failure behind for later launches
    return e;
  }
  g_attr[fn] = cap;
  return cudaSuccess;
}

int grid_for(int64_t total) {
  int64_t g = (total + kThreads - 1) / kThreads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

// threads per block for a W-column tile: the largest power-of-two number of
// lanes per column T with T * W <= kThreads
int tile_threads(int W) {
  int t = 1;
  while (2 * t * W <= kThreads) t *= 2;
  return (t * W + 31) / 32 * 32;  // whole warps (block reductions use full-warp shuffles)
}

// rows per CTA, tile width and shared memory of the contiguous-axis kernels
// (tiles of (n+2) x W complex, W = ceil(R*C/2); `extra` = the old-strain
// staging of the update variant)
// shared memory of a row kernel: twiddles, two tiles, the side-field rows
// (solver epilogues; up to 32 bytes of padding between rows) and, with the
// local operator, the tile's phase ids and the staged phase table.  This is
// the kernels' exact layout (each region aligned to 16 bytes): three CTAs
// per SM of the FP64 c2r update kernel at n = 128 fit with 96 bytes to spare.
size_t rows_smem(int dtype, int n, int C, int r, int w, bool update, bool local, int nphase,
                 int entry = 2, bool padded = false) {
  const size_t cs = dtype == F64 ? 16 : 8;
  // staged table reals (2 * kTabStage at most)
  const size_t treal = (size_t)nphase * entry;
  const size_t staged = treal <= 2 * (size_t)kTabStage ? treal : 0;
  auto a16 = [](size_t v) { return (v + 15) / 16 * 16; };
  // twiddles | A | B; A and B hold (n + 2) w complex, plus r for the padding
  // of r spectral rows when the rows are padded
  const size_t pr = padded ? (size_t)r : 0;
  size_t off = a16(n * cs) + ((size_t)(n + 2) * w + pr) * cs;
  off = a16(off) + ((size_t)(n + 2) * w + pr) * cs;
  if (update) off = a16(off) + (size_t)r * n * C * (cs / 2) + (size_t)(r - 1) * 32;
  if (local) off = a16(off + (size_t)r * n * 4) + staged * (cs / 2);
  return off;
}

bool rows_shape(int dtype, int n, int C, bool update, int* R, int* W, size_t* smem,
                bool local = false, int nphase = 0, int entry = 2, bool padded = false) {
  const size_t cs = dtype == F64 ? 16 : 8;
  int r = (24 + C - 1) / C;
  for (;;) {
    const int w = (r * C + 1) / 2;
    const size_t bytes = rows_smem(dtype, n, C, r, w, update, local, nphase, entry, padded);
    if (bytes <= kSmemBudget || r == 1) {
      if (bytes > kSmemCap - 4096) return false;
      *R = r;
      *W = w;
      *smem = bytes;
      return true;
    }
    --r;
  }
}

bool cols_shape(int dtype, int n, int unit, int* W, size_t* smem) {
  const size_t cs = dtype == F64 ? 16 : 8;
  int w = unit == 1 ? 16 : unit * (12 / unit > 0 ? 12 / unit : 1);
  if (w < unit) w = unit;
  for (;;) {
    const size_t bytes = n * cs + 2 * (size_t)n * w * cs + 32;  // + alignment
    if (bytes <= kSmemBudget || w == unit) {
      if (bytes > kSmemCap - 4096) return false;
      *W = w;
      *smem = bytes;
      return true;
    }
    w -= unit;
  }
}

bool contiguous_rows(const RealGeom& g, int n, int C) {
  if (g.cs != 1 || g.es != C) return false;
  if (g.n1r == 1) return g.s0 == (int64_t)n * C;
  return g.s1 == (int64_t)n * C && g.s0 == g.n1r * n * C;
}

constexpr size_t kPipeBudget = 113 * 1024;  // two persistent CTAs per SM

int sm_count() {
  static int count = 0;
  if (count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        count <= 0)
      count = 148;
  }
  return count;
}

template <typename K>
int persistent_grid(K kernel, int threads, size_t smem, int64_t tiles) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int64_t g = (int64_t)per_sm * sm_count();
  return (int)(tiles < g ? tiles : g);
}

// tile width and shared memory of the tensor-TMA column kernel: two input
// tiles and one compute partner of n x W complex, 128-byte aligned
bool cols_tma_shape(int dtype, int n, int unit, int* W, size_t* smem, int* nbuf,
                    bool stage_ax0, const ColsTuning* tune, bool inplace = false) {
  const size_t cs = dtype == F64 ? 16 : 8;
  // built-in rule, measured on B200 (128^3 x 6, FP64): W = 8 columns for
  // plain passes, 12 (two 6-component coefficients) for the Green pass
  int w = unit == 1 ? 8 : unit * (12 / unit > 0 ? 12 / unit : 1);
  if (tune && tune->w >= unit && tune->w % unit == 0 && tune->w <= 128) w = tune->w;
  if (w < unit) w = unit;
  // + the axis-0 Green values (4 reals per row, unless tabulated) and alignment
  // input tiles, plus the transforms' partner tile unless they run in place
  auto bytes_for = [&](int ww, int nb) {
    const int nt = inplace ? nb : nb + 1;
    return n * cs + nt * 128 + nt * (size_t)n * ww * cs +
           (stage_ax0 ? (size_t)n * 2 * cs + 128 : 0);
  };
  // a TMA box row must span a multiple of 16 bytes: widths that do not
  // (odd multiples of 3 columns in FP32 2D) are skipped
  for (;; w -= unit) {
    // a third input tile for FP32, where two CTAs per SM still fit (measured
    // on B200, 128^3 x 6: FP32 plain passes 8% faster with three; FP64
    // slower, the third tile costing a resident CTA)
    int nb = dtype == F32 ? 3 : 2;
    if (tune && (tune->nbuf == 2 || tune->nbuf == 3)) nb = tune->nbuf;
    if (bytes_for(w, nb) > kPipeBudget) nb = 2;
    const size_t bytes = bytes_for(w, nb);
    const bool aligned = (w * cs) % 16 == 0;
    if (aligned && (bytes <= kPipeBudget || w <= unit)) {
      if (bytes > kSmemCap - 4096) return false;
      *W = w;
      *smem = bytes;
      *nbuf = nb;
      return true;
    }
    if (w <= unit) break;
  }
  // no aligned width fits the two-CTA budget (long axes): the narrowest
  // aligned width, one CTA per SM
  for (w = unit; w <= 128; w += unit) {
    if ((w * cs) % 16 != 0) continue;
    const size_t bytes = bytes_for(w, 2);
    if (bytes > kSmemCap - 4096) return false;
    *W = w;
    *smem = bytes;
    *nbuf = 2;
    return true;
  }
  return false;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

// 3D map of a complex [outer][n][inner] array seen as reals [outer][n][2 inner],
// box = 2W reals x nbox rows x 1
bool make_cols_map(CUtensorMap* m, const void* base, bool f64, int64_t inner, int64_t pitch,
                   int n, int64_t outer, int W, int nbox) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t rs = f64 ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)(2 * inner), (cuuint64_t)n, (cuuint64_t)outer};
  cuuint64_t strides[2] = {(cuuint64_t)(2 * pitch) * rs, (cuuint64_t)(2 * pitch) * rs * n};
  cuuint32_t box[3] = {(cuuint32_t)(2 * W), (cuuint32_t)nbox, 1};
  cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = enc(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         3, const_cast<void*>(base), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename T, int CC, bool LOCAL>
cudaError_t r2c_go(const RowsArgs<T>& a, dim3 grid, int threads, size_t smem, cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(&rows_r2c_kernel<T, CC, LOCAL>);
  cudaError_t e = ensure_smem(fn, smem);
  if (e != cudaSuccess) return e;
  rows_r2c_kernel<T, CC, LOCAL><<<grid, threads, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int CC, int EPI>
cudaError_t c2r_go(const RowsArgs<T>& a, dim3 grid, int threads, size_t smem, cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(&rows_c2r_kernel<T, CC, EPI>);
  cudaError_t e = ensure_smem(fn, smem);
  if (e != cudaSuccess) return e;
  rows_c2r_kernel<T, CC, EPI><<<grid, threads, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int EPI>
cudaError_t c2r_go_c(int C, const RowsArgs<T>& a, dim3 grid, int threads, size_t smem,
                     cudaStream_t st) {
  if (C == 3) return c2r_go<T, 3, EPI>(a, grid, threads, smem, st);
  if (C == 6) return c2r_go<T, 6, EPI>(a, grid, threads, smem, st);
  return cudaErrorInvalidValue;
}

template <typename T, int CC, bool LOCAL, int N, int W>
cudaError_t r2c_ct_go(const RowsArgs<T>& a, dim3 grid, size_t smem, cudaStream_t st) {
  auto k = &rows_r2c_kernel<T, CC, LOCAL, N, W>;
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<grid, ct_threads<N, W>(), smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int CC, int EPI, int N, int W>
cudaError_t c2r_ct_go(const RowsArgs<T>& a, dim3 grid, size_t smem, cudaStream_t st) {
  auto k = &rows_c2r_kernel<T, CC, EPI, N, W>;
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<grid, ct_threads<N, W>(), smem, st>>>(a);
  return cudaGetLastError();
}

// cudaErrorNotSupported: no compile-time variant for this combination
template <typename T, int N, int W>
cudaError_t c2r_ct_dispatch(int C, int epi, const RowsArgs<T>& a, dim3 grid, size_t smem,
                            cudaStream_t st) {
  if (C == 6) {
    switch (epi) {
      case kEpiPlain: return c2r_ct_go<T, 6, kEpiPlain, N, W>(a, grid, smem, st);
      case kEpiUpdate: return c2r_ct_go<T, 6, kEpiUpdate, N, W>(a, grid, smem, st);
      case kEpiResid:
        if constexpr (sizeof(T) == 8) return c2r_ct_go<T, 6, kEpiResid, N, W>(a, grid, smem, st);
        return cudaErrorInvalidValue;
      case kEpiRhs: return c2r_ct_go<T, 6, kEpiRhs, N, W>(a, grid, smem, st);
    }
  } else if (C == 3) {
    switch (epi) {
      case kEpiPlain: return c2r_ct_go<T, 3, kEpiPlain, N, W>(a, grid, smem, st);
      case kEpiUpdate: return c2r_ct_go<T, 3, kEpiUpdate, N, W>(a, grid, smem, st);
      case kEpiResid:
        if constexpr (sizeof(T) == 8) return c2r_ct_go<T, 3, kEpiResid, N, W>(a, grid, smem, st);
        return cudaErrorInvalidValue;
      case kEpiRhs: return c2r_ct_go<T, 3, kEpiRhs, N, W>(a, grid, smem, st);
    }
  }
  return cudaErrorNotSupported;
}

// Long contiguous rows (n = 384, 512, 768, 1024, three components): the persistent
// kernels of jb_rows_long.cuh when every row satisfies their bulk-copy rules
// (16-byte aligned bases and pitches, a spectral row of a multiple of 16
// bytes, a tail of the spectral row of 3 or 4 complex); cudaErrorNotSupported
// otherwise, and the general kernels run.
template <typename T>
cudaError_t long_r2c_launch(const RowsArgs<T>& a, int n, const LocalDesc* local, cudaStream_t st) {
  using C = cx<T>;
  const int ib = local ? local->index_bytes : 0;
  if (!a.contig || !al16(a.x) || !al16(a.out) || (a.sp * sizeof(C)) % 16 != 0 ||
      (a.cstride_l * sizeof(C)) % 16 != 0 || (a.g.ls * sizeof(T)) % 16 != 0 ||
      (ib != 0 && ib != 1 && ib != 4) || (ib != 0 && !al16(local->phase)))
    return cudaErrorNotSupported;
  const int tabn = local ? local->nphase * local_entry(local->kind, 2) : 0;
  const size_t tabb = (local && tabn <= 2 * kTabStage) ? (size_t)tabn * sizeof(T) : 0;
  const size_t smem = long_r2c_layout(sizeof(C), n, a.sp, (size_t)n * ib, tabb).total;
  if (smem > kSmemCap - 4096) return cudaErrorNotSupported;
  const int64_t tiles = a.g.rows * a.L;
  auto go = [&](auto k, int threads) {
    cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    k<<<persistent_grid(k, threads, smem, tiles), threads, smem, st>>>(a);
    return cudaGetLastError();
  };
  constexpr int TH = 192;
  if (n == 1024) return local ? go(&rows_long_r2c_kernel<T, 1024, true>, TH)
                              : go(&rows_long_r2c_kernel<T, 1024, false>, TH);
  if (n == 768) return local ? go(&rows_long_r2c_kernel<T, 768, true>, TH)
                             : go(&rows_long_r2c_kernel<T, 768, false>, TH);
  if (n == 384) return local ? go(&rows_long_r2c_kernel<T, 384, true>, TH)
                             : go(&rows_long_r2c_kernel<T, 384, false>, TH);
  return local ? go(&rows_long_r2c_kernel<T, 512, true>, TH)
               : go(&rows_long_r2c_kernel<T, 512, false>, TH);
}

template <typename T>
cudaError_t long_c2r_launch(const RowsArgs<T>& a, int n, int epi, int* nb_out, cudaStream_t st) {
  using C = cx<T>;
  const int64_t tail = a.sp - 3 * (int64_t)(n / 2);
  if (epi == kEpiResid || !a.contig || !al16(a.cin) || !al16(a.y) ||
      (epi == kEpiRhs && !al16(a.rhs)) || (a.sp * sizeof(C)) % 16 != 0 ||
      (tail * (int64_t)sizeof(C)) % 16 != 0 || tail < 3 || tail > 4 ||
      (a.cstride_l * sizeof(C)) % 16 != 0 || (a.g.ls * sizeof(T)) % 16 != 0)
    return cudaErrorNotSupported;
  const size_t smem = long_c2r_layout(sizeof(C), n).total;
  const int64_t tiles = a.g.rows * a.L;
  auto go = [&](auto k) {
    cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    // at most one CTA per row: the partials hold rows slots per load case
    int grid = persistent_grid(k, 192, smem, tiles);
    if (grid > a.g.rows) grid = (int)a.g.rows;
    if (nb_out) *nb_out = grid;
    k<<<grid, 192, smem, st>>>(a);
    return cudaGetLastError();
  };
  if (n == 1024) {
    switch (epi) {
      case kEpiUpdate: return go(&rows_long_c2r_kernel<T, 1024, kEpiUpdate>);
      case kEpiRhs: return go(&rows_long_c2r_kernel<T, 1024, kEpiRhs>);
      default: return go(&rows_long_c2r_kernel<T, 1024, kEpiPlain>);
    }
  }
  if (n == 768) {
    switch (epi) {
      case kEpiUpdate: return go(&rows_long_c2r_kernel<T, 768, kEpiUpdate>);
      case kEpiRhs: return go(&rows_long_c2r_kernel<T, 768, kEpiRhs>);
      default: return go(&rows_long_c2r_kernel<T, 768, kEpiPlain>);
    }
  }
  if (n == 384) {
    switch (epi) {
      case kEpiUpdate: return go(&rows_long_c2r_kernel<T, 384, kEpiUpdate>);
      case kEpiRhs: return go(&rows_long_c2r_kernel<T, 384, kEpiRhs>);
      default: return go(&rows_long_c2r_kernel<T, 384, kEpiPlain>);
    }
  }
  switch (epi) {
    case kEpiUpdate: return go(&rows_long_c2r_kernel<T, 512, kEpiUpdate>);
    case kEpiRhs: return go(&rows_long_c2r_kernel<T, 512, kEpiRhs>);
    default: return go(&rows_long_c2r_kernel<T, 512, kEpiPlain>);
  }
}

template <typename T>
cudaError_t rows_r2c_t(const AxisData& ax, int C, int L, const void* x, const RealGeom& g,
                       void* out, const LocalDesc* local, cudaStream_t st, int64_t spitch) {
  RowsArgs<T> a{};
  int R, W;
  size_t smem;
  const int n = ax.plan.n;
  if (C != 1 && C != 3 && C != 6) return cudaErrorInvalidValue;
  if (local && C == 1) return cudaErrorInvalidValue;
  const int nphase = local ? local->nphase : 0;
  const int entry = local ? local_entry(local->kind, local->dim) : 2;
  const bool padded = spitch > (int64_t)(n / 2 + 1) * C;
  if (!rows_shape(sizeof(T) == 8 ? F64 : F32, n, C, false, &R, &W, &smem, local != nullptr,
                  nphase, entry, padded))
    return cudaErrorInvalidValue;
  a.x = static_cast<const T*>(x);
  a.out = static_cast<cx<T>*>(out);
  a.tw = static_cast<const cx<T>*>(ax.tw);
  a.plan = ax.plan;
  a.g = g;
  a.R = R;
  a.W = W;
  a.m = n / 2 + 1;
  a.sp = spitch > 0 ? spitch : (int64_t)a.m * C;
  if (a.sp < (int64_t)a.m * C || a.sp > (int64_t)a.m * C + 1 ||
      (C == 6 && a.sp != (int64_t)a.m * C))
    return cudaErrorInvalidValue;
  a.contig = contiguous_rows(g, n, C);
  a.cstride_l = g.rows * a.sp;
  a.L = L;
  if (local) {
    a.phase = local->phase;
    a.index_bytes = local->index_bytes;
    a.table = static_cast<const T*>(local->table);
    a.nphase = local->nphase;
    a.kind = local->kind;
    a.dim = local->dim;
  }
  if ((n == 384 || n == 512 || n == 768 || n == 1024) && C == 3) {
    const cudaError_t e = long_r2c_launch<T>(a, n, local, st);
    if (e != cudaErrorNotSupported) return e;
  }
  if ((n == 64 || n == 128 || n == 256) && (C == 3 || C == 6)) {
    // compile-time tiles: W = 12 columns (6 for n = 256), R = 2 W / C rows
    const int wct = n <= 128 ? 12 : 6;
    const int rct = 2 * wct / C;
    const size_t sct = rows_smem(sizeof(T) == 8 ? F64 : F32, n, C, rct, wct, false,
                                 local != nullptr, nphase, entry, padded);
    if (sct <= kSmemBudget + 24 * 1024) {
      RowsArgs<T> b = a;
      b.R = rct;
      b.W = wct;
      dim3 grid((unsigned)((g.rows + rct - 1) / rct), (unsigned)L);
      switch (n * 16 + C * 2 + (local ? 1 : 0)) {
        case 64 * 16 + 6: return r2c_ct_go<T, 3, false, 64, 12>(b, grid, sct, st);
        case 64 * 16 + 7: return r2c_ct_go<T, 3, true, 64, 12>(b, grid, sct, st);
        case 64 * 16 + 12: return r2c_ct_go<T, 6, false, 64, 12>(b, grid, sct, st);
        case 64 * 16 + 13: return r2c_ct_go<T, 6, true, 64, 12>(b, grid, sct, st);
        case 128 * 16 + 6: return r2c_ct_go<T, 3, false, 128, 12>(b, grid, sct, st);
        case 128 * 16 + 7: return r2c_ct_go<T, 3, true, 128, 12>(b, grid, sct, st);
        case 128 * 16 + 12: return r2c_ct_go<T, 6, false, 128, 12>(b, grid, sct, st);
        case 128 * 16 + 13: return r2c_ct_go<T, 6, true, 128, 12>(b, grid, sct, st);
        case 256 * 16 + 6: return r2c_ct_go<T, 3, false, 256, 6>(b, grid, sct, st);
        case 256 * 16 + 7: return r2c_ct_go<T, 3, true, 256, 6>(b, grid, sct, st);
        case 256 * 16 + 12: return r2c_ct_go<T, 6, false, 256, 6>(b, grid, sct, st);
        case 256 * 16 + 13: return r2c_ct_go<T, 6, true, 256, 6>(b, grid, sct, st);
        default: break;
      }
    }
  }
  const int threads = tile_threads(W);
  dim3 grid((unsigned)((g.rows + R - 1) / R), (unsigned)L);
  if (local) {
    return C == 3 ? r2c_go<T, 3, true>(a, grid, threads, smem, st)
                  : r2c_go<T, 6, true>(a, grid, threads, smem, st);
  }
  if (C == 1) return r2c_go<T, 1, false>(a, grid, threads, smem, st);
  if (C == 3) return r2c_go<T, 3, false>(a, grid, threads, smem, st);
  return r2c_go<T, 6, false>(a, grid, threads, smem, st);
}

template <typename T>
cudaError_t rows_c2r_t(const AxisData& ax, int C, int L, const void* in, void* y,
                       const RealGeom& g, double scale, const UpdateDesc* upd, int* nb_out,
                       cudaStream_t st, int64_t spitch) {
  RowsArgs<T> a{};
  int R, W;
  size_t smem;
  const int n = ax.plan.n;
  if (C != 1 && C != 3 && C != 6) return cudaErrorInvalidValue;
  if (upd && C == 1) return cudaErrorInvalidValue;
  const bool padded = spitch > (int64_t)(n / 2 + 1) * C;
  if (!rows_shape(sizeof(T) == 8 ? F64 : F32, n, C, upd != nullptr, &R, &W, &smem, false, 0, 2,
                  padded))
    return cudaErrorInvalidValue;
  a.cin = static_cast<const cx<T>*>(in);
  a.y = static_cast<T*>(upd ? upd->eps : y);
  a.tw = static_cast<const cx<T>*>(ax.tw);
  a.plan = ax.plan;
  a.g = g;
  a.R = R;
  a.W = W;
  a.m = n / 2 + 1;
  a.sp = spitch > 0 ? spitch : (int64_t)a.m * C;
  if (a.sp < (int64_t)a.m * C || a.sp > (int64_t)a.m * C + 1 ||
      (C == 6 && a.sp != (int64_t)a.m * C))
    return cudaErrorInvalidValue;
  a.contig = contiguous_rows(g, n, C);
  a.cstride_l = g.rows * a.sp;
  a.scale = static_cast<T>(scale);
  a.L = L;
  const int epi = upd ? upd->mode : kEpiPlain;
  if (upd) {
    a.E = upd->E;
    a.partials = upd->partials;
    a.rhs = static_cast<const T*>(upd->rhs);
    a.rout = upd->rout;
    if ((epi == kEpiResid || epi == kEpiRhs) && !a.contig) return cudaErrorInvalidValue;
    if (epi == kEpiResid && (sizeof(T) != 8 || !upd->rout)) return cudaErrorInvalidValue;
    if (epi == kEpiRhs && !upd->rhs) return cudaErrorInvalidValue;
  }
  if ((n == 384 || n == 512 || n == 768 || n == 1024) && C == 3) {
    const cudaError_t e = long_c2r_launch<T>(a, n, epi, nb_out, st);
    if (e != cudaErrorNotSupported) return e;
  }
  if ((n == 64 || n == 128 || n == 256) && (C == 3 || C == 6)) {
    const int wct = n <= 128 ? 12 : 6;
    const int rct = 2 * wct / C;
    const size_t sct = rows_smem(sizeof(T) == 8 ? F64 : F32, n, C, rct, wct, upd != nullptr,
                                 false, 0, 2, padded);
    if (sct <= kSmemBudget + 24 * 1024) {
      RowsArgs<T> b = a;
      b.R = rct;
      b.W = wct;
      dim3 grid((unsigned)((g.rows + rct - 1) / rct), (unsigned)L);
      if (nb_out) *nb_out = (int)grid.x;
      cudaError_t e = cudaErrorNotSupported;
      if (n == 64) e = c2r_ct_dispatch<T, 64, 12>(C, epi, b, grid, sct, st);
      if (n == 128) e = c2r_ct_dispatch<T, 128, 12>(C, epi, b, grid, sct, st);
      if (n == 256) e = c2r_ct_dispatch<T, 256, 6>(C, epi, b, grid, sct, st);
      if (e != cudaErrorNotSupported) return e;
    }
  }
  const int threads = tile_threads(W);
  dim3 grid((unsigned)((g.rows + R - 1) / R), (unsigned)L);
  if (nb_out) *nb_out = (int)grid.x;
  switch (epi) {
    case kEpiUpdate: return c2r_go_c<T, kEpiUpdate>(C, a, grid, threads, smem, st);
    case kEpiResid:
      if constexpr (sizeof(T) == 8) return c2r_go_c<T, kEpiResid>(C, a, grid, threads, smem, st);
      return cudaErrorInvalidValue;
    case kEpiRhs: return c2r_go_c<T, kEpiRhs>(C, a, grid, threads, smem, st);
    default: break;
  }
  if (C == 1) return c2r_go<T, 1, kEpiPlain>(a, grid, threads, smem, st);
  if (C == 3) return c2r_go<T, 3, kEpiPlain>(a, grid, threads, smem, st);
  return c2r_go<T, 6, kEpiPlain>(a, grid, threads, smem, st);
}

template <typename T> GreenTables<T> to_tables(const GreenDeviceTables* gt) {
  GreenTables<T> t{};
  if (!gt) return t;
  for (int d = 0; d < 3; ++d) {
    t.kt[d] = static_cast<const T*>(gt->kt[d]);
    t.kn[d] = static_cast<const T*>(gt->kn[d]);
    t.kp[d] = static_cast<const T*>(gt->kp[d]);
    t.wn[d] = static_cast<const T*>(gt->wn[d]);
    t.wp[d] = static_cast<const T*>(gt->wp[d]);
  }
  t.inv2g = static_cast<T>(gt->inv2g);
  t.c1 = static_cast<T>(gt->c1);
  t.variant = gt->variant;
  return t;
}

template <typename T, int MODE, int DIM>
cudaError_t cols_launch(const ColsArgs<T>& a, dim3 grid, int threads, size_t smem,
                        cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(&cols_kernel<T, MODE, DIM>);
  cudaError_t e = ensure_smem(fn, smem);
  if (e != cudaSuccess) return e;
  cols_kernel<T, MODE, DIM><<<grid, threads, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int MODE, int DIM, int N, int W>
cudaError_t cols_ct_launch(const CUtensorMap& tin, const CUtensorMap& tout,
                           const ColsArgs<T>& a, int nbox, size_t smem, int64_t tiles,
                           cudaStream_t st) {
  auto k = &cols_tma_kernel<T, MODE, DIM, N, W>;
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  const int threads = ct_threads<N, W>();
  const int grid = persistent_grid(k, threads, smem, tiles);
  k<<<grid, threads, smem, st>>>(tin, tout, a, nbox);
  return cudaGetLastError();
}

template <typename T, int DIM, int N, int W>
cudaError_t cols_inplace_launch(const CUtensorMap& tin, const CUtensorMap& tout,
                                const ColsArgs<T>& a, int nbox, size_t smem, int64_t tiles,
                                cudaStream_t st) {
  auto k = &cols_tma_inplace_kernel<T, DIM, N, W>;
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  const int threads = ct_threads_inplace<N, W>();
  const int grid = persistent_grid(k, threads, smem, tiles);
  k<<<grid, threads, smem, st>>>(tin, tout, a, nbox);
  return cudaGetLastError();
}

template <typename T, int N>
cudaError_t cols_ct_dispatch(int mode, int dim, const CUtensorMap& tin, const CUtensorMap& tout,
                             const ColsArgs<T>& a, int nbox, size_t smem, int64_t tiles,
                             cudaStream_t st) {
  if (mode == 0) return cols_ct_launch<T, 0, 2, N, 8>(tin, tout, a, nbox, smem, tiles, st);
  if (mode == 1) return cols_ct_launch<T, 1, 2, N, 8>(tin, tout, a, nbox, smem, tiles, st);
  if constexpr (N == 128 || N == 256) {
    // six-column Green tiles (one 3D coefficient, two 2D ones): the width
    // FP64 tiles of 256 rows fit; at 128 rows an autotuner candidate
    if (a.W == 6) {
      if (dim == 2) return cols_ct_launch<T, 2, 2, N, 6>(tin, tout, a, nbox, smem, tiles, st);
      return cols_ct_launch<T, 2, 3, N, 6>(tin, tout, a, nbox, smem, tiles, st);
    }
  }
  if (dim == 2) return cols_ct_launch<T, 2, 2, N, 12>(tin, tout, a, nbox, smem, tiles, st);
  return cols_ct_launch<T, 2, 3, N, 12>(tin, tout, a, nbox, smem, tiles, st);
}

template <typename T, int MODE, int DIM>
cudaError_t cols_tma_launch(const CUtensorMap& tin, const CUtensorMap& tout,
                            const ColsArgs<T>& a, int nbox, int threads, size_t smem,
                            int64_t tiles, cudaStream_t st) {
  auto k = &cols_tma_kernel<T, MODE, DIM>;
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  const int grid = persistent_grid(k, threads, smem, tiles);
  k<<<grid, threads, smem, st>>>(tin, tout, a, nbox);
  return cudaGetLastError();
}

template <typename T>
cudaError_t cols_t(const AxisData& ax, int mode, int64_t outer, int64_t inner, const void* in,
                   void* out, int C, int dim, const GreenDeviceTables* gt, int64_t m_last,
                   cudaStream_t st, const ColsTuning* tune, int64_t pitch) {
  ColsArgs<T> a{};
  int W;
  size_t smem;
  const int n = ax.plan.n;
  if (outer < 1 || outer > 65535 || inner < 1) return cudaErrorInvalidValue;
  if (mode == 2 && (inner % C) != 0) return cudaErrorInvalidValue;
  if (!cols_shape(sizeof(T) == 8 ? F64 : F32, n, mode == 2 ? C : 1, &W, &smem))
    return cudaErrorInvalidValue;
  a.in = static_cast<const cx<T>*>(in);
  a.out = static_cast<cx<T>*>(out);
  a.tw = static_cast<const cx<T>*>(ax.tw);
  a.plan = ax.plan;
  a.inner = inner;
  a.pitch = pitch > 0 ? pitch : inner;
  if (a.pitch < inner) return cudaErrorInvalidValue;
  a.W = W;
  a.C = C;
  a.m_last = m_last;
  a.gt = to_tables<T>(gt);
  a.mn = gt ? static_cast<const T*>(gt->mn) : nullptr;
  a.outer = outer;
  {
    int Wp, nbuf;
    size_t sp;
    const size_t cs = sizeof(cx<T>);
    // Green tiles transformed in place: 24 columns at n = 128, 12 at n = 256,
    // where that width fits.  Tuning value ct = 2 asks for them; the built-in
    // rule (no schedule set) takes them for 3D grids at n = 256 and in FP32
    // at n = 128 (measured on B200, 128^3 x 6 and 256^3 x 2: Green pass FP64
    // 256: -17%, FP32 256: -8%, FP32 128: -5%, FP64 128: equal)
    const bool rule = !tune || (tune->w == 0 && tune->nbuf == 0 && tune->ct == 1);
    // the register-tile Green pass (n = 32 ... 1024): tuning value ct = 3;
    // the built-in rule takes it except where the in-place or column tiles
    // measured faster on B200 (3D n = 256: 1.22 vs 1.41 ms FP64 at 256^3 x 2;
    // FP32 on the fly at 3D n = 128: 0.191 vs 0.210 ms at 128^3 x 6; FP32 at
    // 3D n = 192: 0.50 vs 0.57 ms filtered at 192^3 x 2)
    const bool rule_reg = rule && !(dim == 3 && n == 256) &&
                          !(dim == 3 && n == 128 && sizeof(T) == 4 && a.mn == nullptr) &&
                          !(dim == 3 && n == 192 && sizeof(T) == 4);
    if (mode == 2 && gt && green_axis0_regs_supported(n, C, dim) &&
        ((tune && tune->ct == 3) || rule_reg)) {
      GreenDeviceTables g2 = *gt;
      g2.mn = a.mn;
      const cudaError_t e = launch_green_axis0_regs(sizeof(T) == 8 ? F64 : F32, ax, outer, inner,
                                                  a.pitch, in, out, C, dim, g2, m_last, st);
      if (e != cudaErrorNotSupported) return e;
    }
    const bool want_inplace =
        (tune && tune->ct == 2) || (rule && dim == 3 && (n == 256 || sizeof(T) == 4));
    if (mode == 2 && want_inplace && (n == 128 || n == 256) && (C == 3 || C == 6) &&
        al16(in) && al16(out) && (a.pitch * cs) % 16 == 0) {
      const int wi = n == 128 ? 24 : 12;
      ColsTuning ti = tune ? *tune : ColsTuning{};
      ti.w = wi;
      if (cols_tma_shape(sizeof(T) == 8 ? F64 : F32, n, C, &Wp, &sp, &nbuf, a.mn == nullptr, &ti,
                         true) &&
          Wp == wi) {
        CUtensorMap tin, tout;
        if (make_cols_map(&tin, in, sizeof(T) == 8, inner, a.pitch, n, outer, Wp, n) &&
            make_cols_map(&tout, out, sizeof(T) == 8, inner, a.pitch, n, outer, Wp, n)) {
          ColsArgs<T> b = a;
          b.W = Wp;
          b.nbuf = nbuf;
          const int64_t tiles = (inner + Wp - 1) / Wp * outer;
          if (n == 128)
            return dim == 2 ? cols_inplace_launch<T, 2, 128, 24>(tin, tout, b, n, sp, tiles, st)
                            : cols_inplace_launch<T, 3, 128, 24>(tin, tout, b, n, sp, tiles, st);
          return dim == 2 ? cols_inplace_launch<T, 2, 256, 12>(tin, tout, b, n, sp, tiles, st)
                          : cols_inplace_launch<T, 3, 256, 12>(tin, tout, b, n, sp, tiles, st);
        }
      }
    }
    // rows 16-byte aligned; a last chunk reaching past `inner` is zero-filled
    // by the load and clipped by the store
    if (al16(in) && al16(out) && (a.pitch * cs) % 16 == 0 &&
        cols_tma_shape(sizeof(T) == 8 ? F64 : F32, n, mode == 2 ? C : 1, &Wp, &sp, &nbuf,
                       mode == 2 && a.mn == nullptr, tune)) {
      // rows per box: the largest divisor of n up to 256 whose boxes start
      // on 128-byte boundaries of the tile (a tensor copy's shared-memory
      // address must be 128-byte aligned: n = 700 in FP64 takes 140-row
      // boxes, not 175)
      int nbox = n <= 256 ? n : 256;
      while (nbox > 1 && (n % nbox != 0 || (nbox < n && (nbox * (size_t)Wp * cs) % 128 != 0)))
        --nbox;
      CUtensorMap tin, tout;
      if (nbox >= 8 &&
          make_cols_map(&tin, in, sizeof(T) == 8, inner, a.pitch, n, outer, Wp, nbox) &&
          make_cols_map(&tout, out, sizeof(T) == 8, inner, a.pitch, n, outer, Wp, nbox)) {
        ColsArgs<T> b = a;
        b.W = Wp;
        b.nbuf = nbuf;
        const int thr = tile_threads(Wp);
        const int64_t tiles = (inner + Wp - 1) / Wp * outer;
        const bool ct_w = (mode == 2 ? (Wp == 12 || (Wp == 6 && n >= 128)) : Wp == 8) &&
                          (mode != 2 || C == 3 || C == 6);
        if (ct_w && (!tune || tune->ct)) {
          if (n == 64) return cols_ct_dispatch<T, 64>(mode, dim, tin, tout, b, nbox, sp, tiles, st);
          if (n == 128)
            return cols_ct_dispatch<T, 128>(mode, dim, tin, tout, b, nbox, sp, tiles, st);
          if (n == 256)
            return cols_ct_dispatch<T, 256>(mode, dim, tin, tout, b, nbox, sp, tiles, st);
        }
        if (mode == 0) return cols_tma_launch<T, 0, 2>(tin, tout, b, nbox, thr, sp, tiles, st);
        if (mode == 1) return cols_tma_launch<T, 1, 2>(tin, tout, b, nbox, thr, sp, tiles, st);
        if (dim == 2) return cols_tma_launch<T, 2, 2>(tin, tout, b, nbox, thr, sp, tiles, st);
        return cols_tma_launch<T, 2, 3>(tin, tout, b, nbox, thr, sp, tiles, st);
      }
    }
  }
  const int threads = tile_threads(W);
  dim3 grid((unsigned)((inner + W - 1) / W), (unsigned)outer);
  if (mode == 0) return cols_launch<T, 0, 2>(a, grid, threads, smem, st);
  if (mode == 1) return cols_launch<T, 1, 2>(a, grid, threads, smem, st);
  if (dim == 2) return cols_launch<T, 2, 2>(a, grid, threads, smem, st);
  return cols_launch<T, 2, 3>(a, grid, threads, smem, st);
}

}  // namespace

int max_axis_length(int dtype) { return dtype == F64 ? 4096 : 8192; }

cudaError_t fetch_fault_async(unsigned* host, cudaStream_t st) {
  return cudaMemcpyFromSymbolAsync(host, g_jb_fault, sizeof(unsigned), 0,
                                   cudaMemcpyDeviceToHost, st);
}

cudaError_t set_first_wait_limit(int polls) {
  const unsigned v = polls < 0 ? kWaitLimit : (unsigned)polls;
  return cudaMemcpyToSymbol(c_jb_wait_first, &v, sizeof(unsigned));
}

cudaError_t read_and_clear_fault(unsigned* out) {
  unsigned zero = 0;
  cudaError_t e = cudaMemcpyFromSymbol(out, g_jb_fault, sizeof(unsigned));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(g_jb_fault, &zero, sizeof(unsigned));
}

cudaError_t launch_rows_r2c(int dtype, const AxisData& ax, int C, int L, const void* x,
                            const RealGeom& g, void* out, const LocalDesc* local,
                            cudaStream_t st, int64_t spitch) {
  return dtype == F64 ? rows_r2c_t<double>(ax, C, L, x, g, out, local, st, spitch)
                      : rows_r2c_t<float>(ax, C, L, x, g, out, local, st, spitch);
}

cudaError_t launch_rows_c2r(int dtype, const AxisData& ax, int C, int L, const void* in,
                            void* y, const RealGeom& g, double scale, const UpdateDesc* upd,
                            int* nb_out, cudaStream_t st, int64_t spitch) {
  return dtype == F64 ? rows_c2r_t<double>(ax, C, L, in, y, g, scale, upd, nb_out, st, spitch)
                      : rows_c2r_t<float>(ax, C, L, in, y, g, scale, upd, nb_out, st, spitch);
}

cudaError_t launch_cols(int dtype, const AxisData& ax, int mode, int64_t outer, int64_t inner,
                        const void* in, void* out, int C, int dim,
                        const GreenDeviceTables* gt, int64_t n1, int64_t m_last,
                        cudaStream_t st, const ColsTuning* tune, int64_t pitch) {
  (void)n1;
  return dtype == F64
             ? cols_t<double>(ax, mode, outer, inner, in, out, C, dim, gt, m_last, st, tune, pitch)
             : cols_t<float>(ax, mode, outer, inner, in, out, C, dim, gt, m_last, st, tune, pitch);
}

cudaError_t launch_local(int dtype, const LocalDesc& loc, int C, int L, int64_t nvox,
                         const void* x, void* y, cudaStream_t st) {
  if (C != 3 && C != 6) return cudaErrorInvalidValue;
  const size_t es = dtype == F64 ? 8 : 4;
  // six-component voxels move as 2-element vectors: the fields must be
  // aligned to two elements (three-component voxels move element-wise)
  if (C == 6 && (reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % (2 * es) != 0)
    return cudaErrorInvalidValue;
  const int g = grid_for(nvox);
  for (int64_t l0 = 0; l0 < L; l0 += 65535) {  // load cases on grid.y
    const dim3 grid((unsigned)g, (unsigned)std::min<int64_t>(65535, L - l0));
    const size_t o = (size_t)l0 * nvox * C * es;
    const void* xl = static_cast<const char*>(x) + o;
    void* yl = static_cast<char*>(y) + o;
    if (dtype == F64) {
      const double* t = static_cast<const double*>(loc.table);
      if (C == 6)
        local_kernel<double, 6><<<grid, kThreads, 0, st>>>(
            loc, t, nvox, static_cast<const double*>(xl), static_cast<double*>(yl));
      else
        local_kernel<double, 3><<<grid, kThreads, 0, st>>>(
            loc, t, nvox, static_cast<const double*>(xl), static_cast<double*>(yl));
    } else {
      const float* t = static_cast<const float*>(loc.table);
      if (C == 6)
        local_kernel<float, 6><<<grid, kThreads, 0, st>>>(
            loc, t, nvox, static_cast<const float*>(xl), static_cast<float*>(yl));
      else
        local_kernel<float, 3><<<grid, kThreads, 0, st>>>(
            loc, t, nvox, static_cast<const float*>(xl), static_cast<float*>(yl));
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_local_sum(int dtype, const LocalDesc& loc, int C, int L, int64_t nvox,
                             const void* eps, double* partials, int* nb_out, cudaStream_t st) {
  int g = grid_for(nvox);
  if (g > 1024) g = 1024;
  *nb_out = g;
  dim3 grid((unsigned)g, (unsigned)L);
  if (dtype == F64)
    local_sum_kernel<double><<<grid, kThreads, 0, st>>>(
        loc, static_cast<const double*>(loc.table), C, nvox, static_cast<const double*>(eps),
        partials);
  else
    local_sum_kernel<float><<<grid, kThreads, 0, st>>>(
        loc, static_cast<const float*>(loc.table), C, nvox, static_cast<const float*>(eps),
        partials);
  return cudaGetLastError();
}

cudaError_t launch_local_gradient(int dtype, int dim, int64_t nvox, int L, const void* eps,
                                  const void* zeta, double scale, double* out,
                                  cudaStream_t st) {
  const int grid = grid_for(nvox);
  if (dtype == F64)
    local_gradient_kernel<double><<<grid, kThreads, 0, st>>>(
        dim, nvox, L, static_cast<const double*>(eps), static_cast<const double*>(zeta), scale,
        out);
  else
    local_gradient_kernel<float><<<grid, kThreads, 0, st>>>(
        dim, nvox, L, static_cast<const float*>(eps), static_cast<const float*>(zeta), scale,
        out);
  return cudaGetLastError();
}

cudaError_t launch_block_linear(int dtype, int64_t nvox, int L, int osz, int isz, const void* a,
                                const void* x, void* y, int transpose, cudaStream_t st) {
  if (osz > 8 || isz > 8) return cudaErrorInvalidValue;
  const int grid = grid_for((int64_t)L * nvox);
  if (dtype == F64)
    block_linear_kernel<double><<<grid, kThreads, 0, st>>>(
        nvox, L, osz, isz, static_cast<const double*>(a), static_cast<const double*>(x),
        static_cast<double*>(y), transpose);
  else
    block_linear_kernel<float><<<grid, kThreads, 0, st>>>(
        nvox, L, osz, isz, static_cast<const float*>(a), static_cast<const float*>(x),
        static_cast<float*>(y), transpose);
  return cudaGetLastError();
}

cudaError_t launch_green_by_freq(int dtype, int dim, const GreenDeviceTables& gt, int64_t count,
                                 const int* b, const void* tau, void* eta, cudaStream_t st) {
  const int grid = grid_for(count);
  if (dtype == F64) {
    auto t = to_tables<double>(&gt);
    if (dim == 2)
      green_by_freq_kernel<double, 2><<<grid, kThreads, 0, st>>>(
          t, count, b, static_cast<const double2*>(tau), static_cast<double2*>(eta));
    else
      green_by_freq_kernel<double, 3><<<grid, kThreads, 0, st>>>(
          t, count, b, static_cast<const double2*>(tau), static_cast<double2*>(eta));
  } else {
    auto t = to_tables<float>(&gt);
    if (dim == 2)
      green_by_freq_kernel<float, 2><<<grid, kThreads, 0, st>>>(
          t, count, b, static_cast<const float2*>(tau), static_cast<float2*>(eta));
    else
      green_by_freq_kernel<float, 3><<<grid, kThreads, 0, st>>>(
          t, count, b, static_cast<const float2*>(tau), static_cast<float2*>(eta));
  }
  return cudaGetLastError();
}

cudaError_t launch_green_table(int dtype, int dim, const GreenDeviceTables& gt, int64_t n0,
                               int64_t n1, int64_t m_last, void* out, cudaStream_t st) {
  const int64_t total = (dim == 3 ? n1 * m_last : m_last) * n0;
  const int grid = grid_for(total);
  if (dtype == F64) {
    auto t = to_tables<double>(&gt);
    if (dim == 2)
      green_table_kernel<double, 2><<<grid, kThreads, 0, st>>>(t, n0, n1, m_last,
                                                                 static_cast<double*>(out));
    else
      green_table_kernel<double, 3><<<grid, kThreads, 0, st>>>(t, n0, n1, m_last,
                                                                 static_cast<double*>(out));
  } else {
    auto t = to_tables<float>(&gt);
    if (dim == 2)
      green_table_kernel<float, 2><<<grid, kThreads, 0, st>>>(t, n0, n1, m_last,
                                                                static_cast<float*>(out));
    else
      green_table_kernel<float, 3><<<grid, kThreads, 0, st>>>(t, n0, n1, m_last,
                                                                static_cast<float*>(out));
  }
  return cudaGetLastError();
}

cudaError_t launch_fill_macro(int dtype, int C, int L, int64_t nvox, const double* E, void* eps,
                              cudaStream_t st) {
  const int grid = grid_for((int64_t)L * nvox * C);
  if (dtype == F64)
    fill_macro_kernel<double><<<grid, kThreads, 0, st>>>(C, L, nvox, E, static_cast<double*>(eps));
  else
    fill_macro_kernel<float><<<grid, kThreads, 0, st>>>(C, L, nvox, E, static_cast<float*>(eps));
  return cudaGetLastError();
}

cudaError_t launch_axpy_to_f64(int dtype, int64_t n, const void* d, double* y,
                               cudaStream_t st) {
  if (dtype == F32) return launch_axpy_f32_to_f64(n, static_cast<const float*>(d), y, st);
  if (n <= 0) return cudaSuccess;
  axpy_f64_kernel<<<grid_for(n / 2 + 1), kThreads, 0, st>>>(n, static_cast<const double*>(d), y);
  return cudaGetLastError();
}

cudaError_t launch_axpy_f32_to_f64(int64_t n, const float* d, double* y, cudaStream_t st) {
  const bool vec = (reinterpret_cast<uintptr_t>(d) & 15u) == 0 &&
                   (reinterpret_cast<uintptr_t>(y) & 15u) == 0;
  if (!vec) return cudaErrorInvalidValue;
  axpy_f32_to_f64_kernel<<<grid_for(n / 4 + 1), kThreads, 0, st>>>(n, d, y);
  return cudaGetLastError();
}

cudaError_t launch_reduce_rows(const double* partials, int L, int nb, double* out, double factor,
                               const double* factors, int take_sqrt, cudaStream_t st) {
  reduce_rows_kernel<<<L, kThreads, 0, st>>>(partials, nb, out, factor, factors, take_sqrt);
  return cudaGetLastError();
}

cudaError_t launch_reduce_cols(const double* partials, int L, int C, int nb, double* out,
                               double factor, cudaStream_t st) {
  reduce_rows_kernel<<<L * C, kThreads, 0, st>>>(partials, nb, out, factor, nullptr, 0);
  return cudaGetLastError();
}

}  // namespace jb
