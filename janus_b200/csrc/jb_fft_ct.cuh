// Compile-time Stockham FFT over a shared-memory tile of W columns for the
// grid sizes the solver is benchmarked on (N = 64, 128, 256; 2D sizes 512
// and 1024).  Transform length, radices, tile width and thread count are
// template constants, so every index, loop bound and twiddle step folds to
// constants; each stage is one fully unrolled loop of radix-8/16 butterflies
// held in registers, and a transform is two (three for N >= 512) stages.
// Same algorithm and twiddle table as fft_tile in jb_device.cuh.
#pragma once

#include "jb_device.cuh"

namespace jb {

template <int N> struct CtSched;
template <> struct CtSched<64> { static constexpr int R0 = 8, R1 = 8, R2 = 1; };
template <> struct CtSched<128> { static constexpr int R0 = 16, R1 = 8, R2 = 1; };
template <> struct CtSched<256> { static constexpr int R0 = 16, R1 = 16, R2 = 1; };
template <> struct CtSched<512> { static constexpr int R0 = 8, R1 = 8, R2 = 8; };
template <> struct CtSched<1024> { static constexpr int R0 = 16, R1 = 8, R2 = 8; };

// threads of a compile-time tile: the largest butterfly count of a stage,
// rounded up to whole warps
template <int N, int W> __host__ __device__ constexpr int ct_threads() {
  using S = CtSched<N>;
  int m = (N / S::R0) * W;
  if ((N / S::R1) * W > m) m = (N / S::R1) * W;
  if (S::R2 > 1 && (N / S::R2) * W > m) m = (N / S::R2) * W;
  return (m + 31) / 32 * 32;
}

template <int R, int Ns, int N, int W, int THREADS, int DIR, typename C>
__device__ __forceinline__ void stage_ct(const C* __restrict__ x, C* __restrict__ y,
                                         const C* __restrict__ tw) {
  constexpr int NR = N / R;
  constexpr int BF = NR * W;
  constexpr int TSTEP = N / (Ns * R);
  constexpr int ITER = (BF + THREADS - 1) / THREADS;
#pragma unroll
  for (int i = 0; i < ITER; ++i) {
    const int b = threadIdx.x + i * THREADS;
    if ((BF % THREADS) != 0 && b >= BF) break;
    const int col = b % W;
    const int j = b / W;
    const int k = j % Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = x[(j + r * NR) * W + col];
    if (Ns > 1 && k != 0) {
      const int kt = k * TSTEP;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<DIR>(tw, kt * r));
    }
    Dft<R, DIR, C>::run(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) y[(base + r * Ns) * W + col] = v[r];
  }
}

// Transform the W columns of tile `a` (ping-pong partner `b`); returns the
// tile holding the result.  blockDim.x must equal ct_threads<N, W>().
template <int N, int W, int DIR, typename C>
__device__ __forceinline__ C* fft_ct(C* a, C* b, const C* tw) {
  using S = CtSched<N>;
  constexpr int TH = ct_threads<N, W>();
  stage_ct<S::R0, 1, N, W, TH, DIR>(a, b, tw);
  __syncthreads();
  stage_ct<S::R1, S::R0, N, W, TH, DIR>(b, a, tw);
  __syncthreads();
  if constexpr (S::R2 > 1) {
    stage_ct<S::R2, S::R0 * S::R1, N, W, TH, DIR>(a, b, tw);
    __syncthreads();
    return b;
  } else {
    return a;
  }
}

// In-place form: each thread holds all of its butterflies' inputs of a stage
// in registers before any output is stored (a barrier between), so a tile
// needs no ping-pong partner.  Threads: the butterfly count of the stage
// with the largest radix (the other stages take several butterflies a
// thread), rounded up to whole warps.
template <int N, int W> __host__ __device__ constexpr int ct_threads_inplace() {
  using S = CtSched<N>;
  int r = S::R0 > S::R1 ? S::R0 : S::R1;
  if (S::R2 > r) r = S::R2;
  return ((N / r) * W + 31) / 32 * 32;
}

template <int R, int Ns, int N, int W, int THREADS, int DIR, typename C>
__device__ __forceinline__ void stage_ct_inplace(C* __restrict__ x, const C* __restrict__ tw) {
  constexpr int NR = N / R;
  constexpr int BF = NR * W;
  constexpr int TSTEP = N / (Ns * R);
  constexpr int ITER = (BF + THREADS - 1) / THREADS;
  C v[ITER][R];
#pragma unroll
  for (int i = 0; i < ITER; ++i) {
    const int b = threadIdx.x + i * THREADS;
    if ((BF % THREADS) == 0 || b < BF) {
      const int col = b % W;
      const int j = b / W;
      const int k = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = x[(j + r * NR) * W + col];
      if (Ns > 1 && k != 0) {
        const int kt = k * TSTEP;
#pragma unroll
        for (int r = 1; r < R; ++r) v[i][r] = cmul(v[i][r], twid<DIR>(tw, kt * r));
      }
      Dft<R, DIR, C>::run(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITER; ++i) {
    const int b = threadIdx.x + i * THREADS;
    if ((BF % THREADS) == 0 || b < BF) {
      const int col = b % W;
      const int j = b / W;
      const int k = j % Ns;
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) x[(base + r * Ns) * W + col] = v[i][r];
    }
  }
  __syncthreads();
}

// transform the W columns of tile `a` in place; blockDim.x must equal
// ct_threads_inplace<N, W>()
template <int N, int W, int DIR, typename C>
__device__ __forceinline__ void fft_ct_inplace(C* a, const C* tw) {
  using S = CtSched<N>;
  constexpr int TH = ct_threads_inplace<N, W>();
  stage_ct_inplace<S::R0, 1, N, W, TH, DIR>(a, tw);
  stage_ct_inplace<S::R1, S::R0, N, W, TH, DIR>(a, tw);
  if constexpr (S::R2 > 1) stage_ct_inplace<S::R2, S::R0 * S::R1, N, W, TH, DIR>(a, tw);
}

}  // namespace jb
