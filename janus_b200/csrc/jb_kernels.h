// Host-side launch interface of the janus_b200 pass kernels (internal; the
// public interface is the C ABI in include/janus_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "jb_device.cuh"

namespace jb {

enum Dtype { F64 = 0, F32 = 1 };
enum Variant { TRUNCATED = 0, FILTERED = 1 };

// per-axis FFT data: plan + device twiddle table (T complex, n entries)
struct AxisData {
  AxisPlan plan;
  void* tw = nullptr;  // device, cx<T>[n]
};

// discrete Green operator tables on the device (type T)
struct GreenDeviceTables {
  void* kt[3] = {nullptr, nullptr, nullptr};
  void* kn[3] = {nullptr, nullptr, nullptr};
  void* kp[3] = {nullptr, nullptr, nullptr};
  void* wn[3] = {nullptr, nullptr, nullptr};
  void* wp[3] = {nullptr, nullptr, nullptr};
  double inv2g = 0, c1 = 0;
  int variant = 0;
  const void* mn = nullptr;  // per-coefficient operator table (T), built by launch_green_table
};

// Real-side geometry of a batch of fields [L][rows][n][C] with arbitrary
// element strides: element (l, row, e, c) lives at
//   l*ls + (row / n1r)*s0 + (row % n1r)*s1 + e*es + c*cs.
struct RealGeom {
  int64_t rows;  // rows per load case (n0 or n0*n1)
  int64_t n1r;   // 1 (2D) or n1 (3D)
  int64_t ls, s0, s1, es, cs;
};

// Local operator (C - C0):eps on a phase map; table holds (tr, dev) pairs
// in the field's precision.
struct LocalDesc {
  const void* phase = nullptr;  // uint8 or int32 per voxel, row-major grid (index_bytes 0: none)
  int index_bytes = 1;          // 0 (one entry per voxel), 1 or 4
  const void* table = nullptr;  // device: kind 0 T[nphase][2] = (tr, dev); kind 1 T[nphase][s][s]
  int nphase = 1;
  int dim = 2;
  int kind = 0;                 // 0 isotropic (tr, dev), 1 full s x s matrix per entry
};

// Solver epilogue of the last pass (y = scale * c2r(spectrum)):
//  mode 1: eps <- E - y in place, partials = sum (new - old)^2
//  mode 2: rout <- (E - y) - eps as FP32 (FP64 fields only), partials = sum r^2
//  mode 3: eps <- rhs - y in place (rhs a field of the same type)
struct UpdateDesc {
  int mode = 1;
  void* eps = nullptr;          // field read/updated (layout of RealGeom)
  const double* E = nullptr;    // device [L][C] macroscopic strains (FP64)
  double* partials = nullptr;   // device [L][gridDim.x]
  const void* rhs = nullptr;    // mode 3
  float* rout = nullptr;        // mode 2
};

// BiCGSTAB scalars of one load case (device); active: 1 iterating, 2 last
// update pending, 0 frozen (converged or broken down)
struct KrylovState {
  double rho, alpha, omega, rho1;
  int active;
};
// blocks per load case of the Krylov vector kernels (partials per dot)
int krylov_blocks(int64_t nel, int L);
// partials[(l*2+q)*nb+b]: q 0 = a.b, q 1 = c.d (c may be NULL), per load case
cudaError_t launch_krylov_dot(int dtype, int64_t nel, int L, const void* a, const void* b,
                              const void* c, const void* d, double* partials, cudaStream_t st);
// stage 0: init + rho1, 1: alpha, 2: omega, 3: rho1 after the x/r update
cudaError_t launch_krylov_scalars(int stage, int64_t nel, int L, const double* partials,
                                  KrylovState* state, cudaStream_t st);
// which 0: x(=p) = r + beta (x - omega t(=v)); 1: x(=s) = r - alpha t(=v);
// 2: x += alpha p + omega s, r = s - omega t, partials of rh.r
cudaError_t launch_krylov_update(int dtype, int which, int64_t nel, int L, void* x, const void* p,
                                 const void* s, const void* t, void* r, const void* rh,
                                 const KrylovState* state, double* partials, cudaStream_t st);

// y[i] += (double) d[i] over n elements (FP64 field, FP32 correction)
// GMRES(m) vector kernels (FP64, batched over L load cases; basis vector i of
// load case l at V + i * vs + l * nel; at most gmres_chunk() vectors a launch)
int gmres_chunk();
// out[l * ldo + o0 + i] = w . V_{j0+i}, i < cnt (partials: L * chunk * blocks)
cudaError_t launch_gmres_dots(int64_t nel, int L, const double* w, const double* V, int64_t vs,
                              int j0, int cnt, double* partials, double* out, int ldo, int o0,
                              cudaStream_t st);
// w += sign * sum_{i < cnt} coef[l * ldc + c0 + i] V_{j0+i}; with partials
// and sq (both or neither), sq[l] = |w|^2 after the update
cudaError_t launch_gmres_axpys(int64_t nel, int L, double* w, const double* V, int64_t vs, int j0,
                               int cnt, const double* coef, int ldc, int c0, double sign,
                               double* partials, double* sq, cudaStream_t st);
// w /= sqrt(sq[l]) (0 where the norm is 0 or not finite)
cudaError_t launch_gmres_scale(int64_t nel, int L, double* w, const double* sq, cudaStream_t st);
// r[l][v][c] = E[l][c] - ax[l][v][c] (r may alias ax)
cudaError_t launch_gmres_resid(int64_t nvox, int C, int L, const double* E, const double* ax,
                               double* r, cudaStream_t st);
cudaError_t launch_axpy_f32_to_f64(int64_t n, const float* d, double* y, cudaStream_t st);
// y[i] += d[i], d of the dtype (FP32 or FP64)
cudaError_t launch_axpy_to_f64(int dtype, int64_t n, const void* d, double* y, cudaStream_t st);

int max_axis_length(int dtype);
// bit 0: a kernel gave up a bounded wait (see jb_async.cuh); cleared on read
cudaError_t read_and_clear_fault(unsigned* out);
// queue a copy of the fault word to `host` on `st` (read after a stream sync)
cudaError_t fetch_fault_async(unsigned* host, cudaStream_t st);
// polls of the first bounded wait of every copy (0: the default limit)
cudaError_t set_first_wait_limit(int polls);  // negative: the default

// Spectral row pitch (complex elements) of the solver's internal half
// spectrum: m * C, plus one where FP32 rows of m * C complex would not span a
// multiple of 16 bytes (2D, C = 3, m odd), so that rows start on 16-byte
// boundaries and the column passes can use tensor TMA.
inline int64_t spectral_pitch(int dtype, int64_t m, int C) {
  const int64_t p = m * C;
  return (dtype == F32 && (p % 2) != 0) ? p + 1 : p;
}
// r2c along the contiguous axis: real x (geom) -> complex out [L][rows][sp]
// (the first m * C of each row's sp complex elements; sp = spitch, default
// m * C, at most m * C + 1).
cudaError_t launch_rows_r2c(int dtype, const AxisData& ax, int C, int L, const void* x,
                            const RealGeom& g, void* out, const LocalDesc* local,
                            cudaStream_t st, int64_t spitch = 0);
// c2r along the contiguous axis: complex in [L][rows][sp] -> real y (geom),
// y = scale * c2r(in), or the solver update when upd != nullptr.
cudaError_t launch_rows_c2r(int dtype, const AxisData& ax, int C, int L, const void* in,
                            void* y, const RealGeom& g, double scale,
                            const UpdateDesc* upd, int* nblocks_out, cudaStream_t st,
                            int64_t spitch = 0);
// tile schedule of a column pass (0 = the built-in rule): tile width in
// complex columns (a multiple of the coefficient size for the Green pass),
// rotating input tiles (2 or 3), and whether compile-time FFT tiles may be
// used where they exist (0 no, 1 yes, 2 Green tiles transformed in place:
// 24 columns at n = 128, 12 at n = 256, no partner tile; 3 the register-tile
// Green pass, n = 32 ... 1024).  Chosen per operator by the autotuner.
struct ColsTuning {
  int w = 0;
  int nbuf = 0;
  int ct = 1;
};

// complex transform along a strided axis of [outer][n][pitch] (complex
// units; the first `inner` of each row's `pitch` elements, pitch 0 = inner).
// mode 0: forward, 1: inverse, 2: forward -> Green contraction -> inverse
// (axis 0 only; dim/m_last/grid describe the spectrum for the contraction).
cudaError_t launch_cols(int dtype, const AxisData& ax, int mode, int64_t outer,
                        int64_t inner, const void* in, void* out, int C, int dim,
                        const GreenDeviceTables* gt, int64_t n1, int64_t m_last,
                        cudaStream_t st, const ColsTuning* tune = nullptr,
                        int64_t pitch = 0);
// Axis-0 Green pass for n0 = 32 ... 1024 (powers of two) as register tiles
// (five phases up to 256, seven at 512 and 1024; jb_green_axis0.cu): in/out complex
// [L][n0][pitch] (the first `inner` = F * C of each row), in place allowed;
// gt.mn, when set, is the operator table of launch_green_table.
bool green_axis0_regs_supported(int n0, int C, int dim);
cudaError_t launch_green_axis0_regs(int dtype, const AxisData& ax0, int64_t L, int64_t inner,
                                  int64_t pitch, const void* in, void* out, int C, int dim,
                                  const GreenDeviceTables& gt, int64_t m_last,
                                  cudaStream_t st);
// Table of the Green operator on the half spectrum of an n0 x n1 (x n2) grid:
// the symmetric Mandel matrix of each coefficient, upper triangle (order in
// jb_green.cuh, GSize), component-major: table[(f12 * NT + c) * n0 + b0],
// f12 = b1 * m + b2 (3D) or b1 (2D), NT = 21 (3D) / 6 (2D).  `out` has
// n0 * n1 * m * NT (3D) reals of the dtype.
cudaError_t launch_green_table(int dtype, int dim, const GreenDeviceTables& gt, int64_t n0,
                               int64_t n1, int64_t m_last, void* out, cudaStream_t st);
// y[l][v] = (C - C0)(v) : x[l][v] on a phase map (contiguous fields)
cudaError_t launch_local(int dtype, const LocalDesc& loc, int C, int L, int64_t nvox,
                         const void* x, void* y, cudaStream_t st);
// per-voxel matrices: y[l][v] = a[v] x[l][v] (or a[v]^T x[l][v])
cudaError_t launch_block_linear(int dtype, int64_t nvox, int L, int osz, int isz,
                                const void* a, const void* x, void* y, int transpose,
                                cudaStream_t st);
// Green contraction at an explicit list of indices b (int32 [count][dim]),
// tau/eta complex [count][C] (may alias)
cudaError_t launch_green_by_freq(int dtype, int dim, const GreenDeviceTables& gt,
                                 int64_t count, const int* b, const void* tau, void* eta,
                                 cudaStream_t st);
// eps[l][v][c] = E[l][c]
cudaError_t launch_fill_macro(int dtype, int C, int L, int64_t nvox, const double* E,
                              void* eps, cudaStream_t st);
// out[l] = f(sum_b partials[l][b]) * factor * (factors ? factors[l] : 1),
// f = sqrt or identity; fixed summation order (deterministic)
cudaError_t launch_reduce_rows(const double* partials, int L, int nb, double* out,
                               double factor, const double* factors, int take_sqrt,
                               cudaStream_t st);
// sum over voxels of (C - C0):eps, per load case and component (FP64 partials)
cudaError_t launch_local_sum(int dtype, const LocalDesc& loc, int C, int L, int64_t nvox,
                             const void* eps, double* partials, int* nblocks_out,
                             cudaStream_t st);
// per-voxel strain / adjoint-strain contractions (gradient of mean stresses
// with respect to the (sph, dev) field): out double[nvox][2]
cudaError_t launch_local_gradient(int dtype, int dim, int64_t nvox, int L, const void* eps,
                                  const void* zeta, double scale, double* out,
                                  cudaStream_t st);
cudaError_t launch_reduce_cols(const double* partials, int L, int C, int nb, double* out,
                               double factor, cudaStream_t st);

}  // namespace jb
