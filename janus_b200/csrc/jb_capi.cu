// C ABI of janus_b200 (declared in include/janus_b200.h): handle objects,
// argument validation with the reference's error semantics, host-side
// per-wave-vector Green matrices, and the orchestration of the pass kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/janus_b200.h"
#include "jb_kernels.h"

using jb::AxisData;
using jb::F32;
using jb::F64;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define JB_CUDA(expr)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? JB_ENOMEM : JB_ECUDA,                \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

#define JB_TRY(expr)          \
  do {                        \
    int r_ = (expr);          \
    if (r_ != JB_OK) return r_; \
  } while (0)

size_t real_size(int dtype) { return dtype == F64 ? 8 : 4; }

// radices used on the device: 8, 4, 2 for powers of two, then 3, 5, then
// any remaining prime handled by the generic butterfly
void factorize(int n, jb::AxisPlan& p) {
  p.n = n;
  p.nf = 0;
  int m = n;
  while (m % 8 == 0) { p.fac[p.nf++] = 8; m /= 8; }
  while (m % 4 == 0) { p.fac[p.nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p.fac[p.nf++] = 2; m /= 2; }
  while (m % 3 == 0) { p.fac[p.nf++] = 3; m /= 3; }
  while (m % 5 == 0) { p.fac[p.nf++] = 5; m /= 5; }
  for (int f = 7; m > 1 && (long)f * f <= m; f += 2)
    while (m % f == 0) { p.fac[p.nf++] = f; m /= f; }
  if (m > 1) p.fac[p.nf++] = m;
  int Ns = 1;
  for (int f = 0; f < p.nf; ++f) {
    p.tstep[f] = n / (Ns * p.fac[f]);
    // ceil(2^32 / Ns): q = umulhi(j, magic) == j / Ns for j < 2^16
    p.nsmagic[f] = Ns > 1 ? (unsigned)((((uint64_t)1 << 32) + Ns - 1) / Ns) : 0u;
    Ns *= p.fac[f];
  }
}

struct DeviceBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

int dev_alloc(void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? JB_ENOMEM : JB_ECUDA,
                std::string("cudaMalloc(") + std::to_string(bytes) +
                    " bytes): " + cudaGetErrorString(e));
  }
  return JB_OK;
}

int ensure_buf(DeviceBuf& b, size_t bytes) {
  if (b.bytes >= bytes && b.p) return JB_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  JB_TRY(dev_alloc(&b.p, bytes));
  b.bytes = bytes;
  return JB_OK;
}

// twiddle table exp(-2 pi i t / n) computed in long double, rounded once
int make_axis(int n, int dtype, AxisData& ax) {
  factorize(n, ax.plan);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  if (dtype == F64) {
    std::vector<double> h(2 * (size_t)n);
    for (int t = 0; t < n; ++t) {
      long double a = two_pi * (long double)t / (long double)n;
      h[2 * t] = (double)cosl(a);
      h[2 * t + 1] = (double)-sinl(a);
    }
    JB_TRY(dev_alloc(&ax.tw, h.size() * sizeof(double)));
    JB_CUDA(cudaMemcpy(ax.tw, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> h(2 * (size_t)n);
    for (int t = 0; t < n; ++t) {
      long double a = two_pi * (long double)t / (long double)n;
      h[2 * t] = (float)cosl(a);
      h[2 * t + 1] = (float)-sinl(a);
    }
    JB_TRY(dev_alloc(&ax.tw, h.size() * sizeof(float)));
    JB_CUDA(cudaMemcpy(ax.tw, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  return JB_OK;
}

int check_shape(int dim, const int64_t* shape, int dtype) {
  if (dim != 2 && dim != 3)
    return fail(JB_EINVAL, "length of shape must be 2 or 3 (was " + std::to_string(dim) + ")");
  if (!shape) return fail(JB_EINVAL, "shape must not be NULL");
  if (dtype != F64 && dtype != F32)
    return fail(JB_EINVAL, "dtype must be JB_F64 or JB_F32");
  for (int d = 0; d < dim; ++d) {
    if (shape[d] <= 0)
      return fail(JB_EINVAL, "shape" + std::to_string(d) + " should be > 0 (was " +
                                 std::to_string(shape[d]) + ")");
    if (shape[d] > jb::max_axis_length(dtype))
      return fail(JB_EINVAL, "axis " + std::to_string(d) + " of length " +
                                 std::to_string(shape[d]) + " exceeds the supported maximum " +
                                 std::to_string(jb::max_axis_length(dtype)));
  }
  return JB_OK;
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

int launch_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return JB_OK;
  if (e == cudaErrorInvalidValue)
    return fail(JB_EINVAL, std::string(what) + ": unsupported size for the tiled kernels");
  return fail(JB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Outcome of each load case of a solve, updated at every residual readback:
// a non-finite residual or one grown kDivergeFactor-fold over the smallest
// seen stops the load case for good (JB_SOLVE_NON_FINITE / _DIVERGING).
constexpr double kDivergeFactor = 1e4;

struct Outcome {
  std::vector<double> best, last;
  std::vector<int> stopped;  // 0, JB_SOLVE_NON_FINITE or JB_SOLVE_DIVERGING
  explicit Outcome(int L) : best(L, INFINITY), last(L, INFINITY), stopped(L, 0) {}
  // record residual r of load case l; true when the case no longer holds the
  // iteration back (converged or stopped)
  bool update(int l, double r, double tol) {
    if (stopped[l]) return true;
    last[l] = r;
    if (!std::isfinite(r)) {
      stopped[l] = JB_SOLVE_NON_FINITE;
      return true;
    }
    if (r > tol && best[l] > 0.0 && r > kDivergeFactor * best[l]) {
      stopped[l] = JB_SOLVE_DIVERGING;
      return true;
    }
    best[l] = std::min(best[l], r);
    return r <= tol;
  }
  void write(double tol, int* status, int off = 0) const {
    if (!status) return;
    for (size_t l = 0; l < stopped.size(); ++l)
      status[off + l] = stopped[l]       ? stopped[l]
                        : last[l] <= tol ? JB_SOLVE_CONVERGED
                                         : JB_SOLVE_MAX_ITER;
  }
};

// after a stream synchronisation: the fault word fetched with it
// (fetch_fault_async) must be clear, else the call's results are invalid
int check_fault(unsigned fetched, const char* what) {
  if (fetched == 0) return JB_OK;
  unsigned f = 0;
  jb::read_and_clear_fault(&f);
  return fail(JB_EFAULT, std::string(what) +
                             ": a kernel gave up a bounded wait for its asynchronous copies "
                             "(device fault word " + std::to_string(fetched) +
                             "); the results of this call are invalid");
}

// ---------------------------------------------------------------------------
// continuous Green operator, isotropic.pyx:158-182 / 227-290, same operations
// ---------------------------------------------------------------------------
struct GreenAux {
  double d1, d2, d3, d4;
};

GreenAux green_aux(double g, double nu) {
  // isotropic.pyx:135-138
  return {1.0 / g, 0.5 / (g * (1.0 - nu)), 0.25 / g, 0.5 / g};
}

void green_matrix2(const GreenAux& a, const double* k, double* out) {
  const double k0 = k[0], k1 = k[1];
  double k0k0 = k0 * k0, k1k1 = k1 * k1;
  double g00, g01, g02, g11, g12, g22;
  if (k0k0 + k1k1 == 0.) {
    g00 = g01 = g02 = g11 = g12 = g22 = 0.;
  } else {
    const double s = 1.0 / (k0k0 + k1k1);
    k0k0 *= s;
    k1k1 *= s;
    const double k0k1 = s * k0 * k1;
    g00 = k0k0 * (a.d1 - a.d2 * k0k0);
    g11 = k1k1 * (a.d1 - a.d2 * k1k1);
    const double dummy = -a.d2 * k0k0 * k1k1;
    g01 = dummy;
    g22 = 2 * (a.d3 + dummy);
    g02 = M_SQRT2 * k0k1 * (a.d4 - a.d2 * k0k0);
    g12 = M_SQRT2 * k0k1 * (a.d4 - a.d2 * k1k1);
  }
  const double m[9] = {g00, g01, g02, g01, g11, g12, g02, g12, g22};
  std::memcpy(out, m, sizeof(m));
}

void green_matrix3(const GreenAux& a, const double* k, double* out) {
  const double k0 = k[0], k1 = k[1], k2 = k[2];
  double k0k0 = k0 * k0, k1k1 = k1 * k1, k2k2 = k2 * k2;
  double g[6][6];
  if (k0k0 + k1k1 + k2k2 == 0.) {
    std::memset(out, 0, 36 * sizeof(double));
    return;
  }
  const double s = 1.0 / (k0k0 + k1k1 + k2k2);
  k0k0 *= s;
  k1k1 *= s;
  k2k2 *= s;
  const double k1k2 = s * k1 * k2, k2k0 = s * k2 * k0, k0k1 = s * k0 * k1;
  const double d1 = a.d1, d2 = a.d2, d3 = a.d3, d4 = a.d4;
  g[0][0] = k0k0 * (d1 - d2 * k0k0);
  g[1][1] = k1k1 * (d1 - d2 * k1k1);
  g[2][2] = k2k2 * (d1 - d2 * k2k2);
  g[3][3] = 2. * (d3 * (k1k1 + k2k2) - d2 * k1k1 * k2k2);
  g[4][4] = 2. * (d3 * (k2k2 + k0k0) - d2 * k2k2 * k0k0);
  g[5][5] = 2. * (d3 * (k0k0 + k1k1) - d2 * k0k0 * k1k1);
  g[0][1] = -d2 * k0k0 * k1k1;
  g[0][2] = -d2 * k0k0 * k2k2;
  g[0][3] = -M_SQRT2 * d2 * k0k0 * k1k2;
  g[0][4] = M_SQRT2 * k2k0 * (d4 - d2 * k0k0);
  g[0][5] = M_SQRT2 * k0k1 * (d4 - d2 * k0k0);
  g[1][2] = -d2 * k1k1 * k2k2;
  g[1][3] = M_SQRT2 * k1k2 * (d4 - d2 * k1k1);
  g[1][4] = -M_SQRT2 * d2 * k1k1 * k2k0;
  g[1][5] = M_SQRT2 * k0k1 * (d4 - d2 * k1k1);
  g[2][3] = M_SQRT2 * k1k2 * (d4 - d2 * k2k2);
  g[2][4] = M_SQRT2 * k2k0 * (d4 - d2 * k2k2);
  g[2][5] = -M_SQRT2 * d2 * k2k2 * k0k1;
  g[3][4] = 2 * k0k1 * (d3 - d2 * k2k2);
  g[3][5] = 2 * k2k0 * (d3 - d2 * k1k1);
  g[4][5] = 2 * k1k2 * (d3 - d2 * k0k0);
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) {
      out[i * 6 + j] = g[i][j];
      out[j * 6 + i] = g[i][j];
    }
}

void green_matrix_dim(int dim, const GreenAux& a, const double* k, double* out) {
  if (dim == 2)
    green_matrix2(a, k, out);
  else
    green_matrix3(a, k, out);
}

}  // namespace

// ===========================================================================
// handles
// ===========================================================================

struct jb_fft_s {
  int dim = 0, dtype = 0;
  int64_t n[3] = {1, 1, 1};
  AxisData ax[3];
  DeviceBuf scratch;
};

struct jb_green_s {
  int dim = 0, dtype = 0, variant = 0;
  int64_t n[3] = {1, 1, 1};
  double h = 1, g = 1, nu = 0;
  double s[3] = {0, 0, 0};
  AxisData ax[3];
  jb::GreenDeviceTables gt;
  std::vector<void*> tables;
  DeviceBuf spec;
  DeviceBuf bidx;
  DeviceBuf mnbuf;        // per-coefficient operator table, built on first use
  jb::ColsTuning tune_plain, tune_green;  // column-pass schedules (autotuner)
  int tune_table = 0;  // Green contraction: 0 built-in rule, 1 table, 2 on the fly
  bool use_table = true;  // false: evaluate the operator on the fly
};

struct jb_local_s {
  int dim = 0, dtype = 0, nphase = 0, index_bytes = 1, kind = 0;
  int64_t n[3] = {1, 1, 1};
  int64_t nvox = 0;
  void* phase = nullptr;
  void* table = nullptr;
};

// CUDA events recorded between the passes of solver steps (benchmarks)
struct PassRecorder {
  std::vector<cudaEvent_t> ev;
  int npass = 0;
  int max_steps = 0;
  int steps = 0;
  size_t cursor = 0;
  bool active = false;
  void mark(cudaStream_t st) {
    if (active && cursor < ev.size()) cudaEventRecord(ev[cursor++], st);
  }
  void release() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    ev.clear();
    active = false;
  }
};

struct jb_solver_s {
  jb_green* green = nullptr;
  jb_local* local = nullptr;
  int L = 1;
  DeviceBuf spec, partials, E, res, mean, normd;
  std::vector<double> Eh;
  std::vector<double> norm;  // 1 / (sqrt(N) |E_l|)
  int nb_rows = 0;
  bool load_set = false;
  PassRecorder rec;
};

namespace {

void free_axes(AxisData* ax) {
  for (int d = 0; d < 3; ++d)
    if (ax[d].tw) {
      cudaFree(ax[d].tw);
      ax[d].tw = nullptr;
    }
}

int upload_table(jb_green* g, int dtype, const std::vector<double>& v, void** out) {
  void* p = nullptr;
  const size_t rs = real_size(dtype);
  JB_TRY(dev_alloc(&p, v.size() * rs));
  g->tables.push_back(p);
  if (dtype == F64) {
    JB_CUDA(cudaMemcpy(p, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(v.begin(), v.end());
    JB_CUDA(cudaMemcpy(p, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
  }
  *out = p;
  return JB_OK;
}

// spectral passes shared by jb_green_apply and the solver
// x: real fields (or eps with local), spec: complex scratch, y: output
// whether the Green pass contracts through the table (else on the fly):
// the tuned choice, or the built-in rule (the table for the filtered
// operator's 2^d aliases per coefficient, on the fly for one alias)
bool green_uses_table(const jb_green* g) {
  return g->use_table &&
         (g->tune_table == 1 || (g->tune_table == 0 && g->variant == JB_FILTERED));
}

// the operator's symmetric Mandel matrix at every half-spectrum coefficient, built once
// on first use (or ahead of a graph capture)
int green_prepare(jb_green* g, cudaStream_t st) {
  if (!g->use_table || g->gt.mn) return JB_OK;
  const int dim = g->dim;
  const int64_t n0 = g->n[0], n1 = g->n[1];
  const int64_t m = (dim == 2 ? g->n[1] : g->n[2]) / 2 + 1;
  const int NT = dim == 3 ? 21 : 6;
  const size_t bytes = (size_t)n0 * (dim == 3 ? n1 * m : m) * NT * real_size(g->dtype);
  JB_TRY(ensure_buf(g->mnbuf, bytes));
  JB_TRY(launch_status(jb::launch_green_table(g->dtype, dim, g->gt, n0, n1, m, g->mnbuf.p, st),
                       "green_table"));
  g->gt.mn = g->mnbuf.p;
  return JB_OK;
}

int green_passes(jb_green* g, const void* x, void* y, int64_t L, void* spec,
                 const jb::LocalDesc* local, const jb::UpdateDesc* upd, int* nb_rows,
                 cudaStream_t st, PassRecorder* rec = nullptr) {
  PassRecorder dummy;
  if (!rec) rec = &dummy;
  const int dim = g->dim;
  const int C = dim == 2 ? 3 : 6;
  const int64_t n0 = g->n[0], n1 = g->n[1], n2 = g->n[2];
  const int64_t nlast = dim == 2 ? n1 : n2;
  const int64_t m = nlast / 2 + 1;
  const int64_t N = dim == 2 ? n0 * n1 : n0 * n1 * n2;
  jb::RealGeom geom{};
  geom.cs = 1;
  geom.es = C;
  geom.ls = N * C;
  if (dim == 2) {
    geom.rows = n0;
    geom.n1r = 1;
    geom.s0 = n1 * C;
    geom.s1 = 0;
  } else {
    geom.rows = n0 * n1;
    geom.n1r = n1;
    geom.s0 = n1 * n2 * C;
    geom.s1 = n2 * C;
  }
  const AxisData& last = g->ax[dim - 1];
  if ((int64_t)L > 65535) return fail(JB_EINVAL, "batch too large (max 65535)");
  // 2D spectral rows padded to 16 bytes (FP32, odd m * C); 3D rows (C = 6)
  // always are
  const int64_t sp = dim == 2 ? jb::spectral_pitch(g->dtype, m, C) : m * C;
  rec->mark(st);
  JB_TRY(launch_status(
      jb::launch_rows_r2c(g->dtype, last, C, (int)L, x, geom, spec, local, st, sp), "rows_r2c"));
  rec->mark(st);
  if (dim == 3) {
    JB_TRY(launch_status(jb::launch_cols(g->dtype, g->ax[1], 0, L * n0, m * C, spec, spec, C,
                                         dim, nullptr, n1, m, st, &g->tune_plain),
                         "cols_fwd_axis1"));
    rec->mark(st);
  }
  const int64_t inner0 = (dim == 2 ? m : n1 * m) * C;
  // the contraction reads the table (built once) or evaluates the
  // operator on the fly; built-in rule: the table for the filtered operator
  // (2^d aliases per coefficient), on the fly for the single-alias ones
  const bool table = green_uses_table(g);
  jb::GreenDeviceTables gt = g->gt;
  if (table) {
    JB_TRY(green_prepare(g, st));
    gt.mn = g->gt.mn;
  } else {
    gt.mn = nullptr;
  }
  JB_TRY(launch_status(jb::launch_cols(g->dtype, g->ax[0], 2, L, inner0, spec, spec, C, dim,
                                       &gt, n1, m, st, &g->tune_green,
                                       dim == 2 ? sp : inner0),
                       "cols_green_axis0"));
  rec->mark(st);
  if (dim == 3) {
    JB_TRY(launch_status(jb::launch_cols(g->dtype, g->ax[1], 1, L * n0, m * C, spec, spec, C,
                                         dim, nullptr, n1, m, st, &g->tune_plain),
                         "cols_inv_axis1"));
    rec->mark(st);
  }
  // mode 4 (x + Gamma0[..]): the right-hand-side epilogue rhs - scale*y with
  // a negative scale
  double scale = 1.0 / (double)N;
  jb::UpdateDesc add;
  if (upd && upd->mode == 4) {
    add = *upd;
    add.mode = 3;
    upd = &add;
    scale = -scale;
  }
  JB_TRY(launch_status(jb::launch_rows_c2r(g->dtype, last, C, (int)L, spec, y, geom, scale, upd,
                                           nb_rows, st, sp),
                       "rows_c2r"));
  rec->mark(st);
  return JB_OK;
}

// complex elements of one field's internal half spectrum (2D rows padded as
// green_passes lays them out)
int64_t spec_elems(const jb_green* g) {
  const int C = g->dim == 2 ? 3 : 6;
  const int64_t nlast = g->dim == 2 ? g->n[1] : g->n[2];
  const int64_t m = nlast / 2 + 1;
  if (g->dim == 2) return g->n[0] * jb::spectral_pitch(g->dtype, m, C);
  return g->n[0] * g->n[1] * m * C;
}

}  // namespace

extern "C" {

int jb_version(void) { return 100; }

const char* jb_last_error(void) { return g_err.c_str(); }

int jb_max_axis_length(int dtype) { return jb::max_axis_length(dtype); }

int jb_device_status(unsigned* fault) {
  if (!fault) return fail(JB_EINVAL, "NULL argument");
  JB_CUDA(jb::read_and_clear_fault(fault));
  return JB_OK;
}

int jb_set_wait_limit(int polls) {
  JB_CUDA(jb::set_first_wait_limit(polls));
  return JB_OK;
}

// ---------------------------------------------------------------------------
// FFT
// ---------------------------------------------------------------------------

int jb_fft_create(int dim, const int64_t* shape, int dtype, unsigned flags, jb_fft** out) {
  (void)flags;
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  JB_TRY(check_shape(dim, shape, dtype));
  jb_fft* f = new jb_fft();
  f->dim = dim;
  f->dtype = dtype;
  for (int d = 0; d < dim; ++d) f->n[d] = shape[d];
  for (int d = 0; d < dim; ++d) {
    int r = make_axis((int)shape[d], dtype, f->ax[d]);
    if (r != JB_OK) {
      free_axes(f->ax);
      delete f;
      return r;
    }
  }
  *out = f;
  return JB_OK;
}

int jb_fft_destroy(jb_fft* f) {
  if (!f) return JB_OK;
  free_axes(f->ax);
  if (f->scratch.p) cudaFree(f->scratch.p);
  delete f;
  return JB_OK;
}

static jb::RealGeom fft_geom(const jb_fft* f, const int64_t* strides) {
  jb::RealGeom g{};
  g.cs = 0;
  g.ls = 0;
  if (f->dim == 2) {
    g.rows = f->n[0];
    g.n1r = 1;
    g.s0 = strides ? strides[0] : f->n[1];
    g.s1 = 0;
    g.es = strides ? strides[1] : 1;
  } else {
    g.rows = f->n[0] * f->n[1];
    g.n1r = f->n[1];
    g.s0 = strides ? strides[0] : f->n[1] * f->n[2];
    g.s1 = strides ? strides[1] : f->n[2];
    g.es = strides ? strides[2] : 1;
  }
  return g;
}

int jb_fft_r2c(jb_fft* f, const void* r, const int64_t* r_strides, void* c, void* stream) {
  if (!f || !r || !c) return fail(JB_EINVAL, "NULL argument");
  cudaStream_t st = as_stream(stream);
  const jb::RealGeom g = fft_geom(f, r_strides);
  const int dim = f->dim;
  const int64_t nlast = f->n[dim - 1];
  const int64_t m = nlast / 2 + 1;
  JB_TRY(launch_status(jb::launch_rows_r2c(f->dtype, f->ax[dim - 1], 1, 1, r, g, c, nullptr, st),
                       "fft rows_r2c"));
  if (dim == 3)
    JB_TRY(launch_status(jb::launch_cols(f->dtype, f->ax[1], 0, f->n[0], m, c, c, 1, dim,
                                         nullptr, f->n[1], m, st),
                         "fft cols axis1"));
  const int64_t inner0 = dim == 2 ? m : f->n[1] * m;
  JB_TRY(launch_status(
      jb::launch_cols(f->dtype, f->ax[0], 0, 1, inner0, c, c, 1, dim, nullptr, f->n[1], m, st),
      "fft cols axis0"));
  return JB_OK;
}

int jb_fft_c2r(jb_fft* f, const void* c, void* r, const int64_t* r_strides, void* stream) {
  if (!f || !r || !c) return fail(JB_EINVAL, "NULL argument");
  cudaStream_t st = as_stream(stream);
  const int dim = f->dim;
  const int64_t nlast = f->n[dim - 1];
  const int64_t m = nlast / 2 + 1;
  const int64_t rows = dim == 2 ? f->n[0] : f->n[0] * f->n[1];
  const size_t bytes = (size_t)rows * m * 2 * real_size(f->dtype);
  JB_TRY(ensure_buf(f->scratch, bytes));
  void* s = f->scratch.p;
  const int64_t inner0 = dim == 2 ? m : f->n[1] * m;
  JB_TRY(launch_status(
      jb::launch_cols(f->dtype, f->ax[0], 1, 1, inner0, c, s, 1, dim, nullptr, f->n[1], m, st),
      "fft cols axis0"));
  if (dim == 3)
    JB_TRY(launch_status(jb::launch_cols(f->dtype, f->ax[1], 1, f->n[0], m, s, s, 1, dim,
                                         nullptr, f->n[1], m, st),
                         "fft cols axis1"));
  const jb::RealGeom g = fft_geom(f, r_strides);
  double N = 1;
  for (int d = 0; d < dim; ++d) N *= (double)f->n[d];
  JB_TRY(launch_status(jb::launch_rows_c2r(f->dtype, f->ax[dim - 1], 1, 1, s, r, g, 1.0 / N,
                                           nullptr, nullptr, st),
                       "fft rows_c2r"));
  return JB_OK;
}

// ---------------------------------------------------------------------------
// continuous Green operator
// ---------------------------------------------------------------------------

int jb_green_continuous_matrix(int dim, double g, double nu, const double* k, double* out) {
  if (dim != 2 && dim != 3) return fail(JB_EINVAL, "dim must be 2 or 3");
  if (!k || !out) return fail(JB_EINVAL, "NULL argument");
  green_matrix_dim(dim, green_aux(g, nu), k, out);
  return JB_OK;
}

int jb_green_continuous_apply(int dim, double g, double nu, const double* k, const double* x,
                              double* y) {
  if (dim != 2 && dim != 3) return fail(JB_EINVAL, "dim must be 2 or 3");
  if (!k || !x || !y) return fail(JB_EINVAL, "NULL argument");
  double m[36];
  green_matrix_dim(dim, green_aux(g, nu), k, m);
  const int S = dim == 2 ? 3 : 6;
  double xv[6];
  for (int i = 0; i < S; ++i) xv[i] = x[i];
  for (int i = 0; i < S; ++i) {
    double s = m[i * S] * xv[0];
    for (int j = 1; j < S; ++j) s = s + m[i * S + j] * xv[j];
    y[i] = s;
  }
  return JB_OK;
}

int jb_isotropic_apply(int dim, double sph, double dev, const double* x, double* y) {
  if (dim != 2 && dim != 3) return fail(JB_EINVAL, "dim must be 2 or 3");
  if (!x || !y) return fail(JB_EINVAL, "NULL argument");
  const double tr = (sph - dev) / (double)dim;  // operators.pyx:299
  if (dim == 2) {
    const double x0 = x[0], x1 = x[1], x2 = x[2];
    const double aux = tr * (x0 + x1);
    y[0] = aux + dev * x0;
    y[1] = aux + dev * x1;
    y[2] = dev * x2;
  } else {
    const double x0 = x[0], x1 = x[1], x2 = x[2], x3 = x[3], x4 = x[4], x5 = x[5];
    const double aux = tr * (x0 + x1 + x2);
    y[0] = aux + dev * x0;
    y[1] = aux + dev * x1;
    y[2] = aux + dev * x2;
    y[3] = dev * x3;
    y[4] = dev * x4;
    y[5] = dev * x5;
  }
  return JB_OK;
}

// ---------------------------------------------------------------------------
// discrete Green operators
// ---------------------------------------------------------------------------

int jb_green_create(int dim, const int64_t* shape, double h, double g, double nu, int variant,
                    int dtype, jb_green** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  JB_TRY(check_shape(dim, shape, dtype));
  if (!(h > 0.)) return fail(JB_EINVAL, "h must be > 0 (was " + std::to_string(h) + ")");
  if (variant != JB_TRUNCATED && variant != JB_FILTERED && variant != JB_WILLOT)
    return fail(JB_EINVAL, "variant must be JB_TRUNCATED, JB_FILTERED or JB_WILLOT");
  jb_green* G = new jb_green();
  G->dim = dim;
  G->dtype = dtype;
  G->variant = variant;
  G->h = h;
  G->g = g;
  G->nu = nu;
  for (int d = 0; d < dim; ++d) {
    G->n[d] = shape[d];
    // green.pyx:140-141, 305-307
    G->s[d] = 2. * M_PI / (h * (double)shape[d]);
  }
  auto cleanup = [&](int r) {
    free_axes(G->ax);
    for (void* p : G->tables) cudaFree(p);
    delete G;
    return r;
  };
  for (int d = 0; d < dim; ++d) {
    int r = make_axis((int)shape[d], dtype, G->ax[d]);
    if (r != JB_OK) return cleanup(r);
  }
  G->gt.variant = variant;
  G->gt.inv2g = 0.5 / g;
  G->gt.c1 = 1.0 / (1.0 - nu);
  for (int d = 0; d < dim; ++d) {
    const int64_t n = shape[d];
    const double sd = G->s[d];
    if (variant == JB_TRUNCATED) {
      std::vector<double> kt(n);
      for (int64_t b = 0; b < n; ++b) kt[b] = 2 * b > n ? sd * (b - n) : sd * b;
      int r = upload_table(G, dtype, kt, &G->gt.kt[d]);
      if (r != JB_OK) return cleanup(r);
    } else if (variant == JB_WILLOT) {
      // sin and cos of phi = 0.5 * s * h * b (green.pyx:983-989, 1001-1013)
      std::vector<double> sn(n), cs(n);
      for (int64_t b = 0; b < n; ++b) {
        const double phi = 0.5 * sd * h * (double)b;
        sn[b] = sin(phi);
        cs[b] = cos(phi);
      }
      int r = upload_table(G, dtype, sn, &G->gt.kn[d]);
      if (r == JB_OK) r = upload_table(G, dtype, cs, &G->gt.kp[d]);
      if (r != JB_OK) return cleanup(r);
    } else {
      std::vector<double> kn(n), kp(n), wn(n), wp(n);
      for (int64_t b = 0; b < n; ++b) {
        // green.pyx:616-648 / 738-808
        double k = sd * (b - n);
        double w = cos(0.25 * h * k);
        w *= w;
        kn[b] = k;
        wn[b] = w;
        k = sd * b;
        w = cos(0.25 * h * k);
        w *= w;
        kp[b] = k;
        wp[b] = w;
      }
      int r = upload_table(G, dtype, kn, &G->gt.kn[d]);
      if (r == JB_OK) r = upload_table(G, dtype, kp, &G->gt.kp[d]);
      if (r == JB_OK) r = upload_table(G, dtype, wn, &G->gt.wn[d]);
      if (r == JB_OK) r = upload_table(G, dtype, wp, &G->gt.wp[d]);
      if (r != JB_OK) return cleanup(r);
    }
  }
  *out = G;
  return JB_OK;
}

int jb_green_destroy(jb_green* G) {
  if (!G) return JB_OK;
  free_axes(G->ax);
  for (void* p : G->tables) cudaFree(p);
  if (G->spec.p) cudaFree(G->spec.p);
  if (G->bidx.p) cudaFree(G->bidx.p);
  if (G->mnbuf.p) cudaFree(G->mnbuf.p);
  delete G;
  return JB_OK;
}

int jb_green_set_tuning(jb_green* G, const int* v, int count) {
  if (!G || !v) return fail(JB_EINVAL, "NULL argument");
  if (count != 6 && count != 7) return fail(JB_EINVAL, "tuning takes 6 or 7 values");
  if (count == 7 && (v[6] < 0 || v[6] > 2))
    return fail(JB_EINVAL, "contraction mode must be 0 (rule), 1 (table) or 2 (on the fly)");
  const int C = G->dim == 2 ? 3 : 6;
  if (v[0] < 0 || v[0] > 128 || v[3] < 0 || v[3] > 128 || (v[3] % C) != 0)
    return fail(JB_EINVAL, "tile widths must be in [0, 128], the Green one a multiple of s");
  for (int k : {v[1], v[4]})
    if (k != 0 && k != 2 && k != 3) return fail(JB_EINVAL, "input tiles must be 0, 2 or 3");
  if (v[5] < 0 || v[5] > 3)
    return fail(JB_EINVAL,
                "Green compile-time value must be 0, 1, 2 (in place) or 3 (register tiles)");
  G->tune_plain.w = v[0];
  G->tune_plain.nbuf = v[1];
  G->tune_plain.ct = v[2] != 0;
  G->tune_green.w = v[3];
  G->tune_green.nbuf = v[4];
  G->tune_green.ct = v[5];
  if (count == 7) G->tune_table = v[6];
  return JB_OK;
}

int jb_green_get_tuning(jb_green* G, int* v, int count) {
  if (!G || !v) return fail(JB_EINVAL, "NULL argument");
  if (count != 6 && count != 7) return fail(JB_EINVAL, "tuning takes 6 or 7 values");
  if (count == 7) v[6] = G->tune_table;
  v[0] = G->tune_plain.w;
  v[1] = G->tune_plain.nbuf;
  v[2] = G->tune_plain.ct;
  v[3] = G->tune_green.w;
  v[4] = G->tune_green.nbuf;
  v[5] = G->tune_green.ct;
  return JB_OK;
}

int jb_green_apply(jb_green* G, const void* x, void* y, int64_t batch, void* stream) {
  if (!G || !x || !y) return fail(JB_EINVAL, "NULL argument");
  if (batch < 1) return fail(JB_EINVAL, "batch must be >= 1");
  const size_t bytes = (size_t)batch * spec_elems(G) * 2 * real_size(G->dtype);
  JB_TRY(ensure_buf(G->spec, bytes));
  return green_passes(G, x, y, batch, G->spec.p, nullptr, nullptr, nullptr,
                      as_stream(stream));
}

static int check_b(const jb_green* G, const int32_t* b) {
  if (!b) return fail(JB_EINVAL, "b must not be NULL");
  for (int d = 0; d < G->dim; ++d)
    if (b[d] < 0 || b[d] >= G->n[d])
      return fail(JB_EINVAL, "index must be >= 0 and < " + std::to_string(G->n[d]) +
                                 " (was " + std::to_string(b[d]) + ")");
  return JB_OK;
}

int jb_green_matrix(jb_green* G, const int32_t* b, double* out) {
  if (!G || !out) return fail(JB_EINVAL, "NULL argument");
  JB_TRY(check_b(G, b));
  const int dim = G->dim;
  const int S = dim == 2 ? 3 : 6;
  const GreenAux aux = green_aux(G->g, G->nu);
  if (G->variant == JB_TRUNCATED) {
    double k[3];
    for (int d = 0; d < dim; ++d) {
      const int64_t n = G->n[d];
      k[d] = 2 * (int64_t)b[d] > n ? G->s[d] * (b[d] - n) : G->s[d] * b[d];
    }
    green_matrix_dim(dim, aux, k, out);
    return JB_OK;
  }
  if (G->variant == JB_WILLOT) {
    // green.pyx:983-989 (2D), 1001-1016 (3D), products left to right
    double c[3], sn[3], k[3];
    for (int d = 0; d < dim; ++d) {
      const double phi = 0.5 * G->s[d] * G->h * b[d];
      c[d] = cos(phi);
      sn[d] = sin(phi);
    }
    if (dim == 2) {
      k[0] = sn[0] * c[1];
      k[1] = c[0] * sn[1];
    } else {
      k[0] = sn[0] * c[1] * c[2];
      k[1] = c[0] * sn[1] * c[2];
      k[2] = c[0] * c[1] * sn[2];
    }
    green_matrix_dim(dim, aux, k, out);
    return JB_OK;
  }
  // filtered: aliases in the reference's order (all negative first, last
  // axis fastest), weights multiplied axis by axis, terms summed left to
  // right (green.pyx:609-670, 732-910)
  double kk[3][2], ww[3][2];
  for (int d = 0; d < dim; ++d) {
    const int64_t n = G->n[d];
    double k = G->s[d] * (b[d] - n);
    double w = cos(0.25 * G->h * k);
    w *= w;
    kk[d][0] = k;
    ww[d][0] = w;
    k = G->s[d] * b[d];
    w = cos(0.25 * G->h * k);
    w *= w;
    kk[d][1] = k;
    ww[d][1] = w;
  }
  double acc[36], term[36];
  const int na = 1 << dim;
  for (int a = 0; a < na; ++a) {
    double k[3];
    double w = 1.0;
    for (int d = 0; d < dim; ++d) {
      const int c = (a >> (dim - 1 - d)) & 1;
      k[d] = kk[d][c];
      w = d == 0 ? ww[d][c] : w * ww[d][c];
    }
    green_matrix_dim(dim, aux, k, term);
    for (int i = 0; i < S * S; ++i) acc[i] = a == 0 ? w * term[i] : acc[i] + w * term[i];
  }
  std::memcpy(out, acc, sizeof(double) * S * S);
  return JB_OK;
}

int jb_green_apply_by_freq(jb_green* G, const int32_t* b, const double* tau, double* eta) {
  if (!G || !tau || !eta) return fail(JB_EINVAL, "NULL argument");
  double m[36];
  JB_TRY(jb_green_matrix(G, b, m));
  const int S = G->dim == 2 ? 3 : 6;
  double x[6];
  for (int i = 0; i < S; ++i) x[i] = tau[i];
  for (int i = 0; i < S; ++i) {
    // row i of the symmetric matrix times x, summed left to right like the
    // reference's explicit expressions (isotropic.pyx:186-193, 294-313)
    double s = m[i * S] * x[0];
    for (int j = 1; j < S; ++j) s = s + m[i * S + j] * x[j];
    eta[i] = s;
  }
  return JB_OK;
}

int jb_green_apply_by_freq_device(jb_green* G, int64_t count, const int32_t* b, const void* tau,
                                  void* eta, void* stream) {
  if (!G || !b || !tau || !eta) return fail(JB_EINVAL, "NULL argument");
  if (count < 0) return fail(JB_EINVAL, "count must be >= 0");
  if (count == 0) return JB_OK;
  return launch_status(jb::launch_green_by_freq(G->dtype, G->dim, G->gt, count, b, tau, eta,
                                                as_stream(stream)),
                       "green_by_freq");
}

// ---------------------------------------------------------------------------
// local operators
// ---------------------------------------------------------------------------

int jb_local_create(int dim, const int64_t* shape, int nphase, const double* sph,
                    const double* dev, const void* phase, int index_bytes, int dtype,
                    jb_local** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (dim != 2 && dim != 3) return fail(JB_EINVAL, "dim must be 2 or 3");
  if (dtype != F64 && dtype != F32) return fail(JB_EINVAL, "dtype must be JB_F64 or JB_F32");
  if (nphase < 1) return fail(JB_EINVAL, "nphase must be >= 1");
  if (index_bytes != 0 && index_bytes != 1 && index_bytes != 4)
    return fail(JB_EINVAL, "index_bytes must be 0 (per-voxel field), 1 or 4");
  if (index_bytes == 1 && nphase > 256) return fail(JB_EINVAL, "uint8 phase map allows 256 phases");
  if (!sph || !dev || (index_bytes != 0 && !phase)) return fail(JB_EINVAL, "NULL argument");
  jb_local* L = new jb_local();
  L->dim = dim;
  L->dtype = dtype;
  L->nphase = nphase;
  L->index_bytes = index_bytes;
  L->nvox = 1;
  for (int d = 0; d < dim; ++d) {
    if (shape[d] <= 0) {
      delete L;
      return fail(JB_EINVAL, "shape must be > 0");
    }
    L->n[d] = shape[d];
    L->nvox *= shape[d];
  }
  if (index_bytes == 0 && (int64_t)nphase != L->nvox) {
    delete L;
    return fail(JB_EINVAL, "a per-voxel field needs nphase equal to the voxel count");
  }
  std::vector<double> tab(2 * (size_t)nphase);
  for (int p = 0; p < nphase; ++p) {
    tab[2 * p] = (sph[p] - dev[p]) / (double)dim;  // operators.pyx:299
    tab[2 * p + 1] = dev[p];
  }
  const size_t rs = real_size(dtype);
  int r = dev_alloc(&L->table, tab.size() * rs);
  if (r == JB_OK && index_bytes != 0) r = dev_alloc(&L->phase, (size_t)L->nvox * index_bytes);
  if (r != JB_OK) {
    if (L->table) cudaFree(L->table);
    delete L;
    return r;
  }
  cudaError_t e;
  if (dtype == F64) {
    e = cudaMemcpy(L->table, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice);
  } else {
    std::vector<float> f(tab.begin(), tab.end());
    e = cudaMemcpy(L->table, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && index_bytes != 0)
    e = cudaMemcpy(L->phase, phase, (size_t)L->nvox * index_bytes, cudaMemcpyDefault);
  if (e != cudaSuccess) {
    cudaFree(L->table);
    cudaFree(L->phase);
    delete L;
    return fail(JB_ECUDA, std::string("jb_local_create: ") + cudaGetErrorString(e));
  }
  *out = L;
  return JB_OK;
}

int jb_local_create_matrix(int dim, const int64_t* shape, int nphase, const double* mats,
                           const void* phase, int index_bytes, int dtype, jb_local** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (dim != 2 && dim != 3) return fail(JB_EINVAL, "dim must be 2 or 3");
  if (dtype != F64 && dtype != F32) return fail(JB_EINVAL, "dtype must be JB_F64 or JB_F32");
  if (nphase < 1) return fail(JB_EINVAL, "nphase must be >= 1");
  if (index_bytes != 0 && index_bytes != 1 && index_bytes != 4)
    return fail(JB_EINVAL, "index_bytes must be 0 (per-voxel field), 1 or 4");
  if (index_bytes == 1 && nphase > 256) return fail(JB_EINVAL, "uint8 phase map allows 256 phases");
  if (!mats || (index_bytes != 0 && !phase)) return fail(JB_EINVAL, "NULL argument");
  jb_local* L = new jb_local();
  L->dim = dim;
  L->dtype = dtype;
  L->nphase = nphase;
  L->index_bytes = index_bytes;
  L->kind = 1;
  L->nvox = 1;
  for (int d = 0; d < dim; ++d) {
    if (shape[d] <= 0) {
      delete L;
      return fail(JB_EINVAL, "shape must be > 0");
    }
    L->n[d] = shape[d];
    L->nvox *= shape[d];
  }
  if (index_bytes == 0 && (int64_t)nphase != L->nvox) {
    delete L;
    return fail(JB_EINVAL, "a per-voxel field needs nphase equal to the voxel count");
  }
  const int S = dim == 2 ? 3 : 6;
  const size_t count = (size_t)nphase * S * S;
  const size_t rs = real_size(dtype);
  int r = dev_alloc(&L->table, count * rs);
  if (r == JB_OK && index_bytes != 0) r = dev_alloc(&L->phase, (size_t)L->nvox * index_bytes);
  if (r != JB_OK) {
    if (L->table) cudaFree(L->table);
    delete L;
    return r;
  }
  cudaError_t e;
  if (dtype == F64) {
    e = cudaMemcpy(L->table, mats, count * 8, cudaMemcpyHostToDevice);
  } else {
    std::vector<float> f(mats, mats + count);
    e = cudaMemcpy(L->table, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && index_bytes != 0)
    e = cudaMemcpy(L->phase, phase, (size_t)L->nvox * index_bytes, cudaMemcpyDefault);
  if (e != cudaSuccess) {
    cudaFree(L->table);
    cudaFree(L->phase);
    delete L;
    return fail(JB_ECUDA, std::string("jb_local_create_matrix: ") + cudaGetErrorString(e));
  }
  *out = L;
  return JB_OK;
}

int jb_local_destroy(jb_local* L) {
  if (!L) return JB_OK;
  cudaFree(L->table);
  cudaFree(L->phase);
  delete L;
  return JB_OK;
}

static jb::LocalDesc local_desc(const jb_local* L) {
  jb::LocalDesc d;
  d.phase = L->phase;
  d.index_bytes = L->index_bytes;
  d.table = L->table;
  d.nphase = L->nphase;
  d.dim = L->dim;
  d.kind = L->kind;
  return d;
}

int jb_local_apply(jb_local* L, const void* x, void* y, int64_t batch, void* stream) {
  if (!L || !x || !y) return fail(JB_EINVAL, "NULL argument");
  if (batch < 1) return fail(JB_EINVAL, "batch must be >= 1");
  const int C = L->dim == 2 ? 3 : 6;
  return launch_status(jb::launch_local(L->dtype, local_desc(L), C, (int)batch, L->nvox, x, y,
                                        as_stream(stream)),
                       "local");
}

int jb_block_linear_apply(int dtype, int64_t nvox, int osz, int isz, const void* a,
                          const void* x, void* y, int transpose, void* stream) {
  if (!a || !x || !y) return fail(JB_EINVAL, "NULL argument");
  if (dtype != F64 && dtype != F32) return fail(JB_EINVAL, "dtype must be JB_F64 or JB_F32");
  if (nvox < 0 || osz < 1 || isz < 1 || osz > 8 || isz > 8)
    return fail(JB_EINVAL, "block sizes must be in [1, 8]");
  if (nvox == 0) return JB_OK;
  return launch_status(jb::launch_block_linear(dtype, nvox, 1, osz, isz, a, x, y, transpose,
                                               as_stream(stream)),
                       "block_linear");
}

int jb_local_gradient(int dim, int dtype, int64_t nvox, int nload, const void* eps,
                      const void* zeta, double scale, double* out, void* stream) {
  if (!eps || !zeta || !out) return fail(JB_EINVAL, "NULL argument");
  if (dim != 2 && dim != 3) return fail(JB_EINVAL, "dim must be 2 or 3");
  if (dtype != F64 && dtype != F32) return fail(JB_EINVAL, "dtype must be JB_F64 or JB_F32");
  if (nvox < 0 || nload < 1) return fail(JB_EINVAL, "nvox must be >= 0 and nload >= 1");
  if (nvox == 0) return JB_OK;
  return launch_status(jb::launch_local_gradient(dtype, dim, nvox, nload, eps, zeta, scale, out,
                                                 as_stream(stream)),
                       "local_gradient");
}

// ---------------------------------------------------------------------------
// basic fixed-point scheme
// ---------------------------------------------------------------------------

int jb_solver_create(jb_green* G, jb_local* L, int nload, jb_solver** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (!G || !L) return fail(JB_EINVAL, "NULL argument");
  if (nload < 1 || nload > 65535) return fail(JB_EINVAL, "nload must be in [1, 65535]");
  if (G->dim != L->dim || G->dtype != L->dtype)
    return fail(JB_EINVAL, "green and local operators differ in dim or dtype");
  for (int d = 0; d < G->dim; ++d)
    if (G->n[d] != L->n[d]) return fail(JB_EINVAL, "green and local operators differ in shape");
  jb_solver* S = new jb_solver();
  S->green = G;
  S->local = L;
  S->L = nload;
  const int C = G->dim == 2 ? 3 : 6;
  int r = ensure_buf(S->spec, (size_t)nload * spec_elems(G) * 2 * real_size(G->dtype));
  if (r == JB_OK) r = ensure_buf(S->E, sizeof(double) * nload * C);
  if (r == JB_OK) r = ensure_buf(S->res, sizeof(double) * nload);
  if (r == JB_OK) r = ensure_buf(S->mean, sizeof(double) * nload * C);
  if (r == JB_OK) r = ensure_buf(S->normd, sizeof(double) * nload);
  // partials: rows_c2r grid (<= rows) and local_sum grid (<= 1024 per comp)
  const int64_t rows = G->dim == 2 ? G->n[0] : G->n[0] * G->n[1];
  const int64_t np = std::max<int64_t>(rows, 1024 * C);
  if (r == JB_OK) r = ensure_buf(S->partials, sizeof(double) * nload * np);
  if (r != JB_OK) {
    jb_solver_destroy(S);
    return r;
  }
  *out = S;
  return JB_OK;
}

int jb_solver_destroy(jb_solver* S) {
  if (!S) return JB_OK;
  S->rec.release();
  for (DeviceBuf* b : {&S->spec, &S->partials, &S->E, &S->res, &S->mean, &S->normd})
    if (b->p) cudaFree(b->p);
  delete S;
  return JB_OK;
}

int jb_solver_set_load(jb_solver* S, const double* E) {
  if (!S || !E) return fail(JB_EINVAL, "NULL argument");
  const int C = S->green->dim == 2 ? 3 : 6;
  double N = 1;
  for (int d = 0; d < S->green->dim; ++d) N *= (double)S->green->n[d];
  S->Eh.assign(E, E + (size_t)S->L * C);
  S->norm.resize(S->L);
  for (int l = 0; l < S->L; ++l) {
    double s = 0;
    for (int c = 0; c < C; ++c) s += E[l * C + c] * E[l * C + c];
    if (!(s > 0)) return fail(JB_EINVAL, "macroscopic strain must be nonzero");
    S->norm[l] = 1.0 / std::sqrt(N) / std::sqrt(s);  // square_basic.py:86
  }
  JB_CUDA(cudaMemcpy(S->E.p, E, sizeof(double) * S->L * C, cudaMemcpyHostToDevice));
  JB_CUDA(cudaMemcpy(S->normd.p, S->norm.data(), sizeof(double) * S->L, cudaMemcpyHostToDevice));
  S->load_set = true;
  return JB_OK;
}

int jb_solver_step(jb_solver* S, void* eps, double* res_dev, void* stream) {
  if (!S || !eps) return fail(JB_EINVAL, "NULL argument");
  if (!S->load_set) return fail(JB_ESTATE, "jb_solver_set_load must be called first");
  cudaStream_t st = as_stream(stream);
  jb::LocalDesc loc = local_desc(S->local);
  jb::UpdateDesc upd;
  upd.eps = eps;
  upd.E = static_cast<const double*>(S->E.p);
  upd.partials = static_cast<double*>(S->partials.p);
  int nb = 0;
  PassRecorder* rec = nullptr;
  if (S->rec.active && S->rec.steps < S->rec.max_steps) {
    rec = &S->rec;
    ++S->rec.steps;
  }
  JB_TRY(green_passes(S->green, eps, eps, S->L, S->spec.p, &loc, &upd, &nb, st, rec));
  if (res_dev) {
    JB_TRY(launch_status(jb::launch_reduce_rows(static_cast<const double*>(S->partials.p), S->L,
                                                nb, res_dev, 1.0,
                                                static_cast<const double*>(S->normd.p), 1, st),
                         "reduce"));
  }
  if (rec) rec->mark(st);
  S->nb_rows = nb;
  return JB_OK;
}

static const char* kPass3[] = {"rows_r2c_local", "cols_fwd_axis1", "cols_green_axis0",
                               "cols_inv_axis1", "rows_c2r_update", "reduce_residual"};
static const char* kPass2[] = {"rows_r2c_local", "cols_green_axis0", "rows_c2r_update",
                               "reduce_residual"};

int jb_solver_timing_begin(jb_solver* S, int max_steps) {
  if (!S) return fail(JB_EINVAL, "NULL argument");
  if (max_steps < 1) return fail(JB_EINVAL, "max_steps must be >= 1");
  S->rec.release();
  S->rec.npass = S->green->dim == 3 ? 6 : 4;
  S->rec.max_steps = max_steps;
  S->rec.steps = 0;
  S->rec.cursor = 0;
  S->rec.ev.resize((size_t)(S->rec.npass + 1) * max_steps);
  for (auto& e : S->rec.ev) JB_CUDA(cudaEventCreate(&e));
  S->rec.active = true;
  return JB_OK;
}

int jb_solver_timing_end(jb_solver* S, double* pass_ms, int* npass, int* nsteps) {
  if (!S || !pass_ms) return fail(JB_EINVAL, "NULL argument");
  PassRecorder& R = S->rec;
  if (!R.active) return fail(JB_ESTATE, "jb_solver_timing_begin was not called");
  const int P = R.npass;
  for (int i = 0; i < 8; ++i) pass_ms[i] = 0.0;
  const int done = (int)(R.cursor / (P + 1));
  if (R.cursor > 0) JB_CUDA(cudaEventSynchronize(R.ev[R.cursor - 1]));
  for (int s = 0; s < done; ++s)
    for (int p = 0; p < P; ++p) {
      float ms = 0.f;
      JB_CUDA(cudaEventElapsedTime(&ms, R.ev[(size_t)s * (P + 1) + p],
                                   R.ev[(size_t)s * (P + 1) + p + 1]));
      pass_ms[p] += ms;
    }
  if (npass) *npass = P;
  if (nsteps) *nsteps = done;
  R.release();
  return JB_OK;
}

const char* jb_solver_pass_name(jb_solver* S, int i) {
  if (!S || i < 0) return "";
  if (S->green->dim == 3) return i < 6 ? kPass3[i] : "";
  return i < 4 ? kPass2[i] : "";
}

int jb_solver_run(jb_solver* S, const double* E, void* eps, int init, int max_iter, double tol,
                  double* residuals, int* iters_out, double* mean_tau, int* status,
                  void* stream) {
  if (!S || !E || !eps) return fail(JB_EINVAL, "NULL argument");
  if (max_iter < 0) return fail(JB_EINVAL, "max_iter must be >= 0");
  JB_TRY(jb_solver_set_load(S, E));
  cudaStream_t st = as_stream(stream);
  const int C = S->green->dim == 2 ? 3 : 6;
  const int64_t nvox = S->local->nvox;
  if (init)
    JB_TRY(launch_status(jb::launch_fill_macro(S->green->dtype, C, S->L, nvox,
                                               static_cast<const double*>(S->E.p), eps, st),
                         "fill"));
  std::vector<double> r(S->L);
  Outcome out(S->L);
  unsigned fault = 0;
  int it = 0;
  for (; it < max_iter; ++it) {
    JB_TRY(jb_solver_step(S, eps, static_cast<double*>(S->res.p), st));
    JB_CUDA(cudaMemcpyAsync(r.data(), S->res.p, sizeof(double) * S->L, cudaMemcpyDeviceToHost,
                            st));
    JB_CUDA(jb::fetch_fault_async(&fault, st));
    JB_CUDA(cudaStreamSynchronize(st));
    JB_TRY(check_fault(fault, "jb_solver_run"));
    bool done = true;
    for (int l = 0; l < S->L; ++l) {
      if (residuals) residuals[(size_t)it * S->L + l] = r[l];
      if (!out.update(l, r[l], tol)) done = false;
    }
    if (done) {
      ++it;
      break;
    }
  }
  if (iters_out) *iters_out = it;
  out.write(tol, status);
  if (mean_tau) {
    int nb = 0;
    JB_TRY(launch_status(jb::launch_local_sum(S->green->dtype, local_desc(S->local), C, S->L,
                                              nvox, eps, static_cast<double*>(S->partials.p),
                                              &nb, st),
                         "local_sum"));
    JB_TRY(launch_status(jb::launch_reduce_cols(static_cast<const double*>(S->partials.p), S->L,
                                                C, nb, static_cast<double*>(S->mean.p),
                                                1.0 / (double)nvox, st),
                         "reduce"));
    JB_CUDA(cudaMemcpyAsync(mean_tau, S->mean.p, sizeof(double) * S->L * C,
                            cudaMemcpyDeviceToHost, st));
  }
  JB_CUDA(cudaStreamSynchronize(st));
  return JB_OK;
}

}  // extern "C"

// ===========================================================================
// Restarted GMRES(m) on the Lippmann-Schwinger equation
// ===========================================================================
//
// The reference's own examples solve (I + Gamma0 (C - C0)) eps = E with
// scipy's GMRES over a LinearOperator whose matvec is x + Gamma0[(C-C0):x]
// (examples/square_inclusion_scipy.py:52-59, 88).  Here the operator is one
// fused pass sequence (rhs epilogue: out = in + Gamma0[(C - C0):in]) and the
// Krylov vectors stay on the device, one Krylov space per load case.  The
// Arnoldi process runs on K = Gamma0 (C - C0) (same Krylov spaces as A,
// H_A = H_K + I).  Its basis is orthogonalised by classical Gram-Schmidt (each projection
// sweep one pass of dot products and one of updates, up to 8 basis vectors
// streamed per launch, |w|^2 computed with the former and |w'|^2 with the
// latter) and swept a second time only when the first sweep cancelled more
// than half of |w|^2 (|w'| < |w| / sqrt(2), the "twice is enough" test of
// Kahan and Parlett); the small Hessenberg least-squares problems (Givens
// rotations) are solved on the host.  Residuals are relative to
// sqrt(N) |E_l|, the normalisation of the basic scheme's residual
// (square_basic.py:86): for the basic scheme's iterate eps_k, E - A eps_k is
// exactly eps_{k+1} - eps_k.  A load case stops taking part once its
// residual estimate reaches tol (its later basis vectors get zero weight).
struct jb_gmres_s {
  jb_green* green = nullptr;
  jb_local* local = nullptr;
  int L = 1;
  int m = 20;
  DeviceBuf spec, V, partials, E, h, sq, y, mean;
};

extern "C" int jb_gmres_create(jb_green* G, jb_local* Lo, int nload, int restart,
                               jb_gmres** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (!G || !Lo) return fail(JB_EINVAL, "NULL argument");
  if (G->dtype != F64 || Lo->dtype != F64)
    return fail(JB_EINVAL, "jb_gmres_create needs FP64 operators");
  if (nload < 1 || nload > 65535) return fail(JB_EINVAL, "nload must be in [1, 65535]");
  if (restart < 1 || restart > 1000) return fail(JB_EINVAL, "restart must be in [1, 1000]");
  if (G->dim != Lo->dim) return fail(JB_EINVAL, "green and local operators differ in dim");
  for (int d = 0; d < G->dim; ++d)
    if (G->n[d] != Lo->n[d]) return fail(JB_EINVAL, "green and local operators differ in shape");
  jb_gmres* S = new jb_gmres();
  S->green = G;
  S->local = Lo;
  S->L = nload;
  S->m = restart;
  const int C = G->dim == 2 ? 3 : 6;
  const int64_t nel = Lo->nvox * C;
  const int ch = jb::gmres_chunk();
  const int64_t nb = jb::krylov_blocks(nel, nload);
  int r = ensure_buf(S->spec, (size_t)nload * spec_elems(G) * 2 * sizeof(double));
  if (r == JB_OK)
    r = ensure_buf(S->V, sizeof(double) * (size_t)(restart + 1) * (size_t)nload * (size_t)nel);
  if (r == JB_OK)
    r = ensure_buf(S->partials,
                   sizeof(double) * std::max<size_t>((size_t)nload * ch * nb,
                                                     (size_t)nload * std::max<int64_t>(
                                                         G->dim == 2 ? G->n[0]
                                                                     : G->n[0] * G->n[1],
                                                         1024 * C)));
  if (r == JB_OK) r = ensure_buf(S->E, sizeof(double) * nload * C);
  if (r == JB_OK) r = ensure_buf(S->h, sizeof(double) * nload * 2 * (restart + 1));
  if (r == JB_OK) r = ensure_buf(S->sq, sizeof(double) * nload);
  if (r == JB_OK) r = ensure_buf(S->y, sizeof(double) * nload * restart);
  if (r == JB_OK) r = ensure_buf(S->mean, sizeof(double) * nload * C);
  if (r != JB_OK) {
    jb_gmres_destroy(S);
    return r;
  }
  *out = S;
  return JB_OK;
}

extern "C" int jb_gmres_destroy(jb_gmres* S) {
  if (!S) return JB_OK;
  for (DeviceBuf* b : {&S->spec, &S->V, &S->partials, &S->E, &S->h, &S->sq, &S->y, &S->mean})
    if (b->p) cudaFree(b->p);
  delete S;
  return JB_OK;
}

namespace {

// Givens rotation (c, s) with c a + s b = r, -s a + c b = 0
void givens(double a, double b, double& c, double& s) {
  if (b == 0.0) {
    c = 1.0;
    s = 0.0;
  } else if (std::fabs(b) > std::fabs(a)) {
    const double t = a / b, u = std::sqrt(1.0 + t * t);
    s = 1.0 / u;
    c = t * s;
  } else {
    const double t = b / a, u = std::sqrt(1.0 + t * t);
    c = 1.0 / u;
    s = t * c;
  }
}

}  // namespace

extern "C" int jb_gmres_run(jb_gmres* S, const double* E, void* eps, int init, int max_iter,
                            double tol, double* residuals, int* iters_out,
                            double* final_residuals, double* mean_tau, int* status,
                            void* stream) {
  if (!S || !E || !eps) return fail(JB_EINVAL, "NULL argument");
  if (max_iter < 0) return fail(JB_EINVAL, "max_iter must be >= 0");
  if (!(tol >= 0.0)) return fail(JB_EINVAL, "tol must be >= 0");
  cudaStream_t st = as_stream(stream);
  jb_green* G = S->green;
  const int L = S->L, m = S->m, C = G->dim == 2 ? 3 : 6;
  const int64_t nvox = S->local->nvox, nel = nvox * C, vs = (int64_t)L * nel;
  const int ch = jb::gmres_chunk();
  const int ldh = 2 * (m + 1);  // per load case: two projection sweeps of up to m + 1
  double N = 1;
  for (int d = 0; d < G->dim; ++d) N *= (double)G->n[d];
  std::vector<double> bnorm(L);
  for (int l = 0; l < L; ++l) {
    double t = 0;
    for (int c = 0; c < C; ++c) t += E[l * C + c] * E[l * C + c];
    if (!(t > 0)) return fail(JB_EINVAL, "macroscopic strain must be nonzero");
    bnorm[l] = std::sqrt(N) * std::sqrt(t);
  }
  double* Ed = static_cast<double*>(S->E.p);
  double* V = static_cast<double*>(S->V.p);
  double* hd = static_cast<double*>(S->h.p);
  double* sqd = static_cast<double*>(S->sq.p);
  double* yd = static_cast<double*>(S->y.p);
  double* part = static_cast<double*>(S->partials.p);
  double* x = static_cast<double*>(eps);
  JB_CUDA(cudaMemcpyAsync(Ed, E, sizeof(double) * L * C, cudaMemcpyHostToDevice, st));
  if (init)
    JB_TRY(launch_status(jb::launch_fill_macro(F64, C, L, nvox, Ed, eps, st), "fill"));
  std::vector<double> H((size_t)L * (m + 1) * m), cs((size_t)L * m), sn((size_t)L * m),
      g((size_t)L * (m + 1)), hh((size_t)L * ldh), sq(L), beta(L), rel(L), yh((size_t)L * m);
  jb::LocalDesc loc = local_desc(S->local);
  auto apply = [&](const double* in, double* o) {  // o = in + Gamma0[(C - C0):in]
    jb::UpdateDesc u;
    u.mode = 4;
    u.eps = o;
    u.rhs = in;
    return green_passes(G, in, o, L, S->spec.p, &loc, &u, nullptr, st);
  };
  // the Arnoldi process runs on K = Gamma0 (C - C0), whose Krylov spaces are
  // those of A = I + K (H_A = H_K + I): w = K v has no component along v from
  // the identity for the projection to cancel
  auto applyK = [&](const double* in, double* o) {
    return green_passes(G, in, o, L, S->spec.p, &loc, nullptr, nullptr, st);
  };
  auto norm2 = [&](const double* w) {  // sq[l] = w . w on the device
    return launch_status(jb::launch_gmres_dots(nel, L, w, w, 0, 0, 1, part, sqd, 1, 0, st),
                         "gmres_dots");
  };
  // one sweep q on w = V_{j+1}: h[l][q (m+1) + i] = V_i . w for i <= j (sweep 0
  // also w . w at i = j + 1), then w -= sum_{i <= j} h_i V_i and sq = |w|^2
  unsigned fault = 0;
  auto sweep = [&](int j, int q) {
    double* w = V + (int64_t)(j + 1) * vs;
    const int nd = q == 0 ? j + 2 : j + 1;
    for (int i0 = 0; i0 < nd; i0 += ch) {
      const int cnt = std::min(ch, nd - i0);
      JB_TRY(launch_status(
          jb::launch_gmres_dots(nel, L, w, V, vs, i0, cnt, part, hd, ldh, q * (m + 1) + i0, st),
          "gmres_dots"));
    }
    for (int i0 = 0; i0 <= j; i0 += ch) {
      const int cnt = std::min(ch, j + 1 - i0);
      const bool last = i0 + cnt > j;
      JB_TRY(launch_status(jb::launch_gmres_axpys(nel, L, w, V, vs, i0, cnt, hd, ldh,
                                                  q * (m + 1) + i0, -1.0, last ? part : nullptr,
                                                  last ? sqd : nullptr, st),
                           "gmres_axpys"));
    }
    JB_CUDA(cudaMemcpyAsync(hh.data() + (size_t)0, hd, sizeof(double) * L * ldh,
                            cudaMemcpyDeviceToHost, st));
    JB_CUDA(cudaMemcpyAsync(sq.data(), sqd, sizeof(double) * L, cudaMemcpyDeviceToHost, st));
    JB_CUDA(jb::fetch_fault_async(&fault, st));
    JB_CUDA(cudaStreamSynchronize(st));
    return check_fault(fault, "jb_gmres_run");
  };
  std::vector<int> active(L), kuse(L);
  Outcome out(L);
  int it = 0;
  for (;;) {
    // true residual r = E - A x into V_0
    JB_TRY(apply(x, V));
    JB_TRY(launch_status(jb::launch_gmres_resid(nvox, C, L, Ed, V, V, st), "gmres_resid"));
    JB_TRY(norm2(V));
    JB_CUDA(cudaMemcpyAsync(sq.data(), sqd, sizeof(double) * L, cudaMemcpyDeviceToHost, st));
    JB_CUDA(jb::fetch_fault_async(&fault, st));
    JB_CUDA(cudaStreamSynchronize(st));
    JB_TRY(check_fault(fault, "jb_gmres_run"));
    bool done = true;
    for (int l = 0; l < L; ++l) {
      beta[l] = std::sqrt(sq[l]);
      rel[l] = beta[l] / bnorm[l];
      if (!out.update(l, rel[l], tol)) done = false;
    }
    if (final_residuals)
      for (int l = 0; l < L; ++l) final_residuals[l] = rel[l];
    if (done || it >= max_iter) break;
    JB_TRY(launch_status(jb::launch_gmres_scale(nel, L, V, sqd, st), "gmres_scale"));
    std::fill(g.begin(), g.end(), 0.0);
    for (int l = 0; l < L; ++l) {
      g[(size_t)l * (m + 1)] = beta[l];
      active[l] = (rel[l] <= tol || !(beta[l] > 0.0) || !std::isfinite(beta[l]) ||
                   out.stopped[l])
                      ? 0
                      : 1;
      kuse[l] = 0;
    }
    int j = 0;
    for (; j < m && it < max_iter; ++j, ++it) {
      double* w = V + (int64_t)(j + 1) * vs;
      JB_TRY(applyK(V + (int64_t)j * vs, w));
      JB_TRY(sweep(j, 0));
      bool again = false;
      for (int l = 0; l < L; ++l)
        if (active[l] && sq[l] < 0.5 * hh[(size_t)l * ldh + j + 1]) again = true;
      if (again) {
        JB_TRY(sweep(j, 1));
      } else {
        for (int l = 0; l < L; ++l)
          for (int i = 0; i <= j; ++i) hh[(size_t)l * ldh + (m + 1) + i] = 0.0;
      }
      JB_TRY(launch_status(jb::launch_gmres_scale(nel, L, w, sqd, st), "gmres_scale"));
      bool any = false;
      for (int l = 0; l < L; ++l) {
        double* Hl = &H[(size_t)l * (m + 1) * m];  // column-major (m + 1) x m
        double* gl = &g[(size_t)l * (m + 1)];
        if (!active[l]) {
          if (residuals) residuals[(size_t)it * L + l] = std::fabs(gl[kuse[l]]) / bnorm[l];
          continue;
        }
        double* col = Hl + (size_t)j * (m + 1);
        for (int i = 0; i <= j; ++i)
          col[i] = hh[(size_t)l * ldh + i] + hh[(size_t)l * ldh + (m + 1) + i];
        col[j] += 1.0;  // H_A = H_K + I
        const double hn = std::sqrt(sq[l]);
        col[j + 1] = hn;
        for (int i = 0; i < j; ++i) {  // earlier rotations
          const double a = col[i], b = col[i + 1];
          col[i] = cs[(size_t)l * m + i] * a + sn[(size_t)l * m + i] * b;
          col[i + 1] = -sn[(size_t)l * m + i] * a + cs[(size_t)l * m + i] * b;
        }
        double c, s;
        givens(col[j], col[j + 1], c, s);
        cs[(size_t)l * m + j] = c;
        sn[(size_t)l * m + j] = s;
        col[j] = c * col[j] + s * col[j + 1];
        col[j + 1] = 0.0;
        gl[j + 1] = -s * gl[j];
        gl[j] = c * gl[j];
        kuse[l] = j + 1;
        const double est = std::fabs(gl[j + 1]) / bnorm[l];
        if (residuals) residuals[(size_t)it * L + l] = est;
        if (!(est > tol) || !(hn > 0.0) || !std::isfinite(hn) || col[j] == 0.0)
          active[l] = 0;
        else
          any = true;
      }
      if (!any) {
        ++j;
        ++it;
        break;
      }
    }
    // x += V y, R y = g over each load case's kuse columns (back substitution)
    std::fill(yh.begin(), yh.end(), 0.0);
    int kmax = 0;
    for (int l = 0; l < L; ++l) {
      const int k = kuse[l];
      const double* Hl = &H[(size_t)l * (m + 1) * m];
      const double* gl = &g[(size_t)l * (m + 1)];
      double* yl = &yh[(size_t)l * m];
      for (int i = k - 1; i >= 0; --i) {
        double t = gl[i];
        for (int q = i + 1; q < k; ++q) t -= Hl[(size_t)q * (m + 1) + i] * yl[q];
        const double d = Hl[(size_t)i * (m + 1) + i];
        yl[i] = (d != 0.0 && std::isfinite(t / d)) ? t / d : 0.0;
      }
      kmax = std::max(kmax, k);
    }
    if (kmax == 0) break;  // no load case can make progress
    JB_CUDA(cudaMemcpyAsync(yd, yh.data(), sizeof(double) * L * m, cudaMemcpyHostToDevice, st));
    for (int i0 = 0; i0 < kmax; i0 += ch) {
      const int cnt = std::min(ch, kmax - i0);
      JB_TRY(launch_status(jb::launch_gmres_axpys(nel, L, x, V, vs, i0, cnt, yd, m, i0, 1.0,
                                                    nullptr, nullptr, st),
                           "gmres_axpys"));
    }
  }
  if (iters_out) *iters_out = it;
  out.write(tol, status);
  if (mean_tau) {
    int nb = 0;
    JB_TRY(launch_status(jb::launch_local_sum(F64, loc, C, L, nvox, eps,
                                              static_cast<double*>(S->partials.p), &nb, st),
                         "local_sum"));
    JB_TRY(launch_status(jb::launch_reduce_cols(static_cast<const double*>(S->partials.p), L, C,
                                                nb, static_cast<double*>(S->mean.p),
                                                1.0 / (double)nvox, st),
                         "reduce"));
    JB_CUDA(cudaMemcpyAsync(mean_tau, S->mean.p, sizeof(double) * L * C, cudaMemcpyDeviceToHost,
                            st));
  }
  JB_CUDA(cudaStreamSynchronize(st));
  return JB_OK;
}

// ===========================================================================
// Green operator application without any device allocation
// ===========================================================================
//
// For callers that cannot allocate device memory at all: code running under
// an allocator that owns the whole GPU (a memory pool sized at start-up), a
// host application that forbids cudaMalloc/cudaFree outside its set-up phase,
// or a plug-in whose host framework hands it only input and output buffers.
// jb_green_apply_noalloc needs no handle: the twiddle tables, the Green
// operator's k/weight tables and the spectral scratch all live in the one
// file-scope device array below (32 MiB, held by every GPU that loads this
// library until the process exits).
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress) and caches it per device, so
// make the first call on each device before any stream capture.  The cache
// does not survive a device reset (cudaDeviceReset) in the same process.
// Every call fills the twiddles and the k / weight tables on the device with
// one small kernel (no host copies), then runs the passes.  The array keeps
// the last call's contents; nothing in it needs to start at zero (every
// region is written before it is read within a call).  Calls share the
// array, so two calls that overlap on the GPU (different streams, or
// different host threads without ordering) race.
namespace {

constexpr size_t kNoAllocBytes = size_t(32) << 20;       // whole array
constexpr size_t kNoAllocTwOff = 0;                      // 3 x 64 KiB twiddles
constexpr size_t kNoAllocTwBytes = size_t(64) << 10;
constexpr size_t kNoAllocTabOff = size_t(192) << 10;     // 3 axes x 4 tables
constexpr size_t kNoAllocTabBytes = size_t(4096) * 8;    // per table
constexpr size_t kNoAllocSpecOff = size_t(1) << 20;      // spectral scratch
constexpr int kNoAllocMaxAxis = 4096;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

int noalloc_scratch(void** out) {
  int dev = -1;
  JB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(JB_EINVAL, "jb_green_apply_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(JB_ECUDA, std::string("jb_green_apply_noalloc: cudaGetSymbolAddress: ") +
                                cudaGetErrorString(e));
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return JB_OK;
}

// per-axis data of one allocation-free call, passed by value
struct NoallocAxes {
  int dim, variant;
  int n[3];
  double s[3];  // 2 pi / (h n_d), as the handle-based operator computes it
  double h;
};

// twiddles exp(-2 pi i t / n) and the per-axis k (truncated) or k-, k+, w-,
// w+ (filtered) tables of green.pyx:434-445 / 609-670, into the static array
__global__ void noalloc_fill_kernel(NoallocAxes a) {
  for (int d = 0; d < a.dim; ++d) {
    const int n = a.n[d];
    const double sd = a.s[d];
    double2* tw =
        reinterpret_cast<double2*>(g_noalloc_scratch + kNoAllocTwOff + d * kNoAllocTwBytes);
    double* tab[4];
    for (int i = 0; i < 4; ++i)
      tab[i] = reinterpret_cast<double*>(g_noalloc_scratch + kNoAllocTabOff +
                                         (size_t)(d * 4 + i) * kNoAllocTabBytes);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
      double sn, cs;
      sincospi(2.0 * (double)t / (double)n, &sn, &cs);
      tw[t] = make_double2(cs, -sn);
      if (a.variant == JB_TRUNCATED) {
        tab[0][t] = 2 * t > n ? sd * (double)(t - n) : sd * (double)t;
      } else {
        double k = sd * (double)(t - n);
        double w = cos(0.25 * a.h * k);
        tab[0][t] = k;
        tab[2][t] = w * w;
        k = sd * (double)t;
        w = cos(0.25 * a.h * k);
        tab[1][t] = k;
        tab[3][t] = w * w;
      }
    }
  }
}

// x / y must be memory of the current device, and the stream one of its
// streams: the kernels address this device's static array
int noalloc_check_device(const void* x, const void* y, cudaStream_t st) {
  int dev = -1;
  JB_CUDA(cudaGetDevice(&dev));
  for (const void* p : {x, y}) {
    cudaPointerAttributes at{};
    const cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(JB_EINVAL, "jb_green_apply_noalloc: x and y must be device memory");
    }
    if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) ||
        at.device != dev)
      return fail(JB_EINVAL, "jb_green_apply_noalloc: x and y must be memory of the current "
                             "device (" + std::to_string(dev) + ")");
  }
  if (st) {
    int sdev = -1;
    const cudaError_t e = cudaStreamGetDevice(st, &sdev);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(JB_EINVAL, "jb_green_apply_noalloc: invalid stream");
    }
    if (sdev != dev)
      return fail(JB_EINVAL, "jb_green_apply_noalloc: the stream belongs to device " +
                                 std::to_string(sdev) + ", not the current device " +
                                 std::to_string(dev));
  }
  return JB_OK;
}

}  // namespace

extern "C" int jb_green_apply_noalloc(int dim, const int64_t* shape, double h, double g,
                                      double nu, int variant, const double* x, double* y,
                                      void* stream) {
  if (!x || !y) return fail(JB_EINVAL, "NULL argument");
  JB_TRY(check_shape(dim, shape, F64));
  if (!(h > 0.)) return fail(JB_EINVAL, "h must be > 0 (was " + std::to_string(h) + ")");
  if (variant != JB_TRUNCATED && variant != JB_FILTERED)
    return fail(JB_EINVAL, "variant must be JB_TRUNCATED or JB_FILTERED");
  for (int d = 0; d < dim; ++d)
    if (shape[d] > kNoAllocMaxAxis)
      return fail(JB_EINVAL, "jb_green_apply_noalloc: axis longer than 4096");
  const int C = dim == 2 ? 3 : 6;
  const int64_t nlast = shape[dim - 1];
  const int64_t rows = dim == 2 ? shape[0] : shape[0] * shape[1];
  const size_t need = (size_t)rows * (nlast / 2 + 1) * C * 16;
  if (need > kNoAllocBytes - kNoAllocSpecOff)
    return fail(JB_EINVAL, "jb_green_apply_noalloc: this grid needs " + std::to_string(need) +
                               " bytes of spectral scratch; the static scratch holds " +
                               std::to_string(kNoAllocBytes - kNoAllocSpecOff) +
                               " (FP64: 2D up to about 1024 x 1024, 3D up to about 80^3)");
  cudaStream_t st = as_stream(stream);
  JB_TRY(noalloc_check_device(x, y, st));
  void* base = nullptr;
  JB_TRY(noalloc_scratch(&base));
  unsigned char* b8 = static_cast<unsigned char*>(base);

  // a stack-held operator description whose device pointers all point into
  // the static array (no handle, no allocation)
  jb_green G;
  G.use_table = false;  // evaluate the operator on the fly: nothing to allocate
  G.dim = dim;
  G.dtype = F64;
  G.variant = variant;
  G.h = h;
  G.g = g;
  G.nu = nu;
  G.gt.variant = variant;
  G.gt.inv2g = 0.5 / g;
  G.gt.c1 = 1.0 / (1.0 - nu);
  NoallocAxes ax{};
  ax.dim = dim;
  ax.variant = variant;
  ax.h = h;
  int nmax = 1;
  for (int d = 0; d < dim; ++d) {
    const int64_t n = shape[d];
    G.n[d] = n;
    G.s[d] = 2. * M_PI / (h * (double)n);
    factorize((int)n, G.ax[d].plan);
    G.ax[d].tw = b8 + kNoAllocTwOff + d * kNoAllocTwBytes;
    ax.n[d] = (int)n;
    ax.s[d] = G.s[d];
    nmax = std::max(nmax, (int)n);
    void** slots[4] = {variant == JB_TRUNCATED ? &G.gt.kt[d] : &G.gt.kn[d], &G.gt.kp[d],
                       &G.gt.wn[d], &G.gt.wp[d]};
    const int ntab = variant == JB_TRUNCATED ? 1 : 4;
    for (int i = 0; i < ntab; ++i)
      *slots[i] = b8 + kNoAllocTabOff + (size_t)(d * 4 + i) * kNoAllocTabBytes;
  }
  noalloc_fill_kernel<<<(nmax + 255) / 256, 256, 0, st>>>(ax);
  JB_TRY(launch_status(cudaGetLastError(), "noalloc_fill"));
  const int r = green_passes(&G, x, y, 1, b8 + kNoAllocSpecOff, nullptr, nullptr, nullptr, st);
  for (int d = 0; d < 3; ++d) G.ax[d].tw = nullptr;  // not owned
  return r;
}

// ===========================================================================
// mixed-precision basic scheme: FP32 bulk iterations, FP64 defect correction
// ===========================================================================

struct jb_mixed_s {
  jb_green* g64 = nullptr;
  jb_local* l64 = nullptr;
  jb_green* g32 = nullptr;
  jb_local* l32 = nullptr;
  int L = 1;
  int method = JB_INNER_BASIC;
  int idt = F32;  // precision of the inner (correction) operators and fields
  DeviceBuf spec, partials, E, res, normd, r32, d32, mean;
  DeviceBuf kr_rh, kr_p, kr_v, kr_s, kr_t, kr_r, kr_part, kr_state;  // BiCGSTAB
  std::vector<double> norm;
};

extern "C" int jb_mixed_create(jb_green* g64, jb_local* l64, jb_green* g32, jb_local* l32,
                               int nload, jb_mixed** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (!g64 || !l64 || !g32 || !l32) return fail(JB_EINVAL, "NULL argument");
  if (g64->dtype != F64 || l64->dtype != F64 || g32->dtype != l32->dtype)
    return fail(JB_EINVAL, "jb_mixed_create needs FP64 outer operators and inner operators "
                           "of one precision");
  if (nload < 1 || nload > 65535) return fail(JB_EINVAL, "nload must be in [1, 65535]");
  const int dim = g64->dim;
  if (g32->dim != dim || l64->dim != dim || l32->dim != dim)
    return fail(JB_EINVAL, "operators differ in dim");
  for (int d = 0; d < dim; ++d)
    if (g32->n[d] != g64->n[d] || l64->n[d] != g64->n[d] || l32->n[d] != g64->n[d])
      return fail(JB_EINVAL, "operators differ in shape");
  if (g32->variant != g64->variant || g32->g != g64->g || g32->nu != g64->nu ||
      g32->h != g64->h)
    return fail(JB_EINVAL, "FP32 and FP64 Green operators differ");
  jb_mixed* M = new jb_mixed();
  M->g64 = g64;
  M->l64 = l64;
  M->g32 = g32;
  M->l32 = l32;
  M->L = nload;
  M->idt = g32->dtype;
  const int C = dim == 2 ? 3 : 6;
  const int64_t nvox = l64->nvox;
  const int64_t rows = dim == 2 ? g64->n[0] : g64->n[0] * g64->n[1];
  int r = ensure_buf(M->spec, (size_t)nload * spec_elems(g64) * 16);
  if (r == JB_OK) r = ensure_buf(M->partials, sizeof(double) * nload *
                                                  std::max<int64_t>(rows, 1024 * C));
  if (r == JB_OK) r = ensure_buf(M->E, sizeof(double) * nload * C);
  if (r == JB_OK) r = ensure_buf(M->res, sizeof(double) * nload);
  if (r == JB_OK) r = ensure_buf(M->normd, sizeof(double) * nload);
  if (r == JB_OK) r = ensure_buf(M->mean, sizeof(double) * nload * C);
  if (r == JB_OK) r = ensure_buf(M->r32, real_size(M->idt) * nload * nvox * C);
  if (r == JB_OK) r = ensure_buf(M->d32, real_size(M->idt) * nload * nvox * C);
  if (r != JB_OK) {
    jb_mixed_destroy(M);
    return r;
  }
  *out = M;
  return JB_OK;
}

extern "C" int jb_mixed_set_method(jb_mixed* M, int method) {
  if (!M) return fail(JB_EINVAL, "NULL argument");
  if (method != JB_INNER_BASIC && method != JB_INNER_BICGSTAB &&
      method != JB_INNER_BICGSTAB_FIXED)
    return fail(JB_EINVAL,
                "method must be JB_INNER_BASIC, JB_INNER_BICGSTAB or JB_INNER_BICGSTAB_FIXED");
  M->method = method;
  return JB_OK;
}

extern "C" int jb_mixed_destroy(jb_mixed* M) {
  if (!M) return JB_OK;
  for (DeviceBuf* b : {&M->spec, &M->partials, &M->E, &M->res, &M->normd, &M->r32, &M->d32,
                       &M->mean, &M->kr_rh, &M->kr_p, &M->kr_v, &M->kr_s, &M->kr_t, &M->kr_r,
                       &M->kr_part, &M->kr_state})
    if (b->p) cudaFree(b->p);
  delete M;
  return JB_OK;
}

namespace {

// load E (host, L x C) for a mixed solver: device copy, residual
// normalisation 1/(sqrt(N) |E_l|), and eps = E when init
int mixed_set_load(jb_mixed* M, const double* E, void* eps, int init, cudaStream_t st) {
  const int dim = M->g64->dim;
  const int C = dim == 2 ? 3 : 6;
  const int L = M->L;
  double N = 1;
  for (int d = 0; d < dim; ++d) N *= (double)M->g64->n[d];
  M->norm.resize(L);
  for (int l = 0; l < L; ++l) {
    double s = 0;
    for (int c = 0; c < C; ++c) s += E[l * C + c] * E[l * C + c];
    if (!(s > 0)) return fail(JB_EINVAL, "macroscopic strain must be nonzero");
    M->norm[l] = 1.0 / std::sqrt(N) / std::sqrt(s);
  }
  JB_CUDA(cudaMemcpyAsync(M->E.p, E, sizeof(double) * L * C, cudaMemcpyHostToDevice, st));
  JB_CUDA(cudaMemcpyAsync(M->normd.p, M->norm.data(), sizeof(double) * L,
                          cudaMemcpyHostToDevice, st));
  if (init)
    JB_TRY(launch_status(jb::launch_fill_macro(F64, C, L, M->l64->nvox,
                                               static_cast<const double*>(M->E.p), eps, st),
                         "fill"));
  return JB_OK;
}

// FP64 residual pass: r32 = E - eps - Gamma0[(C - C0):eps] (in the inner
// precision), its normalised norms into res_out (device double[L])
int mixed_residual(jb_mixed* M, void* eps, double* res_out, cudaStream_t st) {
  jb::LocalDesc loc64 = local_desc(M->l64);
  if (M->idt == F64) {
    // all-FP64 form: A eps into r, r = E - A eps, |r|^2, then the normalised norm
    const int C = M->g64->dim == 2 ? 3 : 6;
    const int64_t nvox = M->l64->nvox;
    double* r = static_cast<double*>(M->r32.p);
    double* sq = static_cast<double*>(M->partials.p);
    jb::UpdateDesc u;
    u.mode = 4;  // r = eps + Gamma0[(C - C0):eps]
    u.eps = r;
    u.rhs = eps;
    JB_TRY(green_passes(M->g64, eps, r, M->L, M->spec.p, &loc64, &u, nullptr, st));
    JB_TRY(launch_status(jb::launch_gmres_resid(nvox, C, M->L,
                                                static_cast<const double*>(M->E.p), r, r, st),
                         "resid"));
    JB_TRY(launch_status(jb::launch_gmres_dots(nvox * C, M->L, r, r, 0, 0, 1,
                                               sq + M->L, sq, 1, 0, st),
                         "dots"));
    return launch_status(jb::launch_reduce_rows(sq, M->L, 1, res_out, 1.0,
                                                static_cast<const double*>(M->normd.p), 1, st),
                         "reduce");
  }
  jb::UpdateDesc u;
  u.mode = 2;
  u.eps = eps;
  u.E = static_cast<const double*>(M->E.p);
  u.partials = static_cast<double*>(M->partials.p);
  u.rout = static_cast<float*>(M->r32.p);
  int nb = 0;
  JB_TRY(green_passes(M->g64, eps, eps, M->L, M->spec.p, &loc64, &u, &nb, st));
  return launch_status(jb::launch_reduce_rows(static_cast<const double*>(M->partials.p), M->L,
                                              nb, res_out, 1.0,
                                              static_cast<const double*>(M->normd.p), 1, st),
                       "reduce");
}

// correction: d = r, inner - 1 FP32 sweeps d <- r - Gamma0[(C - C0):d],
// eps += d
int mixed_correct(jb_mixed* M, void* eps, int inner, cudaStream_t st) {
  const int C = M->g64->dim == 2 ? 3 : 6;
  const int64_t nel = (int64_t)M->L * M->l64->nvox * C;
  jb::LocalDesc loc32 = local_desc(M->l32);
  void* r32 = M->r32.p;
  void* d32 = M->d32.p;
  JB_CUDA(cudaMemcpyAsync(d32, r32, real_size(M->idt) * nel, cudaMemcpyDeviceToDevice, st));
  for (int j = 1; j < inner; ++j) {
    jb::UpdateDesc v;
    v.mode = 3;
    v.eps = d32;
    v.rhs = r32;
    JB_TRY(green_passes(M->g32, d32, d32, M->L, M->spec.p, &loc32, &v, nullptr, st));
  }
  return launch_status(
      jb::launch_axpy_to_f64(M->idt, nel, d32, static_cast<double*>(eps), st), "axpy");
}

// correction by `inner` BiCGSTAB iterations on A d = r (FP32, A d = d +
// Gamma0[(C - C0):d], from d = 0), eps += d
// the BiCGSTAB work fields and scalars (allocated on first use, before any
// graph capture)
int mixed_krylov_buffers(jb_mixed* M) {
  const int C = M->g64->dim == 2 ? 3 : 6;
  const int L = M->L;
  const int64_t nel = M->l64->nvox * C;
  const size_t fb = real_size(M->idt) * (size_t)L * nel;
  for (DeviceBuf* b : {&M->kr_rh, &M->kr_p, &M->kr_v, &M->kr_s, &M->kr_t, &M->kr_r})
    JB_TRY(ensure_buf(*b, fb));
  JB_TRY(ensure_buf(M->kr_part, sizeof(double) * 2 * L * jb::krylov_blocks(nel, L)));
  return ensure_buf(M->kr_state, sizeof(jb::KrylovState) * L);
}

int mixed_correct_bicgstab(jb_mixed* M, void* eps, int inner, cudaStream_t st) {
  const int C = M->g64->dim == 2 ? 3 : 6;
  const int L = M->L;
  const int64_t nel = M->l64->nvox * C;
  const int dt = M->idt;
  const size_t fb = real_size(dt) * (size_t)L * nel;
  JB_TRY(mixed_krylov_buffers(M));
  jb::LocalDesc loc32 = local_desc(M->l32);
  void* x = M->d32.p;
  void* b = M->r32.p;
  void *rh = M->kr_rh.p, *p = M->kr_p.p, *v = M->kr_v.p, *s = M->kr_s.p, *t = M->kr_t.p,
       *r = M->kr_r.p;
  double* part = static_cast<double*>(M->kr_part.p);
  auto* ks = static_cast<jb::KrylovState*>(M->kr_state.p);
  JB_CUDA(cudaMemsetAsync(x, 0, fb, st));
  JB_CUDA(cudaMemsetAsync(p, 0, fb, st));
  JB_CUDA(cudaMemsetAsync(v, 0, fb, st));
  JB_CUDA(cudaMemcpyAsync(r, b, fb, cudaMemcpyDeviceToDevice, st));
  JB_CUDA(cudaMemcpyAsync(rh, b, fb, cudaMemcpyDeviceToDevice, st));
  JB_TRY(launch_status(jb::launch_krylov_dot(dt, nel, L, rh, r, nullptr, nullptr, part, st),
                       "krylov_dot"));
  JB_TRY(launch_status(jb::launch_krylov_scalars(0, nel, L, part, ks, st), "krylov_scalars"));
  auto apply = [&](const void* in, void* out) {
    jb::UpdateDesc u;
    u.mode = 4;  // out = in + Gamma0[(C - C0):in]
    u.eps = out;
    u.rhs = in;
    return green_passes(M->g32, in, out, L, M->spec.p, &loc32, &u, nullptr, st);
  };
  for (int it = 0; it < inner; ++it) {
    JB_TRY(launch_status(
        jb::launch_krylov_update(dt, 0, nel, L, p, nullptr, nullptr, v, r, nullptr, ks, nullptr,
                                 st),
        "krylov_p"));
    JB_TRY(apply(p, v));
    JB_TRY(launch_status(jb::launch_krylov_dot(dt, nel, L, rh, v, nullptr, nullptr, part, st),
                         "krylov_dot"));
    JB_TRY(launch_status(jb::launch_krylov_scalars(1, nel, L, part, ks, st), "krylov_scalars"));
    JB_TRY(launch_status(
        jb::launch_krylov_update(dt, 1, nel, L, s, nullptr, nullptr, v, r, nullptr, ks, nullptr,
                                 st),
        "krylov_s"));
    JB_TRY(apply(s, t));
    JB_TRY(launch_status(jb::launch_krylov_dot(dt, nel, L, t, s, t, t, part, st), "krylov_dot"));
    JB_TRY(launch_status(jb::launch_krylov_scalars(2, nel, L, part, ks, st), "krylov_scalars"));
    JB_TRY(launch_status(
        jb::launch_krylov_update(dt, 2, nel, L, x, p, s, t, r, rh, ks, part, st), "krylov_xr"));
    JB_TRY(launch_status(jb::launch_krylov_scalars(3, nel, L, part, ks, st), "krylov_scalars"));
  }
  return launch_status(
      jb::launch_axpy_to_f64(dt, (int64_t)L * nel, x, static_cast<double*>(eps), st), "axpy");
}

// mean of (C - C0):eps per load case and component into host mean_tau
int mixed_mean(jb_mixed* M, const void* eps, double* mean_tau, cudaStream_t st) {
  const int C = M->g64->dim == 2 ? 3 : 6;
  jb::LocalDesc loc64 = local_desc(M->l64);
  int nb = 0;
  JB_TRY(launch_status(jb::launch_local_sum(F64, loc64, C, M->L, M->l64->nvox, eps,
                                            static_cast<double*>(M->partials.p), &nb, st),
                       "local_sum"));
  JB_TRY(launch_status(jb::launch_reduce_cols(static_cast<const double*>(M->partials.p), M->L,
                                              C, nb, static_cast<double*>(M->mean.p),
                                              1.0 / (double)M->l64->nvox, st),
                       "reduce"));
  JB_CUDA(cudaMemcpyAsync(mean_tau, M->mean.p, sizeof(double) * M->L * C,
                          cudaMemcpyDeviceToHost, st));
  return JB_OK;
}

}  // namespace

extern "C" int jb_mixed_run(jb_mixed* M, const double* E, void* eps, int init, int max_outer,
                            int inner, double tol, double* residuals, int* outer_out,
                            int* fp32_iters_out, double* mean_tau, int* status,
                            void* stream) {
  if (!M || !E || !eps) return fail(JB_EINVAL, "NULL argument");
  if (max_outer < 0) return fail(JB_EINVAL, "max_outer must be >= 0");
  if (inner < 1) return fail(JB_EINVAL, "inner must be >= 1");
  cudaStream_t st = as_stream(stream);
  const int L = M->L;
  JB_TRY(mixed_set_load(M, E, eps, init, st));
  std::vector<double> r(L);
  Outcome out(L);
  unsigned fault = 0;
  int outer = 0, fp32 = 0;
  double rprev = 0.0;  // largest residual of the previous outer step
  int kprev = 0;       // Krylov iterations of the previous correction
  for (; outer < max_outer; ++outer) {
    JB_TRY(mixed_residual(M, eps, static_cast<double*>(M->res.p), st));
    JB_CUDA(cudaMemcpyAsync(r.data(), M->res.p, sizeof(double) * L, cudaMemcpyDeviceToHost, st));
    JB_CUDA(jb::fetch_fault_async(&fault, st));
    JB_CUDA(cudaStreamSynchronize(st));
    JB_TRY(check_fault(fault, "jb_mixed_run"));
    bool done = true;
    double rmax = 0.0;
    for (int l = 0; l < L; ++l) {
      if (residuals) residuals[(size_t)outer * L + l] = r[l];
      if (!out.update(l, r[l], tol)) {
        done = false;
        rmax = std::max(rmax, r[l]);  // the load cases still iterating
      }
    }
    if (done) {
      ++outer;
      break;
    }
    if (M->method == JB_INNER_BICGSTAB || M->method == JB_INNER_BICGSTAB_FIXED) {
      // iterations this correction needs: the reduction per iteration seen
      // over the previous correction, extrapolated to half the tolerance
      // (at most `inner`; the full count when no rate is known yet)
      int k = inner;
      if (M->method == JB_INNER_BICGSTAB && kprev > 0 && rprev > 0.0 && rmax > 0.0 &&
          rmax < rprev) {
        const double rate = std::pow(rmax / rprev, 1.0 / kprev);
        if (rate > 0.0 && rate < 1.0) {
          const double need = std::log(0.5 * tol / rmax) / std::log(rate);
          if (need > 0.0 && need + 2.0 < (double)inner) k = std::max(2, (int)std::ceil(need) + 2);
        }
      }
      JB_TRY(mixed_correct_bicgstab(M, eps, k, st));
      fp32 += 2 * k;
      rprev = rmax;
      kprev = k;
    } else {
      JB_TRY(mixed_correct(M, eps, inner, st));
      fp32 += inner - 1;
    }
  }
  if (outer_out) *outer_out = outer;
  if (fp32_iters_out) *fp32_iters_out = fp32;
  out.write(tol, status);
  if (mean_tau) JB_TRY(mixed_mean(M, eps, mean_tau, st));
  JB_CUDA(jb::fetch_fault_async(&fault, st));
  JB_CUDA(cudaStreamSynchronize(st));
  JB_TRY(check_fault(fault, "jb_mixed_run"));
  return JB_OK;
}

// ===========================================================================
// batched mixed-precision solves: many problems (uneven grids), one CUDA
// graph launch per outer step
// ===========================================================================

struct jb_batch_s {
  std::vector<jb_mixed*> prob;
  std::vector<int> branch;             // branch stream of each problem
  std::vector<size_t> res_off;         // offset of each problem's residuals in res_all
  int nbranch = 1;
  std::vector<cudaStream_t> streams;   // capture origin + branches
  std::vector<cudaEvent_t> events;     // fork / join
  DeviceBuf res_all;
  size_t nres = 0;
  cudaGraphExec_t exec = nullptr;
  DeviceBuf dstate;                    // persistent run: decision state on the device
  bool persistent = true;              // one graph launch per run (conditional nodes)
  std::vector<char> captured;          // active set of the instantiated graph
  std::vector<void*> captured_eps;     // the strain fields its kernels address
  int captured_inner = 0;
};

extern "C" int jb_batch_destroy(jb_batch* B) {
  if (!B) return JB_OK;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  for (cudaStream_t s : B->streams) cudaStreamDestroy(s);
  for (cudaEvent_t e : B->events) cudaEventDestroy(e);
  if (B->res_all.p) cudaFree(B->res_all.p);
  delete B;
  return JB_OK;
}

extern "C" int jb_batch_set_persistent(jb_batch* B, int on) {
  if (!B) return fail(JB_EINVAL, "NULL argument");
  B->persistent = on != 0;
  return JB_OK;
}

extern "C" int jb_batch_create(int count, jb_mixed* const* problems, int branches,
                               jb_batch** out) {
  if (!out) return fail(JB_EINVAL, "out must not be NULL");
  *out = nullptr;
  if (count < 1 || !problems) return fail(JB_EINVAL, "a batch needs at least one problem");
  if (branches < 1 || branches > 64) return fail(JB_EINVAL, "branches must be in [1, 64]");
  jb_batch* B = new jb_batch();
  B->prob.assign(problems, problems + count);
  for (jb_mixed* M : B->prob)
    if (!M) {
      delete B;
      return fail(JB_EINVAL, "NULL problem");
    }
  // longest-processing-time assignment of problems to branches by work
  B->nbranch = std::min(branches, count);
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  auto work = [&](int i) { return (double)B->prob[i]->L * (double)B->prob[i]->l64->nvox; };
  std::sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  std::vector<double> load(B->nbranch, 0.0);
  B->branch.assign(count, 0);
  for (int i : order) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    B->branch[i] = k;
    load[k] += work(i);
  }
  B->res_off.resize(count);
  for (int i = 0; i < count; ++i) {
    B->res_off[i] = B->nres;
    B->nres += B->prob[i]->L;
  }
  int r = ensure_buf(B->res_all, sizeof(double) * B->nres);
  B->streams.assign(B->nbranch + 1, nullptr);
  B->events.assign(2 * B->nbranch + 1, nullptr);
  for (auto& s : B->streams)
    if (r == JB_OK && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
      r = fail(JB_ECUDA, "jb_batch_create: cudaStreamCreate failed");
  for (auto& e : B->events)
    if (r == JB_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      r = fail(JB_ECUDA, "jb_batch_create: cudaEventCreate failed");
  if (r != JB_OK) {
    cudaGetLastError();
    jb_batch_destroy(B);
    return r;
  }
  *out = B;
  return JB_OK;
}

namespace {

// capture one outer step (correction, then residual) of the active problems:
// the origin stream forks to the branch streams and joins them again
int batch_capture(jb_batch* B, const std::vector<char>& active, void* const* eps, int inner) {
  cudaStream_t origin = B->streams[0];
  double* res = static_cast<double*>(B->res_all.p);
  JB_CUDA(cudaStreamBeginCapture(origin, cudaStreamCaptureModeRelaxed));
  int r = JB_OK;
  cudaError_t e = cudaEventRecord(B->events[0], origin);
  for (int k = 0; k < B->nbranch && e == cudaSuccess; ++k)
    e = cudaStreamWaitEvent(B->streams[k + 1], B->events[0], 0);
  for (size_t i = 0; i < B->prob.size() && r == JB_OK && e == cudaSuccess; ++i) {
    if (!active[i]) continue;
    cudaStream_t st = B->streams[B->branch[i] + 1];
    r = B->prob[i]->method != JB_INNER_BASIC
            ? mixed_correct_bicgstab(B->prob[i], eps[i], inner, st)
            : mixed_correct(B->prob[i], eps[i], inner, st);
    if (r == JB_OK) r = mixed_residual(B->prob[i], eps[i], res + B->res_off[i], st);
  }
  for (int k = 0; k < B->nbranch && e == cudaSuccess; ++k) {
    e = cudaEventRecord(B->events[k + 1], B->streams[k + 1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(origin, B->events[k + 1], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(origin, &graph);
  if (r != JB_OK) {
    if (graph) cudaGraphDestroy(graph);
    return r;
  }
  if (e != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return fail(JB_ECUDA, std::string("jb_batch_run: capture: ") +
                              cudaGetErrorString(e != cudaSuccess ? e : ee));
  }
  if (B->exec) {
    cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
  }
  e = cudaGraphInstantiate(&B->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    B->exec = nullptr;
    return fail(JB_ECUDA, std::string("jb_batch_run: instantiate: ") + cudaGetErrorString(e));
  }
  B->captured = active;
  B->captured_eps.assign(eps, eps + B->prob.size());
  B->captured_inner = inner;
  return JB_OK;
}

}  // namespace

namespace {

// Device-side decision of the persistent batched run: the host loop's
// per-step work (record each active problem's residuals, update each load
// case's outcome, retire problems that converged, stopped or reached
// max_outer) done by one block at the start of every iteration of the
// graph's while node; it sets each problem's IF condition and the while
// condition (any problem active).  Same rule as Outcome::update.
struct BatchDecide {
  int P, max_outer;
  double tol, diverge;
  const int* L;               // [P] load cases
  const int* roff;            // [P] offset of a problem's load cases in res / best / ...
  const int64_t* hoff;        // [P] offset of a problem's history (max_outer x L)
  const double* res;          // [nres] latest residuals
  double* hist;               // residual history
  double* best;               // [nres]
  double* last;               // [nres]
  int* stopped;               // [nres]
  int* active;                // [P]
  int* outer;                 // [P] residual evaluations recorded + 1 while iterating
  int* steps;                 // iterations of the while body so far (bound)
  const cudaGraphConditionalHandle* ifh;  // [P]
  cudaGraphConditionalHandle wh;
};

__global__ void batch_decide_kernel(BatchDecide a) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  // the while body runs at most max_outer + 1 times (every problem retires
  // by then); past that, retire everything
  const bool force = *a.steps > a.max_outer + 1;
  for (int p = threadIdx.x; p < a.P; p += blockDim.x) {
    int act = a.active[p];
    if (act) {
      const int L = a.L[p], o = a.outer[p];
      bool done = true;
      for (int l = 0; l < L; ++l) {
        const int q = a.roff[p] + l;
        const double r = a.res[q];
        a.hist[a.hoff[p] + (int64_t)(o - 1) * L + l] = r;
        bool fin;  // the load case no longer holds the problem back
        if (a.stopped[q]) {
          fin = true;
        } else {
          a.last[q] = r;
          if (!isfinite(r)) {
            a.stopped[q] = JB_SOLVE_NON_FINITE;
            fin = true;
          } else if (r > a.tol && a.best[q] > 0.0 && r > a.diverge * a.best[q]) {
            a.stopped[q] = JB_SOLVE_DIVERGING;
            fin = true;
          } else {
            a.best[q] = fmin(a.best[q], r);
            fin = r <= a.tol;
          }
        }
        done = done && fin;
      }
      if (done || o >= a.max_outer || force)
        act = 0;
      else
        a.outer[p] = o + 1;
      a.active[p] = act;
    }
    cudaGraphSetConditional(a.ifh[p], act ? 1u : 0u);
    if (act) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cudaGraphSetConditional(a.wh, any ? 1u : 0u);
    *a.steps += 1;
  }
}

// One graph launch for the whole batched run: while (any problem active) {
// decide; for each problem: if (active) { correction; FP64 residual } }.
// The first residuals and all lazily built tables come before (on `st`).
// Returns JB_ESTATE when this CUDA build cannot make conditional nodes (the
// caller then runs the per-step loop); fills outer / outc / residuals.
int batch_persistent(jb_batch* B, void* const* eps, int max_outer, int inner, double tol,
                     const std::vector<int64_t>& hoff, double* residuals,
                     std::vector<int>& outer, std::vector<Outcome>& outc, cudaStream_t st) {
  const int P = (int)B->prob.size();
  const int nres = (int)B->nres;
  const int64_t nhist = hoff.empty() ? 0 : hoff.back() + (int64_t)max_outer * B->prob.back()->L;
  // device state: L, roff, hoff, active, outer, stopped, steps | best, last, hist | handles
  auto al8 = [](size_t v) { return (v + 7) / 8 * 8; };
  const size_t o_L = 0, o_roff = al8(o_L + 4 * P), o_hoff = al8(o_roff + 4 * P),
               o_act = al8(o_hoff + 8 * P), o_out = al8(o_act + 4 * P),
               o_stop = al8(o_out + 4 * P), o_steps = al8(o_stop + 4 * nres),
               o_best = al8(o_steps + 8), o_last = al8(o_best + 8 * nres),
               o_hist = al8(o_last + 8 * nres), o_h = al8(o_hist + 8 * nhist),
               total = o_h + 8 * (P + 1);
  JB_TRY(ensure_buf(B->dstate, total));
  std::vector<unsigned char> host(total, 0);
  auto put = [&](size_t off, const void* src, size_t bytes) {
    std::memcpy(host.data() + off, src, bytes);
  };
  std::vector<int> Ls(P), roff(P), ones(P, 1);
  for (int i = 0; i < P; ++i) {
    Ls[i] = B->prob[i]->L;
    roff[i] = (int)B->res_off[i];
  }
  std::vector<double> inf(nres, INFINITY);
  put(o_L, Ls.data(), 4 * P);
  put(o_roff, roff.data(), 4 * P);
  put(o_hoff, hoff.data(), 8 * P);
  put(o_act, ones.data(), 4 * P);
  put(o_out, ones.data(), 4 * P);
  put(o_best, inf.data(), 8 * nres);
  put(o_last, inf.data(), 8 * nres);
  unsigned char* d = static_cast<unsigned char*>(B->dstate.p);

  cudaGraph_t g = nullptr;
  JB_CUDA(cudaGraphCreate(&g, 0));
  std::vector<cudaGraphConditionalHandle> h(P + 1);
  cudaError_t e = cudaGraphConditionalHandleCreate(&h[P], g, 1, cudaGraphCondAssignDefault);
  for (int i = 0; i < P && e == cudaSuccess; ++i)
    e = cudaGraphConditionalHandleCreate(&h[i], g, 0, 0);
  cudaGraphNode_t wnode = nullptr;
  cudaGraphNodeParams wp = {};
  if (e == cudaSuccess) {
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h[P];
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    e = cudaGraphAddNode(&wnode, g, nullptr, 0, &wp);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return fail(JB_ESTATE, std::string("conditional graph nodes unavailable: ") +
                               cudaGetErrorString(e));
  }
  put(o_h, h.data(), 8 * (P + 1));
  JB_CUDA(cudaMemcpyAsync(d, host.data(), total, cudaMemcpyHostToDevice, st));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  cudaStream_t cs = B->streams[1 % B->streams.size()];
  BatchDecide dk;
  dk.P = P;
  dk.max_outer = max_outer;
  dk.tol = tol;
  dk.diverge = kDivergeFactor;
  dk.L = reinterpret_cast<const int*>(d + o_L);
  dk.roff = reinterpret_cast<const int*>(d + o_roff);
  dk.hoff = reinterpret_cast<const int64_t*>(d + o_hoff);
  dk.res = static_cast<const double*>(B->res_all.p);
  dk.hist = reinterpret_cast<double*>(d + o_hist);
  dk.best = reinterpret_cast<double*>(d + o_best);
  dk.last = reinterpret_cast<double*>(d + o_last);
  dk.stopped = reinterpret_cast<int*>(d + o_stop);
  dk.active = reinterpret_cast<int*>(d + o_act);
  dk.outer = reinterpret_cast<int*>(d + o_out);
  dk.steps = reinterpret_cast<int*>(d + o_steps);
  dk.ifh = reinterpret_cast<const cudaGraphConditionalHandle*>(d + o_h);
  dk.wh = h[P];
  // the body: the decision kernel, then one IF node per problem after it
  int r = JB_OK;
  e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    batch_decide_kernel<<<1, 256, 0, cs>>>(dk);
    e = cudaGetLastError();
    cudaGraph_t same = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cs, &same);
    if (e == cudaSuccess) e = ee;
  }
  cudaGraphNode_t decide = nullptr;
  size_t nn = 1;
  if (e == cudaSuccess) e = cudaGraphGetNodes(body, &decide, &nn);
  for (int i = 0; i < P && e == cudaSuccess && r == JB_OK; ++i) {
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = h[i];
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode = nullptr;
    e = cudaGraphAddNode(&inode, body, &decide, 1, &ip);
    if (e != cudaSuccess) break;
    e = cudaStreamBeginCaptureToGraph(cs, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) break;
    jb_mixed* M = B->prob[i];
    r = M->method != JB_INNER_BASIC ? mixed_correct_bicgstab(M, eps[i], inner, cs)
                                    : mixed_correct(M, eps[i], inner, cs);
    if (r == JB_OK)
      r = mixed_residual(M, eps[i], static_cast<double*>(B->res_all.p) + B->res_off[i], cs);
    cudaGraph_t same = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cs, &same);
    if (e == cudaSuccess) e = ee;
  }
  cudaGraphExec_t exec = nullptr;
  if (e == cudaSuccess && r == JB_OK) e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (r != JB_OK) {
    if (exec) cudaGraphExecDestroy(exec);
    return r;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (exec) cudaGraphExecDestroy(exec);
    return fail(JB_ESTATE, std::string("persistent batch graph: ") + cudaGetErrorString(e));
  }
  // after the eager work on the caller's stream, one launch runs to the end
  JB_CUDA(cudaGraphLaunch(exec, st));
  JB_CUDA(cudaMemcpyAsync(host.data(), d, total, cudaMemcpyDeviceToHost, st));
  unsigned fault = 0;
  JB_CUDA(jb::fetch_fault_async(&fault, st));
  const cudaError_t se = cudaStreamSynchronize(st);
  cudaGraphExecDestroy(exec);
  JB_CUDA(se);
  JB_TRY(check_fault(fault, "jb_batch_run"));
  const int* outd = reinterpret_cast<const int*>(host.data() + o_out);
  const int* stopd = reinterpret_cast<const int*>(host.data() + o_stop);
  const double* bestd = reinterpret_cast<const double*>(host.data() + o_best);
  const double* lastd = reinterpret_cast<const double*>(host.data() + o_last);
  const double* histd = reinterpret_cast<const double*>(host.data() + o_hist);
  for (int i = 0; i < P; ++i) {
    outer[i] = outd[i];
    for (int l = 0; l < Ls[i]; ++l) {
      const int q = roff[i] + l;
      outc[i].stopped[l] = stopd[q];
      outc[i].best[l] = bestd[q];
      outc[i].last[l] = lastd[q];
    }
  }
  if (residuals) std::memcpy(residuals, histd, 8 * (size_t)nhist);
  return JB_OK;
}

}  // namespace

extern "C" int jb_batch_run(jb_batch* B, const double* E, void* const* eps, int init,
                            int max_outer, int inner, double tol, double* residuals,
                            int* outer_out, int* fp32_iters_out, double* mean_tau,
                            int* graph_launches_out, int* status, void* stream) {
  if (!B || !E || !eps) return fail(JB_EINVAL, "NULL argument");
  if (max_outer < 1) return fail(JB_EINVAL, "max_outer must be >= 1");
  if (inner < 1) return fail(JB_EINVAL, "inner must be >= 1");
  const size_t P = B->prob.size();
  for (size_t i = 0; i < P; ++i)
    if (!eps[i]) return fail(JB_EINVAL, "NULL strain field");
  cudaStream_t st = as_stream(stream);
  cudaStream_t origin = B->streams[0];
  double* res = static_cast<double*>(B->res_all.p);
  // loads, then the first residual of every problem (eagerly: this also
  // builds each operator's lazily created tables before any capture)
  size_t eoff = 0;
  for (size_t i = 0; i < P; ++i) {
    jb_mixed* M = B->prob[i];
    const int C = M->g64->dim == 2 ? 3 : 6;
    JB_TRY(mixed_set_load(M, E + eoff, eps[i], init, st));
    eoff += (size_t)M->L * C;
  }
  for (size_t i = 0; i < P; ++i) {
    if (green_uses_table(B->prob[i]->g32))  // nothing lazily built inside a capture
      JB_TRY(green_prepare(B->prob[i]->g32, st));
    if (B->prob[i]->method != JB_INNER_BASIC) JB_TRY(mixed_krylov_buffers(B->prob[i]));
    JB_TRY(mixed_residual(B->prob[i], eps[i], res + B->res_off[i], st));
  }
  std::vector<double> rh(B->nres);
  std::vector<int> outer(P, 1);
  std::vector<char> active(P, 1);
  size_t roff = 0;
  std::vector<size_t> hist_off(P);
  for (size_t i = 0; i < P; ++i) {
    hist_off[i] = roff;
    roff += (size_t)max_outer * B->prob[i]->L;
  }
  std::vector<Outcome> outc;
  outc.reserve(P);
  for (size_t i = 0; i < P; ++i) outc.emplace_back(B->prob[i]->L);
  unsigned fault = 0;
  int launches = 0;
  bool done_persistent = false;
  if (B->persistent) {
    std::vector<int64_t> hoff(hist_off.begin(), hist_off.end());
    const int pr = batch_persistent(B, eps, max_outer, inner, tol, hoff, residuals, outer, outc,
                                    st);
    if (pr == JB_OK) {
      done_persistent = true;
      launches = 1;
    } else if (pr == JB_ESTATE) {
      B->persistent = false;  // this CUDA build: the per-step loop from now on
    } else {
      return pr;
    }
  }
  for (int step = 0; !done_persistent; ++step) {
    cudaStream_t rs = step == 0 ? st : origin;
    JB_CUDA(cudaMemcpyAsync(rh.data(), res, sizeof(double) * B->nres, cudaMemcpyDeviceToHost,
                            rs));
    JB_CUDA(jb::fetch_fault_async(&fault, rs));
    JB_CUDA(cudaStreamSynchronize(rs));
    JB_TRY(check_fault(fault, "jb_batch_run"));
    bool any = false;
    for (size_t i = 0; i < P; ++i) {
      if (!active[i]) continue;
      const int L = B->prob[i]->L;
      bool done = true;
      for (int l = 0; l < L; ++l) {
        const double v = rh[B->res_off[i] + l];
        if (residuals) residuals[hist_off[i] + (size_t)(outer[i] - 1) * L + l] = v;
        if (!outc[i].update(l, v, tol)) done = false;
      }
      if (done || outer[i] >= max_outer) active[i] = 0;
      any = any || active[i];
    }
    if (!any) break;
    // the graph holds the fields' addresses and the sweep count: capture
    // again when the active set, a field or inner changes
    const bool same = B->exec && B->captured == active && B->captured_inner == inner &&
                      std::equal(B->captured_eps.begin(), B->captured_eps.end(), eps);
    if (!same) JB_TRY(batch_capture(B, active, eps, inner));
    if (step == 0) {
      // order the graph after the eager work on the caller's stream
      JB_CUDA(cudaEventRecord(B->events[B->nbranch + 1], st));
      JB_CUDA(cudaStreamWaitEvent(origin, B->events[B->nbranch + 1], 0));
    }
    JB_CUDA(cudaGraphLaunch(B->exec, origin));
    ++launches;
    for (size_t i = 0; i < P; ++i)
      if (active[i]) ++outer[i];
  }
  // the caller's stream continues after the graph work
  JB_CUDA(cudaEventRecord(B->events[0], origin));
  JB_CUDA(cudaStreamWaitEvent(st, B->events[0], 0));
  eoff = 0;
  for (size_t i = 0; i < P; ++i) {
    jb_mixed* M = B->prob[i];
    const int C = M->g64->dim == 2 ? 3 : 6;
    if (outer_out) outer_out[i] = outer[i];
    outc[i].write(tol, status, (int)B->res_off[i]);
    if (fp32_iters_out)
      fp32_iters_out[i] =
          (outer[i] - 1) * (M->method != JB_INNER_BASIC ? 2 * inner : inner - 1);
    if (mean_tau) JB_TRY(mixed_mean(M, eps[i], mean_tau + eoff, st));
    eoff += (size_t)M->L * C;
  }
  if (graph_launches_out) *graph_launches_out = launches;
  JB_CUDA(cudaStreamSynchronize(st));
  return JB_OK;
}
