// Row passes along long contiguous axes (n = 384, 512, 768, 1024) of
// three-component 2D fields: persistent, pipelined kernels.  Included by
// jb_kernels.cu inside its kernel namespace (uses RowsArgs, the local
// operator and block_sum).
//
// The general row kernels pair two real columns of the tile into one complex
// column and transform n points; with one 1024-point FP64 row per CTA (three
// real columns, so one half-empty complex column) they hold two CTAs of 8
// warps per SM, wait for each row's load, and run at ~21% of HBM.  Here:
//  * half-length transform per component: z_c[j] = x[2j][c] + i x[2j+1][c],
//    H = n/2 points, unpacked into the half spectrum X_c[0..H] with one
//    twiddle per coefficient pair (k, H-k) (r2c), and packed the other way
//    before the inverse (c2r);
//  * H = N1 * 64 points (N1 = 3, 4, 6, 8) as three register phases (N1-, 8-
//    and 8-point transforms, n' = j + 64 m, j = ja + 8 jb, k = k1 + N1 (kb +
//    8 ka)) on a tile whose rows k1 are PK = 193 (FP64) / 194 (FP32)
//    complex apart, so the lanes of phases 2 and 3 (k1 fastest) meet at most
//    two-way bank conflicts;
//  * one CTA of 192 threads walks the rows (l, r) = t, t + grid, ...; loads
//    and stores are bulk copies issued by thread 0, one row or more ahead.
// Half twiddle table: w_n^i for i < n/2 in shared memory, w_n^(i + n/2) =
// -w_n^i.

template <typename T, int N> struct LongRow {
  static constexpr int H = N / 2;
  static constexpr int N1 = H / 64;
  static constexpr int PK = 192 + (sizeof(T) == 8 ? 1 : 2);
  static constexpr int TILE = N1 * PK;  // complex
  static constexpr int THREADS = 192;
  static constexpr int P23 = N1 * 24;   // lanes of phases 2 and 3
  static constexpr int PAIRS = 3 * N1 * (H / (2 * N1) + 1);  // pair jobs (k <= H/2)
  static constexpr int MINB = sizeof(T) == 8 ? (N <= 512 ? 4 : 2) : (N <= 512 ? 5 : 4);
  static constexpr size_t RAWB = ((size_t)N * 3 * sizeof(T) + 127) / 128 * 128;
};

__host__ __device__ constexpr size_t lr_a128(size_t v) { return (v + 127) / 128 * 128; }

// shared-memory layout of the r2c kernel (byte offsets): twiddles | two raw
// rows | tile | spectral row | two phase-id rows | staged table
struct LongR2cLayout {
  size_t raw, tile, outs, ph, tab, total;
};
__host__ __device__ inline LongR2cLayout long_r2c_layout(size_t cs, int n, int64_t sp,
                                                         size_t phb, size_t tabb) {
  LongR2cLayout o{};
  const size_t rawb = lr_a128((size_t)n * 3 * (cs / 2));
  const int n1 = n / 128;
  const size_t pk = 192 + (cs == 16 ? 1 : 2);
  o.raw = lr_a128((size_t)(n / 2) * cs);
  o.tile = o.raw + 2 * rawb;
  o.outs = o.tile + lr_a128(n1 * pk * cs);
  o.ph = o.outs + lr_a128((size_t)sp * cs);
  o.tab = o.ph + lr_a128(2 * phb);
  o.total = o.tab + lr_a128(tabb);
  return o;
}

// c2r: twiddles | two spectral rows (tile + tail) | two real rows
struct LongC2rLayout {
  size_t spec, real, total;
};
__host__ __device__ inline LongC2rLayout long_c2r_layout(size_t cs, int n) {
  LongC2rLayout o{};
  const int n1 = n / 128;
  const size_t pk = 192 + (cs == 16 ? 1 : 2);
  const size_t specb = lr_a128((n1 * pk + 4) * cs);
  o.spec = lr_a128((size_t)(n / 2) * cs);
  o.real = o.spec + 2 * specb;
  o.total = o.real + 2 * lr_a128((size_t)n * 3 * (cs / 2));
  return o;
}

// tile position of natural coefficient k (component c) after phase 3
template <typename K> __device__ __forceinline__ int lr_zpos(int k, int c) {
  const int k1 = k % K::N1, k2 = k / K::N1;
  return k1 * K::PK + ((k2 >> 3) + 8 * (k2 & 7)) * 3 + c;
}

// tile position of natural index k of the phase-1 input (k <= H: the tail)
template <typename K> __device__ __forceinline__ int lr_ipos(int k, int c) {
  return (k >> 6) * K::PK + (k & 63) * 3 + c;
}

// w_n^i, 0 <= i < n, from the half table
template <int N, typename C> __device__ __forceinline__ C lr_tw(const C* tw, int i) {
  const bool hi = i >= N / 2;
  const C w = tw[hi ? i - N / 2 : i];
  return hi ? mkc(-w.x, -w.y) : w;
}

// phases 1-3 of the H-point transform of the three columns in tile z.
// DIR -1: phase 1 reads z_c from the raw row x (r2c) into the tile;
// DIR +1: phase 1 runs in place on the packed spectrum (c2r).
// Barriers after phases 1 and 2; the caller orders phase 3 with what follows.
template <typename K, int DIR, int N, typename T>
__device__ __forceinline__ void lr_phase1(cx<T>* z, const T* x, const cx<T>* tw, int tid) {
  using C = cx<T>;
  constexpr int N1 = K::N1;
  const int c = tid % 3, j = tid / 3;
  C v[N1];
  if constexpr (DIR < 0) {
#pragma unroll
    for (int m = 0; m < N1; ++m) {
      const T* p = x + (2 * (j + 64 * m)) * 3 + c;
      v[m] = mkc(p[0], p[3]);
    }
  } else {
#pragma unroll
    for (int m = 0; m < N1; ++m) v[m] = z[m * K::PK + j * 3 + c];
  }
  Dft<N1, DIR, C>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) {
    const C w = lr_tw<N>(tw, 2 * j * k1);
    v[k1] = DIR < 0 ? cmul(v[k1], w) : cmulc(v[k1], w);
  }
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) z[k1 * K::PK + j * 3 + c] = v[k1];
}

template <typename K, int DIR, int N, typename T>
__device__ __forceinline__ void lr_phase2(cx<T>* z, const cx<T>* tw, int tid) {
  using C = cx<T>;
  constexpr int N1 = K::N1;
  if (tid < K::P23) {
    const int k1 = tid % N1, c = (tid / N1) % 3, ja = tid / (3 * N1);
    C* s = z + k1 * K::PK + ja * 3 + c;
    C w[8];
#pragma unroll
    for (int jb = 0; jb < 8; ++jb) w[jb] = s[jb * 24];
    Dft<8, DIR, C>::run(w);
#pragma unroll
    for (int kb = 1; kb < 8; ++kb) {
      const C t = lr_tw<N>(tw, (N / 64) * ja * kb);
      w[kb] = DIR < 0 ? cmul(w[kb], t) : cmulc(w[kb], t);
    }
#pragma unroll
    for (int kb = 0; kb < 8; ++kb) s[kb * 24] = w[kb];
  }
}

template <typename K, int DIR, typename T>
__device__ __forceinline__ void lr_phase3(cx<T>* z, int tid) {
  using C = cx<T>;
  constexpr int N1 = K::N1;
  if (tid < K::P23) {
    const int k1 = tid % N1, c = (tid / N1) % 3, kb = tid / (3 * N1);
    C* s = z + k1 * K::PK + kb * 24 + c;
    C u[8];
#pragma unroll
    for (int ja = 0; ja < 8; ++ja) u[ja] = s[ja * 3];
    Dft<8, DIR, C>::run(u);
#pragma unroll
    for (int ka = 0; ka < 8; ++ka) s[ka * 3] = u[ka];
  }
}

// r2c of the rows, the local operator (C - C0):eps applied to each voxel
// first when LOCAL (phase ids by bulk copy beside the row, or the voxel
// index).  Row i: wait for its raw row; local operator in place; phase 1
// (raw -> tile), after which the raw buffer takes the row two tiles ahead;
// phases 2, 3; the unpacked half spectrum into the spectral staging row,
// stored by one bulk copy once the previous row's store has read it.
template <typename T, int N, bool LOCAL>
__global__ void __launch_bounds__(LongRow<T, N>::THREADS, LongRow<T, N>::MINB)
    rows_long_r2c_kernel(RowsArgs<T> a) {
  using C = cx<T>;
  using K = LongRow<T, N>;
  constexpr int H = K::H, N1 = K::N1;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int fail_flag;
  const int tid = threadIdx.x;
  const int ib = LOCAL ? a.index_bytes : 0;
  const size_t phb = (size_t)N * ib;
  const int tabn = LOCAL ? a.nphase * local_entry(a.kind, 2) : 0;
  const bool staged = LOCAL && tabn <= 2 * kTabStage;
  const LongR2cLayout lay =
      long_r2c_layout(sizeof(C), N, a.sp, phb, staged ? (size_t)tabn * sizeof(T) : 0);
  C* tw = reinterpret_cast<C*>(smem);
  C* tile = reinterpret_cast<C*>(smem + lay.tile);
  C* outs = reinterpret_cast<C*>(smem + lay.outs);
  T* tabs = reinterpret_cast<T*>(smem + lay.tab);
  auto raw = [&](int b) { return reinterpret_cast<T*>(smem + lay.raw + b * K::RAWB); };
  auto phs = [&](int b) { return smem + lay.ph + b * phb; };
  const int64_t rows = a.g.rows;
  const int64_t total = rows * a.L;
  const int64_t G = gridDim.x;
  if (tid == 0) {
    fail_flag = 0;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  for (int i = tid; i < H; i += K::THREADS) tw[i] = a.tw[i];
  const T* tab = a.table;
  if (staged) {
    for (int i = tid; i < tabn; i += K::THREADS) tabs[i] = a.table[i];
    tab = tabs;
  }
  __syncthreads();
  auto issue = [&](int64_t t, int b) {
    const int64_t l = t / rows, r = t - l * rows;
    const uint32_t xb = (uint32_t)(N * 3 * sizeof(T));
    mbar_arrive_expect_tx(&bar[b], xb + (uint32_t)phb);
    bulk_load(raw(b), a.x + l * a.g.ls + r * N * 3, xb, &bar[b]);
    if (phb > 0)
      bulk_load(phs(b), static_cast<const unsigned char*>(a.phase) + r * (int64_t)phb,
                (uint32_t)phb, &bar[b]);
  };
  const int64_t t0 = blockIdx.x;
  if (tid == 0) {
    if (t0 < total) issue(t0, 0);
    if (t0 + G < total) issue(t0 + G, 1);
  }
  int i = 0;
  for (int64_t t = t0; t < total; t += G, ++i) {
    const int b = i & 1;
    const int64_t l = t / rows, r = t - l * rows;
    if (!mbar_wait(&bar[b], (i >> 1) & 1)) atomicOr(&fail_flag, 1);
    __syncthreads();
    if (fail_flag) {
      // the other buffer's row may still be in flight: let it land
      if (t + G < total) mbar_wait(&bar[b ^ 1], ((i + 1) >> 1) & 1);
      break;
    }
    T* x = raw(b);
    if constexpr (LOCAL) {
      const unsigned char* ph = phs(b);
      for (int e = tid; e < N; e += K::THREADS) {
        T v[3] = {x[e * 3], x[e * 3 + 1], x[e * 3 + 2]};
        const int p = ib == 0   ? (int)(r * N + e)
                      : ib == 1 ? (int)ph[e]
                                : reinterpret_cast<const int32_t*>(ph)[e];
        local_apply<T>(v, tab, p, a.kind, 2);
        x[e * 3] = v[0];
        x[e * 3 + 1] = v[1];
        x[e * 3 + 2] = v[2];
      }
      __syncthreads();
    }
    lr_phase1<K, -1, N, T>(tile, x, tw, tid);
    fence_async_shared();  // the raw row's generic writes before the next bulk load into it
    __syncthreads();
    if (tid == 0 && t + 2 * G < total) issue(t + 2 * G, b);
    lr_phase2<K, -1, N, T>(tile, tw, tid);
    __syncthreads();
    lr_phase3<K, -1, T>(tile, tid);
    if (tid == 0) bulk_wait_read();  // the previous row's store has read `outs`
    __syncthreads();
    for (int q = tid; q < K::PAIRS; q += K::THREADS) {
      const int k1 = q % N1, c = (q / N1) % 3, k2 = q / (3 * N1);
      const int k = k1 + N1 * k2;
      if (k > H / 2) continue;
      const C Z = tile[lr_zpos<K>(k, c)];
      const C Zh = tile[lr_zpos<K>(k == 0 ? 0 : H - k, c)];
      // A = (Z + conj Zh)/2, P = w^k (Z - conj Zh):
      // X[k] = A - (i/2) P, X[H-k] = conj A - (i/2) conj P
      const T ax = T(0.5) * (Z.x + Zh.x), ay = T(0.5) * (Z.y - Zh.y);
      const C P = cmul(tw[k], mkc(Z.x - Zh.x, Z.y + Zh.y));
      outs[k * 3 + c] = mkc(ax + T(0.5) * P.y, ay - T(0.5) * P.x);
      if (2 * k != H) outs[(H - k) * 3 + c] = mkc(ax - T(0.5) * P.y, -ay - T(0.5) * P.x);
    }
    if (tid == 0 && a.sp > 3 * (H + 1)) outs[3 * (H + 1)] = mkc(T(0), T(0));  // row padding
    fence_async_shared();
    __syncthreads();
    if (tid == 0) {
      bulk_store(a.out + l * a.cstride_l + r * a.sp, outs, (uint32_t)(a.sp * sizeof(C)));
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait_read();
}

// c2r of the rows with the row kernels' epilogues except kEpiResid
// (y = scale * c2r(spectrum); update: eps <- E - y with its squared-increment
// partials per load case; rhs: d <- rhs - y).  Row i: wait for its spectral
// row (loaded as N1 chunks of 64 coefficients into the tile rows, plus the
// tail X[H]); pack in place; phases 1-3 in place, after phase 1 the side row
// of the next tile heads for its buffer; the epilogue writes the result over
// the side row, which one bulk copy stores; the spectral buffer then takes the
// row two tiles ahead.  Partials: one slot per (load case, CTA), the CTA's
// rows of a load case being consecutive.
template <typename T, int N, int EPI>
__global__ void __launch_bounds__(LongRow<T, N>::THREADS, LongRow<T, N>::MINB)
    rows_long_c2r_kernel(RowsArgs<T> a) {
  using C = cx<T>;
  using K = LongRow<T, N>;
  constexpr int H = K::H, N1 = K::N1;
  constexpr bool kSide = EPI != kEpiPlain;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar_in[2];
  __shared__ __align__(8) uint64_t bar_sd[2];
  __shared__ int fail_flag;
  __shared__ double red[K::THREADS / 32];
  const int tid = threadIdx.x;
  const LongC2rLayout lay = long_c2r_layout(sizeof(C), N);
  constexpr size_t SPECB = lr_a128(((size_t)K::TILE + 4) * sizeof(C));
  C* tw = reinterpret_cast<C*>(smem);
  auto spec = [&](int b) { return reinterpret_cast<C*>(smem + lay.spec + b * SPECB); };
  auto real = [&](int b) { return reinterpret_cast<T*>(smem + lay.real + b * K::RAWB); };
  const int64_t rows = a.g.rows;
  const int64_t total = rows * a.L;
  const int64_t G = gridDim.x;
  if (tid == 0) {
    fail_flag = 0;
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bar_in[b], 1);
      mbar_init(&bar_sd[b], 1);
    }
    fence_mbar_init();
    if (EPI == kEpiUpdate)
      for (int l = 0; l < a.L; ++l) a.partials[(int64_t)l * G + blockIdx.x] = 0.0;
  }
  for (int i = tid; i < H; i += K::THREADS) tw[i] = a.tw[i];
  __syncthreads();
  const uint32_t tailb = (uint32_t)((a.sp - 3 * H) * sizeof(C));
  auto issue_in = [&](int64_t t, int b) {
    const int64_t l = t / rows, r = t - l * rows;
    const C* src = a.cin + l * a.cstride_l + r * a.sp;
    C* dst = spec(b);
    mbar_arrive_expect_tx(&bar_in[b], (uint32_t)(a.sp * sizeof(C)));
    for (int m = 0; m < N1; ++m)
      bulk_load(dst + m * K::PK, src + m * 192, (uint32_t)(192 * sizeof(C)), &bar_in[b]);
    bulk_load(dst + N1 * K::PK, src + 3 * H, tailb, &bar_in[b]);
  };
  auto issue_sd = [&](int64_t t, int b) {
    const int64_t l = t / rows, r = t - l * rows;
    const T* src = (EPI == kEpiRhs ? a.rhs : a.y) + l * a.g.ls + r * N * 3;
    mbar_arrive_expect_tx(&bar_sd[b], (uint32_t)(N * 3 * sizeof(T)));
    bulk_load(real(b), src, (uint32_t)(N * 3 * sizeof(T)), &bar_sd[b]);
  };
  const int64_t t0 = blockIdx.x;
  if (tid == 0) {
    if (t0 < total) {
      issue_in(t0, 0);
      if (kSide) issue_sd(t0, 0);
    }
    if (t0 + G < total) issue_in(t0 + G, 1);
  }
  double acc = 0.0;
  int i = 0;
  for (int64_t t = t0; t < total; t += G, ++i) {
    const int b = i & 1;
    const uint32_t par = (i >> 1) & 1, par1 = ((i + 1) >> 1) & 1;
    const bool next = t + G < total;
    const int64_t l = t / rows, r = t - l * rows;
    if (!mbar_wait(&bar_in[b], par)) atomicOr(&fail_flag, 1);
    __syncthreads();
    if (fail_flag) {
      if (kSide) mbar_wait(&bar_sd[b], par);
      if (next) mbar_wait(&bar_in[b ^ 1], par1);
      break;
    }
    C* z = spec(b);
    // pack: Z[k] = E + i O, Z[H-k] = conj E + i conj O with E = X[k] +
    // conj X[H-k], O = (X[k] - conj X[H-k]) w^-k (imaginary parts of X[0]
    // and X[H] ignored, as a c2r transform does)
    for (int q = tid; q < K::PAIRS; q += K::THREADS) {
      const int k1 = q % N1, c = (q / N1) % 3, k2 = q / (3 * N1);
      const int k = k1 + N1 * k2;
      if (k > H / 2) continue;
      C x0 = z[lr_ipos<K>(k, c)], x1 = z[lr_ipos<K>(H - k, c)];
      if (k == 0) {
        x0.y = T(0);
        x1.y = T(0);
      }
      const T ex = x0.x + x1.x, ey = x0.y - x1.y;
      const C O = cmulc(mkc(x0.x - x1.x, x0.y + x1.y), tw[k]);
      z[lr_ipos<K>(k, c)] = mkc(ex - O.y, ey + O.x);
      if (k != 0 && 2 * k != H) z[lr_ipos<K>(H - k, c)] = mkc(ex + O.y, O.x - ey);
    }
    __syncthreads();
    lr_phase1<K, +1, N, T>(z, nullptr, tw, tid);
    __syncthreads();
    // the next tile's side row: its buffer's last store (two rows back) is
    // waited for here, long after it was issued
    if (tid == 0 && kSide && next) {
      bulk_wait_read();
      issue_sd(t + G, b ^ 1);
    }
    lr_phase2<K, +1, N, T>(z, tw, tid);
    __syncthreads();
    lr_phase3<K, +1, T>(z, tid);
    bool ok = true;
    if (kSide) ok = mbar_wait(&bar_sd[b], par);
    if (!ok) atomicOr(&fail_flag, 1);
    if (tid == 0) bulk_wait_read_1();  // the store two rows back has read real(b)
    __syncthreads();
    if (fail_flag) {
      if (next) {
        mbar_wait(&bar_in[b ^ 1], par1);
        if (kSide) mbar_wait(&bar_sd[b ^ 1], par1);
      }
      break;
    }
    T* y = real(b);
    T e0 = T(0), e1 = T(0), e2 = T(0);
    if (EPI == kEpiUpdate) {
      e0 = static_cast<T>(a.E[l * 3]);
      e1 = static_cast<T>(a.E[l * 3 + 1]);
      e2 = static_cast<T>(a.E[l * 3 + 2]);
    }
    for (int q = tid; q < 3 * H; q += K::THREADS) {
      const int k1 = q % N1, c = (q / N1) % 3, j2 = q / (3 * N1);
      const int jp = k1 + N1 * j2;
      const C v = z[lr_zpos<K>(jp, c)];
      T* p = y + jp * 6 + c;  // voxels 2 jp and 2 jp + 1, component c
      const T val[2] = {v.x, v.y};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const T s = mul_rn(a.scale, val[h]);
        if (EPI == kEpiUpdate) {
          const T ev = c == 0 ? e0 : (c == 1 ? e1 : e2);
          const T nv = sub_rn(ev, s);
          const double d = static_cast<double>(nv) - static_cast<double>(p[3 * h]);
          acc += d * d;
          p[3 * h] = nv;
        } else if (EPI == kEpiRhs) {
          p[3 * h] = sub_rn(p[3 * h], s);
        } else {
          p[3 * h] = s;
        }
      }
    }
    fence_async_shared();
    __syncthreads();
    if (tid == 0) {
      bulk_store(a.y + l * a.g.ls + r * N * 3, y, (uint32_t)(N * 3 * sizeof(T)));
      bulk_commit();
      if (t + 2 * G < total) issue_in(t + 2 * G, b);
    }
    if (EPI == kEpiUpdate && (!next || (t + G) / rows != l)) {
      const double s = block_sum(acc, red);
      if (tid == 0) a.partials[l * G + blockIdx.x] = s;
      acc = 0.0;
    }
  }
  if (tid == 0) bulk_wait_read();
}
