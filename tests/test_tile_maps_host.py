"""CPU restatements of the index maps of two register-tile kernels, checked
against numpy's FFT (no GPU; host logic only).

* The long-row kernels (janus_b200/csrc/jb_rows_long.cuh): a row of n reals
  per component is packed as z[j] = x[2j] + i x[2j+1] (n/2 points), the n/2 =
  N1 * 64 points are transformed in three phases on a tile whose k1 rows are
  PK complex apart, and the half spectrum is unpacked pair by pair (k, n/2-k)
  (r2c); the c2r side packs E + iO, runs the inverse phases in place and
  splits z back into even and odd voxels.  Each loop below follows the
  kernel's lane mapping and tile addresses, so a wrong position or twiddle
  index shows up as a wrong spectrum.
* The seven-phase Green tiles (green_axis0_r16_kernel): n0 = N1 * 8 * 8 with
  N1 = 3, 6, 8, 12, 16, forward transform, a per-coefficient s x s operator,
  inverse transform, against numpy.
"""
import numpy as np
import pytest


def _dft(v, sign):
    n = len(v)
    k = np.arange(n)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / n) @ v


def _w(n, i, sign=-1):
    return np.exp(sign * 2j * np.pi * i / n)


class _LongRow:
    def __init__(self, n, f64):
        self.n, self.H = n, n // 2
        self.N1 = self.H // 64
        self.PK = 192 + (1 if f64 else 2)

    def pos(self, k1, p, c):
        return k1 * self.PK + p * 3 + c

    def zpos(self, k, c):  # natural coefficient after phase 3
        k1, k2 = k % self.N1, k // self.N1
        return self.pos(k1, (k2 >> 3) + 8 * (k2 & 7), c)

    def ipos(self, k, c):  # natural index of the phase-1 input (k <= H: tail)
        return (k >> 6) * self.PK + (k & 63) * 3 + c

    def pairs(self):
        N1 = self.N1
        for q in range(3 * N1 * (self.H // (2 * N1) + 1)):
            k1, c, k2 = q % N1, (q // N1) % 3, q // (3 * N1)
            k = k1 + N1 * k2
            if k <= self.H // 2:
                yield c, k

    def phases(self, T, sign, raw=None):
        n, N1, PK = self.n, self.N1, self.PK
        for tid in range(192):  # phase 1: lane (c, j)
            c, j = tid % 3, tid // 3
            if raw is not None:
                v = np.array([raw[(2 * (j + 64 * m)) * 3 + c] + 1j * raw[(2 * (j + 64 * m) + 1) * 3 + c]
                              for m in range(N1)])
            else:
                v = np.array([T[m * PK + j * 3 + c] for m in range(N1)])
            v = _dft(v, sign)
            for k1 in range(N1):
                T[k1 * PK + j * 3 + c] = v[k1] * _w(n, 2 * j * k1, sign)
        for tid in range(N1 * 24):  # phase 2: lane (k1, c, ja)
            k1, c, ja = tid % N1, (tid // N1) % 3, tid // (3 * N1)
            idx = [k1 * PK + ja * 3 + c + 24 * jb for jb in range(8)]
            w = _dft(T[idx], sign)
            T[idx] = w * np.array([_w(n, (n // 64) * ja * kb, sign) for kb in range(8)])
        for tid in range(N1 * 24):  # phase 3: lane (k1, c, kb)
            k1, c, kb = tid % N1, (tid // N1) % 3, tid // (3 * N1)
            idx = [k1 * PK + kb * 24 + c + 3 * ja for ja in range(8)]
            T[idx] = _dft(T[idx], sign)

    def r2c(self, x):
        H = self.H
        T = np.full(self.N1 * self.PK, np.nan + 0j)
        self.phases(T, -1, raw=x.reshape(-1))
        X = np.full((H + 1) * 3, np.nan + 0j)
        for c, k in self.pairs():
            Z, Zh = T[self.zpos(k, c)], T[self.zpos(0 if k == 0 else H - k, c)]
            ax, ay = 0.5 * (Z.real + Zh.real), 0.5 * (Z.imag - Zh.imag)
            P = _w(self.n, k) * complex(Z.real - Zh.real, Z.imag + Zh.imag)
            X[k * 3 + c] = complex(ax + 0.5 * P.imag, ay - 0.5 * P.real)
            if 2 * k != H:
                X[(H - k) * 3 + c] = complex(ax - 0.5 * P.imag, -ay - 0.5 * P.real)
        return X.reshape(H + 1, 3)

    def c2r(self, X):
        H = self.H
        T = np.full(self.N1 * self.PK + 4, np.nan + 0j)
        for k in range(H + 1):
            for c in range(3):
                T[self.ipos(k, c)] = X[k, c]
        for c, k in self.pairs():
            x0, x1 = T[self.ipos(k, c)], T[self.ipos(H - k, c)]
            if k == 0:
                x0, x1 = complex(x0.real, 0.0), complex(x1.real, 0.0)
            ex, ey = x0.real + x1.real, x0.imag - x1.imag
            O = complex(x0.real - x1.real, x0.imag + x1.imag) * np.conj(_w(self.n, k))
            T[self.ipos(k, c)] = complex(ex - O.imag, ey + O.real)
            if k != 0 and 2 * k != H:
                T[self.ipos(H - k, c)] = complex(ex + O.imag, O.real - ey)
        self.phases(T, +1)
        y = np.zeros((self.n, 3))
        for q in range(3 * H):
            k1, c, j2 = q % self.N1, (q // self.N1) % 3, q // (3 * self.N1)
            jp = k1 + self.N1 * j2
            z = T[self.zpos(jp, c)]
            y[2 * jp, c], y[2 * jp + 1, c] = z.real, z.imag
        return y


@pytest.mark.parametrize("n", [384, 512, 768, 1024])
@pytest.mark.parametrize("f64", [True, False])
def test_long_row_maps(n, f64):
    rng = np.random.default_rng(n)
    S = _LongRow(n, f64)
    x = rng.standard_normal((n, 3))
    ref = np.fft.rfft(x, axis=0)
    X = S.r2c(x)
    assert np.abs(X - ref).max() <= 1e-12 * np.abs(ref).max()
    spec = ref.copy()
    spec[0] += 0.7j  # imaginary parts of X[0] and X[n/2] are ignored
    spec[-1] -= 0.3j
    y = S.c2r(spec)
    yref = np.fft.irfft(ref, n=n, axis=0) * n
    assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()


@pytest.mark.parametrize("N1", [3, 6, 8, 12, 16])
@pytest.mark.parametrize("dim", [2, 3])
def test_seven_phase_green_tile_maps(N1, dim):
    """Tile S[k1][p][c] (p = ja + 8 jb, then ja + 8 kb, then ka + 8 kb), six
    columns, pad 1 on the k1 stride; the phases and job maps of the kernel."""
    A = B = 8
    M = 64
    n0 = N1 * M
    WC, PJ = 6, 6
    PK = M * PJ + 1
    C = 6 if dim == 3 else 3
    rng = np.random.default_rng(N1 * 10 + dim)
    X = rng.standard_normal((n0, WC)) + 1j * rng.standard_normal((n0, WC))
    G = rng.standard_normal((WC // C, n0, C, C))
    G = G + np.transpose(G, (0, 1, 3, 2))

    def off(k1, p, c):
        return k1 * PK + p * PJ + c

    S = np.full(N1 * PK, np.nan + 0j)
    for t in range(WC * M):  # P1: lane (c, j)
        c, j = t % WC, t // WC
        v = _dft(np.array([X[j + M * m, c] for m in range(N1)]), -1)
        for k1 in range(N1):
            S[off(k1, j, c)] = v[k1] * _w(n0, j * k1)
    for job in range(N1 * A * WC):  # 2a: (k1, ja, c), over jb
        k1, ja, c = job % N1, (job // N1) % A, job // (N1 * A)
        idx = [off(k1, ja + A * jb, c) for jb in range(B)]
        S[idx] = _dft(S[idx], -1) * np.array([_w(n0, (n0 // M) * ja * kb) for kb in range(B)])
    for job in range(N1 * B * WC):  # 2a': (k1, kb, c), over ja
        k1, kb, c = job % N1, (job // N1) % B, job // (N1 * B)
        idx = [off(k1, ja + A * kb, c) for ja in range(A)]
        S[idx] = _dft(S[idx], -1)
    for job in range(N1 * M):  # 2b: (k1, kb, ka), the contraction at b0
        k1, kb, ka = job % N1, (job // N1) % B, job // (N1 * B)
        b0 = k1 + N1 * (kb + B * ka)
        for g in range(WC // C):
            idx = [off(k1, ka + A * kb, g * C + q) for q in range(C)]
            S[idx] = G[g, b0] @ S[idx]
    for job in range(N1 * B * WC):  # 2c'
        k1, kb, c = job % N1, (job // N1) % B, job // (N1 * B)
        idx = [off(k1, ja + A * kb, c) for ja in range(A)]
        S[idx] = _dft(S[idx], +1)
    for job in range(N1 * A * WC):  # 2c
        k1, ja, c = job % N1, (job // N1) % A, job // (N1 * A)
        idx = [off(k1, ja + A * kb, c) for kb in range(B)]
        tw = np.array([np.conj(_w(n0, (n0 // M) * ja * kb)) for kb in range(B)])
        S[idx] = _dft(S[idx] * tw, +1)
    Y = np.zeros_like(X)
    for t in range(WC * M):  # P3
        c, j = t % WC, t // WC
        v = np.array([S[off(k1, j, c)] * np.conj(_w(n0, j * k1)) for k1 in range(N1)])
        v = _dft(v, +1)
        for m in range(N1):
            Y[j + M * m, c] = v[m]
    F = np.fft.fft(X, axis=0)
    for g in range(WC // C):
        F[:, g * C:(g + 1) * C] = np.einsum("kij,kj->ki", G[g], F[:, g * C:(g + 1) * C])
    R = np.fft.ifft(F, axis=0) * n0
    assert np.abs(Y - R).max() <= 1e-12 * np.abs(R).max()
