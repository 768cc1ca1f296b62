"""Oracle: a CPU (numpy) restatement of the reference's Lippmann-Schwinger path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline legs of ``bench.py`` may import this module, and only as the
checker.  The janus_b200 product never imports ``oracle/``.

Parity is pinned: ``tests/test_oracle.py`` checks this module against the
reference's 18 golden ``apply`` files (sampled into ``tests/golden``), the
closed-form Green tensor of the reference's tests, the tutorial's published
C_1212 and, when it has been built, the reference's own Cython modules
compiled against ``oracle/fftw_shim`` (``oracle/_ref``).

Conventions follow the reference: Mandel components (xx, yy, xy) in 2D and
(xx, yy, zz, sqrt2*yz, sqrt2*zx, sqrt2*xy) in 3D, fields ``float64[n0, n1,
(n2,) s]`` with the component fastest.  FFTs are numpy's (``numpy.fft``
computes the same unnormalised DFT the reference obtains from FFTW).
"""
from __future__ import annotations

import itertools
import math

import numpy as np

SQRT2 = math.sqrt(2.0)


# --------------------------------------------------------------------------
# material (janus/material/elastic/linear/isotropic.pyx)
# --------------------------------------------------------------------------

def bulk_modulus(g: float, nu: float, dim: int) -> float:
    """Plane-strain (dim 2) or 3D bulk modulus, isotropic.pyx:74-77."""
    if dim == 2:
        return g / (1. - 2. * nu)
    return 2. / 3. * (1. + nu) / (1. - 2. * nu) * g


def green_aux(g: float, nu: float):
    """daux1..daux4 of isotropic.pyx:135-138."""
    return 1.0 / g, 0.5 / (g * (1.0 - nu)), 0.25 / g, 0.5 / g


def green_matrix(k, g: float, nu: float) -> np.ndarray:
    """Continuous Green operator for strains in Mandel form at wave-vector k.

    Restates _GreenOperatorForStrains2D.c_set_frequency (isotropic.pyx:158-182)
    and _GreenOperatorForStrains3D.c_set_frequency (isotropic.pyx:227-290),
    operation by operation; the zero wave-vector gives the zero matrix.
    """
    k = np.asarray(k, dtype=np.float64)
    d1, d2, d3, d4 = green_aux(g, nu)
    if k.shape[0] == 2:
        k0, k1 = float(k[0]), float(k[1])
        k0k0, k1k1 = k0 * k0, k1 * k1
        out = np.zeros((3, 3))
        if k0k0 + k1k1 == 0.:
            return out
        s = 1.0 / (k0k0 + k1k1)
        k0k0 *= s
        k1k1 *= s
        k0k1 = s * k0 * k1
        g00 = k0k0 * (d1 - d2 * k0k0)
        g11 = k1k1 * (d1 - d2 * k1k1)
        dummy = -d2 * k0k0 * k1k1
        g01 = dummy
        g22 = 2 * (d3 + dummy)
        g02 = SQRT2 * k0k1 * (d4 - d2 * k0k0)
        g12 = SQRT2 * k0k1 * (d4 - d2 * k1k1)
        out[:] = [[g00, g01, g02], [g01, g11, g12], [g02, g12, g22]]
        return out
    k0, k1, k2 = float(k[0]), float(k[1]), float(k[2])
    k0k0, k1k1, k2k2 = k0 * k0, k1 * k1, k2 * k2
    out = np.zeros((6, 6))
    if k0k0 + k1k1 + k2k2 == 0.:
        return out
    s = 1.0 / (k0k0 + k1k1 + k2k2)
    k0k0 *= s
    k1k1 *= s
    k2k2 *= s
    k1k2 = s * k1 * k2
    k2k0 = s * k2 * k0
    k0k1 = s * k0 * k1
    g = {}
    g[0, 0] = k0k0 * (d1 - d2 * k0k0)
    g[1, 1] = k1k1 * (d1 - d2 * k1k1)
    g[2, 2] = k2k2 * (d1 - d2 * k2k2)
    g[3, 3] = 2. * (d3 * (k1k1 + k2k2) - d2 * k1k1 * k2k2)
    g[4, 4] = 2. * (d3 * (k2k2 + k0k0) - d2 * k2k2 * k0k0)
    g[5, 5] = 2. * (d3 * (k0k0 + k1k1) - d2 * k0k0 * k1k1)
    g[0, 1] = -d2 * k0k0 * k1k1
    g[0, 2] = -d2 * k0k0 * k2k2
    g[0, 3] = -SQRT2 * d2 * k0k0 * k1k2
    g[0, 4] = SQRT2 * k2k0 * (d4 - d2 * k0k0)
    g[0, 5] = SQRT2 * k0k1 * (d4 - d2 * k0k0)
    g[1, 2] = -d2 * k1k1 * k2k2
    g[1, 3] = SQRT2 * k1k2 * (d4 - d2 * k1k1)
    g[1, 4] = -SQRT2 * d2 * k1k1 * k2k0
    g[1, 5] = SQRT2 * k0k1 * (d4 - d2 * k1k1)
    g[2, 3] = SQRT2 * k1k2 * (d4 - d2 * k2k2)
    g[2, 4] = SQRT2 * k2k0 * (d4 - d2 * k2k2)
    g[2, 5] = -SQRT2 * d2 * k2k2 * k0k1
    g[3, 4] = 2 * k0k1 * (d3 - d2 * k2k2)
    g[3, 5] = 2 * k2k0 * (d3 - d2 * k1k1)
    g[4, 5] = 2 * k1k2 * (d3 - d2 * k0k0)
    for (i, j), v in g.items():
        out[i, j] = v
        out[j, i] = v
    return out


# --------------------------------------------------------------------------
# discrete Green operators (janus/green.pyx)
# --------------------------------------------------------------------------

def truncated_wavevector(b, n, h: float) -> np.ndarray:
    """k(b) of TruncatedGreenOperator{2,3}D.c_set_frequency (green.pyx:434-445,
    507-523): k_i = s_i*(b_i - n_i) if 2*b_i > n_i else s_i*b_i, s_i = 2pi/(h n_i)."""
    k = np.empty(len(n))
    for i, (bi, ni) in enumerate(zip(b, n)):
        s = 2. * math.pi / (h * ni)
        k[i] = s * (bi - ni) if 2 * bi > ni else s * bi
    return k


def truncated_matrix(b, n, h, g, nu) -> np.ndarray:
    return green_matrix(truncated_wavevector(b, n, h), g, nu)


def filtered_matrix(b, n, h, g, nu) -> np.ndarray:
    """Filtered Green operator at index b: the 2^d-alias weighted sum of
    FilteredGreenOperator{2,3}D.c_set_frequency (green.pyx:609-670, 732-910),
    w = prod_i cos^2(h k_i / 4) over k_i in {s_i (b_i - n_i), s_i b_i}.
    The sum is accumulated alias by alias in the reference's order (the alias
    with all components negative first, the last component varying fastest)."""
    dim = len(n)
    s = [2. * math.pi / (h * ni) for ni in n]
    parts = []
    for i in range(dim):
        kneg = s[i] * (b[i] - n[i])
        kpos = s[i] * b[i]
        wneg = math.cos(0.25 * h * kneg)
        wneg *= wneg
        wpos = math.cos(0.25 * h * kpos)
        wpos *= wpos
        parts.append(((kneg, wneg), (kpos, wpos)))
    acc = None
    for choice in itertools.product((0, 1), repeat=dim):
        k = np.array([parts[i][c][0] for i, c in enumerate(choice)])
        w = parts[0][choice[0]][1]
        for i in range(1, dim):
            w *= parts[i][choice[i]][1]
        term = w * green_matrix(k, g, nu)
        acc = term if acc is None else acc + term
    return acc


def willot_wavevector(b, n, h: float) -> np.ndarray:
    """k(b) of FiniteDifferences{2,3}D.c_set_frequency (green.pyx:983-989,
    1001-1016): phi_i = 0.5*s_i*h*b_i (b_i not wrapped), k_0 = sin(phi_0)
    cos(phi_1) [cos(phi_2)], k_1 = cos(phi_0) sin(phi_1) [cos(phi_2)],
    k_2 = cos(phi_0) cos(phi_1) sin(phi_2); products left to right."""
    dim = len(n)
    phi = [0.5 * (2. * math.pi / (h * ni)) * h * bi for bi, ni in zip(b, n)]
    c = [math.cos(v) for v in phi]
    sn = [math.sin(v) for v in phi]
    if dim == 2:
        return np.array([sn[0] * c[1], c[0] * sn[1]])
    return np.array([sn[0] * c[1] * c[2], c[0] * sn[1] * c[2], c[0] * c[1] * sn[2]])


def willot_matrix(b, n, h, g, nu) -> np.ndarray:
    return green_matrix(willot_wavevector(b, n, h), g, nu)


def _half_spectrum_k(n, h):
    """Per-axis truncated wave-numbers on the r2c half spectrum."""
    ks = []
    for i, ni in enumerate(n):
        s = 2. * np.pi / (h * ni)
        nb = ni if i < len(n) - 1 else ni // 2 + 1
        b = np.arange(nb)
        ks.append(np.where(2 * b > ni, s * (b - ni), s * b))
    return ks


def _green_field(kgrid, g, nu):
    """Vectorised green_matrix over a grid of wave-vectors (same formulas)."""
    dim = len(kgrid)
    d1, d2, d3, d4 = green_aux(g, nu)
    kk = [kc * kc for kc in kgrid]
    tot = kk[0] + kk[1] + (kk[2] if dim == 3 else 0.)
    zero = tot == 0.
    s = np.where(zero, 0., 1.0 / np.where(zero, 1., tot))
    if dim == 2:
        k0k0, k1k1 = kk[0] * s, kk[1] * s
        k0k1 = s * kgrid[0] * kgrid[1]
        G = np.zeros(tot.shape + (3, 3))
        G[..., 0, 0] = k0k0 * (d1 - d2 * k0k0)
        G[..., 1, 1] = k1k1 * (d1 - d2 * k1k1)
        dummy = -d2 * k0k0 * k1k1
        G[..., 0, 1] = G[..., 1, 0] = dummy
        G[..., 2, 2] = 2 * (d3 + dummy)
        G[..., 0, 2] = G[..., 2, 0] = SQRT2 * k0k1 * (d4 - d2 * k0k0)
        G[..., 1, 2] = G[..., 2, 1] = SQRT2 * k0k1 * (d4 - d2 * k1k1)
        G[zero] = 0.
        return G
    k0k0, k1k1, k2k2 = kk[0] * s, kk[1] * s, kk[2] * s
    k1k2 = s * kgrid[1] * kgrid[2]
    k2k0 = s * kgrid[2] * kgrid[0]
    k0k1 = s * kgrid[0] * kgrid[1]
    G = np.zeros(tot.shape + (6, 6))

    def put(i, j, v):
        G[..., i, j] = v
        G[..., j, i] = v
    put(0, 0, k0k0 * (d1 - d2 * k0k0))
    put(1, 1, k1k1 * (d1 - d2 * k1k1))
    put(2, 2, k2k2 * (d1 - d2 * k2k2))
    put(3, 3, 2. * (d3 * (k1k1 + k2k2) - d2 * k1k1 * k2k2))
    put(4, 4, 2. * (d3 * (k2k2 + k0k0) - d2 * k2k2 * k0k0))
    put(5, 5, 2. * (d3 * (k0k0 + k1k1) - d2 * k0k0 * k1k1))
    put(0, 1, -d2 * k0k0 * k1k1)
    put(0, 2, -d2 * k0k0 * k2k2)
    put(0, 3, -SQRT2 * d2 * k0k0 * k1k2)
    put(0, 4, SQRT2 * k2k0 * (d4 - d2 * k0k0))
    put(0, 5, SQRT2 * k0k1 * (d4 - d2 * k0k0))
    put(1, 2, -d2 * k1k1 * k2k2)
    put(1, 3, SQRT2 * k1k2 * (d4 - d2 * k1k1))
    put(1, 4, -SQRT2 * d2 * k1k1 * k2k0)
    put(1, 5, SQRT2 * k0k1 * (d4 - d2 * k1k1))
    put(2, 3, SQRT2 * k1k2 * (d4 - d2 * k2k2))
    put(2, 4, SQRT2 * k2k0 * (d4 - d2 * k2k2))
    put(2, 5, -SQRT2 * d2 * k2k2 * k0k1)
    put(3, 4, 2 * k0k1 * (d3 - d2 * k2k2))
    put(3, 5, 2 * k2k0 * (d3 - d2 * k1k1))
    put(4, 5, 2 * k1k2 * (d3 - d2 * k0k0))
    G[zero] = 0.
    return G


def spectral_green_field(n, h, g, nu, variant="truncated") -> np.ndarray:
    """Gamma-hat on the r2c half spectrum, shape (n0, [n1,] n_last//2+1, s, s).

    truncated: the k-map of green.pyx:464-481 / 542-566 (Nyquist -> +pi/h);
    filtered: the 2^d-alias weighted sum of green.pyx:609-670 / 732-910;
    willot: the finite-difference wave-vector of green.pyx:976-1036.
    """
    dim = len(n)
    if variant == "truncated":
        kgrid = np.meshgrid(*_half_spectrum_k(n, h), indexing="ij")
        return _green_field(kgrid, g, nu)
    if variant == "willot":
        cs, sn = [], []
        for i, ni in enumerate(n):
            nb = ni if i < dim - 1 else ni // 2 + 1
            phi = 0.5 * (2. * np.pi / (h * ni)) * h * np.arange(nb)
            cs.append(np.cos(phi))
            sn.append(np.sin(phi))
        if dim == 2:
            C0, C1 = np.meshgrid(cs[0], cs[1], indexing="ij")
            S0, S1 = np.meshgrid(sn[0], sn[1], indexing="ij")
            return _green_field([S0 * C1, C0 * S1], g, nu)
        C0, C1, C2 = np.meshgrid(*cs, indexing="ij")
        S0, S1, S2 = np.meshgrid(*sn, indexing="ij")
        return _green_field([S0 * C1 * C2, C0 * S1 * C2, C0 * C1 * S2], g, nu)
    acc = None
    s = [2. * np.pi / (h * ni) for ni in n]
    axes = []
    for i, ni in enumerate(n):
        nb = ni if i < dim - 1 else ni // 2 + 1
        b = np.arange(nb)
        kneg, kpos = s[i] * (b - ni), s[i] * b
        wneg = np.cos(0.25 * h * kneg) ** 2
        wpos = np.cos(0.25 * h * kpos) ** 2
        axes.append(((kneg, wneg), (kpos, wpos)))
    for choice in itertools.product((0, 1), repeat=dim):
        kgrid = np.meshgrid(*[axes[i][c][0] for i, c in enumerate(choice)],
                            indexing="ij")
        wgrid = np.meshgrid(*[axes[i][c][1] for i, c in enumerate(choice)],
                            indexing="ij")
        w = wgrid[0]
        for i in range(1, dim):
            w = w * wgrid[i]
        term = w[..., None, None] * _green_field(kgrid, g, nu)
        acc = term if acc is None else acc + term
    return acc


def green_apply(x, g, nu, h=1.0, variant="truncated", G=None) -> np.ndarray:
    """y = F^-1[Gamma-hat . F[x]] for x of shape (n0, n1[, n2], s).

    Restates DiscreteGreenOperator{2,3}D.c_apply (green.pyx:185-216, 356-390)
    and the truncated fused loops (green.pyx:456-495, 534-580): r2c of each
    component, Gamma-hat applied to the real and imaginary parts of every
    half-spectrum coefficient, c2r with the 1/N scaling of
    janus/fft/serial/_serial_fft.pyx:74, 174-175.
    """
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[:-1]
    axes = tuple(range(len(n)))
    if G is None:
        G = spectral_green_field(n, h, g, nu, variant)
    X = np.fft.rfftn(x, axes=axes)
    Y = np.einsum("...ij,...j->...i", G, X.real) + 1j * np.einsum(
        "...ij,...j->...i", G, X.imag)
    return np.fft.irfftn(Y, s=n, axes=axes)


# --------------------------------------------------------------------------
# local operators (janus/operators.pyx)
# --------------------------------------------------------------------------

def isotropic_tr(sph: float, dev: float, dim: int) -> float:
    """tr = (sph - dev) / dim, operators.pyx:299."""
    return (sph - dev) / float(dim)


def isotropic_apply(x, sph, dev, dim) -> np.ndarray:
    """FourthRankIsotropicTensor{2,3}D.c_apply (operators.pyx:317-324,
    354-365), vectorised; ``sph``/``dev`` broadcast against x[..., 0]."""
    x = np.asarray(x, dtype=np.float64)
    sph = np.asarray(sph, dtype=np.float64)
    dev = np.asarray(dev, dtype=np.float64)
    tr = (sph - dev) / float(dim)
    y = np.empty_like(x)
    if dim == 2:
        aux = tr * (x[..., 0] + x[..., 1])
        y[..., 0] = aux + dev * x[..., 0]
        y[..., 1] = aux + dev * x[..., 1]
        y[..., 2] = dev * x[..., 2]
    else:
        aux = tr * (x[..., 0] + x[..., 1] + x[..., 2])
        for i in range(3):
            y[..., i] = aux + dev * x[..., i]
        for i in range(3, 6):
            y[..., i] = dev * x[..., i]
    return y


def phase_apply(x, phase, sph_table, dev_table, dim) -> np.ndarray:
    """BlockDiagonalOperator{2,3}D.c_apply (operators.pyx:657-664, 708-716)
    over a phase map: voxel v uses isotropic_4(sph[phase[v]], dev[phase[v]])."""
    phase = np.asarray(phase)
    sph = np.asarray(sph_table, dtype=np.float64)[phase]
    dev = np.asarray(dev_table, dtype=np.float64)[phase]
    return isotropic_apply(x, sph, dev, dim)


def cubic2d_matrix(t1111, t1122, t1212, theta) -> np.ndarray:
    """Mandel matrix of FourthRankCubicTensor2D (operators.pyx:413-450), same
    operation order."""
    c = math.cos(4 * theta)
    s = math.sin(4 * theta)
    aux = t1111 - t1122 - 2 * t1212
    t11 = 0.25 * (3 * t1111 + t1122 + 2 * t1212 + c * aux)
    t12 = 0.25 * (t1111 + 3 * t1122 - 2 * t1212 - c * aux)
    t13 = 0.25 * math.sqrt(2.0) * s * aux
    t23 = -t13
    t33 = 0.50 * (t1111 - t1122 + 2 * t1212 - c * aux)
    return np.array([[t11, t12, t13], [t12, t11, t23], [t13, t23, t33]])


def block_linear_apply(a, x, transpose=False) -> np.ndarray:
    """BlockDiagonalLinearOperator{2,3}D.c_apply / c_apply_transpose
    (operators.pyx:739-774, 823-861): y[v,i] = sum_j a[v,i,j] x[v,j] summed in
    j order (or a[v,j,i] for the transpose)."""
    a = np.asarray(a, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    if transpose:
        a = np.swapaxes(a, -1, -2)
    y = np.zeros(a.shape[:-1])
    for j in range(a.shape[-1]):
        y = y + a[..., :, j] * x[..., None, j]
    return y


# --------------------------------------------------------------------------
# basic fixed-point scheme (sphinx/tutorials/square_basic/square_basic.py)
# --------------------------------------------------------------------------

def basic_scheme(phase, sph_table, dev_table, g0, nu0, avg_eps, num_iter,
                 h=1.0, variant="truncated", tol=None, callback=None, mats=None):
    """The tutorial loop square_basic.py:83-97 with a phase-map local operator.

    eps0 = E; eps_{k+1} = E - Gamma0[(C - C0):eps_k];
    res_k = ||eps_{k+1} - eps_k|| / (sqrt(N) ||E||) (square_basic.py:86, 91).
    Stops after ``num_iter`` iterations, or earlier once res_k <= tol.
    Returns (eps, residuals, mean_tau) where mean_tau is the mean of
    (C - C0):eps over the grid for the final eps (square_basic.py:95-96).
    With ``mats`` (nphase x s x s), phase p's local operator is the matrix
    mats[p] (BlockDiagonalOperator over LinearOperator / cubic tensors)
    instead of isotropic_4(sph[p], dev[p]).
    """
    phase = np.asarray(phase)
    n = phase.shape
    dim = len(n)
    avg_eps = np.asarray(avg_eps, dtype=np.float64)
    G = spectral_green_field(n, h, g0, nu0, variant)
    if mats is not None:
        mats = np.asarray(mats, dtype=np.float64)

        def local(x):
            return block_linear_apply(mats[phase], x)
    else:
        def local(x):
            return phase_apply(x, phase, sph_table, dev_table, dim)
    eps = np.empty(n + (avg_eps.shape[0],))
    eps[...] = avg_eps
    num_cells = int(np.prod(n))
    normalization = 1 / np.sqrt(num_cells) / np.linalg.norm(avg_eps)
    res = []
    for it in range(num_iter):
        tau = local(eps)
        y = green_apply(tau, g0, nu0, h, variant, G=G)
        new_eps = avg_eps - y
        res.append(normalization * np.linalg.norm(new_eps - eps))
        eps = new_eps
        if callback is not None:
            callback(it, eps)
        if tol is not None and res[-1] <= tol:
            break
    tau = local(eps)
    mean_tau = np.mean(tau, axis=tuple(range(dim)))
    return eps, np.asarray(res), mean_tau


def delta_c(mat_g, mat_nu, g0, nu0, dim):
    """(sph, dev) of C - C0 as built in square_basic.py:26-29:
    isotropic_4(dim*(k - k0), 2*(g - g0), dim)."""
    k = bulk_modulus(mat_g, mat_nu, dim)
    k0 = bulk_modulus(g0, nu0, dim)
    return dim * (k - k0), 2 * (mat_g - g0)


# --------------------------------------------------------------------------
# gradients with respect to a stiffness field (no reference counterpart: the
# reference has no derivatives; these restate the adjoint of its basic
# scheme, square_basic.py:83-97, and check it by differencing that scheme)
# --------------------------------------------------------------------------

def local_gradient(eps, zeta, dim, scale):
    """Per voxel, scale * sum over load cases of the contractions of the
    adjoint strain zeta and the strain eps with the isotropic projectors
    J and K of operators.pyx:257-303 (Mandel form):
        out[..., 0] = scale * sum_j tr(zeta_j) tr(eps_j) / dim
        out[..., 1] = scale * sum_j (zeta_j . eps_j - tr(zeta_j) tr(eps_j) / dim)
    eps, zeta: (nload, *grid, s)."""
    eps = np.asarray(eps, dtype=np.float64)
    zeta = np.asarray(zeta, dtype=np.float64)
    tre = eps[..., :dim].sum(axis=-1)
    trz = zeta[..., :dim].sum(axis=-1)
    j = tre * trz / dim
    k = (zeta * eps).sum(axis=-1) - j
    return scale * np.stack([j.sum(axis=0), k.sum(axis=0)], axis=-1)


def field_tables(mu, nu, g0, nu0):
    """(phase map, sph, dev) of C - C0 for a per-voxel shear modulus mu at a
    uniform Poisson ratio nu: one table entry per voxel (square_basic.py:26-29
    applied voxel by voxel)."""
    mu = np.asarray(mu, dtype=np.float64)
    dim = mu.ndim
    phase = np.arange(mu.size).reshape(mu.shape)
    k = bulk_modulus(mu.ravel(), nu, dim)
    k0 = bulk_modulus(g0, nu0, dim)
    return phase, dim * (k - k0), 2 * (mu.ravel() - g0)


def field_mean_stress(mu, nu, g0, nu0, avg_eps, num_iter, tol, variant="truncated"):
    """Mean stress C0:E + <tau> of a stiffness field under one load case,
    by the oracle basic scheme."""
    phase, sph, dev = field_tables(mu, nu, g0, nu0)
    dim = np.asarray(mu).ndim
    _, res, tau = basic_scheme(phase, sph, dev, g0, nu0, avg_eps, num_iter,
                               variant=variant, tol=tol)
    k0 = bulk_modulus(g0, nu0, dim)
    return isotropic_apply(np.asarray(avg_eps, dtype=np.float64), dim * k0, 2 * g0, dim) + tau
