"""Host-side operator design: WLSQ FIR operators, phase-shift operators and the compact table.

Restates py_src/operatorsPreparation/{preparation,util}.py of the reference with numpy arrays
instead of per-element numba loops, keeping every arithmetic step (and dtype) of the reference so
that the tables agree with the reference's to rounding (bitwise for the table rows, which use the
same numpy call per row as preparation.py:110).

The dense (nextrap, nw, nx, 2M+1) table of preparation.py:101-115 is, for the all-symmetric
operator choice main.py:66 uses (gIdx = M everywhere, util.py:19-21), a gather of the compact
(nk, 2M+1) table built here: T[l, j, i, :] = compact[find_nearest(kappa, w[j] / v[l, i])].
The CUDA library consumes the compact table directly.
"""
import cmath
import math

import numpy as np


def find_nearest(array, value):
    """util.py:5-8: index of the element nearest to value, first one on ties."""
    return int(np.abs(np.asarray(array) - value).argmin())


def create_kappa(cmax, cmin, dw, wmax, dense):
    """util.py:39-45: uniform wavenumber grid kappa[i] = i * deltak covering [0, wmax/cmin]."""
    deltak = dw / cmax / dense
    maxk = wmax / cmin
    nk = int(maxk / deltak) + math.ceil(cmax / cmin)
    return np.arange(nk, dtype=np.float64) * deltak


def kappa_grid(nk, dk):
    """kappa[i] = i*dk as the reference forms it (float64 products)."""
    return np.arange(nk, dtype=np.float64) * dk


def nearest_index(omega, velocity, dk, nk):
    """Vectorised find_nearest(kappa, w/v) for kappa[i] = i*dk: returns int array of w/v's shape.

    Exactly numpy's argmin semantics (ties -> lower index), checked over the candidates around
    floor(value/dk), with value = w / v in float64 as preparation.py:109 computes it.
    """
    value = np.asarray(omega, dtype=np.float64) / np.asarray(velocity, dtype=np.float64)
    q = value / dk
    i0 = np.where(q > 0, np.floor(np.minimum(q, nk - 1)), 0).astype(np.int64)
    best = np.clip(i0 - 1, 0, nk - 1)
    bestd = np.abs(best * dk - value)
    for off in (0, 1, 2):
        cand = np.clip(i0 + off, 0, nk - 1)
        d = np.abs(cand * dk - value)
        better = d < bestd
        best = np.where(better, cand, best)
        bestd = np.where(better, d, bestd)
    return best


def make_forw_ps_operators(kappa, wavenumbers, dz):
    """preparation.py:10-25: psOp[i, j] = exp(-i kz dz), kz = sqrt(k^2 - kx^2) or -i sqrt(kx^2 - k^2)."""
    k = np.asarray(kappa, dtype=np.float64)[:, None]
    kx = np.asarray(wavenumbers, dtype=np.float64)[None, :]
    prop = np.abs(k) >= np.abs(kx)
    kz = np.where(prop, np.sqrt(np.where(prop, k ** 2 - kx ** 2, 0.0)) + 0j,
                  -1j * np.sqrt(np.where(prop, 0.0, kx ** 2 - k ** 2)))
    return np.exp(-1j * kz * dz).astype(np.complex64)


def make_back_ps_operators(kappa, wavenumbers, dz):
    """preparation.py:29-44: psOp[i, j] = exp(+i kz dz), kz = sqrt(k^2 - kx^2) or +i sqrt(kx^2 - k^2)."""
    k = np.asarray(kappa, dtype=np.float64)[:, None]
    kx = np.asarray(wavenumbers, dtype=np.float64)[None, :]
    prop = np.abs(k) >= np.abs(kx)
    kz = np.where(prop, np.sqrt(np.where(prop, k ** 2 - kx ** 2, 0.0)) + 0j,
                  1j * np.sqrt(np.where(prop, 0.0, kx ** 2 - k ** 2)))
    return np.exp(1j * kz * dz).astype(np.complex64)


def create_wlsq_operators(N, M, kx, x, only_symmetric=False):
    """preparation.py:64-97: op[g] = pinv(G^H G) G^H for the 2M+1 one-sided/symmetric stencils.

    gamma[g, n, m] = exp(i kx[n] x[m]) on the stencil's support, complex64 as in the reference.
    With only_symmetric=True only op[M] (the operator main.py:66 selects everywhere) is formed and
    the others are left zero.
    """
    L = 2 * M + 1
    Nk = 2 * N + 1
    kx = np.asarray(kx)
    x = np.asarray(x)
    # element by element with cmath.exp as preparation.py:75-90 does: numpy's vectorised complex exp
    # differs from it in the last bits for some arguments, which survives the cast to complex64
    full = np.array([[cmath.exp(1j * kx[n] * x[m]) for m in range(L)] for n in range(Nk)],
                    dtype=np.complex128).astype(np.complex64)  # (Nk, L)
    op = np.zeros((L, L, Nk), dtype=np.complex64)
    gs = [M] if only_symmetric else range(L)
    for g in gs:
        mask = np.ones(L, dtype=bool)
        if g < M:
            mask = np.arange(L) > M - g - 1
        elif g > M:
            mask = np.arange(L) < M + M - (g - M - 1)
        gamma = np.where(mask[None, :], full, np.complex64(0))
        gamma_h = np.transpose(np.conjugate(gamma))
        op[g] = np.matmul(np.linalg.pinv(np.matmul(gamma_h, gamma)), gamma_h)
    return op


def compact_table(op_sym, ps_op):
    """Row k = op_sym @ ps_op[k] with the same numpy call per row as preparation.py:110."""
    nk = ps_op.shape[0]
    out = np.empty((nk, op_sym.shape[0]), dtype=np.complex64)
    for k in range(nk):
        out[k] = np.matmul(op_sym, ps_op[k, :])
    return out


def dense_table(compact, omega, velocity, nextrap, x0=0, width=None, nk=None, dk=None, conj=False):
    """Gather the dense (nextrap, nf, width, L) table of preparation.py:101-115 from a compact table."""
    nf = len(omega)
    nx = velocity.shape[1]
    width = nx if width is None else width
    nk = compact.shape[0] if nk is None else nk
    idx = nearest_index(np.asarray(omega)[None, :, None], velocity[:nextrap, None, x0:x0 + width], dk, nk)
    out = compact[idx]
    return np.conjugate(out) if conj else out


def odd_wavenumber_grid(nx, dx):
    """kx grid with an odd number of points for any nx (the reference's N = int((nx-1)/2) gives
    nx-1 points for even nx, problemConfig.py:42-43, which breaks preparation.py:110).  Returns
    (N, kx) with 2N+1 = nx for odd nx and nx+1 for even nx, spacing 2*pi/(nx*dx)."""
    N = nx // 2 if nx % 2 == 0 else (nx - 1) // 2
    Nk = 2 * N + 1
    dkx = 2.0 * math.pi / float(nx * dx)
    kx = np.fft.fftfreq(Nk) * Nk * dkx
    return N, kx


def local_x(M, dx):
    """problemConfig.py:51-53: stencil positions (-M..M)*dx as float32."""
    xmin = -M * dx
    return np.array([xmin + i * dx for i in range(2 * M + 1)], dtype=np.float32)


def design_compact_table(nx, dx, dz, M, nk, dk, back=False):
    """Compact forward (or backward) operator table for a model of width nx: (nk, 2M+1) complex64."""
    N, kx = odd_wavenumber_grid(nx, dx)
    op = create_wlsq_operators(N, M, kx, local_x(M, dx), only_symmetric=True)
    kappa = kappa_grid(nk, dk)
    ps = make_back_ps_operators(kappa, kx, dz) if back else make_forw_ps_operators(kappa, kx, dz)
    return compact_table(op[M], ps)
