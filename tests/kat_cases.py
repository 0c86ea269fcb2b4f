"""Known-answer cases of the reference's unit tests for the extrapolation path, rebuilt as data.

Each case gives the inputs in the reference's host argument order and the expected values.
  cpu_*  unittests/test_cpp_src.py:115-295   (CPU library, also test_py_src_extrapolation.py:150-314)
  gpu_*  unittests/test_cpp_src_cuda.py:23-211 and :216-384 (device libraries; image and the
         in-place wavefields of the revOp library)
  py_*   unittests/test_py_src_extrapolation.py:52-148 (real-valued operators and pulses)
Tolerance of the reference tests: 1e-5 absolute (test_cpp_src.py:13).
"""
import numpy as np

SDELTA = 1e-5


def _cpu_base(nextrap=1, nz=1):
    ns, nw, nx, M = 1, 2, 4, 1
    op_f = np.zeros((nextrap, nw, nx, 3), dtype=np.complex64)
    op_b = np.zeros_like(op_f)
    pf = np.array([[1 + 1j, 2 + 2j, 3 + 3j, 4 + 4j], [5 + 5j, 6 + 6j, 7 + 7j, 8 + 8j]], dtype=np.complex64)
    return dict(ns=ns, nextrap=nextrap, nz=nz, nx=nx, nf=nw, nt=nw, M=M), op_f, op_b, pf


def cpu_cases():
    cases = []
    # test_cpp_src_extrapolate_1 (test_cpp_src.py:115-148): point 0, complex frequencies
    d, f, b, pf = _cpu_base()
    freq = np.array([1 + 1j, 2 + 0j], dtype=np.complex64)
    for i in range(2):
        f[0, i, 0, :] = freq[i]
        b[0, i, 0, :] = freq[i]
    pb = np.array([[1 - 1j, 2 - 2j, 3 - 3j, 4 - 4j], [5 + 5j, 6 + 6j, 7 + 7j, 8 + 8j]], dtype=np.complex64)
    cases.append(("cpu_1", d, f, b, pf, pb, {(0, 0): 968.0}))
    # test_cpp_src_extrapolate_2..4 (:150-256)
    freq = np.array([1 + 0j, 2 + 0j], dtype=np.complex64)
    for name, pts, exp in (("cpu_2", [2], {(0, 2): -3690.0}), ("cpu_3", [3], {(0, 3): -1898.0}),
                           ("cpu_4", [2, 3], {(0, 2): -3690.0, (0, 3): -1898.0})):
        d, f, b, pf = _cpu_base()
        for i in range(2):
            for p in pts:
                f[0, i, p, :] = freq[i]
                b[0, i, p, :] = -freq[i]
        cases.append((name, d, f, b, pf, pf.copy(), exp))
    # test_cpp_src_extrapolate_5 (:258-295): two depths
    d, f, b, pf = _cpu_base(nextrap=2, nz=2)
    for l in range(2):
        for i in range(2):
            f[l, i, 3, :] = freq[i]
            b[l, i, 3, :] = -freq[i]
    cases.append(("cpu_5", d, f, b, pf, pf.copy(), {(0, 3): -1898.0, (1, 3): 7298.0}))
    return cases


def gpu_cases():
    """Device-order cases; returned in host order fields plus expected wavefield values."""
    cases = []

    def base(nextrap, nz, nf, nx, M, col, first_row, rows):
        L = 2 * M + 1
        op = np.zeros((nextrap, nf, nx, L), dtype=np.complex64)
        op2 = np.zeros_like(op)
        for l in range(nextrap):
            for i in range(nf):
                for v in range(3 + M):
                    op2[l, i, col, v] = 1 + 1j
                    op[l, i, col, v] = 1 - 1j
        pulse = np.zeros((nf, nx), dtype=np.complex64)
        pulse[first_row, rows] = np.array([1, 2, 3, 4], dtype=np.complex64)
        pulse2 = np.zeros_like(pulse)
        pulse2[1, rows] = np.array([5 + 1j, 6 - 2j, 7, 8], dtype=np.complex64)
        return dict(ns=1, nextrap=nextrap, nz=nz, nx=nx, nf=nf, nt=nf, M=M), op, op2, pulse, pulse2

    # test_cuda_extrapolation_rearranged_operators_1 (test_cpp_src_cuda.py:23-55)
    d, op, op2, p, p2 = base(1, 5, 2, 6, 2, 1, 1, slice(0, 4))
    cases.append(("gpu_1", d, op, op2, p, p2, {(0, 1): 20.0}, {"pulse": ((1, 1), 10 - 10j), "pulse2": ((1, 1), 27 + 25j)}))
    # _2 (:57-91): source in row 0 only -> zero image
    d, op, op2, p, p2 = base(1, 5, 2, 6, 2, 1, 0, slice(0, 4))
    cases.append(("gpu_2", d, op, op2, p, p2, "zero", {"pulse": ((0, 1), 10 - 10j), "pulse2": ((1, 1), 27 + 25j)}))
    # _3 (:93-129)
    d, op, op2, p, p2 = base(1, 5, 2, 6, 2, 2, 1, slice(1, 5))
    cases.append(("gpu_3", d, op, op2, p, p2, {(0, 2): 20.0}, {"pulse": ((1, 2), 10 - 10j), "pulse2": ((1, 2), 27 + 25j)}))
    # _4 (:131-170): two depths
    d, op, op2, p, p2 = base(2, 5, 2, 6, 2, 2, 1, slice(1, 5))
    cases.append(("gpu_4", d, op, op2, p, p2, {(0, 2): 20.0, (1, 2): -1040.0},
                  {"pulse": ((1, 2), 0 - 20j), "pulse2": ((1, 2), 2 + 52j)}))
    # _5 (:172-211): larger grid, M = 5
    d, op, op2, p, p2 = base(2, 10, 20, 16, 5, 2, 1, slice(1, 5))
    cases.append(("gpu_5", d, op, op2, p, p2, {(0, 2): 20.0, (1, 2): -1040.0},
                  {"pulse": ((1, 2), 0 - 20j), "pulse2": ((1, 2), 2 + 52j)}))
    return cases


def py_float_cases():
    """test_py_src_extrapolation.py:52-148 (real operators/pulses, run as complex with zero imag)."""
    cases = []
    freq = np.array([1, 2])
    pulse = np.array([[1, 2, 3, 4], [5, 6, 7, 8]], dtype=np.complex64)

    def mk():
        return np.zeros((1, 2, 4, 3), dtype=np.complex64), np.zeros((1, 2, 4, 3), dtype=np.complex64)

    f, b = mk()
    for i in range(2):
        f[0, i, 1, :] = freq[i]
        b[0, i, 1, :] = -freq[i]
    cases.append(("py_1", f, b, {(0, 1): -1332.0}))
    f2 = f.copy()
    for i in range(2):
        f2[0, i, 1, :] = np.array([0, 0, 1])
    cases.append(("py_2", f2, b.copy(), {(0, 1): -270.0}))
    f, b = mk()
    for i in range(2):
        f[0, i, 0, :] = freq[i]
        b[0, i, 0, :] = -freq[i]
    cases.append(("py_3", f, b, {(0, 0): -493.0}))
    return [(n, dict(ns=1, nextrap=1, nz=1, nx=4, nf=2, nt=2, M=1), f, b, pulse.copy(), pulse.copy(), e)
            for n, f, b, e in cases]


def check_image(image, expected, nz, nx):
    """image (nz, nx); expected dict {(l, x): value} or 'zero'.  Every other entry must be zero."""
    img = np.asarray(image).reshape(nz, nx)
    if expected == "zero":
        return np.all(np.abs(img) <= SDELTA), "image not zero"
    for (l, x), v in expected.items():
        if abs(img[l, x] - v) > SDELTA:
            return False, f"image[{l},{x}] = {img[l, x]} expected {v}"
    mask = np.ones_like(img, dtype=bool)
    for (l, x) in expected:
        mask[l, x] = False
    if np.any(np.abs(img[mask]) > SDELTA):
        return False, "non-zero image outside the expected points"
    return True, ""
