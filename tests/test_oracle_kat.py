"""Pins the CPU oracle (oracle/wlsq_oracle.c) to the reference's known answers, and to the
reference's own CPU library built from its sources (oracle/_ref) when that library is present."""
import numpy as np
import pytest

from oracle import oracle
from tests import kat_cases as K


def _run_f32(d, f, b, pf, pb):
    img = np.zeros((d["ns"], d["nz"], d["nx"]), dtype=np.float32)
    w, s = pf.copy(), pb.copy()
    oracle.extrapolate_f32(d["ns"], d["nextrap"], d["nz"], d["nx"], d["nf"], d["nt"], d["M"], f, b, w, s, img)
    return img, w, s


def _run_ref(d, f, b, pf, pb, v0=False):
    img = np.zeros((d["ns"], d["nz"], d["nx"]), dtype=np.float32)
    w, s = pf.copy(), pb.copy()
    oracle.ref_extrapolate(d["ns"], d["nextrap"], d["nz"], d["nx"], d["nf"], d["nt"], d["M"], f, b, w, s, img, v0=v0)
    return img, w, s


ALL = K.cpu_cases() + [c[:7] for c in K.gpu_cases()] + K.py_float_cases()


@pytest.mark.parametrize("case", ALL, ids=[c[0] for c in ALL])
def test_oracle_f32_known_answers(case):
    name, d, f, b, pf, pb, exp = case
    img, _, _ = _run_f32(d, f, b, pf, pb)
    ok, msg = K.check_image(img[0], exp, d["nz"], d["nx"])
    assert ok, f"{name}: {msg}"


@pytest.mark.parametrize("case", ALL, ids=[c[0] for c in ALL])
def test_oracle_f64_known_answers(case):
    name, d, f, b, pf, pb, exp = case
    img, _, _ = oracle.extrapolate_f64(d["ns"], d["nextrap"], d["nz"], d["nx"], d["nf"], d["nt"], d["M"], f, b, pf, pb)
    ok, msg = K.check_image(img[0], exp, d["nz"], d["nx"])
    assert ok, f"{name}: {msg}"


@pytest.mark.parametrize("case", K.gpu_cases(), ids=[c[0] for c in K.gpu_cases()])
def test_oracle_wavefield_write_back(case):
    # test_cpp_src_cuda.py:51-54, :159-162: in-place final wavefields of the revOp library
    name, d, f, b, pf, pb, _, waves = case
    _, w, s = _run_f32(d, f, b, pf, pb)
    (pi, pv), (ri, rv) = waves["pulse"], waves["pulse2"]
    assert abs(w[pi] - pv) <= K.SDELTA, f"{name}: pulse{pi} = {w[pi]} expected {pv}"
    assert abs(s[ri] - rv) <= K.SDELTA, f"{name}: pulse2{ri} = {s[ri]} expected {rv}"


@pytest.mark.skipif(not oracle.have_ref(), reason="reference CPU library not built (no reference sources)")
@pytest.mark.parametrize("case", ALL, ids=[c[0] for c in ALL])
def test_reference_library_known_answers(case):
    name, d, f, b, pf, pb, exp = case
    for v0 in (False, True):
        img, _, _ = _run_ref(d, f, b, pf, pb, v0=v0)
        ok, msg = K.check_image(img[0], exp, d["nz"], d["nx"])
        assert ok, f"{name} (v0={v0}): {msg}"


@pytest.mark.skipif(not oracle.have_ref(), reason="reference CPU library not built (no reference sources)")
@pytest.mark.parametrize("ns,nextrap,nz,nx,nf,nt,M", [(1, 3, 4, 17, 5, 7, 2), (3, 6, 8, 40, 6, 6, 5),
                                                       (2, 4, 4, 33, 9, 12, 12)])
def test_oracle_matches_reference_library(ns, nextrap, nz, nx, nf, nt, M):
    rng = np.random.default_rng(ns * 100 + nx)
    L = 2 * M + 1

    def c(*shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)

    f, b = c(nextrap, nf, nx, L) * 0.3, c(nextrap, nf, nx, L) * 0.3
    pf, pb = c(ns, nt, nx), c(ns, nt, nx)
    d = dict(ns=ns, nextrap=nextrap, nz=nz, nx=nx, nf=nf, nt=nt, M=M)
    io, wo, so = _run_f32(d, f, b, pf, pb)
    ir, wr, sr = _run_ref(d, f, b, pf, pb)
    # same loop order and summation order: agreement to a few ulps
    np.testing.assert_allclose(io, ir, rtol=2e-5, atol=1e-5 * np.abs(ir).max())
    np.testing.assert_allclose(wo, wr, rtol=2e-5, atol=1e-6 * np.abs(wr).max())
    np.testing.assert_allclose(so, sr, rtol=2e-5, atol=1e-6 * np.abs(sr).max())
    # untouched rows stay untouched
    assert np.all(io[:, nextrap:, :] == 0)
    # FP64 restatement agrees with the FP32 reference to FP32 accuracy
    i64, _, _ = oracle.extrapolate_f64(ns, nextrap, nz, nx, nf, nt, M, f, b, pf, pb)
    assert np.linalg.norm(i64 - ir) / np.linalg.norm(i64) < 1e-5


def test_nearest_kappa_matches_numpy_argmin():
    rng = np.random.default_rng(3)
    for nk, dk in ((10, 0.3), (1000, 1.7e-3), (4000, 7.1e-4)):
        kappa = np.arange(nk) * dk
        vals = np.concatenate([rng.uniform(-0.1, kappa[-1] * 1.3, 500), kappa[1:200] - 0.5 * dk,
                               kappa[1:50] + 0.5 * dk, [0.0, kappa[-1], kappa[-1] + 5 * dk]])
        for v in vals:
            assert oracle.nearest_kappa(v, dk, nk) == int(np.abs(kappa - v).argmin()), (nk, dk, v)
