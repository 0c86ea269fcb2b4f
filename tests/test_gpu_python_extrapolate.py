"""The mirror of the reference's Python extrapolation (wavefield_propagation.extrapolate) on the GPU
against the known answers of unittests/test_py_src_extrapolation.py (real-valued cases :52-148 and
the complex cases :150-314, which are those of test_cpp_src.py), at the reference tests' 1e-5."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import wavefield_propagation as wp
from tests import kat_cases as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", K.py_float_cases() + K.cpu_cases(), ids=lambda c: c[0])
def test_python_extrapolate_known_answers(case):
    name, d, f, b, pf, pb, expected = case
    wave, shot = pf.copy(), pb.copy()
    img = wp.extrapolate(d["nextrap"], d["nz"], d["nx"], d["nf"], d["M"], f, b, wave, shot)
    ok, msg = K.check_image(img, expected, d["nz"], d["nx"])
    assert ok, f"{name}: {msg}"
    # the caller's wavefields are left as they were, as in the reference's Python function
    assert np.array_equal(wave, pf) and np.array_equal(shot, pb)


def test_python_extrapolate_accepts_complex128_and_checks_depth():
    name, d, f, b, pf, pb, expected = K.cpu_cases()[0]
    img = wp.extrapolate(d["nextrap"], d["nz"], d["nx"], d["nf"], d["M"], f.astype(np.complex128),
                         b.astype(np.complex128), pf.astype(np.complex128), pb.astype(np.complex128))
    assert K.check_image(img, expected, d["nz"], d["nx"])[0]
    with pytest.raises(ValueError):
        wp.extrapolate(2, 1, d["nx"], d["nf"], d["M"], f, b, pf, pb)
