"""The C-ABI library loads and exports every symbol include/*.h declares; the drop-in shims export
the reference's symbols; host-side validation works without a GPU."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import imaging2d_wlsq_b200 as pkg
from imaging2d_wlsq_b200 import _lib
from tests.conftest import ROOT, cuda_available


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(img2d_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("img2d_extrapolate_host_order", "img2d_extrapolate_device_order", "img2d_migrate_compact",
                     "img2d_plan_create", "img2d_plan_execute", "img2d_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    syms = exported(pkg.LIB_PATH)
    missing = [n for n in declared_functions() if n not in syms]
    assert not missing, f"declared in include/*.h but not exported: {missing}"
    ctypes.CDLL(pkg.LIB_PATH)  # loads


@pytest.mark.parametrize("name,symbols", [("extrapolation_cpu.so", {"extrapolate", "extrapolate_v0"}),
                                          ("extrapolation_gpu.so", {"extrapolate"}),
                                          ("extrapolation_revOp_gpu.so", {"extrapolate"}),
                                          ("extrapolation_sh_revOp_gpu.so", {"extrapolate"})])
def test_dropin_shims_export_reference_symbols(name, symbols):
    path = os.path.join(pkg.DROPIN_DIR, name)
    assert symbols <= exported(path)
    ctypes.CDLL(path)


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU error path")
def test_no_device_reports_enodev():
    lib = _lib.lib()
    img = np.zeros((1, 1, 4), dtype=np.float32)
    op = np.zeros((1, 2, 4, 3), dtype=np.complex64)
    p = np.zeros((1, 2, 4), dtype=np.complex64)
    rc = lib.img2d_extrapolate_host_order(1, 1, 1, 4, 2, 2, 1, op, op, p, p.copy(), img)
    assert rc == _lib.IMG2D_ENODEV
    assert b"no CUDA device" in lib.img2d_last_error()
    with pytest.raises(_lib.LibraryError):
        from imaging2d_wlsq_b200 import interface
        interface.extrapolate(1, 1, 1, 4, 2, 2, 1, op, op, p, p.copy(), img)


def test_version():
    assert _lib.lib().img2d_version() >= 10000


@pytest.mark.parametrize("dims", [dict(ns=0, nextrap=2, nf=2), dict(ns=2, nextrap=0, nf=2),
                                  dict(ns=2, nextrap=2, nf=0)], ids=["ns0", "nextrap0", "nf0"])
def test_degenerate_sizes_behave_like_reference(dims):
    """Sizes for which the reference's loops do no extrapolation (no shots, no depth steps, no
    frequencies) leave the buffers as the reference's own CPU library does (nf = 0 writes zero
    image rows); no GPU is needed."""
    from oracle import oracle
    from imaging2d_wlsq_b200 import interface, interface_cuda
    ns, nextrap, nf = dims["ns"], dims["nextrap"], dims["nf"]
    nz, nx, nt, M = 3, 5, 3, 1
    rng = np.random.default_rng(1)
    op = (rng.standard_normal((max(nextrap, 1), max(nf, 1), nx, 3)) + 0j).astype(np.complex64)
    wave = (rng.standard_normal((max(ns, 1), nt, nx)) + 1j).astype(np.complex64)
    shot = (rng.standard_normal((max(ns, 1), nt, nx)) - 1j).astype(np.complex64)
    img0 = np.full((max(ns, 1), nz, nx), 7.0, dtype=np.float32)
    outs = []
    calls = [lambda w, s, i: interface.extrapolate(ns, nextrap, nz, nx, nf, nt, M, op, op, w, s, i),
             lambda w, s, i: interface_cuda.extrapolate_revOp(ns, nextrap, nz, nt, nf, nx, M, op, w, op, s, i)]
    if oracle.have_ref():
        calls.append(lambda w, s, i: oracle.ref_extrapolate(ns, nextrap, nz, nx, nf, nt, M, op, op, w, s, i))
    for call in calls:
        w, s, i = wave.copy(), shot.copy(), img0.copy()
        call(w, s, i)
        outs.append((w, s, i))
    for w, s, i in outs:
        np.testing.assert_array_equal(w, wave)
        np.testing.assert_array_equal(s, shot)
        expect = img0.copy()
        if nf == 0:
            expect[:ns, :nextrap] = 0.0
        np.testing.assert_array_equal(i, expect)
