"""Front-end kernels (source wavelets, record spectra) on the GPU against the front-end checker and
the reference's own demo outputs; the GPU-prepared demo sources then migrate to the reference CPU
library's demo image.

Tolerances: wavelets to float32 rounding (1e-6 of the peak); spectra within 2e-6 relative L2 of the
float64 checker (a single-precision FFT, like the reference's) and 1e-5 of the reference's float32
FFT; demo image within 1e-5 relative L2 of the reference CPU library's image.
"""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import frontend, migration
from oracle import frontend_oracle as fo
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _frontend_case():
    g = dict(np.load("tests/golden/frontend_case.npz"))
    p = {k: float(g[k]) for k in ("dx", "dz", "dt", "xmin", "zinit", "v")}
    return g, int(g["nt"]), int(g["nw"]), int(g["nx"]), p


def test_ricker_sources_match_checker_and_reference():
    import torch
    g, nt, nw, nx, p = _frontend_case()
    isx = g["shot_isx"]
    sx = p["xmin"] + isx * p["dx"]
    got = frontend.ricker_sources(len(isx), nt, nx, p["dt"], p["xmin"] + p["dx"], p["dx"], p["dz"] - p["zinit"],
                                  p["v"], sx).cpu().numpy()
    ref = fo.ricker_sources(len(isx), nt, nx, p["dt"], p["xmin"] + p["dx"], p["dx"], p["dz"] - p["zinit"], p["v"], sx)
    peak = np.abs(ref).max()
    assert np.max(np.abs(got - ref)) <= 1e-6 * peak
    assert np.max(np.abs(got[0] - g["wavelet_t"])) <= 1e-6 * peak
    torch.cuda.synchronize()


def test_ricker_reference_unit_test_case():
    # unittests/test_py_src_util.py:19-50 parameters, expected values within 1e-5
    isx, nt, dt, nx, dx, xmin, z1, z2, v = -600, 500, 0.001, 151, 15, -800, 0, 10, 2600
    got = frontend.ricker_sources(1, nt, nx, dt, xmin, dx, z2 - z1, v, [isx]).cpu().numpy()[0]
    xi = xmin + np.arange(nx) * dx
    r = np.sqrt((z2 - z1) ** 2 + (isx - xi) ** 2)
    tau = np.arange(nt)[:, None] * dt - (r / v)[None, :]
    term = np.pi ** 2 * 30.0 ** 2 * tau ** 2
    assert np.max(np.abs(got - (1 - 2 * term) * np.exp(-term) / np.sqrt(r)[None, :])) <= 1e-5


def test_demo_spectra_match_reference(golden_demo):
    import torch
    g, nt, nw, nx, p = _frontend_case()
    rec = torch.from_numpy(g["rec_t"][None]).cuda()
    got = frontend.records_to_spectra(rec, nw).cpu().numpy().reshape(nw, nx)
    assert rel_l2(got, fo.records_to_spectra(g["rec_t"][None], nw).reshape(nw, nx)) <= 2e-6
    assert rel_l2(got, g["rec_f"]) <= 1e-5
    # all nine sources through prepare_shots' source path
    isx = g["shot_isx"]
    src_t = frontend.ricker_sources(len(isx), nt, nx, p["dt"], p["xmin"] + p["dx"], p["dx"], p["dz"] - p["zinit"],
                                    p["v"], p["xmin"] + isx * p["dx"])
    src_f = frontend.records_to_spectra(src_t, nw).cpu().numpy().reshape(len(isx), nw, nx)
    assert rel_l2(src_f, golden_demo["src"]) <= 1e-5


def test_prepare_shots_and_migrate_demo(golden_demo):
    """Sources prepared on the GPU (main.py:111-119 path) with the demo's reference receiver spectra
    migrate to the reference CPU library's demo image."""
    import torch
    g, nt, nw, nx, p = _frontend_case()
    d = golden_demo
    ns = d["src"].shape[0]
    fake_records = torch.zeros((ns, nt, nx), dtype=torch.float32, device="cuda")
    wave, _ = frontend.prepare_shots(fake_records, g["shot_isx"], nw, p["xmin"], p["dx"], p["dt"], p["zinit"],
                                     p["dz"], p["v"])
    wave = wave.cpu().numpy()
    shot = d["rec"].reshape(-1).copy()
    nz, M, nk = int(d["nz"]), int(d["M"]), int(d["nk"])
    img, _ = migration.migrate(ns, int(d["nextrap"]), nz, nx, nw, nw, M, nk, float(d["dk"]), d["omega"],
                               d["velocity"], d["tab_f"], wave, shot, tab_back=d["tab_b"], two_tables=True)
    assert rel_l2(img, d["image_ref_cpu"]) <= 1e-5


def test_apertures_rows_and_errors():
    import torch
    from imaging2d_wlsq_b200._lib import LibraryError
    rng = np.random.default_rng(7)
    ns, nt, nx, nf, nt_rows = 5, 300, 70, 237, 240  # nf > nt/2: upper rows by conjugate symmetry
    rec_np = rng.standard_normal((ns, nt, nx)).astype(np.float32)
    x0 = np.array([0, 10, 33, 50, 69], dtype=np.int32)
    wn = np.array([70, 23, 30, 20, 1], dtype=np.int32)
    rec = torch.from_numpy(rec_np).cuda()
    total = int(nt_rows * wn.sum())
    out = torch.full((total,), 9 + 9j, dtype=torch.complex64, device="cuda")
    frontend.records_to_spectra(rec, nf, nt_rows=nt_rows, shot_x0=x0, shot_nx=wn, out=out)
    got = out.cpu().numpy()
    ref = fo.records_to_spectra(rec_np, nf, nt_rows=nt_rows, shot_x0=x0, shot_nx=wn)
    off = 0
    for s in range(ns):
        blk, rb = got[off:off + nt_rows * wn[s]].reshape(nt_rows, wn[s]), ref[off:off + nt_rows * wn[s]].reshape(nt_rows, wn[s])
        assert rel_l2(blk[:nf], rb[:nf]) <= 2e-6
        assert np.all(blk[nf:] == 9 + 9j)  # rows beyond nf untouched
        off += nt_rows * wn[s]
    with pytest.raises(LibraryError, match="nf <= nt"):
        frontend.records_to_spectra(rec, nt + 1)
    with pytest.raises(LibraryError, match="aperture"):
        frontend.records_to_spectra(rec, nf, shot_x0=[0, 0, 0, 0, 60], shot_nx=[1, 1, 1, 1, 11])
