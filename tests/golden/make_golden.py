"""Generate the golden fixtures in tests/golden/ from the reference implementation.

Run on a machine that has the reference sources (their root in IMG2D_REFERENCE) and the reference
CPU library built by oracle/build_ref.sh:

    IMG2D_REFERENCE=<reference source tree> python tests/golden/make_golden.py

Writes
  operators_small.npz  outputs of the reference's own Python operator design
                       (py_src/operatorsPreparation/{preparation,util}.py, run with numba) for a
                       small odd-width model: createWLSQoperators, make{Forw,Back}PSoperators,
                       createKappa, find_nearest and makeTableOfOperators.
  frontend_case.npz    the demo's data-preparation parameters (main.py:105-123), the reference's
                       util.makeRickerWavelet output and the time-domain CSV record of one shot, and
                       the first nw rows of scipy.fftpack.fft of that record (the receiver spectra the
                       demo feeds to the extrapolation); the source spectra of all shots are in
                       demo_case.npz
  driver_case.npz      inputs of the reference driver for all nine demo shots (the raw velocity model,
                       the time-domain CSV records and their source indices) and the image that the
                       reference flow (main.py: its Python operator design and data preparation, then
                       oracle/_ref/extrapolation_cpu.so on the dense tables) produces from them
  demo_case.npz        the reference demo (demo-data/, problemSetup.txt) reduced to the compact form
                       this library consumes: smoothed velocity, angular frequencies, kappa step,
                       compact forward/backward tables (rows = op[M] @ psOp[k], the numpy call of
                       preparation.py:110), source/receiver spectra prepared as main.py:105-123 does;
                       plus two expected images: the reference's shipped demo-result/final_image.csv
                       and the image of oracle/_ref/extrapolation_cpu.so on the same inputs.
"""
import glob
import math
import os
import re
import sys

import numpy as np

REF = os.environ.get("IMG2D_REFERENCE")
if not REF:
    sys.exit("set IMG2D_REFERENCE to the reference source tree")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REF, "py_src", "operatorsPreparation"))
sys.path.insert(0, ROOT)

import preparation as prep  # noqa: E402  (reference code)
import util  # noqa: E402  (reference code)
from scipy import ndimage  # noqa: E402
import scipy.fftpack as spfft  # noqa: E402

from oracle import oracle  # noqa: E402


def operators_small():
    nx, M, dx, dz = 31, 5, 10.0, 7.5
    N = (nx - 1) // 2
    dkx = 2 * math.pi / (nx * dx)
    kx = np.fft.fftfreq(nx) * nx * dkx
    xil = np.array([-M * dx + i * dx for i in range(2 * M + 1)], dtype=np.float32)
    op = prep.createWLSQoperators(N, M, kx, xil)
    dw = 2 * math.pi / 0.5
    wmax = (0.5 * 64 - 1) * dw
    kappa = util.createKappa(3000.0, 1500.0, dw, wmax, 0.25)
    psf = prep.makeForwPSoperators(kappa, kx, dz)
    psb = prep.makeBackPSoperators(kappa, kx, dz)
    rng = np.random.default_rng(7)
    nextrap, nw = 3, 4
    vel = rng.uniform(1500.0, 3000.0, (nextrap, nx))
    w = (np.fft.fftfreq(64) * 64 * dw)[:nw] + 1.0
    gidx = util.defWLSQIndices(nx=nx, M=M, flip=False, sym=True, extent=5)
    table_f = prep.makeTableOfOperators(nextrap, nx, nw, kappa, kx, w, vel, gidx, op, psf)
    table_b = prep.makeTableOfOperators(nextrap, nx, nw, kappa, kx, w, vel, gidx, op, psb)
    values = np.concatenate([rng.uniform(0, kappa[-1] * 1.2, 200), kappa[5:25] + 0.5 * (kappa[1] - kappa[0])])
    nearest = np.array([util.find_nearest(kappa, v) for v in values])
    np.savez_compressed(os.path.join(HERE, "operators_small.npz"), nx=nx, M=M, dx=dx, dz=dz, kx=kx, xilocal=xil,
                        op=op, kappa=kappa, dw=dw, wmax=wmax, psf=psf, psb=psb, vel=vel, w=w, table_f=table_f,
                        table_b=table_b, values=values, nearest=nearest)


def parse_setup(path):
    vals = {}
    for line in open(path):
        line = line.strip()
        if "_" in line and not line.startswith("key"):
            k, v = line.split("_", 1)
            vals[k] = float(v)
    return vals


def demo_case():
    vel0 = np.genfromtxt(os.path.join(REF, "demo-data", "velmod.csv"), delimiter=",")
    slow = ndimage.gaussian_filter(1.0 / vel0, sigma=2)          # main.py:40-41
    vel = 1.0 / slow
    cfg = parse_setup(os.path.join(REF, "demo-data", "problemSetup.txt"))
    nz, nx = vel.shape
    nt, nw, M = int(cfg["nt"]), int(cfg["nw"]), int(cfg["M"])
    dz = (cfg["zmax"] - cfg["zmin"]) / nz                         # problemConfig.py:24-30
    nextrap = math.ceil((cfg["zfinal"] - cfg["zinit"]) / dz)
    dx = (cfg["xmax"] - cfg["xmin"]) / nx
    dt = (cfg["tmax"] - cfg["tmin"]) / nt
    N = int((nx - 1) / 2)
    dkx = 2 * math.pi * 1 / float(cfg["xmax"] - cfg["xmin"])
    kx = np.fft.fftfreq(nx) * nx * dkx
    dw = 2 * math.pi * 1 / float(cfg["tmax"] - cfg["tmin"])
    w = np.fft.fftfreq(nt) * nt * dw
    wmax = +(0.5 * nt - 1) * dw
    xil = np.array([(-M * dx) + i * dx for i in range(2 * M + 1)], dtype=np.float32)
    op = prep.createWLSQoperators(N, M, kx, xil)                    # main.py:65
    kappa = util.createKappa(np.amax(vel), np.amin(vel), dw, wmax, 0.25)  # main.py:71-73
    psf = prep.makeForwPSoperators(kappa, kx, dz)
    psb = prep.makeBackPSoperators(kappa, kx, dz)
    nk = len(kappa)
    tab_f = np.stack([np.matmul(op[M, :, :], psf[k, :]) for k in range(nk)]).astype(np.complex64)
    tab_b = np.stack([np.matmul(op[M, :, :], psb[k, :]) for k in range(nk)]).astype(np.complex64)
    dk = kappa[1] - kappa[0]
    assert np.array_equal(kappa, np.arange(nk) * dk) or np.allclose(kappa, np.arange(nk) * dk, rtol=0, atol=0)
    # shots (main.py:105-123; glob order as the reference)
    files = glob.glob(os.path.join(REF, "demo-data", "seismicShots") + "/*.csv")
    isx = [int(re.search(r"seis(.+?)_", os.path.basename(f)).group(1)) for f in files]
    v = vel[0, 0]
    tj = [j * dt for j in range(nt)]
    xi = [cfg["xmin"] + (i + 1) * dx for i in range(nx)]
    ns = len(files)
    src = np.zeros((ns, nt, nx), dtype=np.complex64)
    rec = np.zeros((ns, nt, nx), dtype=np.complex64)
    for s in range(ns):
        st = util.makeRickerWavelet([cfg["xmin"] + isx[s] * dx], cfg["zinit"], nt, nx, tj, xi, dz, v)
        src[s] = spfft.fft(st, axis=0)
        rec[s] = spfft.fft(np.genfromtxt(files[s], delimiter=",", dtype=np.float32), axis=0)
    omega = w[:nw].astype(np.float64)
    # reference CPU library on the dense tables gathered from the compact ones
    dense_f = oracle.gather_dense_slab(0, nextrap, nx, 0, nx, nw, M, nk, dk, omega, vel, tab_f)
    dense_b = oracle.gather_dense_slab(0, nextrap, nx, 0, nx, nw, M, nk, dk, omega, vel, tab_b)
    image = np.zeros((ns, nz, nx), dtype=np.float32)
    s_in, r_in = src.copy(), rec.copy()
    oracle.ref_extrapolate(ns, nextrap, nz, nx, nw, nt, M, dense_f, dense_b, s_in, r_in, image)
    ref_cpu = np.zeros((nz, nx), dtype=np.float32)
    for s in range(ns):
        ref_cpu += image[s]
    shipped = np.genfromtxt(os.path.join(REF, "demo-result", "final_image.csv"), delimiter=",").astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "demo_case.npz"), nz=nz, nx=nx, nw=nw, nextrap=nextrap, M=M, nk=nk,
                        dk=dk, dx=dx, dz=dz, omega=omega, velocity=vel, tab_f=tab_f, tab_b=tab_b,
                        src=src[:, :nw, :], rec=rec[:, :nw, :], shot_isx=np.array(isx),
                        image_ref_cpu=ref_cpu, image_shipped=shipped)
    rel = np.linalg.norm(ref_cpu - shipped) / np.linalg.norm(shipped)
    print(f"demo: reference CPU library vs shipped final_image.csv rel-L2 {rel:.3e}")


def frontend_case():
    vel0 = np.genfromtxt(os.path.join(REF, "demo-data", "velmod.csv"), delimiter=",")
    vel = 1.0 / ndimage.gaussian_filter(1.0 / vel0, sigma=2)     # main.py:40-41
    cfg = parse_setup(os.path.join(REF, "demo-data", "problemSetup.txt"))
    nz, nx = vel.shape
    nt, nw = int(cfg["nt"]), int(cfg["nw"])
    dz = (cfg["zmax"] - cfg["zmin"]) / nz
    dx = (cfg["xmax"] - cfg["xmin"]) / nx
    dt = (cfg["tmax"] - cfg["tmin"]) / nt
    files = glob.glob(os.path.join(REF, "demo-data", "seismicShots") + "/*.csv")
    isx = [int(re.search(r"seis(.+?)_", os.path.basename(f)).group(1)) for f in files]
    v = vel[0, 0]
    tj = [j * dt for j in range(nt)]
    xi = [cfg["xmin"] + (i + 1) * dx for i in range(nx)]
    wavelet = util.makeRickerWavelet([cfg["xmin"] + isx[0] * dx], cfg["zinit"], nt, nx, tj, xi, dz, v)
    rec = np.genfromtxt(files[0], delimiter=",", dtype=np.float32)
    rec_f = spfft.fft(rec, axis=0)[:nw]
    np.savez_compressed(os.path.join(HERE, "frontend_case.npz"), nt=nt, nw=nw, nx=nx, dx=dx, dz=dz, dt=dt,
                        xmin=cfg["xmin"], zinit=cfg["zinit"], v=v, shot_isx=np.array(isx),
                        wavelet_t=wavelet, rec_t=rec, rec_f=rec_f.astype(np.complex64))


def driver_case(nshots=None):
    vel0 = np.genfromtxt(os.path.join(REF, "demo-data", "velmod.csv"), delimiter=",")
    vel = 1.0 / ndimage.gaussian_filter(1.0 / vel0, sigma=2)     # main.py:40-41
    cfg = parse_setup(os.path.join(REF, "demo-data", "problemSetup.txt"))
    nz, nx = vel.shape
    nt, nw, M = int(cfg["nt"]), int(cfg["nw"]), int(cfg["M"])
    dz = (cfg["zmax"] - cfg["zmin"]) / nz
    nextrap = math.ceil((cfg["zfinal"] - cfg["zinit"]) / dz)
    dx = (cfg["xmax"] - cfg["xmin"]) / nx
    dt = (cfg["tmax"] - cfg["tmin"]) / nt
    N = int((nx - 1) / 2)
    kx = np.fft.fftfreq(nx) * nx * (2 * math.pi / float(cfg["xmax"] - cfg["xmin"]))
    dw = 2 * math.pi / float(cfg["tmax"] - cfg["tmin"])
    w = np.fft.fftfreq(nt) * nt * dw
    wmax = +(0.5 * nt - 1) * dw
    xil = np.array([(-M * dx) + i * dx for i in range(2 * M + 1)], dtype=np.float32)
    op = prep.createWLSQoperators(N, M, kx, xil)
    kappa = util.createKappa(np.amax(vel), np.amin(vel), dw, wmax, 0.25)
    gidx = util.defWLSQIndices(nx=nx, M=M, flip=False, sym=True, extent=5)
    tf = prep.makeTableOfOperators(nextrap, nx, nw, kappa, kx, w, vel, gidx, op,
                                   prep.makeForwPSoperators(kappa, kx, dz))       # main.py:82-88
    tb = prep.makeTableOfOperators(nextrap, nx, nw, kappa, kx, w, vel, gidx, op,
                                   prep.makeBackPSoperators(kappa, kx, dz))
    files = sorted(glob.glob(os.path.join(REF, "demo-data", "seismicShots") + "/*.csv"))[:nshots]
    nshots = len(files)
    isx = [int(re.search(r"seis(.+?)_", os.path.basename(f)).group(1)) for f in files]
    v = vel[0, 0]
    tj = [j * dt for j in range(nt)]
    xi = [cfg["xmin"] + (i + 1) * dx for i in range(nx)]
    records = np.stack([np.genfromtxt(f, delimiter=",", dtype=np.float32) for f in files])
    src = np.zeros((nshots, nt, nx), dtype=np.complex64)
    rec = np.zeros((nshots, nt, nx), dtype=np.complex64)
    for s in range(nshots):
        src[s] = spfft.fft(util.makeRickerWavelet([cfg["xmin"] + isx[s] * dx], cfg["zinit"], nt, nx, tj, xi, dz, v),
                           axis=0)
        rec[s] = spfft.fft(records[s], axis=0)
    image = np.zeros((nshots, nz, nx), dtype=np.float32)
    oracle.ref_extrapolate(nshots, nextrap, nz, nx, nw, nt, M, np.ascontiguousarray(tf, dtype=np.complex64),
                           np.ascontiguousarray(tb, dtype=np.complex64), src, rec, image)
    np.savez_compressed(os.path.join(HERE, "driver_case.npz"), velmod=vel0, records=records, shot_isx=np.array(isx),
                        image=image.sum(axis=0))


if __name__ == "__main__":
    # all fixtures, or only those named on the command line (e.g. `make_golden.py driver_case`)
    makers = {f.__name__: f for f in (operators_small, frontend_case, driver_case, demo_case)}
    for name in sys.argv[1:] or list(makers):
        makers[name]()
    print("wrote", os.listdir(HERE))
