"""The reference driver's migration flow (main.py) on this library.

main.py:38-186 reads a CSV velocity model and CSV shot records, smooths the model, designs the WLSQ
and phase-shift operators, builds dense operator tables, prepares source and receiver spectra, calls
an extrapolation library per option and sums the per-shot images.  migrate_survey runs the same
flow with the compact table (operators.py), the device front end (frontend.py) and one batched
migration (migration.Plan); the result is the summed image of main.py:184-186.
"""
import glob
import os
import re

import numpy as np
from scipy import ndimage

from . import frontend, operators
from .config import ProblemConfig
from .migration import Plan


def read_velocity(path):
    """main.py:39 (CSV) or a .npy file of the same array."""
    if path.endswith(".npy"):
        return np.load(path).astype(np.float64)
    return np.genfromtxt(path, delimiter=",")


def smooth_velocity(vel):
    """main.py:40-42: Gaussian smoothing (sigma = 2 samples) of the slowness."""
    return 1.0 / ndimage.gaussian_filter(1.0 / vel, sigma=2)


def shot_files(shots_dir, extension="csv", low="seis", up="_"):
    """readShotFiles.py:4-13: shot files of a directory and the source index in their names
    (seis<isx>_<...>.csv); glob order, as the reference."""
    prefix = shots_dir if shots_dir.endswith(os.sep) else shots_dir + os.sep
    files = glob.glob(prefix + "*." + extension)
    isx = [int(re.search(re.escape(prefix) + low + "(.+?)" + up, f).group(1)) for f in files]
    return isx, files


def read_record(path):
    """One shot record (nt, nx) float32: CSV as main.py:121, or .npy (no text parsing)."""
    if path.endswith(".npy"):
        return np.load(path).astype(np.float32)
    return np.genfromtxt(path, delimiter=",", dtype=np.float32)


def operator_tables(config, velocity):
    """Compact forward and backward tables for the model (main.py:65-76 with the all-symmetric
    stencil choice of main.py:66): returns (tab_forw, tab_back, dk)."""
    op = operators.create_wlsq_operators(config.N, config.M, config.kx, config.xilocal, only_symmetric=True)
    kappa = operators.create_kappa(np.amax(velocity), np.amin(velocity), config.dw, config.wmax, 0.25)
    psf = operators.make_forw_ps_operators(kappa, config.kx, config.dz)
    psb = operators.make_back_ps_operators(kappa, config.kx, config.dz)
    M = config.M
    return operators.compact_table(op[M], psf), operators.compact_table(op[M], psb), float(kappa[1] - kappa[0])


def migrate_survey(config, velocity, records, shot_isx, device=None):
    """Summed migrated image (nz, nx) float32 of the shots, main.py's flow on the B200.
    velocity: the smoothed model (nz, nx); records: (ns, nt, nx) float32 array or CUDA tensor."""
    import torch
    dev = device or torch.device("cuda")
    tab_f, tab_b, dk = operator_tables(config, velocity)
    rec = records if torch.is_tensor(records) else torch.from_numpy(np.ascontiguousarray(records, dtype=np.float32))
    rec = rec.to(dev)
    ns = rec.shape[0]
    nw = config.nw
    wave, shot = frontend.prepare_shots(rec, shot_isx, nw, config.xmin, config.dx, config.dt, config.zinit,
                                        config.dz, velocity[0, 0])
    del rec
    plan = Plan(ns, config.nextrap, config.nz, config.nx, nw, nw, config.M, tab_f.shape[0], two_tables=True)
    try:
        plan.set_model(torch.from_numpy(np.ascontiguousarray(config.w[:nw], dtype=np.float64)).to(dev),
                       torch.from_numpy(np.ascontiguousarray(velocity, dtype=np.float64)).to(dev), dk,
                       torch.from_numpy(tab_f).to(dev), torch.from_numpy(tab_b).to(dev))
        image = torch.zeros((config.nz, config.nx), dtype=torch.float32, device=dev)
        plan.execute(wave, shot, image)
        return image.cpu().numpy()
    finally:
        plan.close()


def run(velocity_path, config_path, shots_dir, device=None):
    """main.py's command line flow: returns (summed image, smoothed velocity, config)."""
    vel = smooth_velocity(read_velocity(velocity_path))
    config = ProblemConfig(config_path, nz=vel.shape[0], nx=vel.shape[1], ny=1)
    isx, files = shot_files(shots_dir)
    records = np.stack([read_record(f) for f in files])
    return migrate_survey(config, vel, records, isx, device=device), vel, config
