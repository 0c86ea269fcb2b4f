"""Problem configuration of the reference driver without pandas.

Restates py_src/operatorsPreparation/problemConfig.py:6-53.  The reference reads the key_value file
with pandas.read_csv(delimiter="_") and indexes each row with df.loc[key][0]; on pandas 3 that
positional access on a label-indexed Series raises, so the reference driver no longer runs there.
This parser reads the same file (first line "key_value", then one "key_value" pair per line) and
derives the same quantities with the same arithmetic.
"""
import math

import numpy as np


class ProblemConfig:
    def __init__(self, filename=None, nz=0, nx=0, ny=1, text=None):
        if text is None:
            with open(filename) as f:
                text = f.read()
        vals = {}
        for line in text.splitlines():
            line = line.strip()
            if not line or "_" not in line:
                continue
            key, value = line.split("_", 1)
            if key == "key":
                continue
            vals[key] = float(value)  # the reference's single value column is inferred as float64
        self.filename = filename
        self.nz, self.nx, self.ny = int(nz), int(nx), int(ny)
        self.nt = int(vals["nt"])
        self.nw = int(vals["nw"])
        if self.nt < self.nw:
            raise ValueError("nt must be greater than or equal to nw")
        self.zmin, self.zmax = vals["zmin"], vals["zmax"]
        self.dz = (self.zmax - self.zmin) / self.nz
        self.zinit, self.zfinal = vals["zinit"], vals["zfinal"]
        self.nextrap = math.ceil((self.zfinal - self.zinit) / self.dz)
        self.xmin, self.xmax = vals["xmin"], vals["xmax"]
        self.dx = (self.xmax - self.xmin) / self.nx
        self.tmin, self.tmax = vals["tmin"], vals["tmax"]
        self.dt = (self.tmax - self.tmin) / self.nt
        self.M = int(vals["M"])
        self.length_M = 2 * self.M + 1
        self.N = int((self.nx - 1) / 2)
        self.length_N = 2 * self.N + 1
        self.dkx = 2 * math.pi * 1 / float(self.xmax - self.xmin)
        self.kx = np.fft.fftfreq(self.nx) * self.nx * self.dkx
        self.dw = 2 * math.pi * 1 / float(self.tmax - self.tmin)
        self.w = np.fft.fftfreq(self.nt) * self.nt * self.dw
        self.wmax = +(0.5 * self.nt - 1) * self.dw
        self.xminlocal = -self.M * self.dx
        self.xmaxlocal = +self.M * self.dx
        self.xilocal = np.array([self.xminlocal + i * self.dx for i in range(self.length_M)], dtype=np.float32)
