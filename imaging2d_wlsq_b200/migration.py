"""Python API over the compact-table C ABI.

`migrate(...)` takes host numpy arrays (the C entry point copies to and from the GPU).
`Plan` keeps everything on the device: inputs and outputs are torch CUDA tensors, calls are
asynchronous on the current torch stream, and the operator index table is built once per model.
"""
import ctypes
import json

import numpy as np

from . import _lib
from ._lib import check, lib, ptr


def migrate(ns, nextrap, nz, nx, nf, nt, M, nk, dk, omega, velocity, tab_forw, wave_fs, shot_fs,
            tab_back=None, shot_x0=None, shot_nx=None, image=True, image_shots=False, two_tables=False,
            generic=False, no_cluster=False, cluster_v1=False):
    """Host-buffer migration.  wave_fs/shot_fs (packed complex64) are overwritten with the final
    wavefields.  Returns (image (nz, nx) float32 or None, image_shots (ns, nz, nx) or None); rows
    [nextrap, nz) are zero."""
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    velocity = np.ascontiguousarray(velocity, dtype=np.float64)
    tab_forw = np.ascontiguousarray(tab_forw, dtype=np.complex64)
    if tab_back is not None:
        tab_back = np.ascontiguousarray(tab_back, dtype=np.complex64)
    for a in (wave_fs, shot_fs):
        if a.dtype != np.complex64 or not a.flags.c_contiguous:
            raise TypeError("wave_fs/shot_fs must be C-contiguous complex64 arrays (updated in place)")
    x0 = None if shot_x0 is None else np.ascontiguousarray(shot_x0, dtype=np.int32)
    wn = None if shot_nx is None else np.ascontiguousarray(shot_nx, dtype=np.int32)
    img = np.zeros((nz, nx), dtype=np.float32) if image else None
    imgs = np.zeros((ns, nz, nx), dtype=np.float32) if image_shots else None
    flags = (_lib.FLAG_TWO_TABLES if two_tables else 0) | (_lib.FLAG_GENERIC if generic else 0) | \
        (_lib.FLAG_NO_CLUSTER if no_cluster else 0) | (_lib.FLAG_CLUSTER_V1 if cluster_v1 else 0)
    check(lib().img2d_migrate_compact(ns, nextrap, nz, nx, nf, nt, M, nk, float(dk), ptr(omega), ptr(velocity),
                                      ptr(tab_forw), ptr(tab_back), ptr(x0), ptr(wn), ptr(wave_fs), ptr(shot_fs),
                                      ptr(img), ptr(imgs), flags))
    return img, imgs


def migrate_workload(w, two_tables=False, table_back=None, image_shots=False, generic=False, no_cluster=False,
                     cluster_v1=False):
    """Run a synthetic.Workload through the host entry point on copies of its spectra."""
    wave = w.wave.copy()
    shot = w.shot.copy()
    img, imgs = migrate(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega, w.velocity, w.table,
                        wave, shot, tab_back=table_back, shot_x0=w.shot_x0, shot_nx=w.shot_nx,
                        image_shots=image_shots, two_tables=two_tables, generic=generic, no_cluster=no_cluster,
                        cluster_v1=cluster_v1)
    return img, imgs, wave, shot


def fp32_peak_tflops():
    """Measured FP32 FMA throughput of the current GPU (TFLOP/s)."""
    v = ctypes.c_double()
    check(lib().img2d_measure_fp32_peak(ctypes.byref(v)))
    return v.value


class Plan:
    """Device-resident migration plan (torch CUDA tensors in, torch CUDA tensors out)."""

    def __init__(self, ns, nextrap, nz, nx, nf, nt, M, nk, shot_x0=None, shot_nx=None, two_tables=False,
                 generic=False, no_cluster=False, cluster_v1=False, variant=0, table="fp32"):
        """table: operator-table storage, "fp32" (default), "fp16" or "bf16" (reduced-precision
        storage, FP32 arithmetic; cluster kernel only)."""
        self.ns, self.nextrap, self.nz, self.nx, self.nf, self.nt, self.M, self.nk = \
            ns, nextrap, nz, nx, nf, nt, M, nk
        x0 = None if shot_x0 is None else np.ascontiguousarray(shot_x0, dtype=np.int32)
        wn = None if shot_nx is None else np.ascontiguousarray(shot_nx, dtype=np.int32)
        flags = (_lib.FLAG_TWO_TABLES if two_tables else 0) | (_lib.FLAG_GENERIC if generic else 0) | \
            (_lib.FLAG_NO_CLUSTER if no_cluster else 0) | (_lib.FLAG_CLUSTER_V1 if cluster_v1 else 0) | \
            (int(variant) << _lib.FLAG_VARIANT_SHIFT) | \
            {"fp32": 0, "fp16": _lib.FLAG_TABLE_FP16, "bf16": _lib.FLAG_TABLE_BF16}[table]
        h = ctypes.c_void_p()
        check(lib().img2d_plan_create(ctypes.byref(h), ns, nextrap, nz, nx, nf, nt, M, nk, ptr(x0), ptr(wn), flags))
        self._h = h
        self._keep = []

    @classmethod
    def for_workload(cls, w, **kw):
        return cls(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.shot_x0, w.shot_nx, **kw)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().img2d_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self, stream):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        return ctypes.c_void_p(s.cuda_stream)

    def set_model(self, omega, velocity, dk, table, table_back=None, stream=None):
        """omega (nf,) float64, velocity (nz, nx) float64, table (nk, L) complex64: CUDA tensors."""
        self._keep = [omega, velocity, table, table_back]
        check(lib().img2d_plan_set_model(self._h, ptr(omega), ptr(velocity), float(dk), ptr(table),
                                         ptr(table_back), self._stream(stream)))

    def execute(self, wave, shot, image=None, image_shots=None, stream=None):
        check(lib().img2d_plan_execute(self._h, ptr(wave), ptr(shot), ptr(image), ptr(image_shots),
                                       self._stream(stream)))

    def execute_naive(self, wave, shot, image, stream=None):
        check(lib().img2d_plan_execute_naive(self._h, ptr(wave), ptr(shot), ptr(image), self._stream(stream)))

    def kernel_ms(self):
        """Device time of the migration kernel of the last execute (waits for it)."""
        v = ctypes.c_float()
        check(lib().img2d_plan_kernel_ms(self._h, ctypes.byref(v)))
        return v.value

    def shot_offset(self, s):
        return lib().img2d_plan_shot_offset(self._h, s)

    @property
    def wavefield_elems(self):
        return lib().img2d_plan_wavefield_elems(self._h)

    @property
    def workspace_bytes(self):
        return lib().img2d_plan_workspace_bytes(self._h)

    def describe(self):
        buf = ctypes.create_string_buffer(512)
        check(lib().img2d_plan_describe(self._h, buf, 512))
        return json.loads(buf.value.decode())
