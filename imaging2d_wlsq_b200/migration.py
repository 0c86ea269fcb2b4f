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
            generic=False, no_cluster=False, cluster_v1=False, variant=0, wide=False, wide_scalar=False,
            cluster2=False, wide_bulk=False, line_packing=False):
    """Host-buffer migration.  wave_fs/shot_fs (packed complex64) are overwritten with the final
    wavefields.  Returns (image (nz, nx) float32 or None, image_shots (ns, nz, nx) or None); rows
    [nextrap, nz) are zero.  variant: cluster-kernel variant (1-based, 0 = default)."""
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
        (_lib.FLAG_NO_CLUSTER if no_cluster else 0) | (_lib.FLAG_CLUSTER_V1 if cluster_v1 else 0) | \
        (int(variant) << _lib.FLAG_VARIANT_SHIFT) | _wide_flags(wide, wide_scalar, wide_bulk) | \
        (_lib.FLAG_CLUSTER2 if cluster2 else 0) | (_lib.FLAG_LINE_PACKING if line_packing else 0)
    check(lib().img2d_migrate_compact(ns, nextrap, nz, nx, nf, nt, M, nk, float(dk), ptr(omega), ptr(velocity),
                                      ptr(tab_forw), ptr(tab_back), ptr(x0), ptr(wn), ptr(wave_fs), ptr(shot_fs),
                                      ptr(img), ptr(imgs), flags))
    return img, imgs


def migrate_workload(w, two_tables=False, table_back=None, image_shots=False, generic=False, no_cluster=False,
                     cluster_v1=False, variant=0, wide=False, wide_scalar=False, cluster2=False, wide_bulk=False,
                     line_packing=False):
    """Run a synthetic.Workload through the host entry point on copies of its spectra."""
    wave = w.wave.copy()
    shot = w.shot.copy()
    img, imgs = migrate(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, w.omega, w.velocity, w.table,
                        wave, shot, tab_back=table_back, shot_x0=w.shot_x0, shot_nx=w.shot_nx,
                        image_shots=image_shots, two_tables=two_tables, generic=generic, no_cluster=no_cluster,
                        cluster_v1=cluster_v1, variant=variant, wide=wide, wide_scalar=wide_scalar,
                        cluster2=cluster2, wide_bulk=wide_bulk, line_packing=line_packing)
    return img, imgs, wave, shot


def plan_flags(two_tables=False, generic=False, no_cluster=False, cluster_v1=False, variant=0, table="fp32",
               demig_ring=True, wide=False, wide_scalar=False, cluster2=False, wide_bulk=False,
               line_packing=False):
    """The C ABI `flags` word of a kernel configuration given as Plan keyword arguments."""
    return (_lib.FLAG_TWO_TABLES if two_tables else 0) | (_lib.FLAG_GENERIC if generic else 0) | \
        (_lib.FLAG_NO_CLUSTER if no_cluster else 0) | (_lib.FLAG_CLUSTER_V1 if cluster_v1 else 0) | \
        (int(variant) << _lib.FLAG_VARIANT_SHIFT) | \
        {"fp32": 0, "fp16": _lib.FLAG_TABLE_FP16, "bf16": _lib.FLAG_TABLE_BF16}[table] | \
        (0 if demig_ring else _lib.FLAG_DEMIG_NO_RING) | _wide_flags(wide, wide_scalar, wide_bulk) | \
        (_lib.FLAG_CLUSTER2 if cluster2 else 0) | (_lib.FLAG_LINE_PACKING if line_packing else 0)


def _wide_flags(wide, wide_scalar, wide_bulk=False):
    """Flags of the wide cluster kernel (8 slots x 1024 positions per CTA): packed FMAs by default,
    scalar FMAs with wide_scalar, the operator-pair ring filled by 1-D bulk copies with wide_bulk."""
    if not (wide or wide_scalar or wide_bulk):
        return 0
    return _lib.FLAG_WIDE | (_lib.FLAG_WIDE_SCALAR if wide_scalar else 0) | (_lib.FLAG_WIDE_BULK if wide_bulk else 0)


def pack_shots(shot_x0, shot_nx, nx, M, windows=True, K=None):
    """The wide kernel's packing of shots into items of up to 8 lane slots, computed on the host
    (no GPU): windows=True the window-first packing on clusters of K CTAs (default: just wide enough
    for the widest shot), False the line packing.  Returns a dict with per-shot `group` and `slot`,
    per-group `u0` and `width`, and the modelled `cost` of one frequency's items in CTA units."""
    x0 = np.ascontiguousarray(shot_x0, dtype=np.int32)
    wn = np.ascontiguousarray(shot_nx, dtype=np.int32)
    ns = len(x0)
    if K is None:
        K = -(-int(wn.max()) // 1024) if windows else 0
    group = np.empty(ns, np.int32)
    slot = np.empty(ns, np.int32)
    u0 = np.empty(ns, np.int32)
    width = np.empty(ns, np.int32)
    ng = ctypes.c_int()
    cost = ctypes.c_double()
    check(lib().img2d_pack_shots(ns, int(nx), int(M), ptr(x0), ptr(wn), int(bool(windows)), int(K), ptr(group),
                                 ptr(slot), ptr(u0), ptr(width), ctypes.byref(ng), ctypes.byref(cost)))
    n = ng.value
    return {"group": group, "slot": slot, "u0": u0[:n].copy(), "width": width[:n].copy(), "cost": cost.value,
            "K": int(K)}


def fp32_peak_tflops():
    """Measured FP32 FMA throughput of the current GPU (TFLOP/s)."""
    v = ctypes.c_double()
    check(lib().img2d_measure_fp32_peak(ctypes.byref(v)))
    return v.value


def l2_read_bandwidth_gbs():
    """Measured L2 read bandwidth of the current GPU (GB/s)."""
    v = ctypes.c_double()
    check(lib().img2d_measure_l2_bandwidth(ctypes.byref(v)))
    return v.value


class Plan:
    """Device-resident migration plan (torch CUDA tensors in, torch CUDA tensors out)."""

    def __init__(self, ns, nextrap, nz, nx, nf, nt, M, nk, shot_x0=None, shot_nx=None, two_tables=False,
                 generic=False, no_cluster=False, cluster_v1=False, variant=0, table="fp32", demig_ring=True,
                 wide=False, wide_scalar=False, cluster2=False, wide_bulk=False, line_packing=False):
        """table: operator-table storage, "fp32" (default), "fp16" or "bf16" (reduced-precision
        storage, FP32 arithmetic; cluster kernel only).  demig_ring: the cluster demigration kernel's
        forward steps read their operator pairs through a shared-memory ring (False: through L1)."""
        self.ns, self.nextrap, self.nz, self.nx, self.nf, self.nt, self.M, self.nk = \
            ns, nextrap, nz, nx, nf, nt, M, nk
        x0 = None if shot_x0 is None else np.ascontiguousarray(shot_x0, dtype=np.int32)
        wn = None if shot_nx is None else np.ascontiguousarray(shot_nx, dtype=np.int32)
        flags = plan_flags(two_tables, generic, no_cluster, cluster_v1, variant, table, demig_ring, wide, wide_scalar,
                           cluster2, wide_bulk, line_packing)
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

    def demigrate(self, refl, wave, data, slab_depth=0, source="recompute", stream=None):
        """Demigration, the adjoint of execute() with respect to the receiver spectra: writes
        data = F* refl for the source spectra `wave` (read only).  refl is a float32 (>= nextrap, nx)
        image; data has the packed wavefield layout and must not alias wave.  Source wavefields are
        recomputed per slab of `slab_depth` depth steps (0: the library default) from checkpoints;
        source="keep" keeps those checkpoints on the plan and "reuse" reads them instead of
        computing them (same `wave` as the keeping call, no set_model in between)."""
        mode = {"recompute": _lib.SOURCE_RECOMPUTE, "keep": _lib.SOURCE_KEEP, "reuse": _lib.SOURCE_REUSE}[source]
        check(lib().img2d_plan_demigrate(self._h, ptr(refl), ptr(wave), ptr(data), int(slab_depth), mode,
                                         self._stream(stream)))

    def describe_demigration(self):
        buf = ctypes.create_string_buffer(512)
        check(lib().img2d_plan_describe_demigration(self._h, buf, 512))
        return json.loads(buf.value.decode())

    def dense_table(self, which=0, out=None, stream=None):
        """The legacy ABI's dense operator table (nextrap, nf, nx, 2M+1) complex64, gathered on the
        device from the compact table and the operator index set by set_model (the GPU form of
        makeTableOfOperators, preparation.py:101-115).  which=0: forward rows; 1: receiver rows."""
        import torch
        shape = (self.nextrap, self.nf, self.nx, 2 * self.M + 1)
        if out is None:
            out = torch.empty(shape, dtype=torch.complex64, device="cuda")
        if tuple(out.shape) != shape or out.dtype != torch.complex64 or not out.is_contiguous():
            raise ValueError("out must be a contiguous complex64 tensor of shape %s" % (shape,))
        check(lib().img2d_plan_dense_table(self._h, int(which), ptr(out), self._stream(stream)))
        return out

    def execute_naive(self, wave, shot, image, stream=None):
        check(lib().img2d_plan_execute_naive(self._h, ptr(wave), ptr(shot), ptr(image), self._stream(stream)))

    def kernel_ms(self):
        """Device time of the migration kernel of the last execute (waits for it)."""
        v = ctypes.c_float()
        check(lib().img2d_plan_kernel_ms(self._h, ctypes.byref(v)))
        return v.value

    def check_status(self, stream=None):
        """Raise LibraryError if a bounded wait inside the last migration kernel gave up (its results
        are then invalid); waits for that kernel."""
        check(lib().img2d_plan_status(self._h, self._stream(stream)))

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


# ---------------------------------------------------------------------------------------------
# Autotuning and graph capture
# ---------------------------------------------------------------------------------------------

# Candidate kernel configurations, as Plan keyword arguments.  cluster2 variants differ in warps per
# CTA (positions per CTA), operator-pair prefetch depth, L1 row prefetch, packed arithmetic, and how
# operator indices, Kahan rows and tap pairs reach the tap loop (L1, shared-memory stage or ring).
N_CLUSTER2_VARIANTS = 12
CANDIDATES = [("default", {})] + [("cluster2/v%d" % v, {"variant": v}) for v in range(1, N_CLUSTER2_VARIANTS + 1)] + \
             [("wide/ffma2", {"wide": True}), ("wide/ffma", {"wide_scalar": True}), ("wide/bulk", {"wide_bulk": True}),
              ("wide/lines", {"wide": True, "line_packing": True}),
              ("cluster2", {"cluster2": True}),
              ("cluster1", {"cluster_v1": True}), ("single-cta", {"no_cluster": True})]


def autotune(ns, nextrap, nz, nx, nf, nt, M, nk, dk, omega, velocity, table, wave, shot, shot_x0=None,
             shot_nx=None, trial_depths=12, repeats=2, candidates=None, margin=0.02):
    """Pick the fastest kernel configuration for this geometry.

    Each candidate runs the first `trial_depths` depth steps of the migration (every shot and
    frequency) on copies of the device wavefields; its kernel time is the best of `repeats` runs
    after one warm-up.  Candidates that do not apply to the geometry, or that resolve to the same
    kernel configuration as an earlier one, are skipped.  The first candidate (the plan's default
    configuration) is kept unless another is faster by more than `margin` (a near-tie is timing
    noise, and the default is the configuration the tests cover most).  Returns (chosen Plan
    kwargs, table of (milliseconds, name, describe()) with the chosen row first, the rest fastest
    first)."""
    import torch
    from ._lib import LibraryError
    trial = max(1, min(nextrap, trial_depths))
    seen = set()
    table_rows = []
    for name, kw in (candidates or CANDIDATES):
        try:
            plan = Plan(ns, trial, nz, nx, nf, nt, M, nk, shot_x0, shot_nx, **kw)
        except LibraryError:
            continue
        d = plan.describe()
        key = (d["kernel"], d["variant"], d["cluster"], d["G"], d["block"], d.get("packing"))
        if key in seen:
            plan.close()
            continue
        seen.add(key)
        plan.set_model(omega, velocity, dk, table)
        w2, s2 = wave.clone(), shot.clone()
        img = torch.zeros((nz, nx), dtype=torch.float32, device=wave.device)
        times = []
        for _ in range(repeats + 1):
            plan.execute(w2, s2, img)
            times.append(plan.kernel_ms())
        try:
            plan.check_status()
        except LibraryError:
            plan.close()
            continue
        table_rows.append((min(times[1:]), name, d, kw))
        plan.close()
    if not table_rows:
        raise RuntimeError("no kernel configuration applies to this geometry")
    first = table_rows[0]
    table_rows.sort(key=lambda r: r[0])
    if table_rows[0] is not first and table_rows[0][0] >= first[0] * (1.0 - margin):
        table_rows.remove(first)
        table_rows.insert(0, first)
    return table_rows[0][3], [(t, n, d) for t, n, d, _ in table_rows]


def tuned_plan(w, omega, velocity, table, wave, shot, **kw):
    """Plan for synthetic.Workload-like `w` with the configuration autotune() picks."""
    best, report = autotune(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, omega, velocity, table, wave,
                            shot, shot_x0=w.shot_x0, shot_nx=w.shot_nx, **kw)
    return Plan.for_workload(w, **best), report


class GraphedExecution:
    """One migration of a plan (or its naive per-(shot, w, z) launch sequence) captured as a CUDA
    graph on fixed device buffers; replay() re-runs it with whatever the buffers hold."""

    def __init__(self, plan, wave, shot, image, naive=False):
        import torch
        self.plan, self.naive = plan, naive
        self.buffers = (wave, shot, image)
        run = plan.execute_naive if naive else plan.execute
        # one eager run creates the plan's lazily made resources (events, scratch) before capture
        run(wave, shot, image)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            run(wave, shot, image)
        torch.cuda.synchronize()

    def replay(self):
        self.graph.replay()
