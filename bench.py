#!/usr/bin/env python
"""Benchmark of the extrapolation + imaging path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One step = one full migration (every shot x frequency x depth step, imaging included) of the
workload with inputs resident in HBM.  The default workload is `batched_uneven`: nz=1000,
nx=2048, nf=512 (2-50 Hz), 2M+1=35 taps, nk=4000, 256 shots with apertures U[256, 2048] (seeded
synthetic data).  Metric: extrapolated points (shot, w, z, x) per second, whole job.

Multi-GPU (torchrun, one rank per GPU): weak scaling; every rank migrates the single-GPU survey
(the same seeded shot set) and the stacked images are summed with one all-reduce per step.

Prints one JSON line (rank 0).  Other modes:
  --impl reference   the reference's own CPU library (oracle/_ref/extrapolation_cpu.so, all host
                     threads) on a fixed bounded sample of the same workload (ReferenceSample, the
                     sample of the GPU arm's cpu_baseline leg), same metric and config.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

import numpy as np  # noqa: E402

METRIC = "extrapolated pts/s (shot*w*z*x), batched vs plain on 1 GPU; rel-L2 err vs FP64"
UNIT = "pts/s"


# DRAM and L2 traffic per extrapolated point of the migration kernels, measured by one ncu capture of
# the small case of the batched_uneven workload (nz=60, nf=64: 9.68e8 points per launch):
# dram = (dram__bytes_read.sum + dram__bytes_write.sum) / points, l2 = lts__t_sectors.sum * 32 / points.
# Keyed by (kernel, variant) of describe(); the bench scales them by the points of its launch.
TRAFFIC_PER_POINT = {
    ("migrate_wide", 3): {"dram": 2.38, "l2": 82.4,
                          "capture": "migrate_wide_kernel<1, 1, 0>, window packing, nz=60 nf=64"},
    ("migrate_cluster2", 11): {"dram": 0.980, "l2": 45.8, "capture": "migrate_cluster2_kernel ring variant, nz=60 nf=64"},
}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="batched_uneven")
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--e2e-steps", type=int, default=0, help="end-to-end calls timed (0: as many as --steps)")
    p.add_argument("--strong", action="store_true",
                   help="strong scaling: the ranks split one survey's shots (sharding.migrate_sharded's "
                        "decomposition) instead of each migrating the whole survey")
    p.add_argument("--variant", type=int, default=0, help="cluster-kernel variant (1-based; 0 = default)")
    p.add_argument("--no-autotune", action="store_true", help="use the plan's default kernel configuration")
    p.add_argument("--nz", type=int, default=None, help="override depth steps (profiling a reduced case)")
    p.add_argument("--nf", type=int, default=None, help="override frequency count (profiling a reduced case)")
    p.add_argument("--taps", type=int, default=None,
                   help="override the operator length 2M+1 (odd; timing the per-step overhead)")
    p.add_argument("--cpu-seconds", type=float, default=8.0,
                   help="reference-library time of the GPU arm's CPU-baseline leg (passes over the fixed sample)")
    p.add_argument("--ref-step-seconds", type=float, default=2.0,
                   help="reference-library time per step of --impl reference (passes over the fixed sample)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-naive", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-lsm", action="store_true", help="skip the demigration / least-squares migration leg")
    p.add_argument("--lsm-iters", type=int, default=10)
    p.add_argument("--lsm-scale", type=float, default=1.0, help="shrink the lsm configuration (profiling)")
    p.add_argument("--no-frontend", action="store_true", help="skip the front-end (wavelet, record spectra) leg")
    p.add_argument("--no-accuracy", action="store_true",
                   help="skip the rel-L2 check of the image against the FP64 checker on a sub-volume")
    p.add_argument("--kernel", default="auto", choices=["auto", "cluster2", "wide", "wide-scalar", "wide-bulk", "wide-lines",
                                                           "cluster1", "single"],
                   help="kernel family (comparison runs and profiling); auto = the autotuner's choice")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = [num(r[2]) for r in rows if num(r[2])]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


class quiet_stdout:
    """Send file descriptor 1 to stderr while a C library that prints on stdout runs (its stdio
    buffer is flushed before fd 1 is restored)."""

    def __enter__(self):
        import ctypes
        self.libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self.libc.fflush(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


class ReferenceSample:
    """A fixed, bounded sample of workload w for the reference's own CPU library
    (oracle/_ref/extrapolation_cpu.so): `shots` shots at evenly spaced ranks of the aperture widths
    (narrowest to widest), `freqs` of the frequencies (evenly spaced over the band), the first
    `depth` depth steps, each shot one call of the reference's `extrapolate` on its own aperture
    (ns = 1, nx = the aperture width, as the reference handles one geometry per call).  The dense
    tables are gathered once here and are not timed, as the reference's EXTRAPOLATION and IMAGING
    timers exclude table building.  The same sample serves the reference arm and the CPU leg of
    the GPU arm, so the two rates measure the same thing."""

    def __init__(self, w, shots=8, freqs=64, depth=8):
        from oracle import oracle
        if not oracle.have_ref():
            raise RuntimeError("oracle/_ref/extrapolation_cpu.so missing")
        self.oracle = oracle
        order = np.argsort(w.shot_nx, kind="stable")
        pick = order[np.unique(np.linspace(0, len(order) - 1, min(shots, w.ns)).round().astype(int))]
        jsel = np.unique(np.linspace(0, w.nf - 1, min(freqs, w.nf)).round().astype(int))
        self.depth = depth = int(min(depth, w.nextrap))
        self.nf = nf = len(jsel)
        self.M = w.M
        self.calls = []
        for s in pick:
            x0, n = int(w.shot_x0[s]), int(w.shot_nx[s])
            om = np.ascontiguousarray(w.omega[jsel])
            tf = oracle.gather_dense_slab(0, depth, w.nx, x0, n, nf, w.M, w.nk, w.dk, om, w.velocity, w.table)
            tb = oracle.gather_dense_slab(0, depth, w.nx, x0, n, nf, w.M, w.nk, w.dk, om, w.velocity, w.table,
                                          conj_rows=True)
            wave = np.ascontiguousarray(w.block(w.wave, s)[jsel][None])
            shot = np.ascontiguousarray(w.block(w.shot, s)[jsel][None])
            self.calls.append((n, tf, tb, wave, shot))
        self.points = sum(n * nf * depth for n, *_ in self.calls)
        self.desc = (f"reference extrapolation_cpu.so, {len(self.calls)} shots at evenly spaced ranks of the "
                     f"aperture widths ({', '.join(str(c[0]) for c in self.calls)} traces), {nf} of {w.nf} "
                     f"frequencies, first {depth} depth steps, one call per shot; {self.points:.3g} points per "
                     "pass; dense tables gathered beforehand and not timed")

    def run_pass(self):
        """One pass over the sample; returns the seconds spent inside the reference's calls."""
        secs = 0.0
        with quiet_stdout():  # the reference library prints its phase timers on stdout
            for n, tf, tb, wave0, shot0 in self.calls:
                wave, shot = wave0.copy(), shot0.copy()
                img = np.zeros((1, self.depth, n), dtype=np.float32)
                t0 = time.perf_counter()
                self.oracle.ref_extrapolate(1, self.depth, self.depth, n, self.nf, self.nf, self.M, tf, tb, wave,
                                            shot, img)
                secs += time.perf_counter() - t0
        return secs

    def timed(self, seconds):
        """Passes until `seconds` of reference time have accumulated (at least one); returns
        (points, seconds)."""
        pts, secs = 0, 0.0
        while secs < seconds or pts == 0:
            secs += self.run_pass()
            pts += self.points
        return pts, secs


def cpu_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def run_reference_impl(args):
    """The reference arm: the reference's own CPU library on this host's cores, on the fixed sample
    of the GPU arm's workload (ReferenceSample); one step = passes over the sample for about
    `--ref-step-seconds` of reference time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from imaging2d_wlsq_b200 import synthetic
    world = int(os.environ.get("WORLD_SIZE", "1"))
    maker = synthetic.WORKLOADS[args.workload]
    over = {k: v for k, v in (("nz", args.nz), ("nf", args.nf)) if v}
    w = maker(scale=args.scale, **over)
    sample = ReferenceSample(w)
    pts_all, t_all = 0, 0.0
    for i in range(args.warmup + args.steps):
        pts, secs = sample.timed(args.ref_step_seconds)
        if i >= args.warmup:
            pts_all += pts
            t_all += secs
    value = pts_all / t_all
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_all / max(1, args.steps),
        "higher_is_better": True, "scaling": scaling(args, world), "vs_baseline": None,
        "dtype": "c64 (fp32 complex)", "data": "synthetic (seeded)", "config": run_config(w, args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu_threads(), "kind": "reference",
                         "sample": sample.desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def lsm_leg(dev, iters, scale=1.0):
    """Demigration (adjoint) and least-squares migration on the lsm configuration: nz=500, nx=1024,
    nf=256 (2-40 Hz), 31 taps, 64 full-aperture shots, 0.5% sparse reflectivity; observed data
    synthesised by the demigration kernel."""
    import torch
    from imaging2d_wlsq_b200 import lsm, synthetic
    w = synthetic.lsm(scale=scale)
    op = lsm.MigrationOperator.for_workload(w, device=dev)
    m_true = torch.from_numpy(w.reflectivity[:w.nextrap]).to(dev)
    # source checkpoints recomputed in the call (what a single demigration costs)
    scratch = op.zeros_data()
    for _ in range(3):
        op.plan.demigrate(m_true, op.wave, scratch, source="recompute")
    op.plan.demigrate(m_true, op.wave, scratch, source="recompute")
    kms_recompute = op.plan.kernel_ms()
    del scratch
    # the operator keeps them on its first call and reuses them after (the least-squares loop)
    for _ in range(3):
        d_obs = op.demigrate(m_true)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    d_obs = op.demigrate(m_true)
    e1.record()
    e1.synchronize()
    t_dem = e0.elapsed_time(e1) / 1e3
    kms_dem = op.plan.kernel_ms()
    d_obs = d_obs.clone()
    e0.record()
    op.migrate(d_obs)
    e1.record()
    e1.synchronize()
    t_mig = e0.elapsed_time(e1) / 1e3
    pts = w.points()
    dots = [lsm.dot_product_test(op, seed=sd) for sd in range(5)]
    dots_sep = [lsm.dot_product_test(op, seed=sd, separation=3.0) for sd in range(5)]
    rng = np.random.default_rng(5)
    pts16 = [(int(rng.integers(0, w.nextrap)), int(rng.integers(0, w.nx))) for _ in range(16)]
    ga, fd = lsm.finite_difference_check(op, torch.zeros_like(m_true), d_obs, pts16, h=1.0)
    _, hist = lsm.lsm_cg(op, d_obs, niter=iters)
    _, hist2 = lsm.cgls(op, d_obs, niter=iters)
    out = {
        "workload": f"lsm: nz={w.nz} nx={w.nx} nf={w.nf} taps={w.L} nk={w.nk} ns={w.ns} full aperture, "
                    "reflectivity 0.5% spikes * [1,2,1]/4 (z, x), d_obs = F* m_true",
        "demigration": {"value": pts / t_dem, "unit": UNIT, "seconds": t_dem, "kernel_ms": kms_dem,
                        "source": "kept checkpoints reused (every call after the operator's first)",
                        "recompute": {"value": pts / (kms_recompute / 1e3), "kernel_ms": kms_recompute,
                                      "source": "checkpoint pass inside the call"},
                        "kernel_config": op.plan.describe_demigration()},
        "migration": {"value": pts / t_mig, "unit": UNIT, "seconds": t_mig},
        "dot_product": {"rel": [d[2] for d in dots_sep], "rel_norms": [d[3] for d in dots_sep],
                        "rel_independent": [d[2] for d in dots], "rel_norms_independent": [d[3] for d in dots],
                        "seeds": 5, "vectors": "Gaussian d (complex); m Gaussian plus sign(z) * 3 * Fd/||Fd|| "
                                               "(projection on Fd kept >= 3 norms from orthogonality); "
                                               "*_independent: m Gaussian",
                        "rel_def": "|<Fd,m> - <d,F*m>| / max(|<Fd,m>|, |<d,F*m>|)",
                        "rel_norms_def": "|<Fd,m> - <d,F*m>| / (||Fd|| ||m||)"},
        "fd_gradient": {"points": 16, "h": 1.0, "max_abs_err_over_max_grad": float(np.max(np.abs(ga - fd)) /
                                                                                    np.abs(ga).max())},
        "cg_autograd": {"iterations": iters, "residual_ratio": hist[-1][1] / hist[0][1],
                        "s_per_iteration": hist[-1][2] / iters,
                        "per_iteration": "1 demigration + 1 migration (autograd backward) + 1 demigration (step)"},
        "cgls": {"iterations": iters, "residual_ratio": hist2[-1][1] / hist2[0][1],
                 "s_per_iteration": hist2[-1][2] / iters, "per_iteration": "1 demigration + 1 migration"},
    }
    op.plan.close()
    return out


def plain_medium_leg(dev):
    """The plain medium configuration in full (nz=500, nx=1024, nf=256 over 2-40 Hz, 31 taps, 32
    full-aperture shots: 4.19e9 points), migrated once by the batched kernel and once in the naive
    form, one launch per (shot, frequency, depth step): batched against plain on the same data."""
    import torch
    from imaging2d_wlsq_b200 import migration, synthetic
    w = synthetic.plain_medium()
    plan = migration.Plan.for_workload(w)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    wave0 = torch.from_numpy(w.wave).to(dev)
    shot0 = torch.from_numpy(w.shot).to(dev)
    img = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(run):
        wv, sh = wave0.clone(), shot0.clone()
        e0.record()
        run(wv, sh, img)
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    timed(plan.execute)
    t_batched = timed(plan.execute)
    t_naive = timed(plan.execute_naive)
    pts = w.points()
    out = {"workload": f"plain_medium: nz={w.nz} nx={w.nx} nf={w.nf} taps={w.L} ns={w.ns} full aperture",
           "batched": {"value": pts / t_batched, "unit": UNIT, "seconds": t_batched,
                       "kernel": plan.describe()["kernel"]},
           "naive": {"value": pts / t_naive, "unit": UNIT, "seconds": t_naive,
                     "launches": w.ns * w.nf * (w.nextrap + 1)},
           "batched_over_naive": t_naive / t_batched}
    plan.close()
    return out


def frontend_leg(dev, w):
    """Front end on the workload's shot geometry: time-domain records (ns, nt = 2 nf, nx) float32,
    resident on the device, to the first nf frequency rows of each shot's aperture; and the source
    wavelets of all shots (built and transformed).  CPU: the reference's own call of main.py:119
    (scipy.fftpack.fft along time) on one shot record, and the wavelet restatement on one shot."""
    import time as _time
    import torch
    import scipy.fftpack as spfft
    from imaging2d_wlsq_b200 import frontend
    ns, nx, nf = w.ns, w.nx, w.nf
    nt, dt = 2 * nf, 0.004
    g = torch.Generator(device=dev).manual_seed(11)
    rec = torch.randn((ns, nt, nx), generator=g, device=dev, dtype=torch.float32)
    out = torch.empty(int(nf * w.shot_nx.astype(np.int64).sum()), dtype=torch.complex64, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=3):
        fn()
        best = 1e30
        for _ in range(reps):
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        return best

    t_rec = timed(lambda: frontend.records_to_spectra(rec, nf, shot_x0=w.shot_x0, shot_nx=w.shot_nx, out=out))
    del rec
    sx = w.shot_pos.astype(np.float64) * w.dx
    src_out = torch.empty(ns * nf * nx, dtype=torch.complex64, device=dev)

    def sources():
        st = frontend.ricker_sources(ns, nt, nx, dt, 0.0, w.dx, 10.0, 2000.0, sx, device=dev)
        frontend.records_to_spectra(st, nf, out=src_out)

    t_src = timed(sources)
    samples = int(nt * w.shot_nx.astype(np.int64).sum())
    # CPU: one shot, the reference's transform call and the wavelet restatement
    one = np.random.default_rng(11).standard_normal((nt, nx)).astype(np.float32)
    c0 = _time.perf_counter()
    spfft.fft(one, axis=0)[:nf]
    c_fft = _time.perf_counter() - c0
    from oracle import frontend_oracle
    c0 = _time.perf_counter()
    frontend_oracle.ricker_sources(1, nt, nx, dt, 0.0, w.dx, 10.0, 2000.0, sx[:1])
    c_ric = _time.perf_counter() - c0
    return {
        "workload": f"ns={ns} nt={nt} nx={nx} nf={nf}, receiver records on the {w.name} apertures "
                    f"(mean {w.shot_nx.mean():.0f} traces); sources full aperture",
        "records": {"value": samples / t_rec, "unit": "time samples/s", "ms": t_rec * 1e3,
                    "hbm_gbs": (4.0 * ns * nt * nx + 8.0 * 2 * ns * (nt // 2 + 1) * nx + 8.0 * nf * w.shot_nx.sum())
                               / t_rec / 1e9,
                    "kernel": "cuFFT real-to-complex along time + pack_spectra_kernel (first nf rows, apertures)"},
        "sources": {"value": ns * nt * nx / t_src, "unit": "time samples/s", "ms": t_src * 1e3},
        "cpu_reference_fft": {"value": nt * nx / c_fft, "unit": "time samples/s", "ms_per_shot": c_fft * 1e3,
                              "cores": 1, "kind": "reference",
                              "sample": f"scipy.fftpack.fft of one ({nt}, {nx}) record, the call of main.py:119"},
        "cpu_port_ricker": {"value": nt * nx / c_ric, "unit": "time samples/s", "ms_per_shot": c_ric * 1e3,
                            "cores": 1, "kind": "port", "sample": "oracle wavelet restatement, one shot"},
    }


def dense_table_leg(dev, nl=100, cpu_nl=2):
    """The legacy ABI's dense operator table built on the device (img2d_plan_dense_table) for the
    plain medium geometry (nx=1024, nf=256 over 2-40 Hz, 31 taps, nk=2000): the first `nl` depth steps
    (6.5 GB of complex64, written once).  CPU: the numpy gather of operators.dense_table (the
    vectorised form of preparation.py:101-115) on the first `cpu_nl` depth steps, one host core; its
    rows are compared bit for bit with the device's."""
    import time as _time
    import torch
    from imaging2d_wlsq_b200 import migration, operators, synthetic
    w = synthetic.plain_medium()
    L = 2 * w.M + 1
    plan = migration.Plan(w.ns, nl, w.nz, w.nx, w.nf, w.nt, w.M, w.nk)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev))
    out = torch.empty((nl, w.nf, w.nx, L), dtype=torch.complex64, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    plan.dense_table(0, out=out)
    best = 1e30
    for _ in range(3):
        e0.record()
        plan.dense_table(0, out=out)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    head = out[:cpu_nl].cpu().numpy()
    plan.close()
    nbytes = out.numel() * 8
    del out
    torch.cuda.empty_cache()
    c0 = _time.perf_counter()
    host = operators.dense_table(w.table, w.omega, w.velocity, cpu_nl, dk=w.dk)
    c_s = _time.perf_counter() - c0
    rows = nl * w.nf * w.nx
    return {"workload": f"plain_medium geometry: first {nl} of {w.nz} depth steps, nf={w.nf} nx={w.nx} "
                        f"taps={L} nk={w.nk}, forward rows ({nbytes / 1e9:.2f} GB)",
            "value": rows / best, "unit": "operator rows/s", "ms": best * 1e3, "hbm_write_gbs": nbytes / best / 1e9,
            "kernel": "dense_table_kernel (img2d_plan_dense_table)",
            "cpu_port": {"value": cpu_nl * w.nf * w.nx / c_s, "unit": "operator rows/s", "cores": 1,
                         "kind": "port", "sample": f"operators.dense_table (numpy gather), first {cpu_nl} depth steps"},
            "bitwise_equal_to_host_gather": bool(np.array_equal(head, host))}


def workload_config(w, args):
    return {"workload": f"{w.name}: nz={w.nz} nx={w.nx} dx={w.dx} nf={w.nf} taps={w.L} nk={w.nk} ns={w.ns} "
                        f"apertures {int(w.shot_nx.min())}-{int(w.shot_nx.max())} (mean {w.shot_nx.mean():.0f})",
            "points_per_step": w.points(), "scale": args.scale, "seed": w.seed,
            "l2": "inputs (wavefields %.2f GB) larger than L2 (126 MB); no flush" % (2 * w.wave.nbytes / 1e9)}


def scaling(args, world):
    return "strong" if (args.strong and world > 1) else "weak"


def run_config(w, args, world):
    """The `config` object of both arms' JSON lines (identical for the same workload and N)."""
    return dict(workload_config(w, args), parallelism=f"shots x{world} ({scaling(args, world)})")


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference_impl(args)

    import torch
    import torch.distributed as dist
    from imaging2d_wlsq_b200 import migration, synthetic
    from imaging2d_wlsq_b200.sharding import sum_images_f64 as sharding_sum

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    # weak scaling: every rank migrates the full single-GPU survey (the same seeded shot set as N=1)
    maker = synthetic.WORKLOADS[args.workload]
    over = {k: v for k, v in (("nz", args.nz), ("nf", args.nf)) if v}
    w = maker(scale=args.scale, **over)
    if args.taps:
        from imaging2d_wlsq_b200 import operators
        w.M = (args.taps - 1) // 2
        w.table = operators.design_compact_table(w.nx, w.dx, w.dz, w.M, w.nk, w.dk)
    survey = w
    if args.strong and world > 1:
        # strong scaling: this rank's LPT share of the survey's shots
        from imaging2d_wlsq_b200 import sharding
        w = sharding.sub_workload(survey, sharding.assign_shots(survey.shot_nx, world)[rank])
    om = torch.from_numpy(w.omega).to(dev)
    vel = torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev)
    tab = torch.from_numpy(w.table).to(dev)
    wave0 = torch.from_numpy(w.wave).to(dev)
    shot0 = torch.from_numpy(w.shot).to(dev)
    tune_report = None
    if args.kernel == "auto" and args.variant == 0 and not args.no_autotune:
        # autotuner: every candidate kernel configuration on the first depth steps of this workload
        best, rows = migration.autotune(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.dk, om, vel, tab,
                                        wave0, shot0, shot_x0=w.shot_x0, shot_nx=w.shot_nx, trial_depths=8)
        tune_report = {"trial_depths": 8, "picked": rows[0][1],
                       "ms": {n: round(t, 3) for t, n, _ in rows}}
    else:
        best = dict(no_cluster=args.kernel == "single", cluster_v1=args.kernel == "cluster1", variant=args.variant,
                    wide=args.kernel in ("wide", "wide-lines"), wide_scalar=args.kernel == "wide-scalar",
                    wide_bulk=args.kernel == "wide-bulk", cluster2=args.kernel == "cluster2",
                    line_packing=args.kernel == "wide-lines")
    plan = migration.Plan.for_workload(w, **best)
    plan.set_model(om, vel, w.dk, tab)
    wave = torch.empty_like(wave0)
    shot = torch.empty_like(shot0)
    image = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
    pts_rank = w.points()

    def step():
        wave.copy_(wave0)
        shot.copy_(shot0)
        plan.execute(wave, shot, image)
        if world > 1:
            # the stacked image over all ranks, reduced in float64 (sharding.sum_images_f64)
            image.copy_(sharding_sum(image))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    e0.record()
    for _ in range(args.steps):
        step()
        kernel_ms.append(plan.kernel_ms())
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    plan.check_status()  # no bounded wait inside the timed launches gave up
    elapsed = e0.elapsed_time(e1) / 1e3
    t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    elapsed = float(t.item())
    total_pts = survey.points() if (args.strong and world > 1) else pts_rank * world
    value = total_pts * args.steps / elapsed
    k_s = float(np.mean(kernel_ms)) / 1e3
    describe = plan.describe()

    extra = {}
    if rank == 0:
        fp32 = migration.fp32_peak_tflops()
        flops_pt = 16 * w.L + 4
        bytes_pt = 8 * w.L
        hbm, hbm_src = peaks()
        ach = pts_rank * flops_pt / k_s / 1e12
        roof = {"bound": "fp32", "achieved": ach, "peak": fp32, "unit": "TFLOP/s", "frac": ach / fp32,
                "traffic": None, "kernel": describe["kernel"], "kernel_ms": k_s * 1e3,
                "per_point": f"{flops_pt} flop (16L+4, L={w.L})",
                "peak_source": "FP32 FMA probe kernel timed in this run (img2d_measure_fp32_peak); "
                               "MEASURED_PEAKS.json has no FP32 CUDA-core peak"}
        # per-point figures of the captured configuration only (batched_uneven geometry, 35 taps)
        tp = TRAFFIC_PER_POINT.get((describe.get("kernel"), describe.get("variant"))) \
            if (w.name == "batched_uneven" and w.L == 35) else None
        l2 = migration.l2_read_bandwidth_gbs()
        ach_alg = pts_rank * bytes_pt / k_s / 1e9
        roof_hbm = {"bound": "hbm", "achieved": None, "peak": hbm, "unit": "GB/s", "frac": None,
                    "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({hbm_src})",
                    "algorithmic_gbs": ach_alg,
                    "algorithmic_per_point": f"{bytes_pt} B (8L operator bytes, no cross-shot reuse credit); "
                                             "the rows are reused by the slots of an item from shared memory, "
                                             "so this rate is not a DRAM stream"}
        roof_l2 = {"bound": "l2", "achieved": None, "peak": l2, "unit": "GB/s", "frac": None,
                   "peak_source": "L2 read probe timed in this run (img2d_measure_l2_bandwidth); "
                                  "MEASURED_PEAKS.json has no L2 figure"}
        if tp:
            # measured bytes per point (small-case ncu capture) x the points of this launch
            traffic = tp["dram"] * pts_rank
            roof["traffic"] = traffic
            roof["traffic_unit"] = "DRAM bytes per launch"
            roof["traffic_source"] = (f"{tp['dram']} B/point from ncu of the small case ({tp['capture']}), "
                                      "scaled by this launch's points")
            roof_hbm.update(achieved=traffic / k_s / 1e9, frac=traffic / k_s / 1e9 / hbm,
                            per_point=f"{tp['dram']} B measured DRAM traffic (scaled from the small case)")
            l2b = tp["l2"] * pts_rank
            roof_l2.update(achieved=l2b / k_s / 1e9, frac=l2b / k_s / 1e9 / l2,
                           per_point=f"{tp['l2']} B measured L2 traffic (lts__t_sectors x 32, scaled from the "
                                     "small case)")
        extra["roofline"] = roof
        extra["roofline_hbm"] = roof_hbm
        extra["roofline_l2"] = roof_l2
        extra["binding"] = ("fp32: FP32 FMA work is the largest fraction of its measured peak; L2 and DRAM "
                            "carry measured traffic far below their peaks (operator rows reused from shared "
                            "memory; DRAM traffic is mostly the per-CTA Kahan partial-image rows)")
        extra["kernel_config"] = describe
        if tune_report:
            extra["autotune"] = tune_report

    # end to end through the host C entry point, pinned host buffers, copies inside the timed region
    if rank == 0 and not args.no_e2e:
        hw = torch.from_numpy(w.wave).pin_memory()
        hs = torch.from_numpy(w.shot).pin_memory()
        wave_h = hw.numpy()
        shot_h = hs.numpy()
        img_h = torch.zeros((w.nz, w.nx), dtype=torch.float32).pin_memory().numpy()
        from imaging2d_wlsq_b200._lib import check, lib, ptr
        x0 = np.ascontiguousarray(w.shot_x0, dtype=np.int32)
        wn = np.ascontiguousarray(w.shot_nx, dtype=np.int32)
        vel_h = np.ascontiguousarray(w.velocity)

        def e2e_call():
            wave_h[:] = w.wave
            shot_h[:] = w.shot
            ta = torch.cuda.Event(enable_timing=True)
            tb = torch.cuda.Event(enable_timing=True)
            ta.record(torch.cuda.default_stream())
            check(lib().img2d_migrate_compact(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, float(w.dk),
                                              ptr(w.omega), ptr(vel_h), ptr(w.table), None, ptr(x0), ptr(wn),
                                              ptr(wave_h), ptr(shot_h), ptr(img_h), None,
                                              migration.plan_flags(**best)))
            tb.record(torch.cuda.default_stream())
            tb.synchronize()
            return ta.elapsed_time(tb) / 1e3

        e2e_call()
        secs = [e2e_call() for _ in range(max(1, args.e2e_steps or args.steps))]
        h2d = w.wave.nbytes + w.shot.nbytes + w.omega.nbytes + w.nextrap * w.nx * 8 + w.table.nbytes
        d2h = w.wave.nbytes + w.shot.nbytes + w.nextrap * w.nx * 4
        extra["e2e"] = {"value": pts_rank / float(np.median(secs)), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h), "calls": len(secs),
                        "api": "img2d_migrate_compact (host buffers, flags of the timed kernel configuration)",
                        "n_gpus": 1}

    # naive one-launch-per-(shot, w, z) form on a sample of the same workload
    if rank == 0 and not args.no_naive:
        nf_s = min(w.nf, 4)
        ns_s = 1
        sub = synthetic.Workload(w.name, w.nz, w.nx, w.dx, w.dz, nf_s, w.M, w.nk, w.dk, w.omega[:nf_s], w.velocity,
                                 w.table, w.shot_x0[:ns_s], w.shot_nx[:ns_s], w.shot_pos[:ns_s], nextrap=w.nextrap)
        sub.wave = np.ascontiguousarray(w.block(w.wave, 0)[:nf_s]).reshape(-1)
        sub.shot = np.ascontiguousarray(w.block(w.shot, 0)[:nf_s]).reshape(-1)
        nplan = migration.Plan.for_workload(sub)
        nplan.set_model(torch.from_numpy(sub.omega.copy()).to(dev), vel, w.dk, tab)
        sw = torch.from_numpy(sub.wave).to(dev)
        ss = torch.from_numpy(sub.shot).to(dev)
        si = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
        nplan.execute_naive(sw, ss, si)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        nplan.execute_naive(sw, ss, si)
        a1.record()
        a1.synchronize()
        nsec = a0.elapsed_time(a1) / 1e3
        npts = sub.points()
        # the same launch sequence captured once as a CUDA graph and replayed
        g = migration.GraphedExecution(nplan, sw, ss, si, naive=True)
        a0.record()
        g.replay()
        a1.record()
        a1.synchronize()
        gsec = a0.elapsed_time(a1) / 1e3
        extra["plain_naive"] = {"value": npts / nsec, "unit": UNIT, "launches": ns_s * nf_s * (w.nextrap + 1),
                                "sample": f"1 shot x {nf_s} frequencies x {w.nextrap} depths, one launch per "
                                          "(shot, w, z)", "batched_over_naive": value / world / (npts / nsec),
                                "graph_replay_value": npts / gsec}
        del g
        nplan.close()

    if rank == 0 and not args.no_cpu_baseline and world == 1:
        # CPU leg: the reference's own library timed on a bounded sample, and the FP64 checker's image
        # of a sub-volume (first 40 depth steps, all shots and frequencies) against this run's kernel
        try:
            sample = ReferenceSample(w)
            sample.run_pass()  # warm-up pass (first touch of the library's buffers)
            pts, secs = sample.timed(args.cpu_seconds)
            extra["cpu_baseline"] = {"value": pts / secs, "unit": UNIT, "cores": cpu_threads(),
                                     "kind": "reference", "sample": sample.desc, "seconds": secs}
            del sample
        except Exception as ex:  # reference library not shipped with this tree
            extra["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                     "sample": f"unavailable: {ex}"}
        if not args.no_accuracy:
            from oracle import oracle
            sub_n = min(w.nextrap, 40)
            plan_a = migration.Plan(w.ns, sub_n, w.nz, w.nx, w.nf, w.nt, w.M, w.nk, w.shot_x0, w.shot_nx)
            plan_a.set_model(om, vel, w.dk, tab)
            wa = torch.from_numpy(w.wave).to(dev)
            sa = torch.from_numpy(w.shot).to(dev)
            ia = torch.zeros((w.nz, w.nx), dtype=torch.float32, device=dev)
            plan_a.execute(wa, sa, ia)
            torch.cuda.synchronize()
            stack, _, _, _ = oracle.migrate_workload_f64(w, nextrap=sub_n)
            got = ia.cpu().numpy().astype(np.float64)
            extra["accuracy"] = {"rel_l2": float(np.linalg.norm(got - stack) / np.linalg.norm(stack)),
                                 "max_abs_rel": float(np.abs(got - stack).max() / np.abs(stack).max()),
                                 "sub_volume": f"first {sub_n} depth steps, all shots and frequencies",
                                 "reference": "FP64 CPU checker"}
            plan_a.close()

    if rank == 0 and world == 1 and not args.no_naive:
        try:
            extra["plain_medium"] = plain_medium_leg(dev)
        except Exception as ex:
            extra["plain_medium"] = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0 and world == 1 and not args.no_frontend:
        try:
            extra["frontend"] = frontend_leg(dev, w)
        except Exception as ex:
            extra["frontend"] = {"error": f"{type(ex).__name__}: {ex}"}
        try:
            extra["dense_table"] = dense_table_leg(dev)
        except Exception as ex:
            extra["dense_table"] = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0 and world == 1 and not args.no_lsm:
        try:
            extra["lsm"] = lsm_leg(dev, args.lsm_iters, args.lsm_scale)
        except Exception as ex:
            extra["lsm"] = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": scaling(args, world), "vs_baseline": None, "dtype": "c64 (fp32 complex)",
            "data": "synthetic (seeded)", "config": run_config(survey, args, world),
            "clocks": clk, "gpu_launches": 2 * args.steps,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
