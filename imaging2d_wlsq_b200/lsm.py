"""Least-squares migration on the B200 kernels: the migration operator, its adjoint (demigration),
torch.autograd bindings, and conjugate-gradient solvers.

No counterpart in the reference, which only migrates (main.py:136-186 calls the extrapolation
libraries once and stacks the per-shot images).  The forward map here is the reference's
migration, cpp_src/extrapolation_cpu.cpp:39-89, seen as a linear map of the receiver spectra d for
a fixed source:

    F d = image,  image[l, x] = Re sum_{shots, w} S_{l+1}[x] conj(R_{l+1}[x]),  R_0 = d

(Plan.execute), and the modelling operator of least-squares migration is its adjoint

    F* m = demigrated receiver spectra of the reflectivity m      (Plan.demigrate)

with <F d, m> = Re sum d conj(F* m).  Least-squares migration solves min_m 1/2 ||F* m - d_obs||^2.

Data live on the device in the packed wavefield layout of the plan (complex64, per shot nt rows of
that shot's aperture); images are float32 (nextrap, nx).

Several GPUs: each rank builds its operator on its own shots (sharding.assign_shots) and passes the
process group.  Its migration all-reduces the image, so images (reflectivity, gradient, search
direction) are the same on every rank, and inner products of data (residuals stay with their shots)
are all-reduced; the solvers below then run unchanged, one image all-reduce per migration.
"""
import time

import numpy as np

from .migration import Plan


class MigrationOperator:
    """F (migrate) and F* (demigrate) for one survey geometry, model and source.

    plan    a migration.Plan whose model is set (single-table mode)
    wave    device complex64 source spectra in the plan's packed layout; kept, never modified
    """

    def __init__(self, plan, wave, slab_depth=0, keep_source=True, group=None):
        """keep_source: the first demigration keeps the source checkpoints on the plan and later
        ones reuse them (the source does not change between calls); False recomputes every time.
        group: torch.distributed process group when the shots are shared out over ranks."""
        import torch
        self.plan = plan
        self.wave = wave
        self.slab_depth = slab_depth
        self.keep_source = keep_source
        self.group = group
        self._kept = False
        self.nextrap, self.nx = plan.nextrap, plan.nx
        self.device = wave.device
        self._src = torch.empty_like(wave)
        self._rec = torch.empty_like(wave)

    @classmethod
    def for_workload(cls, w, device=None, slab_depth=0, keep_source=True, group=None, **plan_kw):
        import torch
        dev = device or torch.device("cuda")
        plan = Plan.for_workload(w, **plan_kw)
        plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                       w.dk, torch.from_numpy(w.table).to(dev))
        return cls(plan, torch.from_numpy(w.wave).to(dev), slab_depth=slab_depth, keep_source=keep_source,
                   group=group)

    def data_dot(self, a, b):
        """Real inner product of two data vectors, summed over the ranks that share the shots."""
        return _allreduce_scalar(_dot_r(a, b), self.group, self.device)

    def image_dot(self, a, b):
        """Real inner product of two images (replicated on every rank: no communication)."""
        return _dot_r(a, b)

    def zeros_data(self):
        import torch
        return torch.zeros_like(self.wave)

    def zeros_image(self):
        import torch
        return torch.zeros((self.nextrap, self.nx), dtype=torch.float32, device=self.device)

    def migrate(self, data, image=None):
        """F d: stacked image (nextrap, nx) of the receiver spectra `data` (not modified)."""
        import torch
        image = self.zeros_image() if image is None else image
        self._src.copy_(self.wave)
        self._rec.copy_(data)
        self.plan.execute(self._src, self._rec, image, stream=torch.cuda.current_stream(self.device))
        if self.group is not None:
            import torch.distributed as dist
            dist.all_reduce(image, group=self.group)
        return image

    def demigrate(self, refl, data=None):
        """F* m: receiver spectra (packed layout) of the reflectivity `refl` (nextrap, nx)."""
        import torch
        data = self.zeros_data() if data is None else data
        source = "recompute"
        if self.keep_source:
            source = "reuse" if self._kept else "keep"
        self.plan.demigrate(refl.contiguous(), self.wave, data, slab_depth=self.slab_depth, source=source,
                            stream=torch.cuda.current_stream(self.device))
        self._kept = self._kept or source == "keep"
        return data


def _functions():
    import torch

    class Demigrate(torch.autograd.Function):
        """refl (real) -> data (complex).  Backward: the gradient of a real loss with respect to
        refl is F applied to the complex gradient of the data (torch's convention
        dL/dRe + i dL/dIm)."""

        @staticmethod
        def forward(ctx, refl, op):
            ctx.op = op
            return op.demigrate(refl)

        @staticmethod
        def backward(ctx, grad_data):
            return ctx.op.migrate(grad_data.contiguous()), None

    class Migrate(torch.autograd.Function):
        """data (complex) -> image (real).  Backward: F* of the image gradient."""

        @staticmethod
        def forward(ctx, data, op):
            ctx.op = op
            return op.migrate(data)

        @staticmethod
        def backward(ctx, grad_image):
            return ctx.op.demigrate(grad_image.contiguous()), None

    return Demigrate, Migrate


_FN = None


def _fn():
    global _FN
    if _FN is None:
        _FN = _functions()
    return _FN


def demigrate(refl, op):
    """Differentiable F* refl."""
    return _fn()[0].apply(refl, op)


def migrate(data, op):
    """Differentiable F data."""
    return _fn()[1].apply(data, op)


def _dot_r(a, b):
    """Real inner product in float64: sum a b for real tensors, Re sum a conj(b) for complex."""
    import torch
    if a.is_complex():
        return float(torch.sum(a.real.double() * b.real.double() + a.imag.double() * b.imag.double()))
    return float(torch.sum(a.double() * b.double()))


def _allreduce_scalar(v, group, device):
    if group is None:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    return float(t.item())


def _sync(op):
    import torch
    if op.device.type == "cuda":
        torch.cuda.synchronize(op.device)


def dot_product_test(op, seed=0, data=None, refl=None, separation=0.0):
    """<F d, m> against Re sum d conj(F* m) for seeded Gaussian d and m.  Returns
    (lhs, rhs, rel, rel_norms) with rel = |lhs - rhs| / max(|lhs|, |rhs|) and
    rel_norms = |lhs - rhs| / (||F d|| ||m||).

    For independent Gaussian vectors lhs = ||F d|| z with z ~ N(0, 1) the normalised projection of m
    on F d, while the FP32 rounding of F and F* contributes |lhs - rhs| ~ eps ||F d|| with eps a
    few 1e-7; so rel ~ eps / |z| is ill-conditioned for seeds where m is nearly orthogonal to F d.
    separation > 0 adds sign(z) * separation * F d / ||F d|| to the Gaussian m (a vector of norm
    `separation`, against ||m|| ~ sqrt(image size)), which makes |z| >= separation for every seed
    while m stays a Gaussian vector to within that tiny component; rel then measures eps.  A wrong
    tap, row or depth order gives rel ~ 1e-3 either way."""
    import torch
    g = torch.Generator(device=op.device).manual_seed(seed)
    if data is None:
        data = torch.randn(op.wave.shape, dtype=torch.complex64, device=op.device, generator=g)
    if refl is None:
        refl = torch.randn((op.nextrap, op.nx), dtype=torch.float32, device=op.device, generator=g)
    img = op.migrate(data)
    if separation > 0.0:
        nimg = np.sqrt(op.image_dot(img, img))
        sgn = 1.0 if op.image_dot(img, refl) >= 0.0 else -1.0
        refl = (refl.double() + (sgn * separation / nimg) * img.double()).float()
    lhs = op.image_dot(img, refl)
    rhs = op.data_dot(data, op.demigrate(refl))
    scale = np.sqrt(op.image_dot(img, img) * op.image_dot(refl, refl))
    return lhs, rhs, abs(lhs - rhs) / max(abs(lhs), abs(rhs)), abs(lhs - rhs) / scale


def misfit(op, refl, d_obs):
    """J(m) = 1/2 ||F* m - d_obs||^2 in float64."""
    r = op.demigrate(refl) - d_obs
    return 0.5 * op.data_dot(r, r)


def finite_difference_check(op, refl, d_obs, points, h):
    """Gradient of J at `refl` by autograd (through Demigrate) against central differences
    (J(m + h e_i) - J(m - h e_i)) / 2h at the image points `points` [(l, x), ...].  J is quadratic,
    so the central difference is exact up to rounding for any h.  Returns (autograd, fd) arrays."""
    import torch
    m = refl.detach().clone().requires_grad_(True)
    r = demigrate(m, op) - d_obs
    # each rank back-propagates its shots' misfit; the migration in the backward sums the ranks
    loss = 0.5 * (r.real.double().pow(2).sum() + r.imag.double().pow(2).sum())
    loss.backward()
    grad = m.grad.detach()
    ga, fd = [], []
    with torch.no_grad():
        for (l, x) in points:
            mp = refl.detach().clone()
            mp[l, x] += h
            jp = misfit(op, mp, d_obs)
            mp[l, x] -= 2 * h
            jm = misfit(op, mp, d_obs)
            ga.append(float(grad[l, x]))
            fd.append((jp - jm) / (2 * h))
    return np.array(ga), np.array(fd)


def lsm_cg(op, d_obs, niter, refl0=None, callback=None):
    """Least-squares migration by conjugate gradients on 1/2 ||F* m - d_obs||^2 with the gradient
    from torch autograd: each iteration evaluates the misfit through Demigrate, back-propagates
    (one migration), takes the Fletcher-Reeves direction and the exact step along it (one more
    demigration).  Returns (m, history) with history rows (iteration, ||r||, seconds)."""
    import torch
    m = op.zeros_image() if refl0 is None else refl0.detach().clone()
    p = None
    gg_prev = None
    hist = []
    _sync(op)
    t0 = time.perf_counter()
    for it in range(niter + 1):
        m.requires_grad_(True)
        r = demigrate(m, op) - d_obs
        rr = r.real.double().pow(2).sum() + r.imag.double().pow(2).sum()
        loss = 0.5 * rr
        rnorm = float(np.sqrt(_allreduce_scalar(float(rr.detach()), op.group, op.device)))
        if it == niter:
            _sync(op)
            hist.append((it, rnorm, time.perf_counter() - t0))
            m = m.detach()
            break
        loss.backward()
        g = m.grad.detach()
        m = m.detach()
        _sync(op)
        hist.append((it, rnorm, time.perf_counter() - t0))
        if callback:
            callback(it, m, rnorm)
        gg = op.image_dot(g, g)
        p = -g if p is None else -g + (gg / gg_prev) * p
        gg_prev = gg
        with torch.no_grad():
            q = op.demigrate(p)
            alpha = -op.image_dot(g, p) / op.data_dot(q, q)
            m = m + alpha * p
    return m, hist


def cgls(op, d_obs, niter, refl0=None):
    """The same least-squares problem by CGLS without autograd: one demigration and one migration
    per iteration, residual updated by recursion.  Returns (m, history) like lsm_cg."""
    import torch
    m = op.zeros_image() if refl0 is None else refl0.detach().clone()
    r = d_obs - op.demigrate(m) if refl0 is not None else d_obs.clone()
    s = op.migrate(r)
    p = s.clone()
    gamma = op.image_dot(s, s)
    hist = []
    _sync(op)
    t0 = time.perf_counter()
    hist.append((0, float(np.sqrt(op.data_dot(r, r))), 0.0))
    for it in range(niter):
        q = op.demigrate(p)
        alpha = gamma / op.data_dot(q, q)
        m = m + alpha * p
        r = r - alpha * q
        s = op.migrate(r)
        gamma_new = op.image_dot(s, s)
        p = s + (gamma_new / gamma) * p
        gamma = gamma_new
        _sync(op)
        hist.append((it + 1, float(np.sqrt(op.data_dot(r, r))), time.perf_counter() - t0))
    return m, hist
