"""Least-squares migration over ranks that share the shots, on CPU with gloo.

A small dense operator stands in for the GPU migration (F d = Re(A d), F* m = conj(A)^T m, the same
real-linear pair as the migration and its demigration).  Each of two ranks holds the columns of A
of its own data.  The solvers in imaging2d_wlsq_b200.lsm (CGLS, and CG with the autograd
gradient) must reproduce the single-process solution of the stacked system, and the dot-product
test must hold across the ranks.
"""
import datetime
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from imaging2d_wlsq_b200 import lsm

NI = (6, 10)          # image shape (depth steps, positions)
ND = (40, 35)         # data samples on rank 0 and rank 1


class DenseOperator(lsm.MigrationOperator):
    """Host stand-in with the operator interface the solvers use."""

    def __init__(self, A, group=None):
        self.A = A
        self.group = group
        self.device = torch.device("cpu")
        self.nextrap, self.nx = NI
        self.wave = torch.zeros(A.shape[1], dtype=torch.complex64)

    def zeros_data(self):
        return torch.zeros(self.A.shape[1], dtype=torch.complex64)

    def migrate(self, data, image=None):
        img = (self.A @ data.to(self.A.dtype)).real.to(torch.float32).reshape(NI).contiguous()
        if self.group is not None:
            dist.all_reduce(img, group=self.group)
        return img

    def demigrate(self, refl, data=None):
        return (self.A.conj().T @ refl.reshape(-1).to(self.A.dtype)).contiguous()


def _system():
    g = torch.Generator().manual_seed(0)
    ni = NI[0] * NI[1]
    A = [torch.complex(torch.randn(ni, n, generator=g), torch.randn(ni, n, generator=g)) for n in ND]
    m_true = torch.randn(NI, generator=g)
    d = [(a.conj().T @ m_true.reshape(-1).to(a.dtype)) for a in A]
    return A, d


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    A, d = _system()
    op = DenseOperator(A[rank], group=dist.group.WORLD)
    m_cg, h_cg = lsm.cgls(op, d[rank], 6)
    m_ag, h_ag = lsm.lsm_cg(op, d[rank], 6)
    dots = lsm.dot_product_test(op, seed=1, data=torch.randn(ND[rank], dtype=torch.complex64),
                                refl=torch.full(NI, 0.5))
    if rank == 0:
        q.put((m_cg.numpy(), [h[1] for h in h_cg], m_ag.numpy(), [h[1] for h in h_ag], dots))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_single_process_solution():
    A, d = _system()
    op = DenseOperator(torch.cat(A, dim=1))
    dd = torch.cat(d)
    m_cg, h_cg = lsm.cgls(op, dd, 6)
    m_ag, h_ag = lsm.lsm_cg(op, dd, 6)

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    dm_cg, dh_cg, dm_ag, dh_ag, dots = res
    scale = np.linalg.norm(m_cg.numpy())
    assert np.linalg.norm(dm_cg - m_cg.numpy()) <= 1e-4 * scale
    assert np.linalg.norm(dm_ag - m_ag.numpy()) <= 1e-4 * scale
    np.testing.assert_allclose(dh_cg, [h[1] for h in h_cg], rtol=1e-4)
    np.testing.assert_allclose(dh_ag, [h[1] for h in h_ag], rtol=1e-4)
    assert dh_cg[-1] < 0.5 * dh_cg[0]
    assert dots[3] <= 1e-6  # <F d, m> = <d, F* m> summed over the ranks
