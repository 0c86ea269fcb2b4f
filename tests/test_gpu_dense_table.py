"""The legacy ABI's dense operator table gathered on the GPU (img2d_plan_dense_table), against the
oracle's gather of the same rows, and fed through the reference's dense-table `extrapolate`."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import interface, migration, operators, synthetic
from oracle import oracle
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _plan(w, two_tables=False, table_back=None):
    import torch
    plan = migration.Plan.for_workload(w, two_tables=two_tables)
    dev = torch.device("cuda")
    tb = None if table_back is None else torch.from_numpy(table_back).to(dev)
    plan.set_model(torch.from_numpy(w.omega).to(dev), torch.from_numpy(np.ascontiguousarray(w.velocity)).to(dev),
                   w.dk, torch.from_numpy(w.table).to(dev), tb)
    return plan


def _oracle_dense(w, table, conj=False):
    return oracle.gather_dense_slab(0, w.nextrap, w.nx, 0, w.nx, w.nf, w.M, w.nk, w.dk, w.omega, w.velocity,
                                    table, conj_rows=conj)


@pytest.mark.parametrize("make", [lambda: synthetic.plain_small(scale=0.25),
                                  lambda: synthetic.batched_uneven(scale=0.05)])
def test_dense_table_is_the_gathered_rows(make):
    """Forward rows and the conjugated receiver rows of a single-table plan, bit for bit."""
    w = make()
    plan = _plan(w)
    fwd = plan.dense_table(0).cpu().numpy()
    rec = plan.dense_table(1).cpu().numpy()
    plan.close()
    assert fwd.shape == (w.nextrap, w.nf, w.nx, 2 * w.M + 1)
    assert np.array_equal(fwd, _oracle_dense(w, w.table))
    assert np.array_equal(rec, _oracle_dense(w, w.table, conj=True))


def test_dense_back_table_of_a_two_table_plan():
    """A two-table plan gathers its receiver rows from tab_back (the reference's psBack table)."""
    w = synthetic.plain_small(scale=0.25)
    back = operators.design_compact_table(w.nx, w.dx, w.dz, w.M, w.nk, w.dk, back=True)
    plan = _plan(w, two_tables=True, table_back=back)
    rec = plan.dense_table(1).cpu().numpy()
    plan.close()
    assert np.array_equal(rec, _oracle_dense(w, back))


def test_dense_tables_through_the_legacy_extrapolate():
    """main.py's flow with the tables made on the GPU: dense forward and back tables into the
    reference's host-order `extrapolate`, against the compact-table entry point on the same data."""
    w = synthetic.plain_small(scale=0.25)
    back = operators.design_compact_table(w.nx, w.dx, w.dz, w.M, w.nk, w.dk, back=True)
    plan = _plan(w, two_tables=True, table_back=back)
    opF = np.ascontiguousarray(plan.dense_table(0).cpu().numpy())
    opB = np.ascontiguousarray(plan.dense_table(1).cpu().numpy())
    plan.close()
    wave, shot = w.wave.copy(), w.shot.copy()
    image = np.zeros((w.ns, w.nz, w.nx), dtype=np.float32)
    interface.extrapolate(w.ns, w.nextrap, w.nz, w.nx, w.nf, w.nt, w.M, opF, opB, wave, shot, image)
    stack, _, wave_c, shot_c = migration.migrate_workload(w, two_tables=True, table_back=back)
    assert rel_l2(image.sum(axis=0), stack) <= 1e-5
    assert rel_l2(wave, wave_c) <= 1e-5 and rel_l2(shot, shot_c) <= 1e-5


def test_dense_table_needs_a_model():
    w = synthetic.plain_small(scale=0.25)
    plan = migration.Plan.for_workload(w)
    with pytest.raises(Exception, match="set_model"):
        plan.dense_table(0)
    plan.close()
