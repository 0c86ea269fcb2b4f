"""Host parts of the driver flow: the pandas-free problem configuration (problemConfig.py:6-53),
shot-file discovery (readShotFiles.py:4-13), record reading and the operator tables, checked
against the values the reference computed for its demo (tests/golden/demo_case.npz)."""
import numpy as np

from imaging2d_wlsq_b200 import config as cfgmod
from imaging2d_wlsq_b200 import driver
from tests.conftest import rel_l2

# the demo's problemSetup.txt values (key_value lines)
DEMO_SETUP = """key_value

nt_800
nw_60

zmin_0
zmax_2000

zinit_0
zfinal_1800

xmin_-1000
xmax_1000

tmin_0.0
tmax_0.8

M_21
"""


def test_problem_config_matches_reference_demo(golden_demo):
    g = golden_demo
    c = cfgmod.ProblemConfig(text=DEMO_SETUP, nz=int(g["nz"]), nx=int(g["nx"]), ny=1)
    assert (c.nt, c.nw, c.M, c.nextrap) == (800, 60, int(g["M"]), int(g["nextrap"]))
    assert c.dx == float(g["dx"]) and c.dz == float(g["dz"])
    np.testing.assert_array_equal(c.w[:c.nw], g["omega"])
    assert c.N == (int(g["nx"]) - 1) // 2 and c.xilocal.dtype == np.float32 and len(c.xilocal) == 2 * c.M + 1


def test_operator_tables_match_reference_demo(golden_demo):
    g = golden_demo
    c = cfgmod.ProblemConfig(text=DEMO_SETUP, nz=int(g["nz"]), nx=int(g["nx"]), ny=1)
    tf, tb, dk = driver.operator_tables(c, g["velocity"])
    assert tf.shape == g["tab_f"].shape and dk == float(g["dk"])
    # bit-identical to the rows of the reference's makeTableOfOperators
    np.testing.assert_array_equal(tf, g["tab_f"])
    np.testing.assert_array_equal(tb, g["tab_b"])


def test_shot_files_and_records(tmp_path):
    rng = np.random.default_rng(0)
    recs = {}
    for isx in (7, 42, 105):
        r = rng.standard_normal((5, 4)).astype(np.float32)
        np.savetxt(tmp_path / f"seis{isx}_4.csv", r, delimiter=",")
        np.save(tmp_path / f"seis{isx}_4.npy", r)
        recs[isx] = r
    isx, files = driver.shot_files(str(tmp_path))
    assert sorted(isx) == [7, 42, 105]
    for i, f in zip(isx, files):
        np.testing.assert_allclose(driver.read_record(f), recs[i], rtol=1e-6)
        np.testing.assert_array_equal(driver.read_record(f[:-4] + ".npy"), recs[i])
    isx_npy, _ = driver.shot_files(str(tmp_path), extension="npy")
    assert sorted(isx_npy) == [7, 42, 105]
