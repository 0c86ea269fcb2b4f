"""The reference driver's flow end to end on this library: CSV velocity model and the nine CSV shot
records of the reference demo (written from tests/golden/driver_case.npz into the reference's
directory layout), problem setup, operator design, device front end and one batched migration,
against the image the reference flow (its Python preparation and its CPU extrapolation library)
produced from the same shots, within 1e-5 relative L2 (the bar of the migration parity tests), and
against the reference's shipped demo result (demo-result/final_image.csv) within 3e-5 (that file
was written by another build of the reference, whose FP32 sums ran in another order)."""
import numpy as np
import pytest

from imaging2d_wlsq_b200 import driver
from tests.conftest import rel_l2
from tests.test_driver_host import DEMO_SETUP

pytestmark = pytest.mark.gpu


def test_driver_reproduces_reference_flow(tmp_path):
    g = dict(np.load("tests/golden/driver_case.npz"))
    vel_path = tmp_path / "velmod.csv"
    np.savetxt(vel_path, g["velmod"], delimiter=",", fmt="%.17g")
    cfg_path = tmp_path / "problemSetup.txt"
    cfg_path.write_text(DEMO_SETUP)
    shots = tmp_path / "seismicShots"
    shots.mkdir()
    nx = g["records"].shape[2]
    for isx, rec in zip(g["shot_isx"], g["records"]):
        np.savetxt(shots / f"seis{int(isx)}_{nx}.csv", rec, delimiter=",", fmt="%.9g")
    image, vel, config = driver.run(str(vel_path), str(cfg_path), str(shots))
    assert image.shape == (config.nz, config.nx)
    assert len(g["records"]) == 9
    assert rel_l2(image, g["image"]) <= 1e-5
    shipped = np.load("tests/golden/demo_case.npz")["image_shipped"]
    assert rel_l2(image, shipped) <= 3e-5
    assert np.all(image[config.nextrap:] == 0)
