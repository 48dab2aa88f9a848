"""Host-side arithmetic of bench.py: the per-kernel byte counts, the launch
count per step and the roofline table, on the 384 x 192 x 192 torus shape
(no GPU: the functions take the per-kernel times as plain numbers)."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from hamr_gamma_wind_b200 import problems  # noqa: E402

C3 = {"n1": 384, "n2": 192, "n3": 192}
# per-step kernel times (ms) of a mixed step with the inversion inside the
# update (the fallback pass a few % of it) and of one with the two kernels
FUSED = {"flux3": 2.24, "flux2": 1.72, "flux1": 1.65, "emf_centre": 0.005, "emf_edge": 0.58,
         "face_update": 0.66, "update": 4.25, "invert": 0.18}
SPLIT = dict(FUSED, update=2.56, invert=2.33)


def test_fused_inversion_is_told_from_the_slot_times():
    assert bench.inversion_fused(FUSED, C3)
    assert not bench.inversion_fused(SPLIT, C3)
    assert not bench.inversion_fused(FUSED, {"n1": 64, "n2": 64, "n3": 16})   # no bulk-copy update


def test_update_bytes_with_and_without_the_inversion():
    zones = 384 * 192 * 192
    cols = 384 * 192
    for width, per_zone in ((4.0, 352), (8.0, 460)):
        assert bench.kernel_bytes("update_invert", C3, width) == per_zone * zones + 488 * cols
    # fusing drops the seven W words written and read back and the guess's
    # reload (23 words per zone), and the inversion's own metric columns
    for width in (4.0, 8.0):
        split = bench.kernel_bytes("update", C3, width) + bench.kernel_bytes("invert", C3, width)
        fused = bench.kernel_bytes("update_invert", C3, width)
        assert split - fused == 23 * 8 * zones + 23 * 8 * cols


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_roofline_rows(prec):
    r = bench.kernel_rooflines(FUSED, C3, prec, 6500.0)
    assert "invert" not in r and "emf_centre" not in r   # timed inside update and flux3
    zones = 384 * 192 * 192
    for slot, row in r.items():
        assert row["achieved_gbs"] == pytest.approx(2 * row["algorithmic_bytes"] / (row["ms_per_step"] * 1e-3) / 1e9)
        assert 0 < row["frac"] < 1.5
        assert row["bound"] in ("fp64", "issue", "latency")
        assert row["traffic"] > 0.5 * row["algorithmic_bytes"]
    key = "update_invert"
    assert r["update"]["traffic"] == bench.NCU_DRAM_BYTES_PER_ZONE[prec][key] * zones
    assert r["update"]["limiter"] == bench.KERNEL_LIMITER[key]
    rs = bench.kernel_rooflines(SPLIT, C3, prec, 6500.0)
    assert "invert" in rs and rs["update"]["traffic"] == bench.NCU_DRAM_BYTES_PER_ZONE[prec]["update"] * zones


def test_launches_per_step_of_the_torus():
    pb = problems.fm_torus(24, 16, 40, rout=40.0)   # 3-D, transmissive poles
    # per sub-step: 3 flux directions, edge EMFs, polar EMF average, face
    # update, conserved update, inversion (1 or 2 passes), 3 ghost fills
    assert bench.launches_per_step(pb, True) == 2 * 11 + 1
    assert bench.launches_per_step(pb, False) == 2 * 12 + 1
