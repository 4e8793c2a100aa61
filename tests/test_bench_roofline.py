"""The bench line's roofline and per-category table from the event-timed categories: algorithmic
bytes and FLOPs per launch from the units and pairs, the DRAM traffic scaled from the ncu
captures' bytes per row, the fractions of the peaks, and the counter-derived limiter."""

import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _prof(**over):
    cats = ["lists", "density", "forces", "flow", "marks", "levels", "cooling", "eos", "gradients"]
    prof = {c: {"ms": 0.0, "launches": 0, "units": 0.0, "pairs": 0.0} for c in cats}
    for c, v in over.items():
        prof[c] = v
    return prof


def test_roofline_of_the_dominant_category():
    import bench

    pk = {"hbm_gbs": 6548.5, "bf16_tflops": 1590.0, "source": "measured"}
    # 4 list builds of 4,194,304 particles and 160 entries per row in 42 ms, a smaller density
    prof = _prof(lists={"ms": 42.0, "launches": 4, "units": 4 * 4194304.0, "pairs": 4 * 671088640.0},
                 density={"ms": 40.0, "launches": 10, "units": 10 * 2.7e6, "pairs": 10 * 3.5e8})
    rf, dom = bench.roofline(prof, "fp32", True, pk)
    assert dom == "lists" and rf["kernel"] == "lists" and rf["bound"] == "hbm"
    bytes_ = 4194304.0 * 40.0 + 671088640.0 * 4.0
    assert math.isclose(rf["bytes_per_launch"], bytes_)
    assert math.isclose(rf["achieved"], round(bytes_ / 10.5e-3 / 1e9, 2))
    assert math.isclose(rf["frac"], round(rf["achieved"] / pk["hbm_gbs"], 4), rel_tol=1e-3)
    assert math.isclose(rf["traffic"], bench.DRAM_BYTES_PER_ROW["lists"] * 4194304.0)
    assert rf["limiter"] == bench.LIMITER["lists"]
    assert "pipe" not in rf  # a list build has no FLOP model


def test_kernel_table_fractions_and_limiters():
    import bench

    pk = {"hbm_gbs": 6548.5, "bf16_tflops": 1590.0, "source": "measured"}
    prof = _prof(density={"ms": 35.6, "launches": 10, "units": 10 * 2.72e6, "pairs": 10 * 3.57e8},
                 forces={"ms": 42.6, "launches": 10, "units": 10 * 2.35e6, "pairs": 10 * 1.35e8})
    kt = bench.kernel_table(prof, "fp32", True, pk)
    assert set(kt) == {"density", "forces"}  # categories without launches are left out
    d = kt["density"]
    b = 2.72e6 * 88.0 + 3.57e8 * 4.0
    f = 3.57e8 * bench.FLOP_PER_DENSITY_EVAL
    assert math.isclose(d["gbs"], round(b / 3.56e-3 / 1e9, 1))
    assert math.isclose(d["tflops"], round(f / 3.56e-3 / 1e12, 3))
    assert math.isclose(d["pipe_frac"], round(d["tflops"] / bench.FP32_NOMINAL_TFLOPS, 4), rel_tol=1e-3)
    assert d["limiter"] == bench.LIMITER["density"]
    # disc viscosity adds its 20 FLOP per pair to the force pass
    fo = kt["forces"]
    assert math.isclose(fo["flop_per_launch"], round(1.35e8 * (bench.FLOP_PER_FORCE_PAIR + 20.0)))
