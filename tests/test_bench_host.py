"""The bench's own arithmetic (no GPU): the per-configuration row's fractions of the
D2D copy and of the HBM roofline, and the geomean over configurations, on values
computed by hand."""
import math

import bench


def test_mode_row_fractions():
    # N = 300 MB in, S = 100 MB out, compress at 2000 GB/s of N, decompress at 4000,
    # a 3000 GB/s copy, a 6000 GB/s roofline over N + S moved bytes
    r = bench._mode_row(300e6, 100e6, 2000.0, 4000.0, 3000.0, 6000.0)
    assert r["ratio"] == 3.0
    assert r["frac_of_memcpy"] == {"compress": round(2000 / 3000, 3), "decompress": round(4000 / 3000, 3)}
    assert r["roofline_frac"]["compress"] == round(2000 * 400 / 300 / 6000, 3)
    assert r["roofline_frac"]["decompress"] == round(4000 * 400 / 300 / 6000, 3)


def test_geomean():
    assert math.isclose(bench._geomean([1.0, 4.0, 16.0]), 4.0)
    assert math.isclose(bench._geomean([2.5]), 2.5)
    assert bench._geomean([]) is None
