"""The layout/mode sweep driver on a subset (one layout, m = 1 and 64, float)."""
import pytest

pytestmark = pytest.mark.gpu


def test_sweep_subset(cuda):
    from ttm_b200.sweep import extent_sets, layouts, sweep
    assert layouts(3, 10, 0)[:2] == [[1, 2, 3], [3, 2, 1]] and len(layouts(3, 10, 0)) == 6
    assert len({tuple(x) for x in layouts(5, 10, 1)}) == 10
    res = sweep(dtypes=("f32",), ms=(1, 64), n_layouts=1, reps=1, log=lambda s: None)
    assert len(res["cases"]) == 2 * sum(len(n) for n in extent_sets())
    for c in res["cases"]:
        assert c["gbs"] > 0 and c["kernel"] in ("rowdot", "colvec", "stream_cols", "stream_rows", "simt_gemm", "bvec")
    assert set(res["summary"]) == {"f32_m1", "f32_m64"}
