"""Host-side arithmetic of the bench line, without a GPU: the dominant kernel, its algorithmic
bytes (SoA u/f/d of 3 components, 1-byte activity and support flags, 4-byte element
weights), the achieved / peak fraction and the ncu traffic of the chosen variant."""
import bench


class _Level:
    nv, ne = 1081665, 128 * 128 * 64


class _Hier:
    def __getitem__(self, i):
        return _Level()


def test_roofline_of_the_dominant_kernel():
    stats = {"fine_cheby_f32": (100, 5.9), "st_cheby_f32_l1": (800, 4.0), "restrict_f32": (300, 5.0)}
    tuning = {"chebyshev_f32": {"variant": "smem_tile", "rows": 4, "zchunk": 8}}
    r = bench.roofline(None, stats, _Hier(), {"hbm_gbs": 6534.5}, tuning)
    nv, ne = _Level.nv, _Level.ne
    b = nv * (3 * 4 * 5 + 2) + ne * 4
    assert r["kernel"] == "fine_cheby_f32" and r["launches"] == 100
    assert r["algorithmic_bytes"] == b
    assert abs(r["avg_us"] - 59.0) < 1e-9
    assert abs(r["achieved"] - round(b / 59.0e-6 / 1e9, 1)) < 1e-9
    assert abs(r["frac"] - round(r["achieved"] / 6534.5, 4)) < 1e-4 and r["peak_source"] == "measured"
    assert r["traffic"] == int(bench.NCU_TRAFFIC_PER_NODE[("fine_cheby_f32", "smem_tile")] * nv)
    assert abs(r["share"] - 5.9 / 14.9) < 1e-12
    assert tuple(r["rows_zchunk"]) == (4, 8)


def test_roofline_without_a_byte_model_and_fallback_peak():
    r = bench.roofline(None, {"st_cheby_f32": (10, 1.0)}, _Hier(), {}, None)
    assert r["achieved"] is None and r["frac"] is None and r["bound"] == "hbm"
    r = bench.roofline(None, {"fine_applyK_f64": (10, 1.0)}, _Hier(), {}, None)
    assert r["peak_source"] == "fallback" and r["traffic"] is None
    assert r["algorithmic_bytes"] == _Level.nv * (3 * 8 * 2 + 2) + _Level.ne * 4
