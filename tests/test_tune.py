"""Autotuner (gwf_tune*): the per-bucket table, its JSON file, and that tuned AUTO runs give the
same distances as any fixed launch shape."""
import json

import numpy as np
import pytest


def test_table_json_round_trip_without_gpu(G, tmp_path):
    p = tmp_path / "tune.json"
    p.write_text(json.dumps({"version": 1, "device": 0, "name": "x", "sm_count": 148, "buckets": []})[:-2]
                 + '\n  {"bucket": 0, "ql_max": 1500, "form": "persistent", "ctas_per_sm": 2, "reads_per_s": 123.5},'
                 + '\n  {"bucket": 3, "ql_max": 12000, "form": "plain", "ctas_per_sm": 0, "reads_per_s": 7.0}\n]}\n')
    G.tune_clear(0)
    t = G.tune_load(str(p), device=0)
    assert t == {0: (G.MODE_PERSISTENT, 2, pytest.approx(123.5)), 3: (G.MODE_PLAIN, 0, pytest.approx(7.0))}
    assert G.tune_table(0, with_warps=True)[0][2] == 1  # tables without the field: one warp per read
    G.tune_clear(0)
    assert G.tune_table(0) == {}
    q = tmp_path / "warps.json"
    q.write_text('{"buckets": [\n  {"bucket": 4, "ql_max": -1, "form": "persistent", "ctas_per_sm": 3, '
                 '"reads_per_s": 55.0, "warps_per_read": 8}\n]}\n')
    G.tune_load(str(q), device=0)
    assert G.tune_table(0, with_warps=True) == {4: (G.MODE_PERSISTENT, 3, 8, pytest.approx(55.0))}
    q.write_text('{"buckets": [{"bucket": 4, "ql_max": -1, "form": "persistent", "ctas_per_sm": 3, '
                 '"reads_per_s": 55.0, "warps_per_read": 3}]}')
    with pytest.raises(G.GwfError):
        G.tune_load(str(q), device=0)
    G.tune_clear(0)
    bad = tmp_path / "bad.json"
    bad.write_text('{"buckets": [{"bucket": 9, "ql_max": 1, "form": "plain", "ctas_per_sm": 0, "reads_per_s": 1}]}')
    with pytest.raises(G.GwfError):
        G.tune_load(str(bad), device=0)
    with pytest.raises(G.GwfError):
        G.tune_load(str(tmp_path / "missing.json"), device=0)


@pytest.mark.gpu
def test_tuned_auto_equals_fixed_shapes(G, tmp_path):
    w = G.load_workload("config3", n=1500)
    g = w["graph"]
    g.index()
    reads = (w["cat"], w["offs"], w["lens"])
    G.tune_clear()
    path = str(tmp_path / "tune.json")
    table = G.tune(g, reads, w["v0"], max_reads_per_bucket=150, json_path=path)
    present = {min(b for b, hi in enumerate(G.TUNE_BUCKET_MAX) if hi is None or q < hi) for q in w["lens"]}
    assert set(table) == present
    for form, cps, rps in table.values():
        assert form in (G.MODE_PLAIN, G.MODE_PERSISTENT) and rps > 0
        assert cps >= 1 or form == G.MODE_PLAIN
    shapes = G.tune_table(with_warps=True)
    assert all(v[2] in (1, 2, 4, 8) for v in shapes.values())
    d_auto, s_auto = g.ed_batch(reads, w["v0"], mode=G.MODE_AUTO)
    d_pers, s_pers = g.ed_batch(reads, w["v0"], mode=G.MODE_PERSISTENT)
    assert np.array_equal(d_auto, d_pers) and np.array_equal(s_auto, s_pers)
    G.tune_clear()
    loaded = G.tune_load(path)
    assert {b: v[:2] for b, v in loaded.items()} == {b: v[:2] for b, v in table.items()}
    assert {b: v[:3] for b, v in G.tune_table(with_warps=True).items()} == {b: v[:3] for b, v in shapes.items()}
    for b, v in table.items():
        assert loaded[b][2] == pytest.approx(v[2], abs=0.06)  # the file keeps reads/s to 0.1
    G.tune_clear()
