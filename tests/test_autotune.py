"""Autotuner bookkeeping on the CPU: buckets, the table file, and that every
candidate launch shape is a valid parameter block."""
import ctypes

from cuppa_b200 import autotune as at


def test_bucket_names():
    assert at.bucket(10 ** 8, 16, 64) == "n2^26_d16_i64"
    assert at.bucket(2 ** 30, 4, 64) == "n2^30_d4_i64"
    assert at.bucket(1, 1, 32) == "n2^1_d1_i32"


def test_candidates_are_valid(pa):
    for shape in at.candidates():
        prm = at.apply(pa.make_params(100_000, 4, 0.5), shape)
        assert pa.lib().pa_params_check(ctypes.byref(prm)) == pa.PA_OK, shape


def test_table_round_trip_and_apply(pa, tmp_path):
    path = str(tmp_path / "t.json")
    table = {at.bucket(50_000, 8, 32): {"shape": {"blocks": 100}, "ms": 1.0}}
    at.save(table, path)
    assert at.load(path) == table
    prm = at.tuned_params(50_000, 8, 0.3, table=at.load(path))
    assert prm.blocks == 100 and prm.n == 50_000 and prm.d == 8
    prm = at.tuned_params(10 ** 6, 8, 0.3, table=at.load(path))   # other bucket: defaults
    assert prm.blocks == 0
    assert at.load(str(tmp_path / "missing.json")) == {}
