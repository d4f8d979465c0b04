"""The autotuner's JSON cache (rtk_b200.ops): keys that identify the kernel,
the device and the problem sizes independently of problem order, and
whole-file replacement on every write."""
import json

from rtk_b200 import ops
from rtk_b200.image import make_desc


def _probs(sizes):
    return [(None, make_desc(v), make_desc(p), None, None, None) for v, p in sizes]


def test_key_ignores_problem_order_and_separates_kernels_and_devices():
    a = _probs([((64, 64, 64), (128, 96, 90)), ((32, 40, 48), (64, 64, 30))])
    b = list(reversed(a))
    assert ops._tune_key(a, True, "B200") == ops._tune_key(b, True, "B200")
    assert ops._tune_key(a, True, "B200") != ops._tune_key(a, False, "B200")
    assert ops._tune_key(a, True, "B200") != ops._tune_key(a, True, "H100")
    assert ops._tune_key(a, True, "B200") != ops._tune_key(a[:1], True, "B200")


def test_cache_put_get_round_trip(tmp_path):
    path = str(tmp_path / "t.json")
    assert ops._cache_get(path, "k") is None
    ops._cache_put(path, "k", {"config": 2, "ms": 1.5, "ms_per_config": [2.0, 1.7, 1.5]})
    ops._cache_put(path, "k2", {"config": 0, "ms": 3.0, "ms_per_config": [3.0]})
    assert ops._cache_get(path, "k") == {"config": 2, "ms": 1.5, "ms_per_config": [2.0, 1.7, 1.5]}
    with open(path) as f:
        assert set(json.load(f)) == {"k", "k2"}
    assert not list(tmp_path.glob("*.tmp"))
    (tmp_path / "bad.json").write_text("{not json")
    assert ops._cache_get(str(tmp_path / "bad.json"), "k") is None
