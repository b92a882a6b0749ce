"""The batch autotuner's search and cache (host logic, no GPU): a stand-in
handle whose execute time depends on the tuning lets the test check that the
coordinate descent finds the fastest candidate, skips rejected candidates,
leaves the handle planned with the winner, and reuses the JSON cache."""
import json
import time

from spgemm_b200 import autotune


class FakeCM:
    def __init__(self, rows, cols, nnz):
        self.num_rows, self.num_cols, self.nnz = rows, cols, nnz


class FakeHandle:
    """Execute time = a cost table over two tuning fields; one value rejected."""

    def __init__(self):
        self.precision = 0
        self.t = {"warp_table_max": 256, "warp_p_max": 4096, "warp_cap_max": 2048,
                  "long_p": 4096, "mid_cols": 1 << 18, "long_o_num": 4096, "esc_p_min": 0}
        self.plans = []

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, **kw):
        if kw.get("warp_cap_max") == 512:
            raise RuntimeError("rejected")
        self.t.update(kw)

    def batch_plan(self, A, B):
        self.plans.append(dict(self.t))
        return 0

    def batch_execute(self, graph=True):
        cost = {256: 3.0, 512: 2.0, 1024: 1.0}[self.t["warp_table_max"]]
        cost += {1024: 0.5, 2048: 0.2, 4096: 0.4}[self.t["warp_p_max"]]
        time.sleep(cost * 1e-3)


def test_search_finds_fastest_and_caches(tmp_path):
    A = [FakeCM(10, 10, 30), FakeCM(20, 20, 50)]
    B = [FakeCM(10, 10, 30), FakeCM(20, 20, 50)]
    cache = tmp_path / "tune.json"
    h = FakeHandle()
    res = autotune.tune_batch(h, A, B, device_name="gpu0", reps=2, cache=cache)
    assert not res["cached"]
    assert res["tuning"]["warp_table_max"] == 1024
    assert res["tuning"]["warp_p_max"] == 2048
    assert h.plans[-1]["warp_table_max"] == 1024   # left planned with the winner
    stored = json.loads(cache.read_text())
    key = autotune.batch_key("gpu0", 0, [(10, 10, 30, 30), (20, 20, 50, 50)])
    assert stored[key]["tuning"] == res["tuning"]
    h2 = FakeHandle()
    res2 = autotune.tune_batch(h2, A, B, device_name="gpu0", reps=2, cache=cache)
    assert res2["cached"] and res2["tried"] == 0
    assert h2.t["warp_table_max"] == 1024 and len(h2.plans) == 1


def test_key_depends_on_device_precision_and_shape():
    s = [(1, 2, 3, 4)]
    assert autotune.batch_key("a", 0, s) != autotune.batch_key("b", 0, s)
    assert autotune.batch_key("a", 0, s) != autotune.batch_key("a", 1, s)
    assert autotune.batch_key("a", 0, s) != autotune.batch_key("a", 0, [(1, 2, 3, 5)])
