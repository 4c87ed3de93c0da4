"""The batched form's autotuner (runtime.Batch.autotune): the queue-form
narrow-phase kernels' persistent grids (CTAs per SM) picked by measurement
and cached in JSON by device and scene-size bucket.  The CPU test drives the
search and the cache through a stand-in batch whose step times are a known
function of the grids; the GPU test runs it on real scenes and checks that
the grid changes the time only, never the results."""
import json

import numpy as np
import pytest

from nexdynipc_b200 import runtime, scenes


class FakeBatch(runtime.Batch):
    """Batch without a device: set_queue_ctas records the grids, timed_steps
    returns a cost with a known minimum (rows at 8 CTAs/SM, emit at 2)."""

    def __init__(self, scene_list):
        self.scenes = list(scene_list)
        self.h = None
        self.grid = {0: 4, 1: 4}
        self.calls = []

    def set_queue_ctas(self, kernel, ctas_per_sm):
        self.grid[kernel] = ctas_per_sm
        self.calls.append((kernel, ctas_per_sm))

    def step(self, n=1):
        pass

    def timed_steps(self, n):
        return n * (abs(np.log2(self.grid[0] / 8)) + abs(np.log2(self.grid[1] / 2)) + 1.0)


def test_autotune_search_and_cache(tmp_path, monkeypatch):
    monkeypatch.setattr(runtime, "device_info", lambda: (148, "NVIDIA B200"))
    scs = scenes.batched_scenes(n_scenes=8)
    path = str(tmp_path / "tune.json")
    b = FakeBatch(scs)
    out = b.autotune(cache_path=path, steps=2)
    assert not out["cached"] and out["choice"] == {"narrow_rows": 8, "narrow_emit": 2}
    assert b.grid == {0: 8, 1: 2}
    assert len(out["timings_ms"]) == 2 * len(runtime.AUTOTUNE_CTAS)
    with open(path) as f:
        cache = json.load(f)
    assert out["key"] in cache and out["key"].startswith("NVIDIA B200|sm148|scenes8_")
    # a second batch of the same bucket takes the cached choice without timing
    b2 = FakeBatch(scs)
    out2 = b2.autotune(cache_path=path)
    assert out2["cached"] and out2["choice"] == out["choice"] and b2.grid == {0: 8, 1: 2}
    assert sorted(b2.calls) == [(0, 8), (1, 2)]
    # another bucket is tuned afresh and added beside the first
    b3 = FakeBatch(scenes.batched_scenes(n_scenes=40))
    assert not b3.autotune(cache_path=path)["cached"]
    with open(path) as f:
        assert len(json.load(f)) == 2


@pytest.mark.gpu
def test_queue_grid_changes_time_not_results(tmp_path):
    scs = scenes.batched_scenes(n_scenes=24)
    ref = runtime.Batch(scs)
    ref.set_queue_ctas(runtime.QUEUE_KERNELS["narrow_rows"], 1)
    ref.set_queue_ctas(runtime.QUEUE_KERNELS["narrow_emit"], 1)
    ref.step(6)
    tuned = runtime.Batch(scs)
    out = tuned.autotune(cache_path=str(tmp_path / "tune.json"), steps=1)
    assert set(out["choice"]) == set(runtime.QUEUE_KERNELS)
    # the search stepped 2 kernels x 5 candidates x (1 untimed + 1 timed) =
    # 20 steps; the reference catches up
    ref.step(14)
    for i in range(len(scs)):
        a, b = ref.state(i), tuned.state(i)
        assert np.array_equal(a["position"], b["position"]) and np.array_equal(a["orientation"], b["orientation"])
        assert tuned.diagnostics(i)["status"] == 0
    ref.close()
    tuned.close()
