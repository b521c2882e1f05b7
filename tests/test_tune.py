"""Host logic of the autotuner (CPU): coordinate descent keeps the fastest
candidate of each parameter, and the JSON cache round-trips."""
import pytest

from iitmglobalrouter_b200 import tune


class FakeRouter:
    device, Z = 0, 10

    def __init__(self):
        self.v = {p: c[0] for p, c in tune.CANDIDATES.items()}

    def tune_get(self, p):
        return self.v[p]

    def tune_set(self, p, v):
        self.v[p] = v


def test_autotune_picks_fastest_per_parameter(monkeypatch):
    want = {p: c[-1] for p, c in tune.CANDIDATES.items()}  # the fake time is lowest at the last candidate

    def fake_time(router, mst, pat, b0, b1, reps):
        return sum(abs(tune.CANDIDATES[p].index(router.v[p]) - (len(tune.CANDIDATES[p]) - 1)) for p in router.v)

    monkeypatch.setattr(tune, "time_range", fake_time)
    R = FakeRouter()
    best = tune.autotune(R, None, None)
    assert R.v == want
    assert best == {tune.NAMES[p]: v for p, v in want.items()}


def test_autotune_keeps_current_value_when_nothing_is_faster(monkeypatch):
    monkeypatch.setattr(tune, "time_range", lambda *a, **k: 1.0)
    R = FakeRouter()
    start = dict(R.v)
    tune.autotune(R, None, None)
    assert R.v == start


def test_cache_round_trip(tmp_path):
    path = tmp_path / "t.json"
    assert tune.load("gpu|Z=9", path) is None
    vals = {"mst_mid_threads": 256, "mst_cluster_min_pins": 0}
    tune.save(vals, "gpu|Z=9", path)
    tune.save({"mst_mid_threads": 512}, "gpu|Z=10", path)
    assert tune.load("gpu|Z=9", path) == vals
    R = FakeRouter()
    tune.apply(R, tune.load("gpu|Z=9", path))
    assert R.v[0] == 256 and R.v[3] == 0
    tune.apply(R, None)  # nothing cached: no change
    assert R.v[0] == 256


def test_committed_cache_names_known_parameters():
    data = tune.json.loads(tune.DEFAULT_PATH.read_text())
    for values in data.values():
        assert set(values) <= set(tune.NAMES.values())
        for name, v in values.items():
            assert isinstance(v, int)


@pytest.mark.parametrize("p", sorted(tune.CANDIDATES))
def test_candidates_are_valid_values(p):
    for v in tune.CANDIDATES[p]:
        if p == 3:
            assert v == 0 or 128 < v <= 4096
        elif p == 4:
            assert v in (0, 1, 2, 4)
        elif p == 5:
            assert v in (0, 1)
        else:
            assert 64 <= v <= 1024 and v % 32 == 0
