"""Autotuner logic on a fake engine (no GPU): picks the fastest shape and
caches it by signature."""
import time

from osprey_dpd_b200 import autotune


class FakeEngine:
    costs = {(32, 0, -1): 0.002, (40, 0, -1): 0.001, (24, 0, -1): 0.003}

    def __init__(self):
        self.shape = None
        self.created = True

    def set_launch_shape(self, *shape):
        self.shape = tuple(shape)

    def step(self, t, n):
        time.sleep(self.costs[self.shape] * n / 10)

    def status(self):
        return 0

    def close(self):
        pass


def test_tune_picks_fastest_and_caches(tmp_path):
    cache = str(tmp_path / "shapes.json")
    made = []

    def make():
        e = FakeEngine()
        made.append(e)
        return e

    sig = autotune.signature("B200", 1000, 100, 2, 0, 1)
    res = autotune.tune(make, sig, candidates=list(FakeEngine.costs), steps=5, reps=2, cache_path=cache)
    assert res["shape"] == [40, 0, -1]
    assert len(made) == 3
    again = autotune.tune(make, sig, candidates=list(FakeEngine.costs), steps=5, reps=2, cache_path=cache)
    assert again == res and len(made) == 3          # served from the cache


class FakeSchemeEngine(FakeEngine):
    costs = {(32, 0, -1, 0): 0.003, (32, 0, -1, 1): 0.001, (24, 0, -1): 0.002}

    def set_launch_shape(self, *shape):
        self.shape = tuple(shape) + (0,)

    def set_pair_scheme(self, scheme):
        self.shape = self.shape[:3] + (scheme,)

    def step(self, t, n):
        key = self.shape if self.shape in self.costs else self.shape[:3]
        time.sleep(self.costs[key] * n / 10)


def test_tune_can_select_the_half_shell_scheme(tmp_path):
    cache = str(tmp_path / "shapes.json")
    sig = autotune.signature("B200", 1000, 100, 2, 0, 1, reproducible=False)
    assert sig.endswith("|half") and sig != autotune.signature("B200", 1000, 100, 2, 0, 1)
    res = autotune.tune(FakeSchemeEngine, sig, candidates=[(32, 0, -1, 0), (32, 0, -1, 1), (24, 0, -1)],
                        steps=5, reps=2, cache_path=cache)
    assert res["shape"] == [32, 0, -1, 1]
    e = FakeSchemeEngine()
    autotune.apply_shape(e, res["shape"])
    assert e.shape == (32, 0, -1, 1)
    assert all(len(c) == 5 and c[3] == 1 and c[4] in (64, 128) for c in autotune.HALF_SHELL_CANDIDATES)
    assert {c[4] for c in autotune.HALF_SHELL_CANDIDATES} == {64, 128}


class FakeTileEngine(FakeEngine):
    """Half-shell shapes whose cost depends on the tile (beads per block)."""
    costs = {(32, 0, -1, 1, 64): 0.001, (32, 0, -1, 1, 128): 0.002}

    def set_launch_shape(self, *shape):
        self.shape = tuple(shape)

    def set_pair_scheme(self, scheme):
        self.shape = self.shape[:3] + (scheme,)

    def set_pair_tile(self, tile):
        self.shape = self.shape[:4] + (tile,)

    def step(self, t, n):
        time.sleep(self.costs[self.shape] * n / 10)


def test_tune_selects_the_tile(tmp_path):
    cache = str(tmp_path / "shapes.json")
    sig = autotune.signature("B200", 1000, 100, 2, 0, 1, reproducible=False)
    res = autotune.tune(FakeTileEngine, sig, candidates=list(FakeTileEngine.costs), steps=5, reps=2,
                        cache_path=cache)
    assert res["shape"] == [32, 0, -1, 1, 64]
    e = FakeTileEngine()
    autotune.apply_shape(e, (32, 0, -1, 1, 128))
    assert e.shape == (32, 0, -1, 1, 128)
