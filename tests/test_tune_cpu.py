"""CPU tests of the launch autotuner's host logic (ncs_b200/tune.py): it keeps
the fastest candidate, leaves the solver set to it, caches the choice per
workload key in memory and in a JSON file, and keys batches by tile and
stack counts rounded up to powers of two.  The timer is replaced by a fake,
so no GPU is needed."""
import json


class FakeSolver:
    def __init__(self):
        self.params = {}
        self.sets = []

    def set_params(self, **kw):
        self.params.update(kw)
        self.sets.append(dict(kw))


def test_autotune_picks_caches_and_persists(monkeypatch, tmp_path):
    from ncs_b200 import tune
    monkeypatch.setattr(tune, "_cache", {})
    cost = {(2, 1): 5.0, (4, 1): 3.0, (4, 2): 4.0}
    s = FakeSolver()
    monkeypatch.setattr(tune, "_time_ms", lambda fn, w, r: cost[(s.params["ctas_per_sm"],
                                                                 s.params["m"])])
    cands = [{"ctas_per_sm": 2, "m": 1}, {"ctas_per_sm": 4, "m": 1}, {"ctas_per_sm": 4, "m": 2}]
    path = str(tmp_path / "tune.json")
    best, ms = tune.autotune(s, lambda: None, "k1", candidates=cands, path=path)
    assert best == {"ctas_per_sm": 4, "m": 1} and s.params == best
    assert sorted(t for t, _ in ms) == [3.0, 4.0, 5.0]
    assert json.load(open(path))["k1"]["best"] == best
    # cached in memory: no timing, the solver is set to the choice
    monkeypatch.setattr(tune, "_time_ms", lambda *a: (_ for _ in ()).throw(AssertionError))
    s2 = FakeSolver()
    assert tune.autotune(s2, lambda: None, "k1", candidates=cands)[0] == best
    assert s2.params == best
    # a new process (empty memory cache) reads the file
    monkeypatch.setattr(tune, "_cache", {})
    s3 = FakeSolver()
    assert tune.autotune(s3, lambda: None, "k1", candidates=cands, path=path)[0] == best


def test_batch_key_rounds_up():
    from ncs_b200 import tune

    class S:
        batch_tiles = 1000
        _batch = [1, 2, 3]
    assert tune.batch_key(S()) == "batch/t1024/s4"
    S.batch_tiles, S._batch = 1024, [1] * 4
    assert tune.batch_key(S()) == "batch/t1024/s4"
