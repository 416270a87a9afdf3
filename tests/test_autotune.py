"""Host logic of the autotuner (no GPU): the staged search, the 1 % rule
that keeps the default kernels unless a variant clearly beats them, the
table it writes and the lookup SweepPlan uses, and candidates whose batch
does not fit in memory (efie:nomem) counted as no candidate."""
import importlib
import json

import pytest

from conftest import pkg

PKG = "matlab-cuda-efief-vs-cpu_b200"


@pytest.fixture
def tuner(tmp_path, monkeypatch):
    pkg()
    at = importlib.import_module(PKG + ".autotune")
    monkeypatch.setattr(at, "TABLE", str(tmp_path / "tuned.json"))
    monkeypatch.setattr(at, "_sms", lambda: 148)
    return at


def _fake_time(rates, calls):
    def t(plan_args, freqs, repeats, **kw):
        key = (kw["batch"], kw["lu_nb"], kw.get("tile_chain", 256), kw.get("tile_bulk", 256),
               kw.get("resident_chain", 0), kw.get("resident_bulk", 0), kw.get("share_factors", 0))
        calls.append(key)
        return 6968, rates(key)
    return t


def test_staged_search_and_table(tuner, monkeypatch):
    calls = []
    # (batch 0, panel 512) wins the first stage; the 128/256 tiles beat it by
    # 2 %, then sharing one factorization among 6 batches by 5 %
    def rates(k):
        base = {0: 200.0, 16: 180.0, 32: 190.0}[k[0]] * {128: 0.8, 256: 0.9, 512: 1.0}[k[1]]
        base *= 1.02 if k[2:4] == (128, 256) and k[4:6] == (0, 0) else 1.0
        return base * {0: 1.0, 2: 0.95, 4: 1.03, 6: 1.05, 8: 1.04}[k[6]]
    monkeypatch.setattr(tuner, "_time", _fake_time(rates, calls))
    best, res = tuner.tune([None] * 20, [2e9, 3e9], repeats=1)
    assert best == (0, 512, 128, 256, 0, 0, 6)
    # every (batch, panel) pair, then the tile variants at the winner, then
    # the shares at the winning tiles
    n1 = len(tuner.BATCHES) * len(tuner.PANELS)
    assert len(calls) == n1 + len(tuner.TILES) - 1 + len(tuner.SHARES) - 1
    assert all(c[:2] == (0, 512) for c in calls[n1:])
    assert all(c[:6] == (0, 512, 128, 256, 0, 0) for c in calls[n1 + len(tuner.TILES) - 1:])
    with open(tuner.TABLE) as f:
        table = json.load(f)
    e = table["ne8192_sm148"]
    assert (e["batch"], e["lu_nb"], e["tile_chain"], e["tile_bulk"], e["share_factors"]) == (0, 512, 128, 256, 6)
    assert tuner.tuned_opts(6968, sms=148) == (0, 512, 128, 256, 0, 0, 6)
    assert tuner.tuned_opts(6968, sms=132) is None        # another GPU: untuned


def test_one_percent_rule_keeps_default_kernels(tuner, monkeypatch):
    calls = []
    def rates(k):
        return 100.0 * (1.005 if k[2:6] == (128, 128, 0, 0) or k[6] == 4 else 1.0)   # within the noise
    monkeypatch.setattr(tuner, "_time", _fake_time(rates, calls))
    best, _ = tuner.tune([None] * 20, [2e9], repeats=1, save=False)
    assert best[2:] == (256, 256, 0, 0, 0)


def test_candidates_that_do_not_fit_are_skipped(tuner, monkeypatch):
    nat = importlib.import_module(PKG + "._native")
    api = importlib.import_module(PKG + ".api")

    class OOMPlan:
        def __init__(self, *a, **k):
            raise nat.MexError("efie:nomem", "cudaMalloc failed: out of memory")

    monkeypatch.setattr(api, "SweepPlan", OOMPlan)
    monkeypatch.setattr(api, "sweep_opts", lambda **kw: kw)
    plan_args = [None, None, list(range(1234))] + [None] * 17
    assert tuner._time(plan_args, [2e9], 1, batch=64, lu_nb=512) == (1234, None)

    class BadPlan:
        def __init__(self, *a, **k):
            raise nat.MexError("mex:E", "E must be [Ne x 2] int32.")

    monkeypatch.setattr(api, "SweepPlan", BadPlan)
    with pytest.raises(nat.MexError):
        tuner._time(plan_args, [2e9], 1, batch=0, lu_nb=512)
