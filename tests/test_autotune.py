"""The autotuner's table lookups (host logic, no GPU): the workspace count for the nearest tuned N
with the same tile size, rule and precision, capped at the batch; the fallback without a match; and
the per-tile-size report at the nearest tuned N."""
import json

from adaptive_tlr_pilots_b200 import autotune as A


def _entry(n, b, best, rates, loglik=None, rule="adaptive", value=0.9, precision="mixed"):
    return {"n": n, "b": b, "rule": rule, "value": value, "precision": precision, "best": best,
            "evals_per_s": {str(k): v for k, v in rates.items()}, "loglik_theta0": loglik,
            "stored_factor": 10 * n}


def _table(tmp_path):
    t = {
        "a": _entry(50000, 500, 8, {4: 5.5, 8: 5.7}, 3040.57),
        "b": _entry(50000, 1000, 8, {4: 2.3, 8: 2.6}, 3039.31),
        "c": _entry(20000, 500, 4, {2: 9.0, 4: 11.0}, 1123.45),
        "d": _entry(50000, 500, 2, {2: 4.0}, precision="fp64"),
    }
    p = tmp_path / "tuning.json"
    p.write_text(json.dumps(t))
    return str(p)


def test_best_workspaces(tmp_path):
    path = _table(tmp_path)
    assert A.best_workspaces(50000, 500, 64, path=path) == 8
    assert A.best_workspaces(50000, 500, 6, path=path) == 6            # capped at the batch
    assert A.best_workspaces(25000, 500, 64, path=path) == 4           # nearest N (log scale): 20,000
    assert A.best_workspaces(45000, 500, 64, path=path) == 8
    assert A.best_workspaces(50000, 500, 64, precision="fp64", path=path) == 2
    assert A.best_workspaces(50000, 250, 64, path=path) == A.DEFAULT_WORKSPACES   # no tuned b = 250
    assert A.best_workspaces(50000, 250, 2, path=path) == 2
    assert A.best_workspaces(50000, 500, 64, path=str(tmp_path / "missing.json")) == A.DEFAULT_WORKSPACES


def test_tile_sizes(tmp_path):
    path = _table(tmp_path)
    got = A.tile_sizes(60000, path=path)
    assert set(got) == {500, 1000}
    assert got[500] == (5.7, 3040.57, 500000) and got[1000][0] == 2.6
    assert set(A.tile_sizes(18000, path=path)) == {500}
    assert A.tile_sizes(50000, rule="fixed", path=path) == {}
