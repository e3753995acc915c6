"""CPU checks of the autotuner's cache handling (no GPU needed)."""
import json

from strata_b200 import tune


def test_load_filters_unknown_knobs_and_values(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text(json.dumps({"GPU A": {"1": 19, "2": 13, "3": 5}, "GPU B": {"1": 12}}))
    assert tune.load(p, gpu="GPU A") == {1: 19, 2: 13}
    assert tune.load(p, gpu="GPU B") == {}
    assert tune.load(p, gpu="GPU C") == {}


def test_save_merges_per_gpu(tmp_path):
    p = tmp_path / "sub" / "tune.json"
    tune.save({"gpu": "GPU A", "best": {1: 23, 2: 7}}, p)
    tune.save({"gpu": "GPU B", "best": {1: 11, 2: 9}}, p)
    assert tune.load(p, gpu="GPU A") == {1: 23, 2: 7}
    assert tune.load(p, gpu="GPU B") == {1: 11, 2: 9}


def test_corrupt_cache_is_ignored(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    assert tune.load(p, gpu="GPU A") == {}


def test_load_keeps_every_swept_knob():
    """Every knob the sweep times (radix tiles and ranking, triangle probe,
    batch graph rounds and blocks, dense-word threshold) survives the cache
    round trip; values outside a knob's choices are dropped."""
    import tempfile
    from pathlib import Path
    best = {1: 15, 2: 9, 3: 3, 4: 4, 5: 2, 7: 3, 8: 24}
    with tempfile.TemporaryDirectory() as d:
        p = Path(d) / "tune.json"
        tune.save({"gpu": "GPU A", "best": best}, p)
        assert tune.load(p, gpu="GPU A") == best
        p.write_text(json.dumps({"GPU A": {"8": 34, "4": 3}}))
        assert tune.load(p, gpu="GPU A") == {}
