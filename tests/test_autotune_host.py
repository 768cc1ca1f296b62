"""Host logic of the autotuner (no GPU): candidate sets and the result
cache (file location, keys, round trip)."""
import json

import torch

from janus_b200 import autotune


class _FakeGreen:
    ishape = (32, 32, 32, 6)
    dtype = torch.float64


def test_candidates_respect_the_coefficient_size():
    for dim, s in ((2, 3), (3, 6)):
        plain, green = autotune.candidates(dim, torch.float64)
        sized = [c for c in green if c[2] != 3]
        assert all(w % s == 0 and nb in (2, 3) and ct in (0, 1, 2) for w, nb, ct in sized)
        assert {w for w, _, ct in sized if ct != 2} == {s, 2 * s, 3 * s}
        # the in-place variants: 24 columns (n = 128) and 12 (n = 256)
        assert sorted(c for c in green if c[2] == 2) == [(12, 2, 2), (24, 2, 2)]
        # the register-tile pass has a fixed tile (width and tiles 0)
        assert [c for c in green if c[2] == 3] == [(0, 0, 3)]
        if dim == 2:
            assert plain == []   # 2D has no plain column pass
        else:
            assert all(nb in (2, 3) for _, nb, _ in plain) and (8, 2, 1) in plain


def test_cache_path_follows_the_environment(tmp_path, monkeypatch):
    monkeypatch.setenv("JB_TUNE_CACHE", str(tmp_path / "t.json"))
    assert autotune._cache_path() == str(tmp_path / "t.json")


def test_cache_key_names_grid_precision_operator_and_loads():
    k = autotune._key(_FakeGreen(), 6)
    assert "32x32x32" in k and "f64" in k and "_FakeGreen" in k and k.endswith("|6")


def test_cached_tuning_is_applied_without_timing(tmp_path, monkeypatch):
    path = tmp_path / "t.json"
    monkeypatch.setenv("JB_TUNE_CACHE", str(path))
    g = _FakeGreen()
    key = autotune._key(g, 2)
    path.write_text(json.dumps({key: {"tuning": [8, 2, 1, 12, 3, 1, 2], "plain_ms": 1.0,
                                      "green_ms": 2.0}}))
    applied = []
    monkeypatch.setattr(autotune, "set_tuning", lambda op, v: applied.append(list(v)))
    r = autotune.tune(g, None, nload=2)
    assert r["cached"] and r["tuning"] == [8, 2, 1, 12, 3, 1, 2]
    assert applied == [[8, 2, 1, 12, 3, 1, 2]]
