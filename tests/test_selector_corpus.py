"""Host side of the learned selector: the corpus is a pure function of its
seed and covers the four graph families with the stated parameter ranges,
the regret measure is the time-weighted loss against the per-level best, and
the committed model has the layout the C ABI expects."""
import json
import os

import numpy as np

import gswitch_b200 as gs
from gswitch_b200.selector_train import corpus, load_model, regret

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_corpus_is_seeded_and_in_range():
    a, b = corpus(400, 7), corpus(400, 7)
    assert a == b
    assert corpus(400, 8) != a
    kinds = {s["kind"] for s in a}
    assert kinds == {"rmat", "er", "grid", "powerlaw"}
    for s in a:
        if s["kind"] == "rmat":
            assert 14 <= s["scale"] <= 20 and 0.45 <= s["a"] <= 0.65
            assert abs(s["a"] + s["b"] + s["c"] + 0.05 - 1) < 1e-12
        elif s["kind"] == "er":
            assert 2**14 <= s["n"] <= 2**20 and 4 <= 2 * s["m_pairs"] / s["n"] <= 32
        elif s["kind"] == "grid":
            assert 64 <= s["side"] <= 1024
        else:
            assert 1.8 <= s["gamma"] <= 3.0


def test_regret_is_time_weighted_against_the_best():
    T = np.zeros((3, gs.MLP_CLASSES), dtype=np.float32)
    T[0, :3] = [1, 2, 4]
    T[1, :3] = [3, 1, 0]   # class 2 untimed
    T[2, :3] = [2, 2, 2]
    r = regret(T, np.array([1, 0, 2]))
    assert r["rows"] == 3
    assert abs(r["chosen_ms"] - 7) < 1e-9 and abs(r["best_ms"] - 4) < 1e-9
    assert abs(r["time_weighted"] - 0.75) < 1e-9
    assert regret(T, np.array([2, 2, 2]))["rows"] == 2  # an untimed choice is not counted


def test_committed_model_layout():
    model, conf = load_model()
    assert model is not None
    assert model.shape == (gs.MLP_MODEL_FLOATS,) and np.all(np.isfinite(model))
    assert np.all(model[gs.MLP_NPARAM + gs.MLP_FEATURES:] > 0)  # inverse deviations
    d = json.load(open(os.path.join(ROOT, "gswitch_b200", "models", "selector_mlp.json")))
    rep = d["report"]
    assert rep["test_graphs"] >= 100 and rep["train_graphs"] >= 1000
    assert rep["regret_mlp"]["time_weighted"] <= 0.10


def test_class_names_cover_the_standalone_variants():
    names = {gs.mlp_class_name(k) for k in range(gs.MLP_CLASSES)}
    assert len(names) == 20
    assert "Push-Queue-TM" in names and "Pull-Bitmap-TWC" in names


def test_committed_fusion_model_layout():
    from gswitch_b200.selector_train import load_fusion_model

    model, _ = load_fusion_model()
    assert model is not None
    assert model.shape == (gs.MLP_MODEL_FLOATS,) and np.all(np.isfinite(model))
    d = json.load(open(os.path.join(ROOT, "gswitch_b200", "models", "fusion_mlp.json")))
    t = d["report"]["sssp_ms_test"]
    assert d["report"]["test_graphs"] >= 50
    assert t["mlp"] < t["tree"] and t["mlp"] <= 1.05 * t["best"]
