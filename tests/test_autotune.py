"""The launch autotuner: keys, the on-disk cache round trip (CPU, with a
stand-in for the GPU timing) and, on the GPU, that a tuned launch gives the
default launch's PerturbationTable bit for bit."""
import json

import numpy as np
import pytest

from abcmb_b200 import autotune


def test_key_buckets_queue_length_and_separates_kinds():
    k1 = autotune.make_key("fd", "B200", 100, True, 330000)
    assert k1 == autotune.make_key("fd", "B200", 100, True, 300000)      # same power-of-two bucket
    assert k1 != autotune.make_key("fd", "B200", 100, True, 600000)
    assert k1 != autotune.make_key("tangent", "B200", 100, True, 330000, 4)
    assert k1 != autotune.make_key("fd", "B200", 46, False, 330000)


def test_cache_round_trip(tmp_path):
    """The fastest candidate is measured once, written to the cache and read
    back by a new tuner without measuring again; the knobs end at the choice
    and go back to the defaults."""
    path = str(tmp_path / "tune.json")
    calls = []

    def fake(kind, choice):
        calls.append((kind, choice))
        w, v = choice
        return 10.0 + abs(w - 2) + (0.5 if v == 1 else 0.0)          # (2, 2) is fastest

    t = autotune.Autotuner(path, measure=fake)
    key = autotune.make_key("fd", "fake", 100, True, 1000)
    assert t.tune("fd", key) == (2, 2)
    assert len(calls) == len(autotune.FD_CANDIDATES)
    saved = json.load(open(path))
    assert saved[key]["choice"] == [2, 2] and len(saved[key]["ms"]) == len(autotune.FD_CANDIDATES)
    t2 = autotune.Autotuner(path, measure=lambda *a: pytest.fail("measured again"))
    assert t2.tune("fd", key) == (2, 2)
    tk = autotune.make_key("tangent", "fake", 100, True, 1000, 4)
    t3 = autotune.Autotuner(path, measure=lambda kind, c: {0: 5.0, 1: 9.0, 2: 4.0, 3: 6.0, 4: 7.0}[c])
    assert t3.tune("tangent", tk) == 2
    assert autotune.Autotuner(path).lookup(tk) == 2 and autotune.Autotuner(path).lookup(key) == (2, 2)
    autotune.apply("fd", autotune.DEFAULT["fd"])
    autotune.apply("tangent", autotune.DEFAULT["tangent"])


@pytest.mark.gpu
def test_tuned_launch_reproduces_default_bit_for_bit(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from abcmb_b200 import configs, engine, gradients
    w = configs.c4(n_cosmo=3, nk_range=(20, 30), seed=5)
    for mode in ("fd", "tangent", "ind"):
        gw = gradients.expand(w, processes=1, mode=mode)
        st = w.pert_settings()
        autotune.apply("fd", autotune.DEFAULT["fd"])
        autotune.apply("tangent", autotune.DEFAULT["tangent"])
        db = engine.DeviceBatch.upload(gw.batch)
        db.pt.zero_()
        db.pert_forward_grad(gw, st)
        db.check_status()
        ref = db.pt.cpu().numpy()
        tuner = autotune.Autotuner(str(tmp_path / "tune.json"))
        kind, key, choice = autotune.tune_batch(db, gw, st, tuner, sample_items=50)
        assert kind == mode and tuner.lookup(key) == choice
        db.pt.zero_()
        db.pert_forward_grad(gw, st)
        db.check_status()
        np.testing.assert_array_equal(db.pt.cpu().numpy(), ref)
    autotune.apply("fd", autotune.DEFAULT["fd"])
    autotune.apply("tangent", autotune.DEFAULT["tangent"])
