"""Host logic of the launch-shape autotuner (no GPU): keys, the choice
among timed candidates, the cache and its JSON file."""

import json

import pytest

from sap_warp_b200.autotune import SolveAutotuner, contact_bucket, tuning_key


def test_keys_bucket_contacts_and_name_the_gpu():
    assert [contact_bucket(c) for c in (0, 8, 9, 32, 33, 64)] == [8, 8, 16, 32, 64, 64]
    k = tuning_key(35, 32, "fp32", "armijo_decay", "NVIDIA B200", 148)
    assert k == "n35-c32-fp32-armijo_decay-NVIDIA_B200-148sm"
    assert tuning_key(35, 30, "fp32", "armijo_decay", "NVIDIA B200", 148) == k  # same bucket


def test_tune_picks_the_fastest_and_caches(tmp_path):
    path = tmp_path / "tune.json"
    tuner = SolveAutotuner(path, repeats=2)
    times = {1: 3.0, 2: 1.5, 3: 1.2, 4: 1.3}  # 3 beats the bound 4 by more than the 3 % margin
    calls = []

    def time_ms(k):
        calls.append(k)
        return times[k]

    assert tuner.tune("shape", [1, 2, 3, 4], time_ms) == 3
    assert sorted(calls) == [1, 1, 2, 2, 3, 3, 4, 4]  # each candidate timed `repeats` times
    assert tuner.tune("shape", [1, 2, 3, 4], time_ms) == 3  # cached: not timed again
    assert len(calls) == 8
    data = json.loads(path.read_text())
    assert data["shape"]["ctas_per_sm"] == 3 and set(data["shape"]["ms"]) == {"1", "2", "3", "4"}
    assert SolveAutotuner(path).lookup("shape") == 3  # reloaded from the file


def test_ties_take_more_ctas_and_bad_candidates_fail():
    tuner = SolveAutotuner()
    assert tuner.tune("s", [1, 2, 3], lambda k: 1.0) == 3
    with pytest.raises(ValueError):
        tuner.tune("t", [0, -1], lambda k: 1.0)


def test_the_occupancy_bound_stays_within_the_margin():
    tuner = SolveAutotuner(margin=0.05)
    assert tuner.tune("s", [1, 2, 3, 4], {1: 2.0, 2: 1.0, 3: 0.99, 4: 1.03}.get) == 4
    assert tuner.tune("t", [1, 2, 3, 4], {1: 2.0, 2: 1.0, 3: 0.90, 4: 1.03}.get) == 3
