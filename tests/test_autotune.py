"""The traits autotuner's selection and cache logic (no GPU: the trial solves
are a fake timing function)."""
import json

from adaptivegriddiscretizations_b200.Eikonal.Autotune import Autotuner, bucket_key, candidates


def test_bucket_keys_round_up_to_powers_of_two():
    assert bucket_key("Riemann2", (512, 512), 128, "B200") == "Riemann2|512x512|128|B200"
    assert bucket_key("Riemann2", (300, 513), 100, "B200") == "Riemann2|512x1024|128|B200"
    assert bucket_key("Riemann3", (200, 200, 200), 1) == "Riemann3|256x256x256|1|"


def test_candidates_follow_the_compiled_tile_shapes():
    c2 = candidates("Riemann2")
    assert {tuple(c["shape_i"]) for c in c2} == {(8, 8), (16, 16)}
    assert {c["niter_i"] for c in c2} == {4, 6, 8, 12, 16}
    assert {tuple(c["shape_i"]) for c in candidates("Rander2")} == {(8, 8)}
    assert {tuple(c["shape_i"]) for c in candidates("Riemann3")} == {(4, 4, 4)}


def test_tune_picks_the_fastest_and_caches_it(tmp_path):
    path = tmp_path / "cache" / "autotune.json"
    calls = []

    def run(tr):  # fastest: 16x16 tiles with 12 iterations
        calls.append((tuple(tr["shape_i"]), tr["niter_i"]))
        return 1.0 + abs(tr["niter_i"] - 12) * 0.1 + (0.0 if tr["shape_i"] == (16, 16) else 0.05)

    key = bucket_key("Riemann2", (512, 512), 128, "dev")
    t = Autotuner(str(path))
    choice, trials = t.choose(key, run, candidates("Riemann2"), repeats=2)
    assert choice == {"shape_i": (16, 16), "niter_i": 12}
    assert len(calls) == 2 * len(candidates("Riemann2"))
    entry = json.loads(path.read_text())[key]
    assert entry["shape_i"] == [16, 16] and entry["niter_i"] == 12 and len(entry["trials"]) == len(trials)
    # a new tuner reads the cache: no trial solve
    calls.clear()
    choice2, trials2 = Autotuner(str(path)).choose(key, run, candidates("Riemann2"))
    assert choice2 == choice and trials2 is None and not calls
    # another bucket is tuned separately; a failing candidate (inf) is never chosen
    key3 = bucket_key("Riemann2", (64, 64), 1, "dev")
    choice3, _ = Autotuner(str(path)).choose(key3, lambda tr: float("inf") if tr["niter_i"] != 4 else 2.0,
                                              candidates("Riemann2"), repeats=1)
    assert choice3["niter_i"] == 4
    assert set(json.loads(path.read_text())) == {key, key3}


def test_unreadable_cache_is_ignored(tmp_path):
    path = tmp_path / "autotune.json"
    path.write_text("not json")
    assert Autotuner(str(path)).lookup("anything") is None
