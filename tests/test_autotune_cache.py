"""The autotuner's JSON cache (rhmc_tune_cache_load / _save / rhmc_tune_report) without a GPU:
entries written by one process are read back by the next, keyed by device name, volume and
kernel; entries already known win over the file; a missing file is an empty cache that is
created on save; malformed choices are ignored."""
import json

import rhmc_b200 as rb

ENTRY = "NVIDIA B200|vh=524288|dslash f32_12 nr=4 y=1 red=1"


def _write(path, entries):
    with open(path, "w") as f:
        json.dump({"version": 1, "entries": entries}, f)


def test_cache_round_trip(tmp_path):
    rb.tune_clear()
    src = tmp_path / "in.json"
    _write(src, [
        {"key": ENTRY, "choice": 1, "shapes": [[256, 2], [128, 4], [128, 3]], "us": [87.1, 86.2, 92.5]},
        {"key": "NVIDIA B200|vh=524288|pack f64_18 n=30 y=0", "choice": 2, "shapes": [[8, 0], [4, 0], [3, 0]],
         "us": [900.0, 880.5, 870.25]},
        {"key": "bad entry", "choice": 7, "shapes": [[256, 2]], "us": [1.0]},  # choice out of range: ignored
    ])
    rb.tune_cache_load(str(src))
    rep = {e["key"]: e for e in rb.tune_report()["entries"]}
    assert set(rep) == {ENTRY, "NVIDIA B200|vh=524288|pack f64_18 n=30 y=0"}
    assert rep[ENTRY]["choice"] == 1 and rep[ENTRY]["shapes"][1] == [128, 4]
    assert abs(rep[ENTRY]["us"][2] - 92.5) < 1e-9
    out = tmp_path / "out.json"
    rb.tune_cache_save(str(out))
    rb.tune_clear()
    assert rb.tune_report()["entries"] == []
    rb.tune_cache_load(str(out))
    assert {e["key"]: e for e in rb.tune_report()["entries"]} == rep
    # entries already in the table are kept when a file disagrees
    _write(src, [{"key": ENTRY, "choice": 2, "shapes": [[256, 2], [128, 4], [128, 3]], "us": [1, 2, 0.5]}])
    rb.tune_cache_load(str(src))
    assert {e["key"]: e for e in rb.tune_report()["entries"]}[ENTRY]["choice"] == 1
    rb.tune_clear()


def test_missing_cache_file_is_empty(tmp_path):
    rb.tune_clear()
    rb.tune_cache_load(str(tmp_path / "none.json"))
    assert rb.tune_report()["entries"] == []
    rb.tune_cache_save(None)  # writes the (empty) table to the cache file
    assert json.loads((tmp_path / "none.json").read_text()) == {"version": 1, "entries": []}


def test_switches():
    prev = rb.autotune(False)
    assert rb.autotune(prev) is False
    assert rb.autotune_override(2) == -1
    assert rb.autotune_override(-1) == 2
