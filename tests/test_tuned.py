"""CPU: the autotuner's committed header is what it renders from its committed
JSON (libnt_b200/tune.py writes both; a hand edit of one would desynchronise
the library from its recorded timings)."""
from libnt_b200 import tune


def test_tuned_header_matches_json():
    assert tune.render_header(tune.load_tuned()) == tune.TUNED_H.read_text()


def test_tuned_values_in_range():
    t = tune.load_tuned()
    assert t["pass8_variant"] in (0, 1, 2, 3)
    assert t["batch_chunk"] >= 1 and t["tile_dense_div"] >= 1
    for e in t["sort"]:
        assert 0 <= e["variant"] and e["key_bits_max"] <= 64
