"""The gate autotuner's choice rule and header on CPU (synthetic measurements; the measuring itself needs a
B200): only candidates bit-identical to the default build count, a shape replaces the default only when it is
at least MIN_GAIN faster, and the default choice writes the committed csrc/gate_tuned.h byte for byte."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "desert-search_b200")
sys.path.insert(0, PKG)
import tune_gate as tg  # noqa: E402


def row(pg, fg, pre_ms, full_ms, same=True):
    return {"pregate_blocks_per_sm": pg, "fullgate_blocks_per_sm": fg[0], "fullgate_rows": fg[1],
            "pregate_ms": pre_ms, "fullgate_ms": full_ms, "bit_identical": same}


def rows(pre_alt, full_alt, same=True):
    """The tuner's candidate order: the default, then the pre-gate shapes, then the full-gate shapes."""
    d = row(tg.PREGATE[0], tg.FULLGATE[0], 100.0, 50.0)
    out = [d] + [row(pg, tg.FULLGATE[0], 101.0, 50.0) for pg in tg.PREGATE[1:]]
    out += [row(tg.PREGATE[0], fg, 100.0, 51.0) for fg in tg.FULLGATE[1:]]
    out[1]["pregate_ms"] = pre_alt
    out[len(tg.PREGATE)]["fullgate_ms"] = full_alt
    out[1]["bit_identical"] = out[len(tg.PREGATE)]["bit_identical"] = same
    return out


def chosen(r):
    pg, fg = tg.choose(r)
    return pg["pregate_blocks_per_sm"], (fg["fullgate_blocks_per_sm"], fg["fullgate_rows"])


def test_default_kept_within_noise():
    assert chosen(rows(99.5, 49.8)) == (tg.PREGATE[0], tg.FULLGATE[0])


def test_faster_shapes_chosen_independently():
    assert chosen(rows(97.0, 48.0)) == (tg.PREGATE[1], tg.FULLGATE[1])
    assert chosen(rows(97.0, 50.0)) == (tg.PREGATE[1], tg.FULLGATE[0])


def test_shapes_with_other_amplitudes_never_chosen():
    r = rows(50.0, 20.0, same=False)
    assert chosen(r) == (tg.PREGATE[0], tg.FULLGATE[0])
    r.append({"pregate_blocks_per_sm": 9, "fullgate_blocks_per_sm": 9, "fullgate_rows": 9, "failed": "ptxas error"})
    assert chosen(r) == (tg.PREGATE[0], tg.FULLGATE[0])


def test_default_choice_writes_the_committed_header():
    pg, fg = tg.choose(rows(100.0, 50.0))
    with open(os.path.join(PKG, "csrc", "gate_tuned.h")) as f:
        assert tg.header_text(pg, fg) == f.read()


def _combo_rows():
    r = rows(97.0, 48.0)
    for x in r:
        x["total_ms"] = x["pregate_ms"] + x["fullgate_ms"]
    return r


def test_combined_shape_measured_and_kept_when_identical_and_faster():
    r = _combo_rows()
    pg, fg = tg.choose(r)
    seen = []

    def measure_pair(p, f):
        seen.append((p, f))
        return row(p, f, 97.0, 48.0) | {"total_ms": 145.0}
    pg2, fg2, combo = tg.confirm_combined(r, pg, fg, measure_pair)
    assert seen == [(tg.PREGATE[1], tg.FULLGATE[1])]
    assert (pg2, fg2) == (pg, fg) and combo["total_ms"] == 145.0


def test_combined_shape_rejected_keeps_the_larger_single_gain():
    r = _combo_rows()
    pg, fg = tg.choose(r)
    for bad in (row(0, (0, 0), 97.0, 48.0, same=False) | {"total_ms": 100.0}, row(0, (0, 0), 99.0, 52.0) | {"total_ms": 151.0},
                {"failed": "ptxas error"}):
        pg2, fg2, _ = tg.confirm_combined(r, pg, fg, lambda p, f, b=bad: b)
        # the pre-gate change saves 3 ms, the full-gate change 2 ms: the pre-gate one alone is kept
        assert pg2["pregate_blocks_per_sm"] == tg.PREGATE[1]
        assert (fg2["fullgate_blocks_per_sm"], fg2["fullgate_rows"]) == tg.FULLGATE[0]


def test_no_combined_measurement_when_one_winner_is_the_default():
    r = rows(97.0, 50.0)
    pg, fg = tg.choose(r)
    _, _, combo = tg.confirm_combined(r, pg, fg, lambda p, f: (_ for _ in ()).throw(AssertionError("measured")))
    assert combo is None
