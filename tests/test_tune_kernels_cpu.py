"""The kernel autotuner's choice rule and header on CPU (synthetic measurements; measuring needs a B200): one
knob varied at a time, only builds whose outputs hash like the default build's count, a value replaces the
default only when its stage gets MIN_GAIN faster, and the default choice writes the committed header."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "desert-search_b200")
sys.path.insert(0, PKG)
import tune_kernels as tk  # noqa: E402


def rows(changes=(), bad=()):
    """Measured rows in the tuner's candidate order; changes = {name: {stage: seconds}}, bad = names with other hashes."""
    base = {"tables": 1.0, "flood": 2.0, "proxy": 0.5}
    out = []
    for name, defs in tk.candidates():
        sec = dict(base)
        sec.update(dict(changes).get(name, {}))
        out.append({"name": name, "defines": defs, "seconds": sec, "hashes": {"x": "bad" if name in bad else "ok"}})
    return out


def test_default_kept_within_noise():
    assert tk.choose(rows({"DSG_EVAL_RUN=8": {"flood": 1.99}})) == {k: v[0][0] for k, v in tk.KNOBS.items()}


def test_faster_values_chosen_per_knob():
    c = tk.choose(rows({"DSG_EVAL_RUN=8": {"flood": 1.8}, "DSG_EVAL_RUN=32": {"flood": 1.7}, "DSG_TAB_WAVES=8": {"tables": 0.9},
                        "DSG_PROXY_MINB=1": {"proxy": 0.45}}))
    assert c["DSG_EVAL_RUN"] == 32 and c["DSG_TAB_WAVES"] == 8 and c["DSG_ZONE_CHUNK"] == 2048 and c["DSG_EVAL_BLOCKS"] == 0
    assert c["DSG_PROXY_MINB"] == 1                       # the proxy stage's two knobs are chosen independently


def test_builds_with_other_outputs_never_chosen():
    r = rows({"DSG_ZONE_CHUNK=4096": {"proxy": 0.1}}, bad={"DSG_ZONE_CHUNK=4096"})
    r.append({"name": "DSG_ZONE_CHUNK=8192", "defines": {}, "failed": "launch error"})
    assert tk.choose(r)["DSG_ZONE_CHUNK"] == 2048


def test_default_choice_writes_the_committed_header():
    with open(os.path.join(PKG, "csrc", "kernels_tuned.h")) as f:
        assert tk.header_text(tk.choose(rows())) == f.read()
