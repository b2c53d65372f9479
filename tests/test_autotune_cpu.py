"""Host logic of the near-field tile-shape autotuner (no GPU): selection,
table validation, and the shape list against the C header."""
import json
import os
import re

from fmm2d_b200 import autotune as at

HDR = os.path.join(os.path.dirname(__file__), "..", "include", "fmm2d_b200.h")


def test_select_takes_the_fastest_shape_per_class():
    times = [[3.0, 2.0, 4.0], [1.0, 1.5, 1.2], [9.0, 9.0, 8.5]]
    assert at.select(times) == [1, 0, 2]


def test_shape_list_matches_the_header():
    h = open(HDR).read()
    assert int(re.search(r"#define B2FMM_P2P_SHAPES (\d+)", h).group(1)) == len(at.SHAPES)
    assert int(re.search(r"#define B2FMM_P2P_CLASSES (\d+)", h).group(1)) == at.NCLASSES
    assert len(at.CLASS_NDIV) == at.NCLASSES


def test_load_rejects_malformed_tables(tmp_path):
    p = tmp_path / "t.json"
    for bad in ({"shapes": [0, 1]}, {"shapes": [0, 1, 7]}, {"shapes": [0, -1, 0]}, {}):
        p.write_text(json.dumps(bad))
        assert at.load(str(p)) is None
    p.write_text(json.dumps({"shapes": [2, 0, 1]}))
    assert at.load(str(p))["shapes"] == [2, 0, 1]
    assert at.load(str(tmp_path / "missing.json")) is None


def test_committed_table_is_valid():
    t = at.load()
    if t is not None:
        assert len(t["shapes"]) == at.NCLASSES
        assert t["shape_list"] == at.SHAPES
