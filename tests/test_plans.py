"""Plan files: the launcher's version 1/2 JSON, read and written; plan reuse (CPU only)."""
import json
import os
import tempfile

import pytest

from asz_b200 import plans
from conftest import REFERENCE_DIR


def test_round_trip_and_launcher_layout():
    entries = {1e-3: (["cubic2_012", "cubic1_120", "cubic0_021"], "quintic"), 1e-2: (["cubic0_012"], "cubic")}
    with tempfile.TemporaryDirectory() as wd:
        path = os.path.join(wd, "p.json")
        plans.write(path, entries)
        doc = json.load(open(path))
        assert doc["version"] == 2 and [p["rel_eb"] for p in doc["plans"]] == [1e-2, 1e-3]
        assert doc["plans"][1]["layers"][1] == {"prediction_direction": 1, "traversal_order": [1, 2, 0]}
        back = {e: (p, f) for e, p, f in plans.load(path)}
        assert back == entries
        assert plans.for_rel_eb(plans.load(path), 0.001) == entries[1e-3]


def test_version_one_defaults_to_cubic():
    doc = {"version": 1, "plans": [{"rel_eb": 0.01, "layers": [{"prediction_direction": 0, "traversal_order": [0, 1, 2]}]}]}
    with tempfile.TemporaryDirectory() as wd:
        path = os.path.join(wd, "v1.json")
        json.dump(doc, open(path, "w"))
        assert plans.load(path) == [(0.01, ["cubic0_012"], "cubic")]


@pytest.mark.parametrize("doc", [
    {"version": 3, "plans": []},
    {"version": 2, "plans": [{"rel_eb": 0.01, "layers": []}]},
    {"version": 2, "plans": [{"rel_eb": 0.01, "layers": [{"prediction_direction": 3, "traversal_order": [0, 1, 2]}]}]},
    {"version": 2, "plans": [{"rel_eb": 0.01, "layers": [{"prediction_direction": 0, "traversal_order": [2, 1, 0]}]}]},
    {"version": 2, "plans": [{"rel_eb": 0.01, "layers": [{"prediction_direction": 0, "traversal_order": [0, 1, 2], "x": 1}]}]},
    {"version": 2, "plans": [{"rel_eb": 0.01, "predictor_family": "linear",
                              "layers": [{"prediction_direction": 0, "traversal_order": [0, 1, 2]}]}]},
])
def test_rejects_malformed(doc):
    with tempfile.TemporaryDirectory() as wd:
        path = os.path.join(wd, "bad.json")
        json.dump(doc, open(path, "w"))
        with pytest.raises(plans.PlanFormatError):
            plans.load(path)


def test_exactly_one_plan_per_error_bound():
    ps = [(1e-3, ["cubic0_012"], "cubic"), (1e-3 * (1 + 1e-13), ["cubic1_012"], "cubic")]
    with pytest.raises(plans.PlanFormatError):
        plans.for_rel_eb(ps, 1e-3)
    with pytest.raises(plans.PlanFormatError):
        plans.for_rel_eb(ps, 1e-4)


def test_record_plan_replaces_the_entry():
    class Rep:
        plan = b"cubic2_012,cubic2_021"
        quintic = 1
    with tempfile.TemporaryDirectory() as wd:
        path = os.path.join(wd, "r.json")
        plans.write(path, {1e-3: (["cubic0_012"], "cubic"), 1e-4: (["cubic1_012"], "cubic")})
        plans.record_plan(path, 1e-3, Rep())
        got = {e: (p, f) for e, p, f in plans.load(path)}
        assert got == {1e-3: (["cubic2_012", "cubic2_021"], "quintic"), 1e-4: (["cubic1_012"], "cubic")}


REF_PLANS = os.path.join(REFERENCE_DIR, "plans")


@pytest.mark.skipif(not os.path.isdir(REF_PLANS), reason="reference plan files not present")
def test_reads_the_reference_plan_files():
    """The launcher's own plan files load, and rewrite to documents that load back the same."""
    paths = []
    for root, _, files in os.walk(REF_PLANS):
        paths += [os.path.join(root, f) for f in files if f.endswith(".json")]
    assert paths
    for path in paths:
        ps = plans.load(path)
        with tempfile.TemporaryDirectory() as wd:
            out = os.path.join(wd, "copy.json")
            plans.write(out, {e: (p, f) for e, p, f in ps})
            assert sorted(plans.load(out)) == sorted(ps)
