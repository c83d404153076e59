"""Predictor-plan files: the launcher's JSON format (versions 1 and 2) and plan reuse.

A plan file holds one plan per relative error bound:

    {"version": 2, "plans": [{"rel_eb": 0.001, "predictor_family": "cubic",
                              "layers": [{"prediction_direction": 2, "traversal_order": [0, 1, 2]}, ...]}]}

Version 1 has no "predictor_family" (cubic). A layer's traversal order is one of [1,2,0], [0,2,1],
[0,1,2] and its direction 0..2; in plan-string form the layer is "cubic<direction>_<order>". The
reader validates like the launcher (t1_start_compressors.py:224-250) and the writer produces the
version-2 document it writes (:292-311), so files move between the two freely.

`compress_with_plan_file` compresses with the plan stored for an error bound; `record_plan` stores
the plan (and family) a compression used, e.g. one found by the plan search on the first time step
and reused for the next ones.
"""
from __future__ import annotations

import json
import math
import os
import re
from pathlib import Path

ORDERS = {(1, 2, 0): "120", (0, 2, 1): "021", (0, 1, 2): "012"}


class PlanFormatError(ValueError):
    pass


def load(path) -> list[tuple[float, list[str], str]]:
    """[(rel_eb, predictors, family)] from a version 1 or 2 plan file."""
    with open(path, encoding="utf-8") as f:
        doc = json.load(f)
    if not isinstance(doc, dict) or doc.get("version") not in (1, 2) or not isinstance(doc.get("plans"), list):
        raise PlanFormatError(f"invalid plan file: {path}")
    out = []
    for pid, plan in enumerate(doc["plans"]):
        if (not isinstance(plan, dict) or not isinstance(plan.get("rel_eb"), (int, float))
                or isinstance(plan.get("rel_eb"), bool) or not isinstance(plan.get("layers"), list) or not plan["layers"]):
            raise PlanFormatError(f"plan {pid} is malformed: {path}")
        preds = []
        for lid, layer in enumerate(plan["layers"]):
            if not isinstance(layer, dict) or set(layer) != {"prediction_direction", "traversal_order"}:
                raise PlanFormatError(f"plan {pid} layer {lid} is malformed: {path}")
            d, t = layer["prediction_direction"], layer["traversal_order"]
            if not isinstance(d, int) or isinstance(d, bool) or d not in (0, 1, 2):
                raise PlanFormatError(f"plan {pid} layer {lid} has an invalid prediction direction: {path}")
            if not isinstance(t, list) or tuple(t) not in ORDERS:
                raise PlanFormatError(f"plan {pid} layer {lid} has an invalid traversal order: {path}")
            preds.append(f"cubic{d}_{ORDERS[tuple(t)]}")
        family = plan.get("predictor_family", "cubic")
        if family not in ("cubic", "quintic"):
            raise PlanFormatError(f"plan {pid} has an invalid predictor_family: {path}")
        out.append((float(plan["rel_eb"]), preds, family))
    return out


def for_rel_eb(plans, rel_eb: float, path="plan file") -> tuple[list[str], str]:
    """The single plan stored for rel_eb (compared with a relative tolerance of 1e-12)."""
    m = [(p, f) for e, p, f in plans if math.isclose(e, rel_eb, rel_tol=1e-12, abs_tol=0.0)]
    if len(m) != 1:
        raise PlanFormatError(f"{path} must hold exactly one plan for rel_eb={rel_eb:g}, found {len(m)}")
    return m[0]


def document(entries: dict) -> dict:
    """Version-2 document from {rel_eb: (predictors, family)}, plans in descending rel_eb."""
    plans = []
    for rel_eb, (preds, family) in sorted(entries.items(), reverse=True):
        layers = []
        for p in preds:
            m = re.fullmatch(r"cubic([012])_(120|021|012)", p)
            if m is None:
                raise PlanFormatError(f"cannot write unknown predictor: {p}")
            layers.append({"prediction_direction": int(m.group(1)), "traversal_order": [int(c) for c in m.group(2)]})
        plans.append({"rel_eb": rel_eb, "predictor_family": family, "layers": layers})
    return {"version": 2, "plans": plans}


def write(path, entries: dict) -> None:
    """Write {rel_eb: (predictors, family)} atomically (temporary file, then rename)."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(path.name + ".tmp")
    with open(tmp, "w", encoding="utf-8") as f:
        json.dump(document(entries), f, indent=2)
        f.write("\n")
    os.replace(tmp, path)


def record_plan(path, rel_eb: float, report) -> None:
    """Add (or replace) the plan a compression used (its asz_report) under rel_eb in a plan file."""
    entries = {}
    if os.path.exists(path):
        for e, p, f in load(path):
            entries[e] = (p, f)
    for e in [e for e in entries if math.isclose(e, rel_eb, rel_tol=1e-12, abs_tol=0.0)]:
        del entries[e]
    plan = report.plan.decode() if isinstance(report.plan, bytes) else report.plan
    entries[float(rel_eb)] = (plan.split(","), "quintic" if report.quintic else "cubic")
    write(path, entries)


def compress_with_plan_file(ctx, data, rel_eb: float, path, params=None):
    """Compress with the plan and family stored for rel_eb in a plan file (asz_b200.api.Context)."""
    preds, family = for_rel_eb(load(path), rel_eb, path)
    return ctx.compress(data, rel_eb, ",".join(preds), family, params)
