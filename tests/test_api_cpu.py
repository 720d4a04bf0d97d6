"""The Python drop-in keeps the reference module's call surface: every public function of
the reference's fastcone.py (fastcone.py:52, :147, :260, :272, :294, :306) exists here with
the same parameters in the same order, of the same kinds, with equal defaults (numpy array
defaults by dtype and values); any parameter added here comes after them and has a default,
so every call written against the reference binds the same way.  The reference's signatures
are the committed fixture tests/golden/fastcone_api.json (written by
tests/golden/make_golden.py from the reference's own module)."""
import inspect
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "fastcone_api.json")) as f:
    REF = json.load(f)

FUNCS = sorted(k for k in REF if k != "constants")


def _same_default(ref, ours):
    if ref.get("required"):
        return ours is inspect.Parameter.empty
    if "array" in ref:
        return (isinstance(ours, np.ndarray) and str(ours.dtype) == ref["dtype"]
                and ours.tolist() == ref["array"])
    return not isinstance(ours, np.ndarray) and ours == ref["value"] and type(ours) is type(ref["value"])


@pytest.mark.parametrize("name", FUNCS)
def test_signature_matches_reference(name):
    from fastcone_b200 import fastcone as fc

    params = list(inspect.signature(getattr(fc, name)).parameters.values())
    ref = REF[name]
    assert len(params) >= len(ref), [p.name for p in params]
    for r, p in zip(ref, params):
        assert p.name == r["name"], (name, p.name, r["name"])
        assert p.kind.name == r["kind"], (name, p.name)
        assert _same_default(r, p.default), (name, p.name, p.default, r)
    for p in params[len(ref):]:
        assert p.default is not inspect.Parameter.empty, (name, p.name, "added parameters need a default")


def test_module_constants_match_reference():
    from fastcone_b200 import fastcone as fc

    assert np.dtype(fc.FLOAT_TYPE).name == REF["constants"]["FLOAT_TYPE"]
    assert np.dtype(fc.INT_TYPE).name == REF["constants"]["INT_TYPE"]

