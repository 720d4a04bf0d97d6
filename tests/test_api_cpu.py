"""The Python drop-in keeps the reference module's call surface: every public function of
the reference's fastcone.py (fastcone.py:52, :147, :260, :272, :294, :306) exists here with
the same parameters in the same order, of the same kinds, with equal defaults (numpy array
defaults by dtype and values); any parameter added here comes after them and has a default,
so every call written against the reference binds the same way.  And the calls reach the C
ABI with the arguments the reference's module passes for them.  The reference's signatures
and recorded C-call arguments are the committed fixtures tests/golden/fastcone_api.json and
tests/golden/fastcone_calls.json (written by tests/golden/make_golden.py from the
reference's own module)."""
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



with open(os.path.join(HERE, "golden", "fastcone_calls.json")) as f:
    CALLS = json.load(f)


@pytest.mark.parametrize("idx", range(len(CALLS)))
def test_c_call_arguments_match_reference(idx, monkeypatch):
    """The same project / backproject call reaches the C ABI with the arguments the
    reference's fastcone.py passes (the fixture recorded them through a stand-in library):
    same entry point, scalars, reversed dimension arrays, offsets, default normalisation and
    misalignments, pointers to the caller's own vol / proj; and proj afterwards (the
    projector's column-0 zeroing) is the same."""
    import sys

    sys.path.insert(0, os.path.join(HERE, "golden"))
    import api_calls

    from fastcone_b200 import _lib
    from fastcone_b200 import fastcone as fc

    rec = api_calls.Recorder()
    monkeypatch.setattr(fc, "lib", lambda: rec)
    monkeypatch.setattr(_lib, "check_last", lambda: None)
    fn, kw = api_calls.calls()[idx]
    want = CALLS[idx]
    assert want["fn"] == fn
    vol, proj = api_calls.arrays()
    getattr(fc, fn)(vol, proj, **kw)
    (name, args), = rec.calls
    got = api_calls.decode(name, args, vol, proj)
    assert got == want["c_call"]
    assert proj.tolist() == want["proj_after"]
