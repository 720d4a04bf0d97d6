"""Generates golden vectors for the Python-layer pre-processing by running the reference's
OWN fastcone.py (fastcone.py:260-319) in this container.

    python tests/golden/make_golden.py [/path/to/reference] [all|api]

(the reference tree: the first argument, else $FASTCONE_REFERENCE)

It also records the signatures of the module's public functions (names, kinds and defaults
of their parameters, fastcone.py:52, :147, :260, :272, :294, :306) in fastcone_api.json,
and, in fastcone_calls.json, the C-ABI arguments that its project / backproject pass for
the calls of api_calls.py (through a recording stand-in for the library); the ``api``
argument writes only those two files.

Three shims, applied to the imported module only, make it runnable on numpy >= 1.12 without
touching its code: ``np.zeros`` accepts the float shape the reference builds
(``proj.shape[2]*2.0``, fastcone.py:274); ``backproject`` is replaced by a no-op so
``fbp`` stops after its pre-processing (the C library is not involved); and the module gets
the ``scipy`` name that gaussrampfilter uses without importing (fastcone.py:310-311), with
``scipy.signal.gaussian`` pointing at its current home ``scipy.signal.windows.gaussian``.
"""
import importlib.util
import os
import sys
import types

import numpy as np
import scipy.ndimage
import scipy.signal

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref_dir):
    spec = importlib.util.spec_from_file_location("fastcone_ref", os.path.join(ref_dir, "fastcone.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    compat = types.ModuleType("numpy_compat")
    compat.__dict__.update(np.__dict__)
    compat.zeros = lambda shape, *a, **k: np.zeros(int(shape) if np.ndim(shape) == 0 else [int(s) for s in shape],
                                                   *a, **k)
    mod.np = compat
    return mod


API_FUNCTIONS = ("project", "backproject", "fbp", "rampfilter", "cosrampfilter", "gaussrampfilter")


def describe_default(v):
    """JSON form of a parameter default (numpy arrays by dtype and values)."""
    import inspect

    if v is inspect.Parameter.empty:
        return {"required": True}
    if isinstance(v, np.ndarray):
        return {"array": v.tolist(), "dtype": str(v.dtype)}
    return {"value": v}


def api_signatures(mod):
    """Parameter names, kinds and defaults of the module's public functions."""
    import inspect

    out = {}
    for name in API_FUNCTIONS:
        sig = inspect.signature(getattr(mod, name))
        out[name] = [{"name": p.name, "kind": p.kind.name, **describe_default(p.default)}
                     for p in sig.parameters.values()]
    out["constants"] = {"FLOAT_TYPE": np.dtype(mod.FLOAT_TYPE).name, "INT_TYPE": np.dtype(mod.INT_TYPE).name}
    return out


def record_calls(ref):
    """Runs the reference's project / backproject on the calls of api_calls.py with a
    recording stand-in for ctypes.CDLL("libFastcone.so"); returns each call's C-ABI
    arguments and the proj array afterwards (the projector zeroes column 0)."""
    import ctypes

    sys.path.insert(0, HERE)
    import api_calls

    rec = api_calls.Recorder()
    shim = types.SimpleNamespace(CDLL=lambda name: rec, c_int=ctypes.c_int, c_float=ctypes.c_float,
                                 POINTER=ctypes.POINTER)
    real = ref.ctypes
    ref.ctypes = shim
    out = []
    try:
        for fn, kw in api_calls.calls():
            vol, proj = api_calls.arrays()
            rec.calls.clear()
            getattr(ref, fn)(vol, proj, **kw)
            (name, args), = rec.calls
            out.append({"fn": fn, "c_call": api_calls.decode(name, args, vol, proj),
                        "proj_after": proj.tolist()})
    finally:
        ref.ctypes = real
    return out


def write_api(ref):
    import json

    with open(os.path.join(HERE, "fastcone_api.json"), "w") as f:
        json.dump(api_signatures(ref), f, indent=1)
        f.write("\n")
    with open(os.path.join(HERE, "fastcone_calls.json"), "w") as f:
        json.dump(record_calls(ref), f)
        f.write("\n")


def main(ref_dir=None, what="all"):
    # the reference checkout: the first argument, else $FASTCONE_REFERENCE, else the
    # conventional location
    ref_dir = ref_dir or os.environ.get("FASTCONE_REFERENCE", "/root/reference")
    ref = load_reference(ref_dir)
    write_api(ref)
    if what == "api":
        print("API signatures written to", HERE)
        return
    rng = np.random.default_rng(20240601)
    for name, shape in (("rampfilter_a", (3, 16, 24)), ("rampfilter_b", (2, 9, 37))):
        x = rng.standard_normal(shape).astype(np.float32)
        y = x.copy()
        ref.rampfilter(y)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), input=x, output=y)
    # fbp pre-processing: cosine weight (then ramp filter)
    x = rng.random((4, 20, 28)).astype(np.float32)
    z = np.array([9.5, 10.0, 10.25, 11.0])
    D = 60.0
    w = x.copy()
    real_ramp, real_bp = ref.rampfilter, ref.backproject
    ref.rampfilter = lambda p: None
    ref.backproject = lambda *a, **k: 1
    ref.fbp(np.zeros((4, 4, 4), np.float32), w, np.zeros(4), D, z)
    f = w.copy()
    real_ramp(f)
    ref.rampfilter, ref.backproject = real_ramp, real_bp
    np.savez_compressed(os.path.join(HERE, "fbp_weight.npz"), input=x, zOrigin=z, D=D, weighted=w, filtered=f)
    # apodised ramps (fastcone.py:294-319), view by view: the reference stores only the last
    # view of a multi-view call and needs an even row length
    ref.scipy = types.SimpleNamespace(signal=types.SimpleNamespace(gaussian=scipy.signal.windows.gaussian),
                                      ndimage=scipy.ndimage)
    for name, shape, call in (("cosramp_a", (3, 16, 24), lambda p: ref.cosrampfilter(p)),
                              ("gaussramp_a", (3, 16, 24), lambda p: ref.gaussrampfilter(p)),
                              ("gaussramp_b", (2, 9, 38), lambda p: ref.gaussrampfilter(p, scale=0.3))):
        x = rng.standard_normal(shape).astype(np.float32)
        y = x.copy()
        for t in range(shape[0]):
            v = x[t:t + 1].copy()
            call(v)
            y[t] = v[0]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), input=x, output=y)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
