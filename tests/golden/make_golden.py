"""Generates golden vectors for the Python-layer pre-processing by running the reference's
OWN fastcone.py (fastcone.py:260-319) in this container.

    python tests/golden/make_golden.py [/path/to/reference]

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
    compat.zeros = lambda shape, *a, **k: np.zeros([int(s) for s in shape], *a, **k)
    mod.np = compat
    return mod


def main(ref_dir="/root/reference"):
    ref = load_reference(ref_dir)
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
