"""The product never routes through the checker: no module or source of fastcone_b200/
imports, includes or links the oracle, nothing in it reads the reference's source tree, and
the library has no CPU fallback that would stand in for a missing CUDA build."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fastcone_b200")


def _sources():
    for d, _, files in os.walk(PKG):
        if "_build" in d or "__pycache__" in d:
            continue
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h", ".cuh")):
                p = os.path.join(d, f)
                with open(p, encoding="utf-8") as fh:
                    yield os.path.relpath(p, ROOT), fh.read()


def test_no_oracle_in_the_product():
    bad = []
    for path, text in _sources():
        if re.search(r"^\s*(from\s+oracle\b|import\s+oracle\b)", text, re.M):
            bad.append((path, "imports the oracle"))
        if re.search(r"fc_oracle|libfc_oracle|oracle/_ref", text):
            bad.append((path, "names the oracle's library"))
        if "/root/reference" in text:
            bad.append((path, "reads the reference tree"))
    assert not bad, bad


def test_library_loader_fails_loudly_without_the_build(monkeypatch):
    """With the shared object missing, the first call raises instead of falling back."""
    import pytest

    from fastcone_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", os.path.join(PKG, "_build", "does_not_exist.so"))
    with pytest.raises(_lib.FastconeError, match="not built"):
        _lib.lib()


def test_torch_entry_points_refuse_host_tensors():
    """The torch API has no CPU path: host tensors are refused before any library call."""
    import numpy as np
    import pytest
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry((8, 8, 8), (12, 10), np.linspace(0, 1, 4), 40.0, 1.0)
    with pytest.raises(ValueError, match="no CPU path"):
        ops.backproject(torch.zeros(g.proj_shape), g)
    with pytest.raises(ValueError, match="no CPU path"):
        ops.project(torch.zeros(g.vol_shape), g)
    with pytest.raises(ValueError, match="no CPU path"):
        ops.project_adjoint(torch.zeros(g.proj_shape), g)
