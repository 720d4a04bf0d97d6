"""bench.py's reference arm on CPU: the line it prints for `--impl reference` carries the
contract's keys (metric, unit, steps, warm-up, config with the GPU arm's workload name,
cpu_baseline, e2e with no host-device bytes), timed over W untimed and K timed bounded
samples of the CPU reference path.  A small geometry stands in for the 1024^3 workload so
that the check takes seconds."""
import json
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line_has_contract_keys():
    sys.path.insert(0, ROOT)
    import bench

    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.circular((32, 32, 32), 1.0, (48, 32), 1.0, 500.0, 1000.0, 20)
    g = g.with_norm(np.full(20, 1.0 / 20, np.float32))
    args = types.SimpleNamespace(steps=2, warmup=1, gpus=1)
    out = bench.reference_line(args, g, budget_s=0.5)
    json.dumps(out)
    assert out["impl"] == "reference"
    assert out["metric"] == bench.METRIC and out["unit"] == bench.UNIT
    assert out["value"] > 0 and out["higher_is_better"] is True and out["vs_baseline"] is None
    assert (out["steps"], out["warmup"], out["n_gpus"]) == (2, 1, 1)
    assert out["ms_per_step"] > 0
    assert out["config"]["workload"] == bench.WORKLOAD
    cb = out["cpu_baseline"]
    assert cb["value"] == out["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert "2 x " in cb["sample"] and "32x32x32 / 20-view" in cb["sample"]
    e2e = out["e2e"]
    assert e2e["value"] == out["value"] and e2e["unit"] == bench.UNIT
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_cpu_reference_samples_count_updates():
    """One sample backprojects whole voxel columns: updates = columns x nz x views."""
    sys.path.insert(0, ROOT)
    import bench

    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.circular((24, 20, 16), 1.0, (40, 24), 1.0, 300.0, 600.0, 12)
    ref = bench.CpuReferencePath(g)
    dt, upd = ref.sample(5)
    assert dt > 0 and upd == 5 * 16 * 12
