"""Host-side pieces of the measurement tools, on the CPU: the bench's reference
arm prints one JSON line of the contract, and the study helpers (relMSE,
time to reach an error, the seeded batched workload) compute what their
docstrings say."""
from __future__ import annotations

import json
import math
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    """One JSON line of the contract, from the oracle alone: the GPU package
    and its native library are never loaded by the reference arm."""
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
    code = ("import sys, bench\n"
            "rc = bench.main(['--impl', 'reference', '--steps', '1', '--warmup', '3'])\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(int('wgpu_spectral_rt_b200' in sys.modules), int('libsrt_b200' in maps), "
            "int('liboracle' in maps), file=sys.stderr)\n"
            "sys.exit(rc)\n")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stderr.strip().splitlines()[-1] == "0 0 1"  # no GPU package, no libsrt_b200.so, the oracle
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert "1568780 triangles" in d["config"]["workload"]
    assert d["impl"] == "reference" and d["metric"] == "Mpaths/s" and d["unit"] == "Mpaths/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 3
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("config2")
    # beside the port: the reference's own shaders (translated, built from the
    # reference tree) on whole frames at their own constants, or why not
    rs = d["reference_shaders"]
    assert ("unavailable" in rs) or (rs["kind"] == "reference" and rs["value"] > 0 and rs["frames"] >= 1
                                     and "2^20 photons" in rs["sample"])


def test_relmse_and_time_to_reach():
    from wgpu_spectral_rt_b200.guide_study import _time_to_reach, relmse

    ref = np.full((2, 2, 3), 0.1)
    x = ref + 0.1
    assert math.isclose(relmse(x, ref), 0.01 / (0.01 + 0.01))  # (x - ref)^2 / (ref^2 + 0.01)
    # error ~ 1 / t on a log-log line: reaching 0.25 between t = 2 (0.5) and t = 8 (0.125) gives t = 4
    curve = [(1.0, 10, 1.0), (2.0, 20, 0.5), (8.0, 80, 0.125)]
    assert math.isclose(_time_to_reach(curve, 0.25), 4.0, rel_tol=1e-9)
    assert _time_to_reach(curve, 2.0) == 1.0  # reached at the first checkpoint
    assert _time_to_reach(curve, 0.01) is None  # never reached


def test_batched_workload_is_seeded_and_in_range():
    from wgpu_spectral_rt_b200.batch_guide_study import _workload

    a = _workload(16, (256, 512, 1024, 2048), (1e6, 16e6), 777)
    b = _workload(16, (256, 512, 1024, 2048), (1e6, 16e6), 777)
    assert a == b
    sizes, photons = a
    assert len(sizes) == len(photons) == 16
    assert all(w == h and w in (256, 512, 1024, 2048) for w, h in sizes)
    assert all(1e6 <= p <= 16e6 for p in photons)
    assert _workload(16, (256, 512), (1e6, 2e6), 778) != a


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 times the reference; the other ranks print nothing and exit 0."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
