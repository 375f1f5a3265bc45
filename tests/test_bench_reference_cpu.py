"""bench.py's reference arm (`--impl reference`: the reference's own per-pair code from oracle/_ref on all
host threads, no GPU) prints one JSON line with the keys of the benchmark line: the same metric, unit
and workload as the CUDA arm, its CPU baseline and an end-to-end figure with no host-device traffic."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    from oracle import LIB_REF

    if not os.path.exists(LIB_REF):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "pair-contacts/s" and d["unit"] == "pairs/s"
    for k in ("value", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
              "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_workload_loads_nothing_of_this_library():
    """The reference arm builds its meshes with the reference's own build_mesh: the process that times
    the reference never maps libzdemx.so."""
    from oracle import LIB_REF

    if not os.path.exists(LIB_REF):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    code = ("import sys, types; sys.argv = ['bench.py']; sys.path.insert(0, %r); import bench; "
            "a = types.SimpleNamespace(seed=3, lib_per_level=2, pairs=16); "
            "lib, pm, pp = bench.workload(a, 0, builder='reference'); "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libzdem_ref' in maps and 'libzdemx' not in maps, 'libzdemx mapped'; "
            "assert lib.n_mesh == 8 and pm.shape == (16, 2); print('ok')") % ROOT
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert p.returncode == 0 and p.stdout.strip().endswith("ok"), p.stderr[-2000:]
