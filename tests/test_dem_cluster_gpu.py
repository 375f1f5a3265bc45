"""The spinning 8-particle cluster on the GPU against the reference program (the comparison of
tests/test_dem_gpu.py): broad phase, multi-pair scatter order and history with split_contacts off.  The
scene's config holds plain floats (numpy 2 reprs would not parse in either program), and the oracle's
DEM step reproduces the reference on it bit for bit (tests/test_oracle_dem_cpu.py)."""
import numpy as np
import pytest

from _dem_helpers import fmt, write_binary_stl
from test_dem_gpu import MAT, _compare_run

pytestmark = pytest.mark.gpu


def test_cluster_with_spin_and_split_off(tmp_path):
    """Eight particles in a tight cluster with spin: broad phase, multi-pair scatter order, history."""
    from zdemx import synth

    rng = np.random.default_rng(2)
    write_binary_stl(str(tmp_path / "a.stl"), synth.noised_icosphere(1, 1e-3, 0.15, rng))
    write_binary_stl(str(tmp_path / "b.stl"), synth.noised_icosphere(2, 1e-3, 0.1, rng))
    parts = []
    for i in range(8):
        pos = np.array([(i % 2) * 1.85e-3, ((i // 2) % 2) * 1.85e-3, (i // 4) * 1.85e-3]) + rng.uniform(-5e-5, 5e-5, 3)
        q = synth.random_unit_quat(rng)
        parts.append(dict(stl=str(tmp_path / ("a.stl" if i % 3 else "b.stl")), pos=fmt(pos),
                          vel=fmt(rng.normal(size=3) * 0.02), quat=fmt(q), omega=fmt(rng.normal(size=3) * 5.0),
                          scale=1, **MAT))
    _compare_run(tmp_path, {"steps": 40, "dt": 1e-6, "split_contacts": 0, "gravity": "0 0 -9.81",
                            "output_interval": 2}, parts, min_contact_steps=5)
