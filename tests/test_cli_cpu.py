"""zdem_gpu's command line against zdem_cpu's (src/main.cpp:1691-1708, 1872-1881), run as programs on the
CPU: the cases that end before any device work (bad or missing arguments, a config that cannot be read
or has nothing to simulate) give the same stdout, stderr and exit status, with the program's name
changed in the usage line."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU_EXE = os.path.join(ROOT, "zedm-x_b200", "bin", "zdem_gpu")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "zdem_cpu")


def _run(exe, args, cwd):
    p = subprocess.run([exe] + args, capture_output=True, text=True, timeout=60, cwd=cwd)
    return p.returncode, p.stdout.replace("zdem_gpu", "zdem").replace("zdem_cpu", "zdem"), p.stderr


@pytest.mark.parametrize("args", [[], ["--help"], ["--config"], ["--bogus"], ["--config", "x.txt", "--what"],
                                  ["--config", "missing.txt"], ["--config", "empty.txt"],
                                  ["--config", "only_globals.txt"]])
def test_cli_matches_reference_before_device_work(tmp_path, args):
    if not os.path.exists(GPU_EXE):
        pytest.fail("zdem_gpu is not built (make -C zedm-x_b200)")
    if not os.path.exists(REF_EXE):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    (tmp_path / "empty.txt").write_text("")
    (tmp_path / "only_globals.txt").write_text("dt = 1e-6\nsteps = 10\n# no particles, no stl\n")
    got = _run(GPU_EXE, args, str(tmp_path))
    want = _run(REF_EXE, args, str(tmp_path))
    usage = "Usage: zdem --config path.txt"
    assert got[0] == want[0] == 1, (got, want)
    assert got[2] == want[2], (got, want)
    if want[1].startswith(usage):
        assert got[1].startswith(usage), got
    else:
        assert got[1] == want[1], (got, want)
