"""The float identities the kernels use instead of the reference's double
arithmetic (tracking: reciprocal, rounding of projections, thresholds, the
Sobel scale) and instead of IEEE division (integration: quotients sharing one
reciprocal, Markstein's correction step), checked on the host over every
significand or dense samples (tests/host_c/float_identities.c).  The GPU
parity tests then check the kernels' results bit for bit."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_float_identities(tmp_path):
    exe = tmp_path / "float_identities"
    src = os.path.join(HERE, "host_c", "float_identities.c")
    try:
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), src, "-lm"])
    except (OSError, subprocess.CalledProcessError) as e:
        pytest.skip(f"no C compiler: {e}")
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, timeout=300).stdout
    rows = {line.split()[0]: (int(line.split()[1]), int(line.split()[2])) for line in out.splitlines()}
    assert set(rows) == {"fd_rcp", "trunc_half_up", "floor_half_up", "thresholds", "quotients"}, out
    for name, (n, bad) in rows.items():
        assert n > 0 and bad == 0, (name, n, bad)
