"""The bounds-checked build (libfdtd_b200_check.so) on tiny and ragged
grids: every step path (split, fused with the split-pass shell, the column march, fused with
the marched shell, one-plane z chunks, the batched tile queue) runs with
every global access of its kernels checked against the library's live
allocations and every shared index against its array, and must report no
violation (FDTD_ERR_BOUNDS) while matching the oracle bit for bit. Runs in a
child process, which loads the checked library instead of the normal one."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CHECK_LIB = os.path.join(os.path.dirname(HERE), 'sar-pixel-simulator_b200', 'fdtdsarsim_b200',
                         'libfdtd_b200_check.so')


def test_checked_build_reports_no_violation_and_matches_the_oracle():
    assert os.path.exists(CHECK_LIB), 'build it: python sar-pixel-simulator_b200/build.py --bounds-check'
    env = dict(os.environ, FDTDSARSIM_B200_LIBRARY='check')
    out = subprocess.run([sys.executable, os.path.join(HERE, 'bounds_cases.py')], env=env,
                         capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res['library'] == 'libfdtd_b200_check.so' and res['checked'] is True
    bad = [r for r in res['runs'] if r['error'] is not None or r.get('bit_exact') is False]
    assert not bad, bad
    assert len(res['runs']) >= 25
