"""The C-ABI from plain C: a C99 program including include/fdtd_b200.h,
linked against libfdtd_b200.so, calls the entry points that need no device
(version, error text, argument validation that precedes any device use)."""
import os
import shutil
import subprocess

import pytest

from fdtdsarsim_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include <stdio.h>
#include <string.h>
#include "fdtd_b200.h"

int main(void) {
    char msg[256];
    if (fdtd_version() < 100) return 10;
    fdtd_sim *sim = NULL;
    fdtd_geometry g;
    memset(&g, 0, sizeof(g));
    g.nx = g.ny = g.nz = 5; g.npml = 10; g.tfsf_z = 2; g.nt = 10; g.nt_inc = 5;
    g.dtype = FDTD_F32; g.cell_size = 1e-3; g.timestep = 1e-12; g.frequency = 5.4e9;
    if (fdtd_create(&g, 0, &sim) != FDTD_ERR_INVALID || sim != NULL) return 11;
    fdtd_last_error(msg, (int)sizeof(msg));
    if (!strstr(msg, "too small")) return 12;
    if (fdtd_run(NULL, 1) != FDTD_ERR_INVALID) return 13;
    if (fdtd_batch_run(NULL, 1) == FDTD_OK) return 14;
    int out[7 * 64], n = 0;
    if (fdtd_fused_plan_boxes(761, 761, 203, 10, 156, 4, 0, 0, out, 64, &n) != FDTD_OK || n < 2) return 15;
    printf("ok %d boxes\n", n);
    return 0;
}
'''


@pytest.mark.skipif(shutil.which('gcc') is None, reason='no C compiler')
def test_c_program_links_and_calls(tmp_path):
    src = tmp_path / 'consumer.c'
    src.write_text(PROGRAM)
    exe = tmp_path / 'consumer'
    libdir = os.path.dirname(_native.LIB_PATH)
    cmd = ['gcc', '-std=c99', '-Wall', '-Werror', '-I', os.path.join(ROOT, 'include'), str(src),
           '-o', str(exe), '-L', libdir, '-l:libfdtd_b200.so', f'-Wl,-rpath,{libdir}']
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith('ok')


PRELUDE = r'''
#include <stddef.h>
#include "fdtd_b200.h"
int nx, ny, nz, tfsf_z, nt, nt_inc, size_t_pulse, size_t_inc, i;
double dx, dt, db, dtm0, dte0dx, theta, phi, radius;
float *profiles, *ca, *cb, *ex, *ey, *hx, *hy, *ex_ph_u, *all24, *out;
double *k_vals, *pulse_fft;
fdtd_geometry g;
fdtd_sim *sim;                  /* a main simulation of an earlier example */
'''


EXAMPLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'examples')


@pytest.mark.skipif(shutil.which('gcc') is None, reason='no C compiler')
def test_c_call_examples_compile_against_the_header(tmp_path):
    """The C call sequences of tests/examples (those a reference-side
    integration makes) compile, syntax and types, against
    include/fdtd_b200.h, so they keep the header's names and arguments."""
    import glob
    files = sorted(glob.glob(os.path.join(EXAMPLES, '*.c')))
    assert len(files) >= 3
    for k, path in enumerate(files):
        block = open(path).read()
        body = '\n'.join(line for line in block.splitlines() if not line.startswith('#include'))
        src = tmp_path / f'example{k}.c'
        src.write_text(PRELUDE + f'void example{k}(void) {{\n{body}\n}}\n')
        r = subprocess.run(['gcc', '-std=c99', '-fsyntax-only', '-Werror=implicit-function-declaration',
                            '-Werror=incompatible-pointer-types', '-I', os.path.join(ROOT, 'include'),
                            str(src)], capture_output=True, text=True)
        assert r.returncode == 0, (path, r.stderr)


def test_python_call_examples_parse():
    """The Python call sequences of tests/examples are valid Python (each
    read as the body of a function, since the selector branch returns)."""
    import glob
    files = sorted(glob.glob(os.path.join(EXAMPLES, '*.py')))
    assert len(files) >= 3
    for path in files:
        block = open(path).read()
        src = 'def _example():\n' + '\n'.join('    ' + line for line in block.splitlines())
        compile(src, path, 'exec')
