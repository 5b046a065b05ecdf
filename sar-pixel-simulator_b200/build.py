"""Build libfdtd_b200.so (the CUDA kernels + C-ABI) in-tree for sm_100a.

    python sar-pixel-simulator_b200/build.py [--force] [--verbose] [--bounds-check]

Each .cu under csrc/ is compiled to an object in csrc/_build/ (in parallel)
and linked into fdtdsarsim_b200/libfdtd_b200.so next to the Python package
that loads it. Objects are rebuilt when a source or header is newer.
--bounds-check builds the bounds-checked library instead
(-DFDTD_BOUNDS_CHECK, relocatable device code so that one allocation table
serves every source file; objects in csrc/_build_check/) as
fdtdsarsim_b200/libfdtd_b200_check.so; the package loads it when
FDTDSARSIM_B200_LIBRARY=check is set.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(CSRC, '_build')
INCLUDE = os.path.join(ROOT, 'include')
LIB = os.path.join(HERE, 'fdtdsarsim_b200', 'libfdtd_b200.so')

NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC,-ffp-contract=off',
         '-I', INCLUDE, '-I', CSRC]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False, extra_flags=(), bounds_check=False):
    build_dir = BUILD + '_check' if bounds_check else BUILD
    lib = LIB[:-3] + '_check.so' if bounds_check else LIB
    check_flags = ['-DFDTD_BOUNDS_CHECK', '-rdc=true'] if bounds_check else []
    os.makedirs(build_dir, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    headers = glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(CSRC, '*.h')) \
        + glob.glob(os.path.join(INCLUDE, '*.h'))
    hdr_time = _newest(headers) if headers else 0.0
    jobs = []
    objs = []
    for src in sources:
        obj = os.path.join(build_dir, os.path.basename(src)[:-3] + '.o')
        objs.append(obj)
        if force or not os.path.exists(obj) or \
                os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_time):
            cmd = [NVCC] + ARCH + FLAGS + check_flags + list(extra_flags) + ['-c', src, '-o', obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(' '.join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    failed = []
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for cmd, p in ex.map(run, jobs):
            if verbose and (p.stdout or p.stderr):
                print(p.stdout + p.stderr, flush=True)
            if p.returncode != 0:
                failed.append((cmd, p.stdout + p.stderr))
    if failed:
        msg = '\n'.join(' '.join(c) + '\n' + out for c, out in failed)
        raise RuntimeError('nvcc failed:\n' + msg)
    if force or jobs or not os.path.exists(lib) or os.path.getmtime(lib) < _newest(objs):
        cmd = [NVCC] + ARCH + check_flags[1:] + ['-shared', '-o', lib] + objs + ['-lcudart', '-lcuda', '-lcufft']
        if verbose:
            print(' '.join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError('link failed:\n' + p.stdout + p.stderr)
    return lib


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    ap.add_argument('--ptxas-info', action='store_true', help='print register/smem use')
    ap.add_argument('--bounds-check', action='store_true', help='build libfdtd_b200_check.so')
    a = ap.parse_args()
    extra = ['-Xptxas', '-v'] if a.ptxas_info else []
    print(build(a.force or a.ptxas_info, a.verbose or a.ptxas_info, extra, a.bounds_check))
    sys.exit(0)
