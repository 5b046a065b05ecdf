"""bench.py's multi-GPU path (replicas: one process per GPU, no data
exchanged) on the CPU with two gloo ranks: rank set-up from the launcher's
environment, the max-over-ranks time, the whole-job rate, the reference arm
running on rank 0 only, and a rank that leaves early ending its peer's next
collective with an error instead of a hang."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out_dir, leave_early):
    os.environ.update({'RANK': str(rank), 'WORLD_SIZE': str(world), 'LOCAL_RANK': str(rank),
                       'MASTER_ADDR': '127.0.0.1', 'MASTER_PORT': str(port)})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    r, w, local = bench.init_replicas('gloo', timeout_s=20)
    res = {'rank': r, 'world': w, 'local': local}
    if leave_early:
        if r == 1:
            dist.destroy_process_group()
            return
        try:
            dist.barrier()
            res['barrier'] = 'passed'
        except Exception as e:   # the peer is gone: an error, not a hang
            res['barrier'] = 'error: ' + type(e).__name__
    else:
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0 * r, w, 'cpu')
        res['ms_max'] = ms
        res['rate'] = bench.job_rate(1000, 4, ms, w)
        res['reference_arm_ran'] = bench.run_reference(None) is not None if r != 0 else None
        dist.barrier()
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f'rank{r}.json'), 'w') as fh:
        json.dump(res, fh)


def run(tmp_path, leave_early):
    ctx = mp.get_context('spawn')
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, str(tmp_path), leave_early))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode is not None, 'rank hung'
    return [json.load(open(tmp_path / f'rank{r}.json')) for r in range(2)
            if (tmp_path / f'rank{r}.json').exists()]


def test_two_replicas_max_time_and_job_rate(tmp_path):
    res = run(tmp_path, False)
    assert len(res) == 2
    for r in res:
        assert r['world'] == 2 and r['local'] == r['rank']
        assert r['ms_max'] == 15.0                      # the slower replica's time
        assert r['rate'] == pytest.approx(2 * 1000 * 4 / 0.015 / 1e6)
    assert res[1]['reference_arm_ran'] is False         # rank 1 does no reference work


def test_rank_that_leaves_early_ends_peer_collective(tmp_path):
    res = run(tmp_path, True)
    assert len(res) == 1 and res[0]['rank'] == 0
    assert res[0]['barrier'].startswith('error')


def test_reference_arm_line_on_the_host():
    """bench.py --impl reference needs no GPU: it times the C restatement
    on the host cores and prints one line with the contract's keys."""
    import subprocess
    # run bench.py in a process that then reports whether the product
    # library was ever mapped: the reference arm must not load it
    code = ('import runpy, sys\n'
            f'sys.argv = [{os.path.join(ROOT, "bench.py")!r}, "--impl", "reference", '
            '"--workload", "plain_8x8", "--steps", "1", "--warmup", "1"]\n'
            f'runpy.run_path({os.path.join(ROOT, "bench.py")!r}, run_name="__main__")\n'
            'maps = open("/proc/self/maps").read()\n'
            'print("MAPPED", "libfdtd_b200" in maps, "fdtdsarsim_b200._native" in sys.modules, '
            'file=sys.stderr)\n')
    out = subprocess.run([sys.executable, '-c', code], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, check=True)
    assert 'MAPPED False False' in out.stderr, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line['impl'] == 'reference' and line['metric'] == 'Mcell-updates/s'
    assert line['value'] > 0 and line['higher_is_better'] is True and line['n_gpus'] == 1
    assert line['cpu_baseline']['kind'] == 'port' and line['cpu_baseline']['cores'] >= 1
    assert line['e2e'] == {'value': line['value'], 'unit': 'Mcell-updates/s',
                           'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}
    assert line['config']['grid'] == [101, 381, 381]
    assert '0.35 GB' in line['config']['l2']
