"""bench.py's multi-process plumbing on CPU with gloo (world size 2): the
max over replicas that the job time is taken from, and the reference arm
under torchrun (rank 0 alone works and prints one JSON line)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        v = bench.replica_max(10.0 * (rank + 1), world, 0)
        dist.barrier()
        out.put((rank, v))
    finally:
        dist.destroy_process_group()


def test_replica_max_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 20.0, 1: 20.0}


def test_reference_arm_under_torchrun():
    port = free_port()
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', '--nproc-per-node', '2',
           '--master-addr', '127.0.0.1', '--master-port', str(port), 'bench.py', '--impl', 'reference',
           '--gpus', '2', '--steps', '1', '--warmup', '0', '--n-el', '96', '--fit-sizes', '24,36,48',
           '--no-c2-ref']
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d['impl'] == 'reference' and d['unit'] == 's' and d['higher_is_better'] is False
    assert d['cpu_baseline']['kind'] in ('reference', 'port')
    assert d['e2e']['h2d_bytes_per_step'] == 0
    assert d['extrapolated'] is True and d['fit']['sizes_el'] == [24, 36, 48]
