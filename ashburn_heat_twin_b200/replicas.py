"""Replicas across GPUs: one process per GPU, each stepping its own domain(s), no data-path collective.

The live solver's step has no exchange between domains (the reference runs one domain per device), so scaling is
by replicas: every rank steps an independent domain and the only collectives are a barrier around the timed region
and the max over ranks of the measured time. These helpers are that coordination, shared by bench.py (NCCL on GPUs)
and the multi-process tests (gloo on CPU).
"""
from __future__ import annotations


def env_ranks():
    """(rank, world, local rank) from the torchrun environment (single process when unset)."""
    import os
    return (int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
            int(os.environ.get('LOCAL_RANK', '0')))


def max_over_ranks(x, dist=None, device='cpu'):
    """The maximum of a float over all ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist=None, sync=None):
    """Barrier across ranks, then the local device synchronisation `sync` (if given)."""
    if dist is not None:
        dist.barrier()
    if sync is not None:
        sync()


def aggregate_rate(units_per_rank, world, seconds_max):
    """Whole-job throughput of weak-scaled replicas: every rank processed units_per_rank in at most seconds_max."""
    return world * units_per_rank / seconds_max


def launch_ranks(script, argv, n, port=None):
    """Run `script argv` as n ranks on this node under torch.distributed.run (rendezvous on 127.0.0.1) and return the
    launcher's exit status; every rank reads RANK / LOCAL_RANK / WORLD_SIZE from its environment."""
    import socket
    import subprocess
    import sys
    if port is None:
        with socket.socket() as sk:
            sk.bind(('127.0.0.1', 0))
            port = sk.getsockname()[1]
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', f'--nproc-per-node={int(n)}',
           '--master-addr', '127.0.0.1', '--master-port', str(port), script] + list(argv)
    return subprocess.call(cmd)
