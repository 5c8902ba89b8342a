"""Replica sharding on CPU: SETFREQIP's round-robin and the site-result all-gather (gloo, world_size 2)."""
import os
import socket

import numpy as np
import pytest

from actfemtide_b200.dist import gather_site_results, setfreqip


def reference_setfreqip(nfreq, ip, np_):
    # n_ebfem_bxyz_mpi.f90:97-101, 343-349 written out with 1-based loops
    nfreq_ip = nfreq // np_
    if nfreq - nfreq_ip * np_ > 0:
        nfreq_ip += 1
    freq_ip = [-1] * nfreq_ip
    for i in range(1, nfreq_ip + 1):
        ii = ip + 1 + (i - 1) * np_
        if ii <= nfreq:
            freq_ip[i - 1] = ii
    return [f - 1 for f in freq_ip if f > 0]


@pytest.mark.parametrize("nfreq", [1, 2, 7, 8, 16, 17])
@pytest.mark.parametrize("np_", [1, 2, 3, 8])
def test_setfreqip_partition(nfreq, np_):
    seen = []
    for ip in range(np_):
        mine = setfreqip(nfreq, ip, np_)
        assert mine == reference_setfreqip(nfreq, ip, np_)
        seen += mine
    assert sorted(seen) == list(range(nfreq))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, nfreq, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        local = {}
        for k in setfreqip(nfreq, rank, ws):
            # stand-in for one solve's (5, nobs) site response
            local[k] = (k + 1) * (np.arange(10).reshape(5, 2) + 1j * np.arange(10).reshape(5, 2))
        full = gather_site_results(local, nfreq, (5, 2))
        q.put((rank, full))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nfreq", [3, 8])
def test_gather_two_ranks_gloo(nfreq):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, nfreq, q)) for r in range(2)]
    for p in ps:
        p.start()
    outs = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.stack([(k + 1) * (np.arange(10).reshape(5, 2) + 1j * np.arange(10).reshape(5, 2))
                       for k in range(nfreq)])
    for _, full in outs:
        assert np.array_equal(full, expect)
