"""Multi-GPU sharding logic on CPU: two gloo ranks, each taking its slice of
the lanes (devices.zig capacity split) with the same lead-lane tape, solved by
the CPU oracle; the gathered result equals a single-process run lane for
lane, so results do not depend on the rank count (multi.zig:1-5)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from egspice_b200.multi import split_lanes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_split_lanes():
    assert split_lanes(10, [1, 1]) == [(0, 5), (5, 5)]
    assert split_lanes(7, [1, 1, 1]) == [(0, 3), (3, 2), (5, 2)]
    assert split_lanes(100, [3, 1]) == [(0, 75), (75, 25)]
    with pytest.raises(ValueError):
        split_lanes(0, [1])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    from egspice_b200 import abi, decks
    from egspice_b200.multi import gather_rows, shard
    from oracle import pyoracle as po
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    net = decks.inverter_chain(10)
    local, start = shard(net, rank, world)
    x, res = po.op_lanes(local, abi.newton_opts())
    lead_extra = 1 if start != 0 else 0
    allx = gather_rows(x, start, lead_extra)
    if rank == 0:
        np.save(out, allx)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_match_one(tmp_path):
    from egspice_b200 import abi, decks
    from oracle import pyoracle as po
    out = str(tmp_path / "x.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    allx = np.load(out)
    net = decks.inverter_chain(10)
    x1, _ = po.op_lanes(net, abi.newton_opts())
    assert allx.shape == x1.shape
    assert np.array_equal(allx, x1)
