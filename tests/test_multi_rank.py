"""Multi-GPU sharding logic on CPU: two gloo ranks, each taking its slice of
the lanes (devices.zig capacity split) with the same lead-lane tape, solved by
the CPU oracle; the gathered result equals a single-process run lane for
lane, so results do not depend on the rank count (multi.zig:1-5); and the
points layer's split of pending points across ranks with every rank
receiving every result."""
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


def _points_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    from egspice_b200 import points as pt
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    pt.LANE_WIDTH = 4  # batches of the lead lane and 3 points, so 11 points make 4 batches
    p = pt.Points(POINTS_DECK, ["rval"])
    seen = []
    calls = []

    def fake_run_ids(ids):  # stands in for the GPU run: a result that names its point
        calls.append(list(ids))
        seen.extend(ids)
        return {k: (np.array([p.rows[k][0], -float(k)]), k % 3) for k in ids}

    p._run_ids = fake_run_ids
    p.append_points(np.arange(1, 12, dtype=np.float64)[:, None] * 1e3)
    p.append_points([[np.nan]])  # refused as appended: no rank runs it
    p.run()
    v, r = p.copy_point_measures(0, 12, ["t50", "v2n"])
    ran = np.array(sorted(seen) + [-1] * (12 - len(seen)), dtype=np.float64)
    np.save(out + f".{rank}.npy", np.concatenate([v, r[:, None], ran[:, None]], axis=1))
    # every batch a rank ran is a whole batch of the one-process batching,
    # led by the deck's own value of the live parameter
    one = [b for b in p.batches(list(range(11)))]
    assert all(c in one for c in calls), (calls, one)
    assert p.lead is not None and p.lead.tolist() == [1000.0]
    dist.barrier()
    dist.destroy_process_group()


POINTS_DECK = """RC points
vin in 0 dc 0 pulse(0 1 0 0.2n 0.2n 1 2)
r1 in out {rval}
c1 out 0 1p
.param rval=1k
.tran 1p 6n
.meas tran t50 when v(out)=0.5
.meas tran v2n find v(out) at=2n
.end
"""


def test_points_split_across_two_ranks(tmp_path):
    """Points.run under torch.distributed (gloo, two ranks, the GPU run
    replaced by a result naming its point): the one-process batches of the
    11 pending points (the lead lane and 3 points each) split into
    contiguous runs of whole batches, one per rank, and both ranks end with
    every point's result, equal to a one-process run."""
    out = str(tmp_path / "p")
    mp.spawn(_points_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    a, b = np.load(out + ".0.npy"), np.load(out + ".1.npy")
    np.testing.assert_array_equal(a[:, :3], b[:, :3])
    rows = np.arange(1, 12) * 1e3
    np.testing.assert_array_equal(a[:11, 0], rows)
    np.testing.assert_array_equal(a[:11, 1], -np.arange(11))
    np.testing.assert_array_equal(a[:11, 2], np.arange(11) % 3)
    assert np.isnan(a[11, :2]).all() and a[11, 2] == 9  # INVALID_PARAMETER
    # rank 0 ran points 0..5, rank 1 points 6..10
    np.testing.assert_array_equal(a[:6, 3], np.arange(6))
    np.testing.assert_array_equal(b[:5, 3], np.arange(6, 11))
