"""The multi-GPU host logic of bench.py on two gloo ranks on the CPU: every rank gets its own
seed range (weak scaling, no overlap), and the whole-job figures are the max step time and
the sum of the units over ranks."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    import datetime
    import sys
    import torch.distributed as D
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    D.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, _ = bench.dist()
        seeds = bench.seeds_of("0-9", r)
        step, kern, tot = bench.reduce_over_ranks(1.0 + r, 0.5 * (r + 1), [10.0 * (r + 1), 3.0], "cpu")
        q.put((r, w, seeds, step, kern, tot))
    finally:
        D.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, s0, st0, k0, t0), (r1, w1, s1, st1, k1, t1) = out
    assert w0 == w1 == 2
    assert s0 == list(range(0, 10)) and s1 == list(range(10, 20))  # disjoint, same size
    assert st0 == st1 == 2.0 and k0 == k1 == 1.0                     # max over ranks
    assert t0 == t1 == [30.0, 6.0]                                   # sums over ranks
