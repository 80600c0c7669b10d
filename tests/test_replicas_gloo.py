"""World-size-2 run of the multi-GPU path on CPU (gloo): independent replicas, each building the
same pressure system and hierarchy on its host, and the max-over-ranks timing summary."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import cfd_b200 as cb
    import oracle as O
    from cfd_b200 import workloads as W
    from cfd_b200.multi import replica_summary
    case = W.graded(8)
    up, lo, dg, dv = O.assemble(case.n, case.owner, case.neighbour, case.flux, case.gamma,
                                case.delta, 0.0)
    diag, src = case.finalize(up, lo, dg, dv)
    pat = cb.build_csr_pattern(case.n, case.owner, case.neighbour)
    val = np.zeros(pat.nnz)
    val[pat.diag_pos], val[pat.upper_pos], val[pat.lower_pos] = diag, up, lo
    h = cb.AmgHierarchy(cb.CsrView(case.n, pat.row_ptr, pat.col, val))
    ci = h.coarse_inverse()
    ms, rate = replica_summary(10.0 + 5.0 * rank, steps=4, world=world)
    out[rank] = (ms, rate, float(ci.sum()), h.levels())
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0                    # max over ranks
    assert abs(res[0][1] - world * 4 / 0.015) < 1e-9          # total solves/s of the job
    assert res[0][2] == res[1][2] and res[0][3] == res[1][3]  # replicas are deterministic
