"""The sharded step as separate processes: two ranks, each its own process with its own CUDA
context, exchanging halo points through a gloo process group (host-staged buffers, every wait on
the host), against the unsharded batched step, bit for bit.

Both processes use the one GPU a test box has: no kernel of one rank waits on the other's (the
all-to-all between the fill phases is on the host), so the two contexts may be scheduled in any
order. With NCCL between GPUs the same ShardedGHProblem.step runs the exchange on the device.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    f = tgh.hole_forest(c, 8, 2, [3.0, 1.8, 1.4], path=((0.0, 0.0, 0.0), (0.05, 0.0, 0.0)))
    return c, f, 0.3


def _worker(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(HERE))
    from conftest import load_package
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    tgh = load_package()
    case, forest, t = _case(tgh)
    dt = 0.25 * (forest.h0 / 2 ** int(forest.level.max())) / 2.0
    S = tgh.ShardedGHProblem(case, forest, 4, rank, world, margin_check=False)
    u = S.initial_state(S.statevector(), t)
    u += S.local(torch.from_numpy(tgh.perturbation(forest, amplitude=1e-6, seed=5)).cuda())
    S.step(u, t, dt, nsteps=2)
    torch.cuda.synchronize()
    np.save(Path(out_dir) / f"rank{rank}.npy", u.cpu().numpy())
    np.save(Path(out_dir) / f"leaves{rank}.npy", S.leaves)
    dist.barrier()
    S.close()
    dist.destroy_process_group()


def test_two_processes_over_gloo_equal_the_unsharded_step(tgh, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    case, forest, t = _case(tgh)
    dt = 0.25 * (forest.h0 / 2 ** int(forest.level.max())) / 2.0
    P = tgh.GHProblem(case, forest, 4, margin_check=False)
    u = P.initial_state(P.statevector(), t)
    u += torch.from_numpy(tgh.perturbation(forest, amplitude=1e-6, seed=5)).cuda()
    P.step_batched(u, t, dt, 2)
    ref = u.cpu().numpy().reshape(forest.nblocks, -1)
    covered = np.zeros(forest.nblocks, dtype=bool)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        leaves = np.load(tmp_path / f"leaves{r}.npy")
        assert len(leaves) > 0
        assert np.array_equal(got.reshape(len(leaves), -1), ref[leaves]), f"rank {r} differs"
        covered[leaves] = True
    assert covered.all()
    P.close()
