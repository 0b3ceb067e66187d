"""The sharded step's host logic without a GPU: the partition (per level, Morton order, even
runs: TreeAMR's block distribution, src/distributed.jl:1-22), and the exchange lists of every
fill phase, exchanged for real between two gloo ranks.

Each rank sends, for every point of its send list, the point's (leaf, work index) encoded as
one double; the receiver checks that what arrives is, in order, the list it expects. That
holds only if the two ranks derive the same lists independently, which the step relies on
(no host communication precedes it).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package


def _forests(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, halfwidth=4.0, r0=0.8, r1=1.3, gauge="algebraic")
    hier = tgh.hole_forest(c, 8, 2, [3.0, 1.8, 1.4], path=((0.0, 0.0, 0.0), (0.05, 0.0, 0.0)))
    g = tgh.gauge_wave_case(eps_ko=0.5, gamma0=1.0, gamma2=-0.5)
    return [("hierarchy", c, hier), ("periodic", g, tgh.gh_forest(g, 8, 3))]


def _morton(b):
    code = 0
    for bit in range(21):
        for d in range(3):
            code |= ((int(b[d]) >> bit) & 1) << (3 * bit + d)
    return code


def test_partition_spreads_every_level_in_morton_order(tgh):
    for name, case, f in _forests(tgh):
        for R in (1, 2, 3, 4):
            owner = tgh.partition(f, R)
            assert owner.min() >= 0 and owner.max() < R
            for l in np.unique(f.level):
                idx = np.nonzero(f.level == l)[0]
                cnt = np.bincount(owner[idx], minlength=R)
                assert cnt.max() - cnt.min() <= 1, (name, R, l, cnt)
                order = sorted(idx, key=lambda b: _morton(f.corner[b] // f.N))
                assert np.all(np.diff(owner[order]) >= 0), (name, R, l)


def test_one_rank_exchanges_nothing(tgh):
    for name, case, f in _forests(tgh):
        owner = tgh.partition(f, 1)
        for ph in range(int(f.level.max()) + 1):
            plan = tgh.exchange_plan(case, f, 4, owner, 0, 1, ph)
            assert plan["send"].size == 0 and plan["recv"].size == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _exchange_worker(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tgh = load_package()
        for name, case, f in _forests(tgh):
            q = 4
            G = q // 2 + 1
            Wd = f.N + 2 * G + 1
            owner = tgh.partition(f, world)
            total = 0
            for ph in range(int(f.level.max()) + 1):
                plan = tgh.exchange_plan(case, f, q, owner, rank, world, ph)
                snd, rcv = plan["send"], plan["recv"]
                assert np.all(owner[snd[:, 0]] == rank), "a rank sends only its own leaves' points"
                assert np.all(owner[rcv[:, 0]] != rank), "a rank receives only other ranks' points"
                i, j, k = snd[:, 1] % Wd, (snd[:, 1] // Wd) % Wd, snd[:, 1] // (Wd * Wd)
                if ph == 0:
                    # copies read owned points only
                    for a in (i, j, k):
                        assert np.all((a >= G) & (a <= G + f.N))
                else:
                    # level ph's prolongation reads level ph - 1
                    assert np.all(f.level[snd[:, 0]] == ph - 1)
                    assert np.all(f.level[rcv[:, 0]] == ph - 1)
                enc = lambda e: torch.from_numpy(e[:, 0].astype(np.float64) * 2.0 ** 20 + e[:, 1])  # noqa: E731
                recv = torch.zeros(len(rcv), dtype=torch.float64)
                dist.all_to_all_single(recv, enc(snd), output_split_sizes=[int(c) for c in plan["recv_count"]],
                                       input_split_sizes=[int(c) for c in plan["send_count"]])
                assert torch.equal(recv, enc(rcv)), (name, ph)
                total += len(rcv)
            # the hierarchy's fill reads from the other rank in every phase
            if name == "hierarchy":
                assert total > 0
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_exchange_lists_agree_across_two_gloo_ranks():
    mp.spawn(_exchange_worker, args=(2, _free_port()), nprocs=2, join=True)
