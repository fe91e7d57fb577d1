"""k-point distribution and the IBS-force reduction across processes (CPU, gloo).

* the block rule against the examples documented with the reference's
  nofset / firstofset / lastofset (src/src_mpi/modmpi.F90:272-463);
* world_size 2: each rank computes the oracle's IBS force for its own
  k-points, the all-reduce (force.f90:170) must equal the serial sum.
"""
import os
import socket

import numpy as np
import pytest

from exciting_b200.kdist import firstofset, lastofset, my_kpoints, nofset


def test_documented_examples():
    assert [nofset(p, 10, 3) for p in range(3)] == [4, 3, 3]
    assert [firstofset(p, 10, 3) for p in range(3)] == [1, 5, 8]
    assert [lastofset(p, 10, 3) for p in range(3)] == [4, 7, 10]
    assert [nofset(p, 2, 3) for p in range(3)] == [1, 1, 0]
    assert [firstofset(p, 2, 4) for p in range(4)] == [1, 2, 0, 0]
    assert [lastofset(p, 2, 4) for p in range(4)] == [1, 2, -1, -1]


@pytest.mark.parametrize("n,p", [(8, 2), (27, 4), (27, 8), (3, 8), (0, 2)])
def test_blocks_cover_each_kpoint_once(n, p):
    got = sorted(k for r in range(p) for k in my_kpoints(r, n, p))
    assert got == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import torch.distributed as dist
    from datetime import timedelta

    import lapw_oracle as O
    from exciting_b200 import workloads as W
    from exciting_b200.kdist import allreduce_forces, my_kpoints

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    s = W.si_fcc("shipped")
    f = np.zeros((3, s.natmtot), order="F")
    for ik in my_kpoints(rank, len(s.kpoints), world):
        gk = s.gkset(s.kpoints[ik])
        nmat = s.nmat(gk)
        rng = np.random.default_rng(100 + ik)
        c, _ = np.linalg.qr(rng.standard_normal((nmat, 6)) + 1j * rng.standard_normal((nmat, 6)))
        f += O.forcek(s, gk, c, rng.uniform(-0.5, 0.5, 6), np.full(6, 2.0), W.FCC_IRREDUCIBLE_4x4x4_WEIGHTS[ik])
    tot = allreduce_forces(f)
    np.save(os.path.join(out, f"rank{rank}.npy"), tot)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_force_reduction(tmp_path):
    import torch.multiprocessing as mp

    import lapw_oracle as O
    from exciting_b200 import workloads as W

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    s = W.si_fcc("shipped")
    ref = np.zeros((3, s.natmtot))
    for ik in range(len(s.kpoints)):
        gk = s.gkset(s.kpoints[ik])
        nmat = s.nmat(gk)
        rng = np.random.default_rng(100 + ik)
        c, _ = np.linalg.qr(rng.standard_normal((nmat, 6)) + 1j * rng.standard_normal((nmat, 6)))
        ref += O.forcek(s, gk, c, rng.uniform(-0.5, 0.5, 6), np.full(6, 2.0), W.FCC_IRREDUCIBLE_4x4x4_WEIGHTS[ik])
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-14)
