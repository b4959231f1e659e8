"""CPU tests of the slab-decomposed solve (cuhelmholtz_b200.slab): the
partition, and the two all-to-all exchanges across real processes (gloo,
world sizes 2 and 3) with the local steps restated on the host
(oracle.slab.OracleExecutor).  The distributed result must equal the oracle's
whole-grid restatement of the reference solver to 1e-12."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cuhelmholtz_b200.slab import SlabLayout, solve_local, solve_distributed
from oracle import emulation as E
from oracle import gen
from oracle.slab import OracleExecutor
from oracle.stencil import FACE_KEYS

CASES = [((12, 10, 16), (3, 4, 0), -1.0), ((8, 12, 10), (1, 2, 1), -2.5), ((10, 8, 12), (0, 0, 2), -0.7),
         ((14, 6, 14), (2, 3, 4), -4.0), ((8, 8, 8), (0, 3, 3), 0.0)]


def _oracle_whole(p):
    d = p["dom"]
    return E.emulate_solver(d[0], d[1], p["nx"], p["xbc"], p["bcl"], p["bcr"], d[2], d[3], p["ny"], p["ybc"],
                            p["bcb"], p["bct"], d[4], d[5], p["nz"], p["zbc"], p["bcf"], p["bce"], p["lam"], p["f"])


def _slabs(p, layout):
    f = np.ascontiguousarray(p["f"])
    return [torch.from_numpy(f[z0:z0 + n].copy().ravel()) for z0, n in layout.planes]


def test_layout_partition():
    L = SlabLayout(64, 48, 40, (1, 3, 0), 4)
    assert L.planes[0][0] == 0 and sum(n for _, n in L.planes) == 41
    assert all(n >= 2 for _, n in L.planes)
    assert L.rows[0][0] == 0 and sum(n for _, n in L.rows) == 49       # y code 3: rows 0..48
    assert sum(L.nwin(r) for r in range(4)) == L.zcount == 40           # z periodic: planes 0..39
    for r in range(4):
        assert sum(L.send_splits_forward(r)) == L.nwin(r) * 49 * 66
    # what r sends to q is what q receives from r
    for r in range(4):
        for q in range(4):
            assert L.send_splits_forward(r)[q] == L.recv_splits_forward(q)[r]
    with pytest.raises(ValueError):
        SlabLayout(8, 8, 4, (1, 1, 1), 3)                               # 5 planes, 3 ranks
    with pytest.raises(ValueError):
        SlabLayout(8, 8, 16, (1, 1, 1), 2, planes=[(0, 1), (1, 16)])     # a one-plane slab


@pytest.mark.parametrize("dims,codes,lam", CASES)
@pytest.mark.parametrize("world", [2, 3])
def test_local_form_matches_whole_grid(dims, codes, lam, world):
    p = gen.random_problem(*dims, *codes, lam, seed=sum(dims) + world)
    L = SlabLayout(*dims, codes, world)
    ex = OracleExecutor(L, p["dom"], lam, {k: p.get(k) for k in FACE_KEYS})
    slabs = _slabs(p, L)
    solve_local(L, ex, slabs)
    got = np.concatenate([s.numpy() for s in slabs]).reshape(p["f"].shape)
    ref = _oracle_whole(p)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, dims, codes, lam, seed, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = gen.random_problem(*dims, *codes, lam, seed=seed)
        L = SlabLayout(*dims, codes, world)
        ex = OracleExecutor(L, p["dom"], lam, {k: p.get(k) for k in FACE_KEYS})
        z0, n = L.planes[rank]
        f_slab = torch.from_numpy(np.ascontiguousarray(p["f"])[z0:z0 + n].copy().ravel())
        solve_distributed(L, ex, f_slab)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), f_slab.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("dims,codes,lam", [CASES[0], CASES[1], CASES[3]])
def test_distributed_gloo_matches_whole_grid(tmp_path, world, dims, codes, lam):
    seed = 7 * sum(dims) + world
    mp.start_processes(_rank_main, args=(world, _free_port(), dims, codes, lam, seed, str(tmp_path)),
                       nprocs=world, start_method="spawn", join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(world)])
    p = gen.random_problem(*dims, *codes, lam, seed=seed)
    ref = _oracle_whole(p)
    got = got.reshape(ref.shape)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12
