"""GPU test of the slab-decomposed solve's local steps (chz_slab_forward,
chz_slab_z, chz_slab_inverse through cuhelmholtz_b200.slab.GpuExecutor).

All ranks' slabs are held by this one process and the exchanges are copies
(slab.solve_local): every rank's kernels run one after another on one GPU,
with no kernel waiting on another rank.  The result must equal the
single-GPU solve (chz_helmholtz_solve) on the whole grid to 1e-12, for
partitions of 2 to 4 slabs, including the N = 512 x passes and the
TMA-pipelined z pass on the pencils (N = 256, 512)."""
import numpy as np
import pytest
import torch

from cuhelmholtz_b200 import api
from cuhelmholtz_b200.slab import GpuExecutor, SlabLayout, solve_local
from oracle import gen
from oracle.stencil import FACE_KEYS

pytestmark = pytest.mark.gpu

CASES = [((24, 20, 28), (3, 4, 0), -1.0, 2), ((32, 24, 40), (1, 2, 1), -2.5, 3),
         ((40, 16, 32), (0, 0, 2), -0.7, 4), ((48, 40, 64), (2, 3, 4), -4.0, 3), ((32, 32, 32), (0, 3, 3), 0.0, 2),
         ((512, 24, 256), (3, 4, 0), -1.0, 4), ((64, 48, 512), (1, 0, 0), -3.0, 2),
         ((128, 128, 128), (1, 3, 0), -4.0, 4)]


@pytest.mark.parametrize("dims,codes,lam,world", CASES)
def test_slab_local_steps_match_single_gpu_solve(dims, codes, lam, world):
    p = gen.random_problem(*dims, *codes, lam, seed=sum(dims) + world)
    faces = {k: (None if p.get(k) is None else torch.from_numpy(np.ascontiguousarray(p[k]).ravel()).cuda())
             for k in FACE_KEYS}
    f_all = torch.from_numpy(np.ascontiguousarray(p["f"]).ravel()).cuda()
    ref = f_all.clone()
    api.solve_problem(p, ref, faces)

    L = SlabLayout(*dims, codes, world)
    plane = (dims[0] + 1) * (dims[1] + 1)
    slabs = [f_all[z0 * plane:(z0 + n) * plane].clone() for z0, n in L.planes]
    solve_local(L, GpuExecutor(L, p["dom"], lam, faces), slabs)
    api.stream_status()
    got = torch.cat(slabs)
    err = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
    assert err < 1e-12, err


def test_slab_rejects_a_dirichlet_face_split_from_its_plane():
    """With a Dirichlet z face, the slab holding the first unknown plane must
    hold plane 0 (the boundary terms read it)."""
    L = SlabLayout(16, 16, 16, (1, 1, 1), 2, planes=[(0, 2), (2, 15)])
    ws = torch.zeros(18 * 18 * 16, dtype=torch.float64, device="cuda")
    f = torch.zeros(17 * 17 * 16, dtype=torch.float64, device="cuda")
    from cuhelmholtz_b200 import _lib
    st = _lib.lib().chz_slab_forward(0.0, 1.0, 16, 1, 0, 0, 0.0, 1.0, 16, 1, 0, 0, 0.0, 1.0, 16, 1, 0, 0,
                                     f.data_ptr(), 1, 16, ws.data_ptr(), None)
    assert st == api.CHZ_ERROR_INVALID_VALUE
    assert L.planes[0] == (0, 2)
