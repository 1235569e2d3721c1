"""Run-to-run reproducibility of the 3D projector pair on the GPU.

The transpose kernels gather each voxel's sum in one lane, in a fixed order
of views and cells, so repeated transposes are bit-identical.  The direct
kernels accumulate detector cells in shared memory from whichever warp
reaches a band row first (row locks or shared atomics), so the FP32
summation order of a cell changes from run to run: repeated direct
projections differ by FP32 rounding only, far below the 1e-5 parity bound
against the FP64 reference.  Both the group kernels (views related by
quarter turns) and the per-view kernels are checked."""

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import geometry as G, phantoms as P

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-6  # relative L2 between two direct projections of the same input


@pytest.mark.parametrize("symmetry", [2, 0])
def test_pair_run_to_run(symmetry):
    import torch
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz
    sc = G.circular_scan_3d(64, 64, 64, 1.0, 3, 96, 96, 1.0, 1.0, 16, rsc=200.0, rsd=300.0)
    vol = P.ellipsoids_3d(64, 64, 64, n=12, seed=11, dtype=np.float32) + np.float32(0.05)
    pr = Projector3D(sc)
    pr.set_symmetry(symmetry)
    if symmetry:
        assert pr.groups()[2] == 4  # 16 views: 4 quarter-turn quads
    x = columns_from_xyz(torch.tensor(vol, device="cuda"))
    fw = [pr.forward(x, layout="columns").double().cpu().numpy() for _ in range(3)]
    for a in fw[1:]:
        assert rel_l2(a, fw[0]) <= RUN_TOL
    y = torch.tensor(np.random.default_rng(2).random(pr.detector_shape()), dtype=torch.float32,
                     device="cuda")
    bk = [pr.backward(y, layout="columns").cpu().numpy() for _ in range(2)]
    assert np.array_equal(bk[0], bk[1])
    pr.close()
