"""The allocation-free SRD step (mpcd_srd_step_noalloc), for callers that
cannot allocate device memory when they step the fluid, against the regular
handle-based entry point on the same state and draws, over two calls in a
row.  Collected last so that a failure here stops a run only after every
other test has run; it also passes alone in a fresh process, since each call
clears the shared scratch it needs."""
import numpy as np
import pytest

from mpcd_b200 import abi, gpu
from mpcd_b200 import workloads as W
from mpcd_b200.gpu import Solver

pytestmark = pytest.mark.gpu

# same algorithm and draws; only the order of particles within a cell (and
# so of the FP64 sums) can differ
TOL = 1e-12


@pytest.mark.parametrize("dim,L", [(3, (8, 8, 8)), (2, (30, 30))])
def test_noalloc_step_matches_handle_step_twice(dim, L):
    import torch

    if dim == 3:
        cfg = W.cfg_srd3d(L, seed=515)
    else:
        cfg = W.base_config(2, L, coll_op=abi.COLL_ARBAXIS, seed=515)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=516)
    n = len(Q)
    ref = Solver(cfg)
    ref.upload(Q, V, U, sp)
    dq = torch.tensor(Q, dtype=torch.float64, device="cuda")
    dv = torch.tensor(V, dtype=torch.float64, device="cuda")
    glob = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for step in (1, 2):
        kb, av = ref.timestep(step)
        qr, vr, _ = ref.download()
        gpu.srd_step_noalloc(cfg, n, dq.data_ptr(), dv.data_ptr(), step, glob.data_ptr(),
                             stream)
        torch.cuda.synchronize()
        np.testing.assert_allclose(dv.cpu().numpy(), vr, rtol=0, atol=TOL * 10)
        np.testing.assert_allclose(dq.cpu().numpy(), qr, rtol=0, atol=TOL * max(L))
        g = glob.cpu().numpy()
        assert g[0] == pytest.approx(kb, rel=1e-12)
        np.testing.assert_allclose(g[1:], av, rtol=0, atol=1e-13)
    ref.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    cfg = W.cfg_srd3d((40, 40, 40), seed=1)  # 41^3 cells > the compiled maximum
    dq = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.MPCDError, match="-6"):
        gpu.srd_step_noalloc(cfg, 10, dq.data_ptr(), dq.data_ptr(), 1)
    cfg = W.cfg_srd3d((8, 8, 8), seed=1)
    with pytest.raises(gpu.MPCDError, match="-6"):
        gpu.srd_step_noalloc(cfg, 70000, dq.data_ptr(), dq.data_ptr(), 1)
