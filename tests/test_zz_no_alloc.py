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


def _walled_gravity():
    """3D SRD between plain (non-phantom) no-slip walls at y = 0 and y = L1,
    periodic x and z, gravity along x."""
    L = (6, 7, 5)
    walls = W.channel_walls(L)
    for w in walls:
        w.phantom = 0
    return W.base_config(3, L, coll_op=abi.COLL_ARBAXIS, walls=walls,
                         grav=(5e-3, 0.0, 0.0), seed=517)


@pytest.mark.parametrize("case", ["periodic3d", "periodic2d", "walls_gravity"])
def test_noalloc_step_matches_handle_step_twice(case):
    import torch

    if case == "periodic3d":
        cfg, L = W.cfg_srd3d((8, 8, 8), seed=515), (8, 8, 8)
    elif case == "periodic2d":
        cfg, L = W.base_config(2, (30, 30), coll_op=abi.COLL_ARBAXIS, seed=515), (30, 30)
    else:
        cfg = _walled_gravity()
        L = (6, 7, 5)
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=516)
    if case == "walls_gravity":
        Q[:, 1] = 0.02 + Q[:, 1] * (L[1] - 0.04) / L[1]  # off the walls' planes
    n = len(Q)
    ref = Solver(cfg)
    ref.upload(Q, V, U, sp)
    dq = torch.tensor(Q, dtype=torch.float64, device="cuda")
    dv = torch.tensor(V, dtype=torch.float64, device="cuda")
    glob = torch.zeros(4, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(3, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for step in (1, 2):
        kb, av = ref.timestep(step)
        qr, vr, _ = ref.download()
        gpu.srd_step_noalloc(cfg, n, dq.data_ptr(), dv.data_ptr(), step, glob.data_ptr(),
                             stream, cnt.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_allclose(dv.cpu().numpy(), vr, rtol=0, atol=TOL * 10)
        np.testing.assert_allclose(dq.cpu().numpy(), qr, rtol=0, atol=TOL * max(L))
        g = glob.cpu().numpy()
        assert g[0] == pytest.approx(kb, rel=1e-12)
        np.testing.assert_allclose(g[1:], av, rtol=0, atol=1e-13)
    st = ref.status()
    c = cnt.cpu().numpy()
    assert (c[0], c[1], c[2]) == (st.escaped, st.bounce_limit, st.nonfinite)
    ref.close()


def test_noalloc_reports_escapes_to_the_callers_counters():
    """A particle outside a walled box escapes binning (bin(), mpc.c:970-982);
    the count reaches the caller's counters, and accumulates over calls."""
    import torch

    cfg = _walled_gravity()
    Q, V, U, sp = W.synthetic_state(cfg, 10, seed=518)
    Q[:, 1] = 0.02 + Q[:, 1] * (7 - 0.04) / 7
    Q[5, 1] = 9.5  # above the top wall: outside the (L+1) grid whatever the shift
    Q[6, 1] = -2.5  # below the bottom wall: truncates below cell 0 whatever the shift
    n = len(Q)
    dq = torch.tensor(Q, dtype=torch.float64, device="cuda")
    dv = torch.tensor(V, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(3, dtype=torch.int64, device="cuda")
    ref = Solver(cfg)
    ref.set_kernel(abi.KERNEL_SPLIT)  # the kernels the allocation-free step runs
    ref.upload(Q, V, U, sp)
    ref.timestep(1)
    gpu.srd_step_noalloc(cfg, n, dq.data_ptr(), dv.data_ptr(), 1, None,
                         torch.cuda.current_stream().cuda_stream, cnt.data_ptr())
    torch.cuda.synchronize()
    first = cnt.cpu().numpy().copy()
    assert first[0] >= 1
    assert first[0] == ref.status().escaped
    gpu.srd_step_noalloc(cfg, n, dq.data_ptr(), dv.data_ptr(), 2, None,
                         torch.cuda.current_stream().cuda_stream, cnt.data_ptr())
    torch.cuda.synchronize()
    assert cnt.cpu().numpy()[0] >= first[0]
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


def test_noalloc_rejects_several_species():
    """The call carries no species ids, so a multi-species configuration
    would weigh every particle by the first species' mass: rejected."""
    import torch

    cfg = W.cfg_srd3d((6, 6, 6), species=[W._species(mass=1.0), W._species(mass=2.0)],
                      seed=2)
    dq = torch.zeros((10, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.MPCDError, match="-2"):
        gpu.srd_step_noalloc(cfg, 10, dq.data_ptr(), dq.data_ptr(), 1)
