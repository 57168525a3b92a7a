"""The device adjoint (include/a5a.h) of the head observable on the 8 mm
mesh, 200 steps, checkpoints every 20 steps: the program equals the oracle's,
and its gradient with respect to (mu, D, A, B, E_bg) matches the oracle's
tangent-linear run and central finite differences (h = 1e-6 relative) of the
device program, within 1e-3 relative."""
import numpy as np
import pytest
import torch

import a5ref
from a5_streamer_b200 import adjoint, streamer
from adjoint_harness import head_z

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    prob = adjoint.HeadProblem()
    cfg = prob.config()
    sim = streamer.Simulation(cfg)
    sim.init()
    adj = adjoint.HeadAdjoint(sim, prob)
    dts, T = adj.schedule()
    adj.bind()
    p0 = prob.nominal()
    ref = a5ref.Sim(cfg, n_threads=16)
    ref.init()
    yield prob, cfg, sim, adj, dts, T, p0, ref
    adj.close()


def test_schedule_and_program_match_the_oracle(problem):
    prob, cfg, sim, adj, dts, T, p0, ref = problem
    # the oracle's program on the same mesh and schedule
    assert np.array_equal(ref.meta(), sim.tree.export()[0])
    ref.set_init_cond()
    ref.op("compute_fld", 1)
    odts = []
    while len(odts) < prob.n_steps:
        dt = ref.get_max_dt()
        for _ in range(cfg.num_steps_amr):
            ref.step(dt)
            odts.append(dt)
    assert np.array_equal(np.array(odts[:prob.n_steps]), dts)
    J_dev = adj.value(p0)
    J_ref = ref.program(dts, prob.x0, T)
    assert J_dev == J_ref


def test_gradient_matches_the_oracle_tangent(problem):
    prob, cfg, sim, adj, dts, T, p0, ref = problem
    J, g = adj.gradient(p0)
    d, dV = adjoint.param_tangents(p0, cfg.domain_len_z, cfg.lkptbl_size, cfg.lkptbl_max_fld)
    J_ref, g_ref = ref.tl_program(dts, prob.x0, T, d, dV)
    assert J == J_ref
    np.testing.assert_allclose(g, g_ref, rtol=1e-6, atol=0)


def test_gradient_matches_central_differences(problem):
    prob, cfg, sim, adj, dts, T, p0, ref = problem
    _, g = adj.gradient(p0)
    h = 1e-6
    fd = np.zeros(5)
    for k in range(5):
        Jpm = []
        for sg in (1.0, -1.0):
            p = p0.copy()
            p[k] *= 1 + sg * h
            Jpm.append(adj.value(p))
        fd[k] = (Jpm[0] - Jpm[1]) / (2 * h * p0[k])
    adj.set_params(p0)
    np.testing.assert_allclose(g, fd, rtol=1e-3, atol=0)


def test_checkpoint_interval_does_not_change_the_gradient(problem):
    prob, cfg, sim, adj, dts, T, p0, ref = problem
    _, g20 = adj.gradient(p0)
    one = adjoint.HeadAdjoint(sim, adjoint.HeadProblem(checkpoint_every=prob.n_steps))
    one.bind(dts, T)
    try:
        _, g200 = one.gradient(p0)
    finally:
        one.close()
    np.testing.assert_allclose(g20, g200, rtol=1e-10, atol=0)


def test_autograd_function_in_the_harness(problem):
    prob, cfg, sim, adj, dts, T, p0, ref = problem
    x = torch.zeros(5, dtype=torch.float64, requires_grad=True)
    J = head_z(x, adj, p0)
    J.backward()
    _, g = adj.gradient(p0)
    np.testing.assert_allclose(x.grad.numpy(), g * p0, rtol=1e-12)
    # torch's own finite-difference check of the Function (eps = 1e-6 relative)
    ok = torch.autograd.gradcheck(lambda t: head_z(t, adj, p0), (x,), eps=1e-6, atol=1e-12,
                                  rtol=1e-3, nondet_tol=1e-9)
    assert ok


def test_rejects_unsupported_runs():
    from a5_streamer_b200 import config
    from a5_streamer_b200._lib import A5GError
    sim = streamer.Simulation(config.cylindrical_16mm())
    sim.init()
    adj = adjoint.HeadAdjoint(sim, adjoint.HeadProblem(n_steps=2))
    with pytest.raises(A5GError):
        adj.bind(np.array([1e-12, 1e-12]), 1.0)
