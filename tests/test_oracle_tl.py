"""The oracle's tangent-linear run of the fixed-mesh program (the
differentiation check's CPU reference) against central finite differences of
the oracle's own program, on a short horizon."""
import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import adjoint


@pytest.fixture(scope="module")
def setup():
    prob = adjoint.HeadProblem()
    cfg = prob.config()
    s = a5ref.Sim(cfg, n_threads=4)
    s.init()
    p0 = prob.nominal()
    tab, _, _ = s.table()
    # the table built from the configuration's pairs is the one the
    # parameters give
    assert np.array_equal(tab, adjoint.table_rows(p0, cfg.lkptbl_size, cfg.lkptbl_max_fld))
    n = 12
    s.set_init_cond()
    s.op("compute_fld", 1)
    dts = []
    while len(dts) < n:
        dt = s.get_max_dt()
        for _ in range(cfg.num_steps_amr):
            s.step(dt)
            dts.append(dt)
    dts = np.array(dts[:n])
    T = adjoint.head_temperature(s.head_profile(prob.x0), prob.tau)
    return s, cfg, prob, p0, dts, T


def test_program_is_the_step_sequence(setup):
    s, cfg, prob, p0, dts, T = setup
    J = s.program(dts, prob.x0, T)
    J2, _ = s.tl_program(dts, prob.x0, T, np.zeros((1, cfg.lkptbl_size, 4)), [0.0])
    assert J == J2
    assert 0 < J < cfg.domain_len_z


def test_tangent_matches_central_differences(setup):
    s, cfg, prob, p0, dts, T = setup
    d, dV = adjoint.param_tangents(p0, cfg.domain_len_z, cfg.lkptbl_size, cfg.lkptbl_max_fld)
    _, dJ = s.tl_program(dts, prob.x0, T, d, dV)
    h = 1e-6
    fd = np.zeros(5)
    for k in range(5):
        J = []
        for sg in (1.0, -1.0):
            p = p0.copy()
            p[k] *= 1 + sg * h
            s.set_table_rows(adjoint.table_rows(p, cfg.lkptbl_size, cfg.lkptbl_max_fld))
            s.set_applied_fld(p[4])
            J.append(s.program(dts, prob.x0, T))
        fd[k] = (J[0] - J[1]) / (2 * h * p0[k])
    s.set_table_rows(adjoint.table_rows(p0, cfg.lkptbl_size, cfg.lkptbl_max_fld))
    s.set_applied_fld(p0[4])
    # relative tolerance 1e-3 (the differentiation bar), per parameter
    np.testing.assert_allclose(dJ, fd, rtol=1e-3, atol=0)
