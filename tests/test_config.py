"""The reference's text configuration format (fosito/m_config.f90) and the
two workload presets."""
import math

import pytest

from a5_streamer_b200 import config

SAMPLE = """
 # The desired endtime in seconds of the simulation:
 end_time = 0.1500E-07
 box_size = 8
 domain_len = 0.3200E-01
 applied_fld = 0.2500E+07   # trailing comment
 bg_dens = 0.1000E+14
 seed_dens = 0.2000E+20
 seed_rel_r0 = 0.5000E+00 0.6000E+00
 seed_rel_r1 = 0.5000E+00 0.5000E+00
 seed_width = 0.2000E-03
 seed_falloff = 3
 dt_max = 0.1000E-09
 num_steps_amr = 2
 photoi_enabled = F
 lkptbl_size = 1000
"""


def test_parse_and_apply(tmp_path):
    p = tmp_path / "a.txt"
    p.write_text(SAMPLE)
    q = tmp_path / "b.txt"
    q.write_text("applied_fld = 3.0e6\nn_base = 1 1\n")
    cfg = config.load_cfg_files([str(p), str(q)], base=config.cartesian_8mm())
    assert cfg.end_time == 1.5e-8 and cfg.applied_fld == 3.0e6  # later file wins
    assert cfg.domain_len == (0.032, 0.032) and cfg.n_base == (1, 1)
    assert cfg.dr_base == 0.032 / 8
    assert len(cfg.seeds) == 1
    s = cfg.seeds[0]
    assert s.r0 == (0.016, 0.032 * 0.6) and s.r1 == (0.016, 0.016) and s.falloff == 3
    assert cfg.lkptbl_size == 1000 and not cfg.photoi_enabled
    cfg.validate()


def test_presets():
    c = config.cartesian_8mm()
    c.validate()
    assert c.dr_base == 2.5e-4 and c.dr_at(7) == 2.5e-4 / 64
    assert c.applied_voltage == -0.008 * 2.5e6
    assert c.n_cycle_base == 8 and c.crv_refine == 1.0
    assert math.isclose(c.seeds[0].width, math.sqrt(2) * 0.2e-3)
    y = config.cylindrical_16mm()
    y.validate()
    assert y.is_cyl and y.n_cycle_base == 4 and y.crv_refine == 0.0
    assert y.dr_base == 1e-3 and y.dr_at(10) < 2e-6
    xs = config.table_nodes(200, 3e7)
    assert xs[0] == 0.0 and xs[-1] == (199) * (1 / (199 / 3e7))


def test_validate_rejects():
    with pytest.raises(ValueError):
        config.cartesian_8mm(box_size=6).validate()
    with pytest.raises(ValueError):
        config.cartesian_8mm(domain_len=(8e-3, 9e-3)).validate()


def test_batch_runs_generator():
    """The uneven-run workload: seeded, deterministic, within its ranges."""
    a = config.batch_cylindrical_runs(n=64)
    b = config.batch_cylindrical_runs(n=64)
    assert len(a) == 64
    for x, y in zip(a, b):
        assert x == y
    for c in a:
        c.validate()
        z = c.domain_len[1]
        assert 4e-3 <= z <= 16e-3 and c.domain_len[0] == 0.5 * z
        assert 1.5e6 <= c.applied_fld <= 2.5e6
        assert 1e15 <= c.bg_dens <= 1e16
        assert c.dr_at(c.lvls_max) <= 4e-6 < c.dr_at(c.lvls_max - 1)
        assert c.end_time == 5e-9 and c.photoi_enabled and c.is_cyl
        assert c.seeds[0].r0 == (0.0, z - 1e-3)
        assert all(0 < v < 2147483579 for v in c.rng_seed[:3])
    assert len({c.rng_seed for c in a}) == 64
    assert len({round(c.domain_len[1], 9) for c in a}) == 64


def test_cta_mapping_deals_every_block_once():
    from a5_streamer_b200.autotune import cta_mapping
    for cells, total, power in (([100, 200, 50, 5000], 148, 1.0), ([100] * 64, 148, 0.0),
                                ([3000, 10, 10], 148, 0.5), ([5] * 200, 148, 1.0)):
        m = cta_mapping(cells, total, power)
        assert len(m) == len(cells) and min(m) >= 1
        assert sum(m) == max(total, len(cells))
    m = cta_mapping([100, 200, 50, 5000], 148, 1.0)
    assert m[3] == max(m) and m[2] == min(m)
