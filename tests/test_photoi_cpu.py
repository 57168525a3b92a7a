"""Photoionization without a GPU: the oracle's generator, photon tables and
Monte Carlo source against independent restatements and the reference's own
known-answer case (src/test_m_photons.f90), and the library's host-side
photon table against the oracle's."""
import math

import numpy as np
import pytest

import a5ref
from a5_streamer_b200 import config, device

M = 2147483579
DEFAULT_SEED = (521288629, 362436069, 16163801, 1131199299)


def _wrap(v):
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v >= 1 << 31 else v


def mzran(state, n):
    """RNG_t%int4 (fosito/m_random.f90:58-66) with Python integers and
    explicit two's complement wrap-around."""
    s = list(state)
    out = []
    for _ in range(n):
        rr = _wrap(s[0] - s[2])
        if rr < 0:
            rr = _wrap(rr + M)
        s[0], s[1], s[2] = s[1], s[2], rr
        s[3] = _wrap(69069 * s[3] + 1013904243)
        out.append(_wrap(rr + s[3]))
    return out, s


@pytest.mark.parametrize("seed", [DEFAULT_SEED, (-2000000000, 2100000000, 1999999999, -5),
                                  (2147483647, -2147483648, 7, 0)])
def test_mzran_matches_restatement(seed):
    ref, _ = mzran(seed, 200)
    assert list(a5ref.kat_rng(seed, 200)) == ref


def test_uni01_range_and_mean():
    draws = a5ref.kat_rng(DEFAULT_SEED, 200000).astype(np.float64)
    u = 0.5 + draws * 2.0 ** -32
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 5e-3


def _jump(state, k):
    """k draws at once: (s1, s2, s3) -> M^k (s1, s2, s3) mod m and the affine
    map of s4 composed k times; valid while s1..s3 lie in [0, m)."""
    def mat_mul(a, b):
        return [[sum(a[i][t] * b[t][j] for t in range(3)) % M for j in range(3)] for i in range(3)]
    P = [[1, 0, 0], [0, 1, 0], [0, 0, 1]]
    B = [[0, 1, 0], [0, 0, 1], [1, 0, M - 1]]
    a, c = 1, 0
    ab, cb = 69069, 1013904243
    kk = k
    while kk:
        if kk & 1:
            P = mat_mul(B, P)
            a, c = (ab * a) & 0xFFFFFFFF, (ab * c + cb) & 0xFFFFFFFF
        B = mat_mul(B, B)
        ab, cb = (ab * ab) & 0xFFFFFFFF, (ab * cb + cb) & 0xFFFFFFFF
        kk >>= 1
    v = [x % (1 << 32) for x in state[:3]]
    n = [sum(P[i][j] * v[j] for j in range(3)) % M for i in range(3)]
    s4 = (a * (state[3] & 0xFFFFFFFF) + c) & 0xFFFFFFFF
    return [_wrap(n[0]), _wrap(n[1]), _wrap(n[2]), _wrap(s4)]


@pytest.mark.parametrize("k", [1, 2, 3, 7, 64, 1000, 4 * 37888 + 12])
def test_master_jump_equals_sequential_draws(k):
    """The device seeds team generators by jumping the master generator;
    the jump (a linear map mod m while the state is in [0, m)) equals k
    sequential draws."""
    _, s_seq = mzran(DEFAULT_SEED, k)
    assert _jump(list(DEFAULT_SEED), k) == s_seq


@pytest.mark.parametrize("kind,a,b,max_dist", [("air", 0.2, 0.0, 10e-3),
                                               ("logu", 0.2e-3, 2e-3, 32e-3),
                                               ("air", 0.04, 0.0, 64e-3)])
def test_host_photon_table_matches_oracle(kind, a, b, max_dist):
    cfg = config.cylindrical_16mm(photoi=True, photoi_table=(kind, a, b),
                                  domain_len=(max_dist / 4, max_dist / 2))
    d_host, f_host = device.photon_table(cfg)
    d_ref, f_ref = a5ref.kat_photon_table(kind, a, b, max_dist)
    assert len(d_host) == 500
    assert np.array_equal(d_host, d_ref) and f_host == f_ref
    assert d_host[0] == 0.0 and np.all(np.diff(d_host) >= 0) and d_host[-1] <= max_dist


def _truncated_mean(k0, k1, dmax):
    """Mean of the absorption distance for a coefficient log-uniform on
    [k0, k1], truncated at dmax (numerical quadrature)."""
    from scipy.integrate import quad
    f = lambda d: (math.exp(-k0 * d) - math.exp(-k1 * d)) / (d * math.log(k1 / k0)) if d > 0 \
        else (k1 - k0) / math.log(k1 / k0)
    num = quad(lambda d: d * f(d), 0, dmax, limit=400, points=[1 / k1, 1 / k0])[0]
    den = quad(f, 0, dmax, limit=400, points=[1 / k1, 1 / k0])[0]
    return num / den


def test_photon_mean_distance_known_answer():
    """src/test_m_photons.f90: photons absorbed from the origin in air at
    p_O2 = 0.2 bar over a 10 mm table; the mean absorption distance matches
    the absorption function's own mean up to the table's last distance (the
    table ends at the last integration point inside 10 mm)."""
    torr = float(np.float32(133.322368)) * 1e-5
    k0, k1 = 3.5 / torr * 0.2, 200 / torr * 0.2
    d, _ = a5ref.kat_photon_table("air", 0.2, 0.0, 10e-3)
    expect = _truncated_mean(k0, k1, d[-1])
    got = a5ref.kat_photon_dist(0.2, 10e-3, 400000, 8)
    assert abs(got / expect - 1) < 0.01, (got, expect)


def _cyl_photoi(team, **kw):
    cfg = config.cylindrical_16mm(photoi=True, photoi_team=team, **kw)
    sim = a5ref.Sim(cfg, n_threads=4)
    sim.init()
    return cfg, sim


def _absorbed_content(sim, cfg):
    """Sum over leaf cells (levels >= 1) of the source times the cell volume
    2 pi r dr^2: frac_in_tbl / fac per photon absorbed in the domain."""
    geom, pho = sim.geom(), sim.cc(a5ref.I_PHO)
    nc, g = cfg.box_size, cfg.box_size + 2
    total = 0.0
    for lvl, (_, leaves, _) in sim.levels().items():
        if lvl < 1:
            continue
        for i in leaves:
            dr = geom[i, 3]
            r = geom[i, 0] + (np.arange(1, nc + 1) - 0.5) * dr
            v = pho[i].reshape(g, g)[1:nc + 1, 1:nc + 1]
            total += float((v * (2 * np.pi * r[None, :] * dr * dr)).sum())
    return total


def test_photoionization_content_independent_of_team():
    """The absorbed photon content agrees between an execution with one
    thread and one with 64 (different Monte Carlo realisations, same tree)."""
    cfg, sim = _cyl_photoi(64)
    cfg1, sim1 = _cyl_photoi(1)
    t64, t1 = _absorbed_content(sim, cfg), _absorbed_content(sim1, cfg1)
    assert t64 > 0
    assert abs(t1 / t64 - 1) < 0.02, (t1, t64)
    assert np.array_equal(sim.meta(), sim1.meta())


def test_photoionization_team_changes_realisation_not_statistics():
    _, s1 = _cyl_photoi(16)
    _, s2 = _cyl_photoi(512)
    a, b = s1.cc(a5ref.I_PHO), s2.cc(a5ref.I_PHO)
    assert not np.array_equal(a, b)
    assert abs(a.sum() / b.sum() - 1) < 0.05


def test_rng_advances_by_eight_team_draws():
    team = 37
    cfg, sim = _cyl_photoi(team)
    # init made one call: the master gave 4 * team draws to each of the two teams
    _, s = mzran(DEFAULT_SEED, 8 * team)
    assert list(sim.rng_state()) == s
    sim.photoionization(1e-12)
    _, s = mzran(DEFAULT_SEED, 16 * team)
    assert list(sim.rng_state()) == s


def test_photoi_config_validation():
    with pytest.raises(ValueError):
        config.cartesian_8mm(photoi_enabled=True).validate()
    with pytest.raises(ValueError):
        config.cylindrical_16mm(photoi=True, photoi_table=("logu", 2e-3, 1e-3)).validate()
    config.cylindrical_16mm(photoi=True).validate()
    c = config.photoi_coeff_air(0.05, 1.0)
    assert 0.0019 < c < 0.0020
