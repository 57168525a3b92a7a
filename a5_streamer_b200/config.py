"""Run configuration for the streamer time step.

Mirrors the reference's configuration surface (``ST_create_cfg`` in
src/m_streamer.f90:145-228, read by ``ST_read_cfg_files`` / ``ST_load_cfg``,
src/m_streamer.f90:364-417) plus the keys the 8 mm / cylindrical workloads need
that the reference driver does not have: a rectangular base grid of several
boxes, a finest level, and the dielectric-relaxation step limit.

The reference's text format is ``name = v1 v2 # comment``; several files are
applied in order and later ones override earlier ones
(fosito/m_config.f90:83-182). :func:`load_cfg_files` reads that format.
"""
from __future__ import annotations

import dataclasses
import math
import re
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

# Column order of the transport table (src/m_streamer.f90:37-41).
TD_COLUMNS = ("mobility", "diffusion", "alpha", "eta")

# Seed fall-off types (src/m_geom.f90:8-11).
FALLOFF = {"sigmoid": 1, "gaussian": 2, "smoothstep": 3, "step": 4}


def photoi_coeff_air(eta: float = 0.05, gas_pressure: float = 1.0) -> float:
    """Photons per ionization as the cylindrical driver sets it:
    photoi_eta * p_quench / (gas_pressure + p_quench) with p_quench = 30 Torr
    (src/streamer_cyl.f90:572-588; one Torr in bar as in
    fosito/m_units_constants.f90:44, a single-precision literal times 1e-5)."""
    import struct
    torr = struct.unpack("f", struct.pack("f", 133.322368))[0] * 1.0e-5
    p_quench = 30.0 * torr
    return eta * (p_quench / (gas_pressure + p_quench))


@dataclass
class Seed:
    r0: Tuple[float, ...]
    r1: Tuple[float, ...]
    dens: float
    width: float
    falloff: int = 2


@dataclass
class StreamerConfig:
    dim: int = 2
    coord: str = "xyz"                  # "xyz" or "cyl"
    box_size: int = 8
    n_base: Tuple[int, ...] = (4, 4)    # base boxes per direction
    domain_len: Tuple[float, ...] = (8e-3, 8e-3)
    lvls_max: int = 7
    applied_fld: float = 2.5e6
    epsilon_diel: float = 1.0
    bg_dens: float = 1e15
    seeds: List[Seed] = field(default_factory=list)
    dt_max: float = 1e-10
    num_steps_amr: int = 2
    end_time: float = 2e-9
    use_drt: bool = True
    lkptbl_size: int = 200
    lkptbl_max_fld: float = 3e7
    # transport input pairs per column: name -> (x list, y list)
    td: Dict[str, Tuple[List[float], List[float]]] = field(default_factory=dict)
    # photoionization (src/m_streamer.f90:196-203, src/streamer_cyl.f90:572-617)
    photoi_enabled: bool = False
    photoi_num_photons: int = 50 * 1000
    # photons per ionization; the reference uses photoi_eta * quench factor
    # (photoi_coeff_air below)
    photoi_coeff: float = photoi_coeff_air(0.05, 1.0)
    # ("air", O2 partial pressure in bar, 0) for PH_get_tbl_air, or
    # ("logu", shortest, longest absorption length in m)
    photoi_table: Tuple[str, float, float] = ("air", 0.2, 0.0)
    photoi_fac_dx: float = 0.25e-3
    # size of the OpenMP team whose execution of the photon loops is
    # reproduced: each thread draws from its own generator seeded from the
    # master (fosito/m_random.f90:44-55), loops split by the static schedule
    photoi_team: int = 148 * 256
    # master generator state ST_rng (fosito/m_random.f90:12-13 default)
    rng_seed: Tuple[int, int, int, int] = (521288629, 362436069, 16163801, 1131199299)
    # > 0: every box below this level is refined and the rest kept, instead
    # of the streamer's refinement criterion: a uniformly refined mesh, as
    # afivo/examples/multigrid/test_mg_benchmark_2d.f90:40-86 builds
    uniform_lvl: int = 0

    # --- derived quantities -------------------------------------------------
    @property
    def dr_base(self) -> float:
        return self.domain_len[0] / (self.n_base[0] * self.box_size)

    @property
    def domain_len_z(self) -> float:
        return self.domain_len[self.dim - 1]

    @property
    def is_cyl(self) -> bool:
        return self.coord == "cyl"

    @property
    def n_cycle_base(self) -> int:
        # src/streamer_2d.f90:43 (8) and src/streamer_cyl.f90:46 (4)
        return 4 if self.is_cyl else 8

    @property
    def ref_init_time(self) -> float:
        # src/streamer_2d.f90:200, src/streamer_cyl.f90:212, src/streamer_3d.f90
        if self.is_cyl:
            return 5.0e-9
        return 2.0e-9 if self.dim == 2 else 2.5e-9

    @property
    def crv_refine(self) -> float:
        # src/streamer_2d.f90:214 (1), src/streamer_cyl.f90:226 (0), 3D 0.1
        if self.is_cyl:
            return 0.0
        return 1.0 if self.dim == 2 else 0.1

    @property
    def applied_voltage(self) -> float:
        # src/m_streamer.f90:411: ST_applied_voltage = -ST_domain_len * fld
        return -self.domain_len_z * self.applied_fld

    @property
    def photoi_max_dist(self) -> float:
        # src/m_streamer.f90:329-330: table range 2 * ST_domain_len
        return 2 * self.domain_len_z

    def dr_at(self, lvl: int) -> float:
        return self.dr_base * 0.5 ** (lvl - 1)

    def validate(self) -> None:
        if self.dim not in (2, 3):
            raise ValueError("dim must be 2 or 3")
        if self.dim == 3:
            # the 3D octree form runs on uniformly refined octrees
            # (include/a5g3.h): Cartesian, eps = 1, no photoionization
            if self.coord != "xyz" or self.uniform_lvl < 1:
                raise ValueError("the 3D form needs coord 'xyz' and a uniform mesh (uniform_lvl >= 1)")
            if self.photoi_enabled or self.epsilon_diel != 1.0:
                raise ValueError("the 3D form has no photoionization and no dielectric")
        if self.coord not in ("xyz", "cyl"):
            raise ValueError(f"coord must be 'xyz' or 'cyl', got {self.coord!r}")
        nc = self.box_size
        if nc < 4 or nc & (nc - 1):
            raise ValueError("box_size must be a power of two >= 4")
        if len(self.n_base) != self.dim or len(self.domain_len) != self.dim:
            raise ValueError("n_base and domain_len need one entry per dimension")
        for d in range(1, self.dim):
            dy = self.domain_len[d] / (self.n_base[d] * nc)
            if abs(dy - self.dr_base) > 1e-12 * self.dr_base:
                raise ValueError("base cells must be square: domain_len / n_base must agree")
        if len(self.seeds) > 8:
            raise ValueError("at most 8 seeds")
        for name in TD_COLUMNS:
            if name not in self.td:
                raise ValueError(f"transport column {name!r} missing")
            x, y = self.td[name]
            if len(x) != len(y) or len(x) < 1 or len(x) > 4096:
                raise ValueError(f"transport column {name!r}: bad length")
        if not (1 <= self.lvls_max <= 30):
            raise ValueError("lvls_max must be in 1..30")
        if self.uniform_lvl < 0 or self.uniform_lvl > self.lvls_max:
            raise ValueError("uniform_lvl must be in 0..lvls_max")
        if self.photoi_enabled:
            if not self.is_cyl:
                raise ValueError("photoionization is built for the cylindrical form only "
                                 "(PH_set_src_2d with a constant absorption level)")
            kind = self.photoi_table[0]
            if kind not in ("air", "logu"):
                raise ValueError("photoi_table kind must be 'air' or 'logu'")
            if kind == "logu" and not (0 < self.photoi_table[1] < self.photoi_table[2]):
                raise ValueError("log-uniform absorption lengths need 0 < shortest < longest")
            if self.photoi_team < 1 or self.photoi_num_photons < 0:
                raise ValueError("photoi_team must be >= 1 and photoi_num_photons >= 0")


def table_nodes(n_rows: int, x_max: float, x_min: float = 0.0) -> List[float]:
    """The x grid of a lookup table: LT_get_xdata (fosito/m_lookup_table.f90:180-189)."""
    inv_dx = (n_rows - 1) / (x_max - x_min)
    dx = 1 / inv_dx
    return [x_min + (ix - 1) * dx for ix in range(1, n_rows + 1)]


def synthetic_transport(n_rows: int = 200, x_max: float = 3e7, mobility: float = 0.03,
                        diffusion: float = 0.1, alpha_a: float = 4.3e5,
                        alpha_b: float = 1.4e7, eta_a: float = 0.0,
                        eta_b: float = 4e6) -> Dict[str, Tuple[List[float], List[float]]]:
    """Synthetic transport pairs placed exactly on the table nodes, so that the
    table built from them holds the analytic values: mu, D constant,
    alpha = A exp(-B/|E|) (alpha(0) = 0), eta = a exp(-b/|E|)."""
    xs = table_nodes(n_rows, x_max)
    mu = [mobility] * n_rows
    dif = [diffusion] * n_rows
    alpha = [alpha_a * math.exp(-alpha_b / x) if x > 0 else 0.0 for x in xs]
    eta = [eta_a * math.exp(-eta_b / x) if (x > 0 and eta_a != 0.0) else 0.0 for x in xs]
    return {"mobility": (xs, mu), "diffusion": (xs, dif), "alpha": (xs, alpha),
            "eta": (xs, eta)}


def cartesian_8mm(**overrides) -> StreamerConfig:
    """2D Cartesian FP64 case: 8 mm x 8 mm, 4x4 base boxes of 8^2 cells,
    finest dx 3.906 um (level 7), E_bg = 2.5e6 V/m, background 1e15 m^-3,
    Gaussian seed 1e19 m^-3 with sigma 0.2 mm (GM_gaussian width sqrt(2) sigma)
    at (4, 7) mm, synthetic transport, no photoionization, t_end = 2 ns."""
    sigma = 0.2e-3
    cfg = StreamerConfig(
        dim=2, coord="xyz", box_size=8, n_base=(4, 4), domain_len=(8e-3, 8e-3),
        lvls_max=7, applied_fld=2.5e6, epsilon_diel=1.0, bg_dens=1e15,
        seeds=[Seed(r0=(4e-3, 7e-3), r1=(4e-3, 7e-3), dens=1e19,
                    width=math.sqrt(2.0) * sigma, falloff=2)],
        dt_max=1e-10, num_steps_amr=2, end_time=2e-9, use_drt=True,
        lkptbl_size=200, lkptbl_max_fld=3e7, td=synthetic_transport())
    return dataclasses.replace(cfg, **overrides)


def cartesian_uniform(level: int = 6, **overrides) -> StreamerConfig:
    """The 8 mm Cartesian case on a uniformly refined mesh of the given level
    (every box below it refined, as the multigrid benchmark
    afivo/examples/multigrid/test_mg_benchmark_2d.f90:40-86 builds its mesh):
    (32 * 2^(level-1))^2 leaf cells, e.g. 1,048,576 at level 6 (dx = 7.8 um)
    and 4,194,304 at level 7. A large tree for the grid-mode form. The finest
    allowed level is one above: a$D_adjust_refinement never builds the leaf
    list of level lvls_max (afivo/src/m_aX_core.f90:495-532), so boxes there
    would take no transport update."""
    return cartesian_8mm(lvls_max=level + 1, uniform_lvl=level, **overrides)


def cube_16mm_uniform(level: int = 5, **overrides) -> StreamerConfig:
    """The 3D case on a uniformly refined octree: a 16 mm cube of one base
    box (8^3 cells, base dx 2 mm) refined to the given level (dx = 2 mm /
    2^(level-1): 125 um and 2,097,152 leaf cells at level 5, 62.5 um and
    16,777,216 at level 6), E_bg = 2e6 V/m along z, background 1e15 m^-3, two
    Gaussian seeds of 1e19 m^-3 and sigma 0.3 mm at (8, 6.5, 14) mm and
    (8, 9.5, 14) mm, synthetic transport with attachment, no
    photoionization, t_end = 8 ns. The streamer's own refinement criterion
    would refine further near the seeds; on this mesh every level is
    complete."""
    sigma = 0.3e-3
    seeds = [Seed(r0=(8e-3, y, 14e-3), r1=(8e-3, y, 14e-3), dens=1e19, width=math.sqrt(2.0) * sigma,
                  falloff=2) for y in (6.5e-3, 9.5e-3)]
    cfg = StreamerConfig(
        dim=3, coord="xyz", box_size=8, n_base=(1, 1, 1), domain_len=(16e-3, 16e-3, 16e-3),
        lvls_max=level + 1, uniform_lvl=level, applied_fld=2.0e6, epsilon_diel=1.0, bg_dens=1e15,
        seeds=seeds, dt_max=1e-10, num_steps_amr=2, end_time=8e-9, use_drt=True,
        lkptbl_size=200, lkptbl_max_fld=3e7, td=synthetic_transport(eta_a=1.0e3, eta_b=4e6))
    return dataclasses.replace(cfg, **overrides)


def cylindrical_16mm(photoi: bool = False, **overrides) -> StreamerConfig:
    """Axisymmetric (r, z) FP64 case: R = 8 mm, Z = 16 mm (two base boxes
    stacked in z, base dx 1 mm), E_bg = 2e6 V/m, background 1e15 m^-3, seed
    1e19 m^-3 with sigma 0.1 mm on the axis at z = 15 mm, attachment
    eta = 1e3 exp(-4e6/|E|). With ``photoi=True``: Monte Carlo photoionization
    with 1e5 photons per step, absorption length log-uniform between 0.2 and
    2 mm, 0.06 photons per ionization."""
    sigma = 0.1e-3
    cfg = StreamerConfig(
        dim=2, coord="cyl", box_size=8, n_base=(1, 2), domain_len=(8e-3, 16e-3),
        lvls_max=10, applied_fld=2.0e6, epsilon_diel=1.0, bg_dens=1e15,
        seeds=[Seed(r0=(0.0, 15e-3), r1=(0.0, 15e-3), dens=1e19,
                    width=math.sqrt(2.0) * sigma, falloff=2)],
        dt_max=1e-10, num_steps_amr=2, end_time=10e-9, use_drt=True,
        lkptbl_size=200, lkptbl_max_fld=3e7,
        td=synthetic_transport(eta_a=1.0e3, eta_b=4e6),
        photoi_enabled=photoi, photoi_num_photons=100 * 1000, photoi_coeff=0.06,
        photoi_table=("logu", 0.2e-3, 2.0e-3))
    return dataclasses.replace(cfg, **overrides)


def batch_cylindrical_runs(n: int = 64, seed: int = 20261203, photoi: bool = True,
                           end_time: float = 5e-9, min_dx: float = 4e-6) -> List[StreamerConfig]:
    """Independent axisymmetric runs of uneven size for the batched form,
    drawn from ``numpy.random.default_rng(seed)`` in this order per run:
    background density log-uniform in [1e15, 1e16] m^-3, E_bg uniform in
    [1.5e6, 2.5e6] V/m, domain length Z uniform in [4, 16] mm, and the four
    words of the run's photon generator state. The radius is Z/2 (the aspect
    ratio of the 16 mm case), two base boxes stacked in z, the finest level
    the first with dx <= min_dx, the seed (1e19 m^-3, sigma 0.1 mm) on the
    axis 1 mm below the top, transport and photoionization as in the 16 mm
    case; each run to its own end time."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out: List[StreamerConfig] = []
    for _ in range(n):
        bg = float(10.0 ** rng.uniform(15.0, 16.0))
        ebg = float(rng.uniform(1.5e6, 2.5e6))
        z_len = float(rng.uniform(4e-3, 16e-3))
        st = rng.integers(1, 2147483579, size=3)
        s4 = int(rng.integers(-2 ** 31, 2 ** 31))
        r_len = 0.5 * z_len
        dr_base = r_len / 8
        lvls_max = 1 + max(0, math.ceil(math.log2(dr_base / min_dx) - 1e-12))
        sigma = 0.1e-3
        cfg = cylindrical_16mm(
            photoi=photoi, domain_len=(r_len, z_len), applied_fld=ebg, bg_dens=bg,
            lvls_max=lvls_max, end_time=end_time,
            seeds=[Seed(r0=(0.0, z_len - 1e-3), r1=(0.0, z_len - 1e-3), dens=1e19,
                        width=math.sqrt(2.0) * sigma, falloff=2)],
            rng_seed=(int(st[0]), int(st[1]), int(st[2]), s4))
        out.append(cfg)
    return out


# --- the reference's text configuration format -------------------------------
_LINE = re.compile(r"^\s*([A-Za-z_][A-Za-z0-9_]*)\s*=\s*(.*?)\s*$")


def parse_cfg_text(text: str) -> Dict[str, List[str]]:
    """Parse ``name = v1 v2 ...  # comment`` lines (fosito/m_config.f90:83-182)."""
    out: Dict[str, List[str]] = {}
    for raw in text.splitlines():
        line = raw.split("#", 1)[0]
        m = _LINE.match(line)
        if not m:
            continue
        out[m.group(1)] = m.group(2).split()
    return out


def _f(v: Sequence[str]) -> float:
    return float(v[0].replace("d", "e").replace("D", "E"))


def load_cfg_files(paths: Sequence[str], base: StreamerConfig | None = None) -> StreamerConfig:
    """Apply reference-format config files in order on top of ``base``."""
    cfg = base if base is not None else cartesian_8mm()
    kv: Dict[str, List[str]] = {}
    for p in paths:
        with open(p) as fh:
            kv.update(parse_cfg_text(fh.read()))
    upd: Dict[str, object] = {}
    if "end_time" in kv: upd["end_time"] = _f(kv["end_time"])
    if "box_size" in kv: upd["box_size"] = int(kv["box_size"][0])
    if "applied_fld" in kv: upd["applied_fld"] = _f(kv["applied_fld"])
    if "epsilon_diel" in kv: upd["epsilon_diel"] = _f(kv["epsilon_diel"])
    if "bg_dens" in kv: upd["bg_dens"] = _f(kv["bg_dens"])
    if "dt_max" in kv: upd["dt_max"] = _f(kv["dt_max"])
    if "num_steps_amr" in kv: upd["num_steps_amr"] = int(kv["num_steps_amr"][0])
    if "lkptbl_size" in kv: upd["lkptbl_size"] = int(kv["lkptbl_size"][0])
    if "lkptbl_max_fld" in kv: upd["lkptbl_max_fld"] = _f(kv["lkptbl_max_fld"])
    if "photoi_enabled" in kv: upd["photoi_enabled"] = kv["photoi_enabled"][0].upper().startswith("T")
    if "photoi_num_photons" in kv: upd["photoi_num_photons"] = int(kv["photoi_num_photons"][0])
    if any(k in kv for k in ("photoi_eta", "photoi_frac_O2", "gas_pressure")):
        # src/m_streamer.f90:327-330 and src/streamer_cyl.f90:584-588
        eta = _f(kv.get("photoi_eta", ["0.05"]))
        pressure = _f(kv.get("gas_pressure", ["1.0"]))
        frac_o2 = _f(kv.get("photoi_frac_O2", ["0.2"]))
        upd["photoi_coeff"] = photoi_coeff_air(eta, pressure)
        upd["photoi_table"] = ("air", frac_o2 * pressure, 0.0)
    if "lvls_max" in kv: upd["lvls_max"] = int(kv["lvls_max"][0])
    if "use_drt" in kv: upd["use_drt"] = kv["use_drt"][0].upper().startswith("T")
    if "coord" in kv: upd["coord"] = kv["coord"][0]
    if "n_base" in kv: upd["n_base"] = tuple(int(v) for v in kv["n_base"])
    if "domain_len" in kv:
        vals = [_f([v]) for v in kv["domain_len"]]
        if len(vals) == 1:
            vals = vals * cfg.dim
        upd["domain_len"] = tuple(vals)
    out = dataclasses.replace(cfg, **upd)
    if "seed_dens" in kv:
        dl = out.domain_len_z
        dens = [_f([v]) for v in kv["seed_dens"]]
        r0 = [_f([v]) for v in kv.get("seed_rel_r0", [])]
        r1 = [_f([v]) for v in kv.get("seed_rel_r1", [])]
        wid = [_f([v]) for v in kv.get("seed_width", [])]
        fo = [int(v) for v in kv.get("seed_falloff", ["1"] * len(dens))]
        d = out.dim
        if len(r0) != d * len(dens) or len(r1) != d * len(dens) or len(wid) != len(dens):
            raise ValueError("seed_... variables have incompatible size")
        seeds = [Seed(r0=tuple(dl * x for x in r0[d * n:d * n + d]),
                      r1=tuple(dl * x for x in r1[d * n:d * n + d]),
                      dens=dens[n], width=wid[n], falloff=fo[n]) for n in range(len(dens))]
        out = dataclasses.replace(out, seeds=seeds)
    return out
