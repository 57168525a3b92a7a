"""The algorithmic-bytes model: about 253 words per leaf cell on a uniform 2D
tree, and the census of a real tree."""
import a5ref
from a5_streamer_b200 import config, metrics


def test_uniform_tree_figure():
    # uniform tree refined to level L over a 4x4 base: every level full
    nc, L = 8, 7
    cells, leaf, par = {}, {}, {}
    for l in range(-1, L + 1):
        n_box = 16 * (4 ** max(l - 1, 0))
        n = nc // (2 ** (1 - l)) if l < 1 else nc
        cells[l] = n_box * n * n
        leaf[l] = cells[l] if l == L else 0
        par[l] = 0 if l == L else cells[l]
    c = metrics.Census(2, nc, -1, L, cells, leaf, par)
    words = metrics.bytes_per_step(c) / 8 / c.n_leaf
    assert 240 < words < 330


def test_census_of_a_tree():
    cfg = config.cartesian_8mm()
    s = a5ref.Sim(cfg)
    s.init()
    c = metrics.census(s.meta(), s.levels(), cfg.box_size)
    assert c.n_leaf == s.n_leaf_cells()
    assert sum(c.cells.values()) == s.n_cells_all()
    assert metrics.bytes_per_step(c) > 8 * 200 * c.n_leaf
