// a5adj.cu -- adjoint of the fixed-mesh streamer program (include/a5a.h).
//
// Two parts:
//  * a host builder that writes every linear operation of the time step as
//    a list of phases over one index space (all cell and face variables of
//    the run plus the applied voltage): a phase sets rows d to
//    self * x[d] + sum c x[s], reading only values it does not write (its
//    rows' own entries excepted). The builder follows the reference's loops
//    (afivo/src/m_aX_mg.f90:163-565 for the FAS multigrid, m_aX_gc.f90,
//    m_aX_restrict.f90, m_aX_core.f90:818-930, src/streamer_2d.f90:307-381,
//    492-496) on the run's topology. The reverse pass applies each phase
//    transposed (lam[s] += c lam[d], lam[d] = self lam[d]) in reverse order:
//    on a fixed mesh these are fixed matrices, so one list serves every
//    step;
//  * device kernels: the transposed phases, hand-written adjoints of the
//    nonlinear operations (fluxes_koren, update_solution, the cell |E| of
//    fld_from_pot, gc_interp_lim), and the checkpointed reverse sweep, one
//    block per reverse step (the trees of this path are small: the step is
//    ~1,500 dependent phases, which a single block runs behind block
//    barriers).
#include "../../include/a5a.h"
#include "a5_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr int NC = 8;
constexpr int SLOT = (NC + 2) * (NC + 2);
constexpr int FSLOT = (NC + 1) * NC;
constexpr int NVC = 9;                 // cell variables of a run
constexpr int ATHR = 1024;             // threads of the reverse-step block
enum { I_ELEC = 0, I_PION, I_ELEC_OLD, I_PION_OLD, I_PHI, I_FLD, I_RHS, I_PHO, I_EPS };
enum { F_ELEC = 0, F_FLD = 1 };
constexpr int I_TMP = I_FLD;           // the multigrid's tmp variable (mg%i_tmp = i_fld)
constexpr double UC_EPS0 = 8.8541878176e-12;       // fosito/m_units_constants.f90:201-202
constexpr double UC_ELEM_CHARGE = 1.6022e-19;

// Topology tables, afivo/src/m_aX_t.f90:41-81 (2D, 0-based)
constexpr int ch_dix[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
constexpr int ch_adj_nb[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};
constexpr int nb_dix[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};

// ---------------------------------------------------------------------------
// Host topology
struct HBox {
  int in_use = 0, lvl = 0, nc = 0, ix0 = 0, ix1 = 0, parent = 0;
  int ch[4] = {0, 0, 0, 0}, nb[4] = {0, 0, 0, 0};
  double dr = 0, r0 = 0, r1 = 0;
};
struct Topo {
  int max_id = 0, min_lvl = 0, max_lvl = 0, cap = 0;
  std::vector<HBox> b;
  std::vector<std::vector<int>> ids, leaves, parents;  // per level index
  const std::vector<int> &L_ids(int l) const { return ids[l - min_lvl]; }
  const std::vector<int> &L_leaves(int l) const { return leaves[l - min_lvl]; }
  const std::vector<int> &L_parents(int l) const { return parents[l - min_lvl]; }
};

static void topo_from_upload(int max_id, int min_lvl, int max_lvl, const int *meta16,
                             const double *geom4, const std::vector<std::vector<int>> &ids,
                             const std::vector<std::vector<int>> &leaves,
                             const std::vector<std::vector<int>> &parents, int cap, Topo &T) {
  T.max_id = max_id;
  T.min_lvl = min_lvl;
  T.max_lvl = max_lvl;
  T.cap = cap;
  T.b.assign(max_id + 1, HBox());
  for (int id = 1; id <= max_id; id++) {
    const int *m = meta16 + 16 * id;
    HBox &b = T.b[id];
    b.in_use = m[0];
    if (!b.in_use) continue;
    b.lvl = m[1];
    b.ix0 = m[2];
    b.ix1 = m[3];
    b.parent = m[5];
    for (int k = 0; k < 4; k++) b.ch[k] = m[6 + k];
    for (int k = 0; k < 4; k++) b.nb[k] = m[10 + k];
    b.nc = m[14];
    b.r0 = geom4[4 * id + 0];
    b.r1 = geom4[4 * id + 1];
    b.dr = geom4[4 * id + 3];
  }
  T.ids = ids;
  T.leaves = leaves;
  T.parents = parents;
}

// afivo/src/m_aX_utils.f90:227-239 (a$D_get_child_offset), shifted by a
// neighbour direction as the ghost-cell routines use it (nb = -1: none)
static void child_offset(const HBox &b, int nb, int off[2]) {
  for (int d = 0; d < 2; d++) {
    if (b.lvl > 1) off[d] = (((d ? b.ix1 : b.ix0) - 1) & 1) * (b.nc >> 1);
    else off[d] = 0;
    if (nb >= 0) off[d] -= nb_dix[nb][d] * (b.lvl > 1 ? b.nc : (b.nc >> 1));
  }
}

// ---------------------------------------------------------------------------
// Index space: cell variables in the run's slot layout, then the face
// variables (fx of both variables, then fy), then the applied voltage.
struct Ix {
  size_t cap = 0, fx0 = 0, fy0 = 0, v = 0, total = 0;
  void init(size_t c) {
    cap = c;
    fx0 = (size_t)NVC * cap * SLOT;
    fy0 = fx0 + 2 * cap * FSLOT;
    v = fy0 + 2 * cap * FSLOT;
    total = v + 1;
  }
  uint32_t cc(int iv, int id, int i, int j, int nc) const {
    return (uint32_t)(((size_t)iv * cap + id) * SLOT + i + (nc + 2) * j);
  }
  uint32_t fx(int f, int id, int i, int j, int nc) const {
    return (uint32_t)(fx0 + ((size_t)f * cap + id) * FSLOT + (i - 1) + (nc + 1) * (j - 1));
  }
  uint32_t fy(int f, int id, int i, int j, int nc) const {
    return (uint32_t)(fy0 + ((size_t)f * cap + id) * FSLOT + (i - 1) + nc * (j - 1));
  }
};

// Phases of linear rows (CSR).
struct Tape {
  std::vector<int> phase_row{0};
  std::vector<uint32_t> row_d;
  std::vector<double> row_self;
  std::vector<int> row_term{0};
  std::vector<uint32_t> term_s;
  std::vector<double> term_c;
  int n_phase() const { return (int)phase_row.size() - 1; }
};

class Builder {
 public:
  Builder(const Topo &T, const Ix &X, Tape &tp, int n_base) : T(T), X(X), tp(tp), n_base(n_base) {}

  // ---- rows
  void row(uint32_t d, double self) {
    tp.row_d.push_back(d);
    tp.row_self.push_back(self);
  }
  void term(uint32_t s, double c) {
    // the row's own entry goes into its self coefficient
    if (s == tp.row_d.back()) {
      tp.row_self.back() += c;
      return;
    }
    // merge a repeated source of the row
    for (size_t t = (size_t)tp.row_term.back(); t < tp.term_s.size(); t++)
      if (tp.term_s[t] == s) {
        tp.term_c[t] += c;
        return;
      }
    tp.term_s.push_back(s);
    tp.term_c.push_back(c);
  }
  void end_row() { tp.row_term.push_back((int)tp.term_s.size()); }
  void end_phase() { tp.phase_row.push_back((int)tp.row_d.size()); }

  uint32_t c(int iv, int id, int i, int j) const { return X.cc(iv, id, i, j, T.b[id].nc); }

  // ---- multigrid pieces (Cartesian, plain operator), afivo/src/m_aX_mg.f90
  // The recipe of ghost cell k of side nb of box id (a$D_gc_box with
  // mg$D_sides_rb, :261-301, after a$D_gc_prolong0, and sides_bc_pot,
  // src/streamer_2d.f90:620-638), times scale, into the current row.
  void ghost_terms(int id, int nb, int k, double scale) {
    const HBox &b = T.b[id];
    const int nc = b.nc, nb_id = b.nb[nb], dim = nb >> 1;
    int gi, gj;  // ghost cell
    if (dim == 0) { gi = (nb & 1) ? nc + 1 : 0; gj = k; }
    else { gi = k; gj = (nb & 1) ? nc + 1 : 0; }
    if (nb_id > 0) {
      const int ncn = T.b[nb_id].nc;
      int si = gi, sj = gj;
      if (dim == 0) si = (nb & 1) ? 1 : ncn;
      else sj = (nb & 1) ? 1 : ncn;
      term(X.cc(I_PHI, nb_id, si, sj, ncn), scale);
    } else if (nb_id == 0) {
      // prolong0 from the parent, then 0.5 g + f - 0.25 (f_in + f_side)
      int off[2];
      child_offset(b, -1, off);
      const int p = b.parent;
      const int ic1 = off[0] + ((gi + 1) >> 1), jc1 = off[1] + ((gj + 1) >> 1);
      term(c(I_PHI, p, ic1, jc1), 0.5 * scale);
      if (dim == 0) {
        const int i = (nb & 1) ? nc : 1, di = (nb & 1) ? -1 : 1;
        const int dj = -1 + 2 * (k & 1);
        term(c(I_PHI, id, i, k), scale);
        term(c(I_PHI, id, i + di, k), -0.25 * scale);
        term(c(I_PHI, id, i, k + dj), -0.25 * scale);
      } else {
        const int j = (nb & 1) ? nc : 1, dj = (nb & 1) ? -1 : 1;
        const int di = -1 + 2 * (k & 1);
        term(c(I_PHI, id, k, j), scale);
        term(c(I_PHI, id, k + di, j), -0.25 * scale);
        term(c(I_PHI, id, k, j + dj), -0.25 * scale);
      }
    } else {
      switch (nb) {
        case 0: term(c(I_PHI, id, 1, k), scale); break;
        case 1: term(c(I_PHI, id, nc, k), scale); break;
        case 2: term(c(I_PHI, id, k, 1), -scale); break;
        default:
          term((uint32_t)X.v, 2.0 * scale);
          term(c(I_PHI, id, k, nc), -scale);
          break;
      }
    }
  }
  // phi at neighbour (ii, jj) of an interior cell, times scale: the cell
  // itself, or with inl a side ghost through its recipe
  void nbr_terms(int id, int ii, int jj, double scale, bool inl) {
    const int nc = T.b[id].nc;
    if (inl && (ii == 0 || ii == nc + 1)) ghost_terms(id, ii == 0 ? 0 : 1, jj, scale);
    else if (inl && (jj == 0 || jj == nc + 1)) ghost_terms(id, jj == 0 ? 2 : 3, ii, scale);
    else term(c(I_PHI, id, ii, jj), scale);
  }
  // box_gsrb_lpl half-sweep (:714-760) over a level's boxes. inl: the side
  // ghosts it reads are their recipes, which equals reading them after the
  // fill gsrb_boxes makes after every half-sweep (:343-366); without inl the
  // ghost cells in memory are read.
  void gsrb_half(const std::vector<int> &ids, int redblack, bool inl) {
    for (int id : ids) {
      const HBox &b = T.b[id];
      const double dx2 = b.dr * b.dr;
      for (int j = 1; j <= b.nc; j++) {
        int i0 = 2 - ((redblack ^ j) & 1);
        for (int i = i0; i <= b.nc; i += 2) {
          row(c(I_PHI, id, i, j), 0.0);
          nbr_terms(id, i + 1, j, 0.25, inl);
          nbr_terms(id, i - 1, j, 0.25, inl);
          nbr_terms(id, i, j + 1, 0.25, inl);
          nbr_terms(id, i, j - 1, 0.25, inl);
          term(c(I_RHS, id, i, j), -0.25 * dx2);
          end_row();
        }
      }
    }
    end_phase();
  }
  // scale * box_lpl (:662-680) at cell (i, j) into the current row
  void lpl_terms(int id, int i, int j, double scale) {
    const HBox &b = T.b[id];
    const double inv = 1 / (b.dr * b.dr);
    term(c(I_PHI, id, i - 1, j), scale * inv);
    term(c(I_PHI, id, i + 1, j), scale * inv);
    term(c(I_PHI, id, i, j - 1), scale * inv);
    term(c(I_PHI, id, i, j + 1), scale * inv);
    term(c(I_PHI, id, i, j), -4 * scale * inv);
  }
  // ghost cells of phi of a level's boxes (fill_gc_phi, :303-316)
  void fill_gc_phi(const std::vector<int> &ids) {
    for (int id : ids) {
      const int nc = T.b[id].nc;
      for (int nb = 0; nb < 4; nb++)
        for (int k = 1; k <= nc; k++) {
          int gi, gj;
          if ((nb >> 1) == 0) { gi = (nb & 1) ? nc + 1 : 0; gj = k; }
          else { gi = k; gj = (nb & 1) ? nc + 1 : 0; }
          row(c(I_PHI, id, gi, gj), 0.0);
          ghost_terms(id, nb, k, 1.0);
          end_row();
        }
    }
    end_phase();
  }
  // gsrb_boxes (:343-366): the half-sweeps read their side ghosts through the
  // recipes, and the fill after the last one is kept (later phases read the
  // ghost cells from memory). stale: the first half-sweep reads the ghost
  // cells as they are (the base level of a first FMG call, whose ghosts
  // init_phi_rhs does not fill).
  void gsrb_boxes(const std::vector<int> &ids, int n_cycle, bool stale = false) {
    for (int it = 1; it <= 2 * n_cycle; it++) gsrb_half(ids, it, !(stale && it == 1));
    fill_gc_phi(ids);
  }
  // rows of a parent quadrant from one child: dst(parent cell) = 0.25 sum
  // of the 2x2 child cells of var iv (box_rstr_lpl, :683-705)
  void rstr_rows(int cid, int iv_src, int iv_dst) {
    const HBox &cb = T.b[cid];
    const int p = cb.parent, hnc = cb.nc >> 1;
    int off[2];
    child_offset(cb, -1, off);
    for (int j = 1; j <= hnc; j++)
      for (int i = 1; i <= hnc; i++) {
        const int ic = off[0] + i, jc = off[1] + j, i_f = 2 * i - 1, j_f = 2 * j - 1;
        row(c(iv_dst, p, ic, jc), 0.0);
        term(c(iv_src, cid, i_f, j_f), 0.25);
        term(c(iv_src, cid, i_f + 1, j_f), 0.25);
        term(c(iv_src, cid, i_f, j_f + 1), 0.25);
        term(c(iv_src, cid, i_f + 1, j_f + 1), 0.25);
        end_row();
      }
  }
  // box_op_add_copy on the parents of a level: rhs = lpl(phi) + tmp; then,
  // if copy, tmp = phi on every cell
  void op_add_copy(const std::vector<int> &P, bool copy) {
    for (int id : P) {
      const int nc = T.b[id].nc;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          row(c(I_RHS, id, i, j), 0.0);
          lpl_terms(id, i, j, 1.0);
          term(c(I_TMP, id, i, j), 1.0);
          end_row();
        }
    }
    end_phase();
    if (copy) {
      copy_all(P, I_PHI, I_TMP);
      end_phase();
    }
  }
  void copy_all(const std::vector<int> &ids, int from, int to) {
    for (int id : ids) {
      const int g = T.b[id].nc + 2;
      for (int j = 0; j < g; j++)
        for (int i = 0; i < g; i++) {
          row(c(to, id, i, j), 0.0);
          term(c(from, id, i, j), 1.0);
          end_row();
        }
    }
  }
  // update_coarse (:370-410)
  void update_coarse(int lvl) {
    for (int id : T.L_ids(lvl)) {
      const HBox &b = T.b[id];
      const int p = b.parent, hnc = b.nc >> 1;
      int off[2];
      child_offset(b, -1, off);
      for (int j = 1; j <= hnc; j++)
        for (int i = 1; i <= hnc; i++) {
          const int ic = off[0] + i, jc = off[1] + j, i_f = 2 * i - 1, j_f = 2 * j - 1;
          // parent tmp = restriction of the residual rhs - lpl(phi)
          row(c(I_TMP, p, ic, jc), 0.0);
          for (int q = 0; q < 4; q++) {
            const int a = i_f + (q & 1), bb = j_f + (q >> 1);
            term(c(I_RHS, id, a, bb), 0.25);
            lpl_terms(id, a, bb, -0.25);
          }
          end_row();
        }
      rstr_rows(id, I_PHI, I_PHI);
    }
    end_phase();
    fill_gc_phi(T.L_ids(lvl - 1));
    op_add_copy(T.L_parents(lvl - 1), true);
  }
  // set_coarse_phi_rhs (:414-447)
  void set_coarse_phi_rhs(int lvl) {
    if (lvl == T.max_lvl) fill_gc_phi(T.L_ids(lvl));
    for (int id : T.L_ids(lvl)) {
      const int nc = T.b[id].nc;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          row(c(I_TMP, id, i, j), 0.0);
          term(c(I_RHS, id, i, j), 1.0);
          lpl_terms(id, i, j, -1.0);
          end_row();
        }
    }
    end_phase();
    for (int id : T.L_ids(lvl)) {
      rstr_rows(id, I_TMP, I_TMP);
      rstr_rows(id, I_PHI, I_PHI);
    }
    end_phase();
    fill_gc_phi(T.L_ids(lvl - 1));
    op_add_copy(T.L_parents(lvl - 1), false);
  }
  // init_phi_rhs (:450-473)
  void init_phi_rhs() {
    for (int lvl = T.max_lvl; lvl >= T.min_lvl + 1; lvl--) {
      for (int id : T.L_ids(lvl)) {
        const int g = T.b[id].nc + 2;
        for (int j = 0; j < g; j++)
          for (int i = 0; i < g; i++) {
            row(c(I_PHI, id, i, j), 0.0);
            end_row();
          }
        rstr_rows(id, I_RHS, I_RHS);
      }
      end_phase();
    }
  }
  // correct_children (:319-341) with box_corr_lpl (:605-633)
  void correct_children(const std::vector<int> &P) {
    for (int id : P) {
      const int g = T.b[id].nc + 2;
      for (int j = 0; j < g; j++)
        for (int i = 0; i < g; i++) {
          row(c(I_TMP, id, i, j), -1.0);
          term(c(I_PHI, id, i, j), 1.0);
          end_row();
        }
    }
    end_phase();
    for (int id : P)
      for (int q = 0; q < 4; q++) {
        const int cid = T.b[id].ch[q];
        if (cid <= 0) continue;
        const HBox &cb = T.b[cid];
        int off[2];
        child_offset(cb, -1, off);
        for (int j = 1; j <= cb.nc; j++) {
          const int j_c1 = off[1] + ((j + 1) >> 1), j_c2 = j_c1 + 1 - 2 * (j & 1);
          for (int i = 1; i <= cb.nc; i++) {
            const int i_c1 = off[0] + ((i + 1) >> 1), i_c2 = i_c1 + 1 - 2 * (i & 1);
            row(c(I_PHI, cid, i, j), 1.0);
            term(c(I_TMP, id, i_c1, j_c1), 0.5);
            term(c(I_TMP, id, i_c2, j_c1), 0.25);
            term(c(I_TMP, id, i_c1, j_c2), 0.25);
            end_row();
          }
        }
      }
    end_phase();
  }
  // mg$D_fas_vcycle (:208-254), set_residual false; stale_base: the base
  // level's first half-sweep reads the ghost cells as they are
  void vcycle(int max_lvl, bool stale_base = false) {
    for (int lvl = max_lvl; lvl >= T.min_lvl + 1; lvl--) {
      gsrb_boxes(T.L_ids(lvl), n_down);
      update_coarse(lvl);
    }
    gsrb_boxes(T.L_ids(T.min_lvl), n_base, stale_base);
    for (int lvl = T.min_lvl + 1; lvl <= max_lvl; lvl++) {
      correct_children(T.L_parents(lvl - 1));
      fill_gc_phi(T.L_ids(lvl));
      gsrb_boxes(T.L_ids(lvl), n_up);
    }
  }
  // mg$D_fas_fmg (:163-202), set_residual false
  void fmg(bool first_call) {
    if (first_call) init_phi_rhs();
    else
      for (int lvl = T.max_lvl; lvl >= T.min_lvl + 1; lvl--) set_coarse_phi_rhs(lvl);
    for (int lvl = T.min_lvl; lvl <= T.max_lvl; lvl++) {
      copy_all(T.L_ids(lvl), I_PHI, I_TMP);
      end_phase();
      if (lvl > T.min_lvl) {
        correct_children(T.L_parents(lvl - 1));
        fill_gc_phi(T.L_ids(lvl));
      }
      // the first call's first base-level sweep reads the ghost cells as the
      // previous fills left them (init_phi_rhs fills none)
      vcycle(lvl, first_call && lvl == T.min_lvl);
    }
  }

  // ---- transport and field pieces
  // a$D_tree_copy_cc (afivo/src/m_aX_utils.f90:432-453) of n_e and n_i
  void copy_old() {
    for (int lvl = T.min_lvl; lvl <= T.max_lvl; lvl++) {
      copy_all(T.L_ids(lvl), I_ELEC, I_ELEC_OLD);
      copy_all(T.L_ids(lvl), I_PION, I_PION_OLD);
    }
    end_phase();
  }
  // a$D_consistent_fluxes / flux_from_children (afivo/src/m_aX_core.f90:818-930)
  void consistent_fluxes() {
    for (int lvl = T.min_lvl; lvl <= T.max_lvl - 1; lvl++) {
      for (int id : T.L_parents(lvl)) {
        const HBox &p = T.b[id];
        for (int nb = 0; nb < 4; nb++) {
          const int nb_id = p.nb[nb];
          if (nb_id <= 0 || T.b[nb_id].ch[0] > 0) continue;
          const HBox &bn = T.b[nb_id];
          const int nc = p.nc, nch = nc >> 1;
          const bool low = !(nb & 1);
          const int i = low ? 1 : nc + 1, i_nb = low ? nc + 1 : 1;
          for (int k = 0; k < 2; k++) {
            const int i_ch = ch_adj_nb[nb][k], cid = p.ch[i_ch];
            const int cnc = T.b[cid].nc;
            const int ioff0 = nch * ch_dix[i_ch][0], ioff1 = nch * ch_dix[i_ch][1];
            for (int m = 1; m <= nch; m++) {
              if ((nb >> 1) == 0) {
                row(X.fx(F_ELEC, nb_id, i_nb, ioff1 + m, bn.nc), 0.0);
                term(X.fx(F_ELEC, cid, i, 2 * m - 1, cnc), 0.5);
                term(X.fx(F_ELEC, cid, i, 2 * m, cnc), 0.5);
              } else {
                row(X.fy(F_ELEC, nb_id, ioff0 + m, i_nb, bn.nc), 0.0);
                term(X.fy(F_ELEC, cid, 2 * m - 1, i, cnc), 0.5);
                term(X.fy(F_ELEC, cid, 2 * m, i, cnc), 0.5);
              }
              end_row();
            }
          }
        }
      }
      end_phase();
    }
  }
  // a$D_restrict_tree (afivo/src/m_aX_restrict.f90:23-142) of n_e, then n_i
  void restrict_dens() {
    for (int iv : {I_ELEC, I_PION})
      for (int lvl = T.max_lvl - 1; lvl >= T.min_lvl; lvl--) {
        for (int id : T.L_parents(lvl))
          for (int q = 0; q < 4; q++)
            if (T.b[id].ch[q] > 0) rstr_rows(T.b[id].ch[q], iv, iv);
        end_phase();
      }
  }
  // space charge, src/streamer_2d.f90:317-329 (leaves of levels >= 1, every cell)
  void set_rhs() {
    const double fac = UC_ELEM_CHARGE / UC_EPS0;
    for (int lvl = std::max(1, T.min_lvl); lvl <= T.max_lvl; lvl++)
      for (int id : T.L_leaves(lvl)) {
        const int g = T.b[id].nc + 2;
        for (int j = 0; j < g; j++)
          for (int i = 0; i < g; i++) {
            row(c(I_RHS, id, i, j), 0.0);
            term(c(I_ELEC, id, i, j), fac);
            term(c(I_PION, id, i, j), -fac);
            end_row();
          }
      }
    end_phase();
  }
  // the faces of fld_from_pot (src/streamer_2d.f90:346-381) on every box,
  // eps = 1 (the box-edge faces' eps weight 2 eps_g / (eps_i + eps_g) is 1)
  void fld_faces() {
    for (int lvl = T.min_lvl; lvl <= T.max_lvl; lvl++)
      for (int id : T.L_ids(lvl)) {
        const HBox &b = T.b[id];
        const int nc = b.nc;
        const double inv_dr = 1 / b.dr;
        for (int j = 1; j <= nc; j++)
          for (int i = 1; i <= nc + 1; i++) {
            row(X.fx(F_FLD, id, i, j, nc), 0.0);
            term(c(I_PHI, id, i - 1, j), inv_dr);
            term(c(I_PHI, id, i, j), -inv_dr);
            end_row();
          }
        for (int j = 1; j <= nc + 1; j++)
          for (int i = 1; i <= nc; i++) {
            row(X.fy(F_FLD, id, i, j, nc), 0.0);
            term(c(I_PHI, id, i, j - 1), inv_dr);
            term(c(I_PHI, id, i, j), -inv_dr);
            end_row();
          }
      }
    end_phase();
  }
  // a$D_gc_tree(i_fld, a$D_gc_interp, a$D_gc_neumann) (afivo/src/m_aX_gc.f90:28-185, 298-330)
  void gc_fld() {
    const double sixth = 1 / 6.0, third = 1 / 3.0;
    for (int lvl = T.min_lvl; lvl <= T.max_lvl; lvl++) {
      for (int id : T.L_ids(lvl)) {
        const HBox &b = T.b[id];
        const int nc = b.nc;
        for (int nb = 0; nb < 4; nb++) {
          const int nb_id = b.nb[nb], dim = nb >> 1;
          for (int k = 1; k <= nc; k++) {
            int gi, gj;
            if (dim == 0) { gi = (nb & 1) ? nc + 1 : 0; gj = k; }
            else { gi = k; gj = (nb & 1) ? nc + 1 : 0; }
            row(c(I_FLD, id, gi, gj), 0.0);
            if (nb_id > 0) {
              const int ncn = T.b[nb_id].nc;
              int si = gi, sj = gj;
              if (dim == 0) si = (nb & 1) ? 1 : ncn;
              else sj = (nb & 1) ? 1 : ncn;
              term(X.cc(I_FLD, nb_id, si, sj, ncn), 1.0);
            } else if (nb_id == 0) {
              const int pn = T.b[b.parent].nb[nb];
              int off[2];
              child_offset(b, nb, off);
              const int ix_f = (nb & 1) ? nc : 1, ix_c = (nb & 1) ? 1 : nc;
              const int a1 = off[dim == 0 ? 1 : 0] + ((k + 1) >> 1);
              const int a2 = a1 + 1 - 2 * (k & 1);
              if (dim == 0) {
                term(c(I_FLD, pn, ix_c, a1), 0.5);
                term(c(I_FLD, pn, ix_c, a2), sixth);
                term(c(I_FLD, id, ix_f, k), third);
              } else {
                term(c(I_FLD, pn, a1, ix_c), 0.5);
                term(c(I_FLD, pn, a2, ix_c), sixth);
                term(c(I_FLD, id, k, ix_f), third);
              }
            } else {
              switch (nb) {
                case 0: term(c(I_FLD, id, 1, k), 1.0); break;
                case 1: term(c(I_FLD, id, nc, k), 1.0); break;
                case 2: term(c(I_FLD, id, k, 1), 1.0); break;
                default: term(c(I_FLD, id, k, nc), 1.0); break;
              }
            }
            end_row();
          }
        }
      }
      end_phase();
    }
  }
  // average_dens (src/streamer_2d.f90:492-496) on every box and cell
  void average() {
    for (int lvl = T.min_lvl; lvl <= T.max_lvl; lvl++)
      for (int id : T.L_ids(lvl)) {
        const int g = T.b[id].nc + 2;
        for (int v = 0; v < 2; v++)
          for (int j = 0; j < g; j++)
            for (int i = 0; i < g; i++) {
              row(c(v, id, i, j), 0.5);
              term(c(v + 2, id, i, j), 0.5);
              end_row();
            }
      }
    end_phase();
  }

 private:
  const Topo &T;
  const Ix &X;
  Tape &tp;
  int n_base, n_down = 2, n_up = 2;
};

enum { SEG_COPY = 0, SEG_CONS, SEG_RSTR, SEG_RHS, SEG_FMG, SEG_FMG1, SEG_FACES, SEG_GCFLD, SEG_AVG,
       N_SEG };

// Build one tape holding every segment; seg_phase[s], seg_phase[s+1] bound
// segment s. Checks that no phase reads a value it writes (except a row's
// own entry) and that no phase writes an entry twice.
static std::string build_tape(const Topo &T, const Ix &X, int n_base, Tape &tp, int seg_phase[N_SEG + 1]) {
  Builder B(T, X, tp, n_base);
  seg_phase[SEG_COPY] = tp.n_phase();
  B.copy_old();
  seg_phase[SEG_CONS] = tp.n_phase();
  B.consistent_fluxes();
  seg_phase[SEG_RSTR] = tp.n_phase();
  B.restrict_dens();
  seg_phase[SEG_RHS] = tp.n_phase();
  B.set_rhs();
  seg_phase[SEG_FMG] = tp.n_phase();
  B.fmg(false);
  seg_phase[SEG_FMG1] = tp.n_phase();
  B.fmg(true);
  seg_phase[SEG_FACES] = tp.n_phase();
  B.fld_faces();
  seg_phase[SEG_GCFLD] = tp.n_phase();
  B.gc_fld();
  seg_phase[SEG_AVG] = tp.n_phase();
  B.average();
  seg_phase[N_SEG] = tp.n_phase();
  if (X.total >= 0xffffffffull) return "index space too large";
  std::vector<int> stamp(X.total, -1);
  for (int p = 0; p < tp.n_phase(); p++) {
    for (int r = tp.phase_row[p]; r < tp.phase_row[p + 1]; r++) {
      if (stamp[tp.row_d[r]] == p) return "phase " + std::to_string(p) + " writes an entry twice";
      stamp[tp.row_d[r]] = p;
    }
    for (int r = tp.phase_row[p]; r < tp.phase_row[p + 1]; r++)
      for (int t = tp.row_term[r]; t < tp.row_term[r + 1]; t++)
        if (tp.term_s[t] != tp.row_d[r] && stamp[tp.term_s[t]] == p)
          return "phase " + std::to_string(p) + " reads an entry it writes";
  }
  return "";
}

// ---------------------------------------------------------------------------
// Device side
struct DBox {
  int lvl, nc, parent, pad;
  int ch[4], nb[4];
  int ix0, ix1, pad2[2];
  double dr, r0, r1, pad3;
};

struct AdjArgs {
  // tape
  const int *phase_row;
  const uint32_t *row_d;
  const double *row_self;
  const int *row_term;
  const uint32_t *term_s;
  const double *term_c;
  int seg[N_SEG + 1];
  // topology
  const DBox *box;
  const int *lists;            // ids | leaves of every level
  int lv_ids[41], lv_leaves[41];  // offsets per level index (+1 entry)
  int min_lvl, max_lvl, nlev, cap;
  // adjoint vector (cell vars, fx, fy, voltage) and table accumulator
  double *lam;
  double *lam_tbl;             // n_rows x 4
  const double *tbl;           // n_rows x 4 column-major
  int tbl_rows, pad;
  double tbl_xmin, tbl_inv_dx;
};

// Intermediate fields of one step (device pointers): cell blocks of
// capacity * SLOT doubles, face pairs of 2 * capacity * FSLOT (fx then fy).
struct StepSnap {
  const double *n0, *E0, *ff0;  // step start: n_e, |E|, field faces
  const double *F1, *R1e, *R1i, *E1, *ff1;
  const double *F2, *R2e, *R2i, *ff3;
  double dt;
};

// nb_dix of a neighbour direction (afivo/src/m_aX_t.f90:64-67)
__device__ __forceinline__ int nbdx(int nb) { return nb == 0 ? -1 : (nb == 1 ? 1 : 0); }
__device__ __forceinline__ int nbdy(int nb) { return nb == 2 ? -1 : (nb == 3 ? 1 : 0); }
__device__ __forceinline__ size_t lx(const AdjArgs &A, int f, int id, int i, int j, int nc) {
  return (size_t)NVC * A.cap * SLOT + ((size_t)f * A.cap + id) * FSLOT + (i - 1) + (nc + 1) * (j - 1);
}
__device__ __forceinline__ size_t ly(const AdjArgs &A, int f, int id, int i, int j, int nc) {
  return (size_t)NVC * A.cap * SLOT + 2 * (size_t)A.cap * FSLOT + ((size_t)f * A.cap + id) * FSLOT +
         (i - 1) + nc * (j - 1);
}
// offsets inside a snapshot face pair
__device__ __forceinline__ size_t sfx(const AdjArgs &A, int id, int i, int j, int nc) {
  return (size_t)id * FSLOT + (i - 1) + (nc + 1) * (j - 1);
}
__device__ __forceinline__ size_t sfy(const AdjArgs &A, int id, int i, int j, int nc) {
  return (size_t)A.cap * FSLOT + (size_t)id * FSLOT + (i - 1) + nc * (j - 1);
}

// Transposed phases p1-1 down to p0.
__device__ void tape_rev(const AdjArgs &A, int p0, int p1) {
  for (int p = p1 - 1; p >= p0; p--) {
    const int r0 = A.phase_row[p], r1 = A.phase_row[p + 1];
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const uint32_t d = A.row_d[r];
      const double lam = A.lam[d];
      if (lam != 0.0) {
        for (int t = A.row_term[r]; t < A.row_term[r + 1]; t++)
          atomicAdd(&A.lam[A.term_s[t]], A.term_c[t] * lam);
        A.lam[d] = A.row_self[r] * lam;
      }
    }
    __syncthreads();
  }
}
__device__ __forceinline__ void seg_rev(const AdjArgs &A, int s) { tape_rev(A, A.seg[s], A.seg[s + 1]); }

// Table location (fosito/m_lookup_table.f90:117-124): low row (1-based),
// weight of the low row, and d(lookup)/dx per unit row difference
// (inv_dx where not clamped, else 0).
struct TLoc { int low; double w, ddx; };
__device__ __forceinline__ TLoc tloc(const AdjArgs &A, double x) {
  TLoc l;
  const double frac = (x - A.tbl_xmin) * A.tbl_inv_dx;
  l.ddx = A.tbl_inv_dx;
  if (frac < 2.0e9 && frac > -2.0e9) {
    l.low = (int)ceil(frac);
    l.w = l.low - frac;
  } else {
    l.low = frac > 0 ? A.tbl_rows : 0;
    l.w = 0;
    l.ddx = 0;
  }
  if (l.low < 1) { l.low = 1; l.w = 1; l.ddx = 0; }
  else if (l.low >= A.tbl_rows) { l.low = A.tbl_rows - 1; l.w = 0; l.ddx = 0; }
  return l;
}
__device__ __forceinline__ double trow(const AdjArgs &A, int row, int col) {
  return A.tbl[(row - 1) + (size_t)A.tbl_rows * col];
}
__device__ __forceinline__ double tval(const AdjArgs &A, const TLoc &l, int col) {
  return l.w * trow(A, l.low, col) + (1 - l.w) * trow(A, l.low + 1, col);
}
__device__ __forceinline__ double tdx(const AdjArgs &A, const TLoc &l, int col) {
  return l.ddx * (trow(A, l.low + 1, col) - trow(A, l.low, col));
}
// adjoint of a lookup's table rows into the block's accumulator
__device__ __forceinline__ void tacc(double *s_tbl, int rows, const TLoc &l, int col, double g) {
  atomicAdd(&s_tbl[(l.low - 1) + rows * col], l.w * g);
  atomicAdd(&s_tbl[l.low + rows * col], (1 - l.w) * g);
}

// Koren limiter (src/m_streamer.f90:339-362) and its partial derivatives
__device__ __forceinline__ double koren(double a, double b, double &ka, double &kb) {
  const double aa = a * a, ab = a * b;
  ka = kb = 0;
  if (ab <= 0) return 0;
  if (aa <= 0.25 * ab) { ka = 1; return a; }
  if (aa <= 2.5 * ab) { ka = 1.0 / 3.0; kb = 1.0 / 6.0; return (1 / 6.0) * (b + 2 * a); }
  kb = 1;
  return b;
}

// Sources of the second ghost layer of n_e at side nb, index k
// (a$D_gc2_box with gc2_prolong1 / gc2_neumann, afivo/src/m_aX_gc.f90:407-622):
// up to 3 (cell index in the n_e block, coefficient) pairs.
__device__ int gc2_src(const AdjArgs &A, int id, int nb, int k, size_t *src, double *cf) {
  const DBox &m = A.box[id];
  const int nc = m.nc, nb_id = m.nb[nb], dim = nb >> 1;
  if (nb_id > 0) {
    int i, j;
    switch (nb) {
      case 0: i = nc - 1; j = k; break;
      case 1: i = 2; j = k; break;
      case 2: i = k; j = nc - 1; break;
      default: i = k; j = 2; break;
    }
    src[0] = (size_t)nb_id * SLOT + i + (A.box[nb_id].nc + 2) * j;
    cf[0] = 1;
    return 1;
  }
  if (nb_id == 0) {
    int o0, o1;
    if (m.lvl > 1) {
      o0 = ((m.ix0 - 1) & 1) * (nc >> 1) - nbdx(nb) * nc;
      o1 = ((m.ix1 - 1) & 1) * (nc >> 1) - nbdy(nb) * nc;
    } else {
      o0 = -nbdx(nb) * (nc >> 1);
      o1 = -nbdy(nb) * (nc >> 1);
    }
    const int pn = m.parent > 0 ? A.box[m.parent].nb[nb] : 0;
    if (pn <= 0) return 0;  // not a refinement boundary of a valid tree
    const int g = A.box[pn].nc + 2;
    const int ix = (nb & 1) * (nc + 3) - 1;
    const int hs = (ix + 1) >> 1, par = ix & 1;
    int i_c1, i_c2, j_c1, j_c2;
    if (dim == 0) {
      i_c1 = o0 + hs;
      i_c2 = i_c1 + 1 - 2 * par;
      j_c1 = o1 + ((k + 1) >> 1);
      j_c2 = j_c1 + 1 - 2 * (k & 1);
    } else {
      j_c1 = o1 + hs;
      j_c2 = j_c1 + 1 - 2 * par;
      i_c1 = o0 + ((k + 1) >> 1);
      i_c2 = i_c1 + 1 - 2 * (k & 1);
    }
    src[0] = (size_t)pn * SLOT + i_c1 + g * j_c1;
    src[1] = (size_t)pn * SLOT + i_c2 + g * j_c1;
    src[2] = (size_t)pn * SLOT + i_c1 + g * j_c2;
    cf[0] = 0.5;
    cf[1] = 0.25;
    cf[2] = 0.25;
    return 3;
  }
  int i, j;
  switch (nb) {
    case 0: i = 2; j = k; break;
    case 1: i = nc - 1; j = k; break;
    case 2: i = k; j = 2; break;
    default: i = k; j = nc - 1; break;
  }
  src[0] = (size_t)id * SLOT + i + (nc + 2) * j;
  cf[0] = 1;
  return 1;
}

__device__ __forceinline__ void leaf_item(const AdjArgs &A, int q, int per_box, int &id, int &r) {
  // q-th item over the leaves of all levels, per_box items per box
  const int b = q / per_box;
  id = A.lists[A.lv_leaves[0] + b];
  r = q - b * per_box;
}
__device__ __forceinline__ int n_leaves(const AdjArgs &A) { return A.lv_leaves[A.nlev] - A.lv_leaves[0]; }
__device__ __forceinline__ int n_ids(const AdjArgs &A) { return A.lv_ids[A.nlev] - A.lv_ids[0]; }

// Adjoint of fluxes_koren (src/streamer_2d.f90:384-489): the electron flux of
// every leaf face from n_e (with both ghost layers), |E| and the face field.
__device__ void adj_fluxes(const AdjArgs &A, double *s_tbl, const double *ne, const double *E,
                           const double *ff, double dt) {
  const double fac = -0.8 * UC_EPS0 / (UC_ELEM_CHARGE * dt);
  const int nb_all = n_leaves(A);
  const int per = 2 * (NC + 1) * NC;
  double *lam_ne = A.lam + (size_t)I_ELEC * A.cap * SLOT;
  double *lam_E = A.lam + (size_t)I_FLD * A.cap * SLOT;
  for (int q = threadIdx.x; q < nb_all * per; q += blockDim.x) {
    int id, r;
    leaf_item(A, q, per, id, r);
    const DBox &m = A.box[id];
    const int nc = m.nc;
    const int nfx = (nc + 1) * nc;
    if (r >= 2 * nfx) continue;
    const int dim = r < nfx ? 0 : 1;
    const int rr = dim == 0 ? r : r - nfx;
    int i, j;
    if (dim == 0) { i = rr % (nc + 1) + 1; j = rr / (nc + 1) + 1; }
    else { i = rr % nc + 1; j = rr / nc + 1; }
    const size_t fidx = dim == 0 ? lx(A, F_ELEC, id, i, j, nc) : ly(A, F_ELEC, id, i, j, nc);
    const double g = A.lam[fidx];
    if (g == 0.0) continue;
    A.lam[fidx] = 0.0;
    const int g2 = nc + 2;
    const size_t base = (size_t)id * SLOT;
    const int di = dim == 0 ? 1 : 0, dj = dim == 0 ? 0 : 1;
    const int pos = dim == 0 ? i : j;       // face index along the normal
    const int kk = dim == 0 ? j : i;        // index along the side
    // cells c(-2) c(-1) | c(0) c(+1) along the normal
    const size_t i0 = base + i + g2 * j;
    const size_t im = base + (i - di) + g2 * (j - dj);
    const double inv_dr = 1 / m.dr;
    const double E0 = E[i0], Em = E[im];
    const double fa = 0.5 * (E0 + Em);
    const TLoc L = tloc(A, fa);
    const double mob = tval(A, L, 0), dif = tval(A, L, 1);
    const double fld = dim == 0 ? ff[sfx(A, id, i, j, nc)] : ff[sfy(A, id, i, j, nc)];
    const double v = -mob * fld;
    const double c0 = ne[i0], cm = ne[im];
    const double gradc = c0 - cm;
    double l_gradc = -dif * inv_dr * g;
    const double l_dif = -gradc * inv_dr * g;
    double l_fld = 0, l_v = 0;
    double l_c0 = 0, l_cm = 0;
    size_t src[3];
    double cf[3];
    if (v < 0.0) {
      int ns;
      const bool edge = pos == nc + 1;
      double cp;
      if (edge) {
        ns = gc2_src(A, id, dim == 0 ? 1 : 3, kk, src, cf);
        cp = ns == 3 ? 0.5 * ne[src[0]] + 0.25 * ne[src[1]] + 0.25 * ne[src[2]]
                     : (ns == 1 ? ne[src[0]] : 0.0);
      } else {
        ns = 1;
        src[0] = base + (i + di) + g2 * (j + dj);
        cf[0] = 1;
        cp = ne[src[0]];
      }
      const double gradn = cp - c0;
      double ka, kb;
      const double Lm = koren(gradc, gradn, ka, kb);
      const double f = v * (c0 - Lm);
      if (f < fac * fld) {
        l_fld += fac * g;
      } else {
        l_v = (c0 - Lm) * g;
        l_c0 += v * g;
        const double l_L = -v * g;
        l_gradc += ka * l_L;
        const double l_b = kb * l_L;
        for (int t = 0; t < ns; t++) atomicAdd(&lam_ne[src[t]], cf[t] * l_b);
        l_c0 -= l_b;
      }
    } else {
      int ns;
      const bool edge = pos == 1;
      double cmm;
      if (edge) {
        ns = gc2_src(A, id, dim == 0 ? 0 : 2, kk, src, cf);
        cmm = ns == 3 ? 0.5 * ne[src[0]] + 0.25 * ne[src[1]] + 0.25 * ne[src[2]]
                      : (ns == 1 ? ne[src[0]] : 0.0);
      } else {
        ns = 1;
        src[0] = base + (i - 2 * di) + g2 * (j - 2 * dj);
        cf[0] = 1;
        cmm = ne[src[0]];
      }
      const double gradp = cm - cmm;
      double ka, kb;
      const double Lm = koren(gradc, gradp, ka, kb);
      const double f = v * (cm + Lm);
      if (f > fac * fld) {
        l_fld += fac * g;
      } else {
        l_v = (cm + Lm) * g;
        l_cm += v * g;
        const double l_L = v * g;
        l_gradc += ka * l_L;
        const double l_b = kb * l_L;
        l_cm += l_b;
        for (int t = 0; t < ns; t++) atomicAdd(&lam_ne[src[t]], -cf[t] * l_b);
      }
    }
    // v = -mob * fld
    const double l_mob = -fld * l_v;
    l_fld += -mob * l_v;
    l_c0 += l_gradc;
    l_cm -= l_gradc;
    atomicAdd(&lam_ne[i0], l_c0);
    atomicAdd(&lam_ne[im], l_cm);
    // face field (each face is this thread's alone in this operation)
    const size_t ffi = dim == 0 ? lx(A, F_FLD, id, i, j, nc) : ly(A, F_FLD, id, i, j, nc);
    A.lam[ffi] += l_fld;
    // lookups of mobility and diffusion at the face-averaged |E|
    tacc(s_tbl, A.tbl_rows, L, 0, l_mob);
    tacc(s_tbl, A.tbl_rows, L, 1, l_dif);
    const double l_fa = tdx(A, L, 0) * l_mob + tdx(A, L, 1) * l_dif;
    if (l_fa != 0.0) {
      atomicAdd(&lam_E[i0], 0.5 * l_fa);
      atomicAdd(&lam_E[im], 0.5 * l_fa);
    }
  }
  __syncthreads();
}

// Adjoint of update_solution (src/streamer_2d.f90:499-542), Cartesian, eps = 1.
__device__ void adj_update(const AdjArgs &A, double *s_tbl, const double *F, const double *E,
                           double dt) {
  const int nb_all = n_leaves(A);
  const int per = NC * NC;
  const double *lam_ne = A.lam + (size_t)I_ELEC * A.cap * SLOT;
  const double *lam_ni = A.lam + (size_t)I_PION * A.cap * SLOT;
  double *lam_E = A.lam + (size_t)I_FLD * A.cap * SLOT;
  for (int q = threadIdx.x; q < nb_all * per; q += blockDim.x) {
    int id, r;
    leaf_item(A, q, per, id, r);
    const DBox &m = A.box[id];
    const int nc = m.nc;
    if (r >= nc * nc) continue;
    const int i = r % nc + 1, j = r / nc + 1;
    const size_t ci = (size_t)id * SLOT + i + (nc + 2) * j;
    const double gE = lam_ne[ci], gI = lam_ni[ci];
    const double l_src = dt * (gE + gI), l_sflux = dt * gE;
    if (l_src == 0.0 && l_sflux == 0.0) continue;
    const double inv_dr = 1 / m.dr;
    const double fld = E[ci];
    const TLoc L = tloc(A, fld);
    const double alpha = tval(A, L, 2), eta = tval(A, L, 3);
    const double fxl = F[sfx(A, id, i, j, nc)], fxh = F[sfx(A, id, i + 1, j, nc)];
    const double fyl = F[sfy(A, id, i, j, nc)], fyh = F[sfy(A, id, i, j + 1, nc)];
    const double d0 = fxl + fxh, d1 = fyl + fyh;
    const double nrm = sqrt(d0 * d0 + d1 * d1);
    double ld0 = 0, ld1 = 0;
    if (nrm > 0) {
      const double s = 0.5 * (alpha - eta) * l_src / nrm;
      ld0 = s * d0;
      ld1 = s * d1;
    }
    const double l_alpha = 0.5 * nrm * l_src, l_eta = -0.5 * nrm * l_src;
    atomicAdd(&A.lam[lx(A, F_ELEC, id, i, j, nc)], ld0 + inv_dr * l_sflux);
    atomicAdd(&A.lam[lx(A, F_ELEC, id, i + 1, j, nc)], ld0 - inv_dr * l_sflux);
    atomicAdd(&A.lam[ly(A, F_ELEC, id, i, j, nc)], ld1 + inv_dr * l_sflux);
    atomicAdd(&A.lam[ly(A, F_ELEC, id, i, j + 1, nc)], ld1 - inv_dr * l_sflux);
    tacc(s_tbl, A.tbl_rows, L, 2, l_alpha);
    tacc(s_tbl, A.tbl_rows, L, 3, l_eta);
    const double l_fld = tdx(A, L, 2) * l_alpha + tdx(A, L, 3) * l_eta;
    lam_E[ci] += l_fld;  // this cell is this thread's alone here
  }
  __syncthreads();
}

// Adjoint of the cell |E| of fld_from_pot (src/streamer_2d.f90:375-380) on
// every box: |E| = sqrt(sx^2/4 + sy^2/4) from the four face fields.
__device__ void adj_fld_norm(const AdjArgs &A, const double *ff) {
  const int n = n_ids(A);
  const int per = NC * NC;
  double *lam_E = A.lam + (size_t)I_FLD * A.cap * SLOT;
  for (int q = threadIdx.x; q < n * per; q += blockDim.x) {
    const int b = q / per, r = q - b * per;
    const int id = A.lists[A.lv_ids[0] + b];
    const int nc = A.box[id].nc;
    if (r >= nc * nc) continue;
    const int i = r % nc + 1, j = r / nc + 1;
    const size_t ci = (size_t)id * SLOT + i + (nc + 2) * j;
    const double g = lam_E[ci];
    if (g == 0.0) continue;
    lam_E[ci] = 0.0;
    const double sx = ff[sfx(A, id, i, j, nc)] + ff[sfx(A, id, i + 1, j, nc)];
    const double sy = ff[sfy(A, id, i, j, nc)] + ff[sfy(A, id, i, j + 1, nc)];
    const double e = sqrt(0.25 * (sx * sx) + 0.25 * (sy * sy));
    if (!(e > 0)) continue;
    const double lx_ = 0.25 * sx / e * g, ly_ = 0.25 * sy / e * g;
    atomicAdd(&A.lam[lx(A, F_FLD, id, i, j, nc)], lx_);
    atomicAdd(&A.lam[lx(A, F_FLD, id, i + 1, j, nc)], lx_);
    atomicAdd(&A.lam[ly(A, F_FLD, id, i, j, nc)], ly_);
    atomicAdd(&A.lam[ly(A, F_FLD, id, i, j + 1, nc)], ly_);
  }
  __syncthreads();
}

// Adjoint of a$D_gc_tree(iv, a$D_gc_interp_lim, a$D_gc_neumann)
// (afivo/src/m_aX_gc.f90:28-68, 190-330). Levels in reverse order: a level's
// fill reads the coarser level's ghost cells. X is the variable after the
// fill (the limiter's branch).
__device__ void adj_gc_lim(const AdjArgs &A, int iv, const double *X) {
  const double sixth = 1 / 6.0, third = 1 / 3.0;
  double *lam = A.lam + (size_t)iv * A.cap * SLOT;
  for (int li = A.nlev - 1; li >= 0; li--) {
    const int n = A.lv_ids[li + 1] - A.lv_ids[li];
    const int *ids = A.lists + A.lv_ids[li];
    const int per = 4 * NC;
    for (int q = threadIdx.x; q < n * per; q += blockDim.x) {
      const int b = q / per, r = q - b * per;
      const int id = ids[b];
      const DBox &m = A.box[id];
      const int nc = m.nc, g2 = nc + 2;
      if (r >= 4 * nc) continue;
      const int nb = r / nc, k = r % nc + 1, dim = nb >> 1;
      int gi, gj;
      if (dim == 0) { gi = (nb & 1) ? nc + 1 : 0; gj = k; }
      else { gi = k; gj = (nb & 1) ? nc + 1 : 0; }
      const size_t gix = (size_t)id * SLOT + gi + g2 * gj;
      const double g = lam[gix];
      if (g == 0.0) continue;
      lam[gix] = 0.0;
      const int nb_id = m.nb[nb];
      if (nb_id > 0) {
        const int ncn = A.box[nb_id].nc;
        int si = gi, sj = gj;
        if (dim == 0) si = (nb & 1) ? 1 : ncn;
        else sj = (nb & 1) ? 1 : ncn;
        atomicAdd(&lam[(size_t)nb_id * SLOT + si + (ncn + 2) * sj], g);
      } else if (nb_id == 0) {
        int o0, o1;
        if (m.lvl > 1) {
          o0 = ((m.ix0 - 1) & 1) * (nc >> 1) - nbdx(nb) * nc;
          o1 = ((m.ix1 - 1) & 1) * (nc >> 1) - nbdy(nb) * nc;
        } else {
          o0 = -nbdx(nb) * (nc >> 1);
          o1 = -nbdy(nb) * (nc >> 1);
        }
        const int pn = m.parent > 0 ? A.box[m.parent].nb[nb] : 0;
        if (pn <= 0) continue;  // not a refinement boundary of a valid tree
        const int gp = A.box[pn].nc + 2;
        const int ix_f = (nb & 1) ? nc : 1, ix_c = (nb & 1) ? 1 : nc;
        const int a1 = (dim == 0 ? o1 : o0) + ((k + 1) >> 1);
        const int a2 = a1 + 1 - 2 * (k & 1);
        size_t s1, s2, sf;
        if (dim == 0) {
          s1 = (size_t)pn * SLOT + ix_c + gp * a1;
          s2 = (size_t)pn * SLOT + ix_c + gp * a2;
          sf = (size_t)id * SLOT + ix_f + g2 * k;
        } else {
          s1 = (size_t)pn * SLOT + a1 + gp * ix_c;
          s2 = (size_t)pn * SLOT + a2 + gp * ix_c;
          sf = (size_t)id * SLOT + k + g2 * ix_f;
        }
        const double c1 = X[s1], c2 = X[s2], f = X[sf];
        const double v = 0.5 * c1 + sixth * c2 + third * f;
        if (v > 2 * c1) {
          atomicAdd(&lam[s1], 2 * g);
        } else {
          atomicAdd(&lam[s1], 0.5 * g);
          atomicAdd(&lam[s2], sixth * g);
          atomicAdd(&lam[sf], third * g);
        }
      } else {
        int si = gi, sj = gj;
        switch (nb) {
          case 0: si = 1; break;
          case 1: si = nc; break;
          case 2: sj = 1; break;
          default: sj = nc; break;
        }
        atomicAdd(&lam[(size_t)id * SLOT + si + g2 * sj], g);
      }
    }
    __syncthreads();
  }
}

// compute_fld's transpose: ghost cells of |E|, the cell |E|, the faces, the
// FMG, the space charge.
__device__ void adj_compute_fld(const AdjArgs &A, const double *ff, int fmg_seg) {
  seg_rev(A, SEG_GCFLD);
  adj_fld_norm(A, ff);
  seg_rev(A, SEG_FACES);
  seg_rev(A, fmg_seg);
  seg_rev(A, SEG_RHS);
}

__device__ void zero_smem_tbl(double *s_tbl, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) s_tbl[k] = 0;
  __syncthreads();
}
__device__ void flush_smem_tbl(const AdjArgs &A, const double *s_tbl, int n) {
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) A.lam_tbl[k] += s_tbl[k];
}

// The reverse of one full time step (src/streamer_2d.f90:93-128).
__global__ void __launch_bounds__(ATHR) adj_step_kernel(AdjArgs A, StepSnap S) {
  extern __shared__ double s_tbl[];
  const int nt = 4 * A.tbl_rows;
  zero_smem_tbl(s_tbl, nt);
  // final compute_fld
  adj_compute_fld(A, S.ff3, SEG_FMG);
  seg_rev(A, SEG_AVG);
  // stage 2
  adj_gc_lim(A, I_PION, S.R2i);
  adj_gc_lim(A, I_ELEC, S.R2e);
  seg_rev(A, SEG_RSTR);
  adj_update(A, s_tbl, S.F2, S.E1, S.dt);
  seg_rev(A, SEG_CONS);
  adj_fluxes(A, s_tbl, S.R1e, S.E1, S.ff1, S.dt);
  // stage 1
  adj_compute_fld(A, S.ff1, SEG_FMG);
  adj_gc_lim(A, I_PION, S.R1i);
  adj_gc_lim(A, I_ELEC, S.R1e);
  seg_rev(A, SEG_RSTR);
  adj_update(A, s_tbl, S.F1, S.E0, S.dt);
  seg_rev(A, SEG_CONS);
  adj_fluxes(A, s_tbl, S.n0, S.E0, S.ff0, S.dt);
  seg_rev(A, SEG_COPY);
  flush_smem_tbl(A, s_tbl, nt);
}

// The reverse of the first field solve (no guess).
__global__ void __launch_bounds__(ATHR) adj_init_kernel(AdjArgs A, const double *ff0) {
  adj_compute_fld(A, ff0, SEG_FMG1);
}

// ---------------------------------------------------------------------------
std::string g_aerr;
int afail(int code, const std::string &m) {
  g_aerr = m;
  a5g_internal_fail(code, m.c_str());
  return code;
}
#define ACK(call)                                                                   \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return afail(e_ == cudaErrorMemoryAllocation ? A5G_ENOMEM : A5G_ECUDA,        \
                   std::string(#call) + ": " + cudaGetErrorString(e_));             \
  } while (0)
#define ARC(call)            \
  do {                       \
    int r_ = (call);         \
    if (r_) return r_;       \
  } while (0)

template <class T>
int dupload(T *&dev, const std::vector<T> &v, cudaStream_t s) {
  ACK(cudaMalloc(&dev, std::max<size_t>(1, v.size()) * sizeof(T)));
  if (!v.empty()) ACK(cudaMemcpyAsync(dev, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return A5G_OK;
}

// Head profile (host): leaf cells next to x = x0 on either side.
struct PCell { int id, i, j; double y, w; };
static std::vector<PCell> head_profile(const Topo &T, double x0) {
  std::vector<PCell> out;
  for (int lvl = T.min_lvl; lvl <= T.max_lvl; lvl++)
    for (int id : T.L_leaves(lvl)) {
      const HBox &b = T.b[id];
      const double tol = 1e-9 * b.dr;
      int i = 0;
      if (std::fabs(b.r0 + b.nc * b.dr - x0) <= tol) i = b.nc;
      else if (std::fabs(b.r0 - x0) <= tol) i = 1;
      if (!i) continue;
      for (int j = 1; j <= b.nc; j++) out.push_back({id, i, j, b.r1 + (j - 0.5) * b.dr, b.dr});
    }
  return out;
}

}  // namespace

struct a5a_ctx {
  a5g_ctx *run = nullptr;
  a5a_params p{};
  std::vector<double> dts;
  cudaStream_t stream = nullptr;
  int cap = 0, n_rows = 0;
  Topo T;
  Ix X;
  Tape tape;
  int seg[N_SEG + 1] = {};
  std::vector<PCell> prof;
  // device storage
  int *d_phase_row = nullptr, *d_row_term = nullptr, *d_lists = nullptr;
  uint32_t *d_row_d = nullptr, *d_term_s = nullptr;
  double *d_row_self = nullptr, *d_term_c = nullptr;
  DBox *d_box = nullptr;
  double *lam = nullptr, *lam_tbl = nullptr, *tbl = nullptr;
  double *init = nullptr;       // the program's initial state (full run state)
  double *ckpt = nullptr;       // stored states, n_ckpt of them
  double *snap = nullptr;       // intermediate fields of checkpoint_every steps
  double *endst = nullptr;      // the end state
  int n_ckpt = 0;
  size_t state_n = 0, snap_step_n = 0;
  AdjArgs args{};
};

namespace {

// Full state of a run: all cell variables, then fx and fy of both face variables.
int state_copy(a5a_ctx *a, double *dst, bool to_run) {
  A5View v;
  ARC(a5g_internal_view(a->run, &v));
  const size_t ncc = (size_t)NVC * a->cap * SLOT, nf = 2 * (size_t)a->cap * FSLOT;
  cudaStream_t s = a->stream;
  if (to_run) {
    ACK(cudaMemcpyAsync(v.cc, dst, ncc * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ACK(cudaMemcpyAsync(v.fx, dst + ncc, nf * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ACK(cudaMemcpyAsync(v.fy, dst + ncc + nf, nf * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else {
    ACK(cudaMemcpyAsync(dst, v.cc, ncc * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ACK(cudaMemcpyAsync(dst + ncc, v.fx, nf * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ACK(cudaMemcpyAsync(dst + ncc + nf, v.fy, nf * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  return A5G_OK;
}

// Snapshot layout per step (offsets in doubles): 7 cell blocks, 5 face pairs.
enum { SN_N0 = 0, SN_E0, SN_R1E, SN_R1I, SN_E1, SN_R2E, SN_R2I, SN_NCELL };
enum { SF_FF0 = 0, SF_F1, SF_FF1, SF_F2, SF_FF3, SN_NFACE };
double *snap_cell(a5a_ctx *a, int k, int w) {
  return a->snap + a->snap_step_n * k + (size_t)w * a->cap * SLOT;
}
double *snap_face(a5a_ctx *a, int k, int w) {
  return a->snap + a->snap_step_n * k + (size_t)SN_NCELL * a->cap * SLOT +
         (size_t)w * 2 * a->cap * FSLOT;
}
int save_cell(a5a_ctx *a, double *dst, int iv) {
  A5View v;
  ARC(a5g_internal_view(a->run, &v));
  ACK(cudaMemcpyAsync(dst, v.cc + (size_t)iv * a->cap * SLOT, (size_t)a->cap * SLOT * sizeof(double),
                      cudaMemcpyDeviceToDevice, a->stream));
  return A5G_OK;
}
int save_face(a5a_ctx *a, double *dst, int f) {
  A5View v;
  ARC(a5g_internal_view(a->run, &v));
  const size_t nf = (size_t)a->cap * FSLOT;
  ACK(cudaMemcpyAsync(dst, v.fx + f * nf, nf * sizeof(double), cudaMemcpyDeviceToDevice, a->stream));
  ACK(cudaMemcpyAsync(dst + nf, v.fy + f * nf, nf * sizeof(double), cudaMemcpyDeviceToDevice,
                      a->stream));
  return A5G_OK;
}

// One time step through the run's operations, storing the fields the reverse
// step reads (the step sequence of src/streamer_2d.f90:93-128).
int step_recorded(a5a_ctx *a, int k, double dt) {
  a5g_ctx *c = a->run;
  ARC(save_cell(a, snap_cell(a, k, SN_N0), I_ELEC));
  ARC(save_cell(a, snap_cell(a, k, SN_E0), I_FLD));
  ARC(save_face(a, snap_face(a, k, SF_FF0), F_FLD));
  ARC(a5g_tree_copy_cc(c, I_ELEC, I_ELEC_OLD));
  ARC(a5g_tree_copy_cc(c, I_PION, I_PION_OLD));
  for (int st = 1; st <= 2; st++) {
    ARC(a5g_fluxes_koren(c, dt));
    ARC(a5g_consistent_fluxes(c));
    ARC(save_face(a, snap_face(a, k, st == 1 ? SF_F1 : SF_F2), F_ELEC));
    ARC(a5g_update_solution(c, dt));
    ARC(a5g_restrict_tree(c, I_ELEC));
    ARC(a5g_restrict_tree(c, I_PION));
    ARC(a5g_gc_tree(c, I_ELEC, 0));
    ARC(a5g_gc_tree(c, I_PION, 0));
    ARC(save_cell(a, snap_cell(a, k, st == 1 ? SN_R1E : SN_R2E), I_ELEC));
    ARC(save_cell(a, snap_cell(a, k, st == 1 ? SN_R1I : SN_R2I), I_PION));
    if (st == 1) {
      ARC(a5g_compute_fld(c, 0));
      ARC(save_cell(a, snap_cell(a, k, SN_E1), I_FLD));
      ARC(save_face(a, snap_face(a, k, SF_FF1), F_FLD));
    }
  }
  ARC(a5g_average_dens(c));
  ARC(a5g_compute_fld(c, 0));
  ARC(save_face(a, snap_face(a, k, SF_FF3), F_FLD));
  return A5G_OK;
}

int check_run(a5g_ctx *run, A5View &v) {
  ARC(a5g_internal_view(run, &v));
  if (!v.topo) return afail(A5G_ESTATE, "the run has no tree");
  if (!v.has_table) return afail(A5G_ESTATE, "the run has no table");
  if (v.coord != 0) return afail(A5G_EINVAL, "the adjoint supports Cartesian runs only");
  if (v.precision != 0) return afail(A5G_EINVAL, "the adjoint supports FP64 runs only");
  if (v.photoi_enabled) return afail(A5G_EINVAL, "the adjoint does not support photoionization");
  if (v.has_lsf) return afail(A5G_EINVAL, "the adjoint does not support level-set boundaries");
  if (v.epsilon_diel != 1.0) return afail(A5G_EINVAL, "the adjoint does not support dielectrics");
  if (v.tbl_cols != 4) return afail(A5G_EINVAL, "table must have 4 columns");
  return A5G_OK;
}

// J and dJ/d|E| of the end state (host).
int observable(a5a_ctx *a, double *J, std::vector<double> *dJ) {
  A5View v;
  ARC(a5g_internal_view(a->run, &v));
  std::vector<double> E((size_t)a->cap * SLOT);
  ACK(cudaMemcpyAsync(E.data(), v.cc + (size_t)I_FLD * a->cap * SLOT, E.size() * sizeof(double),
                      cudaMemcpyDeviceToHost, a->stream));
  ACK(cudaStreamSynchronize(a->stream));
  const auto &P = a->prof;
  if (P.empty()) return afail(A5G_EINVAL, "no leaf cell next to the line x = x0");
  auto val = [&](const PCell &c) { return E[(size_t)c.id * SLOT + c.i + (a->T.b[c.id].nc + 2) * c.j]; };
  double m = -1.7976931348623157e308;
  for (const PCell &c : P) m = std::max(m, val(c));
  double sw = 0, swy = 0;
  std::vector<double> w(P.size());
  for (size_t k = 0; k < P.size(); k++) {
    w[k] = P[k].w * std::exp((val(P[k]) - m) / a->p.temperature);
    sw += w[k];
    swy += w[k] * P[k].y;
  }
  *J = swy / sw;
  if (!std::isfinite(*J)) return afail(A5G_ENONFINITE, "observable is not finite");
  if (dJ) {
    dJ->assign((size_t)a->cap * SLOT, 0.0);
    for (size_t k = 0; k < P.size(); k++)
      (*dJ)[(size_t)P[k].id * SLOT + P[k].i + (a->T.b[P[k].id].nc + 2) * P[k].j] +=
          w[k] * (P[k].y - *J) / (a->p.temperature * sw);
  }
  return A5G_OK;
}

// Forward pass: initial solve and n_steps steps; stores a state every
// checkpoint_every steps when store.
int forward(a5a_ctx *a, bool store) {
  ARC(state_copy(a, a->init, true));
  ARC(a5g_compute_fld(a->run, 1));
  const int E = a->p.checkpoint_every;
  for (int k = 0; k < a->p.n_steps; k++) {
    if (store && k % E == 0) ARC(state_copy(a, a->ckpt + a->state_n * (k / E), false));
    ARC(a5g_step(a->run, a->dts[k]));
  }
  ARC(state_copy(a, a->endst, false));
  return A5G_OK;
}

}  // namespace

extern "C" {

int a5a_create(a5g_ctx *run, const a5a_params *p, const double *dts, a5a_ctx **out) {
  if (!run || !p || !dts || !out) return afail(A5G_EINVAL, "null argument");
  *out = nullptr;
  if (p->n_steps < 1 || p->checkpoint_every < 1) return afail(A5G_EINVAL, "n_steps and checkpoint_every must be >= 1");
  if (!(p->temperature > 0)) return afail(A5G_EINVAL, "temperature must be > 0");
  for (int k = 0; k < p->n_steps; k++)
    if (!(dts[k] > 0) || !std::isfinite(dts[k])) return afail(A5G_EINVAL, "step sizes must be > 0");
  A5View v;
  ARC(check_run(run, v));
  const A5Topo &tp = *v.topo;
  if (tp.max_lvl - tp.min_lvl + 1 > 40) return afail(A5G_EINVAL, "too many levels");
  a5a_ctx *a = new a5a_ctx();
  a->run = run;
  a->p = *p;
  a->dts.assign(dts, dts + p->n_steps);
  a->stream = (cudaStream_t)v.stream;
  a->cap = v.capacity;
  a->n_rows = v.tbl_rows;
  topo_from_upload(tp.max_id, tp.min_lvl, tp.max_lvl, tp.meta16.data(), tp.geom4.data(), tp.ids,
                   tp.leaves, tp.parents, a->cap, a->T);
  a->X.init(a->cap);
  std::string e = build_tape(a->T, a->X, v.n_cycle_base, a->tape, a->seg);
  if (!e.empty()) {
    delete a;
    return afail(A5G_EINVAL, "adjoint phases: " + e);
  }
  a->prof = head_profile(a->T, p->x0);
  if (a->prof.empty()) {
    delete a;
    return afail(A5G_EINVAL, "no leaf cell next to the line x = x0");
  }
  int r = [&]() -> int {
    cudaStream_t s = a->stream;
    ARC(dupload(a->d_phase_row, a->tape.phase_row, s));
    ARC(dupload(a->d_row_d, a->tape.row_d, s));
    ARC(dupload(a->d_row_self, a->tape.row_self, s));
    ARC(dupload(a->d_row_term, a->tape.row_term, s));
    ARC(dupload(a->d_term_s, a->tape.term_s, s));
    ARC(dupload(a->d_term_c, a->tape.term_c, s));
    std::vector<DBox> db(a->T.max_id + 1);
    std::memset(db.data(), 0, db.size() * sizeof(DBox));
    for (int id = 1; id <= a->T.max_id; id++) {
      const HBox &b = a->T.b[id];
      if (!b.in_use) continue;
      db[id].lvl = b.lvl;
      db[id].nc = b.nc;
      db[id].parent = b.parent;
      for (int q = 0; q < 4; q++) {
        db[id].ch[q] = b.ch[q];
        db[id].nb[q] = b.nb[q];
      }
      db[id].ix0 = b.ix0;
      db[id].ix1 = b.ix1;
      db[id].dr = b.dr;
      db[id].r0 = b.r0;
      db[id].r1 = b.r1;
    }
    ARC(dupload(a->d_box, db, s));
    std::vector<int> lists;
    AdjArgs &A = a->args;
    const int nlev = a->T.max_lvl - a->T.min_lvl + 1;
    for (int li = 0; li < nlev; li++) {
      A.lv_ids[li] = (int)lists.size();
      lists.insert(lists.end(), a->T.ids[li].begin(), a->T.ids[li].end());
    }
    A.lv_ids[nlev] = (int)lists.size();
    for (int li = 0; li < nlev; li++) {
      A.lv_leaves[li] = (int)lists.size();
      lists.insert(lists.end(), a->T.leaves[li].begin(), a->T.leaves[li].end());
    }
    A.lv_leaves[nlev] = (int)lists.size();
    ARC(dupload(a->d_lists, lists, s));
    a->X.init(a->cap);
    ACK(cudaMalloc(&a->lam, a->X.total * sizeof(double)));
    ACK(cudaMalloc(&a->lam_tbl, 4 * (size_t)a->n_rows * sizeof(double)));
    ACK(cudaMalloc(&a->tbl, 4 * (size_t)a->n_rows * sizeof(double)));
    a->state_n = (size_t)NVC * a->cap * SLOT + 4 * (size_t)a->cap * FSLOT;
    a->snap_step_n = (size_t)SN_NCELL * a->cap * SLOT + (size_t)SN_NFACE * 2 * a->cap * FSLOT;
    a->n_ckpt = (p->n_steps + p->checkpoint_every - 1) / p->checkpoint_every;
    ACK(cudaMalloc(&a->init, a->state_n * sizeof(double)));
    ACK(cudaMalloc(&a->endst, a->state_n * sizeof(double)));
    ACK(cudaMalloc(&a->ckpt, a->state_n * a->n_ckpt * sizeof(double)));
    ACK(cudaMalloc(&a->snap, a->snap_step_n * std::min(p->checkpoint_every, p->n_steps) * sizeof(double)));
    ARC(state_copy(a, a->init, false));
    A.phase_row = a->d_phase_row;
    A.row_d = a->d_row_d;
    A.row_self = a->d_row_self;
    A.row_term = a->d_row_term;
    A.term_s = a->d_term_s;
    A.term_c = a->d_term_c;
    for (int k = 0; k <= N_SEG; k++) A.seg[k] = a->seg[k];
    A.box = a->d_box;
    A.lists = a->d_lists;
    A.min_lvl = a->T.min_lvl;
    A.max_lvl = a->T.max_lvl;
    A.nlev = nlev;
    A.cap = a->cap;
    A.lam = a->lam;
    A.lam_tbl = a->lam_tbl;
    A.tbl = a->tbl;
    A.tbl_rows = a->n_rows;
    A.tbl_xmin = v.tbl_xmin;
    A.tbl_inv_dx = v.tbl_inv_dx;
    ACK(cudaFuncSetAttribute(adj_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(4 * a->n_rows * sizeof(double))));
    ACK(cudaStreamSynchronize(s));
    return A5G_OK;
  }();
  if (r) {
    a5a_destroy(a);
    return r;
  }
  if (4 * (size_t)a->n_rows * sizeof(double) > 200 * 1024) {
    a5a_destroy(a);
    return afail(A5G_EINVAL, "table too large for the adjoint's shared accumulator");
  }
  *out = a;
  return A5G_OK;
}

int a5a_destroy(a5a_ctx *a) {
  if (!a) return A5G_OK;
  if (a->stream) cudaStreamSynchronize(a->stream);
  cudaFree(a->d_phase_row);
  cudaFree(a->d_row_d);
  cudaFree(a->d_row_self);
  cudaFree(a->d_row_term);
  cudaFree(a->d_term_s);
  cudaFree(a->d_term_c);
  cudaFree(a->d_box);
  cudaFree(a->d_lists);
  cudaFree(a->lam);
  cudaFree(a->lam_tbl);
  cudaFree(a->tbl);
  cudaFree(a->init);
  cudaFree(a->endst);
  cudaFree(a->ckpt);
  cudaFree(a->snap);
  delete a;
  return A5G_OK;
}

int a5a_forward(a5a_ctx *a, double *J) {
  if (!a || !J) return afail(A5G_EINVAL, "null argument");
  A5View v;
  ARC(check_run(a->run, v));
  if (v.capacity != a->cap) return afail(A5G_ESTATE, "the run's storage changed since a5a_create");
  ARC(forward(a, false));
  return observable(a, J, nullptr);
}

int a5a_gradient(a5a_ctx *a, double *J, double *dJ_dtable, double *dJ_dV) {
  if (!a || !J || !dJ_dtable || !dJ_dV) return afail(A5G_EINVAL, "null argument");
  A5View v;
  ARC(check_run(a->run, v));
  if (v.capacity != a->cap) return afail(A5G_ESTATE, "the run's storage changed since a5a_create");
  if (v.tbl_rows != a->n_rows) return afail(A5G_ESTATE, "the run's table size changed");
  cudaStream_t s = a->stream;
  AdjArgs &A = a->args;
  A.tbl_xmin = v.tbl_xmin;
  A.tbl_inv_dx = v.tbl_inv_dx;
  ACK(cudaMemcpyAsync(a->tbl, v.tbl_host, 4 * (size_t)a->n_rows * sizeof(double),
                      cudaMemcpyHostToDevice, s));
  // forward pass with stored states
  ARC(forward(a, true));
  std::vector<double> seed;
  ARC(observable(a, J, &seed));
  // seed: dJ/d|E| of the end state, every other adjoint 0
  ACK(cudaMemsetAsync(a->lam, 0, a->X.total * sizeof(double), s));
  ACK(cudaMemsetAsync(a->lam_tbl, 0, 4 * (size_t)a->n_rows * sizeof(double), s));
  ACK(cudaMemcpyAsync(a->lam + (size_t)I_FLD * a->cap * SLOT, seed.data(), seed.size() * sizeof(double),
                      cudaMemcpyHostToDevice, s));
  const int E = a->p.checkpoint_every;
  const size_t smem = 4 * (size_t)a->n_rows * sizeof(double);
  for (int c = a->n_ckpt - 1; c >= 0; c--) {
    const int k0 = c * E, k1 = std::min(a->p.n_steps, k0 + E);
    ARC(state_copy(a, a->ckpt + a->state_n * c, true));
    for (int k = k0; k < k1; k++) ARC(step_recorded(a, k - k0, a->dts[k]));
    for (int k = k1 - 1; k >= k0; k--) {
      const int q = k - k0;
      StepSnap S;
      S.n0 = snap_cell(a, q, SN_N0);
      S.E0 = snap_cell(a, q, SN_E0);
      S.ff0 = snap_face(a, q, SF_FF0);
      S.F1 = snap_face(a, q, SF_F1);
      S.R1e = snap_cell(a, q, SN_R1E);
      S.R1i = snap_cell(a, q, SN_R1I);
      S.E1 = snap_cell(a, q, SN_E1);
      S.ff1 = snap_face(a, q, SF_FF1);
      S.F2 = snap_face(a, q, SF_F2);
      S.R2e = snap_cell(a, q, SN_R2E);
      S.R2i = snap_cell(a, q, SN_R2I);
      S.ff3 = snap_face(a, q, SF_FF3);
      S.dt = a->dts[k];
      adj_step_kernel<<<1, ATHR, smem, s>>>(A, S);
      ACK(cudaGetLastError());
    }
  }
  // the first field solve: its faces are step 0's starting faces (interval 0
  // was recomputed last)
  adj_init_kernel<<<1, ATHR, 0, s>>>(A, snap_face(a, 0, SF_FF0));
  ACK(cudaGetLastError());
  ARC(state_copy(a, a->endst, true));
  ACK(cudaMemcpyAsync(dJ_dtable, a->lam_tbl, 4 * (size_t)a->n_rows * sizeof(double),
                      cudaMemcpyDeviceToHost, s));
  ACK(cudaMemcpyAsync(dJ_dV, a->lam + a->X.v, sizeof(double), cudaMemcpyDeviceToHost, s));
  ACK(cudaStreamSynchronize(s));
  for (int k = 0; k < 4 * a->n_rows; k++)
    if (!std::isfinite(dJ_dtable[k])) return afail(A5G_ENONFINITE, "gradient is not finite");
  return A5G_OK;
}

int a5a_debug_tape(int max_id, int min_lvl, int max_lvl, const int *meta16, const double *geom4,
                   const int *lvl_counts, const int *lvl_ids, int capacity, int n_cycle_base,
                   int seg, long long *sizes, int *phase_row, unsigned *row_d, double *row_self,
                   int *row_term, unsigned *term_s, double *term_c) {
  if (!meta16 || !geom4 || !lvl_counts || !lvl_ids || !sizes) return afail(A5G_EINVAL, "null argument");
  if (seg < 0 || seg >= N_SEG) return afail(A5G_EINVAL, "bad segment");
  const int nlev = max_lvl - min_lvl + 1;
  if (nlev < 1 || capacity < max_id + 1) return afail(A5G_EINVAL, "bad levels or capacity");
  std::vector<std::vector<int>> ids(nlev), leaves(nlev), parents(nlev);
  size_t k = 0;
  for (int li = 0; li < nlev; li++) {
    for (int q = 0; q < lvl_counts[3 * li]; q++) ids[li].push_back(lvl_ids[k++]);
    for (int q = 0; q < lvl_counts[3 * li + 1]; q++) leaves[li].push_back(lvl_ids[k++]);
    for (int q = 0; q < lvl_counts[3 * li + 2]; q++) parents[li].push_back(lvl_ids[k++]);
  }
  Topo T;
  topo_from_upload(max_id, min_lvl, max_lvl, meta16, geom4, ids, leaves, parents, capacity, T);
  Ix X;
  X.init(capacity);
  Tape tp;
  int sp[N_SEG + 1];
  std::string e = build_tape(T, X, n_cycle_base, tp, sp);
  if (!e.empty()) return afail(A5G_EINVAL, "adjoint phases: " + e);
  const int p0 = sp[seg], p1 = sp[seg + 1];
  const int r0 = tp.phase_row[p0], r1 = tp.phase_row[p1];
  const int t0 = tp.row_term[r0], t1 = tp.row_term[r1];
  sizes[0] = p1 - p0;
  sizes[1] = r1 - r0;
  sizes[2] = t1 - t0;
  sizes[3] = (long long)X.total;
  if (phase_row)
    for (int p = p0; p <= p1; p++) phase_row[p - p0] = tp.phase_row[p] - r0;
  if (row_d)
    for (int r = r0; r < r1; r++) {
      row_d[r - r0] = tp.row_d[r];
      if (row_self) row_self[r - r0] = tp.row_self[r];
    }
  if (row_term)
    for (int r = r0; r <= r1; r++) row_term[r - r0] = tp.row_term[r] - t0;
  if (term_s)
    for (int t = t0; t < t1; t++) {
      term_s[t - t0] = tp.term_s[t];
      if (term_c) term_c[t - t0] = tp.term_c[t];
    }
  return A5G_OK;
}

}  // extern "C"
