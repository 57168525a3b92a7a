// a5ref — CPU oracle (test infrastructure only) for a5_streamer's per-timestep
// path. Plain C++ restatement of the reference's Fortran; every routine cites
// the reference file:line it follows (paths relative to the reference repo).
// Parity with the reference binary is UNPINNED: the reference is Fortran and
// cannot be compiled here, and ships no golden vectors (see a5ref.h).
//
// Conventions kept from the reference:
//  * box ids are 1-based, 0 = no box, negative = physical boundary;
//  * cell arrays are (0:nc+1, 0:nc+1, n_var), i fastest;
//  * face arrays fx(1:nc+1, 1:nc, n_f), fy(1:nc, 1:nc+1, n_f);
//  * loops run j outer, i inner (Fortran column-major order);
//  * children / neighbour directions are 0-based here (lx, hx, ly, hy).
#include "a5ref.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace a5ref {

// ---------------------------------------------------------------------------
// Topology tables, afivo/src/m_aX_t.f90:41-81 (2D), 0-based.
static const int NCH = 4, NNB = 4;
static const int ch_dix[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
static const int ch_rev[4][2] = {{1, 2}, {0, 3}, {3, 0}, {2, 1}};
static const int ch_adj_nb[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};
static const int nb_dix[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
static const bool nb_low[4] = {true, false, true, false};
static const int nb_hi01[4] = {0, 1, 0, 1};
static const int nb_rev[4] = {1, 0, 3, 2};
static const int nb_dim[4] = {0, 0, 1, 1};
enum { NB_LX = 0, NB_HX = 1, NB_LY = 2, NB_HY = 3 };

// Refinement flag values, afivo/src/m_aX_t.f90:13-26.
static const int RM_REF = -1, KP_REF = 0, DO_REF = 1, DEREFINE = -2,
                 REFINE = 2, NO_BOX = 0;
static const int INIT_TAG = -INT_MAX;
static const int XYZ = 0, CYL = 1;

// Streamer variable indices, src/m_streamer.f90:17-43 (0-based).
// I_LSF, I_BVAL: level-set function and boundary value of the level-set
// multigrid operators (unused unless a level set is set)
enum { I_ELEC = 0, I_PION, I_ELEC_OLD, I_PION_OLD, I_PHI, I_FLD, I_RHS,
       I_PHO, I_EPS, I_LSF, I_BVAL, N_VAR_CELL };
enum { F_ELEC = 0, F_FLD, N_VAR_FACE };
enum { I_MOBILITY = 0, I_DIFFUSION, I_ALPHA, I_ETA };

// fosito/m_units_constants.f90:201-202
static const double UC_EPS0 = 8.8541878176e-12;
static const double UC_ELEM_CHARGE = 1.6022e-19;

// ---------------------------------------------------------------------------
struct Box {
  int lvl = 0;
  bool in_use = false;
  int tag = INIT_TAG;
  int ix[2] = {0, 0};
  int parent = 0;
  int children[4] = {0, 0, 0, 0};
  int neighbors[4] = {0, 0, 0, 0};
  int n_cell = 0;
  double dr = 0;
  double r_min[2] = {0, 0};
  int coord = XYZ;
  std::vector<double> cc, fx, fy;

  int ncg() const { return n_cell + 2; }
  double &c(int i, int j, int v) { return cc[i + ncg() * (j + ncg() * v)]; }
  double c(int i, int j, int v) const { return cc[i + ncg() * (j + ncg() * v)]; }
  double &Fx(int i, int j, int f) {
    return fx[(i - 1) + (n_cell + 1) * ((j - 1) + n_cell * f)];
  }
  double &Fy(int i, int j, int f) {
    return fy[(i - 1) + n_cell * ((j - 1) + (n_cell + 1) * f)];
  }
};

struct Level {
  std::vector<int> ids, leaves, parents;
};

struct Tree {
  int lvls_max = 30, max_lvl = 0, max_id = 0, n_cell = 0;
  int n_var_cell = 0, n_var_face = 0, coord = XYZ, min_lvl = 1;
  double r_base[2] = {0, 0}, dr_base = 0;
  std::vector<Level> lv;      // index lvl - min_lvl, lvl in min_lvl..lvls_max+1
  std::vector<Box> boxes;     // index = id, boxes[0] unused
  Level &L(int lvl) { return lv[lvl - min_lvl]; }
};

static inline bool has_children(const Box &b) { return b.children[0] != NO_BOX; }

// afivo/src/m_aX_core.f90:363-381 (init_box); storage zeroed for determinism.
static void init_box(Box &b, int n_cell, int n_cc, int n_fc) {
  b.in_use = true;
  b.cc.assign((size_t)(n_cell + 2) * (n_cell + 2) * n_cc, 0.0);
  b.fx.assign((size_t)(n_cell + 1) * n_cell * std::max(n_fc, 1), 0.0);
  b.fy.assign((size_t)(n_cell + 1) * n_cell * std::max(n_fc, 1), 0.0);
}

static void clear_box(Box &b) {
  b.in_use = false;
  b.cc.clear(); b.cc.shrink_to_fit();
  b.fx.clear(); b.fx.shrink_to_fit();
  b.fy.clear(); b.fy.shrink_to_fit();
}

// afivo/src/m_aX_core.f90:47-116 (a$D_init)
static void tree_init(Tree &t, int n_cell, int n_var_cell, int n_var_face,
                      double dr, const double r_min[2], int lvls_max,
                      int coarsen_to, int coord) {
  int min_lvl = 1;
  if (coarsen_to > 0) {
    min_lvl = 1 - (int)std::lround(std::log((double)n_cell / coarsen_to) /
                                   std::log(2.0));
  }
  t.min_lvl = min_lvl;
  t.lv.assign(lvls_max + 2 - min_lvl, Level());
  t.n_cell = n_cell;
  t.n_var_cell = n_var_cell;
  t.n_var_face = n_var_face;
  t.r_base[0] = r_min[0];
  t.r_base[1] = r_min[1];
  t.dr_base = dr;
  t.lvls_max = lvls_max;
  t.max_id = 0;
  t.max_lvl = 0;
  t.coord = coord;
  t.boxes.assign(1, Box());
}

static void get_free_ids(Tree &t, int n, int *ids) {
  int prev = t.max_id;
  t.max_id += n;
  if ((int)t.boxes.size() < t.max_id + 1) t.boxes.resize(t.max_id + 1);
  for (int i = 0; i < n; i++) ids[i] = prev + 1 + i;
}

// afivo/src/m_aX_core.f90:134-217 (a$D_set_base). nb_list entries: box index
// (1-based within ix_list), or negative for a physical boundary.
static void set_base(Tree &t, int n_boxes, const int (*ix_list)[2],
                     std::vector<std::array<int, 4>> nb_list) {
  for (int i = 0; i < n_boxes; i++)
    for (int nb = 0; nb < NNB; nb++) {
      int nb_id = nb_list[i][nb];
      if (nb_id > NO_BOX && nb_id != i + 1) nb_list[nb_id - 1][nb_rev[nb]] = i + 1;
    }
  for (int lvl = t.min_lvl; lvl <= 1; lvl++) {
    Level &L = t.L(lvl);
    L.ids.assign(n_boxes, 0);
    get_free_ids(t, n_boxes, L.ids.data());
    int offset = L.ids[0] - 1;
    for (int i = 0; i < n_boxes; i++) {
      int id = L.ids[i];
      Box &b = t.boxes[id];
      b.lvl = lvl;
      b.ix[0] = ix_list[i][0];
      b.ix[1] = ix_list[i][1];
      b.dr = t.dr_base * std::pow(0.5, lvl - 1);
      for (int d = 0; d < 2; d++)
        b.r_min[d] = t.r_base[d] + (ix_list[i][d] - 1) * t.dr_base * t.n_cell;
      b.n_cell = t.n_cell / (1 << (1 - lvl));
      b.coord = t.coord;
      b.parent = NO_BOX;
      for (int c = 0; c < NCH; c++) b.children[c] = NO_BOX;
      for (int nb = 0; nb < NNB; nb++)
        b.neighbors[nb] = nb_list[i][nb] > NO_BOX ? nb_list[i][nb] + offset
                                                   : nb_list[i][nb];
      b.tag = INIT_TAG;
      init_box(b, b.n_cell, t.n_var_cell, t.n_var_face);
    }
    if (lvl == 1) {
      L.leaves = L.ids;
      L.parents.clear();
    } else {
      L.parents = L.ids;
      L.leaves.clear();
    }
    if (lvl > t.min_lvl) {
      Level &Lm = t.L(lvl - 1);
      for (int i = 0; i < n_boxes; i++) {
        t.boxes[Lm.ids[i]].children[0] = L.ids[i];
        t.boxes[L.ids[i]].parent = Lm.ids[i];
      }
    }
  }
  t.max_lvl = 1;
}

// afivo/src/m_aX_core.f90:328-359 (set_leaves_parents)
static void set_leaves_parents(Tree &t, Level &L) {
  L.leaves.clear();
  L.parents.clear();
  for (int id : L.ids) {
    if (has_children(t.boxes[id])) L.parents.push_back(id);
    else L.leaves.push_back(id);
  }
}

// afivo/src/m_aX_core.f90:403-407 (a$D_ix_to_cix), 0-based result
static inline int ix_to_cix(const int ix[2]) {
  return 3 - 2 * (ix[1] & 1) - (ix[0] & 1);
}

// afivo/src/m_aX_core.f90:427-445 (find_nb)
static int find_nb(Tree &t, int id, int nb) {
  int p_id = t.boxes[id].parent;
  int c_ix = ix_to_cix(t.boxes[id].ix);
  int d = nb_dim[nb];
  bool ch_low = ch_dix[c_ix][d] == 0;
  if (ch_low == nb_low[nb]) p_id = t.boxes[p_id].neighbors[nb];
  return t.boxes[p_id].children[ch_rev[c_ix][d]];
}

// afivo/src/m_aX_core.f90:386-400 (set_nbs_$Dd)
static void set_nbs(Tree &t, int id) {
  for (int nb = 0; nb < NNB; nb++) {
    if (t.boxes[id].neighbors[nb] == NO_BOX) {
      int nb_id = find_nb(t, id, nb);
      if (nb_id > NO_BOX) {
        t.boxes[id].neighbors[nb] = nb_id;
        t.boxes[nb_id].neighbors[nb_rev[nb]] = id;
      }
    }
  }
}

// afivo/src/m_aX_core.f90:729-750 (remove_children)
static void remove_children(Tree &t, int id) {
  for (int ic = 0; ic < NCH; ic++) {
    int c_id = t.boxes[id].children[ic];
    for (int nb = 0; nb < NNB; nb++) {
      int nb_id = t.boxes[c_id].neighbors[nb];
      if (nb_id > NO_BOX) t.boxes[nb_id].neighbors[nb_rev[nb]] = NO_BOX;
    }
    clear_box(t.boxes[c_id]);
  }
  for (int ic = 0; ic < NCH; ic++) t.boxes[id].children[ic] = NO_BOX;
}

// afivo/src/m_aX_core.f90:753-788 (add_children)
static void add_children(Tree &t, int id, const int c_ids[4]) {
  Box &p = t.boxes[id];
  for (int i = 0; i < NCH; i++) p.children[i] = c_ids[i];
  int base[2] = {2 * p.ix[0] - 1, 2 * p.ix[1] - 1};
  for (int i = 0; i < NCH; i++) {
    Box &c = t.boxes[c_ids[i]];
    Box &pp = t.boxes[id];
    c.ix[0] = base[0] + ch_dix[i][0];
    c.ix[1] = base[1] + ch_dix[i][1];
    c.lvl = pp.lvl + 1;
    c.parent = id;
    c.tag = INIT_TAG;
    for (int k = 0; k < NCH; k++) c.children[k] = NO_BOX;
    for (int k = 0; k < NNB; k++) c.neighbors[k] = NO_BOX;
    c.n_cell = pp.n_cell;
    c.coord = pp.coord;
    c.dr = 0.5 * pp.dr;
    for (int d = 0; d < 2; d++)
      c.r_min[d] = pp.r_min[d] + 0.5 * pp.dr * ch_dix[i][d] * pp.n_cell;
    init_box(c, pp.n_cell, t.n_var_cell, t.n_var_face);
  }
  for (int nb = 0; nb < NNB; nb++) {
    int pn = t.boxes[id].neighbors[nb];
    if (pn < NO_BOX)
      for (int k = 0; k < 2; k++) t.boxes[c_ids[ch_adj_nb[nb][k]]].neighbors[nb] = pn;
  }
}

// afivo/src/m_aX_core.f90:792-815 (set_child_ids)
static void set_child_ids(Tree &t, const std::vector<int> &p_ids,
                          std::vector<int> &c_ids) {
  c_ids.assign(NCH * p_ids.size(), 0);
  for (size_t i = 0; i < p_ids.size(); i++)
    for (int k = 0; k < NCH; k++) c_ids[NCH * i + k] = t.boxes[p_ids[i]].children[k];
}

using RefFn = std::function<void(Tree &, int, std::vector<int> &)>;

// afivo/src/m_aX_core.f90:624-726 (consistent_ref_flags)
static void consistent_ref_flags(Tree &t, std::vector<int> &rf,
                                 const RefFn &set_ref_flags) {
  rf.assign(t.max_id + 1, -INT_MAX);
  for (int lvl = 1; lvl <= t.max_lvl; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) set_ref_flags(t, L.ids[i], rf);
  }
  for (int i = 1; i <= t.max_id; i++) {
    if (rf[i] > DO_REF) rf[i] = KP_REF;
    if (rf[i] < RM_REF) rf[i] = KP_REF;
  }
  for (int id : t.L(t.lvls_max).ids)
    if (rf[id] == DO_REF) rf[id] = KP_REF;
  for (int lvl = t.max_lvl; lvl >= 1; lvl--) {
    for (int id : t.L(lvl).leaves) {
      if (rf[id] > KP_REF) {
        rf[id] = REFINE;
        for (int nb = 0; nb < NNB; nb++) {
          int nb_id = t.boxes[id].neighbors[nb];
          if (nb_id == NO_BOX) {
            int p_id = t.boxes[id].parent;
            int p_nb_id = t.boxes[p_id].neighbors[nb];
            rf[p_nb_id] = REFINE;
          }
        }
      } else if (rf[id] == RM_REF) {
        for (int nb = 0; nb < NNB; nb++) {
          int nb_id = t.boxes[id].neighbors[nb];
          if (nb_id > NO_BOX) {
            if (has_children(t.boxes[nb_id]) || rf[nb_id] > KP_REF) {
              rf[id] = KP_REF;
              break;
            }
          }
        }
      }
    }
  }
  for (int lvl = t.max_lvl - 1; lvl >= 1; lvl--) {
    for (int id : t.L(lvl).parents) {
      bool all_rm = true;
      for (int k = 0; k < NCH; k++)
        if (rf[t.boxes[id].children[k]] != RM_REF) all_rm = false;
      if (all_rm && rf[id] <= KP_REF) rf[id] = DEREFINE;
      else rf[id] = KP_REF;
    }
  }
}

struct RefInfo {
  int n_add = 0, n_rm = 0;
  std::vector<std::vector<int>> add;  // index lvl (1..max_lvl+1)
};

// afivo/src/m_aX_core.f90:523-584 (set_ref_info)
static void set_ref_info(Tree &t, const std::vector<int> &rf, RefInfo &ri) {
  ri.n_add = ri.n_rm = 0;
  ri.add.assign(t.max_lvl + 2, std::vector<int>());
  for (int id = 1; id < (int)rf.size(); id++) {
    if (rf[id] == REFINE) {
      ri.n_add += NCH;
      int lvl = t.boxes[id].lvl;
      for (int k = 0; k < NCH; k++) ri.add[lvl + 1].push_back(t.boxes[id].children[k]);
    } else if (rf[id] == DEREFINE) {
      ri.n_rm += NCH;
    }
  }
}

// afivo/src/m_aX_core.f90:456-520 (a$D_adjust_refinement)
static void adjust_refinement(Tree &t, const RefFn &set_ref_flags, RefInfo &ri) {
  int max_id_prev = t.max_id;
  std::vector<int> rf;
  consistent_ref_flags(t, rf, set_ref_flags);
  int lvl;
  for (lvl = 1; lvl <= t.lvls_max - 1; lvl++) {
    Level &L = t.L(lvl);
    for (size_t i = 0; i < L.ids.size(); i++) {
      int id = t.L(lvl).ids[i];
      if (id > max_id_prev) continue;
      if (rf[id] == REFINE) {
        int c_ids[4];
        get_free_ids(t, NCH, c_ids);
        add_children(t, id, c_ids);
      } else if (rf[id] == DEREFINE) {
        remove_children(t, id);
      }
    }
    set_leaves_parents(t, t.L(lvl));
    set_child_ids(t, t.L(lvl).parents, t.L(lvl + 1).ids);
    for (int id : t.L(lvl + 1).ids)
      if (id > max_id_prev) set_nbs(t, id);
    if (t.L(lvl + 1).ids.empty()) break;
  }
  if (lvl > t.lvls_max - 1) lvl = t.lvls_max;
  t.max_lvl = lvl;
  set_leaves_parents(t, t.L(t.max_lvl + 1));
  set_ref_info(t, rf, ri);
}

// afivo/src/m_aX_utils.f90:227-239 (a$D_get_child_offset); nb < 0: absent
static inline void child_offset(const Box &b, int nb, int off[2]) {
  if (b.lvl > 1) {
    for (int d = 0; d < 2; d++) {
      off[d] = ((b.ix[d] - 1) & 1) * (b.n_cell >> 1);
      if (nb >= 0) off[d] -= nb_dix[nb][d] * b.n_cell;
    }
  } else {
    for (int d = 0; d < 2; d++) {
      off[d] = 0;
      if (nb >= 0) off[d] -= nb_dix[nb][d] * (b.n_cell >> 1);
    }
  }
}

// afivo/src/m_aX_utils.f90:309-314 (a$D_r_cc)
static inline void r_cc(const Box &b, int i, int j, double xy[2]) {
  xy[0] = b.r_min[0] + (i - 0.5) * b.dr;
  xy[1] = b.r_min[1] + (j - 0.5) * b.dr;
}

// gfortran's inline NORM2 (scaled sum of squares): scale = 0, ssq = 1; for
// each non-zero |x|, rescale when |x| exceeds the running scale.
static inline double norm2(const double *x, int n) {
  double scale = 0.0, ssq = 1.0;
  for (int k = 0; k < n; k++) {
    if (x[k] != 0.0) {
      double ax = std::fabs(x[k]);
      if (scale < ax) {
        double v = scale / ax;
        ssq = 1.0 + ssq * v * v;
        scale = ax;
      } else {
        double v = ax / scale;
        ssq += v * v;
      }
    }
  }
  return scale * std::sqrt(ssq);
}

// ---------------------------------------------------------------------------
// Ghost cells, afivo/src/m_aX_gc.f90
using GcFn = std::function<void(Tree &, int id, int nb, int iv)>;

// afivo/src/m_aX_gc.f90:368-402 (sides_from_nb)
static void sides_from_nb(Box &b, const Box &bn, int nb, int iv) {
  int nc = b.n_cell;
  switch (nb) {
    case NB_LX: for (int j = 1; j <= nc; j++) b.c(0, j, iv) = bn.c(nc, j, iv); break;
    case NB_HX: for (int j = 1; j <= nc; j++) b.c(nc + 1, j, iv) = bn.c(1, j, iv); break;
    case NB_LY: for (int i = 1; i <= nc; i++) b.c(i, 0, iv) = bn.c(i, nc, iv); break;
    case NB_HY: for (int i = 1; i <= nc; i++) b.c(i, nc + 1, iv) = bn.c(i, 1, iv); break;
  }
}

// afivo/src/m_aX_gc.f90:50-68 (a$D_gc_box)
static void gc_box(Tree &t, int id, int iv, const GcFn &rb, const GcFn &bc) {
  for (int nb = 0; nb < NNB; nb++) {
    int nb_id = t.boxes[id].neighbors[nb];
    if (nb_id > NO_BOX) sides_from_nb(t.boxes[id], t.boxes[nb_id], nb, iv);
    else if (nb_id == NO_BOX) rb(t, id, nb, iv);
    else bc(t, id, nb, iv);
  }
}

// afivo/src/m_aX_gc.f90:28-46 (a$D_gc_tree)
static void gc_tree(Tree &t, int iv, const GcFn &rb, const GcFn &bc) {
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) gc_box(t, L.ids[i], iv, rb, bc);
  }
}

// afivo/src/m_aX_gc.f90:90-185 (a$D_gc_interp) and 190-295 (_lim)
static void gc_interp_impl(Tree &t, int id, int nb, int iv, bool lim) {
  const double sixth = 1 / 6.0, third = 1 / 3.0;
  Box &b = t.boxes[id];
  int nc = b.n_cell;
  int p_id = b.parent;
  Box &pn = t.boxes[t.boxes[p_id].neighbors[nb]];
  int off[2];
  child_offset(b, nb, off);
  int ix, ix_f, ix_c;
  if (nb_low[nb]) { ix = 0; ix_f = 1; ix_c = nc; }
  else { ix = nc + 1; ix_f = nc; ix_c = 1; }
  if (nb_dim[nb] == 0) {
    for (int j = 1; j <= nc; j++) {
      int j_c1 = off[1] + ((j + 1) >> 1);
      int j_c2 = j_c1 + 1 - 2 * (j & 1);
      double c1 = pn.c(ix_c, j_c1, iv), c2 = pn.c(ix_c, j_c2, iv);
      double v = 0.5 * c1 + sixth * c2 + third * b.c(ix_f, j, iv);
      if (lim && v > 2 * c1) v = 2 * c1;
      b.c(ix, j, iv) = v;
    }
  } else {
    for (int i = 1; i <= nc; i++) {
      int i_c1 = off[0] + ((i + 1) >> 1);
      int i_c2 = i_c1 + 1 - 2 * (i & 1);
      double c1 = pn.c(i_c1, ix_c, iv), c2 = pn.c(i_c2, ix_c, iv);
      double v = 0.5 * c1 + sixth * c2 + third * b.c(i, ix_f, iv);
      if (lim && v > 2 * c1) v = 2 * c1;
      b.c(i, ix, iv) = v;
    }
  }
}
static void gc_interp(Tree &t, int id, int nb, int iv) { gc_interp_impl(t, id, nb, iv, false); }
static void gc_interp_lim(Tree &t, int id, int nb, int iv) { gc_interp_impl(t, id, nb, iv, true); }

// afivo/src/m_aX_gc.f90:298-330 (a$D_gc_neumann)
static void gc_neumann(Tree &t, int id, int nb, int iv) {
  Box &b = t.boxes[id];
  int nc = b.n_cell;
  switch (nb) {
    case NB_LX: for (int j = 1; j <= nc; j++) b.c(0, j, iv) = b.c(1, j, iv); break;
    case NB_HX: for (int j = 1; j <= nc; j++) b.c(nc + 1, j, iv) = b.c(nc, j, iv); break;
    case NB_LY: for (int i = 1; i <= nc; i++) b.c(i, 0, iv) = b.c(i, 1, iv); break;
    case NB_HY: for (int i = 1; i <= nc; i++) b.c(i, nc + 1, iv) = b.c(i, nc, iv); break;
  }
}

// afivo/src/m_aX_prolong.f90:37-78 (a$D_prolong0_to) over [lo, hi]
static void prolong0_to(Tree &t, int id, int iv, const int lo[2], const int hi[2]) {
  Box &b = t.boxes[id];
  const Box &p = t.boxes[b.parent];
  int off[2];
  child_offset(b, -1, off);
  for (int j = lo[1]; j <= hi[1]; j++) {
    int j_c1 = off[1] + ((j + 1) >> 1);
    for (int i = lo[0]; i <= hi[0]; i++) {
      int i_c1 = off[0] + ((i + 1) >> 1);
      b.c(i, j, iv) = p.c(i_c1, j_c1, iv);
    }
  }
}

// afivo/src/m_aX_gc.f90:71-86 (a$D_gc_prolong0)
static void gc_prolong0(Tree &t, int id, int nb, int iv) {
  int nc = t.boxes[id].n_cell;
  int d = nb_dim[nb];
  int lo[2] = {1, 1}, hi[2] = {nc, nc};
  lo[d] = nb_hi01[nb] * (nc + 1);
  hi[d] = nb_hi01[nb] * (nc + 1);
  prolong0_to(t, id, iv, lo, hi);
}

// afivo/src/m_aX_prolong.f90:99-191 (a$D_prolong1_to), add = false
static void prolong1_to(Tree &t, int id, int iv) {
  Box &b = t.boxes[id];
  const Box &p = t.boxes[b.parent];
  int nc = b.n_cell, hnc = nc >> 1;
  int off[2];
  child_offset(b, -1, off);
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) b.c(i, j, iv) = 0;
  for (int j = 1; j <= hnc; j++) {
    int j_c = j + off[1], j_f = 2 * j - 1;
    for (int i = 1; i <= hnc; i++) {
      int i_c = i + off[0], i_f = 2 * i - 1;
      double f0 = 0.5 * p.c(i_c, j_c, iv);
      double flx = 0.25 * p.c(i_c - 1, j_c, iv);
      double fhx = 0.25 * p.c(i_c + 1, j_c, iv);
      double fly = 0.25 * p.c(i_c, j_c - 1, iv);
      double fhy = 0.25 * p.c(i_c, j_c + 1, iv);
      b.c(i_f, j_f, iv) = f0 + flx + fly + b.c(i_f, j_f, iv);
      b.c(i_f + 1, j_f, iv) = f0 + fhx + fly + b.c(i_f + 1, j_f, iv);
      b.c(i_f, j_f + 1, iv) = f0 + flx + fhy + b.c(i_f, j_f + 1, iv);
      b.c(i_f + 1, j_f + 1, iv) = f0 + fhx + fhy + b.c(i_f + 1, j_f + 1, iv);
    }
  }
}

// afivo/src/m_aX_gc.f90:407-443 (a$D_gc2_box) with a$D_gc2_prolong1 (485-585)
// on refinement boundaries and a$D_gc2_neumann (588-622) on physical ones.
// gc_data[nb][k], k = 0..nc-1.
static void gc2_box(Tree &t, int id, int iv, double gc_data[4][64]) {
  Box &b = t.boxes[id];
  int nc = b.n_cell;
  for (int nb = 0; nb < NNB; nb++) {
    int nb_id = b.neighbors[nb];
    double *g = gc_data[nb];
    if (nb_id > NO_BOX) {  // sides2_from_nb, m_aX_gc.f90:446-482
      const Box &bn = t.boxes[nb_id];
      switch (nb) {
        case NB_LX: for (int j = 1; j <= nc; j++) g[j - 1] = bn.c(nc - 1, j, iv); break;
        case NB_HX: for (int j = 1; j <= nc; j++) g[j - 1] = bn.c(2, j, iv); break;
        case NB_LY: for (int i = 1; i <= nc; i++) g[i - 1] = bn.c(i, nc - 1, iv); break;
        case NB_HY: for (int i = 1; i <= nc; i++) g[i - 1] = bn.c(i, 2, iv); break;
      }
    } else if (nb_id == NO_BOX) {
      const Box &pn = t.boxes[t.boxes[b.parent].neighbors[nb]];
      int off[2];
      child_offset(b, nb, off);
      int ix = nb_hi01[nb] * (nc + 3) - 1;  // -1 or nc+2
      int hs = (ix + 1) >> 1;               // ishft(ix+1, -1); ix+1 >= 0
      int par = ix & 1;                     // iand(ix, 1), two's complement
      if (nb_dim[nb] == 0) {
        int i_c1 = off[0] + hs;
        int i_c2 = i_c1 + 1 - 2 * par;
        for (int j = 1; j <= nc; j++) {
          int j_c1 = off[1] + ((j + 1) >> 1);
          int j_c2 = j_c1 + 1 - 2 * (j & 1);
          g[j - 1] = 0.5 * pn.c(i_c1, j_c1, iv) + 0.25 * pn.c(i_c2, j_c1, iv) +
                     0.25 * pn.c(i_c1, j_c2, iv);
        }
      } else {
        int j_c1 = off[1] + hs;
        int j_c2 = j_c1 + 1 - 2 * par;
        for (int i = 1; i <= nc; i++) {
          int i_c1 = off[0] + ((i + 1) >> 1);
          int i_c2 = i_c1 + 1 - 2 * (i & 1);
          g[i - 1] = 0.5 * pn.c(i_c1, j_c1, iv) + 0.25 * pn.c(i_c2, j_c1, iv) +
                     0.25 * pn.c(i_c1, j_c2, iv);
        }
      }
    } else {
      switch (nb) {
        case NB_LX: for (int j = 1; j <= nc; j++) g[j - 1] = b.c(2, j, iv); break;
        case NB_HX: for (int j = 1; j <= nc; j++) g[j - 1] = b.c(nc - 1, j, iv); break;
        case NB_LY: for (int i = 1; i <= nc; i++) g[i - 1] = b.c(i, 2, iv); break;
        case NB_HY: for (int i = 1; i <= nc; i++) g[i - 1] = b.c(i, nc - 1, iv); break;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Restriction, afivo/src/m_aX_restrict.f90:67-142 (a$D_restrict_box)
static void restrict_box(const Box &bc, Box &bp, int iv, int i_dest) {
  int hnc = bc.n_cell >> 1;
  int off[2];
  child_offset(bc, -1, off);
  if (bp.coord == CYL) {
    double dr16 = 0.0625 * bp.dr;
    for (int j = 1; j <= hnc; j++) {
      int j_c = off[1] + j, j_f = 2 * j - 1;
      for (int i = 1; i <= hnc; i++) {
        int i_c = off[0] + i, i_f = 2 * i - 1;
        // The reference evaluates the radius at parent index [i, j], not
        // [i_c, j_c] (m_aX_restrict.f90:104); kept as written.
        double r = bp.r_min[0] + (i - 0.5) * bp.dr;
        double rfac = dr16 / r;
        double s1 = bc.c(i_f, j_f, iv) + bc.c(i_f, j_f + 1, iv);
        double s2 = bc.c(i_f + 1, j_f, iv) + bc.c(i_f + 1, j_f + 1, iv);
        bp.c(i_c, j_c, i_dest) = (0.25 - rfac) * s1 + (0.25 + rfac) * s2;
      }
    }
  } else {
    for (int j = 1; j <= hnc; j++) {
      int j_c = off[1] + j, j_f = 2 * j - 1;
      for (int i = 1; i <= hnc; i++) {
        int i_c = off[0] + i, i_f = 2 * i - 1;
        double s = bc.c(i_f, j_f, iv) + bc.c(i_f + 1, j_f, iv) +
                   bc.c(i_f, j_f + 1, iv) + bc.c(i_f + 1, j_f + 1, iv);
        bp.c(i_c, j_c, i_dest) = 0.25 * s;
      }
    }
  }
}

// afivo/src/m_aX_restrict.f90:23-64 (restrict_to_box / _boxes / _tree)
static void restrict_tree(Tree &t, int iv) {
  for (int lvl = t.max_lvl - 1; lvl >= t.min_lvl; lvl--) {
    Level &L = t.L(lvl);
    int n = (int)L.parents.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      int id = L.parents[i];
      for (int ic = 0; ic < NCH; ic++) {
        int c_id = t.boxes[id].children[ic];
        if (c_id == NO_BOX) continue;
        restrict_box(t.boxes[c_id], t.boxes[id], iv, iv);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Multigrid, afivo/src/m_aX_mg.f90
enum { MG_NORMAL_BOX = 1, MG_LSF_BOX = 2, MG_CEPS_BOX = 3, MG_VEPS_BOX = 4 };

struct MG {
  int i_phi = -1, i_rhs = -1, i_tmp = -1, i_eps = -1, i_lsf = -1, i_bval = -1;
  int n_cycle_down = 2, n_cycle_up = 2, n_cycle_base = 2;
  GcFn sides_bc, sides_rb;
};

// afivo/src/m_aX_mg.f90:673-712 (mg$D_set_box_tag): a level-set box where
// the level-set function changes sign in the box (ghost and corner cells
// included), an eps box where eps varies or is a constant other than 1.
static void set_box_tag(Box &b, const MG &mg) {
  bool is_lsf = false, is_eps = false, is_deps = false;
  if (mg.i_lsf != -1) {
    const int ncg = b.ncg();
    double a = b.c(0, 0, mg.i_lsf), bb = a;
    for (int j = 0; j < ncg; j++)
      for (int i = 0; i < ncg; i++) {
        a = std::min(a, b.c(i, j, mg.i_lsf));
        bb = std::max(bb, b.c(i, j, mg.i_lsf));
      }
    is_lsf = a * bb < 0;
  }
  if (mg.i_eps != -1) {
    int ncg = b.ncg();
    double a = b.c(0, 0, mg.i_eps), bb = a;
    for (int j = 0; j < ncg; j++)
      for (int i = 0; i < ncg; i++) {
        a = std::min(a, b.c(i, j, mg.i_eps));
        bb = std::max(bb, b.c(i, j, mg.i_eps));
      }
    is_deps = bb > a;
    if (!is_deps) is_eps = (a < 1 || a > 1);
  }
  b.tag = MG_NORMAL_BOX;
  if (is_lsf) b.tag = MG_LSF_BOX;
  if (is_eps) b.tag = MG_CEPS_BOX;
  if (is_deps) b.tag = MG_VEPS_BOX;
}

// lsf_dist_val (afivo/src/m_aX_mg.f90:1077-1104): distance (0..1] from a
// to neighbour b and the value there: where the level set changes sign
// between them, the interface at lsf_a / (lsf_a - lsf_b), with the boundary
// values interpolated; else b itself and its value.
static inline void lsf_dist_val(const double va[3], const double vb[3], double &dist, double &val) {
  if (va[0] * vb[0] < 0) {
    dist = va[0] / (va[0] - vb[0]);
    val = va[2] * (1 - dist) + vb[2] * dist;
  } else {
    dist = 1;
    val = vb[1];
  }
}

// The four neighbours (lx, hx, ly, hy) of cell (i, j) as distances and
// values for the level-set operators.
static inline void lsf_nbrs(const Box &b, int i, int j, const MG &mg, int iv, double dd[4],
                            double val[4]) {
  const double va[3] = {b.c(i, j, mg.i_lsf), b.c(i, j, iv), b.c(i, j, mg.i_bval)};
  const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
  for (int k = 0; k < 4; k++) {
    const double vb[3] = {b.c(i + di[k], j + dj[k], mg.i_lsf), b.c(i + di[k], j + dj[k], iv),
                          b.c(i + di[k], j + dj[k], mg.i_bval)};
    lsf_dist_val(va, vb, dd[k], val[k]);
  }
}

// mg$D_box_gsrb_lpllsf (afivo/src/m_aX_mg.f90:1190-1267, 2D): Gauss-Seidel
// for the Laplacian with neighbours at distances dd dx (Fortran operation
// order kept: 1 / (dd1 dd2 + dd3 dd4) * (...)).
static void box_gsrb_lsf(Box &b, int redblack, const MG &mg) {
  const double dx2 = b.dr * b.dr;
  const int nc = b.n_cell;
  for (int j = 1; j <= nc; j++) {
    const int i0 = 2 - ((redblack ^ j) & 1);
    for (int i = i0; i <= nc; i += 2) {
      double dd[4], val[4];
      lsf_nbrs(b, i, j, mg, mg.i_phi, dd, val);
      const double prod = dd[0] * dd[1] * dd[2] * dd[3];
      b.c(i, j, mg.i_phi) = 1 / (dd[0] * dd[1] + dd[2] * dd[3]) *
                            ((dd[1] * val[0] + dd[0] * val[1]) * dd[2] * dd[3] / (dd[0] + dd[1]) +
                             (dd[3] * val[2] + dd[2] * val[3]) * dd[0] * dd[1] / (dd[2] + dd[3]) -
                             0.5 * prod * dx2 * b.c(i, j, mg.i_rhs));
    }
  }
}

// mg$D_box_lpllsf (afivo/src/m_aX_mg.f90:1270-1340, 2D)
static void box_op_lsf(Box &b, int i_out, const MG &mg) {
  const double inv_dr_sq = 1 / (b.dr * b.dr);
  const int nc = b.n_cell;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) {
      double dd[4], val[4];
      lsf_nbrs(b, i, j, mg, mg.i_phi, dd, val);
      const double f0 = b.c(i, j, mg.i_phi);
      b.c(i, j, i_out) = 2 * inv_dr_sq *
                         ((dd[1] * val[0] + dd[0] * val[1] - (dd[0] + dd[1]) * f0) /
                              ((dd[0] + dd[1]) * dd[0] * dd[1]) +
                          (dd[3] * val[2] + dd[2] * val[3] - (dd[2] + dd[3]) * f0) /
                              ((dd[2] + dd[3]) * dd[2] * dd[3]));
    }
}

// Radius weights of the cylindrical operators at global index g = i + ioff:
// (g - 1) / (g - 1/2) and g / (g - 1/2) (afivo/src/m_aX_mg.f90:1027-1049).
static inline void rfac_cyl(int g, double &rf1, double &rf2) {
  double den = g - 0.5;
  rf1 = (g - 1) / den;
  rf2 = g / den;
}

// Red-black Gauss-Seidel on a box whose eps is not identically 1
// (mg$D_box_gsrb_lpld, afivo/src/m_aX_mg.f90:895-948; cylindrical
// mg2_box_gsrb_clpld, :1499-1531): face weights c = 2 a0 a / (a0 + a) from
// the eps of the cell (a0) and of each neighbour (a), the cylindrical radius
// factors on the x faces, phi = (sum c rfac u - dx^2 rhs) / sum c rfac; sums
// in neighbour order lx, hx, ly, hy.
static void box_gsrb_diel(Box &b, int redblack, const MG &mg) {
  const double dx2 = b.dr * b.dr;
  const int nc = b.n_cell, ip = mg.i_phi, ir = mg.i_rhs, ie = mg.i_eps;
  const bool cyl = b.coord == CYL;
  const int ioff = (b.ix[0] - 1) * nc;
  for (int j = 1; j <= nc; j++) {
    int i0 = 2 - ((redblack ^ j) & 1);
    for (int i = i0; i <= nc; i += 2) {
      const double a0 = b.c(i, j, ie);
      const double u[4] = {b.c(i - 1, j, ip), b.c(i + 1, j, ip), b.c(i, j - 1, ip), b.c(i, j + 1, ip)};
      const double a[4] = {b.c(i - 1, j, ie), b.c(i + 1, j, ie), b.c(i, j - 1, ie), b.c(i, j + 1, ie)};
      double rf[4] = {1, 1, 1, 1};
      if (cyl) rfac_cyl(i + ioff, rf[0], rf[1]);
      double su = 0, sc = 0;
      for (int k = 0; k < 4; k++) {
        const double c = 2 * a0 * a[k] / (a0 + a[k]);
        if (cyl) {
          su = su + c * rf[k] * u[k];
          sc = sc + c * rf[k];
        } else {
          su = su + c * u[k];
          sc = sc + c;
        }
      }
      b.c(i, j, ip) = (su - dx2 * b.c(i, j, ir)) / sc;
    }
  }
}

// Laplacian of a box whose eps is not identically 1 (mg$D_box_lpld,
// afivo/src/m_aX_mg.f90:951-1001; cylindrical mg2_box_clpld, :1467-1495):
// inv_dr^2 * 2 * sum rfac a0 a / (a0 + a) (u - u0).
static void box_op_diel(Box &b, int i_out, const MG &mg) {
  const int nc = b.n_cell, ip = mg.i_phi, ie = mg.i_eps;
  const double inv_dr_sq = 1 / (b.dr * b.dr);
  const bool cyl = b.coord == CYL;
  const int ioff = (b.ix[0] - 1) * nc;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) {
      const double u0 = b.c(i, j, ip), a0 = b.c(i, j, ie);
      const double u[4] = {b.c(i - 1, j, ip), b.c(i + 1, j, ip), b.c(i, j - 1, ip), b.c(i, j + 1, ip)};
      const double a[4] = {b.c(i - 1, j, ie), b.c(i + 1, j, ie), b.c(i, j - 1, ie), b.c(i, j + 1, ie)};
      double rf[4] = {1, 1, 1, 1};
      if (cyl) rfac_cyl(i + ioff, rf[0], rf[1]);
      double sum = 0;
      for (int k = 0; k < 4; k++) {
        if (cyl) sum = sum + rf[k] * a0 * a[k] / (a0 + a[k]) * (u[k] - u0);
        else sum = sum + a0 * a[k] / (a0 + a[k]) * (u[k] - u0);
      }
      b.c(i, j, i_out) = inv_dr_sq * 2 * sum;
    }
}

// afivo/src/m_aX_mg.f90:636-659 (gsrb_lpl) and 998-1024 (gsrb_clpl)
static void box_gsrb(Box &b, int redblack, const MG &mg) {
  if (b.tag == INIT_TAG) set_box_tag(b, mg);
  if (b.tag == MG_LSF_BOX) {
    box_gsrb_lsf(b, redblack, mg);
    return;
  }
  if (b.tag == MG_CEPS_BOX || b.tag == MG_VEPS_BOX) {
    box_gsrb_diel(b, redblack, mg);
    return;
  }
  double dx2 = b.dr * b.dr;
  int nc = b.n_cell, ip = mg.i_phi, ir = mg.i_rhs;
  if (b.coord == CYL) {
    int ioff = (b.ix[0] - 1) * nc;
    for (int j = 1; j <= nc; j++) {
      int i0 = 2 - ((redblack ^ j) & 1);
      for (int i = i0; i <= nc; i += 2) {
        double den = i + ioff - 0.5;
        double rf1 = (i + ioff - 1) / den, rf2 = (i + ioff) / den;
        b.c(i, j, ip) = 0.25 * (rf1 * b.c(i - 1, j, ip) + rf2 * b.c(i + 1, j, ip) +
                                b.c(i, j + 1, ip) + b.c(i, j - 1, ip) -
                                dx2 * b.c(i, j, ir));
      }
    }
  } else {
    for (int j = 1; j <= nc; j++) {
      int i0 = 2 - ((redblack ^ j) & 1);
      for (int i = i0; i <= nc; i += 2)
        b.c(i, j, ip) = 0.25 * (b.c(i + 1, j, ip) + b.c(i - 1, j, ip) +
                                b.c(i, j + 1, ip) + b.c(i, j - 1, ip) -
                                dx2 * b.c(i, j, ir));
    }
  }
}

// afivo/src/m_aX_mg.f90:662-680 (box_lpl) and 1027-1049 (box_clpl)
static void box_op(Box &b, int i_out, const MG &mg) {
  if (b.tag == INIT_TAG) set_box_tag(b, mg);
  if (b.tag == MG_LSF_BOX) {
    box_op_lsf(b, i_out, mg);
    return;
  }
  if (b.tag == MG_CEPS_BOX || b.tag == MG_VEPS_BOX) {
    box_op_diel(b, i_out, mg);
    return;
  }
  int nc = b.n_cell, ip = mg.i_phi;
  double inv_dr_sq = 1 / (b.dr * b.dr);
  if (b.coord == CYL) {
    int ioff = (b.ix[0] - 1) * nc;
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc; i++) {
        double den = i + ioff - 0.5;
        double rf1 = (i + ioff - 1) / den, rf2 = (i + ioff) / den;
        b.c(i, j, i_out) = (rf1 * b.c(i - 1, j, ip) + rf2 * b.c(i + 1, j, ip) +
                            b.c(i, j - 1, ip) + b.c(i, j + 1, ip) -
                            4 * b.c(i, j, ip)) * inv_dr_sq;
      }
  } else {
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc; i++)
        b.c(i, j, i_out) = inv_dr_sq * (b.c(i - 1, j, ip) + b.c(i + 1, j, ip) +
                                        b.c(i, j - 1, ip) + b.c(i, j + 1, ip) -
                                        4 * b.c(i, j, ip));
  }
}

// afivo/src/m_aX_mg.f90:605-633 (box_corr_lpl)
static void box_corr(const Box &p, Box &c, const MG &mg) {
  if (c.tag == INIT_TAG) set_box_tag(c, mg);
  int nc = c.n_cell, ip = mg.i_phi, ic = mg.i_tmp;
  int off[2];
  child_offset(c, -1, off);
  if (c.tag == MG_LSF_BOX) {
    // mg$D_box_corr_lpllsf (afivo/src/m_aX_mg.f90:1106-1187, 2D): the
    // correction interpolated along the lines to the three nearest coarse
    // cells, each cut at the interface (boundary value 0 for a correction)
    for (int j = 1; j <= nc; j++) {
      int j_c1 = off[1] + ((j + 1) >> 1);
      int j_c2 = j_c1 + 1 - 2 * (j & 1);
      for (int i = 1; i <= nc; i++) {
        int i_c1 = off[0] + ((i + 1) >> 1);
        int i_c2 = i_c1 + 1 - 2 * (i & 1);
        const double va[3] = {c.c(i, j, mg.i_lsf), c.c(i, j, ic), 0.0};
        const int pi[3] = {i_c1, i_c2, i_c1}, pj[3] = {j_c1, j_c1, j_c2};
        double dist[3], val[3];
        for (int k = 0; k < 3; k++) {
          const double vb[3] = {p.c(pi[k], pj[k], mg.i_lsf), p.c(pi[k], pj[k], ic), 0.0};
          lsf_dist_val(va, vb, dist[k], val[k]);
        }
        const double cw[3] = {2 * dist[1] * dist[2], dist[0] * dist[2], dist[0] * dist[1]};
        c.c(i, j, ip) = c.c(i, j, ip) + (cw[0] * val[0] + cw[1] * val[1] + cw[2] * val[2]) /
                                            (cw[0] + cw[1] + cw[2]);
      }
    }
    return;
  }
  if (c.tag == MG_CEPS_BOX || c.tag == MG_VEPS_BOX) {
    // mg$D_box_corr_lpld, afivo/src/m_aX_mg.f90:1003-1071 (2D): eps-weighted
    // averages of the parent's correction toward each coarse neighbour
    const int ie = mg.i_eps;
    for (int j = 1; j <= nc; j++) {
      int j_c1 = off[1] + ((j + 1) >> 1);
      int j_c2 = j_c1 + 1 - 2 * (j & 1);
      for (int i = 1; i <= nc; i++) {
        int i_c1 = off[0] + ((i + 1) >> 1);
        int i_c2 = i_c1 + 1 - 2 * (i & 1);
        const double u0 = p.c(i_c1, j_c1, ic), a0 = p.c(i_c1, j_c1, ie);
        const double u1 = p.c(i_c2, j_c1, ic), u2 = p.c(i_c1, j_c2, ic);
        const double a1 = p.c(i_c2, j_c1, ie), a2 = p.c(i_c1, j_c2, ie);
        double sum = 0;
        sum = sum + (a0 * u0 + a1 * u1) / (a0 + a1);
        sum = sum + (a0 * u0 + a2 * u2) / (a0 + a2);
        c.c(i, j, ip) = c.c(i, j, ip) + 0.5 * sum;
      }
    }
    return;
  }
  for (int j = 1; j <= nc; j++) {
    int j_c1 = off[1] + ((j + 1) >> 1);
    int j_c2 = j_c1 + 1 - 2 * (j & 1);
    for (int i = 1; i <= nc; i++) {
      int i_c1 = off[0] + ((i + 1) >> 1);
      int i_c2 = i_c1 + 1 - 2 * (i & 1);
      c.c(i, j, ip) = c.c(i, j, ip) + 0.5 * p.c(i_c1, j_c1, ic) +
                      0.25 * (p.c(i_c2, j_c1, ic) + p.c(i_c1, j_c2, ic));
    }
  }
}

// afivo/src/m_aX_mg.f90:683-705 (box_rstr_lpl)
static void box_rstr(const Box &bc, Box &bp, int iv) {
  int hnc = bc.n_cell >> 1;
  int off[2];
  child_offset(bc, -1, off);
  for (int j = 1; j <= hnc; j++) {
    int j_c = off[1] + j, j_f = 2 * j - 1;
    for (int i = 1; i <= hnc; i++) {
      int i_c = off[0] + i, i_f = 2 * i - 1;
      bp.c(i_c, j_c, iv) = 0.25 * (bc.c(i_f, j_f, iv) + bc.c(i_f + 1, j_f, iv) +
                                   bc.c(i_f, j_f + 1, iv) + bc.c(i_f + 1, j_f + 1, iv));
    }
  }
}

// afivo/src/m_aX_mg.f90:261-301 (mg$D_sides_rb)
static void mg_sides_rb(Tree &t, int id, int nb, int iv) {
  Box &b = t.boxes[id];
  int nc = b.n_cell;
  int ix, dix;
  if (nb_low[nb]) { ix = 1; dix = 1; }
  else { ix = nc; dix = -1; }
  gc_prolong0(t, id, nb, iv);
  if (nb_dim[nb] == 0) {
    int i = ix, di = dix;
    for (int j = 1; j <= nc; j++) {
      int dj = -1 + 2 * (j & 1);
      b.c(i - di, j, iv) = 0.5 * b.c(i - di, j, iv) + b.c(i, j, iv) -
                           0.25 * (b.c(i + di, j, iv) + b.c(i, j + dj, iv));
    }
  } else {
    int j = ix, dj = dix;
    for (int i = 1; i <= nc; i++) {
      int di = -1 + 2 * (i & 1);
      b.c(i, j - dj, iv) = 0.5 * b.c(i, j - dj, iv) + b.c(i, j, iv) -
                           0.25 * (b.c(i + di, j, iv) + b.c(i, j + dj, iv));
    }
  }
}

static void copy_full(Box &b, int from, int to) {
  size_t n = (size_t)b.ncg() * b.ncg();
  std::memcpy(&b.cc[n * to], &b.cc[n * from], n * sizeof(double));
}

// afivo/src/m_aX_mg.f90:303-316 (fill_gc_phi)
static void fill_gc_phi(Tree &t, const std::vector<int> &ids, const MG &mg) {
  int n = (int)ids.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) gc_box(t, ids[i], mg.i_phi, mg.sides_rb, mg.sides_bc);
}

// afivo/src/m_aX_mg.f90:319-341 (correct_children)
static void correct_children(Tree &t, const std::vector<int> &ids, const MG &mg) {
  int n = (int)ids.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    Box &p = t.boxes[ids[i]];
    size_t m = (size_t)p.ncg() * p.ncg();
    double *phi = &p.cc[m * mg.i_phi], *tmp = &p.cc[m * mg.i_tmp];
    for (size_t k = 0; k < m; k++) tmp[k] = phi[k] - tmp[k];
    for (int ic = 0; ic < NCH; ic++) {
      int c_id = p.children[ic];
      if (c_id == NO_BOX) continue;
      box_corr(p, t.boxes[c_id], mg);
    }
  }
}

// afivo/src/m_aX_mg.f90:343-366 (gsrb_boxes)
static void gsrb_boxes(Tree &t, const std::vector<int> &ids, const MG &mg, int n_cycle) {
  int n = (int)ids.size();
  for (int it = 1; it <= 2 * n_cycle; it++) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) box_gsrb(t.boxes[ids[i]], it, mg);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) gc_box(t, ids[i], mg.i_phi, mg.sides_rb, mg.sides_bc);
  }
}

// afivo/src/m_aX_mg.f90:475-484 (residual_box)
static void residual_box(Box &b, const MG &mg) {
  box_op(b, mg.i_tmp, mg);
  int nc = b.n_cell;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++)
      b.c(i, j, mg.i_tmp) = b.c(i, j, mg.i_rhs) - b.c(i, j, mg.i_tmp);
}

static void box_op_add_copy(Box &b, const MG &mg, bool copy_phi_tmp) {
  box_op(b, mg.i_rhs, mg);
  size_t m = (size_t)b.ncg() * b.ncg();
  double *rhs = &b.cc[m * mg.i_rhs], *tmp = &b.cc[m * mg.i_tmp];
  for (size_t k = 0; k < m; k++) rhs[k] = rhs[k] + tmp[k];
  if (copy_phi_tmp) copy_full(b, mg.i_phi, mg.i_tmp);
}

// afivo/src/m_aX_mg.f90:370-410 (update_coarse)
static void update_coarse(Tree &t, int lvl, const MG &mg) {
  Level &L = t.L(lvl);
  int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int id = L.ids[i];
    Box &b = t.boxes[id];
    Box &p = t.boxes[b.parent];
    int nc = b.n_cell;
    double save[64 * 64];
    for (int j = 1; j <= nc; j++)
      for (int ii = 1; ii <= nc; ii++) save[(ii - 1) + nc * (j - 1)] = b.c(ii, j, mg.i_tmp);
    residual_box(b, mg);
    box_rstr(b, p, mg.i_tmp);
    box_rstr(b, p, mg.i_phi);
    for (int j = 1; j <= nc; j++)
      for (int ii = 1; ii <= nc; ii++) b.c(ii, j, mg.i_tmp) = save[(ii - 1) + nc * (j - 1)];
  }
  fill_gc_phi(t, t.L(lvl - 1).ids, mg);
  std::vector<int> &P = t.L(lvl - 1).parents;
  int np = (int)P.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < np; i++) box_op_add_copy(t.boxes[P[i]], mg, true);
}

// afivo/src/m_aX_mg.f90:414-447 (set_coarse_phi_rhs)
static void set_coarse_phi_rhs(Tree &t, int lvl, const MG &mg) {
  if (lvl == t.max_lvl) fill_gc_phi(t, t.L(lvl).ids, mg);
  Level &L = t.L(lvl);
  int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    Box &b = t.boxes[L.ids[i]];
    Box &p = t.boxes[b.parent];
    residual_box(b, mg);
    box_rstr(b, p, mg.i_tmp);
    box_rstr(b, p, mg.i_phi);
  }
  fill_gc_phi(t, t.L(lvl - 1).ids, mg);
  std::vector<int> &P = t.L(lvl - 1).parents;
  int np = (int)P.size();
#pragma omp parallel for schedule(static)
  for (int i = 0; i < np; i++) box_op_add_copy(t.boxes[P[i]], mg, false);
}

// afivo/src/m_aX_mg.f90:450-473 (init_phi_rhs)
static void init_phi_rhs(Tree &t, const MG &mg) {
  for (int lvl = t.max_lvl; lvl >= t.min_lvl + 1; lvl--) {
    Level &L = t.L(lvl);
    int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      Box &b = t.boxes[L.ids[i]];
      size_t m = (size_t)b.ncg() * b.ncg();
      std::fill(&b.cc[m * mg.i_phi], &b.cc[m * mg.i_phi] + m, 0.0);
      box_rstr(b, t.boxes[b.parent], mg.i_rhs);
    }
  }
}

// afivo/src/m_aX_mg.f90:208-254 (mg$D_fas_vcycle)
static void fas_vcycle(Tree &t, const MG &mg, int max_lvl, bool set_residual) {
  int min_lvl = t.min_lvl;
  for (int lvl = max_lvl; lvl >= min_lvl + 1; lvl--) {
    gsrb_boxes(t, t.L(lvl).ids, mg, mg.n_cycle_down);
    update_coarse(t, lvl, mg);
  }
  gsrb_boxes(t, t.L(min_lvl).ids, mg, mg.n_cycle_base);
  for (int lvl = min_lvl + 1; lvl <= max_lvl; lvl++) {
    correct_children(t, t.L(lvl - 1).parents, mg);
    fill_gc_phi(t, t.L(lvl).ids, mg);
    gsrb_boxes(t, t.L(lvl).ids, mg, mg.n_cycle_up);
  }
  if (set_residual) {
    for (int lvl = min_lvl; lvl <= max_lvl; lvl++) {
      Level &L = t.L(lvl);
      int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) residual_box(t.boxes[L.ids[i]], mg);
    }
  }
}

// afivo/src/m_aX_mg.f90:163-202 (mg$D_fas_fmg)
static void fas_fmg(Tree &t, const MG &mg, bool set_residual, bool first_call) {
  int min_lvl = t.min_lvl;
  if (first_call) {
    init_phi_rhs(t, mg);
  } else {
    for (int lvl = t.max_lvl; lvl >= min_lvl + 1; lvl--) set_coarse_phi_rhs(t, lvl, mg);
  }
  for (int lvl = min_lvl; lvl <= t.max_lvl; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) copy_full(t.boxes[L.ids[i]], mg.i_phi, mg.i_tmp);
    if (lvl > min_lvl) {
      correct_children(t, t.L(lvl - 1).parents, mg);
      fill_gc_phi(t, L.ids, mg);
    }
    fas_vcycle(t, mg, lvl, set_residual && lvl == t.max_lvl);
  }
}

// afivo/src/m_aX_utils.f90:559-619 (a$D_tree_max_cc / _min_cc), leaves only
static double tree_max_cc(Tree &t, int iv) {
  double m = -1.7976931348623157e308;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) {
      Box &b = t.boxes[id];
      int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) m = std::max(m, b.c(i, j, iv));
    }
  return m;
}
static double tree_min_cc(Tree &t, int iv) {
  double m = 1.7976931348623157e308;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) {
      Box &b = t.boxes[id];
      int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) m = std::min(m, b.c(i, j, iv));
    }
  return m;
}

// ---------------------------------------------------------------------------
// Lookup table, fosito/m_lookup_table.f90
struct LT {
  int n_rows = 0, n_cols = 0;
  double x_min = 0, inv_dx = 0;
  std::vector<double> rows_cols;  // rows_cols[(row-1) + n_rows * col]
  double rc(int row, int col) const { return rows_cols[(row - 1) + (size_t)n_rows * col]; }
};
struct Loc { int low_ix; double low_frac; };

// fosito/m_lookup_table.f90:46-63 (LT_create)
static LT lt_create(double x_min, double x_max, int n_rows, int n_cols) {
  LT t;
  t.n_rows = n_rows;
  t.x_min = x_min;
  t.inv_dx = (n_rows - 1) / (x_max - x_min);
  t.n_cols = n_cols;
  t.rows_cols.assign((size_t)n_rows * n_cols, 0.0);
  return t;
}

// fosito/m_find_index.f90:26-67: smallest ix (1-based) with val <= list(ix)
static int fi_adaptive(const double *list, int n, double val) {
  int lo = 1, hi = n;
  while (lo < hi) {
    int mid = lo + (hi - lo) / 2;
    if (val <= list[mid - 1]) hi = mid;
    else lo = mid + 1;
  }
  if (val > list[lo - 1]) lo = n + 1;
  return lo;
}

// fosito/m_lookup_table.f90:200-221 (LT_lin_interp_list)
static double lin_interp_list(const double *xl, const double *yl, int n, double x) {
  if (x <= xl[0]) return yl[0];
  if (x >= xl[n - 1]) return yl[n - 1];
  int ix = fi_adaptive(xl, n, x);
  double temp = (x - xl[ix - 2]) / (xl[ix - 1] - xl[ix - 2]);
  return (1 - temp) * yl[ix - 2] + temp * yl[ix - 1];
}

// fosito/m_lookup_table.f90:65-72 (LT_set_col) with LT_get_xdata (180-189)
static void lt_set_col(LT &t, int col, const double *xx, const double *yy, int n) {
  double dx = 1 / t.inv_dx;
  for (int ix = 1; ix <= t.n_rows; ix++) {
    double x = t.x_min + (ix - 1) * dx;
    t.rows_cols[(ix - 1) + (size_t)t.n_rows * col] = lin_interp_list(xx, yy, n, x);
  }
}

// fosito/m_lookup_table.f90:107-125 (get_loc). ceiling() of an argument
// beyond the int range is clamped to the table end.
static inline Loc lt_get_loc(const LT &t, double x) {
  double frac = (x - t.x_min) * t.inv_dx;
  Loc l;
  if (frac < 2.0e9 && frac > -2.0e9) {
    l.low_ix = (int)std::ceil(frac);
    l.low_frac = l.low_ix - frac;
  } else {
    l.low_ix = frac > 0 ? t.n_rows : 0;
    l.low_frac = 0;
  }
  if (l.low_ix < 1) { l.low_ix = 1; l.low_frac = 1; }
  else if (l.low_ix >= t.n_rows) { l.low_ix = t.n_rows - 1; l.low_frac = 0; }
  return l;
}
// fosito/m_lookup_table.f90:154-161 (LT_get_col_at_loc)
static inline double lt_col_at(const LT &t, int col, const Loc &l) {
  return l.low_frac * t.rc(l.low_ix, col) + (1 - l.low_frac) * t.rc(l.low_ix + 1, col);
}
static inline double lt_get_col(const LT &t, int col, double x) {
  return lt_col_at(t, col, lt_get_loc(t, x));
}

// ---------------------------------------------------------------------------
// Random numbers, fosito/m_random.f90. RNG_t holds four default integers and
// draws with Marsaglia's mzran. The reference's integer arithmetic wraps on
// overflow (two's complement, as its gfortran x86-64 build computes it);
// restated here with unsigned arithmetic.
struct Rng {
  int32_t st[4] = {521288629, 362436069, 16163801, 1131199299};  // :12-13
  // int4, :58-66
  int32_t int4() {
    int32_t rr = (int32_t)((uint32_t)st[0] - (uint32_t)st[2]);
    if (rr < 0) rr = (int32_t)((uint32_t)rr + 2147483579u);
    st[0] = st[1];
    st[1] = st[2];
    st[2] = rr;
    st[3] = (int32_t)(69069u * (uint32_t)st[3] + 1013904243u);
    return (int32_t)((uint32_t)rr + (uint32_t)st[3]);
  }
  // uni_01, :75-80: 0.5 + 2^-32 * int4, exact in double
  double uni_01() { return 0.5 + 0x1p-32 * (double)int4(); }
  // uni_ab, :83-88
  double uni_ab(double a, double b) { return a + uni_01() * (b - a); }
  // sphere, :135-151 (Marsaglia's method)
  void sphere(double radius, double xyz[3]) {
    double r0, r1, ss;
    while (true) {
      r0 = uni_ab(-1.0, 1.0);
      r1 = uni_ab(-1.0, 1.0);
      ss = r0 * r0 + r1 * r1;
      if (ss <= 1) break;
    }
    double t = std::sqrt(1 - ss);
    xyz[0] = 2 * r0 * t;
    xyz[1] = 2 * r1 * t;
    xyz[2] = 1 - 2 * ss;
    for (int d = 0; d < 3; d++) xyz[d] = xyz[d] * radius;
  }
};

// PRNG_t%init, fosito/m_random.f90:44-55: stream n takes the master's draws
// 4n+1..4n+4 (0-based n).
static std::vector<Rng> prng_init(Rng &master, int n_proc) {
  std::vector<Rng> r(n_proc);
  for (int n = 0; n < n_proc; n++)
    for (int i = 0; i < 4; i++) r[n].st[i] = master.int4();
  return r;
}

// libgomp's static schedule without a chunk size: iterations [lo, lo+len) of
// thread c out of n_threads for n iterations.
static inline void static_chunk(long n, long n_threads, long c, long &lo, long &len) {
  long q = n / n_threads, t = n % n_threads;
  if (c < t) {
    q++;
    t = 0;
  }
  lo = q * c + t;
  len = q;
}

// ---------------------------------------------------------------------------
// Photon absorption table, src/m_photons.f90:25-140. The absorption function
// is PH_absfunc_air (:122-140) with its two absorption coefficients c0 < c1
// (1/(m bar)) at O2 pressure p: (exp(-c0 p d) - exp(-c1 p d)) / (d log(c1/c0)),
// the distance density of an exponential absorption whose coefficient is
// log-uniform on [c0 p, c1 p]. A log-uniform absorption length [l_lo, l_hi]
// is the same function with c0 = 1/l_hi, c1 = 1/l_lo and p = 1.
struct AbsFn {
  double c0, c1, p;
};
// fosito/m_units_constants.f90:44: one Torr in bar, written with a default
// (single precision) real literal times 1.0D-5.
static const double UC_TORR_TO_BAR = (double)133.322368f * 1.0e-5;

static AbsFn absfn_air(double p_O2) {
  return AbsFn{3.5 / UC_TORR_TO_BAR, 200 / UC_TORR_TO_BAR, p_O2};
}
static AbsFn absfn_logu(double len_lo, double len_hi) {
  return AbsFn{1 / len_hi, 1 / len_lo, 1.0};
}

// src/m_photons.f90:122-140 (PH_absfunc_air)
static double absfunc(const AbsFn &a, double dist) {
  const double eps = 2.220446049250313e-16;
  double r = a.p * dist;
  if (r * (a.c0 + a.c1) < eps)
    return (a.c1 - a.c0 + 0.5 * (a.c0 * a.c0 - a.c1 * a.c1) * r) * a.p / std::log(a.c1 / a.c0);
  if (r * a.c0 > -std::log(eps)) return eps;
  return (std::exp(-a.c0 * r) - std::exp(-a.c1 * r)) / (dist * std::log(a.c1 / a.c0));
}

// src/m_photons.f90:95-117 (rk4_drdF)
static double rk4_drdF(const AbsFn &a, double r, double dF) {
  const double one_sixth = 1 / 6.0;
  double drdF = 1 / absfunc(a, r);
  double sum = drdF;
  drdF = 1 / absfunc(a, r + 0.5 * dF * drdF);
  sum = sum + 2 * drdF;
  drdF = 1 / absfunc(a, r + 0.5 * dF * drdF);
  sum = sum + 2 * drdF;
  drdF = 1 / absfunc(a, r + dF * drdF);
  sum = sum + drdF;
  return one_sixth * sum;
}

struct PhTbl {
  LT tbl;
  double frac_in_tbl = 0;
};

// src/m_photons.f90:25-93 (PH_get_tbl_air) for a given absorption function
static bool ph_get_tbl(const AbsFn &a, double max_dist, PhTbl &out) {
  const int tbl_size = 500;
  double frac_guess = 1.0;
  for (int n = 1; n <= 5; n++) {
    double dF = frac_guess / (tbl_size - 1), r = 0, F = 0;
    while (true) {
      double drdF = rk4_drdF(a, r, dF);
      r = r + dF * drdF;
      F = F + dF;
      if (r > max_dist) {
        frac_guess = F;
        break;
      }
    }
  }
  std::vector<double> fsum(2 * tbl_size), dist(2 * tbl_size);
  double dF = frac_guess / (tbl_size - 1);
  dist[0] = 0;
  fsum[0] = 0;
  int n;  // 1-based index at exit, as the Fortran loop variable
  for (n = 2; n <= 2 * tbl_size; n++) {
    double drdF = rk4_drdF(a, dist[n - 2], dF);
    fsum[n - 1] = fsum[n - 2] + dF;
    dist[n - 1] = dist[n - 2] + dF * drdF;
    if (dist[n - 1] > max_dist) break;
  }
  if (n > tbl_size + 10) return false;  // "integration accuracy fail"
  out.frac_in_tbl = fsum[n - 2];
  const double norm = fsum[n - 2];
  for (int k = 0; k < n - 1; k++) fsum[k] = fsum[k] / norm;
  out.tbl = lt_create(0.0, 1.0, tbl_size, 1);
  lt_set_col(out.tbl, 0, fsum.data(), dist.data(), n - 1);
  return true;
}

// src/m_photons.f90:142-155 (get_lvl_length)
static int get_lvl_length(double dr_base, double length) {
  const double invlog2 = 1 / std::log(2.0);
  double ratio = dr_base / length;
  if (ratio <= 1) return 1;
  return 1 + (int)std::ceil(std::log(ratio) * invlog2);
}

// ---------------------------------------------------------------------------
// Streamer model, src/streamer_2d.f90 and src/streamer_cyl.f90
struct Sim {
  a5ref_params p;
  Tree tree;
  LT td;
  MG mg;
  double time = 0;
  double applied_voltage = 0;
  Rng rng;       // ST_rng (src/m_streamer.f90:69)
  PhTbl ph;      // ST_photoi_tbl
  int pho_lvl = 1;
  long n_photons = 0;  // photons created by the last photoionization call
};

// src/m_streamer.f90:339-362 (koren_mlim)
static inline double koren_mlim(double a, double b) {
  const double sixth = 1 / 6.0;
  double aa = a * a, ab = a * b;
  if (ab <= 0) return 0;
  if (aa <= 0.25 * ab) return a;
  if (aa <= 2.5 * ab) return sixth * (b + 2 * a);
  return b;
}

// src/m_geom.f90:29-46 (GM_dist_line), 2D
static double dist_line(const double r[2], const double r0[2], const double r1[2]) {
  double line_len2 = 0, temp = 0;
  for (int d = 0; d < 2; d++) line_len2 += (r1[d] - r0[d]) * (r1[d] - r0[d]);
  for (int d = 0; d < 2; d++) temp += (r[d] - r0[d]) * (r1[d] - r0[d]);
  double v[2];
  if (temp <= 0.0) {
    for (int d = 0; d < 2; d++) v[d] = r[d] - r0[d];
  } else if (temp >= line_len2) {
    for (int d = 0; d < 2; d++) v[d] = r[d] - r1[d];
  } else {
    for (int d = 0; d < 2; d++) {
      double proj = r0[d] + temp / line_len2 * (r1[d] - r0[d]);
      v[d] = r[d] - proj;
    }
  }
  return norm2(v, 2);
}

// src/m_geom.f90:48-111 (GM_dens_line and the fall-off shapes)
static double dens_line(const double r[2], const double r0[2], const double r1[2],
                        double width, int falloff) {
  double dist = dist_line(r, r0, r1);
  switch (falloff) {
    case 1: {
      double tmp = dist / width;
      if (tmp > std::log(0.5 * 1.7976931348623157e308)) return 0;
      return 2 / (1 + std::exp(tmp));
    }
    case 2: {
      double x = dist / width;
      return std::exp(-(x * x));
    }
    case 3: {
      if (dist < width) return 1;
      if (dist < 2 * width) {
        double temp = dist / width - 1;
        return (1 - (3 * (temp * temp) - 2 * (temp * temp * temp)));
      }
      return 0.0;
    }
    case 4: return dist < width ? 1.0 : 0.0;
    default: return 0;
  }
}

// src/streamer_2d.f90:250-266 (set_box_eps); cylindrical tests r, :271
static void set_box_eps(Sim &s, Box &b) {
  int nc = b.n_cell;
  for (int j = 0; j <= nc + 1; j++)
    for (int i = 0; i <= nc + 1; i++) {
      double xy[2];
      r_cc(b, i, j, xy);
      double rel = (b.coord == CYL ? xy[0] : xy[1]) / s.p.domain_len_z;
      b.c(i, j, I_EPS) = rel < 0.25 ? s.p.epsilon_diel : 1.0;
    }
}

// src/streamer_2d.f90:218-248 (set_init_cond)
static void set_init_cond(Sim &s, Box &b) {
  int nc = b.n_cell;
  const a5ref_params &p = s.p;
  for (int j = 0; j <= nc + 1; j++)
    for (int i = 0; i <= nc + 1; i++) b.c(i, j, I_ELEC) = p.bg_dens;
  for (int j = 0; j <= nc + 1; j++)
    for (int i = 0; i <= nc + 1; i++) {
      double xy[2];
      r_cc(b, i, j, xy);
      for (int n = 0; n < p.n_seeds; n++) {
        double dens = p.seed_dens[n] * dens_line(xy, p.seed_r0[n], p.seed_r1[n],
                                                 p.seed_width[n], p.seed_falloff[n]);
        b.c(i, j, I_ELEC) = b.c(i, j, I_ELEC) + dens;
      }
    }
  for (int j = 0; j <= nc + 1; j++)
    for (int i = 0; i <= nc + 1; i++) {
      b.c(i, j, I_PION) = b.c(i, j, I_ELEC);
      b.c(i, j, I_PHI) = 0;
    }
  set_box_eps(s, b);
}

static void loop_all_boxes(Tree &t, const std::function<void(Box &)> &f) {
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) f(t.boxes[L.ids[i]]);
  }
}
static void loop_leaves(Tree &t, const std::function<void(Box &, int)> &f) {
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.leaves.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) f(t.boxes[L.leaves[i]], L.leaves[i]);
  }
}

// src/streamer_2d.f90:177-216 (set_ref_flags); cyl :190-227
static void set_ref_flags(Sim &s, Tree &t, int id, std::vector<int> &rf) {
  Box &b = t.boxes[id];
  if (s.p.uniform_lvl > 0) {
    // uniformly refined mesh (the multigrid benchmark's,
    // afivo/examples/multigrid/test_mg_benchmark_2d.f90:40-86)
    rf[id] = b.lvl < s.p.uniform_lvl ? DO_REF : KP_REF;
    return;
  }
  int nc = b.n_cell;
  double dr2 = b.dr * b.dr;
  double mrhs = 0, max_fld = -1.7976931348623157e308;
  bool first = true;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) {
      double a = std::fabs(b.c(i, j, I_RHS));
      if (first) { mrhs = a; first = false; }
      else mrhs = std::max(mrhs, a);
      max_fld = std::max(max_fld, b.c(i, j, I_FLD));
    }
  double crv_phi = dr2 * mrhs;
  double alpha = lt_get_col(s.td, I_ALPHA, max_fld);
  double adx = b.dr * alpha;
  if (adx < 0.1 && b.dr < 2.0e-5) rf[id] = RM_REF;
  if (adx < 0.1 && crv_phi < 4.0 && b.dr < 5.0e-5) rf[id] = RM_REF;
  if (s.time < s.p.ref_init_time) {
    double boxlen = b.n_cell * b.dr;
    double ctr[2] = {b.r_min[0] + 0.5 * b.n_cell * b.dr, b.r_min[1] + 0.5 * b.n_cell * b.dr};
    for (int n = 0; n < s.p.n_seeds; n++) {
      double dist = dist_line(ctr, s.p.seed_r0[n], s.p.seed_r1[n]);
      if (dist - s.p.seed_width[n] < boxlen && b.dr > 0.2 * s.p.seed_width[n])
        rf[id] = DO_REF;
    }
  }
  if (adx > 1.0 && crv_phi > s.p.crv_refine) rf[id] = DO_REF;
}

// src/streamer_2d.f90:620-638 (sides_bc_pot); cyl :395-413 also fills the
// high-z corners
static void sides_bc_pot(Sim &s, Tree &t, int id, int nb, int iv) {
  Box &b = t.boxes[id];
  int nc = b.n_cell;
  double V = s.applied_voltage;
  switch (nb) {
    case NB_LX: for (int j = 1; j <= nc; j++) b.c(0, j, iv) = b.c(1, j, iv); break;
    case NB_HX: for (int j = 1; j <= nc; j++) b.c(nc + 1, j, iv) = b.c(nc, j, iv); break;
    case NB_LY: for (int i = 1; i <= nc; i++) b.c(i, 0, iv) = -b.c(i, 1, iv); break;
    case NB_HY:
      if (b.coord == CYL) {
        for (int i = 0; i <= nc + 1; i++) b.c(i, nc + 1, iv) = 2 * V - b.c(i, nc, iv);
      } else {
        for (int i = 1; i <= nc; i++) b.c(i, nc + 1, iv) = 2 * V - b.c(i, nc, iv);
      }
      break;
  }
}

// src/streamer_2d.f90:346-381 (fld_from_pot); cyl :357-392 is identical
static void fld_from_pot(Box &b) {
  int nc = b.n_cell;
  double inv_dr = 1 / b.dr;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc + 1; i++)
      b.Fx(i, j, F_FLD) = inv_dr * (b.c(i - 1, j, I_PHI) - b.c(i, j, I_PHI));
  for (int j = 1; j <= nc + 1; j++)
    for (int i = 1; i <= nc; i++)
      b.Fy(i, j, F_FLD) = inv_dr * (b.c(i, j - 1, I_PHI) - b.c(i, j, I_PHI));
  for (int j = 1; j <= nc; j++) {
    b.Fx(1, j, F_FLD) = 2 * inv_dr * (b.c(0, j, I_PHI) - b.c(1, j, I_PHI)) *
                        b.c(0, j, I_EPS) / (b.c(1, j, I_EPS) + b.c(0, j, I_EPS));
    b.Fx(nc + 1, j, F_FLD) = 2 * inv_dr * (b.c(nc, j, I_PHI) - b.c(nc + 1, j, I_PHI)) *
                             b.c(nc + 1, j, I_EPS) / (b.c(nc + 1, j, I_EPS) + b.c(nc, j, I_EPS));
  }
  for (int i = 1; i <= nc; i++) {
    b.Fy(i, 1, F_FLD) = 2 * inv_dr * (b.c(i, 0, I_PHI) - b.c(i, 1, I_PHI)) *
                        b.c(i, 0, I_EPS) / (b.c(i, 1, I_EPS) + b.c(i, 0, I_EPS));
    b.Fy(i, nc + 1, F_FLD) = 2 * inv_dr * (b.c(i, nc, I_PHI) - b.c(i, nc + 1, I_PHI)) *
                             b.c(i, nc + 1, I_EPS) / (b.c(i, nc + 1, I_EPS) + b.c(i, nc, I_EPS));
  }
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) {
      double sx = b.Fx(i, j, F_FLD) + b.Fx(i + 1, j, F_FLD);
      double sy = b.Fy(i, j, F_FLD) + b.Fy(i, j + 1, F_FLD);
      b.c(i, j, I_FLD) = std::sqrt(0.25 * (sx * sx) + 0.25 * (sy * sy));
    }
}

static void set_rhs(Sim &s) {
  // src/streamer_2d.f90:317-329: rhs = e/eps0 (n_e - n_i) on leaves, incl. ghosts
  const double fac = UC_ELEM_CHARGE / UC_EPS0;
  Tree &t = s.tree;
  for (int lvl = 1; lvl <= t.max_lvl; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.leaves.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      Box &b = t.boxes[L.leaves[i]];
      size_t m = (size_t)b.ncg() * b.ncg();
      double *rhs = &b.cc[m * I_RHS], *e = &b.cc[m * I_ELEC], *pi = &b.cc[m * I_PION];
      for (size_t k = 0; k < m; k++) rhs[k] = fac * (e[k] - pi[k]);
    }
  }
}

// src/streamer_2d.f90:307-343 (compute_fld)
static void compute_fld(Sim &s, int n_cycles, bool no_guess) {
  Tree &t = s.tree;
  set_rhs(s);
  s.applied_voltage = -s.p.domain_len_z * s.p.applied_fld;
  for (int i = 1; i <= n_cycles; i++) fas_fmg(t, s.mg, false, no_guess && i == 1);
  loop_all_boxes(t, [](Box &b) { fld_from_pot(b); });
  gc_tree(t, I_FLD, gc_interp, gc_neumann);
}

// src/streamer_2d.f90:384-489 (fluxes_koren); cyl :416-521 is identical
static void fluxes_koren(Sim &s, Tree &t, int id, double dt) {
  Box &b = t.boxes[id];
  int nc = b.n_cell;
  double inv_dr = 1 / b.dr;
  double fac = -0.8 * UC_EPS0 / (UC_ELEM_CHARGE * dt);
  double gc[4][64];
  gc2_box(t, id, I_ELEC, gc);
  const LT &td = s.td;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc + 1; i++) {
      double fld_avg = 0.5 * (b.c(i, j, I_FLD) + b.c(i - 1, j, I_FLD));
      Loc loc = lt_get_loc(td, fld_avg);
      double mobility = lt_col_at(td, I_MOBILITY, loc);
      double diff_coeff = lt_col_at(td, I_DIFFUSION, loc);
      double fld = b.Fx(i, j, F_FLD);
      double v_drift = -mobility * fld;
      double gradc = b.c(i, j, I_ELEC) - b.c(i - 1, j, I_ELEC);
      double f;
      if (v_drift < 0.0) {
        double tmp = (i == nc + 1) ? gc[NB_HX][j - 1] : b.c(i + 1, j, I_ELEC);
        double gradn = tmp - b.c(i, j, I_ELEC);
        f = v_drift * (b.c(i, j, I_ELEC) - koren_mlim(gradc, gradn));
        if (f < fac * fld) f = fac * fld;
      } else {
        double tmp = (i == 1) ? gc[NB_LX][j - 1] : b.c(i - 2, j, I_ELEC);
        double gradp = b.c(i - 1, j, I_ELEC) - tmp;
        f = v_drift * (b.c(i - 1, j, I_ELEC) + koren_mlim(gradc, gradp));
        if (f > fac * fld) f = fac * fld;
      }
      f = f - diff_coeff * gradc * inv_dr;
      b.Fx(i, j, F_ELEC) = f;
    }
  for (int j = 1; j <= nc + 1; j++)
    for (int i = 1; i <= nc; i++) {
      double fld_avg = 0.5 * (b.c(i, j, I_FLD) + b.c(i, j - 1, I_FLD));
      Loc loc = lt_get_loc(td, fld_avg);
      double mobility = lt_col_at(td, I_MOBILITY, loc);
      double diff_coeff = lt_col_at(td, I_DIFFUSION, loc);
      double fld = b.Fy(i, j, F_FLD);
      double v_drift = -mobility * fld;
      double gradc = b.c(i, j, I_ELEC) - b.c(i, j - 1, I_ELEC);
      double f;
      if (v_drift < 0.0) {
        double tmp = (j == nc + 1) ? gc[NB_HY][i - 1] : b.c(i, j + 1, I_ELEC);
        double gradn = tmp - b.c(i, j, I_ELEC);
        f = v_drift * (b.c(i, j, I_ELEC) - koren_mlim(gradc, gradn));
        if (f < fac * fld) f = fac * fld;
      } else {
        double tmp = (j == 1) ? gc[NB_LY][i - 1] : b.c(i, j - 2, I_ELEC);
        double gradp = b.c(i, j - 1, I_ELEC) - tmp;
        f = v_drift * (b.c(i, j - 1, I_ELEC) + koren_mlim(gradc, gradp));
        if (f > fac * fld) f = fac * fld;
      }
      f = f - diff_coeff * gradc * inv_dr;
      b.Fy(i, j, F_ELEC) = f;
    }
}

// afivo/src/m_aX_core.f90:847-930 (flux_from_children)
static void flux_from_children(Tree &t, int id, int nb, int f) {
  Box &p = t.boxes[id];
  int nc = p.n_cell, nch = nc >> 1;
  int nb_id = p.neighbors[nb];
  Box &bn = t.boxes[nb_id];
  int i, i_nb;
  if (nb_low[nb]) { i = 1; i_nb = nc + 1; }
  else { i = nc + 1; i_nb = 1; }
  for (int k = 0; k < 2; k++) {
    int i_ch = ch_adj_nb[nb][k];
    Box &c = t.boxes[p.children[i_ch]];
    int ioff0 = nch * ch_dix[i_ch][0], ioff1 = nch * ch_dix[i_ch][1];
    if (nb_dim[nb] == 0) {
      for (int m = 1; m <= nch; m++)
        bn.Fx(i_nb, ioff1 + m, f) = 0.5 * (c.Fx(i, 2 * m - 1, f) + c.Fx(i, 2 * m, f));
    } else {
      for (int m = 1; m <= nch; m++)
        bn.Fy(ioff0 + m, i_nb, f) = 0.5 * (c.Fy(2 * m - 1, i, f) + c.Fy(2 * m, i, f));
    }
  }
}

// afivo/src/m_aX_core.f90:818-843 (a$D_consistent_fluxes)
static void consistent_fluxes(Tree &t, int f) {
  for (int lvl = t.min_lvl; lvl <= t.max_lvl - 1; lvl++) {
    Level &L = t.L(lvl);
    int n = (int)L.parents.size();
#pragma omp parallel for schedule(static)
    for (int ii = 0; ii < n; ii++) {
      int id = L.parents[ii];
      for (int nb = 0; nb < NNB; nb++) {
        int nb_id = t.boxes[id].neighbors[nb];
        if (nb_id > NO_BOX && !has_children(t.boxes[nb_id])) flux_from_children(t, id, nb, f);
      }
    }
  }
}

// src/streamer_2d.f90:499-542 (update_solution); cyl :531-570
static void update_solution(Sim &s, Box &b, double dt) {
  int nc = b.n_cell;
  double inv_dr = 1 / b.dr;
  const LT &td = s.td;
  bool cyl = b.coord == CYL;
  int ioff = (b.ix[0] - 1) * nc;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) {
      double fld = b.c(i, j, I_FLD);
      Loc loc = lt_get_loc(td, fld);
      double alpha = lt_col_at(td, I_ALPHA, loc);
      double eta = lt_col_at(td, I_ETA, loc);
      double dflux[2] = {b.Fx(i, j, F_ELEC) + b.Fx(i + 1, j, F_ELEC),
                         b.Fy(i, j, F_ELEC) + b.Fy(i, j + 1, F_ELEC)};
      double src = 0.5 * norm2(dflux, 2) * (alpha - eta);
      if (s.p.photoi_enabled) src = src + b.c(i, j, I_PHO);
      double sflux;
      if (cyl) {
        double den = i + ioff - 0.5;
        double rf1 = (i + ioff - 1) / den, rf2 = (i + ioff) / den;
        sflux = (b.Fy(i, j, F_ELEC) - b.Fy(i, j + 1, F_ELEC) + rf1 * b.Fx(i, j, F_ELEC) -
                 rf2 * b.Fx(i + 1, j, F_ELEC)) * inv_dr;
      } else {
        sflux = (b.Fx(i, j, F_ELEC) - b.Fx(i + 1, j, F_ELEC) + b.Fy(i, j, F_ELEC) -
                 b.Fy(i, j + 1, F_ELEC)) * inv_dr;
      }
      b.c(i, j, I_ELEC) = b.c(i, j, I_ELEC) + (src + sflux) * dt;
      b.c(i, j, I_PION) = b.c(i, j, I_PION) + src * dt;
    }
  if (!cyl) {
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc; i++)
        if (b.c(i, j, I_EPS) > 1.0) {
          b.c(i, j, I_PION) = b.c(i, j, I_PION) - b.c(i, j, I_ELEC);
          b.c(i, j, I_ELEC) = 0;
        }
  }
}

// src/streamer_2d.f90:492-496 (average_dens)
static void average_dens(Box &b) {
  size_t m = (size_t)b.ncg() * b.ncg();
  for (int v = 0; v < 2; v++) {
    double *x = &b.cc[m * v], *o = &b.cc[m * (v + 2)];
    for (size_t k = 0; k < m; k++) x[k] = 0.5 * (x[k] + o[k]);
  }
}

// afivo/src/m_aX_utils.f90:432-453 (a$D_tree_copy_cc)
static void tree_copy_cc(Tree &t, int from, int to) {
  loop_all_boxes(t, [from, to](Box &b) { copy_full(b, from, to); });
}

// src/streamer_2d.f90:271-303 (get_max_dt); cyl :281-314
static void dt_reductions(Sim &s, double out[3]) {
  out[0] = tree_max_cc(s.tree, I_FLD);
  out[1] = tree_min_cc(s.tree, I_FLD);
  out[2] = tree_max_cc(s.tree, I_ELEC);
}
static double get_max_dt(Sim &s) {
  double r[3];
  dt_reductions(s, r);
  double max_fld = r[0], min_fld = r[1], max_dns = r[2];
  Tree &t = s.tree;
  double dr_min = t.dr_base * std::pow(0.5, t.max_lvl - 1);
  double mobility = lt_get_col(s.td, I_MOBILITY, max_fld);
  double max_mobility = lt_get_col(s.td, I_MOBILITY, min_fld);
  double diff_coeff = lt_get_col(s.td, I_DIFFUSION, max_fld);
  double alpha = lt_get_col(s.td, I_ALPHA, max_fld);
  double dt_cfl = dr_min / (mobility * max_fld);
  double dt_dif = 0.25 * (dr_min * dr_min) / diff_coeff;
  double dns = s.tree.coord == CYL ? std::max(2.220446049250313e-16, max_dns) : max_dns;
  double dt_drt = UC_EPS0 / (UC_ELEM_CHARGE * max_mobility * dns);
  double dt_alpha = 1 / std::max(mobility * max_fld * alpha, 2.220446049250313e-16);
  double m = std::min(std::min(1 / (1 / dt_cfl + 1 / dt_dif), dt_alpha), s.p.dt_max);
  if (s.p.use_drt) m = std::min(m, dt_drt);
  return 0.5 * m;
}

// afivo/src/m_aX_utils.f90:244-299 (a$D_get_loc with child_that_contains)
static void get_loc(Tree &t, const double rr[2], int max_lvl, int &id_out, int ix[2]) {
  const Level &L1 = t.L(1);
  int id = 0;
  size_t i;
  for (i = 0; i < L1.ids.size(); i++) {
    id = L1.ids[i];
    const Box &b = t.boxes[id];
    bool inside = true;
    for (int d = 0; d < 2; d++) {
      double r_max = b.r_min[d] + b.dr * b.n_cell;
      if (!(rr[d] >= b.r_min[d] && rr[d] <= r_max)) inside = false;
    }
    if (inside) break;
  }
  if (i == L1.ids.size()) {
    id_out = -1;
    ix[0] = ix[1] = -1;
    return;
  }
  while (t.boxes[id].lvl < max_lvl && has_children(t.boxes[id])) {
    const Box &b = t.boxes[id];
    int i_ch = 0;
    for (int d = 0; d < 2; d++) {
      double cntr = b.r_min[d] + b.dr * (b.n_cell >> 1);
      if (rr[d] > cntr) i_ch += 1 << d;
    }
    id = b.children[i_ch];
  }
  const Box &b = t.boxes[id];
  id_out = id;
  for (int d = 0; d < 2; d++) ix[d] = (int)std::ceil((rr[d] - b.r_min[d]) / b.dr);
}

// afivo/src/m_aX_prolong.f90:99-191 (a$D_prolong1_to) with add = .true.
static void prolong1_add(Tree &t, int id, int iv) {
  Box &b = t.boxes[id];
  const Box &p = t.boxes[b.parent];
  int nc = b.n_cell, hnc = nc >> 1, off[2];
  child_offset(b, -1, off);
  for (int j = 1; j <= hnc; j++) {
    int j_c = j + off[1], j_f = 2 * j - 1;
    for (int i = 1; i <= hnc; i++) {
      int i_c = i + off[0], i_f = 2 * i - 1;
      double f0 = 0.5 * p.c(i_c, j_c, iv);
      double flx = 0.25 * p.c(i_c - 1, j_c, iv), fhx = 0.25 * p.c(i_c + 1, j_c, iv);
      double fly = 0.25 * p.c(i_c, j_c - 1, iv), fhy = 0.25 * p.c(i_c, j_c + 1, iv);
      b.c(i_f, j_f, iv) = f0 + flx + fly + b.c(i_f, j_f, iv);
      b.c(i_f + 1, j_f, iv) = f0 + fhx + fly + b.c(i_f + 1, j_f, iv);
      b.c(i_f, j_f + 1, iv) = f0 + flx + fhy + b.c(i_f, j_f + 1, iv);
      b.c(i_f + 1, j_f + 1, iv) = f0 + fhx + fhy + b.c(i_f + 1, j_f + 1, iv);
    }
  }
}

// afivo/src/m_aX_utils.f90:623-656 (a$D_tree_sum_cc) run by a team of W
// threads: thread c sums fac * (box sum) over its static chunk of each
// level's leaves in level order; the partial sums are then added in thread
// order to the initial 0. Threads without boxes hold +0 and change nothing.
static double tree_sum_team(Tree &t, int iv, long W) {
  const double twopi = 2 * std::acos(-1.0);
  long n_busy = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    n_busy = std::max(n_busy, (long)t.L(lvl).leaves.size());
  n_busy = std::min(n_busy, W);
  double total = 0;
  for (long c = 0; c < n_busy; c++) {
    double my = 0;
    for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) {
      const double dr = t.dr_base * std::pow(0.5, lvl - 1);
      const double fac = dr * dr;
      const Level &L = t.L(lvl);
      long lo, len;
      static_chunk((long)L.leaves.size(), W, c, lo, len);
      for (long k = lo; k < lo + len; k++) {
        const Box &b = t.boxes[L.leaves[k]];
        const int nc = b.n_cell;
        double tmp = 0;
        if (t.coord == CYL) {
          // sum_2pr_box, :661-678
          for (int j = 1; j <= nc; j++)
            for (int i = 1; i <= nc; i++) tmp = tmp + b.c(i, j, iv) * (b.r_min[0] + (i - 0.5) * b.dr);
          tmp = tmp * twopi;
        } else {
          for (int j = 1; j <= nc; j++)
            for (int i = 1; i <= nc; i++) tmp = tmp + b.c(i, j, iv);
        }
        my = my + fac * tmp;
      }
    }
    total = total + my;
  }
  return total;
}

// src/streamer_cyl.f90:595-617 (set_photoi_rate) on one leaf box
static void set_photoi_rate(Sim &s, Box &b, double coeff) {
  const int nc = b.n_cell;
  for (int j = 1; j <= nc; j++)
    for (int i = 1; i <= nc; i++) {
      double fld = b.c(i, j, I_FLD);
      Loc loc = lt_get_loc(s.td, fld);
      double alpha = lt_col_at(s.td, I_ALPHA, loc);
      double mobility = lt_col_at(s.td, I_MOBILITY, loc);
      double tmp = fld * mobility * alpha * b.c(i, j, I_ELEC) * coeff;
      if (tmp < 0) tmp = 0;
      b.c(i, j, I_PHO) = tmp;
    }
}

// src/streamer_cyl.f90:572-593 (set_photoionization) and
// src/m_photons.f90:207-436 (PH_set_src_2d with i_src = i_pho, fac_dx,
// const_dx = .true., use_cyl = .true.), as run by a team of W threads (see
// a5ref.h): creation in thread order, absorption in static chunks.
static void set_photoionization(Sim &s, double dt, bool has_dt) {
  Tree &t = s.tree;
  const a5ref_params &p = s.p;
  const long W = p.photoi_team;
  const int nc = t.n_cell;
  const double pi = std::acos(-1.0);
  loop_leaves(t, [&](Box &b, int) { set_photoi_rate(s, b, p.photoi_coeff); });
  double sum_production = tree_sum_team(t, I_PHO, W);
  const double eps = 2.220446049250313e-16;
  double fac = p.photoi_num_photons / (sum_production + eps);
  if (has_dt) fac = dt < fac ? dt : fac;
  // photon creation, :263-306
  std::vector<Rng> rngs = prng_init(s.rng, (int)W);
  struct Src {
    int id, i, j;
  };
  std::vector<Src> src;
  for (long c = 0; c < W; c++) {
    for (int lvl = 1; lvl <= t.max_lvl; lvl++) {
      const double dr = t.dr_base * std::pow(0.5, lvl - 1);
      const Level &L = t.L(lvl);
      long lo, len;
      static_chunk((long)L.leaves.size(), W, c, lo, len);
      for (long k = lo; k < lo + len; k++) {
        const int id = L.leaves[k];
        const Box &b = t.boxes[id];
        for (int j = 1; j <= nc; j++)
          for (int i = 1; i <= nc; i++) {
            double tmp;
            if (b.coord == CYL) {
              double rc = b.r_min[0] + (i - 0.5) * b.dr;
              tmp = fac * 2 * pi * rc * b.c(i, j, I_PHO) * (dr * dr);
            } else {
              tmp = fac * b.c(i, j, I_PHO) * (dr * dr);
            }
            int n_create = (int)std::floor(tmp);
            if (rngs[c].uni_01() < tmp - n_create) n_create = n_create + 1;
            for (int q = 0; q < n_create; q++) src.push_back(Src{id, i, j});
          }
      }
    }
  }
  const long n_used = (long)src.size();
  s.n_photons = n_used;
  // absorption, PH_do_absorp (:161-205) in 3D, then the radius, :318-329
  std::vector<Rng> arngs = prng_init(s.rng, (int)W);
  std::vector<double> dst(2 * (size_t)n_used);
  for (long w = 0; w < W; w++) {
    long lo, len;
    static_chunk(n_used, W, w, lo, len);
    for (long n = lo; n < lo + len; n++) {
      const Box &b = t.boxes[src[n].id];
      double xin[3] = {b.r_min[0] + (src[n].i - 0.5) * b.dr, b.r_min[1] + (src[n].j - 0.5) * b.dr, 0};
      double rr = arngs[w].uni_01();
      double dist = lt_get_col(s.ph.tbl, 0, rr);
      double sph[3];
      arngs[w].sphere(dist, sph);
      double xo[3] = {xin[0] + sph[0], xin[1] + sph[1], xin[2] + sph[2]};
      dst[2 * n] = std::sqrt(xo[0] * xo[0] + xo[2] * xo[2]);
      dst[2 * n + 1] = xo[1];
    }
  }
  // absorption locations at level pho_lvl, :331-344
  std::vector<int> loc_id(n_used), loc_ix(2 * (size_t)n_used);
  for (long n = 0; n < n_used; n++) get_loc(t, &dst[2 * n], s.pho_lvl, loc_id[n], &loc_ix[2 * n]);
  // clear i_pho, :360-370
  for (int lvl = 1; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).ids) {
      Box &b = t.boxes[id];
      for (int j = 0; j <= nc + 1; j++)
        for (int i = 0; i <= nc + 1; i++) b.c(i, j, I_PHO) = 0;
    }
  // sequential deposit, :372-386
  const double tmp = fac * 2 * pi;
  for (long n = 0; n < n_used; n++) {
    int id = loc_id[n];
    if (id > NO_BOX) {
      int i = loc_ix[2 * n], j = loc_ix[2 * n + 1];
      Box &b = t.boxes[id];
      double dr = b.dr;
      double r0 = b.r_min[0] + (i - 0.5) * b.dr;
      b.c(i, j, I_PHO) = b.c(i, j, I_PHO) + s.ph.frac_in_tbl / (tmp * (dr * dr) * r0);
    }
  }
  // ghost cells and prolongation from the absorption level, :402-427
  for (int lvl = s.pho_lvl; lvl <= t.max_lvl - 1; lvl++) {
    for (int id : t.L(lvl).parents) gc_box(t, id, I_PHO, gc_interp, gc_neumann);
    for (int id : t.L(lvl).parents)
      for (int q = 0; q < NCH; q++) {
        int c_id = t.boxes[id].children[q];
        if (c_id == NO_BOX) continue;
        prolong1_add(t, c_id, I_PHO);
      }
  }
}

// src/streamer_2d.f90:99-127 (cyl :95-130), one iteration of the n loop at
// fixed dt, with set_photoionization first when it is enabled
static void step(Sim &s, double dt) {
  Tree &t = s.tree;
  if (s.p.photoi_enabled) set_photoionization(s, dt, true);
  s.time += dt;
  tree_copy_cc(t, I_ELEC, I_ELEC_OLD);
  tree_copy_cc(t, I_PION, I_PION_OLD);
  for (int i = 1; i <= 2; i++) {
    loop_leaves(t, [&](Box &, int id) { fluxes_koren(s, t, id, dt); });
    consistent_fluxes(t, F_ELEC);
    loop_leaves(t, [&](Box &b, int) { update_solution(s, b, dt); });
    restrict_tree(t, I_ELEC);
    restrict_tree(t, I_PION);
    gc_tree(t, I_ELEC, gc_interp_lim, gc_neumann);
    gc_tree(t, I_PION, gc_interp_lim, gc_neumann);
    if (i == 1) compute_fld(s, 1, false);
  }
  loop_all_boxes(t, [](Box &b) { average_dens(b); });
  compute_fld(s, 1, false);
}

// src/streamer_2d.f90:592-617 (prolong_to_new_boxes)
static void prolong_to_new_boxes(Sim &s, RefInfo &ri) {
  Tree &t = s.tree;
  for (int lvl = 1; lvl <= t.max_lvl; lvl++) {
    if (lvl >= (int)ri.add.size()) break;
    std::vector<int> &add = ri.add[lvl];
    int n = (int)add.size();
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      int id = add[i];
      prolong1_to(t, id, I_ELEC);
      prolong1_to(t, id, I_PION);
      prolong1_to(t, id, I_PHI);
      set_box_eps(s, t.boxes[id]);
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      int id = add[i];
      gc_box(t, id, I_ELEC, gc_interp_lim, gc_neumann);
      gc_box(t, id, I_PION, gc_interp_lim, gc_neumann);
      gc_box(t, id, I_PHI, s.mg.sides_rb, s.mg.sides_bc);
    }
  }
}

static void regrid(Sim &s, RefInfo &ri) {
  adjust_refinement(s.tree,
                    [&s](Tree &t, int id, std::vector<int> &rf) { set_ref_flags(s, t, id, rf); },
                    ri);
}

static bool setup(Sim &s) {
  const a5ref_params &p = s.p;
  double r0[2] = {0, 0};
  tree_init(s.tree, p.box_size, N_VAR_CELL, N_VAR_FACE, p.dr_base, r0, p.lvls_max, 2,
            p.coord);
  int nx = p.n_base[0], ny = p.n_base[1], n = nx * ny;
  std::vector<int> ixl(2 * n);
  std::vector<std::array<int, 4>> nbl(n);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int k = i + nx * j;
      ixl[2 * k] = i + 1;
      ixl[2 * k + 1] = j + 1;
      nbl[k][NB_LX] = i > 0 ? k : -1;              // box index k-1+1
      nbl[k][NB_HX] = i < nx - 1 ? k + 2 : -1;
      nbl[k][NB_LY] = j > 0 ? k + 1 - nx : -1;
      nbl[k][NB_HY] = j < ny - 1 ? k + 1 + nx : -1;
    }
  set_base(s.tree, n, reinterpret_cast<const int(*)[2]>(ixl.data()), nbl);
  s.td = lt_create(0.0, p.lkptbl_max_fld, p.lkptbl_size, 4);
  for (int c = 0; c < 4; c++) lt_set_col(s.td, c, p.td_x[c], p.td_y[c], p.td_n[c]);
  s.mg.i_phi = I_PHI;
  s.mg.i_tmp = I_FLD;
  s.mg.i_rhs = I_RHS;
  s.mg.i_eps = I_EPS;
  s.mg.n_cycle_base = p.n_cycle_base;
  s.mg.n_cycle_down = 2;
  s.mg.n_cycle_up = 2;
  s.mg.sides_rb = mg_sides_rb;
  Sim *sp = &s;
  s.mg.sides_bc = [sp](Tree &t, int id, int nb, int iv) { sides_bc_pot(*sp, t, id, nb, iv); };
  s.time = 0;
  s.applied_voltage = -p.domain_len_z * p.applied_fld;
  for (int i = 0; i < 4; i++) s.rng.st[i] = p.rng_seed[i];
  if (p.photoi_enabled) {
    // src/m_streamer.f90:327-330 builds the table; src/m_photons.f90:331-336
    // picks the absorption level from the length at fraction fac_dx
    AbsFn a = p.photoi_tbl_kind == 0 ? absfn_air(p.photoi_p_O2)
                                     : absfn_logu(p.photoi_len_lo, p.photoi_len_hi);
    if (!ph_get_tbl(a, p.photoi_max_dist, s.ph)) return false;
    s.pho_lvl = get_lvl_length(s.tree.dr_base, lt_get_col(s.ph.tbl, 0, p.photoi_fac_dx));
  }
  return true;
}

}  // namespace a5ref

// ---------------------------------------------------------------------------
// C API
using namespace a5ref;

struct a5ref_sim {
  Sim s;
};

static void apply_threads(const a5ref_params &p) {
#ifdef _OPENMP
  if (p.n_threads > 0) omp_set_num_threads(p.n_threads);
#else
  (void)p;
#endif
}

// a$D_reduction_loc with reduce_max (afivo/src/m_aX_utils.f90:499-555):
// leaves level by level in list order; a box result replaces the running one
// when max(tmp, running) differs from the running value. The reference's
// location is undefined when nothing replaces the initial value; here it is
// id -1 then.
template <class F>
static double reduction_max_loc(Tree &t, F box_subr, double init, int &id_out, int ix_out[2]) {
  double my_val = init;
  int my_id = -1, my_ix[2] = {-1, -1};
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) {
      double tmp;
      int tix[2] = {-1, -1};
      box_subr(t.boxes[id], tmp, tix);
      const double nv = std::max(tmp, my_val);
      if (std::fabs(nv - my_val) > 0) {
        my_id = id;
        my_ix[0] = tix[0];
        my_ix[1] = tix[1];
        my_val = tmp;
      }
    }
  id_out = -1;
  ix_out[0] = ix_out[1] = -1;
  const double nv = std::max(my_val, init);
  if (std::fabs(nv - init) > 0) {
    id_out = my_id;
    ix_out[0] = my_ix[0];
    ix_out[1] = my_ix[1];
    return my_val;
  }
  return init;
}

extern "C" {

a5ref_sim *a5ref_create(const a5ref_params *p) {
  if (!p || p->dim != 2 || p->box_size < 4 || (p->box_size & 1)) return nullptr;
  a5ref_sim *h = new a5ref_sim();
  h->s.p = *p;
  if (p->photoi_enabled && (p->coord != CYL || p->photoi_team < 1 || p->photoi_num_photons < 0)) {
    delete h;
    return nullptr;
  }
  apply_threads(*p);
  if (!setup(h->s)) {
    delete h;
    return nullptr;
  }
  return h;
}

void a5ref_destroy(a5ref_sim *h) { delete h; }

void a5ref_set_init_cond(a5ref_sim *h) {
  Sim &s = h->s;
  loop_all_boxes(s.tree, [&s](Box &b) { set_init_cond(s, b); });
}

int a5ref_init(a5ref_sim *h) {
  Sim &s = h->s;
  int it = 0;
  while (true) {
    it++;
    a5ref_set_init_cond(h);
    compute_fld(s, 1, true);
    RefInfo ri;
    regrid(s, ri);
    if (ri.n_add == 0) break;
    if (it > 100) break;
  }
  // src/streamer_cyl.f90:68-69
  if (s.p.photoi_enabled) set_photoionization(s, 0.0, false);
  return it;
}

void a5ref_dt_reductions(a5ref_sim *h, double out3[3]) { dt_reductions(h->s, out3); }
double a5ref_get_max_dt(a5ref_sim *h) { return get_max_dt(h->s); }
void a5ref_step(a5ref_sim *h, double dt) { step(h->s, dt); }

double a5ref_advance(a5ref_sim *h, int do_regrid) {
  Sim &s = h->s;
  double dt = get_max_dt(s);
  for (int n = 0; n < s.p.num_steps_amr; n++) step(s, dt);
  if (do_regrid) {
    RefInfo ri;
    regrid(s, ri);
    if (ri.n_add > 0 || ri.n_rm > 0) {
      prolong_to_new_boxes(s, ri);
      compute_fld(s, 1, false);
    }
  }
  return dt;
}

int a5ref_run(a5ref_sim *h, double t_end, int max_blocks) {
  int nb = 0;
  while (nb < max_blocks) {
    double dt = get_max_dt(h->s);
    if (dt < 1e-14) break;
    if (h->s.time > t_end) break;
    a5ref_advance(h, 1);
    nb++;
  }
  return nb;
}

double a5ref_time(a5ref_sim *h) { return h->s.time; }
void a5ref_set_time(a5ref_sim *h, double t) { h->s.time = t; }

void a5ref_op_copy_cc(a5ref_sim *h, int a, int b) { tree_copy_cc(h->s.tree, a, b); }
void a5ref_op_fluxes_koren(a5ref_sim *h, double dt) {
  Sim &s = h->s;
  loop_leaves(s.tree, [&](Box &, int id) { fluxes_koren(s, s.tree, id, dt); });
}
void a5ref_op_consistent_fluxes(a5ref_sim *h) { consistent_fluxes(h->s.tree, F_ELEC); }
void a5ref_op_update_solution(a5ref_sim *h, double dt) {
  Sim &s = h->s;
  loop_leaves(s.tree, [&](Box &b, int) { update_solution(s, b, dt); });
}
void a5ref_op_restrict_tree(a5ref_sim *h, int iv) { restrict_tree(h->s.tree, iv); }
void a5ref_op_gc_tree(a5ref_sim *h, int iv, int rb_kind) {
  if (rb_kind == 0) gc_tree(h->s.tree, iv, gc_interp_lim, gc_neumann);
  else gc_tree(h->s.tree, iv, gc_interp, gc_neumann);
}
void a5ref_op_average_dens(a5ref_sim *h) {
  loop_all_boxes(h->s.tree, [](Box &b) { average_dens(b); });
}
void a5ref_op_compute_fld(a5ref_sim *h, int no_guess) { compute_fld(h->s, 1, no_guess != 0); }
void a5ref_op_set_rhs(a5ref_sim *h) { set_rhs(h->s); }
void a5ref_op_fmg(a5ref_sim *h, int set_residual, int first_call) {
  h->s.applied_voltage = -h->s.p.domain_len_z * h->s.p.applied_fld;
  fas_fmg(h->s.tree, h->s.mg, set_residual != 0, first_call != 0);
}
// mg$D_fas_vcycle(tree, mg, set_residual, highest_lvl), afivo/src/m_aX_mg.f90:208-254
void a5ref_op_vcycle(a5ref_sim *h, int max_lvl, int set_residual) {
  h->s.applied_voltage = -h->s.p.domain_len_z * h->s.p.applied_fld;
  fas_vcycle(h->s.tree, h->s.mg, max_lvl, set_residual != 0);
}
void a5ref_op_fld_from_pot(a5ref_sim *h) {
  loop_all_boxes(h->s.tree, [](Box &b) { fld_from_pot(b); });
  gc_tree(h->s.tree, I_FLD, gc_interp, gc_neumann);
}
// a$D_tree_max_cc / _min_cc / _sum_cc, afivo/src/m_aX_utils.f90:559-680;
// the sum as a team of `team` OpenMP threads forms it (team 1: the loop order)
long long a5ref_photons_created(a5ref_sim *h) { return h->s.n_photons; }

// Level-set boundaries of the run's field solves: lsf and bval per cell in
// the export layout (ids 0..max_id); NULL removes them. Every box's
// multigrid tag is set again at its next use (mg$D_set_box_tag).
void a5ref_set_level_set(a5ref_sim *h, const double *lsf, const double *bval) {
  Sim &s = h->s;
  if (!lsf) {
    s.mg.i_lsf = s.mg.i_bval = -1;
  } else {
    a5ref_import_cc(h, I_LSF, lsf);
    a5ref_import_cc(h, I_BVAL, bval);
    s.mg.i_lsf = I_LSF;
    s.mg.i_bval = I_BVAL;
  }
  for (int id = 1; id <= s.tree.max_id; id++) s.tree.boxes[id].tag = INIT_TAG;
}

// ---------------------------------------------------------------------------
// Streamer diagnostics of the axisymmetric program, one thread.

// get_streamer_properties (src/streamer_cyl.f90:682-828): the 39 values in
// the reference's order, with box_maxfld_z / box_maxfld_r (maxloc: first
// maximum in column-major order), box_fld_maxr / box_fld_maxz (:835-903) and
// the alpha column read for both alpha and mu (:708-709, :718-719). The
// boundary stop (:721-723) is not taken.
void a5ref_streamer_properties(a5ref_sim *h, double *props) {
  Sim &s = h->s;
  Tree &t = s.tree;
  const double L = s.p.domain_len_z, V = s.applied_voltage;
  auto maxfld = [](bool radial) {
    return [radial](Box &b, double &val, int ix[2]) {
      const int nc = b.n_cell;
      double best = 0;
      bool first = true;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          const double a = radial ? std::fabs(b.Fx(i, j, F_FLD) + b.Fx(i + 1, j, F_FLD))
                                  : std::fabs(b.Fy(i, j, F_FLD) + b.Fy(i, j + 1, F_FLD));
          if (first || a > best) {
            best = a;
            ix[0] = i;
            ix[1] = j;
            first = false;
          }
        }
      val = radial ? 0.5 * std::fabs(b.Fx(ix[0], ix[1], F_FLD) + b.Fx(ix[0] + 1, ix[1], F_FLD))
                   : 0.5 * std::fabs(b.Fy(ix[0], ix[1], F_FLD) + b.Fy(ix[0], ix[1] + 1, F_FLD));
    };
  };
  auto fld_max_pos = [](double thr, int axis) {
    return [thr, axis](Box &b, double &val, int ix[2]) {
      val = 0;
      const int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++)
          if (b.c(i, j, I_FLD) > thr) {
            const double rz[2] = {b.r_min[0] + (i - 0.5) * b.dr, b.r_min[1] + (j - 0.5) * b.dr};
            if (rz[axis] > val) {
              val = rz[axis];
              ix[0] = i;
              ix[1] = j;
            }
          }
    };
  };
  int ip = 0;
  props[ip++] = s.p.applied_fld;  // ST_get_fld(ST_time), no field modulation
  int ez_id, ez_ix[2], er_id, er_ix[2];
  const double ez_max = reduction_max_loc(t, maxfld(false), -1.0e99, ez_id, ez_ix);
  props[ip++] = ez_max;
  props[ip++] = reduction_max_loc(t, maxfld(true), -1.0e99, er_id, er_ix);
  double rz[2];
  {
    const Box &b = t.boxes[er_id];
    rz[0] = b.r_min[0] + (er_ix[0] - 0.5) * b.dr;
    rz[1] = b.r_min[1] + (er_ix[1] - 0.5) * b.dr;
  }
  props[ip++] = rz[0];
  props[ip++] = rz[1];
  const double z_head = rz[1];
  const double er_norm = t.boxes[er_id].c(er_ix[0], er_ix[1], I_FLD);
  props[ip++] = er_norm;
  for (double e : {ez_max, er_norm}) {
    const double alpha = lt_get_col(s.td, I_ALPHA, e);
    const double mu = lt_get_col(s.td, I_ALPHA, e);
    props[ip++] = alpha;
    props[ip++] = alpha * mu * e;
  }
  int id, ix[2];
  {
    const double rr[2] = {0.0, rz[1]};
    get_loc(t, rr, t.lvls_max, id, ix);
  }
  props[ip++] = t.boxes[id].c(ix[0], ix[1], I_ELEC);
  const double phi_head = t.boxes[id].c(ix[0], ix[1], I_PHI);
  props[ip++] = phi_head - (rz[1] / L) * V;
  {
    const Box &b = t.boxes[ez_id];
    rz[0] = b.r_min[0] + (ez_ix[0] - 0.5) * b.dr;
    rz[1] = b.r_min[1] + (ez_ix[1] - 0.5) * b.dr;
  }
  props[ip++] = rz[1];
  for (double dz : {2.0e-3, 4.0e-3}) {
    const double rr[2] = {0.0, rz[1] + dz};
    int lid, lix[2];
    get_loc(t, rr, t.lvls_max, lid, lix);
    props[ip++] = lid > 0 ? phi_head - t.boxes[lid].c(lix[0], lix[1], I_PHI) : 0.0;
  }
  for (int i = 4; i <= 14; i += 2) {
    const double thr = i * 1e6;
    int lid, lix[2];
    props[ip++] = reduction_max_loc(t, fld_max_pos(thr, 0), 0.0, lid, lix);
    props[ip++] = lid > 0 ? phi_head - t.boxes[lid].c(lix[0], lix[1], I_PHI) : 0.0;
    props[ip++] = reduction_max_loc(t, fld_max_pos(thr, 1), 0.0, lid, lix) - z_head;
    props[ip++] = lid > 0 ? phi_head - t.boxes[lid].c(lix[0], lix[1], I_PHI) : 0.0;
  }
}

// The arrays a$D_write_vtk (afivo/src/m_aX_io.f90:20-207, 2D) builds for a
// file of the leaves of levels 1..max_lvl: node coordinates (2 per node,
// written by m_vtk.f90 as Float32 x 3), connectivity, offsets, cell types and
// the values of n_iv cell variables ivs plus, for n_if face variables ifs, the
// cell means of fx and fy. Any output may be NULL; returns the cell count.
int a5ref_vtk_arrays(a5ref_sim *h, int n_iv, const int *ivs, int n_if, const int *ifs,
                     double *coords, int *connects, int *offsets, int *types, double *vals) {
  Tree &t = h->s.tree;
  const int bc = t.n_cell, bn = t.n_cell + 1;
  const int nodes_per_box = bn * bn, cells_per_box = bc * bc;
  int n_grids = 0;
  for (int lvl = 1; lvl <= t.max_lvl; lvl++) n_grids += (int)t.L(lvl).leaves.size();
  const int n_cells = cells_per_box * n_grids;
  int ig = 0;
  for (int lvl = 1; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) {
      Box &b = t.boxes[id];
      ig++;
      const int cell_ix = (ig - 1) * cells_per_box, node_ix = (ig - 1) * nodes_per_box;
      for (int j = 1; j <= bn; j++)
        for (int i = 1; i <= bn; i++) {
          const int n_ix = 2 * (node_ix + (j - 1) * bn + i);  // 1-based pair end
          if (coords) {
            coords[n_ix - 2] = b.r_min[0] + (i - 1) * b.dr;
            coords[n_ix - 1] = b.r_min[1] + (j - 1) * b.dr;
          }
        }
      for (int j = 1; j <= bc; j++)
        for (int i = 1; i <= bc; i++) {
          const int n_ix = node_ix + (j - 1) * bn + i - 1;
          const int c_ix = cell_ix + (j - 1) * bc + i;  // 1-based
          if (vals) {
            for (int v = 0; v < n_iv; v++) vals[(size_t)v * n_cells + (c_ix - 1)] = b.c(i, j, ivs[v]);
            for (int f = 0; f < n_if; f++) {
              vals[(size_t)(n_iv + 2 * f) * n_cells + (c_ix - 1)] =
                  0.5 * (b.Fx(i, j, ifs[f]) + b.Fx(i + 1, j, ifs[f]));
              vals[(size_t)(n_iv + 2 * f + 1) * n_cells + (c_ix - 1)] =
                  0.5 * (b.Fy(i, j, ifs[f]) + b.Fy(i, j + 1, ifs[f]));
            }
          }
          if (offsets) offsets[c_ix - 1] = 4 * c_ix;
          if (types) types[c_ix - 1] = 8;  // VTK pixel
          if (connects) {
            const int q[4] = {n_ix, n_ix + 1, n_ix + bn, n_ix + bn + 1};
            for (int k = 0; k < 4; k++) connects[4 * (c_ix - 1) + k] = q[k];
          }
        }
    }
  return n_cells;
}

// get_cc_axis(tree, [i_elec, i_pion], [f_fld, f_elec]) (src/streamer_cyl.f90:
// 905-956): per axis cell z, n_e, n_i and the face averages of the field and
// the electron flux, box by box from z = 0 up. out: 5 x n (row-major by
// quantity), capacity cap cells; returns n (call with out NULL to size).
int a5ref_cc_axis(a5ref_sim *h, double *out, int cap) {
  Tree &t = h->s.tree;
  const int nc = t.n_cell;
  std::vector<double> z_l, e_l, i_l, f_l, x_l;
  double z = 0;
  while (true) {
    const double rr[2] = {0.0, z};
    int id, ix[2];
    get_loc(t, rr, t.lvls_max, id, ix);
    if (id == -1) break;
    Box &b = t.boxes[id];
    const double box_z = b.r_min[1], box_dz = b.dr;
    for (int j = 1; j <= nc; j++) {
      z_l.push_back(box_z + (j - 0.5) * box_dz);
      e_l.push_back(b.c(1, j, I_ELEC));
      i_l.push_back(b.c(1, j, I_PION));
      f_l.push_back(0.5 * (b.Fy(1, j, F_FLD) + b.Fy(1, j + 1, F_FLD)));
      x_l.push_back(0.5 * (b.Fy(1, j, F_ELEC) + b.Fy(1, j + 1, F_ELEC)));
    }
    z = box_z + (nc + 1) * box_dz;
  }
  const int n = (int)z_l.size();
  if (out && n <= cap) {
    const std::vector<double> *rows[5] = {&z_l, &e_l, &i_l, &f_l, &x_l};
    for (int r = 0; r < 5; r++)
      for (int k = 0; k < n; k++) out[(size_t)r * n + k] = (*rows[r])[k];
  }
  return n;
}
double a5ref_tree_max_cc(a5ref_sim *h, int iv) { return tree_max_cc(h->s.tree, iv); }
double a5ref_tree_min_cc(a5ref_sim *h, int iv) { return tree_min_cc(h->s.tree, iv); }
double a5ref_tree_sum_cc(a5ref_sim *h, int iv, int team) {
  return tree_sum_team(h->s.tree, iv, team < 1 ? 1 : team);
}
void a5ref_op_ref_flags(a5ref_sim *h, int *out) {
  Sim &s = h->s;
  Tree &t = s.tree;
  std::vector<int> rf(t.max_id + 1, -INT_MAX);
  for (int lvl = 1; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).ids) set_ref_flags(s, t, id, rf);
  for (int i = 0; i <= t.max_id; i++) out[i] = rf[i];
}
int a5ref_op_regrid(a5ref_sim *h, int *n_add, int *n_rm) {
  Sim &s = h->s;
  RefInfo ri;
  regrid(s, ri);
  if (ri.n_add > 0 || ri.n_rm > 0) prolong_to_new_boxes(s, ri);
  if (n_add) *n_add = ri.n_add;
  if (n_rm) *n_rm = ri.n_rm;
  return ri.n_add + ri.n_rm;
}

// Multigrid stages, for stepping the solver in lockstep with other
// implementations in the tests (afivo/src/m_aX_mg.f90:163-447).
void a5ref_dbg_set_rhs_voltage(a5ref_sim *h) {
  set_rhs(h->s);
  h->s.applied_voltage = -h->s.p.domain_len_z * h->s.p.applied_fld;
}
void a5ref_dbg_set_coarse(a5ref_sim *h, int lvl) { set_coarse_phi_rhs(h->s.tree, lvl, h->s.mg); }
void a5ref_dbg_fmg_pre(a5ref_sim *h, int lvl) {
  Tree &t = h->s.tree;
  for (int id : t.L(lvl).ids) copy_full(t.boxes[id], h->s.mg.i_phi, h->s.mg.i_tmp);
  if (lvl > t.min_lvl) {
    correct_children(t, t.L(lvl - 1).parents, h->s.mg);
    fill_gc_phi(t, t.L(lvl).ids, h->s.mg);
  }
}
void a5ref_dbg_gsrb(a5ref_sim *h, int lvl, int n_cycle) {
  gsrb_boxes(h->s.tree, h->s.tree.L(lvl).ids, h->s.mg, n_cycle);
}
void a5ref_dbg_update_coarse(a5ref_sim *h, int lvl) { update_coarse(h->s.tree, lvl, h->s.mg); }
void a5ref_dbg_correct_fill(a5ref_sim *h, int lvl) {
  Tree &t = h->s.tree;
  correct_children(t, t.L(lvl - 1).parents, h->s.mg);
  fill_gc_phi(t, t.L(lvl).ids, h->s.mg);
}

int a5ref_max_id(a5ref_sim *h) { return h->s.tree.max_id; }
int a5ref_max_lvl(a5ref_sim *h) { return h->s.tree.max_lvl; }
int a5ref_min_lvl(a5ref_sim *h) { return h->s.tree.min_lvl; }
int a5ref_n_leaf_cells(a5ref_sim *h) {
  Tree &t = h->s.tree;
  long n = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) n += (long)t.boxes[id].n_cell * t.boxes[id].n_cell;
  return (int)n;
}
int a5ref_n_cells_all(a5ref_sim *h) {
  Tree &t = h->s.tree;
  long n = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).ids) n += (long)t.boxes[id].n_cell * t.boxes[id].n_cell;
  return (int)n;
}

void a5ref_export_meta(a5ref_sim *h, int *meta) {
  Tree &t = h->s.tree;
  for (int id = 0; id <= t.max_id; id++) {
    int *m = meta + 16 * id;
    std::memset(m, 0, 16 * sizeof(int));
    if (id == 0) continue;
    const Box &b = t.boxes[id];
    m[0] = b.in_use;
    if (!b.in_use) continue;
    m[1] = b.lvl;
    m[2] = b.ix[0];
    m[3] = b.ix[1];
    m[4] = 0;
    m[5] = b.parent;
    for (int k = 0; k < 4; k++) m[6 + k] = b.children[k];
    for (int k = 0; k < 4; k++) m[10 + k] = b.neighbors[k];
    m[14] = b.n_cell;
  }
}

void a5ref_export_geom(a5ref_sim *h, double *g) {
  Tree &t = h->s.tree;
  for (int id = 0; id <= t.max_id; id++) {
    double *m = g + 4 * id;
    m[0] = m[1] = m[2] = m[3] = 0;
    if (id == 0 || !t.boxes[id].in_use) continue;
    m[0] = t.boxes[id].r_min[0];
    m[1] = t.boxes[id].r_min[1];
    m[3] = t.boxes[id].dr;
  }
}

int a5ref_export_levels(a5ref_sim *h, int *counts, int *ids, int cap) {
  Tree &t = h->s.tree;
  int k = 0, nl = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++, nl++) {
    Level &L = t.L(lvl);
    counts[3 * nl] = (int)L.ids.size();
    counts[3 * nl + 1] = (int)L.leaves.size();
    counts[3 * nl + 2] = (int)L.parents.size();
    for (const std::vector<int> *v : {&L.ids, &L.leaves, &L.parents})
      for (int id : *v) {
        if (k < cap) ids[k] = id;
        k++;
      }
  }
  return k;
}

void a5ref_export_cc(a5ref_sim *h, int iv, double *out) {
  Tree &t = h->s.tree;
  int S = (t.n_cell + 2) * (t.n_cell + 2);
  for (int id = 0; id <= t.max_id; id++) {
    double *o = out + (size_t)S * id;
    std::memset(o, 0, S * sizeof(double));
    if (id == 0 || !t.boxes[id].in_use) continue;
    const Box &b = t.boxes[id];
    int m = b.ncg() * b.ncg();
    std::memcpy(o, &b.cc[(size_t)m * iv], m * sizeof(double));
  }
}

void a5ref_import_cc(a5ref_sim *h, int iv, const double *in) {
  Tree &t = h->s.tree;
  int S = (t.n_cell + 2) * (t.n_cell + 2);
  for (int id = 1; id <= t.max_id; id++) {
    if (!t.boxes[id].in_use) continue;
    Box &b = t.boxes[id];
    int m = b.ncg() * b.ncg();
    std::memcpy(&b.cc[(size_t)m * iv], in + (size_t)S * id, m * sizeof(double));
  }
}

void a5ref_export_fc(a5ref_sim *h, int dimf, int f, double *out) {
  Tree &t = h->s.tree;
  int S = (t.n_cell + 1) * t.n_cell;
  for (int id = 0; id <= t.max_id; id++) {
    double *o = out + (size_t)S * id;
    std::memset(o, 0, S * sizeof(double));
    if (id == 0 || !t.boxes[id].in_use) continue;
    const Box &b = t.boxes[id];
    int m = (b.n_cell + 1) * b.n_cell;
    const std::vector<double> &src = dimf == 0 ? b.fx : b.fy;
    std::memcpy(o, &src[(size_t)m * f], m * sizeof(double));
  }
}

void a5ref_import_fc(a5ref_sim *h, int dimf, int f, const double *in) {
  Tree &t = h->s.tree;
  int S = (t.n_cell + 1) * t.n_cell;
  for (int id = 1; id <= t.max_id; id++) {
    if (!t.boxes[id].in_use) continue;
    Box &b = t.boxes[id];
    int m = (b.n_cell + 1) * b.n_cell;
    std::vector<double> &dst = dimf == 0 ? b.fx : b.fy;
    std::memcpy(&dst[(size_t)m * f], in + (size_t)S * id, m * sizeof(double));
  }
}

// The tree of a run checkpoint (the layout of a5s_checkpoint_save in the
// product library): per id 0..max_id, 14 ints (in_use, lvl, ix0, ix1,
// parent, n_cell, children[4], neighbors[4]) and 3 doubles (dr, r_min0,
// r_min1); the level lists of levels min_lvl .. min_lvl + n_lists - 1 as
// counts[3 k + {0,1,2}] and the ids concatenated. Boxes in use get zeroed
// storage (init_box) and the initial multigrid tag; cell and face data
// follow through a5ref_import_cc / a5ref_import_fc. Returns 0, or -1 if the
// tree does not fit this run. Lets the oracle resume from a checkpoint the
// device path wrote.
int a5ref_import_tree(a5ref_sim *h, int max_id, int min_lvl, int max_lvl, const int *rec_i,
                      const double *rec_d, int n_lists, const int *counts, const int *ids) {
  Tree &t = h->s.tree;
  if (!rec_i || !rec_d || !counts || max_id < 1 || min_lvl != t.min_lvl ||
      n_lists != (int)t.lv.size() || max_lvl < min_lvl || max_lvl > t.lvls_max)
    return -1;
  t.boxes.assign(max_id + 1, Box());
  for (int id = 1; id <= max_id; id++) {
    Box &b = t.boxes[id];
    const int *r = rec_i + 14 * id;
    const double *d = rec_d + 3 * id;
    b.lvl = r[1];
    b.ix[0] = r[2];
    b.ix[1] = r[3];
    b.parent = r[4];
    b.n_cell = r[5];
    for (int k = 0; k < 4; k++) b.children[k] = r[6 + k];
    for (int k = 0; k < 4; k++) b.neighbors[k] = r[10 + k];
    b.dr = d[0];
    b.r_min[0] = d[1];
    b.r_min[1] = d[2];
    b.coord = t.coord;
    if (r[0]) init_box(b, b.n_cell, t.n_var_cell, t.n_var_face);
  }
  t.max_id = max_id;
  t.max_lvl = max_lvl;
  int k = 0;
  for (int q = 0; q < n_lists; q++) {
    Level &L = t.lv[q];
    L.ids.assign(ids + k, ids + k + counts[3 * q]);
    k += counts[3 * q];
    L.leaves.assign(ids + k, ids + k + counts[3 * q + 1]);
    k += counts[3 * q + 1];
    L.parents.assign(ids + k, ids + k + counts[3 * q + 2]);
    k += counts[3 * q + 2];
  }
  return 0;
}

void a5ref_export_table(a5ref_sim *h, double *rows_cols, double *x_min, double *inv_dx,
                        int *n_rows) {
  const LT &td = h->s.td;
  if (rows_cols) std::memcpy(rows_cols, td.rows_cols.data(), td.rows_cols.size() * sizeof(double));
  if (x_min) *x_min = td.x_min;
  if (inv_dx) *inv_dx = td.inv_dx;
  if (n_rows) *n_rows = td.n_rows;
}

double a5ref_applied_voltage(a5ref_sim *h) { return h->s.applied_voltage; }

double a5ref_koren_mlim(double a, double b) { return koren_mlim(a, b); }

void a5ref_op_photoionization(a5ref_sim *h, double dt, int has_dt) {
  if (!h->s.p.photoi_enabled) return;
  set_photoionization(h->s, dt, has_dt != 0);
}
void a5ref_rng_get(a5ref_sim *h, int *st) {
  for (int i = 0; i < 4; i++) st[i] = h->s.rng.st[i];
}
void a5ref_rng_set(a5ref_sim *h, const int *st) {
  for (int i = 0; i < 4; i++) h->s.rng.st[i] = st[i];
}
int a5ref_photon_table(a5ref_sim *h, double *dist, int cap, double *frac, int *pho_lvl) {
  const PhTbl &ph = h->s.ph;
  if (dist)
    for (int i = 0; i < ph.tbl.n_rows && i < cap; i++) dist[i] = ph.tbl.rc(i + 1, 0);
  if (frac) *frac = ph.frac_in_tbl;
  if (pho_lvl) *pho_lvl = h->s.pho_lvl;
  return ph.tbl.n_rows;
}
int a5ref_kat_photon_table(int kind, double p_O2, double len_lo, double len_hi, double max_dist,
                           double *dist, double *frac) {
  PhTbl ph;
  AbsFn a = kind == 0 ? absfn_air(p_O2) : absfn_logu(len_lo, len_hi);
  if (!ph_get_tbl(a, max_dist, ph)) return -1;
  for (int i = 0; i < ph.tbl.n_rows; i++) dist[i] = ph.tbl.rc(i + 1, 0);
  *frac = ph.frac_in_tbl;
  return ph.tbl.n_rows;
}
double a5ref_kat_photon_dist(double p_O2, double max_dist, int n_photons, int n_team) {
  // src/test_m_photons.f90: PH_get_tbl_air(phtbl, 0.2, 10e-3), photons from
  // the origin, PH_do_absorp in 3D, mean of |xyz_out - xyz_in|
  PhTbl ph;
  if (!ph_get_tbl(absfn_air(p_O2), max_dist, ph)) return -1;
  Rng master;
  std::vector<Rng> r = prng_init(master, n_team);
  double sum = 0;
  for (long w = 0; w < n_team; w++) {
    long lo, len;
    static_chunk(n_photons, n_team, w, lo, len);
    for (long n = lo; n < lo + len; n++) {
      double rr = r[w].uni_01();
      double dist = lt_get_col(ph.tbl, 0, rr);
      double x[3];
      r[w].sphere(dist, x);
      sum += norm2(x, 3);
    }
  }
  return sum / n_photons;
}
void a5ref_kat_rng(const int *st, int n, int *out) {
  Rng r;
  for (int i = 0; i < 4; i++) r.st[i] = st[i];
  for (int k = 0; k < n; k++) out[k] = r.int4();
}

// ---------------------------------------------------------------------------
// Known-answer cases.

// afivo/examples/multigrid/test_mg2_2d.f90 and test_mg_cyl.f90
static int kat_mg(bool cyl, int n_fmg, double *res_out, double *err_out, int *max_lvl_out) {
  struct G { double a, x0, y0, s; };
  G g[2];
  if (cyl) {
    g[0] = G{1.0, 0.1, 0.25, 0.15};
    g[1] = G{1.0e-3, 0.75, 0.75, 0.05};
  } else {
    g[0] = G{1.0, 0.25, 0.25, 0.04};
    g[1] = G{1.0, 0.75, 0.75, 0.04};
  }
  auto gauss = [](const double x[2], const G &q) {
    double xr0 = (x[0] - q.x0) / q.s, xr1 = (x[1] - q.y0) / q.s;
    return std::exp(-(xr0 * xr0 + xr1 * xr1));
  };
  auto phi_sol = [&](const double x[2]) {
    double v = 0;
    for (const G &q : g) v = v + q.a * gauss(x, q);
    return v;
  };
  auto rhs_fn = [&](const double x[2]) {
    double v = 0;
    for (const G &q : g) {
      double xr0 = (x[0] - q.x0) / q.s, xr1 = (x[1] - q.y0) / q.s;
      double sum = xr0 * xr0 + xr1 * xr1;
      double l = cyl ? 4 / (q.s * q.s) * (sum - 1.0 - 0.5 * (x[0] - q.x0) / x[0]) * gauss(x, q)
                     : 4 / (q.s * q.s) * (sum - 1) * gauss(x, q);
      v = v + q.a * l;
    }
    return v;
  };
  const int i_phi = 0, i_tmp = 1, i_rhs = 2, i_err = 3;
  Tree t;
  double r0[2] = {0, 0};
  int box_size = 8;
  tree_init(t, box_size, 4, 0, 1.0 / box_size, r0, 30, 2, cyl ? CYL : XYZ);
  int ixl[1][2] = {{1, 1}};
  std::vector<std::array<int, 4>> nbl(1, std::array<int, 4>{-1, -1, -1, -1});
  set_base(t, 1, ixl, nbl);
  auto init = [&](Box &b) {
    int nc = b.n_cell;
    int lo = cyl ? 0 : 1, hi = cyl ? nc + 1 : nc;
    if (cyl)
      for (int j = 0; j <= nc + 1; j++)
        for (int i = 0; i <= nc + 1; i++) b.c(i, j, i_phi) = 0;
    for (int j = lo; j <= hi; j++)
      for (int i = lo; i <= hi; i++) {
        double xy[2];
        r_cc(b, i, j, xy);
        b.c(i, j, i_rhs) = rhs_fn(xy);
      }
  };
  RefFn ref;
  if (cyl) {
    ref = [](Tree &tt, int id, std::vector<int> &rf) {
      rf[id] = RM_REF;
      if (tt.boxes[id].lvl < 6) rf[id] = DO_REF;
    };
    for (int i = 0; i < 20; i++) {
      RefInfo ri;
      adjust_refinement(t, ref, ri);
      if (ri.n_add == 0) break;
    }
    loop_all_boxes(t, init);
  } else {
    ref = [&](Tree &tt, int id, std::vector<int> &rf) {
      Box &b = tt.boxes[id];
      int nc = b.n_cell;
      double m = 0;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) m = std::max(m, std::fabs(b.c(i, j, i_rhs)));
      if (b.dr * b.dr * m > 5.0e-4) rf[id] = DO_REF;
    };
    while (true) {
      loop_all_boxes(t, init);
      RefInfo ri;
      adjust_refinement(t, ref, ri);
      if (ri.n_add == 0) break;
    }
  }
  MG mg;
  mg.i_phi = i_phi;
  mg.i_tmp = i_tmp;
  mg.i_rhs = i_rhs;
  mg.n_cycle_down = 2;
  mg.n_cycle_up = 2;
  mg.n_cycle_base = 2;
  mg.sides_rb = mg_sides_rb;
  mg.sides_bc = [&](Tree &tt, int id, int nb, int iv) {
    Box &b = tt.boxes[id];
    int nc = b.n_cell;
    double xy[2];
    switch (nb) {
      case NB_LX:
        if (cyl) {
          for (int n = 1; n <= nc; n++) b.c(0, n, iv) = b.c(1, n, iv);
        } else {
          for (int n = 1; n <= nc; n++) {
            xy[0] = b.r_min[0] + (0.5 - 0.5) * b.dr;
            xy[1] = b.r_min[1] + (n - 0.5) * b.dr;
            b.c(0, n, iv) = 2 * phi_sol(xy) - b.c(1, n, iv);
          }
        }
        break;
      case NB_HX:
        for (int n = 1; n <= nc; n++) {
          xy[0] = b.r_min[0] + ((nc + 0.5) - 0.5) * b.dr;
          xy[1] = b.r_min[1] + (n - 0.5) * b.dr;
          b.c(nc + 1, n, iv) = 2 * phi_sol(xy) - b.c(nc, n, iv);
        }
        break;
      case NB_LY:
        for (int n = 1; n <= nc; n++) {
          xy[0] = b.r_min[0] + (n - 0.5) * b.dr;
          xy[1] = b.r_min[1] + (0.5 - 0.5) * b.dr;
          b.c(n, 0, iv) = 2 * phi_sol(xy) - b.c(n, 1, iv);
        }
        break;
      case NB_HY:
        for (int n = 1; n <= nc; n++) {
          xy[0] = b.r_min[0] + (n - 0.5) * b.dr;
          xy[1] = b.r_min[1] + ((nc + 0.5) - 0.5) * b.dr;
          b.c(n, nc + 1, iv) = 2 * phi_sol(xy) - b.c(n, nc, iv);
        }
        break;
    }
  };
  for (int it = 1; it <= n_fmg; it++) {
    fas_fmg(t, mg, true, it == 1);
    double max_err = 0;
    loop_all_boxes(t, [&](Box &b) {
      int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          double xy[2];
          r_cc(b, i, j, xy);
          b.c(i, j, i_err) = b.c(i, j, i_phi) - phi_sol(xy);
        }
    });
    double mn = tree_min_cc(t, i_tmp), mx = tree_max_cc(t, i_tmp);
    double emn = tree_min_cc(t, i_err), emx = tree_max_cc(t, i_err);
    max_err = std::max(std::fabs(emn), std::fabs(emx));
    if (res_out) res_out[it - 1] = std::max(std::fabs(mn), std::fabs(mx));
    if (err_out) err_out[it - 1] = max_err;
  }
  if (max_lvl_out) *max_lvl_out = t.max_lvl;
  long cells = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) cells += (long)t.boxes[id].n_cell * t.boxes[id].n_cell;
  return (int)cells;
}

// afivo/examples/multigrid/test_mg_cyl_diel.f90: cylindrical Poisson
// problem with eps = 100 in the quadrant r < 0.5, z < 0.5 and 1 elsewhere,
// manufactured solution of two Gaussians; rhs = eps * lpl(phi) plus the
// surface charge at the eps jumps, split between the two cells of a face in
// proportion to their eps; Neumann on the axis, Dirichlet phi_sol elsewhere;
// refinement where dr^2 max|rhs / eps| > 5e-4. The multigrid uses the eps
// operators (box tags from the eps of each box).
static int kat_mg_diel(int n_fmg, double *res_out, double *err_out, int *max_lvl_out) {
  struct G { double a, x0, y0, s; };
  const G g[2] = {G{1.0, 0.25, 0.25, 0.04}, G{1.0, 0.75, 0.75, 0.04}};
  auto gauss = [](const double x[2], const G &q) {
    double xr0 = (x[0] - q.x0) / q.s, xr1 = (x[1] - q.y0) / q.s;
    return std::exp(-(xr0 * xr0 + xr1 * xr1));
  };
  auto phi_sol = [&](const double x[2]) {
    double v = 0;
    for (const G &q : g) v = v + q.a * gauss(x, q);
    return v;
  };
  auto phi_grad = [&](const double x[2], double gr[2]) {
    gr[0] = gr[1] = 0;
    for (const G &q : g) {
      double xr0 = (x[0] - q.x0) / q.s, xr1 = (x[1] - q.y0) / q.s, e = gauss(x, q);
      gr[0] = gr[0] + q.a * (-2 * xr0 / q.s * e);
      gr[1] = gr[1] + q.a * (-2 * xr1 / q.s * e);
    }
  };
  auto lpl = [&](const double x[2]) {
    double v = 0;
    for (const G &q : g) {
      double xr0 = (x[0] - q.x0) / q.s, xr1 = (x[1] - q.y0) / q.s;
      double sum = xr0 * xr0 + xr1 * xr1;
      v = v + q.a * (4 / (q.s * q.s) * (sum - 1.0 - 0.5 * (x[0] - q.x0) / x[0]) * gauss(x, q));
    }
    return v;
  };
  const int i_phi = 0, i_tmp = 1, i_rhs = 2, i_err = 3, i_eps = 4;
  Tree t;
  double r0[2] = {0, 0};
  const int box_size = 8;
  tree_init(t, box_size, 5, 0, 1.0 / box_size, r0, 30, 2, CYL);
  int ixl[1][2] = {{1, 1}};
  std::vector<std::array<int, 4>> nbl(1, std::array<int, 4>{-1, -1, -1, -1});
  set_base(t, 1, ixl, nbl);
  auto rr = [](const Box &b, double fi, double fj, double xy[2]) {
    xy[0] = b.r_min[0] + (fi - 0.5) * b.dr;
    xy[1] = b.r_min[1] + (fj - 0.5) * b.dr;
  };
  auto init = [&](Box &b) {
    const int nc = b.n_cell;
    const double dr = b.dr;
    for (int j = 0; j <= nc + 1; j++)
      for (int i = 0; i <= nc + 1; i++) {
        double xy[2];
        r_cc(b, i, j, xy);
        b.c(i, j, i_phi) = 0;
        b.c(i, j, i_eps) = (xy[0] < 0.5 && xy[1] < 0.5) ? 100.0 : 1.0;
        b.c(i, j, i_rhs) = lpl(xy) * b.c(i, j, i_eps);
      }
    for (int j = 1; j <= nc; j++)
      for (int i = 0; i <= nc; i++) {
        double xy[2], gr[2];
        rr(b, i + 0.5, (double)j, xy);
        phi_grad(xy, gr);
        double qbnd = (b.c(i + 1, j, i_eps) - b.c(i, j, i_eps)) * gr[0] / dr;
        double w = b.c(i + 1, j, i_eps) / (b.c(i, j, i_eps) + b.c(i + 1, j, i_eps));
        b.c(i + 1, j, i_rhs) = b.c(i + 1, j, i_rhs) + w * qbnd;
        b.c(i, j, i_rhs) = b.c(i, j, i_rhs) + (1 - w) * qbnd;
      }
    for (int j = 0; j <= nc; j++)
      for (int i = 1; i <= nc; i++) {
        double xy[2], gr[2];
        rr(b, (double)i, j + 0.5, xy);
        phi_grad(xy, gr);
        double qbnd = (b.c(i, j + 1, i_eps) - b.c(i, j, i_eps)) * gr[1] / dr;
        double w = b.c(i, j + 1, i_eps) / (b.c(i, j, i_eps) + b.c(i, j + 1, i_eps));
        b.c(i, j + 1, i_rhs) = b.c(i, j + 1, i_rhs) + w * qbnd;
        b.c(i, j, i_rhs) = b.c(i, j, i_rhs) + (1 - w) * qbnd;
      }
  };
  RefFn ref = [&](Tree &tt, int id, std::vector<int> &rf) {
    Box &b = tt.boxes[id];
    int nc = b.n_cell;
    double m = 0;
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc; i++) m = std::max(m, std::fabs(b.c(i, j, i_rhs) / b.c(i, j, i_eps)));
    if (b.dr * b.dr * m > 5.0e-4) rf[id] = DO_REF;
  };
  while (true) {
    loop_all_boxes(t, init);
    RefInfo ri;
    adjust_refinement(t, ref, ri);
    if (ri.n_add == 0) break;
  }
  loop_all_boxes(t, init);
  MG mg;
  mg.i_phi = i_phi;
  mg.i_tmp = i_tmp;
  mg.i_rhs = i_rhs;
  mg.i_eps = i_eps;
  mg.n_cycle_down = 2;
  mg.n_cycle_up = 2;
  mg.n_cycle_base = 2;
  mg.sides_rb = mg_sides_rb;
  mg.sides_bc = [&](Tree &tt, int id, int nb, int iv) {
    Box &b = tt.boxes[id];
    const int nc = b.n_cell;
    double xy[2];
    for (int n = 1; n <= nc; n++) {
      switch (nb) {
        case NB_LX: b.c(0, n, iv) = b.c(1, n, iv); break;
        case NB_HX:
          rr(b, nc + 0.5, (double)n, xy);
          b.c(nc + 1, n, iv) = 2 * phi_sol(xy) - b.c(nc, n, iv);
          break;
        case NB_LY:
          rr(b, (double)n, 0.5, xy);
          b.c(n, 0, iv) = 2 * phi_sol(xy) - b.c(n, 1, iv);
          break;
        default:
          rr(b, (double)n, nc + 0.5, xy);
          b.c(n, nc + 1, iv) = 2 * phi_sol(xy) - b.c(n, nc, iv);
      }
    }
  };
  for (int it = 1; it <= n_fmg; it++) {
    fas_fmg(t, mg, true, it == 1);
    loop_all_boxes(t, [&](Box &b) {
      int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          double xy[2];
          r_cc(b, i, j, xy);
          b.c(i, j, i_err) = b.c(i, j, i_phi) - phi_sol(xy);
        }
    });
    double mn = tree_min_cc(t, i_tmp), mx = tree_max_cc(t, i_tmp);
    double emn = tree_min_cc(t, i_err), emx = tree_max_cc(t, i_err);
    if (res_out) res_out[it - 1] = std::max(std::fabs(mn), std::fabs(mx));
    if (err_out) err_out[it - 1] = std::max(std::fabs(emn), std::fabs(emx));
  }
  if (max_lvl_out) *max_lvl_out = t.max_lvl;
  int n_diel = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).ids)
      if (t.boxes[id].tag == MG_CEPS_BOX || t.boxes[id].tag == MG_VEPS_BOX) n_diel++;
  return n_diel;
}

int a5ref_kat_mg_cyl_diel(int n_fmg, double *res, double *err, int *ml) {
  return kat_mg_diel(n_fmg, res, err, ml);
}

// afivo/examples/multigrid/test_mg3_2d.f90: a jump in eps (1 below y = 0.5,
// 4 above) on the unit square, 2x2-cell boxes, refined to level 4 everywhere
// and to level 7 within 5 dr of the centre (:90-101), phi = 0 at the bottom
// and 1 at the top, Neumann sides (:120-141), no charge, FMG cycles with
// set_residual (:64-69). The known answer is the layered solution: continuity
// of eps dphi/dy gives phi = 1.6 y below the interface and 0.8 + 0.4 (y - 0.5)
// above it. Per cycle: max |residual| and max |phi - exact| over the leaves.
static int kat_mg3_2d(int n_fmg, double *res_out, double *err_out, int *max_lvl_out) {
  const int i_phi = 0, i_tmp = 1, i_rhs = 2, i_eps = 3, i_err = 4;
  Tree t;
  const double r0[2] = {0, 0};
  const int box_size = 2;
  tree_init(t, box_size, 5, 0, 1.0 / box_size, r0, 30, 0, XYZ);
  const int ixl[1][2] = {{1, 1}};
  std::vector<std::array<int, 4>> nbl(1, std::array<int, 4>{-1, -1, -1, -1});
  set_base(t, 1, ixl, nbl);
  auto exact = [](double y) { return y < 0.5 ? 1.6 * y : 0.8 + 0.4 * (y - 0.5); };
  const RefFn ref = [&](Tree &tt, int id, std::vector<int> &rf) {
    const Box &b = tt.boxes[id];
    const double d = 5 * b.dr;
    bool inside = true;
    for (int k = 0; k < 2; k++) {
      const double r_max = b.r_min[k] + b.dr * b.n_cell;
      if (!(0.5 + d >= b.r_min[k] && 0.5 - d <= r_max)) inside = false;
    }
    rf[id] = (b.lvl < 4 || (b.lvl < 7 && inside)) ? DO_REF : KP_REF;
  };
  for (int it = 0; it < 20; it++) {
    RefInfo ri;
    adjust_refinement(t, ref, ri);
    if (ri.n_add == 0) break;
  }
  loop_all_boxes(t, [&](Box &b) {
    const int nc = b.n_cell;
    for (int j = 0; j <= nc + 1; j++)
      for (int i = 0; i <= nc + 1; i++) {
        double xy[2];
        r_cc(b, i, j, xy);
        b.c(i, j, i_phi) = 0;
        b.c(i, j, i_rhs) = 0;
        b.c(i, j, i_eps) = xy[1] < 0.5 ? 1.0 : 4.0;
      }
  });
  MG mg;
  mg.i_phi = i_phi;
  mg.i_tmp = i_tmp;
  mg.i_rhs = i_rhs;
  mg.i_eps = i_eps;
  mg.n_cycle_down = 2;
  mg.n_cycle_up = 2;
  mg.n_cycle_base = 2;
  mg.sides_rb = mg_sides_rb;
  mg.sides_bc = [](Tree &tt, int id, int nb, int iv) {
    Box &b = tt.boxes[id];
    const int nc = b.n_cell;
    for (int n = 1; n <= nc; n++) {
      switch (nb) {
        case NB_LX: b.c(0, n, iv) = b.c(1, n, iv); break;
        case NB_HX: b.c(nc + 1, n, iv) = b.c(nc, n, iv); break;
        case NB_LY: b.c(n, 0, iv) = -b.c(n, 1, iv); break;
        default: b.c(n, nc + 1, iv) = 2 - b.c(n, nc, iv);
      }
    }
  };
  for (int it = 1; it <= n_fmg; it++) {
    fas_fmg(t, mg, true, it == 1);
    loop_all_boxes(t, [&](Box &b) {
      const int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          double xy[2];
          r_cc(b, i, j, xy);
          b.c(i, j, i_err) = b.c(i, j, i_phi) - exact(xy[1]);
        }
    });
    const double mn = tree_min_cc(t, i_tmp), mx = tree_max_cc(t, i_tmp);
    const double emn = tree_min_cc(t, i_err), emx = tree_max_cc(t, i_err);
    if (res_out) res_out[it - 1] = std::max(std::fabs(mn), std::fabs(mx));
    if (err_out) err_out[it - 1] = std::max(std::fabs(emn), std::fabs(emx));
  }
  if (max_lvl_out) *max_lvl_out = t.max_lvl;
  int n_leaf = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) n_leaf += (int)t.L(lvl).leaves.size();
  return n_leaf;
}

int a5ref_kat_mg3_2d(int n_fmg, double *res, double *err, int *ml) {
  return kat_mg3_2d(n_fmg, res, err, ml);
}

// afivo/examples/multigrid/test_mgb_2d.f90: internal boundaries from a level
// set on the 4 x 4 square (8x8-cell boxes, refined uniformly to level 6,
// :32-44, 83-89), phi = phi0 = 1e3 on the zero contour, phi = 0 at the
// bottom and top, Neumann sides (:115-131), no charge, FMG cycles with the
// level-set operators on the boxes the contour crosses (mg2_auto_*, default
// restriction). shape 0: the example's ellipse sqrt(100 x^2 + y^2) - 1.8
// around the centre (:100-104); shape 1: the plane y = 1.3, whose exact
// solution phi0 y / 1.3 below and phi0 (4 - y) / 2.7 above satisfies the
// operators' one-sided differences exactly. Per cycle: max |residual| and
// (shape 1) max |phi - exact| over the leaves; returns the boxes tagged.
static int kat_mgb_2d(int shape, int n_fmg, double *res_out, double *err_out) {
  const int i_phi = 0, i_tmp = 1, i_rhs = 2, i_lsf = 3, i_bval = 4, i_err = 5;
  const double phi0 = 1e3, y0 = 1.3;
  Tree t;
  const double r0[2] = {0, 0};
  const int box_size = 8;
  tree_init(t, box_size, 6, 0, 4.0 / box_size, r0, 30, 8, XYZ);
  const int ixl[1][2] = {{1, 1}};
  std::vector<std::array<int, 4>> nbl(1, std::array<int, 4>{-1, -1, -1, -1});
  set_base(t, 1, ixl, nbl);
  const RefFn ref = [](Tree &tt, int id, std::vector<int> &rf) {
    if (tt.boxes[id].lvl < 6) rf[id] = DO_REF;
  };
  for (int it = 0; it < 20; it++) {
    RefInfo ri;
    adjust_refinement(t, ref, ri);
    if (ri.n_add == 0) break;
  }
  auto exact = [&](double y) { return y < y0 ? phi0 * y / y0 : phi0 * (4 - y) / (4 - y0); };
  loop_all_boxes(t, [&](Box &b) {
    const int nc = b.n_cell;
    for (int j = 0; j <= nc + 1; j++)
      for (int i = 0; i <= nc + 1; i++) {
        double xy[2];
        r_cc(b, i, j, xy);
        const double x = xy[0] - 2, y = xy[1] - 2;
        b.c(i, j, i_phi) = 0;
        b.c(i, j, i_rhs) = 0;
        b.c(i, j, i_lsf) = shape == 0 ? std::sqrt(100 * (x * x) + y * y) - 1.8 : xy[1] - y0;
        b.c(i, j, i_bval) = phi0;
      }
  });
  MG mg;
  mg.i_phi = i_phi;
  mg.i_tmp = i_tmp;
  mg.i_rhs = i_rhs;
  mg.i_lsf = i_lsf;
  mg.i_bval = i_bval;
  mg.sides_rb = mg_sides_rb;
  mg.sides_bc = [](Tree &tt, int id, int nb, int iv) {
    Box &b = tt.boxes[id];
    const int nc = b.n_cell;
    for (int n = 1; n <= nc; n++) {
      switch (nb) {
        case NB_LX: b.c(0, n, iv) = b.c(1, n, iv); break;
        case NB_HX: b.c(nc + 1, n, iv) = b.c(nc, n, iv); break;
        case NB_LY: b.c(n, 0, iv) = -b.c(n, 1, iv); break;
        default: b.c(n, nc + 1, iv) = -b.c(n, nc, iv);
      }
    }
  };
  for (int it = 1; it <= n_fmg; it++) {
    fas_fmg(t, mg, true, it == 1);
    loop_all_boxes(t, [&](Box &b) {
      const int nc = b.n_cell;
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          double xy[2];
          r_cc(b, i, j, xy);
          b.c(i, j, i_err) = b.c(i, j, i_phi) - exact(xy[1]);
        }
    });
    const double mn = tree_min_cc(t, i_tmp), mx = tree_max_cc(t, i_tmp);
    if (res_out) res_out[it - 1] = std::max(std::fabs(mn), std::fabs(mx));
    if (err_out)
      err_out[it - 1] = std::max(std::fabs(tree_min_cc(t, i_err)), std::fabs(tree_max_cc(t, i_err)));
  }
  int n_lsf = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).ids)
      if (t.boxes[id].tag == MG_LSF_BOX) n_lsf++;
  return n_lsf;
}

int a5ref_kat_mgb_2d(int shape, int n_fmg, double *res, double *err) {
  return kat_mgb_2d(shape, n_fmg, res, err);
}

int a5ref_kat_mg2_2d(int n_fmg, double *res, double *err, int *ml) {
  return kat_mg(false, n_fmg, res, err, ml);
}

// afivo/examples/transport/test_drift_diff_2d.f90: phi advected with velocity
// (1, 1) on the periodic square [0, 2 pi]^2 (one base box of 8 x 8 cells, its
// own neighbour on every side, no coarse levels), exact solution
// sin^4(x - t) cos^4(y - t) (:187-200). Koren-limited upwind fluxes with the
// second ghost layer (:283-348, here with the oracle's koren_mlim), flux
// consistency, the update (:351-361), restriction and limited ghost cells,
// the trapezoidal step of time_step_method 2 (:84-101), dt = 0.5 / (sum |v| /
// dr_min + eps) (:68-70; no diffusion), a regrid after every step with the
// example's criterion (:131-153) and prolong_to_new_children (:369-389).
// This runs the oracle's own transport machinery -- gc2_box, gc_tree with
// gc_interp_lim, consistent_fluxes, restrict_tree, prolong1_to and
// adjust_refinement -- against a known solution.
//  uniform_lvl > 0: refine uniformly to that level instead (no regrid steps);
//  regrid = 0: no regrid after the initial mesh (frozen mesh).
// out: [0] max |error| over the leaves at the end (a$D_tree_max_cc /
// _min_cc of phi - solution, :103-117), [1] mean |error| (cell-size
// weighted), [2] sum of phi at the start and [3] at the end
// (a$D_tree_sum_cc), [4] steps, [5] max level, [6] leaf cells, [7] time.
static int kat_drift_diff(int uniform_lvl, double end_time, int regrid, double *out) {
  const int nc = 8, v_phi = 0, v_old = 1, v_err = 2;
  const double two_pi = 2 * std::acos(-1.0);
  const double vel[2] = {1.0, 1.0}, diff_coeff = 0.0;
  Tree t;
  const double r0[2] = {0, 0};
  tree_init(t, nc, 3, 1, two_pi / nc, r0, 20, 0, XYZ);
  const int ixl[1][2] = {{1, 1}};
  std::vector<std::array<int, 4>> nbl(1, std::array<int, 4>{1, 1, 1, 1});
  set_base(t, 1, ixl, nbl);
  auto solution = [&](double x, double y, double tm) {
    const double a = std::sin(x - vel[0] * tm), b = std::cos(y - vel[1] * tm);
    const double a2 = a * a, b2 = b * b;
    return (a2 * a2) * (b2 * b2);
  };
  auto set_init = [&](Box &b) {
    for (int j = 0; j <= nc + 1; j++)
      for (int i = 0; i <= nc + 1; i++) {
        const double x = b.r_min[0] + (i - 0.5) * b.dr, y = b.r_min[1] + (j - 0.5) * b.dr;
        b.c(i, j, v_phi) = solution(x, y, 0.0);
      }
  };
  int n_bc = 0;  // physical-boundary calls: none exist on the periodic square
  const GcFn no_bc = [&n_bc](Tree &, int, int, int) { n_bc++; };
  const RefFn ref_fn = [&](Tree &tt, int id, std::vector<int> &rf) {
    const Box &b = tt.boxes[id];
    if (uniform_lvl > 0) {
      rf[id] = b.lvl < uniform_lvl ? DO_REF : KP_REF;
      return;
    }
    double diff = 0;
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc + 1; i++)
        diff = std::max(diff, std::fabs(b.c(i, j, v_phi) - b.c(i - 1, j, v_phi)));
    for (int j = 1; j <= nc + 1; j++)
      for (int i = 1; i <= nc; i++)
        diff = std::max(diff, std::fabs(b.c(i, j, v_phi) - b.c(i, j - 1, v_phi)));
    if (b.lvl < 3 || diff > 0.05) rf[id] = DO_REF;
    else if (diff > 0.2 * 0.05) rf[id] = KP_REF;
    else if (b.lvl > 4) rf[id] = RM_REF;
  };
  RefInfo ri;
  do {
    for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
      for (int id : t.L(lvl).ids) set_init(t.boxes[id]);
    gc_tree(t, v_phi, gc_interp_lim, no_bc);
    adjust_refinement(t, ref_fn, ri);
  } while (ri.n_add > 0);
  restrict_tree(t, v_phi);
  gc_tree(t, v_phi, gc_interp_lim, no_bc);

  auto tree_sum = [&]() { return tree_sum_team(t, v_phi, 1); };
  // Koren fluxes of the example (:283-348) for velocity vel and diffusion 0
  auto fluxes = [&](int id) {
    Box &b = t.boxes[id];
    const double inv_dr = 1 / b.dr;
    double gc[4][64];
    gc2_box(t, id, v_phi, gc);
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc + 1; i++) {
        const double gradc = b.c(i, j, v_phi) - b.c(i - 1, j, v_phi);
        double f;
        if (vel[0] < 0.0) {
          const double tmp = i == nc + 1 ? gc[NB_HX][j - 1] : b.c(i + 1, j, v_phi);
          f = vel[0] * (b.c(i, j, v_phi) - koren_mlim(gradc, tmp - b.c(i, j, v_phi)));
        } else {
          const double tmp = i == 1 ? gc[NB_LX][j - 1] : b.c(i - 2, j, v_phi);
          f = vel[0] * (b.c(i - 1, j, v_phi) + koren_mlim(gradc, b.c(i - 1, j, v_phi) - tmp));
        }
        b.Fx(i, j, 0) = f - diff_coeff * gradc * inv_dr;
      }
    for (int j = 1; j <= nc + 1; j++)
      for (int i = 1; i <= nc; i++) {
        const double gradc = b.c(i, j, v_phi) - b.c(i, j - 1, v_phi);
        double f;
        if (vel[1] < 0.0) {
          const double tmp = j == nc + 1 ? gc[NB_HY][i - 1] : b.c(i, j + 1, v_phi);
          f = vel[1] * (b.c(i, j, v_phi) - koren_mlim(gradc, tmp - b.c(i, j, v_phi)));
        } else {
          const double tmp = j == 1 ? gc[NB_LY][i - 1] : b.c(i, j - 2, v_phi);
          f = vel[1] * (b.c(i, j - 1, v_phi) + koren_mlim(gradc, b.c(i, j - 1, v_phi) - tmp));
        }
        b.Fy(i, j, 0) = f - diff_coeff * gradc * inv_dr;
      }
  };
  auto update = [&](Box &b, double dt) {
    const double inv_dr = 1 / b.dr;
    for (int j = 1; j <= nc; j++)
      for (int i = 1; i <= nc; i++)
        b.c(i, j, v_phi) = b.c(i, j, v_phi) +
                           dt * ((b.Fx(i, j, 0) - b.Fx(i + 1, j, 0)) * inv_dr +
                                 (b.Fy(i, j, 0) - b.Fy(i, j + 1, 0)) * inv_dr);
  };
  const double sum0 = tree_sum();
  double time = 0;
  int steps = 0;
  while (true) {
    const double dr_min = t.dr_base * std::pow(0.5, t.max_lvl - 1);
    const double dt = 0.5 / (2 * diff_coeff * (2 / (dr_min * dr_min)) +
                             (std::fabs(vel[0]) / dr_min + std::fabs(vel[1]) / dr_min) +
                             2.220446049250313e-16);
    if (time > end_time) break;
    tree_copy_cc(t, v_phi, v_old);
    for (int stage = 0; stage < 2; stage++) {
      for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) {
        const Level &L = t.L(lvl);
        const int n = (int)L.ids.size();
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n; k++) fluxes(L.ids[k]);
      }
      consistent_fluxes(t, 0);
      for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
        for (int id : t.L(lvl).ids) update(t.boxes[id], dt);
      restrict_tree(t, v_phi);
      gc_tree(t, v_phi, gc_interp_lim, no_bc);
    }
    for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
      for (int id : t.L(lvl).ids) {
        Box &b = t.boxes[id];
        const size_t m = (size_t)b.ncg() * b.ncg();
        for (size_t k = 0; k < m; k++) b.cc[k + m * v_phi] = 0.5 * (b.cc[k + m * v_phi] + b.cc[k + m * v_old]);
      }
    time = time + dt;
    steps++;
    if (regrid && uniform_lvl <= 0) {
      adjust_refinement(t, ref_fn, ri);
      for (int lvl = 1; lvl <= t.max_lvl && lvl < (int)ri.add.size(); lvl++) {
        for (int id : ri.add[lvl]) prolong1_to(t, id, v_phi);
        for (int id : ri.add[lvl]) gc_box(t, id, v_phi, gc_interp_lim, no_bc);
      }
      gc_tree(t, v_phi, gc_interp_lim, no_bc);
    }
  }
  double emax = 0, esum = 0, area = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++)
    for (int id : t.L(lvl).leaves) {
      Box &b = t.boxes[id];
      for (int j = 1; j <= nc; j++)
        for (int i = 1; i <= nc; i++) {
          const double x = b.r_min[0] + (i - 0.5) * b.dr, y = b.r_min[1] + (j - 0.5) * b.dr;
          const double e = b.c(i, j, v_phi) - solution(x, y, time);
          b.c(i, j, v_err) = e;
          emax = std::max(emax, std::fabs(e));
          esum += std::fabs(e) * b.dr * b.dr;
          area += b.dr * b.dr;
        }
    }
  long long n_leaf = 0;
  for (int lvl = t.min_lvl; lvl <= t.max_lvl; lvl++) n_leaf += (long long)t.L(lvl).leaves.size() * nc * nc;
  out[0] = emax;
  out[1] = esum / area;
  out[2] = sum0;
  out[3] = tree_sum();
  out[4] = steps;
  out[5] = t.max_lvl;
  out[6] = (double)n_leaf;
  out[7] = time;
  return n_bc == 0 ? 0 : -1;
}

int a5ref_kat_drift_diff(int uniform_lvl, double end_time, int regrid, double *out8) {
  return kat_drift_diff(uniform_lvl, end_time, regrid, out8);
}
int a5ref_kat_mg_cyl(int n_fmg, double *res, double *err, int *ml) {
  return kat_mg(true, n_fmg, res, err, ml);
}

// fosito/test/test_m_lookup_table.f90:40-60: table of sin(x) built from
// n_pairs samples on (0, x_max], evaluated at n_samples points.
double a5ref_kat_lookup(int n_rows, int n_pairs, double x_max, int n_samples) {
  std::vector<double> xs(n_pairs), ys(n_pairs);
  for (int i = 1; i <= n_pairs; i++) {
    xs[i - 1] = i / ((double)n_pairs / x_max);
    ys[i - 1] = std::sin(xs[i - 1]);
  }
  LT t = lt_create(xs[0], xs[n_pairs - 1], n_rows, 1);
  lt_set_col(t, 0, xs.data(), ys.data(), n_pairs);
  double md = 0;
  int stride = std::max(1, n_pairs / n_samples);
  for (int i = 0; i < n_pairs; i += stride)
    md = std::max(md, std::fabs(lt_get_col(t, 0, xs[i]) - ys[i]));
  return md;
}

}  // extern "C"

// The 3D octree form (uniformly refined octrees), same translation unit.
#include "a5ref3.inc"
#include "a5ref_tl.inc"
