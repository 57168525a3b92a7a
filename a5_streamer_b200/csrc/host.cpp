// Host side of liba5g.so: quadtree topology (a5t_*) and the streamer driver
// loop (a5s_*). The topology routines restate Afivo's core
// (afivo/src/m_aX_core.f90) on structure-of-arrays storage; the driver
// restates src/streamer_2d.f90 / src/streamer_cyl.f90 with all box data on
// the device. Everything here is integer bookkeeping or one-time setup
// (initial conditions, table build); the per-step work runs in a5g.cu.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/a5t.h"
#include "a5_internal.h"

namespace {

// afivo/src/m_aX_t.f90:41-81 (2D), 0-based child / neighbour numbering
const int kChDix[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
const int kChRev[4][2] = {{1, 2}, {0, 3}, {3, 0}, {2, 1}};
const int kChAdjNb[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};
const int kNbRev[4] = {1, 0, 3, 2};
constexpr int kRmRef = -1, kKpRef = 0, kDoRef = 1, kDerefine = -2, kRefine = 2;
constexpr int kUnset = INT_MIN + 1;  // -huge(1)

inline bool nb_is_low(int nb) { return (nb & 1) == 0; }
inline int nb_dim(int nb) { return nb >> 1; }

int err(int code, const std::string &m) { return a5g_internal_fail(code, m.c_str()); }

}  // namespace

struct a5t_tree {
  int nc = 8, lvls_max = 30, min_lvl = 1, max_lvl = 0, max_id = 0, coord = 0;
  double dr_base = 0, r_base[2] = {0, 0};
  // per id (index 0 unused)
  std::vector<char> in_use{0};
  std::vector<int> lvl{0}, ix0{0}, ix1{0}, parent{0}, ncell{0};
  std::vector<std::array<int, 4>> ch{{0, 0, 0, 0}}, nb{{0, 0, 0, 0}};
  std::vector<double> dr{0}, rmin0{0}, rmin1{0};
  // per level, index lvl - min_lvl, levels min_lvl..lvls_max+1
  std::vector<std::vector<int>> ids, leaves, parents, added;

  int li(int l) const { return l - min_lvl; }
  bool has_children(int id) const { return ch[id][0] != 0; }

  int grow_ids(int n) {  // get_free_ids, m_aX_core.f90:588-600
    int first = max_id + 1;
    max_id += n;
    in_use.resize(max_id + 1, 0);
    lvl.resize(max_id + 1, 0);
    ix0.resize(max_id + 1, 0);
    ix1.resize(max_id + 1, 0);
    parent.resize(max_id + 1, 0);
    ncell.resize(max_id + 1, 0);
    ch.resize(max_id + 1, {0, 0, 0, 0});
    nb.resize(max_id + 1, {0, 0, 0, 0});
    dr.resize(max_id + 1, 0);
    rmin0.resize(max_id + 1, 0);
    rmin1.resize(max_id + 1, 0);
    return first;
  }

  void split_level(int l) {  // set_leaves_parents, m_aX_core.f90:328-359
    auto &L = ids[li(l)];
    leaves[li(l)].clear();
    parents[li(l)].clear();
    for (int id : L) (has_children(id) ? parents : leaves)[li(l)].push_back(id);
  }

  int neighbour_via_parent(int id, int n) const {  // find_nb, m_aX_core.f90:427-445
    int p = parent[id];
    int cix = 3 - 2 * (ix1[id] & 1) - (ix0[id] & 1);
    int d = nb_dim(n);
    bool child_low = kChDix[cix][d] == 0;
    if (child_low == nb_is_low(n)) p = nb[p][n];
    return ch[p][kChRev[cix][d]];
  }

  void link_neighbours(int id) {  // set_nbs, m_aX_core.f90:386-400
    for (int n = 0; n < 4; n++) {
      if (nb[id][n] != 0) continue;
      int other = neighbour_via_parent(id, n);
      if (other > 0) {
        nb[id][n] = other;
        nb[other][kNbRev[n]] = id;
      }
    }
  }

  void add_children(int id) {  // add_children, m_aX_core.f90:753-788
    int first = grow_ids(4);
    for (int k = 0; k < 4; k++) ch[id][k] = first + k;
    for (int k = 0; k < 4; k++) {
      int c = first + k;
      in_use[c] = 1;
      ix0[c] = 2 * ix0[id] - 1 + kChDix[k][0];
      ix1[c] = 2 * ix1[id] - 1 + kChDix[k][1];
      lvl[c] = lvl[id] + 1;
      parent[c] = id;
      ch[c] = {0, 0, 0, 0};
      nb[c] = {0, 0, 0, 0};
      ncell[c] = ncell[id];
      dr[c] = 0.5 * dr[id];
      rmin0[c] = rmin0[id] + 0.5 * dr[id] * kChDix[k][0] * ncell[id];
      rmin1[c] = rmin1[id] + 0.5 * dr[id] * kChDix[k][1] * ncell[id];
    }
    for (int n = 0; n < 4; n++)
      if (nb[id][n] < 0)
        for (int q = 0; q < 2; q++) nb[first + kChAdjNb[n][q]][n] = nb[id][n];
  }

  void remove_children(int id) {  // remove_children, m_aX_core.f90:729-750
    for (int k = 0; k < 4; k++) {
      int c = ch[id][k];
      for (int n = 0; n < 4; n++)
        if (nb[c][n] > 0) nb[nb[c][n]][kNbRev[n]] = 0;
      in_use[c] = 0;
    }
    ch[id] = {0, 0, 0, 0};
  }

  // consistent_ref_flags, m_aX_core.f90:624-726, from user flags per id
  std::vector<int> consistent_flags(const int *user) const {
    std::vector<int> rf(max_id + 1, kUnset);
    for (int l = 1; l <= max_lvl; l++)
      for (int id : ids[li(l)]) rf[id] = user[id];
    for (int id = 1; id <= max_id; id++)
      if (rf[id] > kDoRef || rf[id] < kRmRef) rf[id] = kKpRef;
    for (int id : ids[li(lvls_max)])
      if (rf[id] == kDoRef) rf[id] = kKpRef;
    for (int l = max_lvl; l >= 1; l--) {
      for (int id : leaves[li(l)]) {
        if (rf[id] > kKpRef) {
          rf[id] = kRefine;
          for (int n = 0; n < 4; n++)
            if (nb[id][n] == 0) rf[nb[parent[id]][n]] = kRefine;
        } else if (rf[id] == kRmRef) {
          for (int n = 0; n < 4; n++) {
            int o = nb[id][n];
            if (o > 0 && (has_children(o) || rf[o] > kKpRef)) {
              rf[id] = kKpRef;
              break;
            }
          }
        }
      }
    }
    for (int l = max_lvl - 1; l >= 1; l--)
      for (int id : parents[li(l)]) {
        bool all_rm = true;
        for (int k = 0; k < 4; k++) all_rm = all_rm && rf[ch[id][k]] == kRmRef;
        rf[id] = (all_rm && rf[id] <= kKpRef) ? kDerefine : kKpRef;
      }
    return rf;
  }
};

extern "C" {

int a5t_create(int box_size, int lvls_max, double dr_base, const double r_base[2], int coord,
               a5t_tree **out) {
  if (!out) return err(A5G_EINVAL, "null argument");
  *out = nullptr;
  if (box_size < 4 || (box_size & (box_size - 1))) return err(A5G_EINVAL, "box_size must be a power of two >= 4");
  if (lvls_max < 1 || lvls_max > 30) return err(A5G_EINVAL, "lvls_max must be 1..30");
  if (!(dr_base > 0)) return err(A5G_EINVAL, "dr_base must be > 0");
  a5t_tree *t = new a5t_tree();
  t->nc = box_size;
  t->lvls_max = lvls_max;
  t->dr_base = dr_base;
  t->r_base[0] = r_base ? r_base[0] : 0;
  t->r_base[1] = r_base ? r_base[1] : 0;
  t->coord = coord;
  // coarsen_to = 2: min_lvl = 1 - log2(box_size / 2), a$D_init :84-93
  int k = 0;
  while ((2 << k) < box_size) k++;
  t->min_lvl = 1 - k;
  int nlev = lvls_max + 2 - t->min_lvl;
  t->ids.assign(nlev, {});
  t->leaves.assign(nlev, {});
  t->parents.assign(nlev, {});
  t->added.assign(nlev, {});
  *out = t;
  return A5G_OK;
}

int a5t_destroy(a5t_tree *t) {
  delete t;
  return A5G_OK;
}

int a5t_set_base(a5t_tree *t, int n_boxes, const int *ix_list, const int *nb_list) {
  if (!t || !ix_list || !nb_list || n_boxes < 1) return err(A5G_EINVAL, "bad argument");
  if (t->max_id > 0) return err(A5G_ESTATE, "tree already has boxes");
  std::vector<std::array<int, 4>> nbl(n_boxes);
  for (int i = 0; i < n_boxes; i++) {
    if (ix_list[2 * i] < 1 || ix_list[2 * i + 1] < 1) return err(A5G_EINVAL, "need all ix_list > 0");
    for (int n = 0; n < 4; n++) nbl[i][n] = nb_list[4 * i + n];
  }
  for (int i = 0; i < n_boxes; i++)
    for (int n = 0; n < 4; n++) {
      int o = nbl[i][n];
      if (o > n_boxes) return err(A5G_EINVAL, "neighbour index out of range");
      if (o > 0 && o != i + 1) nbl[o - 1][kNbRev[n]] = i + 1;
    }
  for (int i = 0; i < n_boxes; i++)
    for (int n = 0; n < 4; n++)
      if (nbl[i][n] == 0) return err(A5G_EINVAL, "unresolved neighbours");
  // a$D_set_base, m_aX_core.f90:163-212: copies of level 1 down to min_lvl
  std::vector<int> prev;
  for (int l = t->min_lvl; l <= 1; l++) {
    int first = t->grow_ids(n_boxes);
    int offset = first - 1;
    std::vector<int> cur(n_boxes);
    for (int i = 0; i < n_boxes; i++) {
      int id = first + i;
      cur[i] = id;
      t->in_use[id] = 1;
      t->lvl[id] = l;
      t->ix0[id] = ix_list[2 * i];
      t->ix1[id] = ix_list[2 * i + 1];
      t->dr[id] = t->dr_base * std::pow(0.5, l - 1);
      t->rmin0[id] = t->r_base[0] + (ix_list[2 * i] - 1) * t->dr_base * t->nc;
      t->rmin1[id] = t->r_base[1] + (ix_list[2 * i + 1] - 1) * t->dr_base * t->nc;
      t->ncell[id] = t->nc / (1 << (1 - l));
      t->parent[id] = 0;
      t->ch[id] = {0, 0, 0, 0};
      for (int n = 0; n < 4; n++) t->nb[id][n] = nbl[i][n] > 0 ? nbl[i][n] + offset : nbl[i][n];
    }
    t->ids[t->li(l)] = cur;
    if (l == 1) t->leaves[t->li(l)] = cur;
    else t->parents[t->li(l)] = cur;
    if (l > t->min_lvl)
      for (int i = 0; i < n_boxes; i++) {
        t->ch[prev[i]][0] = cur[i];
        t->parent[cur[i]] = prev[i];
      }
    prev = cur;
  }
  t->max_lvl = 1;
  return A5G_OK;
}

int a5t_adjust_refinement(a5t_tree *t, const int *user, int *n_add, int *n_rm) {
  if (!t || !user) return err(A5G_EINVAL, "null argument");
  if (t->max_id == 0) return err(A5G_ESTATE, "no base mesh");
  const int max_id_prev = t->max_id;
  std::vector<int> rf = t->consistent_flags(user);
  int na = 0, nr = 0;
  for (auto &a : t->added) a.clear();
  // a$D_adjust_refinement, m_aX_core.f90:478-515
  int l;
  for (l = 1; l <= t->lvls_max - 1; l++) {
    std::vector<int> here = t->ids[t->li(l)];
    for (int id : here) {
      if (id > max_id_prev) continue;
      if (rf[id] == kRefine) {
        t->add_children(id);
        na += 4;
      } else if (rf[id] == kDerefine) {
        t->remove_children(id);
        nr += 4;
      }
    }
    t->split_level(l);
    auto &next = t->ids[t->li(l + 1)];
    next.clear();
    for (int p : t->parents[t->li(l)])
      for (int k = 0; k < 4; k++) next.push_back(t->ch[p][k]);
    for (int id : next)
      if (id > max_id_prev) t->link_neighbours(id);
    if (next.empty()) break;
  }
  if (l > t->lvls_max - 1) l = t->lvls_max;
  t->max_lvl = l;
  t->split_level(t->max_lvl + 1);
  // ref_info%lvls(lvl)%add: children of refined boxes in id order (:571-583)
  for (int id = 1; id <= max_id_prev; id++)
    if (rf[id] == kRefine)
      for (int k = 0; k < 4; k++) t->added[t->li(t->lvl[id] + 1)].push_back(t->ch[id][k]);
  if (n_add) *n_add = na;
  if (n_rm) *n_rm = nr;
  return A5G_OK;
}

int a5t_max_id(a5t_tree *t) { return t ? t->max_id : -1; }
int a5t_min_lvl(a5t_tree *t) { return t ? t->min_lvl : 0; }
int a5t_max_lvl(a5t_tree *t) { return t ? t->max_lvl : 0; }

int a5t_n_level_ids(a5t_tree *t) {
  if (!t) return -1;
  int n = 0;
  for (int l = t->min_lvl; l <= t->max_lvl; l++)
    n += (int)(t->ids[t->li(l)].size() + t->leaves[t->li(l)].size() + t->parents[t->li(l)].size());
  return n;
}

int a5t_export(a5t_tree *t, int *meta16, double *geom4, int *lvl_counts, int *lvl_ids) {
  if (!t) return err(A5G_EINVAL, "null tree");
  if (meta16) {
    std::memset(meta16, 0, sizeof(int) * 16 * (t->max_id + 1));
    for (int id = 1; id <= t->max_id; id++) {
      int *m = meta16 + 16 * id;
      m[0] = t->in_use[id];
      if (!t->in_use[id]) continue;
      m[1] = t->lvl[id];
      m[2] = t->ix0[id];
      m[3] = t->ix1[id];
      m[5] = t->parent[id];
      for (int k = 0; k < 4; k++) m[6 + k] = t->ch[id][k];
      for (int k = 0; k < 4; k++) m[10 + k] = t->nb[id][k];
      m[14] = t->ncell[id];
    }
  }
  if (geom4) {
    std::memset(geom4, 0, sizeof(double) * 4 * (t->max_id + 1));
    for (int id = 1; id <= t->max_id; id++)
      if (t->in_use[id]) {
        geom4[4 * id] = t->rmin0[id];
        geom4[4 * id + 1] = t->rmin1[id];
        geom4[4 * id + 3] = t->dr[id];
      }
  }
  int k = 0, q = 0;
  for (int l = t->min_lvl; l <= t->max_lvl; l++, q++) {
    const std::vector<int> *v3[3] = {&t->ids[t->li(l)], &t->leaves[t->li(l)], &t->parents[t->li(l)]};
    for (int kind = 0; kind < 3; kind++) {
      if (lvl_counts) lvl_counts[3 * q + kind] = (int)v3[kind]->size();
      for (int id : *v3[kind]) {
        if (lvl_ids) lvl_ids[k] = id;
        k++;
      }
    }
  }
  return k;
}

int a5t_new_boxes(a5t_tree *t, int *counts, int *ids) {
  if (!t) return err(A5G_EINVAL, "null tree");
  int k = 0, q = 0;
  for (int l = t->min_lvl; l <= t->max_lvl; l++, q++) {
    const auto &a = t->added[t->li(l)];
    if (counts) counts[q] = (int)a.size();
    for (int id : a) {
      if (ids) ids[k] = id;
      k++;
    }
  }
  return k;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Streamer driver
namespace {

// gfortran's inline NORM2 (scaled sum of squares)
double norm2v(const double *x, int n) {
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

// GM_dist_line / GM_dens_line, src/m_geom.f90:29-111 (2D)
double seed_density(const double r[2], const double r0[2], const double r1[2], double width,
                    int falloff) {
  double line_len2 = 0, temp = 0, v[2];
  for (int d = 0; d < 2; d++) line_len2 += (r1[d] - r0[d]) * (r1[d] - r0[d]);
  for (int d = 0; d < 2; d++) temp += (r[d] - r0[d]) * (r1[d] - r0[d]);
  for (int d = 0; d < 2; d++) {
    if (temp <= 0.0) v[d] = r[d] - r0[d];
    else if (temp >= line_len2) v[d] = r[d] - r1[d];
    else v[d] = r[d] - (r0[d] + temp / line_len2 * (r1[d] - r0[d]));
  }
  double dist = norm2v(v, 2);
  switch (falloff) {
    case 1: {
      double q = dist / width;
      if (q > std::log(0.5 * 1.7976931348623157e308)) return 0;
      return 2 / (1 + std::exp(q));
    }
    case 2: {
      double q = dist / width;
      return std::exp(-(q * q));
    }
    case 3: {
      if (dist < width) return 1;
      if (dist < 2 * width) {
        double q = dist / width - 1;
        return (1 - (3 * (q * q) - 2 * (q * q * q)));
      }
      return 0.0;
    }
    case 4: return dist < width ? 1.0 : 0.0;
    default: return 0;
  }
}

// FI_adaptive_r / LT_lin_interp_list, fosito/m_find_index.f90:56-67 and
// fosito/m_lookup_table.f90:200-221
double interp_pairs(const double *xl, const double *yl, int n, double x) {
  if (x <= xl[0]) return yl[0];
  if (x >= xl[n - 1]) return yl[n - 1];
  int lo = 1, hi = n;
  while (lo < hi) {
    int mid = lo + (hi - lo) / 2;
    if (x <= xl[mid - 1]) hi = mid;
    else lo = mid + 1;
  }
  double w = (x - xl[lo - 2]) / (xl[lo - 1] - xl[lo - 2]);
  return (1 - w) * yl[lo - 2] + w * yl[lo - 1];
}

// Photon absorption table, src/m_photons.f90:25-140. The absorption
// function is the distance density of PH_absfunc_air (:122-140) with
// coefficients c0 < c1 (per unit pressure) at pressure p.
struct PhAbs {
  double c0, c1, p;
  double f(double dist) const {
    const double eps = 2.220446049250313e-16;
    const double r = p * dist;
    if (r * (c0 + c1) < eps) return (c1 - c0 + 0.5 * (c0 * c0 - c1 * c1) * r) * p / std::log(c1 / c0);
    if (r * c0 > -std::log(eps)) return eps;
    return (std::exp(-c0 * r) - std::exp(-c1 * r)) / (dist * std::log(c1 / c0));
  }
  // rk4_drdF, :95-117
  double drdF(double r, double dF) const {
    const double one_sixth = 1 / 6.0;
    double d = 1 / f(r);
    double sum = d;
    d = 1 / f(r + 0.5 * dF * d);
    sum = sum + 2 * d;
    d = 1 / f(r + 0.5 * dF * d);
    sum = sum + 2 * d;
    d = 1 / f(r + dF * d);
    sum = sum + d;
    return one_sixth * sum;
  }
};

}  // namespace

extern "C" int a5t_photon_table(int kind, double a, double b, double max_dist, double *dist_out,
                                double *frac_out, int *n_rows) {
  if (!dist_out || !frac_out || !n_rows) return err(A5G_EINVAL, "null argument");
  if (!(max_dist > 0)) return err(A5G_EINVAL, "max_dist must be > 0");
  // fosito/m_units_constants.f90:44, a single-precision literal times 1.0D-5
  const double torr_to_bar = (double)133.322368f * 1.0e-5;
  PhAbs fn;
  if (kind == 0) {
    if (!(a > 0)) return err(A5G_EINVAL, "O2 partial pressure must be > 0");
    fn = PhAbs{3.5 / torr_to_bar, 200 / torr_to_bar, a};
  } else if (kind == 1) {
    if (!(a > 0 && a < b)) return err(A5G_EINVAL, "need 0 < shortest < longest absorption length");
    fn = PhAbs{1 / b, 1 / a, 1.0};
  } else {
    return err(A5G_EINVAL, "photon table kind must be 0 or 1");
  }
  const int tbl_size = 500;
  double frac_guess = 1.0;
  for (int it = 0; it < 5; it++) {
    const double dF = frac_guess / (tbl_size - 1);
    double r = 0, F = 0;
    for (long guard = 0;; guard++) {
      r = r + dF * fn.drdF(r, dF);
      F = F + dF;
      if (r > max_dist) break;
      if (guard > 100000000L) return err(A5G_EINVAL, "photon table integration does not reach max_dist");
    }
    frac_guess = F;
  }
  std::vector<double> fsum(2 * tbl_size), dist(2 * tbl_size);
  const double dF = frac_guess / (tbl_size - 1);
  fsum[0] = dist[0] = 0;
  int used = 2 * tbl_size;  // entries 0..used-1 are the table's input pairs
  for (int k = 1; k < 2 * tbl_size; k++) {
    const double d = fn.drdF(dist[k - 1], dF);
    fsum[k] = fsum[k - 1] + dF;
    dist[k] = dist[k - 1] + dF * d;
    if (dist[k] > max_dist) {
      used = k;
      break;
    }
  }
  if (used + 1 > tbl_size + 10) return err(A5G_EINVAL, "photon table: integration accuracy fail");
  const double norm = fsum[used - 1];
  for (int k = 0; k < used; k++) fsum[k] = fsum[k] / norm;
  // LT_create(0, 1, tbl_size, 1) + LT_set_col (fosito/m_lookup_table.f90:46-72)
  const double inv_dx = (tbl_size - 1) / (1.0 - 0.0);
  const double dx = 1 / inv_dx;
  for (int ix = 1; ix <= tbl_size; ix++)
    dist_out[ix - 1] = interp_pairs(fsum.data(), dist.data(), used, 0.0 + (ix - 1) * dx);
  *frac_out = norm;
  *n_rows = tbl_size;
  return A5G_OK;
}

struct a5s_sim {
  a5s_config cfg{};
  std::vector<double> td_x[4], td_y[4];
  a5t_tree *tree = nullptr;
  a5g_ctx *ctx = nullptr;
  double time = 0;
  std::vector<double> table;
  double tbl_xmin = 0, tbl_inv_dx = 0;
  int tbl_rows = 0;
  std::vector<int> meta;
  std::vector<double> geom;

  int upload_tree() {
    int n = t_n();
    meta.assign(16 * (tree->max_id + 1), 0);
    geom.assign(4 * (tree->max_id + 1), 0.0);
    std::vector<int> counts(3 * (tree->max_lvl - tree->min_lvl + 1));
    std::vector<int> ids(std::max(n, 1));
    a5t_export(tree, meta.data(), geom.data(), counts.data(), ids.data());
    return a5g_upload_tree(ctx, tree->max_id, tree->min_lvl, tree->max_lvl, meta.data(),
                           geom.data(), counts.data(), ids.data());
  }
  int t_n() { return a5t_n_level_ids(tree); }

  // set_init_cond + set_box_eps on every box (src/streamer_2d.f90:218-266)
  int init_cond_all() {
    const int S = (cfg.dev.box_size + 2) * (cfg.dev.box_size + 2);
    const int M = tree->max_id + 1;
    std::vector<double> e(S * M, 0.0), pi(S * M, 0.0), phi(S * M, 0.0), eps(S * M, 0.0);
    const bool cyl = cfg.dev.coord == 1;
    for (int id = 1; id < M; id++) {
      if (!tree->in_use[id]) continue;
      int nc = tree->ncell[id], g = nc + 2;
      double *pe = &e[(size_t)S * id];
      for (int k = 0; k < g * g; k++) pe[k] = cfg.bg_dens;
      for (int j = 0; j <= nc + 1; j++)
        for (int i = 0; i <= nc + 1; i++) {
          double xy[2] = {tree->rmin0[id] + (i - 0.5) * tree->dr[id],
                          tree->rmin1[id] + (j - 0.5) * tree->dr[id]};
          for (int s = 0; s < cfg.n_seeds; s++) {
            double d = cfg.seed_dens[s] * seed_density(xy, cfg.dev.seed_r0[s], cfg.dev.seed_r1[s],
                                                       cfg.dev.seed_width[s], cfg.seed_falloff[s]);
            pe[i + g * j] = pe[i + g * j] + d;
          }
          double rel = (cyl ? xy[0] : xy[1]) / cfg.dev.domain_len_z;
          eps[(size_t)S * id + i + g * j] = rel < 0.25 ? cfg.dev.epsilon_diel : 1.0;
        }
      for (int k = 0; k < g * g; k++) pi[(size_t)S * id + k] = pe[k];
    }
    int r;
    if ((r = a5g_upload_cc(ctx, 0, e.data()))) return r;
    if ((r = a5g_upload_cc(ctx, 1, pi.data()))) return r;
    if ((r = a5g_upload_cc(ctx, 4, phi.data()))) return r;
    return a5g_upload_cc(ctx, 8, eps.data());
  }

  int regrid(int *n_add, int *n_rm) {
    std::vector<int> flags(tree->max_id + 1);
    int r = a5g_ref_flags(ctx, time, flags.data());
    if (r) return r;
    if ((r = a5t_adjust_refinement(tree, flags.data(), n_add, n_rm))) return r;
    if (*n_add > 0 || *n_rm > 0) return upload_tree();
    return A5G_OK;
  }
};

extern "C" {

int a5s_create(const a5s_config *cfg, a5s_sim **out) {
  if (!cfg || !out) return err(A5G_EINVAL, "null argument");
  *out = nullptr;
  if (cfg->n_base[0] < 1 || cfg->n_base[1] < 1) return err(A5G_EINVAL, "n_base must be >= 1");
  if (cfg->n_seeds < 0 || cfg->n_seeds > 8) return err(A5G_EINVAL, "n_seeds must be 0..8");
  if (cfg->num_steps_amr < 1) return err(A5G_EINVAL, "num_steps_amr must be >= 1");
  if (cfg->lkptbl_size < 2 || !(cfg->lkptbl_max_fld > 0)) return err(A5G_EINVAL, "bad table size");
  for (int c = 0; c < 4; c++)
    if (cfg->td_n[c] < 1 || !cfg->td_x[c] || !cfg->td_y[c]) return err(A5G_EINVAL, "missing transport column");
  a5s_sim *s = new a5s_sim();
  s->cfg = *cfg;
  for (int c = 0; c < 4; c++) {
    s->td_x[c].assign(cfg->td_x[c], cfg->td_x[c] + cfg->td_n[c]);
    s->td_y[c].assign(cfg->td_y[c], cfg->td_y[c] + cfg->td_n[c]);
    s->cfg.td_x[c] = s->td_x[c].data();
    s->cfg.td_y[c] = s->td_y[c].data();
  }
  // LT_create(0, max_fld, n_rows, 4) + LT_set_col (fosito/m_lookup_table.f90:46-72)
  const int nr = cfg->lkptbl_size;
  s->tbl_rows = nr;
  s->tbl_xmin = 0.0;
  s->tbl_inv_dx = (nr - 1) / (cfg->lkptbl_max_fld - 0.0);
  s->table.assign((size_t)nr * 4, 0.0);
  const double dx = 1 / s->tbl_inv_dx;
  for (int c = 0; c < 4; c++)
    for (int ix = 1; ix <= nr; ix++)
      s->table[(size_t)nr * c + ix - 1] =
          interp_pairs(s->td_x[c].data(), s->td_y[c].data(), cfg->td_n[c], 0.0 + (ix - 1) * dx);
  int r;
  double r0[2] = {0, 0};
  if ((r = a5t_create(cfg->dev.box_size, cfg->dev.lvls_max, cfg->dev.dr_base, r0, cfg->dev.coord,
                      &s->tree))) {
    delete s;
    return r;
  }
  const int nx = cfg->n_base[0], ny = cfg->n_base[1], n = nx * ny;
  std::vector<int> ix(2 * n), nbl(4 * n);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int k = i + nx * j;
      ix[2 * k] = i + 1;
      ix[2 * k + 1] = j + 1;
      nbl[4 * k + 0] = i > 0 ? k : -1;
      nbl[4 * k + 1] = i < nx - 1 ? k + 2 : -1;
      nbl[4 * k + 2] = j > 0 ? k + 1 - nx : -1;
      nbl[4 * k + 3] = j < ny - 1 ? k + 1 + nx : -1;
    }
  if ((r = a5t_set_base(s->tree, n, ix.data(), nbl.data())) ||
      (r = a5g_create(&s->cfg.dev, &s->ctx)) ||
      (r = a5g_set_table(s->ctx, nr, 4, s->tbl_xmin, s->tbl_inv_dx, s->table.data())) ||
      (r = s->upload_tree())) {
    a5s_destroy(s);
    return r;
  }
  if (cfg->dev.photoi_enabled) {
    // src/m_streamer.f90:327-330
    double dist[500], frac = 0;
    int rows = 0;
    if ((r = a5t_photon_table(cfg->photoi_tbl_kind, cfg->photoi_tbl_a, cfg->photoi_tbl_b,
                              cfg->photoi_max_dist, dist, &frac, &rows)) ||
        (r = a5g_set_photon_table(s->ctx, rows, 0.0, (rows - 1) / 1.0, dist, frac))) {
      a5s_destroy(s);
      return r;
    }
  }
  *out = s;
  return A5G_OK;
}

int a5s_destroy(a5s_sim *s) {
  if (!s) return A5G_OK;
  if (s->ctx) a5g_destroy(s->ctx);
  if (s->tree) a5t_destroy(s->tree);
  delete s;
  return A5G_OK;
}

int a5s_init(a5s_sim *s, int *n_iter) {
  if (!s) return err(A5G_EINVAL, "null sim");
  int it = 0, r;
  s->time = 0;
  while (true) {
    it++;
    if ((r = s->init_cond_all())) return r;
    if ((r = a5g_compute_fld(s->ctx, 1))) return r;
    int na = 0, nr = 0;
    if ((r = s->regrid(&na, &nr))) return r;
    if (na == 0 || it > 100) break;
  }
  if (n_iter) *n_iter = it;
  // src/streamer_cyl.f90:68-69
  if (s->cfg.dev.photoi_enabled && (r = a5g_photoionization(s->ctx, 0.0, 0))) return r;
  return a5g_sync(s->ctx);
}

int a5s_set_init_cond(a5s_sim *s) {
  if (!s) return err(A5G_EINVAL, "null sim");
  int r = s->init_cond_all();
  if (r) return r;
  return a5g_sync(s->ctx);
}

// The regrid at the end of a main-loop block (src/streamer_2d.f90:130-141):
// refinement flags, a$D_adjust_refinement, prolongation into new boxes and a
// field solve when the tree changed.
static int regrid_block(a5s_sim *s) {
  int na = 0, nr = 0, r;
  if ((r = s->regrid(&na, &nr))) return r;
  if (na > 0 || nr > 0) {
    int nlev = s->tree->max_lvl - s->tree->min_lvl + 1;
    std::vector<int> counts(nlev), ids(std::max(na, 1));
    a5t_new_boxes(s->tree, counts.data(), ids.data());
    if ((r = a5g_prolong_new(s->ctx, counts.data(), ids.data()))) return r;
    // in FP64 whatever the run's precision: after a prolongation the
    // potential's correction is large and smooth, and the mixed form's FP32
    // correction pass would lose the digits it needs
    if ((r = a5g_compute_fld_fp64(s->ctx, 0))) return r;
  }
  return A5G_OK;
}

static int do_block(a5s_sim *s, double dt, int regrid) {
  int r;
  for (int n = 0; n < s->cfg.num_steps_amr; n++) {
    s->time += dt;
    if ((r = a5g_step(s->ctx, dt))) return r;
  }
  if (!regrid) return A5G_OK;
  return regrid_block(s);
}

int a5s_advance(a5s_sim *s, int regrid, double *dt_used) {
  if (!s) return err(A5G_EINVAL, "null sim");
  double dt = 0;
  int r = a5g_get_max_dt(s->ctx, &dt);
  if (r) return r;
  if (dt_used) *dt_used = dt;
  return do_block(s, dt, regrid);
}

int a5s_run(a5s_sim *s, double t_end, int max_blocks, int *n_blocks) {
  if (!s) return err(A5G_EINVAL, "null sim");
  int nb = 0, r;
  while (nb < max_blocks) {
    double dt = 0;
    if ((r = a5g_get_max_dt(s->ctx, &dt))) return r;
    if (dt < 1e-14) break;  // src/streamer_2d.f90:72-75
    if (s->time > t_end) break;
    if ((r = do_block(s, dt, 1))) return r;
    nb++;
  }
  if (n_blocks) *n_blocks = nb;
  return a5g_sync(s->ctx);
}

// Worker threads that run one job at a time together with the caller: run(f)
// hands f to every worker, runs it on the calling thread too and returns once
// every worker has finished it (jobs share their work through a counter).
class WorkerPool {
 public:
  explicit WorkerPool(int n_threads) {
    for (int t = 1; t < n_threads; t++) th_.emplace_back([this] { loop(); });
  }
  ~WorkerPool() {
    {
      std::lock_guard<std::mutex> l(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  void run(const std::function<void()> &f) {
    {
      std::lock_guard<std::mutex> l(mu_);
      job_ = f;
      gen_++;
      pending_ = (int)th_.size();
    }
    cv_.notify_all();
    f();
    std::unique_lock<std::mutex> l(mu_);
    done_.wait(l, [&] { return pending_ == 0; });
  }

 private:
  void loop() {
    long seen = 0;
    for (;;) {
      std::function<void()> j;
      {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        j = job_;
      }
      j();
      std::lock_guard<std::mutex> l(mu_);
      if (--pending_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::function<void()> job_;
  long gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

// Regrid the given members on the pool's threads (trees and contexts are
// independent; each context works on its own stream), and wait for them.
static int regrid_members(a5s_sim **sims, const std::vector<int> &todo, WorkerPool &pool) {
  std::atomic<size_t> next{0};
  std::vector<int> rc(todo.size(), A5G_OK);
  std::vector<std::string> msg(todo.size());
  pool.run([&]() {
    size_t i;
    while ((i = next++) < todo.size()) {
      rc[i] = regrid_block(sims[todo[i]]);
      if (!rc[i]) rc[i] = a5g_sync(sims[todo[i]]->ctx);
      if (rc[i]) msg[i] = a5g_last_error();
    }
  });
  for (size_t i = 0; i < todo.size(); i++)
    if (rc[i]) return err(rc[i], "regrid of batch member " + std::to_string(todo[i]) + ": " + msg[i]);
  return A5G_OK;
}

int a5s_batch_run(a5s_sim **sims, int n, const double *t_end, int use_graph, int n_threads,
                  int n_groups, int max_blocks, int *n_blocks, double *gpu_ms, double *host_ms,
                  double *cell_updates) {
  if (!sims || !t_end || n < 1) return err(A5G_EINVAL, "bad batch");
  if (n_groups < 1) return err(A5G_EINVAL, "n_groups must be >= 1");
  for (int k = 0; k < n; k++) {
    if (!sims[k]) return err(A5G_EINVAL, "null sim in batch");
    if (sims[k]->cfg.num_steps_amr != sims[0]->cfg.num_steps_amr)
      return err(A5G_EINVAL, "batch members need the same num_steps_amr");
  }
  // members are dealt to groups in turn; each group is a batch of its own
  // with its own stream, so that one group's block runs on the device while
  // the host regrids another group's runs
  const int G = std::min(n_groups, n);
  struct Group {
    std::vector<int> mem;
    a5g_batch *b = nullptr;
    std::vector<double> dt, tm;
    std::vector<int> act;
    std::vector<long long> leaves;
    int blocks = 0;
    bool done = false;
  };
  std::vector<Group> g(G);
  for (int k = 0; k < n; k++) g[k % G].mem.push_back(k);
  const int steps = sims[0]->cfg.num_steps_amr;
  int r = A5G_OK;
  for (auto &q : g) {
    const int m = (int)q.mem.size();
    std::vector<a5g_ctx *> ctxs(m);
    std::vector<double> te(m);
    q.dt.assign(m, 0);
    q.tm.assign(m, 0);
    q.act.assign(m, 0);
    q.leaves.assign(m, 0);
    for (int i = 0; i < m; i++) {
      ctxs[i] = sims[q.mem[i]]->ctx;
      q.tm[i] = sims[q.mem[i]]->time;
      te[i] = t_end[q.mem[i]];
    }
    if ((r = a5g_batch_create(ctxs.data(), m, &q.b)) || (r = a5g_batch_begin(q.b, q.tm.data(), te.data())))
      break;
  }
  double g_ms = 0, h_ms = 0, cu = 0;
  WorkerPool pool(std::max(1, std::min(n_threads, n)));
  auto launch = [&](Group &q) {
    for (size_t i = 0; i < q.mem.size(); i++) a5g_n_leaf_cells(sims[q.mem[i]]->ctx, &q.leaves[i]);
    return a5g_batch_launch(q.b, steps, use_graph);
  };
  if (!r)
    for (auto &q : g)
      if ((r = launch(q))) break;
  bool any = true;
  while (!r && any) {
    any = false;
    for (auto &q : g) {
      if (q.done) continue;
      float ms = 0;
      if ((r = a5g_batch_finish(q.b, q.dt.data(), q.tm.data(), q.act.data(), &ms))) break;
      g_ms += ms;
      std::vector<int> todo;
      for (size_t i = 0; i < q.mem.size(); i++) {
        sims[q.mem[i]]->time = q.tm[i];
        if (q.act[i]) {
          todo.push_back(q.mem[i]);
          cu += (double)q.leaves[i] * steps;
        }
      }
      if (todo.empty()) {
        q.done = true;
        continue;
      }
      q.blocks++;
      const auto t0 = std::chrono::steady_clock::now();
      r = regrid_members(sims, todo, pool);
      h_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (r) break;
      if (q.blocks >= max_blocks) {
        q.done = true;
        continue;
      }
      if ((r = launch(q))) break;
      any = true;
    }
  }
  int nb = 0;
  for (auto &q : g) {
    if (q.b) {
      if (r) a5g_batch_finish(q.b, nullptr, nullptr, nullptr, nullptr);  // drain before destroying
      a5g_batch_destroy(q.b);
    }
    nb = std::max(nb, q.blocks);
  }
  if (n_blocks) *n_blocks = nb;
  if (gpu_ms) *gpu_ms = g_ms;
  if (host_ms) *host_ms = h_ms;
  if (cell_updates) *cell_updates = cu;
  return r;
}

int a5s_time(a5s_sim *s, double *t) {
  if (!s || !t) return err(A5G_EINVAL, "null argument");
  *t = s->time;
  return A5G_OK;
}
int a5s_ctx(a5s_sim *s, a5g_ctx **c) {
  if (!s || !c) return err(A5G_EINVAL, "null argument");
  *c = s->ctx;
  return A5G_OK;
}
int a5s_tree(a5s_sim *s, a5t_tree **t) {
  if (!s || !t) return err(A5G_EINVAL, "null argument");
  *t = s->tree;
  return A5G_OK;
}
int a5s_table(a5s_sim *s, double *rows_cols, double *x_min, double *inv_dx, int *n_rows) {
  if (!s) return err(A5G_EINVAL, "null sim");
  if (rows_cols) std::memcpy(rows_cols, s->table.data(), s->table.size() * sizeof(double));
  if (x_min) *x_min = s->tbl_xmin;
  if (inv_dx) *inv_dx = s->tbl_inv_dx;
  if (n_rows) *n_rows = s->tbl_rows;
  return A5G_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Checkpoint / resume. The reference persists nothing but output snapshots;
// a checkpoint here is the whole state a run's next block depends on: time,
// generator state, the tree (per-id arrays and the level lists exactly as
// a$D_adjust_refinement left them, including the lists of level lvls_max
// that it never rebuilds), and every cell and face variable of ids
// 0..max_id with ghost cells. Layout (native byte order, no padding):
//   u32 magic 'A5CK', u32 version, u64 configuration fingerprint,
//   i32 box_size, coord, lvls_max, min_lvl, max_lvl, max_id, n_lists,
//       cell slot, face slot, photoionization, f64 time, i32 rng[4],
//   per id: i32 in_use, lvl, ix0, ix1, parent, n_cell, ch[4], nb[4];
//           f64 dr, r_min0, r_min1,
//   per list level: i32 n_ids, n_leaves, n_parents, then the three lists,
//   f64 cc[var][id][cell slot], f64 fc[dim][var][id][face slot].
namespace {

constexpr uint32_t kCkMagic = 0x4B433541u;  // "A5CK"
constexpr uint32_t kCkVersion = 1;

struct CkWriter {
  unsigned char *p;
  size_t cap, n = 0;
  void put(const void *src, size_t bytes) {
    if (p && n + bytes <= cap) std::memcpy(p + n, src, bytes);
    n += bytes;
  }
  template <class T> void v(T x) { put(&x, sizeof(T)); }
};

struct CkReader {
  const unsigned char *p;
  size_t len, n = 0;
  bool ok = true;
  void get(void *dst, size_t bytes) {
    if (!ok || n + bytes > len) {
      ok = false;
      return;
    }
    std::memcpy(dst, p + n, bytes);
    n += bytes;
  }
  template <class T> T v() {
    T x{};
    get(&x, sizeof(T));
    return x;
  }
};

// FNV-1a over the settings that change a run's arithmetic: a checkpoint is
// only resumed by a run of the same configuration.
uint64_t ck_fingerprint(const a5s_sim *s) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](const void *q, size_t bytes) {
    const unsigned char *b = static_cast<const unsigned char *>(q);
    for (size_t i = 0; i < bytes; i++) h = (h ^ b[i]) * 1099511628211ull;
  };
  const a5g_params &d = s->cfg.dev;
  const int ints[] = {d.box_size, d.coord, d.lvls_max, d.use_drt, d.n_cycle_base, d.n_seeds,
                      d.photoi_enabled, d.photoi_num_photons, d.photoi_team, d.uniform_lvl,
                      s->cfg.n_base[0], s->cfg.n_base[1], s->cfg.num_steps_amr};
  const double dbl[] = {d.dr_base, d.domain_len_z, d.applied_fld, d.epsilon_diel, d.dt_max,
                        d.ref_init_time, d.crv_refine, d.photoi_coeff, d.photoi_fac_dx};
  mix(ints, sizeof(ints));
  mix(dbl, sizeof(dbl));
  mix(d.seed_r0, sizeof(d.seed_r0));
  mix(d.seed_r1, sizeof(d.seed_r1));
  mix(d.seed_width, sizeof(d.seed_width));
  mix(s->table.data(), s->table.size() * sizeof(double));
  return h;
}

// The invariants a device upload relies on: every box in use is listed
// exactly once, on its own level, among the level lists of min_lvl..max_lvl
// (lists above max_lvl are kept as a$D_adjust_refinement leaves them);
// leaves and parents are boxes of their level; parents, children and
// neighbours of a box in use are in use on the adjacent / same level.
bool tree_consistent(const a5t_tree &t) {
  const int M = t.max_id + 1;
  if (t.max_lvl < t.min_lvl || t.max_lvl - t.min_lvl >= (int)t.ids.size()) return false;
  std::vector<int> seen(M, 0);
  auto ok_id = [&](int id, int lvl) { return id >= 1 && id < M && t.in_use[id] && t.lvl[id] == lvl; };
  for (int k = 0; k <= t.max_lvl - t.min_lvl; k++) {
    const int lvl = t.min_lvl + k;
    for (int id : t.ids[k])
      if (!ok_id(id, lvl) || seen[id]++) return false;
    for (int id : t.leaves[k])
      if (!ok_id(id, lvl)) return false;
    for (int id : t.parents[k])
      if (!ok_id(id, lvl)) return false;
  }
  for (int id = 1; id < M; id++) {
    if (!t.in_use[id]) continue;
    const int l = t.lvl[id], p = t.parent[id];
    if (seen[id] != 1 || l > t.max_lvl) return false;
    if (l == t.min_lvl ? p != 0 : !ok_id(p, l - 1)) return false;
    for (int q = 0; q < 4; q++) {
      const int c = t.ch[id][q], n = t.nb[id][q];
      if (c > 0 && (!ok_id(c, l + 1) || t.parent[c] != id)) return false;
      if (n > 0 && !ok_id(n, l)) return false;
    }
  }
  return true;
}

int ck_write(a5s_sim *s, CkWriter &w) {
  const a5t_tree *t = s->tree;
  const int nc = t->nc, cslot = (nc + 2) * (nc + 2), fslot = (nc + 1) * nc;
  const int nlists = (int)t->ids.size(), M = t->max_id + 1;
  int rng[4] = {0, 0, 0, 0};
  int r;
  if (w.p && s->cfg.dev.photoi_enabled && (r = a5g_get_rng(s->ctx, rng))) return r;
  w.v(kCkMagic);
  w.v(kCkVersion);
  w.v(ck_fingerprint(s));
  for (int x : {nc, t->coord, t->lvls_max, t->min_lvl, t->max_lvl, t->max_id, nlists, cslot, fslot,
                s->cfg.dev.photoi_enabled})
    w.v(x);
  w.v(s->time);
  w.put(rng, sizeof(rng));
  for (int id = 0; id < M; id++) {
    for (int x : {(int)t->in_use[id], t->lvl[id], t->ix0[id], t->ix1[id], t->parent[id], t->ncell[id]})
      w.v(x);
    w.put(t->ch[id].data(), 4 * sizeof(int));
    w.put(t->nb[id].data(), 4 * sizeof(int));
    w.v(t->dr[id]);
    w.v(t->rmin0[id]);
    w.v(t->rmin1[id]);
  }
  for (int k = 0; k < nlists; k++) {
    w.v((int)t->ids[k].size());
    w.v((int)t->leaves[k].size());
    w.v((int)t->parents[k].size());
    w.put(t->ids[k].data(), t->ids[k].size() * sizeof(int));
    w.put(t->leaves[k].data(), t->leaves[k].size() * sizeof(int));
    w.put(t->parents[k].data(), t->parents[k].size() * sizeof(int));
  }
  std::vector<double> buf;
  for (int iv = 0; iv < A5G_N_VAR_CELL; iv++) {
    if (w.p) {
      buf.resize((size_t)M * cslot);
      if ((r = a5g_download_cc(s->ctx, iv, buf.data()))) return r;
    }
    w.put(buf.data(), (size_t)M * cslot * sizeof(double));
  }
  for (int dim = 0; dim < 2; dim++)
    for (int f = 0; f < A5G_N_VAR_FACE; f++) {
      if (w.p) {
        buf.resize((size_t)M * fslot);
        if ((r = a5g_download_fc(s->ctx, dim, f, buf.data()))) return r;
      }
      w.put(buf.data(), (size_t)M * fslot * sizeof(double));
    }
  return A5G_OK;
}

}  // namespace

extern "C" {

int a5t_check(a5t_tree *t) {
  if (!t) return err(A5G_EINVAL, "null tree");
  if (t->max_id == 0) return A5G_OK;
  return tree_consistent(*t) ? A5G_OK : err(A5G_EINVAL, "tree inconsistent");
}

int a5s_checkpoint_size(a5s_sim *s, size_t *bytes) {
  if (!s || !bytes) return err(A5G_EINVAL, "null argument");
  CkWriter w{nullptr, 0};
  int r = ck_write(s, w);
  if (r) return r;
  *bytes = w.n;
  return A5G_OK;
}

int a5s_checkpoint_save(a5s_sim *s, void *buf, size_t cap, size_t *written) {
  if (!s || !buf) return err(A5G_EINVAL, "null argument");
  size_t need = 0;
  int r = a5s_checkpoint_size(s, &need);
  if (r) return r;
  if (cap < need) return err(A5G_EINVAL, "checkpoint buffer too small (a5s_checkpoint_size gives the size)");
  CkWriter w{static_cast<unsigned char *>(buf), cap};
  if ((r = ck_write(s, w))) return r;
  if (written) *written = w.n;
  return A5G_OK;
}

int a5s_checkpoint_load(a5s_sim *s, const void *buf, size_t len) {
  if (!s || !buf) return err(A5G_EINVAL, "null argument");
  CkReader rd{static_cast<const unsigned char *>(buf), len};
  if (rd.v<uint32_t>() != kCkMagic || !rd.ok) return err(A5G_EINVAL, "not a checkpoint");
  if (rd.v<uint32_t>() != kCkVersion) return err(A5G_EINVAL, "checkpoint version not supported");
  if (rd.v<uint64_t>() != ck_fingerprint(s))
    return err(A5G_EINVAL, "checkpoint was written by a run of another configuration");
  int hdr[10];
  for (int &x : hdr) x = rd.v<int>();
  a5t_tree *cur = s->tree;
  const int nc = hdr[0], min_lvl = hdr[3], max_lvl = hdr[4], max_id = hdr[5], nlists = hdr[6];
  if (!rd.ok || nc != cur->nc || hdr[1] != cur->coord || hdr[2] != cur->lvls_max ||
      min_lvl != cur->min_lvl || nlists != (int)cur->ids.size() || hdr[7] != (nc + 2) * (nc + 2) ||
      hdr[8] != (nc + 1) * nc || hdr[9] != s->cfg.dev.photoi_enabled)
    return err(A5G_EINVAL, "checkpoint header does not match this run");
  if (max_id < 1 || max_lvl < 1 || max_lvl > cur->lvls_max)
    return err(A5G_EINVAL, "checkpoint header out of range");
  const int M = max_id + 1, cslot = hdr[7], fslot = hdr[8];
  const size_t body = (size_t)M * (14 * sizeof(int) + 3 * sizeof(double)) +
                      (size_t)M * (A5G_N_VAR_CELL * cslot + 2 * A5G_N_VAR_FACE * fslot) * sizeof(double);
  if (body > len) return err(A5G_EINVAL, "checkpoint truncated");
  const double time = rd.v<double>();
  int rng[4];
  rd.get(rng, sizeof(rng));
  // the tree is built aside and swapped in only once it has been read whole
  a5t_tree nt;
  nt.nc = cur->nc;
  nt.lvls_max = cur->lvls_max;
  nt.dr_base = cur->dr_base;
  nt.r_base[0] = cur->r_base[0];
  nt.r_base[1] = cur->r_base[1];
  nt.coord = cur->coord;
  nt.min_lvl = min_lvl;
  nt.max_lvl = max_lvl;
  nt.grow_ids(max_id);
  for (int id = 0; id < M; id++) {
    nt.in_use[id] = (char)rd.v<int>();
    nt.lvl[id] = rd.v<int>();
    nt.ix0[id] = rd.v<int>();
    nt.ix1[id] = rd.v<int>();
    nt.parent[id] = rd.v<int>();
    nt.ncell[id] = rd.v<int>();
    rd.get(nt.ch[id].data(), 4 * sizeof(int));
    rd.get(nt.nb[id].data(), 4 * sizeof(int));
    nt.dr[id] = rd.v<double>();
    nt.rmin0[id] = rd.v<double>();
    nt.rmin1[id] = rd.v<double>();
  }
  nt.ids.assign(nlists, {});
  nt.leaves.assign(nlists, {});
  nt.parents.assign(nlists, {});
  nt.added.assign(nlists, {});
  auto in_range = [&](const std::vector<int> &v) {
    for (int id : v)
      if (id < 1 || id > max_id) return false;
    return true;
  };
  for (int k = 0; k < nlists && rd.ok; k++) {
    const int a = rd.v<int>(), b = rd.v<int>(), c = rd.v<int>();
    if (!rd.ok || a < 0 || b < 0 || c < 0 || a > M || b > M || c > M)
      return err(A5G_EINVAL, "checkpoint level list out of range");
    nt.ids[k].resize(a);
    nt.leaves[k].resize(b);
    nt.parents[k].resize(c);
    rd.get(nt.ids[k].data(), a * sizeof(int));
    rd.get(nt.leaves[k].data(), b * sizeof(int));
    rd.get(nt.parents[k].data(), c * sizeof(int));
    if (!in_range(nt.ids[k]) || !in_range(nt.leaves[k]) || !in_range(nt.parents[k]))
      return err(A5G_EINVAL, "checkpoint level list names an id out of range");
  }
  for (int id = 1; id < M && rd.ok; id++) {
    for (int q = 0; q < 4; q++)
      if (nt.ch[id][q] < 0 || nt.ch[id][q] > max_id || nt.nb[id][q] > max_id)
        return err(A5G_EINVAL, "checkpoint box links out of range");
    if (nt.parent[id] < 0 || nt.parent[id] > max_id) return err(A5G_EINVAL, "checkpoint box record out of range");
    if (!nt.in_use[id]) continue;
    const int l = nt.lvl[id];
    if (l < min_lvl || l > nt.lvls_max || nt.ncell[id] != (l >= 1 ? nc : nc >> (1 - l)))
      return err(A5G_EINVAL, "checkpoint box record out of range");
  }
  if (!tree_consistent(nt)) return err(A5G_EINVAL, "checkpoint tree inconsistent");
  std::vector<double> cc((size_t)A5G_N_VAR_CELL * M * cslot), fc((size_t)2 * A5G_N_VAR_FACE * M * fslot);
  rd.get(cc.data(), cc.size() * sizeof(double));
  rd.get(fc.data(), fc.size() * sizeof(double));
  if (!rd.ok) return err(A5G_EINVAL, "checkpoint truncated");
  if (rd.n != len) return err(A5G_EINVAL, "checkpoint has trailing bytes");
  *cur = std::move(nt);
  int r;
  if ((r = s->upload_tree())) return r;
  for (int iv = 0; iv < A5G_N_VAR_CELL; iv++)
    if ((r = a5g_upload_cc(s->ctx, iv, cc.data() + (size_t)iv * M * cslot))) return r;
  for (int dim = 0; dim < 2; dim++)
    for (int f = 0; f < A5G_N_VAR_FACE; f++)
      if ((r = a5g_upload_fc(s->ctx, dim, f, fc.data() + ((size_t)dim * A5G_N_VAR_FACE + f) * M * fslot)))
        return r;
  if (s->cfg.dev.photoi_enabled && (r = a5g_set_rng(s->ctx, rng))) return r;
  s->time = time;
  return a5g_sync(s->ctx);
}

}  // extern "C"
