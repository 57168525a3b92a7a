// Phases, operations and kernels of the device path, included by a5g.cu
// once per execution form, inside namespace blk (A5G_GRID 0: a run on one
// thread block) and namespace grd (A5G_GRID 1: a run on a group of blocks,
// and runs with level-set boxes). Everything a phase needs from the group
// goes through TID(), NTH(), LEAD(), PSYNC() and the one-block sections
// below, which the block form reduces to threadIdx.x, NTHR and
// __syncthreads at compile time.
#ifndef A5G_GRID
#error "a5g_phases.cuh is included by a5g.cu with A5G_GRID set"
#endif

constexpr bool kGrid = A5G_GRID != 0;

#if A5G_GRID
__device__ __forceinline__ int TID() { return s_grp.tid0 + (int)threadIdx.x; }
__device__ __forceinline__ int NTH() { return s_grp.nth; }
// the one thread of the group that writes a run's scalars
__device__ __forceinline__ bool LEAD() { return s_grp.tid0 == 0 && threadIdx.x == 0; }
#else
__device__ __forceinline__ int TID() { return (int)threadIdx.x; }
__device__ __forceinline__ int NTH() { return NTHR; }
__device__ __forceinline__ bool LEAD() { return threadIdx.x == 0; }
#endif

// Barrier of the run's block group. One thread per block arrives on the
// group's counter; the last arrival resets it and advances the generation;
// the others wait for the generation to change, at most s_grp.budget SM
// cycles, after which the wait records A5G_TIMEOUT, raises the abort flag
// (every later barrier of the launch then returns at once) and returns.
// The fences order each block's writes before its arrival and the waiting
// block's later reads after the release (gpu-scope acquire also drops stale
// L1 lines), as a grid-wide barrier requires.
__device__ __noinline__ void grid_sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned *bar = s_grp.bar;
    volatile unsigned *vgen = bar + 1, *vabort = bar + 2;
    if (*vabort == 0u) {
      const unsigned gen = *vgen;
      __threadfence();
      const unsigned prev = atomicAdd(bar, 1u);
      if (prev == (unsigned)s_grp.size - 1u) {
        atomicExch(bar, 0u);
        __threadfence();
        atomicAdd(bar + 1, 1u);
      } else {
        const long long budget = s_grp.budget;
        const long long t0 = clock64();
        while (*vgen == gen && *vabort == 0u) {
          if (clock64() - t0 >= budget) {
            atomicExch(bar + 2, 1u);
            atomicExch(s_grp.status, (int)A5G_TIMEOUT);
            break;
          }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
}

// Barrier between two phases of a run.
__device__ __forceinline__ void PSYNC() {
  if (kGrid && s_grp.size > 1) grid_sync();
  else __syncthreads();
}

template <class F>
__device__ __forceinline__ void box_loop(const int *list, int n, F &&f) {
  const int g = TID() / GT, t = threadIdx.x % GT, ng = NTH() / GT;
  for (int b = g; b < n; b += ng) f(list[b], t);
}

// afivo/src/m_aX_utils.f90:227-239 (a$D_get_child_offset); nb < 0: absent
__device__ __forceinline__ void child_offset(const BoxMeta &m, int nb, int &o0, int &o1) {
  if (m.lvl > 1) {
    o0 = ((m.ix0 - 1) & 1) * (m.nc >> 1);
    o1 = ((m.ix1 - 1) & 1) * (m.nc >> 1);
    if (nb >= 0) { o0 -= c_nb_dix[nb][0] * m.nc; o1 -= c_nb_dix[nb][1] * m.nc; }
  } else {
    o0 = 0;
    o1 = 0;
    if (nb >= 0) {
      o0 -= c_nb_dix[nb][0] * (m.nc >> 1);
      o1 -= c_nb_dix[nb][1] * (m.nc >> 1);
    }
  }
}

// gfortran's inline NORM2 for two elements (scaled sum of squares). T is
// double on the plain path and float for the FP32 transport of the mixed form.
template <class T>
__device__ __forceinline__ T norm2_2(T x0, T x1) {
  T scale = T(0), ssq = T(1);
  T xs[2] = {x0, x1};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    if (xs[k] != T(0)) {
      T ax = fabs(xs[k]);
      if (scale < ax) {
        T v = scale / ax;
        ssq = T(1) + ssq * v * v;
        scale = ax;
      } else {
        T v = ax / scale;
        ssq += v * v;
      }
    }
  }
  return scale * sqrt(ssq);
}

// fosito/m_lookup_table.f90:107-125 (get_loc) and 154-161 (LT_get_col_at_loc)
// (T = float: the same lookup on the FP32 copy of the table.)
template <class T> struct Loc { int ix; T fr; };
template <class T>
__device__ __forceinline__ Loc<T> get_loc(const RunDev &R, T x) {
  T frac = (x - T(R.tbl_xmin)) * T(R.tbl_inv_dx);
  Loc<T> l;
  if (frac < T(2.0e9) && frac > T(-2.0e9)) {
    l.ix = (int)ceil(frac);
    l.fr = T(l.ix) - frac;
  } else {
    l.ix = frac > T(0) ? R.tbl_rows : 0;
    l.fr = T(0);
  }
  if (l.ix < 1) { l.ix = 1; l.fr = T(1); }
  else if (l.ix >= R.tbl_rows) { l.ix = R.tbl_rows - 1; l.fr = T(0); }
  return l;
}
template <class T> __device__ __forceinline__ const T *table_of(const RunDev &R);
template <> __device__ __forceinline__ const double *table_of<double>(const RunDev &R) { return R.tbl; }
template <> __device__ __forceinline__ const float *table_of<float>(const RunDev &R) { return R.tbl32; }
template <class T>
__device__ __forceinline__ T col_at(const RunDev &R, int c, const Loc<T> &l) {
  const T *tb = table_of<T>(R) + (size_t)R.tbl_rows * c;
  return l.fr * __ldg(tb + l.ix - 1) + (T(1) - l.fr) * __ldg(tb + l.ix);
}

// src/m_streamer.f90:339-362 (koren_mlim)
template <class T>
__device__ __forceinline__ T koren_mlim(T a, T b) {
  const T sixth = T(1 / 6.0);
  T aa = a * a, ab = a * b;
  if (ab <= T(0)) return T(0);
  if (aa <= T(0.25) * ab) return a;
  if (aa <= T(2.5) * ab) return sixth * (b + T(2) * a);
  return b;
}

// Scale of the densities inside the FP32 fluxes: an exact power of two that
// keeps squares of density differences (up to ~1e21 m^-3) inside the float
// range. The fluxes are homogeneous of degree one in the density, so the
// scaled flux times 1/scale is the flux. 1 on the FP64 path.
template <class T> __device__ __forceinline__ T dens_scale() { return T(1); }
template <> __device__ __forceinline__ float dens_scale<float>() { return 0x1p-40f; }

// ---------------------------------------------------------------------------
// Ghost cells (afivo/src/m_aX_gc.f90). Value of side ghost (nb, k), k = 1..nc,
// of box id for variable iv.
__device__ double ghost_value(const RunDev &R, const BoxMeta &m, int id, int iv, int nb,
                              int k, int kind) {
  const int nc = m.nc, ncg = nc + 2;
  const double *own = CC(R, iv, id);
  const int nb_id = m.nb[nb];
  const int dim = nb >> 1;
  const bool low = (nb & 1) == 0;
  if (nb_id > 0) {
    // sides_from_nb, m_aX_gc.f90:368-402
    const double *nbc = CC(R, iv, nb_id);
    if (dim == 0) return nbc[(low ? nc : 1) + ncg * k];
    return nbc[k + ncg * (low ? nc : 1)];
  }
  if (nb_id == 0) {
    if (kind == GC_PHI) {
      // mg$D_sides_rb (m_aX_mg.f90:261-301) after a$D_gc_prolong0 (m_aX_gc.f90:71-86)
      int o0, o1;
      child_offset(m, -1, o0, o1);
      const BoxMeta &pm = R.meta[m.parent];
      const double *par = CC(R, iv, m.parent);
      const int pncg = pm.nc + 2;
      const int ix = low ? 1 : nc, di = low ? 1 : -1;
      const int dk = -1 + 2 * (k & 1);
      if (dim == 0) {
        int ig = ix - di;
        double g = par[(o0 + ((ig + 1) >> 1)) + pncg * (o1 + ((k + 1) >> 1))];
        return 0.5 * g + own[ix + ncg * k] -
               0.25 * (own[(ix + di) + ncg * k] + own[ix + ncg * (k + dk)]);
      } else {
        int jg = ix - di;
        double g = par[(o0 + ((k + 1) >> 1)) + pncg * (o1 + ((jg + 1) >> 1))];
        return 0.5 * g + own[k + ncg * ix] -
               0.25 * (own[(k + dk) + ncg * ix] + own[k + ncg * (ix + di)]);
      }
    }
    // a$D_gc_interp / a$D_gc_interp_lim, m_aX_gc.f90:90-295
    const double sixth = 1 / 6.0, third = 1 / 3.0;
    int o0, o1;
    child_offset(m, nb, o0, o1);
    const int pn = R.meta[m.parent].nb[nb];
    const double *pc = CC(R, iv, pn);
    const int ix_f = low ? 1 : nc, ix_c = low ? nc : 1;
    double c1, c2, f;
    if (dim == 0) {
      int j_c1 = o1 + ((k + 1) >> 1);
      int j_c2 = j_c1 + 1 - 2 * (k & 1);
      c1 = pc[ix_c + ncg * j_c1];
      c2 = pc[ix_c + ncg * j_c2];
      f = own[ix_f + ncg * k];
    } else {
      int i_c1 = o0 + ((k + 1) >> 1);
      int i_c2 = i_c1 + 1 - 2 * (k & 1);
      c1 = pc[i_c1 + ncg * ix_c];
      c2 = pc[i_c2 + ncg * ix_c];
      f = own[k + ncg * ix_f];
    }
    double v = 0.5 * c1 + sixth * c2 + third * f;
    if (kind == GC_LIM && v > 2 * c1) v = 2 * c1;
    return v;
  }
  // physical boundary
  if (kind == GC_PHI) {
    // sides_bc_pot, src/streamer_2d.f90:620-638 (cyl :395-413)
    switch (nb) {
      case 0: return own[1 + ncg * k];
      case 1: return own[nc + ncg * k];
      case 2: return -own[k + ncg * 1];
      default: return 2 * R.applied_voltage - own[k + ncg * nc];
    }
  }
  // a$D_gc_neumann, m_aX_gc.f90:298-330
  switch (nb) {
    case 0: return own[1 + ncg * k];
    case 1: return own[nc + ncg * k];
    case 2: return own[k + ncg * 1];
    default: return own[k + ncg * nc];
  }
}

__device__ __forceinline__ int ghost_index(int nb, int k, int nc) {
  const int ncg = nc + 2;
  switch (nb) {
    case 0: return 0 + ncg * k;
    case 1: return (nc + 1) + ncg * k;
    case 2: return k;
    default: return k + ncg * (nc + 1);
  }
}

// a$D_gc_box for one box, group thread t (4*nc side ghosts).
__device__ __forceinline__ void gc_box(const RunDev &R, int id, int t, int iv, int kind) {
  const BoxMeta &m = R.meta[id];
  const int nc = m.nc;
  if (t < 4 * nc) {
    int nb = t / nc, k = t % nc + 1;
    double v = ghost_value(R, m, id, iv, nb, k, kind);
    CC(R, iv, id)[ghost_index(nb, k, nc)] = v;
  }
}

// Second ghost layer, afivo/src/m_aX_gc.f90:407-622 (gc2_box with
// gc2_prolong1 on refinement boundaries and gc2_neumann on physical ones)
__device__ double gc2_value(const RunDev &R, const BoxMeta &m, int id, int iv, int nb, int k) {
  const int nc = m.nc, ncg = nc + 2;
  const int nb_id = m.nb[nb];
  const int dim = nb >> 1;
  if (nb_id > 0) {
    const double *n = CC(R, iv, nb_id);
    switch (nb) {
      case 0: return n[(nc - 1) + ncg * k];
      case 1: return n[2 + ncg * k];
      case 2: return n[k + ncg * (nc - 1)];
      default: return n[k + ncg * 2];
    }
  }
  if (nb_id == 0) {
    int o0, o1;
    child_offset(m, nb, o0, o1);
    const double *P = CC(R, iv, R.meta[m.parent].nb[nb]);
    const int ix = (nb & 1) * (nc + 3) - 1;  // -1 or nc+2
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
    return 0.5 * P[i_c1 + ncg * j_c1] + 0.25 * P[i_c2 + ncg * j_c1] +
           0.25 * P[i_c1 + ncg * j_c2];
  }
  const double *own = CC(R, iv, id);
  switch (nb) {
    case 0: return own[2 + ncg * k];
    case 1: return own[(nc - 1) + ncg * k];
    case 2: return own[k + ncg * 2];
    default: return own[k + ncg * (nc - 1)];
  }
}

// ---------------------------------------------------------------------------
// Flux and source update.

// fluxes_koren, src/streamer_2d.f90:384-489 (cyl :416-521 is the same).
// T: arithmetic type of the flux (double; float in the mixed form, where the
// densities enter scaled by dens_scale and the flux leaves unscaled).
template <class T>
__device__ void fluxes_koren(const RunDev &R, double dt) {
  const int *ids;
  int n;
  list_range(R, 1, R.min_lvl, R.max_lvl, ids, n);
  const T ds = dens_scale<T>();
  const T fac = T(-0.8 * UC_EPS0 / (UC_ELEM_CHARGE * dt)) * ds;
  box_loop(ids, n, [&](int id, int t) {
    const BoxMeta &m = R.meta[id];
    const int nc = m.nc, ncg = nc + 2;
    const T inv_dr = T(1 / m.dr);
    const double *e = CC(R, I_ELEC, id), *fl = CC(R, I_FLD, id);
    double *fxe = FX(R, F_ELEC, id), *fye = FY(R, F_ELEC, id);
    const double *fxf = FX(R, F_FLD, id), *fyf = FY(R, F_FLD, id);
    const int nf = (nc + 1) * nc;
    for (int f = t; f < 2 * nf; f += GT) {
      const bool xd = f < nf;
      const int g = xd ? f : f - nf;
      int i, j;
      if (xd) { i = g % (nc + 1) + 1; j = g / (nc + 1) + 1; }
      else { i = (g & (nc - 1)) + 1; j = (g >> (31 - __clz(nc))) + 1; }
      // stride between the two cells adjacent to the face
      const int s = xd ? 1 : ncg;
      const int c = i + ncg * j;          // cell (i, j): high side of the face
      const int pos = xd ? i : j;         // face index along the direction
      T fld_avg = T(0.5) * (T(fl[c]) + T(fl[c - s]));
      Loc<T> loc = get_loc<T>(R, fld_avg);
      T mobility = col_at<T>(R, C_MOB, loc);
      T diff_coeff = col_at<T>(R, C_DIF, loc);
      T fld = T(xd ? fxf[fxi(i, j, nc)] : fyf[fyi(i, j, nc)]);
      T v_drift = -mobility * fld;
      const T ec = T(e[c]) * ds, em = T(e[c - s]) * ds;
      T gradc = ec - em;
      T fv;
      const int k = xd ? j : i;
      if (v_drift < T(0)) {
        T tmp = T((pos == nc + 1) ? gc2_value(R, m, id, I_ELEC, xd ? 1 : 3, k) : e[c + s]) * ds;
        T gradn = tmp - ec;
        fv = v_drift * (ec - koren_mlim(gradc, gradn));
        if (fv < fac * fld) fv = fac * fld;
      } else {
        T tmp = T((pos == 1) ? gc2_value(R, m, id, I_ELEC, xd ? 0 : 2, k) : e[c - 2 * s]) * ds;
        T gradp = em - tmp;
        fv = v_drift * (em + koren_mlim(gradc, gradp));
        if (fv > fac * fld) fv = fac * fld;
      }
      fv = fv - diff_coeff * gradc * inv_dr;
      const double out = (double)fv / (double)ds;
      if (xd) fxe[fxi(i, j, nc)] = out;
      else fye[fyi(i, j, nc)] = out;
    }
  });
}

// a$D_consistent_fluxes([f_elec]) with flux_from_children,
// afivo/src/m_aX_core.f90:818-930. All parent levels in one phase: the faces
// written (coarse leaves next to refined neighbours) are never read here.
__device__ void consistent_fluxes(const RunDev &R) {
  const int *ids;
  int n;
  list_range(R, 2, R.min_lvl, R.max_lvl - 1, ids, n);
  box_loop(ids, n, [&](int id, int t) {
    const BoxMeta &m = R.meta[id];
    const int nc = m.nc, nch = nc >> 1;
    if (t >= 4 * nc) return;
    const int nb = t / nc, mm0 = t % nc, kk = mm0 / nch, mm = mm0 % nch;
    const int nb_id = m.nb[nb];
    if (nb_id <= 0) return;
    if (R.meta[nb_id].ch[0] != 0) return;
    const bool low = (nb & 1) == 0;
    const int i = low ? 1 : nc + 1, i_nb = low ? nc + 1 : 1;
    const int i_ch = c_ch_adj_nb[nb][kk];
    const int cid = m.ch[i_ch];
    if ((nb >> 1) == 0) {
      const int ioff1 = nch * c_ch_dix[i_ch][1];
      const double *cf = FX(R, F_ELEC, cid);
      FX(R, F_ELEC, nb_id)[fxi(i_nb, ioff1 + mm + 1, nc)] =
          0.5 * (cf[fxi(i, 2 * mm + 1, nc)] + cf[fxi(i, 2 * mm + 2, nc)]);
    } else {
      const int ioff0 = nch * c_ch_dix[i_ch][0];
      const double *cf = FY(R, F_ELEC, cid);
      FY(R, F_ELEC, nb_id)[fyi(ioff0 + mm + 1, i_nb, nc)] =
          0.5 * (cf[fyi(2 * mm + 1, i, nc)] + cf[fyi(2 * mm + 2, i, nc)]);
    }
  });
}

// update_solution, src/streamer_2d.f90:499-542 and src/streamer_cyl.f90:531-570.
// T: arithmetic type of the source and flux divergence (float in the mixed
// form); the densities are accumulated in double.
template <class T>
__device__ void update_solution(const RunDev &R, double dt) {
  const int *ids;
  int n;
  list_range(R, 1, R.min_lvl, R.max_lvl, ids, n);
  const bool cyl = R.coord == 1;
  box_loop(ids, n, [&](int id, int t) {
    const BoxMeta &m = R.meta[id];
    const int nc = m.nc, ncg = nc + 2;
    if (t >= nc * nc) return;
    const int i = (t & (nc - 1)) + 1, j = (t >> (31 - __clz(nc))) + 1, c = i + ncg * j;
    const T inv_dr = T(1 / m.dr);
    double *e = CC(R, I_ELEC, id), *pi = CC(R, I_PION, id);
    const double *fxe = FX(R, F_ELEC, id), *fye = FY(R, F_ELEC, id);
    T fld = T(CC(R, I_FLD, id)[c]);
    Loc<T> loc = get_loc<T>(R, fld);
    T alpha = col_at<T>(R, C_ALPHA, loc);
    T eta = col_at<T>(R, C_ETA, loc);
    T fx0 = T(fxe[fxi(i, j, nc)]), fx1 = T(fxe[fxi(i + 1, j, nc)]);
    T fy0 = T(fye[fyi(i, j, nc)]), fy1 = T(fye[fyi(i, j + 1, nc)]);
    T src = T(0.5) * norm2_2<T>(fx0 + fx1, fy0 + fy1) * (alpha - eta);
    if (R.ph_enabled) src = src + T(CC(R, I_PHO, id)[c]);
    T sflux;
    if (cyl) {
      int ioff = (m.ix0 - 1) * nc;
      T den = T(i + ioff) - T(0.5);
      T rf1 = T(i + ioff - 1) / den, rf2 = T(i + ioff) / den;
      sflux = (fy0 - fy1 + rf1 * fx0 - rf2 * fx1) * inv_dr;
    } else {
      sflux = (fx0 - fx1 + fy0 - fy1) * inv_dr;
    }
    const T tdt = T(dt);
    double ne = e[c] + (double)((src + sflux) * tdt);
    double ni = pi[c] + (double)(src * tdt);
    if (!cyl && CC(R, I_EPS, id)[c] > 1.0) {
      ni = ni - ne;
      ne = 0;
    }
    e[c] = ne;
    pi[c] = ni;
  });
}

constexpr int MP = I_PHI, MT = I_FLD, MR = I_RHS;

// ---------------------------------------------------------------------------
// Plan-based operations. The host writes, once per topology, one BoxRec per
// box (level by level, in list order; build_plans) holding the slot bases of
// the box, its parent, its same-level neighbours, its parent's neighbours and
// its children, its offset in the parent and its list membership. Every
// index a phase needs -- neighbour cells, ghost-cell sources, restriction and
// correction stencils -- is derived from that record, and a phase is a flat
// loop of all threads over the (box, cell) items of one level.

__device__ __forceinline__ double *VAR(const RunDev &R, int v) {
  return R.cc + (size_t)v * R.capacity * SLOT;
}

// Where the multigrid variables live during a solve: device memory, or a
// compact copy in shared memory when the tree fits (then every read in a
// phase that follows a write by another thread hits shared memory instead
// of L2). boxes: the BoxRecs addressing those arrays.
// T is the storage and arithmetic type of the solve: double for the plain
// FP64 path, float for the inner correction solve of the mixed form. V is the
// potential of the applied-voltage wall (0 for the homogeneous correction
// equation); sw_*: half-sweeps per level visit (reference: 4 down, 4 up,
// 2 n_cycle_base on the coarsest level).
template <class T>
struct MGV {
  T *phi, *rhs, *tmp;
  const BoxRec *boxes;
  const int *pbx;
  bool plans;  // the cell plans of "Cell plans" are available (shared-memory solve)
  double V;
  int sw_down, sw_up, sw_base;
};

// Side ghost (side, k) of the potential: sides_from_nb, mg$D_sides_rb after
// a$D_gc_prolong0 (m_aX_mg.f90:261-301), or sides_bc_pot
// (src/streamer_2d.f90:620-638). Reads only interior cells of the box and its
// neighbours and ghost cells of the parent. This is the readable statement
// of the recipe; the phases call phi_ghost_sl below, which gives the same
// values with its loads issued together.
template <class T>
__device__ __forceinline__ T phi_ghost(double V, const T *phi, const BoxRec &B, int nc, int ncg,
                                       int side, int k) {
  const int dim = side >> 1;
  const bool low = (side & 1) == 0;
  const int nbb = B.nb[side];
  if (nbb > 0) return phi[nbb + (dim == 0 ? (low ? nc : 1) + ncg * k : k + ncg * (low ? nc : 1))];
  const int ix = low ? 1 : nc;
  const int own = B.base + (dim == 0 ? ix + ncg * k : k + ncg * ix);
  if (nbb == NBR_RB) {
    const int di = low ? 1 : -1, dk = -1 + 2 * (k & 1), ig = ix - di;
    int pc, a, b;
    if (dim == 0) {
      pc = B.pbase + (B.o0 + ((ig + 1) >> 1)) + ncg * (B.o1 + ((k + 1) >> 1));
      a = own + di;
      b = own + ncg * dk;
    } else {
      pc = B.pbase + (B.o0 + ((k + 1) >> 1)) + ncg * (B.o1 + ((ig + 1) >> 1));
      a = own + dk;
      b = own + ncg * di;
    }
    return T(0.5) * phi[pc] + phi[own] - T(0.25) * (phi[a] + phi[b]);
  }
  if (side == 2) return -phi[own];
  if (side == 3) return T(2 * V) - phi[own];
  return phi[own];
}

// Side ghost (side, k) of a density or |E|: sides_from_nb (a copy of the
// neighbour's cell), a$D_gc_interp (lim: a$D_gc_interp_lim) from the
// parent's neighbour, 1/2 c1 + 1/6 c2 + 1/3 own (m_aX_gc.f90:90-295), or
// a$D_gc_neumann. Straight-line form: the source addresses of the side's
// kind are selected first and loaded together, so that a ghost's loads do
// not wait behind branches.
__device__ __forceinline__ double den_ghost_sl(const double *x, const BoxRec &B, int nc, int ncg,
                                               int side, int k, bool lim) {
  const int dim = side >> 1;
  const bool low = (side & 1) == 0;
  const int nbb = B.nb[side];
  const int ix = low ? 1 : nc;
  const int own = B.base + (dim == 0 ? ix + ncg * k : k + ncg * ix);
  const int cp = nbb + (dim == 0 ? (low ? nc : 1) + ncg * k : k + ncg * (low ? nc : 1));
  const bool isnb = nbb > 0, isrb = nbb == NBR_RB;
  const int pn = B.pnb[side], ix_c = low ? nc : 1;
  const int c1 = (dim == 0 ? B.o1 : B.o0) + ((k + 1) >> 1), c2 = c1 + 1 - 2 * (k & 1);
  const int r1 = dim == 0 ? pn + ix_c + ncg * c1 : pn + c1 + ncg * ix_c;
  const int r2 = dim == 0 ? pn + ix_c + ncg * c2 : pn + c2 + ncg * ix_c;
  const int s0 = isnb ? cp : (isrb ? r1 : own), s1 = isrb ? r2 : s0, s2 = isrb ? own : s0;
  const double v0 = x[s0], v1 = x[s1], v2 = x[s2];
  const double sixth = 1 / 6.0, third = 1 / 3.0;
  double v = 0.5 * v0 + sixth * v1 + third * v2;
  if (lim && v > 2 * v0) v = 2 * v0;
  return isrb ? v : v0;
}

// phi_ghost in straight-line form: the addresses of all candidate sources
// are formed first, the values loaded together and the result selected by
// the kind of the side (neighbour copy, refinement boundary, physical wall),
// so that a cell's loads are in flight together instead of behind branches.
// Same values and the same arithmetic as phi_ghost.
template <class T>
__device__ __forceinline__ T phi_ghost_sl(double V, const T *phi, const BoxRec &B, int nc, int ncg,
                                          int side, int k) {
  const int dim = side >> 1;
  const bool low = (side & 1) == 0;
  const int nbb = B.nb[side];
  const int ix = low ? 1 : nc;
  const int own = B.base + (dim == 0 ? ix + ncg * k : k + ncg * ix);
  const int di = low ? 1 : -1, dk = -1 + 2 * (k & 1), ig = ix - di;
  const int h1 = (ig + 1) >> 1, h2 = (k + 1) >> 1;
  const int pc = B.pbase + (dim == 0 ? (B.o0 + h1) + ncg * (B.o1 + h2)
                                     : (B.o0 + h2) + ncg * (B.o1 + h1));
  const int a = own + (dim == 0 ? di : dk);
  const int b = own + ncg * (dim == 0 ? dk : di);
  const int cp = nbb + (dim == 0 ? (low ? nc : 1) + ncg * k : k + ncg * (low ? nc : 1));
  const bool isnb = nbb > 0, isrb = nbb == NBR_RB;
  const int s0 = isnb ? cp : (isrb ? pc : own);
  const int s1 = isrb ? own : s0, s2 = isrb ? a : s0, s3 = isrb ? b : s0;
  const T v0 = phi[s0], v1 = phi[s1], v2 = phi[s2], v3 = phi[s3];
  const T vrb = T(0.5) * v0 + v1 - T(0.25) * (v2 + v3);
  const T vbc = side == 2 ? -v0 : (side == 3 ? T(2 * V) - v0 : v0);
  return isnb ? v0 : (isrb ? vrb : vbc);
}

// phi_ghost_sl with the refinement-boundary source read where the parent's
// ghost cell takes it from: at a refinement boundary the parent has a
// same-level neighbour on that side (2:1 balance), so the parent's ghost
// cell under the fine ghost is a copy of that neighbour's cell (pnb). Right
// after the parent's ghost fill both hold the same value; reading the
// neighbour's cell lets the fills of all levels run in one phase.
template <class T>
__device__ __forceinline__ T phi_ghost_flat(double V, const T *phi, const BoxRec &B, int nc, int ncg,
                                            int side, int k) {
  const int dim = side >> 1;
  const bool low = (side & 1) == 0;
  const int nbb = B.nb[side];
  const int ix = low ? 1 : nc;
  const int own = B.base + (dim == 0 ? ix + ncg * k : k + ncg * ix);
  const int di = low ? 1 : -1, dk = -1 + 2 * (k & 1);
  const int h2 = (k + 1) >> 1, xc = low ? nc : 1;
  const int pc = B.pnb[side] + (dim == 0 ? xc + ncg * (B.o1 + h2) : (B.o0 + h2) + ncg * xc);
  const int a = own + (dim == 0 ? di : dk);
  const int b = own + ncg * (dim == 0 ? dk : di);
  const int cp = nbb + (dim == 0 ? (low ? nc : 1) + ncg * k : k + ncg * (low ? nc : 1));
  const bool isnb = nbb > 0, isrb = nbb == NBR_RB;
  const int s0 = isnb ? cp : (isrb ? pc : own);
  const int s1 = isrb ? own : s0, s2 = isrb ? a : s0, s3 = isrb ? b : s0;
  const T v0 = phi[s0], v1 = phi[s1], v2 = phi[s2], v3 = phi[s3];
  const T vrb = T(0.5) * v0 + v1 - T(0.25) * (v2 + v3);
  const T vbc = side == 2 ? -v0 : (side == 3 ? T(2 * V) - v0 : v0);
  return isnb ? v0 : (isrb ? vrb : vbc);
}

// Neighbours (lx, hx, ly, hy) of interior cell (i, j). A cell has at most
// one ghost neighbour in x and one in y; both are evaluated unconditionally
// (straight-line) and selected where needed.
template <class T>
__device__ __forceinline__ void phi_nbrs(double V, const T *phi, const BoxRec &B, int nc, int ncg,
                                         int i, int j, int g, T &lx, T &hx, T &ly, T &hy) {
  const T gx = phi_ghost_sl(V, phi, B, nc, ncg, i == 1 ? 0 : 1, j);
  const T gy = phi_ghost_sl(V, phi, B, nc, ncg, j == 1 ? 2 : 3, i);
  const T dlx = phi[g - (i > 1 ? 1 : 0)], dhx = phi[g + (i < nc ? 1 : 0)];
  const T dly = phi[g - (j > 1 ? ncg : 0)], dhy = phi[g + (j < nc ? ncg : 0)];
  lx = i > 1 ? dlx : gx;
  hx = i < nc ? dhx : gx;
  ly = j > 1 ? dly : gy;
  hy = j < nc ? dhy : gy;
}

// box_lpl (m_aX_mg.f90:662-680) / box_clpl (:1027-1049) at one cell
// A box the multigrid treats with the eps operators (its tag; device-memory
// multigrid of a dielectric run only).
__device__ __forceinline__ bool diel_box(const RunDev &R, const BoxRec &B) {
  return R.diel && R.tags[B.gbase / SLOT] == TAG_DIEL;
}
// A box the multigrid treats with the level-set operators (its tag); the
// block form is never launched for a run with level-set boxes.
__device__ __forceinline__ bool lsf_box(const RunDev &R, const BoxRec &B) {
  return kGrid && R.has_lsf && R.tags[B.gbase / SLOT] == TAG_LSF;
}

// lsf_dist_val (afivo/src/m_aX_mg.f90:1077-1104): from cell a (level set la,
// boundary value ba) to neighbour b (level set lb, value vb, boundary value
// bb): where the level set changes sign between them, the interface at
// distance la / (la - lb) with the interpolated boundary value; else b.
__device__ __forceinline__ void lsf_dist_val(double la, double ba, double lb, double vb, double bb,
                                             double &dist, double &val) {
  if (la * lb < 0) {
    dist = la / (la - lb);
    val = ba * (1 - dist) + bb * dist;
  } else {
    dist = 1;
    val = vb;
  }
}

// Distances and values of the four neighbours (lx, hx, ly, hy; values u,
// ghost neighbours from their recipes) of cell (i, j) of a level-set box.
__device__ __forceinline__ void lsf_nbrs(const RunDev &R, const BoxRec &B, int ncg, int i, int j,
                                         const double u[4], double dd[4], double val[4]) {
  const double *L = R.lsf + B.gbase, *Bv = R.bval + B.gbase;
  const int loc = i + ncg * j;
  const int nb[4] = {loc - 1, loc + 1, loc - ncg, loc + ncg};
  const double la = L[loc], ba = Bv[loc];
#pragma unroll
  for (int k = 0; k < 4; k++) lsf_dist_val(la, ba, L[nb[k]], u[k], Bv[nb[k]], dd[k], val[k]);
}

// mg$D_box_lpllsf at one cell (afivo/src/m_aX_mg.f90:1270-1340, 2D):
// 2 inv_dr^2 (sum over x and y of (d2 v1 + d1 v2 - (d1 + d2) u0) /
// ((d1 + d2) d1 d2)), in the reference's operation order.
__device__ __forceinline__ double lap_lsf(const RunDev &R, const BoxRec &B, int ncg, int i, int j,
                                          double f0, const double u[4], double inv_dr_sq) {
  double dd[4], val[4];
  lsf_nbrs(R, B, ncg, i, j, u, dd, val);
  return 2 * inv_dr_sq *
         ((dd[1] * val[0] + dd[0] * val[1] - (dd[0] + dd[1]) * f0) / ((dd[0] + dd[1]) * dd[0] * dd[1]) +
          (dd[3] * val[2] + dd[2] * val[3] - (dd[2] + dd[3]) * f0) / ((dd[2] + dd[3]) * dd[2] * dd[3]));
}

// Laplacian of a dielectric box at one cell (mg$D_box_lpld,
// afivo/src/m_aX_mg.f90:951-1001; cylindrical mg2_box_clpld, :1467-1495):
// inv_dr^2 * 2 * sum over lx, hx, ly, hy of rfac a0 a / (a0 + a) (u - u0),
// a0 and a the eps of the cell and of the neighbour.
__device__ __forceinline__ double lap_diel(const RunDev &R, const BoxRec &B, int ncg, int i, int j,
                                           double v, const double u[4], double inv_dr_sq) {
  const double *eps = VAR(R, I_EPS) + B.gbase;
  const int loc = i + ncg * j;
  const double a0 = eps[loc];
  const double a[4] = {eps[loc - 1], eps[loc + 1], eps[loc - ncg], eps[loc + ncg]};
  double rf[4] = {1, 1, 1, 1};
  if (R.coord == 1) {
    const int gi = B.gi0 + i;
    const double den = gi - 0.5;
    rf[0] = (gi - 1) / den;
    rf[1] = gi / den;
  }
  double sum = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (R.coord == 1) sum = sum + rf[k] * a0 * a[k] / (a0 + a[k]) * (u[k] - v);
    else sum = sum + a0 * a[k] / (a0 + a[k]) * (u[k] - v);
  }
  return inv_dr_sq * 2 * sum;
}

template <class T>
__device__ __forceinline__ T lap_at(const RunDev &R, double V, const T *phi, const BoxRec &B, int nc,
                                    int ncg, int i, int j, T inv_dr_sq) {
  const int g = B.base + i + ncg * j;
  T lx, hx, ly, hy;
  phi_nbrs(V, phi, B, nc, ncg, i, j, g, lx, hx, ly, hy);
  const T v = phi[g];
  if (lsf_box(R, B)) {
    const double u[4] = {(double)lx, (double)hx, (double)ly, (double)hy};
    return T(lap_lsf(R, B, ncg, i, j, (double)v, u, (double)inv_dr_sq));
  }
  if (diel_box(R, B)) {
    const double u[4] = {(double)lx, (double)hx, (double)ly, (double)hy};
    return T(lap_diel(R, B, ncg, i, j, (double)v, u, (double)inv_dr_sq));
  }
  if (R.coord == 1) {
    const int gi = B.gi0 + i;
    const T den = T(gi) - T(0.5);
    const T rf1 = T(gi - 1) / den, rf2 = T(gi) / den;
    return (rf1 * lx + rf2 * hx + ly + hy - T(4) * v) * inv_dr_sq;
  }
  return inv_dr_sq * (lx + hx + ly + hy - T(4) * v);
}

struct LvlInfo {
  int nc, ncg, sh, b0, nb, li;
  double dr;
};
__device__ __forceinline__ LvlInfo lvl_info(const RunDev &R, int lvl) {
  const int li = lvl - R.min_lvl;
  LvlInfo L;
  L.nc = R.lv_nc[li];
  L.ncg = L.nc + 2;
  L.sh = 31 - __clz(L.nc);  // log2(nc)
  L.b0 = R.bx_off[li];
  L.nb = R.bx_off[li + 1] - L.b0;
  L.li = li;
  L.dr = R.lv_dr[li];
  return L;
}

// Cursor over the interior cells of every box of every level, level by
// level in plan order, for flat loops in which each thread moves forward:
// cells of different levels can then be in flight together.
struct CellCursor {
  int li, lo, hi;  // level index and the flat range [lo, hi) of its cells
};
__device__ __forceinline__ int level_cells(const RunDev &R, int li) {
  return (R.bx_off[li + 1] - R.bx_off[li]) * R.lv_nc[li] * R.lv_nc[li];
}
__device__ __forceinline__ CellCursor cell_cursor(const RunDev &R) { return CellCursor{0, 0, level_cells(R, 0)}; }
// Flat cell k (not below the previous call's k) as level index, box record
// index and (i, j); false past the last level.
__device__ __forceinline__ bool cell_at(const RunDev &R, CellCursor &c, int k, int &li, int &b, int &i,
                                        int &j) {
  while (k >= c.hi) {
    if (++c.li >= R.nlev) return false;
    c.lo = c.hi;
    c.hi = c.lo + level_cells(R, c.li);
  }
  li = c.li;
  const int nc = R.lv_nc[li], sh = 31 - __clz(nc), t = k - c.lo;
  b = R.bx_off[li] + (t >> (2 * sh));
  i = (t & (nc - 1)) + 1;
  j = ((t >> sh) & (nc - 1)) + 1;
  return true;
}

// Red-black Gauss-Seidel half-sweep `it` on level lvl (box_gsrb_lpl,
// m_aX_mg.f90:636-659; box_gsrb_clpl :998-1024). Ghost neighbours are
// evaluated from their sources, which equals the ghost fill the reference
// performs after every half-sweep (gsrb_boxes, :343-366): those sources are
// cells of the colour not updated here, the updated cell itself (read before
// it is written), or coarser-level cells. mem: read ghosts from memory
// instead (first half-sweep of a first FMG call, where the reference's
// ghosts are not consistent with the interior).
template <class T>
__device__ __noinline__ void p_sweep(const RunDev &R, const MGV<T> &M, int lvl, int it, bool mem) {
  const LvlInfo L = lvl_info(R, lvl);
  T *phi = M.phi;
  const T *rhs = M.rhs;
  const T dx2 = T(L.dr * L.dr);
  const int half = (L.nc * L.nc) >> 1, hsh = 2 * L.sh - 1, hn = L.nc >> 1;
  const int p = it & 1;  // parity (i + j) & 1 of the updated cells
  const bool cyl = R.coord == 1;
  const int n = L.nb * half;
  for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
    const BoxRec &B = M.boxes[L.b0 + (k >> hsh)];
    const int t = k & (half - 1);
    const int j = t / hn + 1, m = t % hn;
    const int i = 2 * m + 2 - ((p + j) & 1);
    const int g = B.base + i + L.ncg * j;
    T lx, hx, ly, hy;
    if (mem) {
      lx = phi[g - 1]; hx = phi[g + 1]; ly = phi[g - L.ncg]; hy = phi[g + L.ncg];
    } else {
      phi_nbrs(M.V, phi, B, L.nc, L.ncg, i, j, g, lx, hx, ly, hy);
    }
    const T r = rhs[g];
    if (lsf_box(R, B)) {
      // mg$D_box_gsrb_lpllsf (afivo/src/m_aX_mg.f90:1190-1267, 2D)
      const double u[4] = {(double)lx, (double)hx, (double)ly, (double)hy};
      double dd[4], val[4];
      lsf_nbrs(R, B, L.ncg, i, j, u, dd, val);
      const double prod = dd[0] * dd[1] * dd[2] * dd[3];
      phi[g] = T(1 / (dd[0] * dd[1] + dd[2] * dd[3]) *
                 ((dd[1] * val[0] + dd[0] * val[1]) * dd[2] * dd[3] / (dd[0] + dd[1]) +
                  (dd[3] * val[2] + dd[2] * val[3]) * dd[0] * dd[1] / (dd[2] + dd[3]) -
                  0.5 * prod * (double)dx2 * (double)r));
    } else if (diel_box(R, B)) {
      // mg$D_box_gsrb_lpld (afivo/src/m_aX_mg.f90:895-948; cylindrical
      // mg2_box_gsrb_clpld, :1499-1531): face weights c = 2 a0 a / (a0 + a),
      // phi = (sum c rfac u - dx^2 rhs) / sum c rfac
      const double *eps = VAR(R, I_EPS) + B.gbase;
      const int loc = i + L.ncg * j;
      const double a0 = eps[loc];
      const double a[4] = {eps[loc - 1], eps[loc + 1], eps[loc - L.ncg], eps[loc + L.ncg]};
      const double u[4] = {(double)lx, (double)hx, (double)ly, (double)hy};
      double rf[4] = {1, 1, 1, 1};
      if (cyl) {
        const int gi = B.gi0 + i;
        const double den = gi - 0.5;
        rf[0] = (gi - 1) / den;
        rf[1] = gi / den;
      }
      double su = 0, sc = 0;
#pragma unroll
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
      phi[g] = T((su - (double)dx2 * (double)r) / sc);
    } else if (cyl) {
      const int gi = B.gi0 + i;
      const T den = T(gi) - T(0.5);
      const T rf1 = T(gi - 1) / den, rf2 = T(gi) / den;
      phi[g] = T(0.25) * (rf1 * lx + rf2 * hx + hy + ly - dx2 * r);
    } else {
      phi[g] = T(0.25) * (hx + lx + hy + ly - dx2 * r);
    }
  }
  PSYNC();
}

// Ghost fill of the potential on level lvl (fill_gc_phi, :303-316), no
// barrier. copy_tmp: also tmp = phi on the ghosts of parent boxes (the
// whole-box copy of update_coarse, :407).
template <class T>
__device__ __forceinline__ void fill_phi_loop(const RunDev &R, const MGV<T> &M, const LvlInfo &L, bool copy_tmp) {
  T *phi = M.phi, *tmp = M.tmp;
  const int per = 4 * L.nc, n = L.nb * per;
  for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
    const BoxRec &B = M.boxes[L.b0 + (k >> (L.sh + 2))];
    const int r = k & (per - 1), side = r >> L.sh, kk = (r & (L.nc - 1)) + 1;
    const T v = phi_ghost_sl(M.V, phi, B, L.nc, L.ncg, side, kk);
    const int dim = side >> 1, gx = (side & 1) ? L.nc + 1 : 0;
    const int d = B.base + (dim == 0 ? gx + L.ncg * kk : kk + L.ncg * gx);
    phi[d] = v;
    if (copy_tmp && (B.flags & CF_PARENT)) tmp[d] = v;
  }
}
template <class T>
__device__ void p_fill(const RunDev &R, const MGV<T> &M, int lvl) {
  fill_phi_loop(R, M, lvl_info(R, lvl), false);
  PSYNC();
}

// For every box of level lvl: the residual rhs - A phi (residual_box,
// :475-484) restricted into the parent's tmp and phi restricted into the
// parent's phi (box_rstr_lpl, :683-705); fill: the ghosts of level lvl are
// filled in the same phase (the residual evaluates ghost neighbours from
// their sources). leaf_rhs: first set the space charge e/eps0 (n_e - n_i) on
// leaf cells (src/streamer_2d.f90:317-329). store_res: keep the residual in
// the box's own tmp (set_coarse_phi_rhs); otherwise tmp is left as it was
// (update_coarse saves and restores it).
template <class T>
__device__ __noinline__ void p_fr(const RunDev &R, const MGV<T> &M, int lvl, bool fill, bool leaf_rhs, bool store_res) {
  const LvlInfo L = lvl_info(R, lvl);
  const int pncg = R.lv_nc[lvl - 1 - R.min_lvl] + 2;
  T *phi = M.phi, *tmp = M.tmp, *rhs = M.rhs;
  const double *e = VAR(R, I_ELEC), *pi = VAR(R, I_PION);
  const T inv_dr_sq = T(1 / (L.dr * L.dr));
  const double fac = UC_ELEM_CHARGE / UC_EPS0;
  // one cell per thread, whole warps per iteration: the 2x2 block of a
  // parent cell is gathered by shuffles (cells of a box are consecutive
  // threads, i fastest) and added in the order of box_rstr_lpl
  const int per = L.nc * L.nc, n = L.nb * per, nw = (n + 31) & ~31;
  for (int k = TID(), nt_ = NTH(); k < nw; k += nt_) {
    const bool act = k < n;
    const BoxRec &B = M.boxes[L.b0 + (act ? k >> (2 * L.sh) : 0)];
    const int t = k & (per - 1), i = (t & (L.nc - 1)) + 1, j = (t >> L.sh) + 1;
    const int g = B.base + i + L.ncg * j;
    T res = 0, ph = 0;
    if (act) {
      T rh;
      if (leaf_rhs && (B.flags & CF_LEAF)) {
        const int gg = B.gbase + i + L.ncg * j;
        rh = T(fac * (e[gg] - pi[gg]));
        rhs[g] = rh;
      } else {
        rh = rhs[g];
      }
      res = rh - lap_at(R, M.V, phi, B, L.nc, L.ncg, i, j, inv_dr_sq);
      if (store_res) tmp[g] = res;
      ph = phi[g];
    }
    const unsigned FULL = 0xffffffffu;
    const T r1 = __shfl_down_sync(FULL, res, 1), r2 = __shfl_down_sync(FULL, res, L.nc),
            r3 = __shfl_down_sync(FULL, res, L.nc + 1);
    const T p1 = __shfl_down_sync(FULL, ph, 1), p2 = __shfl_down_sync(FULL, ph, L.nc),
            p3 = __shfl_down_sync(FULL, ph, L.nc + 1);
    if (act && (i & 1) && (j & 1)) {
      const int d = B.pbase + (B.o0 + (i + 1) / 2) + pncg * (B.o1 + (j + 1) / 2);
      tmp[d] = T(0.25) * (res + r1 + r2 + r3);
      phi[d] = T(0.25) * (ph + p1 + p2 + p3);
    }
  }
  if (fill) fill_phi_loop(R, M, L, false);
  PSYNC();
}

// Ghost fill of level lvl and the coarse right-hand side of its parent
// boxes: rhs = A phi + tmp (box_op then a$D_box_add_cc, :399-402 / :441-444);
// copy_tmp: then tmp = phi (a$D_box_copy_cc, :403).
template <class T>
__device__ void p_fc(const RunDev &R, const MGV<T> &M, int lvl, bool copy_tmp) {
  const LvlInfo L = lvl_info(R, lvl);
  const int li = lvl - R.min_lvl;
  const int *pb = M.pbx + R.pb_off[li];
  const int npb = R.pb_off[li + 1] - R.pb_off[li];
  T *phi = M.phi, *tmp = M.tmp, *rhs = M.rhs;
  const T inv_dr_sq = T(1 / (L.dr * L.dr));
  const int per = L.nc * L.nc, n = npb * per;
  for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
    const BoxRec &B = M.boxes[pb[k >> (2 * L.sh)]];
    const int t = k & (per - 1), i = (t & (L.nc - 1)) + 1, j = (t >> L.sh) + 1;
    const int g = B.base + i + L.ncg * j;
    const T a = lap_at(R, M.V, phi, B, L.nc, L.ncg, i, j, inv_dr_sq);
    const T pv = phi[g];
    rhs[g] = a + tmp[g];
    if (copy_tmp) tmp[g] = pv;
  }
  fill_phi_loop(R, M, L, copy_tmp);
  PSYNC();
}

// Boxes of level lvl: copy: tmp = phi (a$D_boxes_copy_cc in mg$D_fas_fmg,
// :187-188); correct: phi += prolongation of the parent's correction
// (correct_children :319-341 with box_corr_lpl :605-633). The correction
// phi_p - tmp_p is formed where it is used instead of being stored back into
// the parent's tmp; that stored value is never read again by the reference.
template <class T>
__device__ void p_correct(const RunDev &R, const MGV<T> &M, int lvl, bool copy, bool correct) {
  const LvlInfo L = lvl_info(R, lvl);
  const int pncg = correct ? R.lv_nc[lvl - 1 - R.min_lvl] + 2 : 0;
  T *phi = M.phi, *tmp = M.tmp;
  const int per = L.nc * L.nc, n = L.nb * per;
  for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
    const BoxRec &B = M.boxes[L.b0 + (k >> (2 * L.sh))];
    const int t = k & (per - 1), i = (t & (L.nc - 1)) + 1, j = (t >> L.sh) + 1;
    const int g = B.base + i + L.ncg * j;
    const T v = phi[g];
    if (copy) tmp[g] = v;
    if (correct) {
      const int i_c1 = B.o0 + ((i + 1) >> 1), i_c2 = i_c1 + 1 - 2 * (i & 1);
      const int j_c1 = B.o1 + ((j + 1) >> 1), j_c2 = j_c1 + 1 - 2 * (j & 1);
      const int p1 = B.pbase + i_c1 + pncg * j_c1;
      const int p2 = B.pbase + i_c2 + pncg * j_c1;
      const int p3 = B.pbase + i_c1 + pncg * j_c2;
      const T c1 = phi[p1] - tmp[p1], c2x = phi[p2] - tmp[p2], c2y = phi[p3] - tmp[p3];
      if (lsf_box(R, B)) {
        // mg$D_box_corr_lpllsf (afivo/src/m_aX_mg.f90:1106-1187, 2D): the
        // correction along the lines to the three coarse cells, each cut at
        // the interface, where a correction is 0
        const double *lsf = R.lsf;
        const double la = lsf[B.gbase + i + L.ncg * j];
        const int pp[3] = {p1, p2, p3};
        const double cv[3] = {(double)c1, (double)c2x, (double)c2y};
        double dist[3], val[3];
#pragma unroll
        for (int q = 0; q < 3; q++) lsf_dist_val(la, 0.0, lsf[pp[q]], cv[q], 0.0, dist[q], val[q]);
        const double cw[3] = {2 * dist[1] * dist[2], dist[0] * dist[2], dist[0] * dist[1]};
        phi[g] = T((double)v + (cw[0] * val[0] + cw[1] * val[1] + cw[2] * val[2]) /
                                   (cw[0] + cw[1] + cw[2]));
      } else if (diel_box(R, B)) {
        // mg$D_box_corr_lpld (afivo/src/m_aX_mg.f90:1003-1071, 2D): eps-weighted
        // averages of the parent's correction toward each coarse neighbour
        const double *eps = VAR(R, I_EPS);
        const double a0 = eps[p1], a1 = eps[p2], a2 = eps[p3];
        double sum = 0;
        sum = sum + (a0 * (double)c1 + a1 * (double)c2x) / (a0 + a1);
        sum = sum + (a0 * (double)c1 + a2 * (double)c2y) / (a0 + a2);
        phi[g] = T((double)v + 0.5 * sum);
      } else {
        phi[g] = v + T(0.5) * c1 + T(0.25) * (c2x + c2y);
      }
    }
  }
  if (copy) {
    const int pg = 4 * L.nc, ng = L.nb * pg;
    for (int k = TID(), nt_ = NTH(); k < ng; k += nt_) {
      const BoxRec &B = M.boxes[L.b0 + (k >> (L.sh + 2))];
      const int r = k & (pg - 1), side = r >> L.sh, kk = (r & (L.nc - 1)) + 1;
      const int dim = side >> 1, gx = (side & 1) ? L.nc + 1 : 0;
      const int d = B.base + (dim == 0 ? gx + L.ncg * kk : kk + L.ncg * gx);
      tmp[d] = phi[d];
    }
  }
  PSYNC();
}

// init_phi_rhs for one level (m_aX_mg.f90:450-473): phi = 0 on the boxes of
// level lvl and their rhs restricted to the parents.
template <class T>
__device__ __noinline__ void p_init_level(const RunDev &R, const MGV<T> &M, int lvl, bool leaf_rhs) {
  const LvlInfo L = lvl_info(R, lvl);
  const int pncg = R.lv_nc[lvl - 1 - R.min_lvl] + 2;
  T *rhs = M.rhs, *phi = M.phi;
  const double *e = VAR(R, I_ELEC), *pi = VAR(R, I_PION);
  const double fac = UC_ELEM_CHARGE / UC_EPS0;
  const int hn = L.nc >> 1, per = hn * hn, n = L.nb * per;
  for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
    const BoxRec &B = M.boxes[L.b0 + (k >> (2 * L.sh - 2))];
    const int t = k & (per - 1), ii = (t & (hn - 1)) + 1, jj = (t >> (L.sh - 1)) + 1;
    const bool leaf = leaf_rhs && (B.flags & CF_LEAF);
    T rs[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int loc = (2 * ii - 1 + (q & 1)) + L.ncg * (2 * jj - 1 + (q >> 1));
      const int g = B.base + loc;
      if (leaf) {
        rs[q] = T(fac * (e[B.gbase + loc] - pi[B.gbase + loc]));
        rhs[g] = rs[q];
      } else {
        rs[q] = rhs[g];
      }
    }
    rhs[B.pbase + (B.o0 + ii) + pncg * (B.o1 + jj)] = T(0.25) * (rs[0] + rs[1] + rs[2] + rs[3]);
  }
  const int pc = L.ncg * L.ncg, nz = L.nb * pc;
  for (int k = TID(), nt_ = NTH(); k < nz; k += nt_) phi[M.boxes[L.b0 + k / pc].base + k % pc] = T(0);
  PSYNC();
}

// Residual rhs - A phi on every cell of levels min..max (set_residual of
// mg$D_fas_vcycle, :243-253)
template <class T>
__device__ __noinline__ void p_residual_all(const RunDev &R, const MGV<T> &M, int max_lvl) {
  T *phi = M.phi, *tmp = M.tmp;
  const T *rhs = M.rhs;
  for (int lvl = R.min_lvl; lvl <= max_lvl; lvl++) {
    const LvlInfo L = lvl_info(R, lvl);
    const T inv_dr_sq = T(1 / (L.dr * L.dr));
    const int per = L.nc * L.nc, n = L.nb * per;
    for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
      const BoxRec &B = M.boxes[L.b0 + (k >> (2 * L.sh))];
      const int t = k & (per - 1), i = (t & (L.nc - 1)) + 1, j = (t >> L.sh) + 1;
      const int g = B.base + i + L.ncg * j;
      tmp[g] = rhs[g] - lap_at(R, M.V, phi, B, L.nc, L.ncg, i, j, inv_dr_sq);
    }
  }
  PSYNC();
}

// ---------------------------------------------------------------------------
// Cell plans of a level visit. When the multigrid variables are in shared
// memory and every colour of a level has at most one cell per thread, each
// thread forms once per visit, for its red and its black cell, the cell
// address and the first source and kind of each ghost neighbour, and keeps
// them in its two shared-memory plan slots through the half-sweeps (and the
// residual/restriction) of that visit. The values computed are those of
// p_sweep / p_fr; only the address work moves out of the phases.

// Value of a ghost neighbour from its first source v0 and the cell's own
// value vo, its neighbour across the box va and along the side vb.
template <class T>
__device__ __forceinline__ T ghost_eval(T v0, int kind, T vo, T va, T vb, double V) {
  const T vrb = T(0.5) * v0 + vo - T(0.25) * (va + vb);
  const T vw = kind == GK_NEG ? -vo : T(2 * V) - vo;
  return kind == GK_COPY ? v0 : (kind == GK_RB ? vrb : vw);
}

// The four neighbours of the plan's cell (as phi_nbrs; mem: read the ghost
// cells stored in memory instead). The across and along neighbours a ghost
// recipe reads are among the cell's direct neighbours.
template <class T>
__device__ __forceinline__ void plan_nbrs(double V, const T *phi, const int4 &c, int nc, int ncg,
                                          bool mem, T &lx, T &hx, T &ly, T &hy) {
  const int g = c.x, i = c.w & 255, j = (c.w >> 8) & 255;
  const T dlx = phi[g - 1], dhx = phi[g + 1], dly = phi[g - ncg], dhy = phi[g + ncg];
  if (mem) {
    lx = dlx;
    hx = dhx;
    ly = dly;
    hy = dhy;
    return;
  }
  const T vo = phi[g], x0 = phi[c.y], y0 = phi[c.z];
  const T gx = ghost_eval(x0, (c.w >> 16) & 3, vo, i == 1 ? dhx : dlx, (j & 1) ? dhy : dly, V);
  const T gy = ghost_eval(y0, (c.w >> 18) & 3, vo, j == 1 ? dhy : dly, (i & 1) ? dhx : dlx, V);
  lx = i > 1 ? dlx : gx;
  hx = i < nc ? dhx : gx;
  ly = j > 1 ? dly : gy;
  hy = j < nc ? dhy : gy;
}

__device__ __forceinline__ int4 *plan_slots() { return reinterpret_cast<int4 *>(g_dsmem); }
__device__ __forceinline__ double2 *wts_slots() { return reinterpret_cast<double2 *>(g_dsmem + PLAN_DOUBLES); }

struct LevelPlan {
  int bx;    // index of the box record of the thread's cells (-1: none)
  int item;  // cell index within each colour of the box (row-major, nc/2 per row)
};

// Asynchronous 16-byte copies global -> shared (cp.async), used to fetch the
// host-built plans of the next level while the current level's phases run.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const size_t ga = __cvta_generic_to_global(gmem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(ga) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The level index whose plans are being fetched into the slots (-1: none).
// Every thread tracks the same value: the control flow of the multigrid is
// uniform over the block.
struct PlanFetch {
  int li = -1;
};

template <class T>
__device__ __forceinline__ bool plan_fits(const MGV<T> &M, const LvlInfo &L) {
  return M.plans && L.nb * ((L.nc * L.nc) >> 1) <= NTHR;
}

// Forms the thread's two cell plans (colour p = (i + j) & 1). Each thread
// reads only its own slots afterwards, so no barrier is needed.
template <class T>
__device__ __forceinline__ LevelPlan make_level_plan(const RunDev &R, const MGV<T> &M, const LvlInfo &L,
                                                     bool cyl, PlanFetch &pf) {
  LevelPlan P;
  const int half = (L.nc * L.nc) >> 1, hsh = 2 * L.sh - 1, hn = L.nc >> 1;
  const int k = threadIdx.x;
  P.bx = -1;
  P.item = k & (half - 1);
  if (k < L.nb * half) P.bx = L.b0 + (k >> hsh);
  const int blk = R.cplan_blk[L.li];
  if (pf.li >= 0) {
    // a fetch is in flight: let it land (it is this level's plans, or slots
    // about to be overwritten)
    cp_async_wait_all();
    const bool mine = pf.li == L.li;
    pf.li = -1;
    if (mine) return P;
  }
  if (blk >= 0) {
    // plans of this level built on the host at the topology upload
    const size_t o = (size_t)blk * 2 * NTHR + 2 * threadIdx.x;
    plan_slots()[2 * threadIdx.x] = R.cplan[o];
    plan_slots()[2 * threadIdx.x + 1] = R.cplan[o + 1];
    if (cyl) {
      wts_slots()[2 * threadIdx.x] = R.cwts[o];
      wts_slots()[2 * threadIdx.x + 1] = R.cwts[o + 1];
    }
    return P;
  }
  int4 c[2];
  c[0].x = c[1].x = -1;
  if (k < L.nb * half) {
    P.bx = L.b0 + (k >> hsh);
    const BoxRec &B = M.boxes[P.bx];
    const int j = (P.item >> (L.sh - 1)) + 1, m = P.item & (hn - 1);
#pragma unroll
    for (int p = 0; p < 2; p++) c[p] = make_plan(B, L.nc, L.ncg, 2 * m + 2 - ((p + j) & 1), j);
  }
  plan_slots()[2 * threadIdx.x] = c[0];
  plan_slots()[2 * threadIdx.x + 1] = c[1];
  if (cyl && P.bx >= 0) {
    const int gi0 = M.boxes[P.bx].gi0;
#pragma unroll
    for (int p = 0; p < 2; p++) {
      double2 w;
      cyl_weights(gi0 + (c[p].w & 255), w.x, w.y);
      wts_slots()[2 * threadIdx.x + p] = w;
    }
  }
  return P;
}

// Start fetching the host-built plans of level lvl into the slots (each
// thread its own four 16-byte slots), to be taken by make_level_plan. Only
// after the last read of the slots by the current level, which a barrier
// separates from this call.
template <class T>
__device__ __forceinline__ void fetch_level_plan(const RunDev &R, const MGV<T> &M, int lvl, bool cyl,
                                                 PlanFetch &pf) {
  if (lvl < R.min_lvl || lvl > R.max_lvl || pf.li >= 0) return;
  const LvlInfo L = lvl_info(R, lvl);
  const int blk = R.cplan_blk[L.li];
  if (!plan_fits(M, L) || blk < 0) return;
  const size_t o = (size_t)blk * 2 * NTHR + 2 * threadIdx.x;
  cp_async16(&plan_slots()[2 * threadIdx.x], &R.cplan[o]);
  cp_async16(&plan_slots()[2 * threadIdx.x + 1], &R.cplan[o + 1]);
  if (cyl) {
    cp_async16(&wts_slots()[2 * threadIdx.x], &R.cwts[o]);
    cp_async16(&wts_slots()[2 * threadIdx.x + 1], &R.cwts[o + 1]);
  }
  cp_async_commit();
  pf.li = L.li;
}

// One red-black half-sweep `it` from the cell plans (p_sweep).
template <class T>
__device__ __forceinline__ void plan_sweep(const RunDev &R, const MGV<T> &M, const LvlInfo &L,
                                           const LevelPlan &P, int it, bool mem) {
  const int4 c = plan_slots()[2 * threadIdx.x + (it & 1)];
  if (c.x >= 0) {
    T *phi = M.phi;
    T lx, hx, ly, hy;
    plan_nbrs(M.V, phi, c, L.nc, L.ncg, mem, lx, hx, ly, hy);
    const T r = M.rhs[c.x], dx2 = T(L.dr * L.dr);
    if (R.coord == 1) {
      const double2 w = wts_slots()[2 * threadIdx.x + (it & 1)];
      phi[c.x] = T(0.25) * (T(w.x) * lx + T(w.y) * hx + hy + ly - dx2 * r);
    } else {
      phi[c.x] = T(0.25) * (hx + lx + hy + ly - dx2 * r);
    }
  }
  __syncthreads();
}

// Residual of both cells of the plan, restricted with phi into the parent
// (p_fr with fill, without leaf_rhs and store_res). The 2x2 block of cells
// (2ii-1..2ii, 2jj-1..2jj) belongs to the threads of items (2jj-2) hn + ii-1
// (cells (2ii-1, 2jj-1) and (2ii, 2jj-1)) and that item + hn (cells
// (2ii, 2jj) and (2ii-1, 2jj)), which are in the same warp; the first adds
// the four in the order of box_rstr_lpl.
template <class T>
__device__ __forceinline__ void plan_fr(const RunDev &R, const MGV<T> &M, const LvlInfo &L,
                                        const LevelPlan &P, int lvl) {
  T *phi = M.phi, *tmp = M.tmp;
  const T inv_dr_sq = T(1 / (L.dr * L.dr));
  T res[2] = {0, 0}, ph[2] = {0, 0};
#pragma unroll
  for (int p = 0; p < 2; p++) {
    const int4 c = plan_slots()[2 * threadIdx.x + p];
    if (c.x < 0) continue;
    T lx, hx, ly, hy;
    plan_nbrs(M.V, phi, c, L.nc, L.ncg, false, lx, hx, ly, hy);
    const T v = phi[c.x];
    T lap;
    if (R.coord == 1) {
      const double2 w = wts_slots()[2 * threadIdx.x + p];
      lap = (T(w.x) * lx + T(w.y) * hx + ly + hy - T(4) * v) * inv_dr_sq;
    } else {
      lap = inv_dr_sq * (lx + hx + ly + hy - T(4) * v);
    }
    res[p] = M.rhs[c.x] - lap;
    ph[p] = v;
  }
  const int hn = L.nc >> 1;
  // from the item one row up: its even cell (2ii, 2jj) and odd cell (2ii-1, 2jj)
  const T r11 = __shfl_down_sync(0xffffffffu, res[0], hn);
  const T r01 = __shfl_down_sync(0xffffffffu, res[1], hn);
  const T p11 = __shfl_down_sync(0xffffffffu, ph[0], hn);
  const T p01 = __shfl_down_sync(0xffffffffu, ph[1], hn);
  const int row = P.item >> (L.sh - 1);  // j - 1
  if (P.bx >= 0 && (row & 1) == 0) {
    const BoxRec &B = M.boxes[P.bx];
    const int ii = (P.item & (hn - 1)) + 1, jj = (row >> 1) + 1;
    const int pncg = R.lv_nc[lvl - 1 - R.min_lvl] + 2;
    const int d = B.pbase + (B.o0 + ii) + pncg * (B.o1 + jj);
    tmp[d] = T(0.25) * (res[0] + res[1] + r01 + r11);
    phi[d] = T(0.25) * (ph[0] + ph[1] + p01 + p11);
  }
  fill_phi_loop(R, M, L, false);
  __syncthreads();
}

// Grid mode: levels with few cells would spend more time in grid barriers
// than in work, so a run of consecutive phases on such levels goes to block 0
// of the group alone, behind block barriers, while the other blocks wait at
// the grid barrier that ends the section. local_top: the highest level L <=
// max_lvl such that every level min_lvl..L has at most R.local_cells cells
// (min_lvl - 1: none; always none outside grid mode).
__device__ __forceinline__ int local_top(const RunDev &R, int max_lvl) {
  int lc = R.min_lvl - 1;
  if (!kGrid || s_grp.size == 1) return lc;
  for (int lvl = R.min_lvl; lvl <= max_lvl; lvl++) {
    const int li = lvl - R.min_lvl;
    const int cells = (R.bx_off[li + 1] - R.bx_off[li]) * R.lv_nc[li] * R.lv_nc[li];
    if (cells > R.local_cells) break;
    lc = lvl;
  }
  return lc;
}
// Start of a one-block section: true on block 0, which then runs as a group
// of one (its writes are published, and the others' reads ordered, by the
// grid barrier of local_end).
__device__ __forceinline__ bool local_begin() {
  if (!kGrid) return true;
  if (s_grp.rank != 0) return false;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_grp.size = 1;
    s_grp.nth = NTHR;
  }
  __syncthreads();
  return true;
}
// End of the section on every block of a group of `size`.
__device__ __forceinline__ void local_end(int size) {
  if (!kGrid) return;
  if (s_grp.rank == 0) {
    __syncthreads();
    if (threadIdx.x == 0) {
      s_grp.size = size;
      s_grp.nth = size * NTHR;
    }
  }
  grid_sync();
}

// mg$D_fas_vcycle (m_aX_mg.f90:208-254), set_residual handled by the caller.
// Phases per level: down: 4 half-sweeps, residual/restriction (+ ghost fill),
// coarse ghost fill + rhs; base: 2 n_cycle_base half-sweeps + ghost fill;
// up: correction, 4 half-sweeps, ghost fill. In grid mode the levels up to
// local_top run on one block (the down, base and up phases of those levels
// are consecutive).
template <class T>
__device__ __forceinline__ void vcycle_body(const RunDev &R, const MGV<T> &M, int max_lvl, bool stale_base,
                                            PlanFetch &pf, int after) {
  const int min_lvl = R.min_lvl;
  const bool cyl = R.coord == 1;
  // grid mode: the levels min_lvl..lc run on block 0 alone (the others wait
  // at the barrier of local_end); each level's code appears once
  const int lc = local_top(R, max_lvl);
  const int size = s_grp.size;
  bool work = true;
  for (int lvl = max_lvl; lvl >= min_lvl + 1; lvl--) {
    if (lvl == lc) work = local_begin();
    if (!work) continue;
    const LvlInfo L = lvl_info(R, lvl);
    if (plan_fits(M, L)) {
      const LevelPlan P = make_level_plan(R, M, L, cyl, pf);
      #pragma unroll 1
      for (int it = 1; it <= M.sw_down; it++) plan_sweep(R, M, L, P, it, false);
      plan_fr(R, M, L, P, lvl);
    } else {
      for (int it = 1; it <= M.sw_down; it++) p_sweep(R, M, lvl, it, false);
      p_fr(R, M, lvl, true, false, false);
    }
    fetch_level_plan(R, M, lvl - 1, cyl, pf);
    p_fc(R, M, lvl - 1, true);
  }
  if (lc == min_lvl) work = local_begin();
  if (work) {
    const LvlInfo L = lvl_info(R, min_lvl);
    if (plan_fits(M, L)) {
      const LevelPlan P = make_level_plan(R, M, L, cyl, pf);
      #pragma unroll 1
      for (int it = 1; it <= M.sw_base; it++) plan_sweep(R, M, L, P, it, stale_base && it == 1);
    } else {
      for (int it = 1; it <= M.sw_base; it++) p_sweep(R, M, min_lvl, it, stale_base && it == 1);
    }
    fetch_level_plan(R, M, min_lvl < max_lvl ? min_lvl + 1 : after, cyl, pf);
    p_fill(R, M, min_lvl);
  }
  for (int lvl = min_lvl + 1; lvl <= max_lvl; lvl++) {
    if (lvl == lc + 1 && lc >= min_lvl) {
      local_end(size);
      work = true;
    }
    if (!work) continue;
    const LvlInfo L = lvl_info(R, lvl);
    if (plan_fits(M, L)) {
      const LevelPlan P = make_level_plan(R, M, L, cyl, pf);
      p_correct(R, M, lvl, false, true);
      #pragma unroll 1
      for (int it = 1; it <= M.sw_up; it++) plan_sweep(R, M, L, P, it, false);
    } else {
      p_correct(R, M, lvl, false, true);
      for (int it = 1; it <= M.sw_up; it++) p_sweep(R, M, lvl, it, false);
    }
    fetch_level_plan(R, M, lvl < max_lvl ? lvl + 1 : after, cyl, pf);
    p_fill(R, M, lvl);
  }
  if (lc == max_lvl && lc >= min_lvl) local_end(size);
}

// The FP64 V-cycle is inlined into its caller; the FP32 one (mixed form) is
// kept out of line. Measured against the alternatives: with both inlined the
// kernels that contain both forms spilled several times more, with both out
// of line the FP64 step was 5% slower.
template <class T>
__device__ __forceinline__ void p_vcycle(const RunDev &R, const MGV<T> &M, int max_lvl, bool stale_base,
                                         PlanFetch &pf, int after) {
  vcycle_body<T>(R, M, max_lvl, stale_base, pf, after);
}
template <>
__device__ __noinline__ void p_vcycle<float>(const RunDev &R, const MGV<float> &M, int max_lvl, bool stale_base,
                                             PlanFetch &pf, int after) {
  vcycle_body<float>(R, M, max_lvl, stale_base, pf, after);
}

// mg$D_fas_fmg, m_aX_mg.f90:163-202. leaf_rhs: compute the space charge of
// the leaves where it is first needed (compute_fld). Inlined into each
// caller, so that the multigrid variables' descriptor M stays in registers.
template <class T>
__device__ __forceinline__ void p_fmg_in(const RunDev &R, const MGV<T> &M, bool set_residual, bool first_call,
                         bool leaf_rhs) {
  const int min_lvl = R.min_lvl, max_lvl = R.max_lvl;
  if (first_call) {
    for (int lvl = max_lvl; lvl >= min_lvl + 1; lvl--) p_init_level(R, M, lvl, leaf_rhs);
  } else {
    // set_coarse_phi_rhs for lvl = max..min+1 (:414-447)
    for (int lvl = max_lvl; lvl >= min_lvl + 1; lvl--) {
      p_fr(R, M, lvl, lvl == max_lvl, leaf_rhs, true);
      p_fc(R, M, lvl - 1, false);
    }
  }
  PlanFetch pf;
  // grid mode: the FMG's levels up to local_top, whose V-cycles touch only
  // those levels, on block 0 alone
  const int lc = local_top(R, max_lvl);
  const int size = s_grp.size;
  bool work = true;
  if (lc >= min_lvl) work = local_begin();
  for (int lvl = min_lvl; lvl <= max_lvl; lvl++) {
    if (lvl == lc + 1 && lc >= min_lvl) {
      local_end(size);
      work = true;
    }
    if (!work) continue;
    p_correct(R, M, lvl, true, lvl > min_lvl);
    p_vcycle(R, M, lvl, first_call && lvl == min_lvl, pf, lvl + 1);
    if (set_residual && lvl == max_lvl) p_residual_all(R, M, lvl);
  }
  if (lc == max_lvl && lc >= min_lvl) local_end(size);
  if (pf.li >= 0) cp_async_wait_all();
}

// Copy the multigrid variables of every box between device memory and the
// compact shared-memory arrays (in: to shared memory). All slots of all
// levels form one flat range; a thread moves two slots (three variables
// each) per round, loading all six values before storing any.
template <class T>
__device__ void stage_mg(const RunDev &R, const MGV<T> &M, T *g0, T *g1, T *g2, bool in) {
  T *g[3] = {g0, g1, g2};
  T *s[3] = {M.phi, M.rhs, M.tmp};
  auto level_slots = [&](int li) {
    const int ncg = R.lv_nc[li] + 2;
    return (R.bx_off[li + 1] - R.bx_off[li]) * ncg * ncg;
  };
  int li = 0, lo = 0, hi = level_slots(0);
  // slot k (not below the previous call's k): source and destination index
  auto slot_at = [&](int k, int &src, int &dst) {
    while (k >= hi) {
      if (++li >= R.nlev) return false;
      lo = hi;
      hi = lo + level_slots(li);
    }
    const int ncg = R.lv_nc[li] + 2, per = ncg * ncg, t = k - lo;
    const BoxRec &B = M.boxes[R.bx_off[li] + t / per];
    const int c = t % per;
    src = in ? B.gbase + c : B.base + c;
    dst = in ? B.base + c : B.gbase + c;
    return true;
  };
  T *const *from = in ? g : s;
  T *const *to = in ? s : g;
  for (int k = threadIdx.x;; k += 2 * NTHR) {
    int a0, d0, a1 = 0, d1 = 0;
    if (!slot_at(k, a0, d0)) break;
    const bool two = slot_at(k + NTHR, a1, d1);
    T v0[3], v1[3];
#pragma unroll
    for (int v = 0; v < 3; v++) {
      v0[v] = from[v][a0];
      if (two) v1[v] = from[v][a1];
    }
#pragma unroll
    for (int v = 0; v < 3; v++) {
      to[v][d0] = v0[v];
      if (two) to[v][d1] = v1[v];
    }
  }
  __syncthreads();
}


// mg$D_set_box_tag (afivo/src/m_aX_mg.f90:673-712) for every box of a
// dielectric run: the box is treated with the eps operators when its eps
// (interior, ghost and corner cells) is not identically 1 -- varying, or
// constant and different from 1. The reference tags a box at its first
// multigrid use; eps is set when a box is created (set_box_eps) and not
// changed afterwards, so tagging every box at every solve gives the same
// tags. One warp per box.
__device__ void p_set_tags(const RunDev &R) {
  const double *eps = VAR(R, I_EPS);
  const int warp = TID() >> 5, lane = threadIdx.x & 31, nwarp = NTH() >> 5;
  for (int li = 0; li < R.nlev; li++) {
    const int ncg = R.lv_nc[li] + 2, per = ncg * ncg;
    const int b0 = R.bx_off[li], nb = R.bx_off[li + 1] - b0;
    for (int b = warp; b < nb; b += nwarp) {
      const int base = R.boxes[b0 + b].gbase;
      double mn = eps[base], mx = mn;
      double ln = R.has_lsf ? R.lsf[base] : 0.0, lx = ln;
      for (int c = lane; c < per; c += 32) {
        const double v = eps[base + c];
        mn = dmin(mn, v);
        mx = dmax(mx, v);
        if (R.has_lsf) {
          const double w = R.lsf[base + c];
          ln = dmin(ln, w);
          lx = dmax(lx, w);
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        mn = dmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        ln = dmin(ln, __shfl_xor_sync(0xffffffffu, ln, o));
        lx = dmax(lx, __shfl_xor_sync(0xffffffffu, lx, o));
      }
      if (lane == 0) {
        // mg$D_set_box_tag: level set first, eps tags override it
        const bool deps = mx > mn, ceps = !deps && (mn < 1 || mn > 1);
        const bool is_lsf = R.has_lsf && ln * lx < 0;
        R.tags[base / SLOT] = (deps || ceps) ? TAG_DIEL : (is_lsf ? TAG_LSF : TAG_NORMAL);
      }
    }
  }
  PSYNC();
}

// mg$D_fas_fmg in shared memory when the tree fits (the three variables,
// the box records and the parent-box list), else in device memory. A
// dielectric run always takes the device-memory path, whose phases apply the
// eps operators to the boxes tagged dielectric.
template <class F>
__device__ __forceinline__ void mg_staged(const RunDev &R, const F &body);

// The solves run by mg_staged, as function objects whose bodies are inlined
// into both branches (shared-memory and device-memory variables), so that
// each copy sees its descriptor M as constants.
struct FmgBody {
  bool set_residual, first_call, leaf_rhs;
  __device__ __forceinline__ void operator()(const RunDev &R, const MGV<double> &M) const {
    p_fmg_in(R, M, set_residual, first_call, leaf_rhs);
  }
};
// mg$D_fas_vcycle(tree, mg, max_lvl, set_residual) on its own
// (afivo/src/m_aX_mg.f90:208-254): valid potential ghost cells on input and
// output; with set_residual the residual of levels min..max_lvl in tmp.
struct VcycleBody {
  int max_lvl;
  bool set_residual;
  __device__ __forceinline__ void operator()(const RunDev &R, const MGV<double> &M) const {
    PlanFetch pf;
    p_vcycle(R, M, max_lvl, false, pf, R.max_lvl + 1);
    if (set_residual) p_residual_all(R, M, max_lvl);
    if (pf.li >= 0) cp_async_wait_all();
  }
};

__device__ void p_fmg(const RunDev &R, bool set_residual, bool first_call, bool leaf_rhs) {
  mg_staged(R, FmgBody{set_residual, first_call, leaf_rhs});
}

__device__ void p_vcycle_alone(const RunDev &R, int max_lvl, bool set_residual) {
  mg_staged(R, VcycleBody{max_lvl, set_residual});
}

// Runs body(M) on the multigrid variables: staged in shared memory when the
// tree fits, else in device memory (dielectric runs always in device memory).
template <class F>
__device__ __forceinline__ void mg_staged(const RunDev &R, const F &body) {
  if (R.diel || R.has_lsf) p_set_tags(R);
  if (R.smem_doubles > 0 && !R.diel && !R.has_lsf) {
    const int S = R.smem_doubles, nbx = R.bx_off[R.nlev], npb = R.pb_off[R.nlev];
    double *base = g_dsmem + PLAN_DOUBLES + (R.coord == 1 ? WTS_DOUBLES : 0);
    BoxRec *sb = reinterpret_cast<BoxRec *>(base + 3 * S);
    int *spb = reinterpret_cast<int *>(sb + nbx);
    {
      const int4 *src = reinterpret_cast<const int4 *>(R.sboxes);
      int4 *dst = reinterpret_cast<int4 *>(sb);
      const int n4 = nbx * (int)(sizeof(BoxRec) / sizeof(int4));
      for (int k = threadIdx.x; k < n4; k += NTHR) dst[k] = src[k];
      for (int k = threadIdx.x; k < npb; k += NTHR) spb[k] = R.pbx[k];
    }
    __syncthreads();
    MGV<double> M{base, base + S, base + 2 * S, sb, spb, true, R.applied_voltage,
                  4, 4, 2 * R.n_cycle_base};
    stage_mg(R, M, VAR(R, MP), VAR(R, MR), VAR(R, MT), true);
    body(R, M);
    stage_mg(R, M, VAR(R, MP), VAR(R, MR), VAR(R, MT), false);
  } else {
    MGV<double> M{VAR(R, MP), VAR(R, MR), VAR(R, MT), R.boxes, R.pbx, false, R.applied_voltage,
                  4, 4, 2 * R.n_cycle_base};
    body(R, M);
  }
}


// ---------------------------------------------------------------------------
// Mixed-precision field solve: defect correction around an FP32 multigrid.
// One pass is
//  1. FP64, levels max..min (p_mx_residual): on leaf cells the space charge
//     rhs = e/eps0 (n_e - n_i) and the residual r = rhs - A phi of the FP64
//     potential, ghost neighbours evaluated from their recipes (as p_fr); on
//     parent cells the restriction of the children's r. phi and rhs are
//     restricted into the parents as update_coarse does (box_rstr_lpl,
//     afivo/src/m_aX_mg.f90:683-705). The correction c starts at 0.
//  2. FP32: multigrid on A c = r with homogeneous wall values (V = 0), either
//     the reference's FMG schedule (mg$D_fas_fmg, :163-202) or a single
//     V-cycle over all levels (mg$D_fas_vcycle, :208-254), with the half-sweep
//     counts of the run's schedule.
//  3. FP64 (p_mx_accumulate): phi += c on every cell of every level, then the
//     ghost cells of phi level by level (fill_gc_phi, :303-316).
// The correction equation is linear and the ghost recipes are affine in the
// potential, so this is one FAS cycle on phi whose smoothing runs in FP32,
// while the residual (which cancels) and the accumulation stay in FP64.

// Step 1 on level lvl, one cell per thread; whole warps iterate together so
// that the restriction can gather a 2x2 quad by warp shuffles (the cells of
// a box are consecutive threads, i fastest, and a quad's rows lie in one
// warp). The lane of the quad's lower-left cell writes the parent cell.
__device__ __noinline__ void p_mx_residual(const RunDev &R, const MGV<float> &M, int lvl) {
  const LvlInfo L = lvl_info(R, lvl);
  const bool down = lvl > R.min_lvl;
  const int pncg = down ? R.lv_nc[lvl - 1 - R.min_lvl] + 2 : 0;
  double *phi = VAR(R, I_PHI), *rhs = VAR(R, I_RHS);
  const double *e = VAR(R, I_ELEC), *pi = VAR(R, I_PION);
  float *ce = M.phi, *cr = M.rhs, *ct = M.tmp;
  const double inv_dr_sq = 1 / (L.dr * L.dr);
  const double fac = UC_ELEM_CHARGE / UC_EPS0;
  const int per = L.nc * L.nc, n = L.nb * per, nw = (n + 31) & ~31;
  for (int k = TID(), nt_ = NTH(); k < nw; k += nt_) {
    const bool act = k < n;
    const int b = L.b0 + (act ? k >> (2 * L.sh) : 0);
    const BoxRec &B = R.boxes[b];  // device-memory slots (phi, rhs, densities)
    const BoxRec &S = M.boxes[b];  // slots of the FP32 arrays
    const int t = k & (per - 1), i = (t & (L.nc - 1)) + 1, j = (t >> L.sh) + 1;
    const int g = B.base + i + L.ncg * j, sc = S.base + i + L.ncg * j;
    double res = 0, ph = 0, rh = 0;
    if (act) {
      if (B.flags & CF_PARENT) {
        // the children's residual, restricted into cr on the finer level
        rh = rhs[g];
        res = (double)cr[sc];
      } else {
        // leaves get the space charge; a box in neither list (on level
        // lvls_max, whose lists are never rebuilt) keeps its stored rhs, as
        // residual_box of the FP64 solve reads it
        if (B.flags & CF_LEAF) {
          rh = fac * (e[g] - pi[g]);
          rhs[g] = rh;
        } else {
          rh = rhs[g];
        }
        res = rh - lap_at(R, R.applied_voltage, (const double *)phi, B, L.nc, L.ncg, i, j, inv_dr_sq);
        cr[sc] = (float)res;
      }
      ph = phi[g];
      ce[sc] = 0.0f;
      ct[sc] = 0.0f;
    }
    if (down) {
      const unsigned FULL = 0xffffffffu;
      const double r1 = __shfl_down_sync(FULL, res, 1), r2 = __shfl_down_sync(FULL, res, L.nc),
                   r3 = __shfl_down_sync(FULL, res, L.nc + 1);
      const double p1 = __shfl_down_sync(FULL, ph, 1), p2 = __shfl_down_sync(FULL, ph, L.nc),
                   p3 = __shfl_down_sync(FULL, ph, L.nc + 1);
      const double h1 = __shfl_down_sync(FULL, rh, 1), h2 = __shfl_down_sync(FULL, rh, L.nc),
                   h3 = __shfl_down_sync(FULL, rh, L.nc + 1);
      if (act && (i & 1) && (j & 1)) {
        const int o = (B.o0 + (i + 1) / 2) + pncg * (B.o1 + (j + 1) / 2);
        cr[S.pbase + o] = (float)(0.25 * (res + r1 + r2 + r3));
        phi[B.pbase + o] = 0.25 * (ph + p1 + p2 + p3);
        rhs[B.pbase + o] = 0.25 * (rh + h1 + h2 + h3);
      }
    }
  }
  // side ghosts of c and of its tmp start at zero (consistent with c = 0 and V = 0)
  const int pg = 4 * L.nc, ng = L.nb * pg;
  for (int k = TID(), nt_ = NTH(); k < ng; k += nt_) {
    const BoxRec &S = M.boxes[L.b0 + (k >> (L.sh + 2))];
    const int r = k & (pg - 1), side = r >> L.sh, kk = (r & (L.nc - 1)) + 1;
    const int dim = side >> 1, gx = (side & 1) ? L.nc + 1 : 0;
    const int d = S.base + (dim == 0 ? gx + L.ncg * kk : kk + L.ncg * gx);
    ce[d] = 0.0f;
    ct[d] = 0.0f;
  }
  PSYNC();
}

__device__ void p_mx_accumulate(const RunDev &R, const MGV<float> &M) {
  double *phi = VAR(R, I_PHI);
  for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
    const LvlInfo L = lvl_info(R, lvl);
    const int per = L.nc * L.nc, n = L.nb * per;
    for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
      const int b = L.b0 + (k >> (2 * L.sh));
      const int t = k & (per - 1), i = (t & (L.nc - 1)) + 1, j = (t >> L.sh) + 1;
      const int loc = i + L.ncg * j;
      phi[R.boxes[b].base + loc] += (double)M.phi[M.boxes[b].base + loc];
    }
  }
  PSYNC();
  // the FP64 ghost fill of phi on every level in one phase (phi_ghost_flat:
  // no level waits for the coarser level's fill)
  for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
    const LvlInfo L = lvl_info(R, lvl);
    const int per = 4 * L.nc, n = L.nb * per;
    for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
      const BoxRec &B = R.boxes[L.b0 + (k >> (L.sh + 2))];
      const int r = k & (per - 1), side = r >> L.sh, kk = (r & (L.nc - 1)) + 1;
      const double v = phi_ghost_flat(R.applied_voltage, (const double *)phi, B, L.nc, L.ncg, side, kk);
      const int dim = side >> 1, gx = (side & 1) ? L.nc + 1 : 0;
      phi[B.base + (dim == 0 ? gx + L.ncg * kk : kk + L.ncg * gx)] = v;
    }
  }
  PSYNC();
}

// The mixed-precision solve of compute_fld (see above): the FP32 arrays are
// in shared memory when the tree fits (mx_smem floats per variable), else in
// the run's FP32 storage cc32. The FP64 potential and rhs stay in device
// memory: staging them too (with the FP32 arrays) was measured slower, the
// copies in and out costing more than the residual and accumulation save.
__device__ void p_solve_mixed(const RunDev &R) {
  MGV<float> M;
  if (R.mx_smem > 0) {
    const int S = R.mx_smem, nbx = R.bx_off[R.nlev], npb = R.pb_off[R.nlev];
    float *base = reinterpret_cast<float *>(g_dsmem + PLAN_DOUBLES + (R.coord == 1 ? WTS_DOUBLES : 0));
    BoxRec *sb = reinterpret_cast<BoxRec *>(base + 3 * S);
    int *spb = reinterpret_cast<int *>(sb + nbx);
    const int4 *src = reinterpret_cast<const int4 *>(R.sboxes);
    int4 *dst = reinterpret_cast<int4 *>(sb);
    const int n4 = nbx * (int)(sizeof(BoxRec) / sizeof(int4));
    for (int k = threadIdx.x; k < n4; k += NTHR) dst[k] = src[k];
    for (int k = threadIdx.x; k < npb; k += NTHR) spb[k] = R.pbx[k];
    __syncthreads();
    M = MGV<float>{base, base + S, base + 2 * S, sb, spb, true, 0.0, R.mx_sw_down, R.mx_sw_up,
                   R.mx_sw_base};
  } else {
    const size_t n = (size_t)R.capacity * SLOT;
    M = MGV<float>{R.cc32, R.cc32 + n, R.cc32 + 2 * n, R.boxes, R.pbx, false, 0.0, R.mx_sw_down,
                   R.mx_sw_up, R.mx_sw_base};
  }
  PlanFetch pf;
  for (int pass = 0; pass < R.mx_n_corr; pass++) {
    for (int lvl = R.max_lvl; lvl >= R.min_lvl; lvl--) p_mx_residual(R, M, lvl);
    // the plans that follow the last V-cycle of a pass: those of the next
    // pass's first V-cycle (fetched while the FP64 phases run), or none
    const int next = pass + 1 < R.mx_n_corr ? (R.mx_fmg ? R.min_lvl : R.max_lvl) : R.max_lvl + 1;
    if (R.mx_fmg) {
      for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
        p_correct(R, M, lvl, true, lvl > R.min_lvl);
        p_vcycle(R, M, lvl, false, pf, lvl < R.max_lvl ? lvl + 1 : next);
      }
    } else {
      p_vcycle(R, M, R.max_lvl, false, pf, next);
    }
    p_mx_accumulate(R, M);
  }
  if (pf.li >= 0) cp_async_wait_all();
}
// a$D_gc_tree(iv, a$D_gc_interp[_lim], a$D_gc_neumann) for one or two
// variables, levels ascending (m_aX_gc.f90:28-46, 90-330)
__device__ void p_gc_den(const RunDev &R, int iv0, int iv1, bool lim) {
  // grid mode: the small coarse levels (filled first) on block 0 alone
  const int lc = local_top(R, R.max_lvl);
  const int size = s_grp.size;
  bool work = true;
  if (lc >= R.min_lvl) work = local_begin();
  for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
    if (lvl == lc + 1 && lc >= R.min_lvl) {
      local_end(size);
      work = true;
    }
    if (!work) continue;
    const LvlInfo L = lvl_info(R, lvl);
    const int per = 4 * L.nc, n = L.nb * per;
    for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
      const BoxRec &B = R.boxes[L.b0 + (k >> (L.sh + 2))];
      const int r = k & (per - 1), side = r >> L.sh, kk = (r & (L.nc - 1)) + 1;
      const int dim = side >> 1, gx = (side & 1) ? L.nc + 1 : 0;
      const int d = B.base + (dim == 0 ? gx + L.ncg * kk : kk + L.ncg * gx);
      // both variables' ghost values are formed before either is written
      double g[2];
#pragma unroll
      for (int w = 0; w < 2; w++) {
        const int iv = w == 0 ? iv0 : iv1;
        if (iv >= 0) g[w] = den_ghost_sl(VAR(R, iv), B, L.nc, L.ncg, side, kk, lim);
      }
#pragma unroll
      for (int w = 0; w < 2; w++) {
        const int iv = w == 0 ? iv0 : iv1;
        if (iv >= 0) VAR(R, iv)[d] = g[w];
      }
    }
    PSYNC();
  }
  if (lc == R.max_lvl && lc >= R.min_lvl) local_end(size);
}

// a$D_restrict_tree for one or two variables, levels descending
// (afivo/src/m_aX_restrict.f90:54-142; cylindrical weights :95-113 with the
// radius evaluated at the child-local index [i, j] as in :104)
__device__ void p_restrict(const RunDev &R, int iv0, int iv1) {
  const bool cyl = R.coord == 1;
  // grid mode: the small coarse levels (restricted last) on block 0 alone
  const int lc = local_top(R, R.max_lvl);
  const int top = min(lc, R.max_lvl - 1);
  const bool loc = lc >= R.min_lvl && top >= R.min_lvl;
  const int size = s_grp.size;
  bool work = true;
  for (int lvl = R.max_lvl - 1; lvl >= R.min_lvl; lvl--) {
    if (loc && lvl == top) work = local_begin();
    if (!work) continue;
    const LvlInfo L = lvl_info(R, lvl);
    const int li = lvl - R.min_lvl;
    const int *pb = R.pbx + R.pb_off[li];
    const int npb = R.pb_off[li + 1] - R.pb_off[li];
    const int cg = R.lv_nc[li + 1] + 2;
    const int per = L.nc * L.nc, n = npb * per;
    for (int k = TID(), nt_ = NTH(); k < n; k += nt_) {
      const BoxRec &P = R.boxes[pb[k >> (2 * L.sh)]];
      const int t = k & (per - 1), ic = (t & (L.nc - 1)) + 1, jc = (t >> L.sh) + 1;
      int q = 0, i = ic, j = jc;
      if (P.ch[1] != 0) {  // four children, each covering a quadrant
        const int h = L.nc >> 1;
        const int qx = ic > h, qy = jc > h;
        q = qx + 2 * qy;
        i = ic - qx * h;
        j = jc - qy * h;
      }
      const int src = P.ch[q] + (2 * i - 1) + cg * (2 * j - 1);
      const int d = P.base + ic + L.ncg * jc;
      // the children's values of both variables are read before either
      // parent value is written
      double v[2][4];
#pragma unroll
      for (int w = 0; w < 2; w++) {
        const int iv = w == 0 ? iv0 : iv1;
        if (iv < 0) continue;
        const double *x = VAR(R, iv);
        v[w][0] = x[src];
        v[w][1] = x[src + 1];
        v[w][2] = x[src + cg];
        v[w][3] = x[src + cg + 1];
      }
#pragma unroll
      for (int w = 0; w < 2; w++) {
        const int iv = w == 0 ? iv0 : iv1;
        if (iv < 0) continue;
        const double a = v[w][0], b = v[w][1], c = v[w][2], dd = v[w][3];
        if (cyl) {
          const double dr16 = 0.0625 * P.dr;
          const double r = P.r0 + (i - 0.5) * P.dr;
          const double rfac = dr16 / r;
          VAR(R, iv)[d] = (0.25 - rfac) * (a + c) + (0.25 + rfac) * (b + dd);
        } else {
          VAR(R, iv)[d] = 0.25 * (a + b + c + dd);
        }
      }
    }
    PSYNC();
  }
  if (loc) local_end(size);
}

// Field of one face from the potential (fld_from_pot, src/streamer_2d.f90:
// 346-381): g is the cell on the high side, s the stride to the low side,
// pos the face index along its direction (1..nc+1).
__device__ __forceinline__ double face_fld(const double *phi, const double *eps, int g, int s,
                                           int pos, int nc, double inv_dr) {
  if (pos == 1) return 2 * inv_dr * (phi[g - s] - phi[g]) * eps[g - s] / (eps[g] + eps[g - s]);
  if (pos == nc + 1) return 2 * inv_dr * (phi[g - s] - phi[g]) * eps[g] / (eps[g] + eps[g - s]);
  return inv_dr * (phi[g - s] - phi[g]);
}

// fld_from_pot on every box in one phase (each cell writes its low faces and,
// on the high box edges, the high faces; |E| from its four faces), then the
// |E| ghost fill a$D_gc_tree(i_fld, a$D_gc_interp, a$D_gc_neumann). A thread
// takes two cells per round, all levels in one flat range, and loads both
// before it stores either.
__device__ __noinline__ void p_fld_from_pot(const RunDev &R) {
  const double *phi = VAR(R, I_PHI), *eps = VAR(R, I_EPS);
  double *fld = VAR(R, I_FLD);
  CellCursor cur = cell_cursor(R);
  const int nth = NTH();
  for (int k = TID();; k += 2 * nth) {
    int li[2], b[2], ci[2], cj[2];
    bool ok[2];
    ok[0] = cell_at(R, cur, k, li[0], b[0], ci[0], cj[0]);
    ok[1] = ok[0] && cell_at(R, cur, k + nth, li[1], b[1], ci[1], cj[1]);
    if (!ok[0]) break;
    double f[2][4];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      if (!ok[u]) continue;
      const int nc = R.lv_nc[li[u]], ncg = nc + 2, i = ci[u], j = cj[u];
      const double inv_dr = 1 / R.lv_dr[li[u]];
      const int g = R.boxes[b[u]].base + i + ncg * j;
      f[u][0] = face_fld(phi, eps, g, 1, i, nc, inv_dr);
      f[u][1] = face_fld(phi, eps, g + 1, 1, i + 1, nc, inv_dr);
      f[u][2] = face_fld(phi, eps, g, ncg, j, nc, inv_dr);
      f[u][3] = face_fld(phi, eps, g + ncg, ncg, j + 1, nc, inv_dr);
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      if (!ok[u]) continue;
      const int nc = R.lv_nc[li[u]], ncg = nc + 2, i = ci[u], j = cj[u];
      const int base = R.boxes[b[u]].base, id = base / SLOT;
      double *fxf = FX(R, F_FLD, id), *fyf = FY(R, F_FLD, id);
      fxf[fxi(i, j, nc)] = f[u][0];
      if (i == nc) fxf[fxi(nc + 1, j, nc)] = f[u][1];
      fyf[fyi(i, j, nc)] = f[u][2];
      if (j == nc) fyf[fyi(i, nc + 1, nc)] = f[u][3];
      const double sx = f[u][0] + f[u][1], sy = f[u][2] + f[u][3];
      fld[base + i + ncg * j] = sqrt(0.25 * (sx * sx) + 0.25 * (sy * sy));
    }
  }
  PSYNC();
  p_gc_den(R, I_FLD, -1, false);
}

// compute_fld, src/streamer_2d.f90:307-343 (one FMG cycle)
__device__ void p_compute_fld(const RunDev &R, bool no_guess) {
  p_fmg(R, false, no_guess, true);
  p_fld_from_pot(R);
}
// compute_fld of the mixed form: defect-correction solve, FP64 field
__device__ void p_compute_fld_mixed(const RunDev &R) {
  p_solve_mixed(R);
  p_fld_from_pot(R);
}

// Whole-array copy / average over every slot (unused slots included; their
// contents are never read).
// Four slots per thread and round, all loads before the stores.
__device__ void copy_var(const RunDev &R, int from, int to) {
  const size_t n = (size_t)R.capacity * SLOT;
  const double *a = R.cc + (size_t)from * n;
  double *b = R.cc + (size_t)to * n;
  const size_t nth = NTH();
  for (size_t k = TID(); k < n; k += 4 * nth) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (k + u * nth < n) v[u] = a[k + u * nth];
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (k + u * nth < n) b[k + u * nth] = v[u];
  }
  PSYNC();
}
// average_dens, src/streamer_2d.f90:492-496; both densities, two slots per
// thread and round, all loads before the stores
__device__ void average_dens(const RunDev &R) {
  const size_t n = (size_t)R.capacity * SLOT;
  double *x0 = R.cc, *x1 = R.cc + n;
  const double *o0 = R.cc + 2 * n, *o1 = R.cc + 3 * n;
  const size_t nth = NTH();
  for (size_t k = TID(); k < n; k += 2 * nth) {
    const size_t k1 = k + nth;
    const bool two = k1 < n;
    const double a0 = x0[k], b0 = o0[k], a1 = x1[k], b1 = o1[k];
    double c0 = 0, d0 = 0, c1 = 0, d1 = 0;
    if (two) {
      c0 = x0[k1];
      d0 = o0[k1];
      c1 = x1[k1];
      d1 = o1[k1];
    }
    x0[k] = 0.5 * (a0 + b0);
    x1[k] = 0.5 * (a1 + b1);
    if (two) {
      x0[k1] = 0.5 * (c0 + d0);
      x1[k1] = 0.5 * (c1 + d1);
    }
  }
  PSYNC();
}

// ---------------------------------------------------------------------------
// Reductions and refinement flags.

__device__ void dt_reductions(const RunDev &R);


// a$D_tree_max_cc / _min_cc over leaves (afivo/src/m_aX_utils.f90:559-619)
__device__ void dt_reductions(const RunDev &R) {
  __shared__ double red[3][NTHR / 32];
  const int *ids;
  int n;
  list_range(R, 1, R.min_lvl, R.max_lvl, ids, n);
  double mx = -1.7976931348623157e308, mn = 1.7976931348623157e308,
         me = -1.7976931348623157e308;
  box_loop(ids, n, [&](int id, int t) {
    const BoxMeta &m = R.meta[id];
    const int nc = m.nc;
    if (t >= nc * nc) return;
    const int c = ((t & (nc - 1)) + 1) + (nc + 2) * ((t >> (31 - __clz(nc))) + 1);
    double f = CC(R, I_FLD, id)[c];
    mx = dmax(mx, f);
    mn = dmin(mn, f);
    me = dmax(me, CC(R, I_ELEC, id)[c]);
  });
  for (int o = 16; o > 0; o >>= 1) {
    mx = dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = dmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    me = dmax(me, __shfl_xor_sync(0xffffffffu, me, o));
  }
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) { red[0][w] = mx; red[1][w] = mn; red[2][w] = me; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < NTHR / 32; k++) {
      mx = dmax(mx, red[0][k]);
      mn = dmin(mn, red[1][k]);
      me = dmax(me, red[2][k]);
    }
    mx = dmax(red[0][0], mx);
    mn = dmin(red[1][0], mn);
    me = dmax(red[2][0], me);
    if (kGrid && s_grp.size > 1) {
      // grid mode: each block's values, combined by the lead after a barrier
      // (max and min are exact: any order gives the same result)
      double *g = s_grp.red + 4 * s_grp.rank;
      g[0] = mx;
      g[1] = mn;
      g[2] = me;
    }
  }
  if (kGrid && s_grp.size > 1) {
    grid_sync();
    if (LEAD()) {
      for (int r = 1; r < s_grp.size; r++) {
        const double *g = s_grp.red + 4 * r;
        mx = dmax(mx, g[0]);
        mn = dmin(mn, g[1]);
        me = dmax(me, g[2]);
      }
    }
  }
  if (LEAD()) {
    R.scal[0] = mx;
    R.scal[1] = mn;
    R.scal[2] = me;
    if (!isfinite(mx) || !isfinite(mn) || !isfinite(me)) atomicExch(R.status, A5G_ENONFINITE);
  }
  PSYNC();
}

// GM_dist_line (src/m_geom.f90:29-46), 2D, with gfortran's NORM2
// Step size of the next block of the device-driven loop: get_max_dt
// (src/streamer_2d.f90:271-303, cyl :281-314) from the leaf reductions, with
// the same operations in the same order as the host's a5g_get_max_dt (table
// columns at a location, IEEE + - * / only), then the loop's exit tests
// (src/streamer_2d.f90:72-75): the run stays active unless dt < 1e-14 or
// time > end time.
__device__ void block_dt(const RunDev &R) {
  dt_reductions(R);
  if (LEAD()) {
    const double max_fld = R.scal[0], min_fld = R.scal[1], max_dns = R.scal[2];
    const double eps_mach = 2.220446049250313e-16;
    const double dr_min = R.dr_min;
    const double mobility = col_at<double>(R, C_MOB, get_loc<double>(R, max_fld));
    const double max_mobility = col_at<double>(R, C_MOB, get_loc<double>(R, min_fld));
    const double diff_coeff = col_at<double>(R, C_DIF, get_loc<double>(R, max_fld));
    const double alpha = col_at<double>(R, C_ALPHA, get_loc<double>(R, max_fld));
    const double dt_cfl = dr_min / (mobility * max_fld);
    const double dt_dif = 0.25 * (dr_min * dr_min) / diff_coeff;
    const double dns = R.coord == 1 ? dmax(eps_mach, max_dns) : max_dns;
    const double dt_drt = UC_EPS0 / (UC_ELEM_CHARGE * max_mobility * dns);
    const double dt_alpha = 1 / dmax(mobility * max_fld * alpha, eps_mach);
    double m = dmin(dmin(1 / (1 / dt_cfl + 1 / dt_dif), dt_alpha), R.dt_max);
    if (R.use_drt) m = dmin(m, dt_drt);
    const double dt = 0.5 * m;
    R.blk[0] = dt;
    R.blk[3] = (R.blk[3] != 0.0 && !(dt < 1e-14) && !(R.blk[1] > R.blk[2])) ? 1.0 : 0.0;
  }
  PSYNC();
}

__device__ double dist_line(double x, double y, const double r0[2], const double r1[2]) {
  double line_len2 = 0, temp = 0;
  line_len2 += (r1[0] - r0[0]) * (r1[0] - r0[0]);
  line_len2 += (r1[1] - r0[1]) * (r1[1] - r0[1]);
  temp += (x - r0[0]) * (r1[0] - r0[0]);
  temp += (y - r0[1]) * (r1[1] - r0[1]);
  double v0, v1;
  if (temp <= 0.0) { v0 = x - r0[0]; v1 = y - r0[1]; }
  else if (temp >= line_len2) { v0 = x - r1[0]; v1 = y - r1[1]; }
  else {
    double p0 = r0[0] + temp / line_len2 * (r1[0] - r0[0]);
    double p1 = r0[1] + temp / line_len2 * (r1[1] - r0[1]);
    v0 = x - p0;
    v1 = y - p1;
  }
  return norm2_2(v0, v1);
}

// set_ref_flags on every box of levels 1..max_lvl (src/streamer_2d.f90:177-216,
// cyl :190-227). One warp per box (levels >= 1 have nc = 8: two cells/lane).
__device__ void ref_flags(const RunDev &R, double time) {
  for (int id = TID(), nt_ = NTH(); id < R.capacity; id += nt_) R.flags[id] = INT_MIN + 1;
  PSYNC();
  const int *ids;
  int n;
  list_range(R, 0, 1, R.max_lvl, ids, n);
  const int w = TID() / 32, l = threadIdx.x % 32, nw = NTH() / 32;
  for (int b = w; b < n; b += nw) {
    const int id = ids[b];
    const BoxMeta &m = R.meta[id];
    const int nc = m.nc, ncg = nc + 2;
    double mr = 0.0, mf = -1.7976931348623157e308;
    for (int c = l; c < nc * nc; c += 32) {
      int k = (c % nc + 1) + ncg * (c / nc + 1);
      mr = dmax(mr, fabs(CC(R, I_RHS, id)[k]));
      mf = dmax(mf, CC(R, I_FLD, id)[k]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mr = dmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
      mf = dmax(mf, __shfl_xor_sync(0xffffffffu, mf, o));
    }
    if (l == 0 && R.uniform_lvl > 0) {
      // uniformly refined mesh: refine below the level, keep the rest
      R.flags[id] = m.lvl < R.uniform_lvl ? 1 : 0;
    } else if (l == 0) {
      int flag = INT_MIN + 1;
      double dr2 = m.dr * m.dr;
      double crv_phi = dr2 * mr;
      double alpha = col_at(R, C_ALPHA, get_loc(R, mf));
      double adx = m.dr * alpha;
      if (adx < 0.1 && m.dr < 2.0e-5) flag = -1;
      if (adx < 0.1 && crv_phi < 4.0 && m.dr < 5.0e-5) flag = -1;
      if (time < R.ref_init_time) {
        double boxlen = m.nc * m.dr;
        double cx = m.r0 + 0.5 * m.nc * m.dr, cy = m.r1 + 0.5 * m.nc * m.dr;
        for (int s = 0; s < R.n_seeds; s++) {
          double dist = dist_line(cx, cy, R.seed_r0[s], R.seed_r1[s]);
          if (dist - R.seed_width[s] < boxlen && m.dr > 0.2 * R.seed_width[s]) flag = 1;
        }
      }
      if (adx > 1.0 && crv_phi > R.crv_refine) flag = 1;
      R.flags[id] = flag;
    }
  }
  PSYNC();
}

// prolong_to_new_boxes, src/streamer_2d.f90:592-617, with a$D_prolong1_to
// (afivo/src/m_aX_prolong.f90:99-191) and set_box_eps (:250-266).
__device__ void prolong_new(const RunDev &R) {
  const bool cyl = R.coord == 1;
  for (int li = 0; li < R.nlev; li++) {
    const int *ids = R.new_lists + R.new_off[li];
    const int n = R.new_off[li + 1] - R.new_off[li];
    if (n == 0) continue;
    box_loop(ids, n, [&](int id, int t) {
      const BoxMeta &m = R.meta[id];
      const int nc = m.nc, ncg = nc + 2, hnc = nc >> 1;
      const BoxMeta &pm = R.meta[m.parent];
      const int pg = pm.nc + 2;
      if (t < hnc * hnc) {
        int ii = t % hnc + 1, jj = t / hnc + 1;
        int o0, o1;
        child_offset(m, -1, o0, o1);
        int i_c = ii + o0, j_c = jj + o1, i_f = 2 * ii - 1, j_f = 2 * jj - 1;
        const int vars[3] = {I_ELEC, I_PION, I_PHI};
        for (int v = 0; v < 3; v++) {
          const double *p = CC(R, vars[v], m.parent);
          double *b = CC(R, vars[v], id);
          const int pc = i_c + pg * j_c;
          double f0 = 0.5 * p[pc];
          double flx = 0.25 * p[pc - 1], fhx = 0.25 * p[pc + 1];
          double fly = 0.25 * p[pc - pg], fhy = 0.25 * p[pc + pg];
          b[i_f + ncg * j_f] = f0 + flx + fly + 0.0;
          b[(i_f + 1) + ncg * j_f] = f0 + fhx + fly + 0.0;
          b[i_f + ncg * (j_f + 1)] = f0 + flx + fhy + 0.0;
          b[(i_f + 1) + ncg * (j_f + 1)] = f0 + fhx + fhy + 0.0;
        }
      }
      double *eps = CC(R, I_EPS, id);
      for (int c = t; c < ncg * ncg; c += GT) {
        int i = c % ncg, j = c / ncg;
        double x = m.r0 + (i - 0.5) * m.dr, y = m.r1 + (j - 0.5) * m.dr;
        double rel = (cyl ? x : y) / R.domain_len_z;
        eps[c] = rel < 0.25 ? R.epsilon_diel : 1.0;
      }
    });
    PSYNC();
    box_loop(ids, n, [&](int id, int t) {
      gc_box(R, id, t, I_ELEC, GC_LIM);
      gc_box(R, id, t, I_PION, GC_LIM);
      gc_box(R, id, t, I_PHI, GC_PHI);
    });
    PSYNC();
  }
}

// ---------------------------------------------------------------------------
// Photoionization: set_photoionization (src/streamer_cyl.f90:572-617) and
// PH_set_src_2d with use_cyl and a constant absorption level
// (src/m_photons.f90:207-436).
//
// The reference runs the photon loops in OpenMP regions whose outcome
// depends on the team (every thread draws from its own generator, seeded
// from the master by PRNG_t%init, fosito/m_random.f90:44-55; loops use the
// static schedule; photon numbers are taken in a critical section). Here
// the team has R.ph_team threads, photons are numbered thread by thread and
// the per-thread partial sums of a$D_tree_sum_cc are added in thread order:
// one of the executions the reference takes with that many threads.
//
// Three launches: ph_source (one block: production rate, sum, photon
// creation, numbering), a5g_photon_kernel (many blocks: absorption of each
// thread's chunk of photons and the count per absorbing cell), ph_deposit
// (one block, at the start of the step: the source term per cell, ghost
// cells and prolongation). The deposit of the reference adds the same value
// frac_in_tbl / (fac 2 pi dr^2 r) once per photon to a cleared cell, in
// photon order; with every addend equal, that sum depends only on the
// count, so the device counts photons with integer atomics and forms the
// same sequential sum per cell.

// mzran (fosito/m_random.f90:58-66). Default integers wrap on overflow, as
// in the reference's gfortran x86-64 build.
__device__ __forceinline__ int mz_int4(int st[4]) {
  int rr = (int)((unsigned)st[0] - (unsigned)st[2]);
  if (rr < 0) rr = (int)((unsigned)rr + MZ_M);
  st[0] = st[1];
  st[1] = st[2];
  st[2] = rr;
  st[3] = (int)(69069u * (unsigned)st[3] + 1013904243u);
  return (int)((unsigned)rr + (unsigned)st[3]);
}
// uni_01 (fosito/m_random.f90:75-80)
__device__ __forceinline__ double mz_uni01(int st[4]) { return 0.5 + 0x1p-32 * (double)mz_int4(st); }

// x mod m for any 64-bit x (here a row of a jump matrix times a state),
// from 2^31 = m + 69: two folds x -> (x mod 2^31) + 69 floor(x / 2^31) bring
// x below 2^31 + 69 * 2^9 < 2m, one conditional subtraction finishes.
__device__ __forceinline__ unsigned mz_mod(unsigned long long x) {
  x = (x & 0x7fffffffull) + 69ull * (x >> 31);
  x = (x & 0x7fffffffull) + 69ull * (x >> 31);
  return (unsigned)(x >= MZ_M ? x - MZ_M : x);
}

// Advance the master generator by k draws. While s1, s2, s3 all lie in
// [0, m) a draw maps (s1, s2, s3) to (s2, s3, s1 - s3 mod m), a linear map
// mod m, and s4 to 69069 s4 + 1013904243 mod 2^32; J[b] holds both maps for
// 2^b draws. Outside that range (a seed set by the caller) the draws are
// stepped one by one until the state enters it; it then stays there.
__device__ __forceinline__ bool mz_clean(const int st[4]) {
  return st[0] >= 0 && st[0] < (int)MZ_M && st[1] >= 0 && st[1] < (int)MZ_M && st[2] >= 0 &&
         st[2] < (int)MZ_M;
}
// One jump (a clean state stays clean).
__device__ __forceinline__ void mz_apply(int st[4], const MzJump &j) {
  const unsigned long long v0 = (unsigned)st[0], v1 = (unsigned)st[1], v2 = (unsigned)st[2];
  unsigned int n[3];
#pragma unroll
  for (int r = 0; r < 3; r++)
    n[r] = mz_mod((unsigned long long)j.m[3 * r] * v0 + (unsigned long long)j.m[3 * r + 1] * v1 +
                  (unsigned long long)j.m[3 * r + 2] * v2);
  st[0] = (int)n[0];
  st[1] = (int)n[1];
  st[2] = (int)n[2];
  st[3] = (int)(j.a * (unsigned)st[3] + j.c);
}
__device__ void mz_advance(int st[4], unsigned long long k, const MzJump *J) {
  while (k > 0 && !mz_clean(st)) {
    mz_int4(st);
    k--;
  }
  for (int b = 0; k != 0 && b < MZ_NJUMP; b++, k >>= 1)
    if (k & 1) mz_apply(st, J[b]);
}
// Advance by k draws where J[pre] is the jump of exactly k draws: one
// application from a clean state, mz_advance otherwise (a fresh seed).
__device__ __forceinline__ void mz_advance_pre(int st[4], unsigned long long k, const MzJump *J, int pre) {
  if (mz_clean(st)) mz_apply(st, J[pre]);
  else mz_advance(st, k, J);
}

// libgomp's static schedule without a chunk size: thread c of W gets the
// iterations [lo, lo + len) of n (n and W below 2^31).
__device__ __forceinline__ void static_chunk(long long n, long long W, long long c, long long &lo,
                                             long long &len) {
  const unsigned un = (unsigned)n, uw = (unsigned)W;
  unsigned q = un / uw, t = un - q * uw;
  if ((unsigned long long)c < t) {
    q++;
    t = 0;
  }
  lo = (long long)q * c + t;
  len = q;
}

constexpr double PI_DP = 3.141592653589793;   // acos(-1.0_dp)
constexpr double TWOPI_DP = 6.283185307179586; // 2 * acos(-1.0_dp)

// Position of leaf k of level lvl in the leaf lists of all levels.
__device__ __forceinline__ int leaf_pos(const RunDev &R, int lvl, long long k) {
  return R.lv_off[1][lvl - R.min_lvl] - R.lv_off[1][0] + (int)k;
}

// Exclusive prefix sum of two values per lane over a warp, lane order, the
// lane's first value before its second: returns the sums before each and the
// warp total.
__device__ __forceinline__ void warp_scan2(int a, int b, int &ea, int &eb, int &total) {
  const int lane = threadIdx.x & 31;
  int x = a;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const int tot_a = __shfl_sync(0xffffffffu, x, 31);
  ea = x - a;
  int z = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, z, o);
    if (lane >= o) z += y;
  }
  eb = tot_a + z - b;
  total = tot_a + __shfl_sync(0xffffffffu, z, 31);
}

// ph_source: everything up to the photon numbers. Only the generators'
// draws are sequential per team thread; sums and counts run in parallel
// over boxes and cells and are combined in the team's order. Photons are
// numbered team thread by team thread, each thread's boxes in its loop order
// (levels up, then its chunk of the level's leaves), cells in (j, i) order.
// Work arrays (cap = box capacity):
//   ph_part[0, cap)      sum of leaf box k's production, reference order
//   ph_part[cap, 2cap)   team thread c's partial sum
//   ph_ipart[0, cap)     photons of leaf box k, then its first photon number
//   ph_ipart[cap, 2cap)  photons of team thread c, then its first number
//   ph_ipart[2cap, 3cap) boxes of team thread c, then its first box rank
//   ph_ipart[3cap, 4cap) first photon number of the box of rank r
//   ph_ipart[4cap, 5cap) id of the box of rank r
//   ph_u                 the draw of each leaf cell (int4 output)
//   ph_ncr               first photon number of each leaf cell
//   ph_cnt               absorbed photons per cell, zeroed here
__device__ void ph_source(const RunDev &R, double dt, bool has_dt) {
  __shared__ double s_fac;
  __shared__ double s_prod[NTHR / 32][64];
  const bool cyl = R.coord == 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long W = R.ph_team;
  const int cap = R.capacity;
  double *box_sum = R.ph_part, *team_sum = R.ph_part + cap;
  int *box_cnt = R.ph_ipart, *team_cnt = R.ph_ipart + cap, *team_nbx = R.ph_ipart + 2 * cap;
  int *rank_first = R.ph_ipart + 3 * cap, *rank_id = R.ph_ipart + 4 * cap;
  int *draw = reinterpret_cast<int *>(R.ph_u);
  for (size_t k = threadIdx.x; k < (size_t)cap * SLOT; k += NTHR) R.ph_cnt[k] = 0;
  // set_photoi_rate on all leaves (src/streamer_cyl.f90:595-617)
  {
    const int *ids;
    int n;
    list_range(R, 1, R.min_lvl, R.max_lvl, ids, n);
    box_loop(ids, n, [&](int id, int t) {
      const int nc = R.meta[id].nc, ncg = nc + 2;
      if (t >= nc * nc) return;
      const int c = (t % nc + 1) + ncg * (t / nc + 1);
      const double fld = CC(R, I_FLD, id)[c];
      const Loc<double> loc = get_loc(R, fld);
      const double alpha = col_at(R, C_ALPHA, loc);
      const double mobility = col_at(R, C_MOB, loc);
      double tmp = fld * mobility * alpha * CC(R, I_ELEC, id)[c] * R.ph_coeff;
      if (tmp < 0) tmp = 0;
      CC(R, I_PHO, id)[c] = tmp;
    });
  }
  __syncthreads();
  int max_l = 0, max_l1 = 0;
  for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
    const int L = list_n(R, 1, lvl);
    max_l = max(max_l, L);
    if (lvl >= 1) max_l1 = max(max_l1, L);
  }
  const int n_sum = (int)min((long long)max_l, W), n_cr = (int)min((long long)max_l1, W);
  int st0[4];
#pragma unroll
  for (int q = 0; q < 4; q++) st0[q] = R.ph_rng[q];
  // a$D_tree_sum_cc (afivo/src/m_aX_utils.f90:623-680): per leaf box the sum
  // over its cells in the reference's order (sum_2pr_box for cyl), one warp
  // per box; the products are formed in parallel, the additions in order.
  // Meanwhile the threads of the first n_cr team threads draw their
  // generators' uniforms for photon creation (src/m_photons.f90:263-306):
  // team thread c draws once per cell of its boxes, in its loop order, from
  // the generator seeded with the master's draws 4c+1..4c+4.
  {
    const int *ids;
    int n;
    list_range(R, 1, R.min_lvl, R.max_lvl, ids, n);
    for (int k = warp; k < n; k += NTHR / 32) {
      const int id = ids[k];
      const BoxMeta &m = R.meta[id];
      const int nc = m.nc, ncg = nc + 2, nn = nc * nc;
      const double *x = CC(R, I_PHO, id);
      for (int t = lane; t < nn; t += 32) {
        const int i = t % nc + 1, j = t / nc + 1;
        const double v = x[i + ncg * j];
        s_prod[warp][t] = cyl ? v * (m.r0 + (i - 0.5) * m.dr) : v;
      }
      __syncwarp();
      if (lane == 0) {
        double res = 0;
#pragma unroll 8
        for (int t = 0; t < nn; t++) res = res + s_prod[warp][t];
        box_sum[k] = cyl ? res * TWOPI_DP : res;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n_cr; c += NTHR) {
    int st[4] = {st0[0], st0[1], st0[2], st0[3]};
    mz_advance(st, 4ull * (unsigned long long)c, R.ph_jump);
    int rs[4];
#pragma unroll
    for (int q = 0; q < 4; q++) rs[q] = mz_int4(st);
    for (int lvl = 1; lvl <= R.max_lvl; lvl++) {
      long long lo, len;
      static_chunk(list_n(R, 1, lvl), W, c, lo, len);
      const int *lv = list_p(R, 1, lvl);
      for (long long k = lo; k < lo + len; k++) {
        int *u = draw + (size_t)lv[k] * SLOT;
        // leaf boxes on levels >= 1 have NC x NC cells; cell t is (i, j) =
        // (t % NC + 1, t / NC + 1), the reference's loop order
#pragma unroll 8
        for (int t = 0; t < NC * NC; t++) u[t] = mz_int4(rs);
      }
    }
  }
  // team thread c: fac_l * box sum over its static chunk of each level
  for (int c = threadIdx.x; c < n_sum; c += NTHR) {
    double my = 0;
    for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
      long long lo, len;
      static_chunk(list_n(R, 1, lvl), W, c, lo, len);
      const double dr = R.lv_dr[lvl - R.min_lvl], fac = dr * dr;
      for (long long k = lo; k < lo + len; k++) my = my + fac * box_sum[leaf_pos(R, lvl, k)];
    }
    team_sum[c] = my;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0;
#pragma unroll 8
    for (int c = 0; c < n_sum; c++) total = total + team_sum[c];
    double fac = R.ph_num_photons / (total + 2.220446049250313e-16);
    if (has_dt) fac = dt < fac ? dt : fac;
    s_fac = fac;
  }
  __syncthreads();
  const double fac = s_fac;
  // photons per cell and their numbers within each box, one warp per box
  {
    const int *ids;
    int n;
    list_range(R, 1, 1, R.max_lvl, ids, n);
    const int pos0 = n > 0 ? leaf_pos(R, 1, 0) : 0;
    for (int k = warp; k < n; k += NTHR / 32) {
      const int id = ids[k];
      const BoxMeta &m = R.meta[id];
      const double dr2 = m.dr * m.dr;
      const double *x = CC(R, I_PHO, id);
      const int *u = draw + (size_t)id * SLOT;
      int cnt[2], cell[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int t = lane + 32 * h;
        const int i = t % NC + 1, j = t / NC + 1;
        cell[h] = i + (NC + 2) * j;
        double tmp;
        if (cyl) tmp = fac * 2 * PI_DP * (m.r0 + (i - 0.5) * m.dr) * x[cell[h]] * dr2;
        else tmp = fac * x[cell[h]] * dr2;
        const double fl = floor(tmp);
        int n_create = 0;
        if (fl >= 0 && fl < 1.0e9) n_create = (int)fl;
        else atomicExch(R.status, A5G_ENONFINITE);
        // uni_01 (fosito/m_random.f90:75-80)
        if (0.5 + 0x1p-32 * (double)u[t] < tmp - n_create) n_create = n_create + 1;
        cnt[h] = n_create;
      }
      int e0, e1, tot;
      warp_scan2(cnt[0], cnt[1], e0, e1, tot);
      int *first = R.ph_ncr + (size_t)id * SLOT;
      first[cell[0]] = e0;
      first[cell[1]] = e1;
      if (lane == 0) box_cnt[pos0 + k] = tot;
    }
  }
  __syncthreads();
  // photons and boxes per team thread
  for (int c = threadIdx.x; c < n_cr; c += NTHR) {
    long long tot = 0;
    int nb = 0;
    for (int lvl = 1; lvl <= R.max_lvl; lvl++) {
      long long lo, len;
      static_chunk(list_n(R, 1, lvl), W, c, lo, len);
      for (long long k = lo; k < lo + len; k++) tot += box_cnt[leaf_pos(R, lvl, k)];
      nb += (int)len;
    }
    team_cnt[c] = (int)min(tot, (long long)INT_MAX);
    team_nbx[c] = nb;
  }
  __syncthreads();
  // photon numbers and box ranks: threads in order
  if (threadIdx.x == 0) {
    long long acc = 0;
    int nbx = 0;
#pragma unroll 8
    for (int c = 0; c < n_cr; c++) {
      const int v = team_cnt[c], b = team_nbx[c];
      team_cnt[c] = (int)min(acc, (long long)INT_MAX);
      team_nbx[c] = nbx;
      acc += v;
      nbx += b;
    }
    if (acc > R.ph_cap) {
      atomicExch(R.status, A5G_ENOMEM);
      acc = 0;
    }
    R.ph_scal->n_used = acc;
    R.ph_scal->n_boxes = nbx;
    R.ph_scal->fac = fac;
    for (int q = 0; q < 4; q++) R.ph_scal->st0[q] = st0[q];
    // the master has given 4W draws to the creation team and gives 4W to
    // the absorption team
    int st[4] = {st0[0], st0[1], st0[2], st0[3]};
    mz_advance_pre(st, 8ull * (unsigned long long)W, R.ph_jump, MZ_JSTEP);
    for (int q = 0; q < 4; q++) R.ph_rng[q] = st[q];
  }
  __syncthreads();
  // first photon number and rank of each box, in its team thread's order
  for (int c = threadIdx.x; c < n_cr; c += NTHR) {
    long long off = team_cnt[c];
    int rank = team_nbx[c];
    for (int lvl = 1; lvl <= R.max_lvl; lvl++) {
      long long lo, len;
      static_chunk(list_n(R, 1, lvl), W, c, lo, len);
      const int *lv = list_p(R, 1, lvl);
      for (long long k = lo; k < lo + len; k++) {
        const int p = leaf_pos(R, lvl, k);
        const int v = box_cnt[p];
        box_cnt[p] = (int)off;
        rank_first[rank] = (int)off;
        rank_id[rank] = lv[k];
        rank++;
        off += v;
      }
    }
  }
  __syncthreads();
  // first photon number of each cell
  {
    const int *ids;
    int n;
    list_range(R, 1, 1, R.max_lvl, ids, n);
    const int pos0 = n > 0 ? leaf_pos(R, 1, 0) : 0;
    const int g = threadIdx.x / GT, t = threadIdx.x % GT;
    for (int b = g; b < n; b += NGRP) {
      const int cell = (t % NC + 1) + (NC + 2) * (t / NC + 1);
      R.ph_ncr[(size_t)ids[b] * SLOT + cell] += box_cnt[pos0 + b];
    }
  }
  __syncthreads();
}

// LT_get_col on the photon table (fosito/m_lookup_table.f90:107-161)
__device__ __forceinline__ double ph_dist(const RunDev &R, double x) {
  double frac = (x - R.ph_xmin) * R.ph_inv_dx;
  int ix;
  double fr;
  if (frac < 2.0e9 && frac > -2.0e9) {
    ix = (int)ceil(frac);
    fr = ix - frac;
  } else {
    ix = frac > 0 ? R.ph_rows : 0;
    fr = 0;
  }
  if (ix < 1) {
    ix = 1;
    fr = 1;
  } else if (ix >= R.ph_rows) {
    ix = R.ph_rows - 1;
    fr = 0;
  }
  return fr * R.ph_tbl[ix - 1] + (1 - fr) * R.ph_tbl[ix];
}

// ph_deposit: clear i_pho on levels 1..max_lvl, the source term from the
// photon counts, then ghost cells and prolongation from the absorption
// level (src/m_photons.f90:358-427).
__device__ void ph_deposit(const RunDev &R) {
  const double fac = R.ph_scal->fac;
  const double tmp = fac * 2 * PI_DP;
  {
    const int *ids;
    int n;
    list_range(R, 0, 1, R.max_lvl, ids, n);
    box_loop(ids, n, [&](int id, int t) {
      const BoxMeta &m = R.meta[id];
      const int ncg = m.nc + 2;
      double *x = CC(R, I_PHO, id);
      const int *cnt = R.ph_cnt + (size_t)id * SLOT;
      for (int c = t; c < ncg * ncg; c += GT) {
        const int k = cnt[c];
        double v = 0;
        if (k > 0) {
          const double r0 = m.r0 + (c % ncg - 0.5) * m.dr;
          const double add = R.ph_frac / (tmp * (m.dr * m.dr) * r0);
          for (int q = 0; q < k; q++) v = v + add;
        }
        x[c] = v;
      }
    });
  }
  PSYNC();
  for (int lvl = max(R.ph_lvl, R.min_lvl); lvl <= R.max_lvl - 1; lvl++) {
    const int *par = list_p(R, 2, lvl);
    const int np = list_n(R, 2, lvl);
    box_loop(par, np, [&](int id, int t) { gc_box(R, id, t, I_PHO, GC_INTERP); });
    PSYNC();
    // a$D_prolong1_from(boxes, id, i_pho, add=.true.), m_aX_prolong.f90:81-191
    box_loop(par, np, [&](int id, int t) {
      const BoxMeta &pm = R.meta[id];
      const int q = t >> 4, cc = t & 15;
      const int cid = pm.ch[q];
      if (cid <= 0) return;
      const BoxMeta &m = R.meta[cid];
      const int nc = m.nc, ncg = nc + 2, hnc = nc >> 1;
      if (cc >= hnc * hnc) return;
      int o0, o1;
      child_offset(m, -1, o0, o1);
      const int ii = cc % hnc + 1, jj = cc / hnc + 1;
      const int i_c = ii + o0, j_c = jj + o1, i_f = 2 * ii - 1, j_f = 2 * jj - 1;
      const int pg = pm.nc + 2;
      const double *p = CC(R, I_PHO, id);
      double *b = CC(R, I_PHO, cid);
      const int pc = i_c + pg * j_c;
      const double f0 = 0.5 * p[pc];
      const double flx = 0.25 * p[pc - 1], fhx = 0.25 * p[pc + 1];
      const double fly = 0.25 * p[pc - pg], fhy = 0.25 * p[pc + pg];
      b[i_f + ncg * j_f] = f0 + flx + fly + b[i_f + ncg * j_f];
      b[(i_f + 1) + ncg * j_f] = f0 + fhx + fly + b[(i_f + 1) + ncg * j_f];
      b[i_f + ncg * (j_f + 1)] = f0 + flx + fhy + b[i_f + ncg * (j_f + 1)];
      b[(i_f + 1) + ncg * (j_f + 1)] = f0 + fhx + fhy + b[(i_f + 1) + ncg * (j_f + 1)];
    });
    PSYNC();
  }
}

// a$D_tree_max_cc / a$D_tree_min_cc / a$D_tree_sum_cc over the interior
// cells of the leaves (afivo/src/m_aX_utils.f90:559-680); result in scal[4].
// kind 0: max, 1: min (exact, so any order gives the reference's value);
// kind 2: the sum as a team of `team` OpenMP threads forms it: thread c adds
// lvl_dr^2 * (box sum) over its static chunk of each level's leaves, levels
// ascending, and the partial sums are added to 0 in thread order. The box sum
// runs over (j, i) in column-major order; the cylindrical form weights each
// cell by its radius and multiplies by 2 pi (sum_2pr_box, :661-678).
__device__ void tree_reduce(const RunDev &R, int iv, int kind, int team) {
  __shared__ double red[NTHR / 32];
  const int *ids;
  int n;
  list_range(R, 1, R.min_lvl, R.max_lvl, ids, n);
  if (kind < 2) {
    const bool mx = kind == 0;
    double v = mx ? -1.7976931348623157e308 : 1.7976931348623157e308;
    box_loop(ids, n, [&](int id, int t) {
      const int nc = R.meta[id].nc;
      if (t >= nc * nc) return;
      const int c = ((t & (nc - 1)) + 1) + (nc + 2) * ((t >> (31 - __clz(nc))) + 1);
      const double x = CC(R, iv, id)[c];
      v = mx ? dmax(v, x) : dmin(v, x);
    });
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, v, o);
      v = mx ? dmax(v, y) : dmin(v, y);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 0; k < NTHR / 32; k++) v = mx ? dmax(v, red[k]) : dmin(v, red[k]);
      R.scal[4] = v;
    }
    __syncthreads();
    return;
  }
  const bool cyl = R.coord == 1;
  const long long W = team;
  int max_l = 0;
  for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) max_l = max(max_l, list_n(R, 1, lvl));
  const int n_busy = (int)min((long long)max_l, W);
  for (int c = threadIdx.x; c < n_busy; c += NTHR) {
    double my = 0;
    for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) {
      long long lo, len;
      static_chunk(list_n(R, 1, lvl), W, c, lo, len);
      const int *lv = list_p(R, 1, lvl);
      const double dr = R.lv_dr[lvl - R.min_lvl], fac = dr * dr;
      for (long long k = lo; k < lo + len; k++) {
        const BoxMeta &m = R.meta[lv[k]];
        const int nc = m.nc, ncg = nc + 2;
        const double *x = CC(R, iv, lv[k]);
        double tmp = 0;
        for (int j = 1; j <= nc; j++)
          for (int i = 1; i <= nc; i++) {
            const double v = x[i + ncg * j];
            tmp = tmp + (cyl ? v * (m.r0 + (i - 0.5) * m.dr) : v);
          }
        if (cyl) tmp = tmp * TWOPI_DP;
        my = my + fac * tmp;
      }
    }
    R.sumbuf[c] = my;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0;
    for (int c = 0; c < n_busy; c++) total = total + R.sumbuf[c];
    R.scal[4] = total;
  }
  __syncthreads();
}

// One full time step, src/streamer_2d.f90:99-127; with deposit, the photon
// source term of this step's photoionization first (src/streamer_cyl.f90:95-97).
// MIXED: the mixed-precision form -- FP32 fluxes, source update and lookups,
// field solves by defect correction around an FP32 multigrid (p_solve_mixed);
// densities, the space charge, the potential, the field and the step size
// stay in FP64.
template <bool MIXED>
__device__ void step(const RunDev &R, double dt, bool deposit) {
  if (deposit) ph_deposit(R);
  {
    const size_t n = (size_t)R.capacity * SLOT;
    const double *e = VAR(R, I_ELEC), *pi = VAR(R, I_PION);
    double *eo = VAR(R, I_ELEC_OLD), *po = VAR(R, I_PION_OLD);
    // two slots per thread and round, all loads before the stores
    const size_t nth = NTH();
    for (size_t k = TID(); k < n; k += 2 * nth) {
      const size_t k1 = k + nth;
      const bool two = k1 < n;
      const double a0 = e[k], b0 = pi[k], a1 = two ? e[k1] : 0.0, b1 = two ? pi[k1] : 0.0;
      eo[k] = a0;
      po[k] = b0;
      if (two) {
        eo[k1] = a1;
        po[k1] = b1;
      }
    }
    PSYNC();
  }
  using T = typename std::conditional<MIXED, float, double>::type;
  for (int stage = 1; stage <= 2; stage++) {
    fluxes_koren<T>(R, dt);
    PSYNC();
    consistent_fluxes(R);
    PSYNC();
    update_solution<T>(R, dt);
    PSYNC();
    p_restrict(R, I_ELEC, I_PION);
    p_gc_den(R, I_ELEC, I_PION, true);
    if (stage == 1) {
      if (MIXED) p_compute_fld_mixed(R);
      else p_compute_fld(R, false);
    }
  }
  average_dens(R);
  if (MIXED) p_compute_fld_mixed(R);
  else p_compute_fld(R, false);
}

__device__ void run_op(const RunDev &R, const Op &op) {
  switch (op.code) {
    case OP_COPY: copy_var(R, op.i0, op.i1); break;
    case OP_FLUXES: fluxes_koren<double>(R, op.d0); PSYNC(); break;
    case OP_CONSISTENT: consistent_fluxes(R); PSYNC(); break;
    case OP_UPDATE: update_solution<double>(R, op.d0); PSYNC(); break;
    case OP_RESTRICT: p_restrict(R, op.i0, -1); break;
    case OP_GC: p_gc_den(R, op.i0, -1, op.i1 == GC_LIM); break;
    case OP_AVERAGE: average_dens(R); break;
    case OP_COMPUTE_FLD: p_compute_fld(R, op.i0 != 0); break;
    case OP_FMG: p_fmg(R, op.i0 != 0, op.i1 != 0, false); break;
    case OP_FLD_FROM_POT: p_fld_from_pot(R); break;
    case OP_DT_RED: dt_reductions(R); break;
    case OP_REF_FLAGS: ref_flags(R, op.d0); break;
    case OP_PROLONG_NEW: prolong_new(R); break;
    case OP_STEP:
    case OP_STEP_MIXED: {
      // i1 = 1: the block's dt and active flag come from the device block state
      double dt = op.d0;
      if (op.i1) {
        if (R.blk[3] == 0.0) break;
        dt = R.blk[0];
      }
      if (op.code == OP_STEP) step<false>(R, dt, op.i0 != 0);
      else step<true>(R, dt, op.i0 != 0);
      if (op.i1 && LEAD()) R.blk[1] = R.blk[1] + dt;
      break;
    }
    case OP_BLOCK_DT: block_dt(R); break;
    case OP_COMPUTE_FLD_MIXED: p_compute_fld_mixed(R); break;
    case OP_PH_SOURCE:
      if (op.i1 && R.blk[3] == 0.0) {
        // inactive run of a device-driven batch: no photons this step
        if (threadIdx.x == 0) R.ph_scal->n_used = 0;
        break;
      }
      ph_source(R, op.i1 ? R.blk[0] : op.d0, op.i0 != 0);
      break;
    case OP_PH_DEPOSIT: ph_deposit(R); break;
    case OP_VCYCLE: p_vcycle_alone(R, op.i0, op.i1 != 0); break;
    case OP_TREE_RED: tree_reduce(R, op.i0, op.i1, op.i2); break;
    case OP_NOP: break;
    default: if (LEAD()) atomicExch(R.status, A5G_EINVAL);
  }
}

// The run descriptor staged in shared memory, and the block's group: a
// single-run launch of g blocks is the group of all its blocks (grid mode
// when g > 1, launched cooperatively so that they are co-resident); in a
// batch every block is a group of its own.
__device__ __forceinline__ void stage_run(const RunDev *src, RunDev &sR, int size, int rank) {
  const int *s = reinterpret_cast<const int *>(src);
  int *d = reinterpret_cast<int *>(&sR);
  for (int k = threadIdx.x; k < (int)(sizeof(RunDev) / sizeof(int)); k += NTHR) d[k] = s[k];
  if (threadIdx.x == 0) {
    s_grp.size = size;
    s_grp.rank = rank;
    s_grp.tid0 = rank * NTHR;
    s_grp.nth = size * NTHR;
    s_grp.bar = src->gbar;
    s_grp.budget = src->gbudget;
    s_grp.status = src->status;
    s_grp.red = src->gred;
  }
  __syncthreads();
}

// One block per run of a batch, or one run on all blocks of the launch.
__global__ void __launch_bounds__(NTHR, 1)
a5g_run_kernel(const RunDev *single, Op single_op, const RunDev *const *runs, const Op *ops) {
  __shared__ RunDev sR;
  if (runs) stage_run(runs[blockIdx.x], sR, 1, 0);
  else stage_run(single, sR, (int)gridDim.x, (int)blockIdx.x);
  Op op = runs ? ops[blockIdx.x] : single_op;
  run_op(sR, op);
}

// One full time step of one run (a5g_step) on the launch's blocks; a kernel
// of its own so that profilers can select the hot launch by name.
__global__ void __launch_bounds__(NTHR, 1) a5g_step_kernel(const RunDev *run, double dt, int deposit) {
  __shared__ RunDev sR;
  stage_run(run, sR, (int)gridDim.x, (int)blockIdx.x);
  step<false>(sR, dt, deposit != 0);
}

// One full time step of one run in the mixed-precision form.
__global__ void __launch_bounds__(NTHR, 1) a5g_step_mixed_kernel(const RunDev *run, double dt,
                                                                 int deposit) {
  __shared__ RunDev sR;
  stage_run(run, sR, (int)gridDim.x, (int)blockIdx.x);
  step<true>(sR, dt, deposit != 0);
}

// Same work as a5g_run_kernel, with each block's run and operation read from
// a descriptor table (the fixed array below).
__global__ void __launch_bounds__(NTHR, 1) a5g_run_kernel_slots(const BatchSlot *slots) {
  __shared__ RunDev sR;
  stage_run(slots[blockIdx.x].run, sR, 1, 0);
  Op op = slots[blockIdx.x].op;
  run_op(sR, op);
}

#if A5G_GRID
// A device-driven batch whose members take several blocks each (the
// members' a5g_set_ctas): block b runs operation ops[k] of run k as rank r of
// its run's group of m blocks, gmap[3 b ..] = {k, r, m}; one cooperative
// launch holds every member's group, each synchronising on its own barrier.
__global__ void __launch_bounds__(NTHR, 1) a5g_batch_map_kernel(const RunDev *const *runs, const Op *ops,
                                                                const int *gmap) {
  __shared__ RunDev sR;
  const int k = gmap[3 * blockIdx.x], r = gmap[3 * blockIdx.x + 1], m = gmap[3 * blockIdx.x + 2];
  stage_run(runs[k], sR, m, r);
  run_op(sR, ops[k]);
}
#endif

#if !A5G_GRID
// Absorption of the photons of one photoionization call (PH_do_absorp,
// src/m_photons.f90:161-205, then the radius, :318-329, and a$D_get_loc at
// the absorption level, :331-344). Thread w of the team absorbs its static
// chunk of the photons in order with its own generator (the master's draws
// 4W + 4w + 1..4 of the call) and counts each photon in its absorbing cell.
// A photon's source cell follows from its number: the last ranked box whose
// first number is not above it, then the last cell of that box whose first
// number is not above it. blockIdx.y selects the run of a batch. The per-box
// geometry and the box ranks are staged in shared memory when they fit
// (ph_smem: bytes available).
__device__ __forceinline__ int ph_cell_index(int t) { return (t % NC + 1) + (NC + 2) * (t / NC + 1); }

__global__ void __launch_bounds__(PH_THREADS, PH_BLOCKS_PER_SM) a5g_photon_kernel(const RunDev *single,
                                                               const RunDev *const *runs,
                                                               const BatchSlot *slots,
                                                               int ph_smem) {
  const RunDev *rp = runs ? runs[blockIdx.y] : slots ? slots[blockIdx.y].run : single;
  // the run's descriptor in shared memory: the photon loop reads its fields
  // after every atomic, which the compiler cannot keep in registers
  __shared__ RunDev sR;
  {
    const int *src = reinterpret_cast<const int *>(rp);
    int *d = reinterpret_cast<int *>(&sR);
    for (int k = threadIdx.x; k < (int)(sizeof(RunDev) / sizeof(int)); k += PH_THREADS) d[k] = src[k];
  }
  __syncthreads();
  const RunDev &R = sR;
  if (!R.ph_enabled) return;
  const long long W = R.ph_team;
  const long long w0 = (long long)blockIdx.x * PH_THREADS;
  if (w0 >= W) return;
  const long long n_used = R.ph_scal->n_used;
  if (n_used == 0) return;
  const int nbx = R.ph_scal->n_boxes, cap = R.capacity;
  const PhBox *tb = R.ph_boxes;
  const int *rank_first = R.ph_ipart + 3 * cap, *rank_id = R.ph_ipart + 4 * cap;
  const size_t need = (size_t)R.n_ids * sizeof(PhBox) + 2 * (size_t)nbx * sizeof(int);
  if (need <= (size_t)ph_smem) {
    PhBox *sb = reinterpret_cast<PhBox *>(g_dsmem);
    int *sf = reinterpret_cast<int *>(sb + R.n_ids), *si = sf + nbx;
    for (int k = threadIdx.x; k < R.n_ids; k += PH_THREADS) sb[k] = R.ph_boxes[k];
    for (int k = threadIdx.x; k < nbx; k += PH_THREADS) {
      sf[k] = rank_first[k];
      si[k] = rank_id[k];
    }
    __syncthreads();
    tb = sb;
    rank_first = sf;
    rank_id = si;
  }
  // Generator of team thread w: the master's state at draw 4W + 4w. One
  // thread jumps the master to the block's first team thread (4W + 4 w0),
  // then every thread jumps from there by 4 threadIdx.x: jumps compose
  // exactly. Both jumps are single precomputed matrices of the run's table.
  __shared__ int s_base[4];
  if (threadIdx.x == 0) {
    int b[4] = {R.ph_scal->st0[0], R.ph_scal->st0[1], R.ph_scal->st0[2], R.ph_scal->st0[3]};
    mz_advance_pre(b, 4ull * (unsigned long long)W + 4ull * (unsigned long long)w0, R.ph_jump,
                   MZ_JBLK + (int)blockIdx.x);
#pragma unroll
    for (int q = 0; q < 4; q++) s_base[q] = b[q];
  }
  __syncthreads();
  const long long w = w0 + threadIdx.x;
  if (w >= W) return;
  long long lo, len;
  static_chunk(n_used, W, w, lo, len);
  if (len == 0) return;
  int st[4] = {s_base[0], s_base[1], s_base[2], s_base[3]};
  mz_advance_pre(st, 4ull * (unsigned long long)threadIdx.x, R.ph_jump, MZ_JTHR + (int)threadIdx.x);
  int rs[4];
#pragma unroll
  for (int q = 0; q < 4; q++) rs[q] = mz_int4(st);
  const int *l1 = list_p(R, 0, 1);
  const int n1 = list_n(R, 0, 1);
  const int lvl_max = R.ph_lvl;
  int sid = 0, scell = 0;
  long long cell_end = -1;  // photons [.., cell_end) come from (sid, scell)
  for (long long p = lo; p < lo + len; p++) {
    if (p >= cell_end) {
      // box: last rank with first <= p
      int a = 0, b = nbx - 1;
      while (a < b) {
        const int mid = (a + b + 1) >> 1;
        if (rank_first[mid] <= p) a = mid;
        else b = mid - 1;
      }
      sid = rank_id[a];
      const long long box_end = a + 1 < nbx ? rank_first[a + 1] : n_used;
      const int *first = R.ph_ncr + (size_t)sid * SLOT;
      int ta = 0, tbb = NC * NC - 1;
      while (ta < tbb) {
        const int mid = (ta + tbb + 1) >> 1;
        if (first[ph_cell_index(mid)] <= p) ta = mid;
        else tbb = mid - 1;
      }
      scell = ph_cell_index(ta);
      cell_end = ta + 1 < NC * NC ? first[ph_cell_index(ta + 1)] : box_end;
    }
    const int si = scell % (NC + 2), sj = scell / (NC + 2);
    const PhBox &S = tb[sid];
    const double x0 = S.r0 + (si - 0.5) * S.dr, y0 = S.r1 + (sj - 0.5) * S.dr;
    const double dist = ph_dist(R, mz_uni01(rs));
    // RNG_t%sphere, fosito/m_random.f90:135-151
    double a, b, ss;
    int tries = 0;
    while (true) {
      a = -1.0 + mz_uni01(rs) * (1.0 - -1.0);
      b = -1.0 + mz_uni01(rs) * (1.0 - -1.0);
      ss = a * a + b * b;
      if (ss <= 1) break;
      if (++tries > 100000) {
        atomicExch(R.status, A5G_ENONFINITE);
        break;
      }
    }
    const double t = sqrt(1 - ss);
    const double sx = 2 * a * t * dist, sy = 2 * b * t * dist, sz = (1 - 2 * ss) * dist;
    const double xo = x0 + sx, yo = y0 + sy, zo = 0.0 + sz;
    const double x = sqrt(xo * xo + zo * zo), y = yo;
    // a$D_get_loc (afivo/src/m_aX_utils.f90:244-299)
    int id = -1;
    for (int k = 0; k < n1; k++) {
      const PhBox &B = tb[l1[k]];
      const double xm = B.r0 + B.dr * B.nc, ym = B.r1 + B.dr * B.nc;
      if (x >= B.r0 && y >= B.r1 && x <= xm && y <= ym) {
        id = l1[k];
        break;
      }
    }
    if (id < 0) continue;
    for (int guard = 0; guard < 64; guard++) {
      const PhBox &B = tb[id];
      if (!(B.lvl < lvl_max && B.ch[0] != 0)) break;
      const double hc = (double)(B.nc >> 1);
      const int i_ch = (x > B.r0 + B.dr * hc ? 1 : 0) + (y > B.r1 + B.dr * hc ? 2 : 0);
      id = B.ch[i_ch];
    }
    const PhBox &B = tb[id];
    const int ix = (int)ceil((x - B.r0) / B.dr), iy = (int)ceil((y - B.r1) / B.dr);
    if (ix < 0 || iy < 0 || ix > B.nc + 1 || iy > B.nc + 1) {
      atomicExch(R.status, A5G_EINVAL);
      continue;
    }
    atomicAdd(R.ph_cnt + (size_t)id * SLOT + ix + (B.nc + 2) * iy, 1);
  }
}
#endif  // !A5G_GRID
