// a5g3 -- the 3D octree form of the device path on sm_100a (see
// include/a5g3.h): uniformly refined octrees of 8^3-cell boxes resident in
// HBM, one kernel per phase over a level's (or the leaves') box list, one
// thread block per box, the whole time step replayed from a CUDA graph.
//
// Arithmetic follows the reference expression by expression (compiled with
// --fmad=false, so every multiply and add is rounded on its own) and gives
// the same doubles as the CPU restatement of src/streamer_3d.f90 and afivo's
// m_a3_* routines.
//
// Memory layout in HBM: cell variable iv of box id is the slot
// cc[iv][id][(nc+2)^3] of SLOT3 = (box_size+2)^3 doubles (i fastest, then j,
// k); face variable f of direction d is fc[d][f][id][FSLOT3]. Box ids index
// slots directly. A box is one thread block: its slot is 8 KB of contiguous
// doubles per variable, read with coalesced loads.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "a5g3.h"

namespace {

constexpr int NC3 = 8;                                  // box_size on levels >= 1
constexpr int G3 = NC3 + 2;
constexpr int SLOT3 = G3 * G3 * G3;                     // 1000 doubles
constexpr int FSLOT3 = (NC3 + 1) * NC3 * NC3;           // 576 doubles
constexpr int NV3 = A5G_N_VAR_CELL, NF3 = A5G_N_VAR_FACE;
enum { I_ELEC = 0, I_PION, I_ELEC_OLD, I_PION_OLD, I_PHI, I_FLD, I_RHS, I_PHO, I_EPS };
enum { F_ELEC = 0, F_FLD };
enum { C_MOB = 0, C_DIF, C_ALPHA, C_ETA };
constexpr int NTH3 = 256;                               // threads per box block
constexpr double UC_EPS0 = 8.8541878176e-12;            // fosito/m_units_constants.f90:201
constexpr double UC_ELEM_CHARGE = 1.6022e-19;           // :202

// Device view of one run, passed by value to every kernel.
struct Run3 {
  double *cc;          // NV3 variables x cap slots
  double *fc;          // 3 directions x NF3 variables x cap face slots
  const int *nc;       // [cap] cells per box edge
  const int *nbr;      // [cap][6] neighbours (lx hx ly hy lz hz), < 0 physical
  const int *chl;      // [cap][8] children
  const int *par;      // [cap] parent
  const int *off;      // [cap][3] offset of the box's cells in its parent (child offset)
  const double *geo;   // [cap][4] r_min[3], dr
  const double *lt;    // transport table, rows x 4, column-major
  const float *lt32;   // its FP32 copy (the mixed form's lookups)
  double *scal;        // device scalars (S_*)
  double *part;        // per-block partial reductions
  long long cap;       // slots (max_id + 1)
  int lt_rows;
  double lt_xmin, lt_inv_dx;
  double voltage;      // applied potential at the high-z wall
  // the levels: ids of level lo + q at ids[lv_off[q] .. + lv_n[q]], lv_nc[q]
  // cells per box edge
  const int *ids;
  int lo, nlev, n_cycle_base;
  int lv_off[16], lv_n[16], lv_nc[16];
  int lv_first[16];    // a level's ids are lv_first .. lv_first + lv_n - 1
};
enum { S_DT = 0, S_RED = 1 };  // scal[0] dt; scal[1..3] reductions; scal[4] tree max/min

__device__ __forceinline__ double *VAR(const Run3 &R, int iv) { return R.cc + (size_t)iv * R.cap * SLOT3; }
__device__ __forceinline__ double *CC(const Run3 &R, int iv, int id) {
  return R.cc + ((size_t)iv * R.cap + id) * SLOT3;
}
__device__ __forceinline__ double *FC(const Run3 &R, int d, int f, int id) {
  return R.fc + (((size_t)d * NF3 + f) * R.cap + id) * FSLOT3;
}
__device__ __forceinline__ int ix3(int g, int i, int j, int k) { return i + g * (j + g * k); }

// gfortran's NORM2 of a 3-vector: scaled sum of squares, the scale raised
// whenever a larger |x| appears
__device__ __forceinline__ double norm2_3(const double x[3]) {
  double scale = 0.0, ssq = 1.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (x[k] != 0.0) {
      const double ax = fabs(x[k]);
      if (scale < ax) {
        const double v = scale / ax;
        ssq = 1.0 + ssq * v * v;
        scale = ax;
      } else {
        const double v = ax / scale;
        ssq += v * v;
      }
    }
  }
  return scale * sqrt(ssq);
}

// The same lookup, limiter and norm in the arithmetic type T of the transport
// (double: the expressions above; float: the mixed form, on the FP32 table).
template <class T>
struct LocT {
  int ix;
  T fr;
};
template <class T>
__device__ __forceinline__ const T *lt_tab(const Run3 &R);
template <>
__device__ __forceinline__ const double *lt_tab<double>(const Run3 &R) { return R.lt; }
template <>
__device__ __forceinline__ const float *lt_tab<float>(const Run3 &R) { return R.lt32; }
template <class T>
__device__ __forceinline__ LocT<T> lt_locT(const Run3 &R, T x) {
  const T frac = (x - T(R.lt_xmin)) * T(R.lt_inv_dx);
  LocT<T> l;
  if (frac < T(2.0e9) && frac > T(-2.0e9)) {
    l.ix = (int)ceil(frac);
    l.fr = T(l.ix) - frac;
  } else {
    l.ix = frac > T(0) ? R.lt_rows : 0;
    l.fr = 0;
  }
  if (l.ix < 1) {
    l.ix = 1;
    l.fr = 1;
  } else if (l.ix >= R.lt_rows) {
    l.ix = R.lt_rows - 1;
    l.fr = 0;
  }
  return l;
}
template <class T>
__device__ __forceinline__ T lt_colT(const Run3 &R, int col, const LocT<T> &l) {
  const T *c = lt_tab<T>(R) + (size_t)R.lt_rows * col;
  return l.fr * c[l.ix - 1] + (T(1) - l.fr) * c[l.ix];
}
template <class T>
__device__ __forceinline__ T koren_mlimT(T a, T b) {
  const T sixth = T(1 / 6.0);
  const T aa = a * a, ab = a * b;
  if (ab <= T(0)) return 0;
  if (aa <= T(0.25) * ab) return a;
  if (aa <= T(2.5) * ab) return sixth * (b + 2 * a);
  return b;
}
template <class T>
__device__ __forceinline__ T norm2_3T(const T x[3]) {
  T scale = 0, ssq = 1;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (x[k] != T(0)) {
      const T ax = fabs(x[k]);
      if (scale < ax) {
        const T v = scale / ax;
        ssq = T(1) + ssq * v * v;
        scale = ax;
      } else {
        const T v = ax / scale;
        ssq += v * v;
      }
    }
  }
  return scale * sqrt(ssq);
}
// Densities enter the FP32 fluxes scaled by 2^-40, an exact power of two:
// Koren's limiter and the flux are homogeneous of degree one in the density,
// and the squares of density differences stay inside the float range.
template <class T>
__device__ __forceinline__ T dscale() { return T(1); }
template <>
__device__ __forceinline__ float dscale<float>() { return 0x1p-40f; }

// ---------------------------------------------------------------------------
// a3_tree_copy_cc for two variable pairs at once (elec -> elec_old, pion ->
// pion_old at the start of a step); whole slots, two doubles per thread.
__global__ void k3_copy2(Run3 R, int a0, int b0, int a1, int b1) {
  const size_t n2 = (size_t)R.cap * SLOT3 / 2;
  const double2 *s0 = reinterpret_cast<const double2 *>(VAR(R, a0));
  const double2 *s1 = reinterpret_cast<const double2 *>(VAR(R, a1));
  double2 *d0 = reinterpret_cast<double2 *>(VAR(R, b0));
  double2 *d1 = reinterpret_cast<double2 *>(VAR(R, b1));
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n2; k += (size_t)gridDim.x * blockDim.x) {
    const double2 x = s0[k];
    d0[k] = x;
    if (a1 >= 0) d1[k] = s1[k];
  }
}

// average_dens (src/streamer_3d.f90:557-563): x = 0.5 (x + x_old) for n_e
// and n_i, whole slots.
__global__ void k3_average(Run3 R) {
  const size_t n = (size_t)R.cap * SLOT3;
  double *e = VAR(R, I_ELEC), *p = VAR(R, I_PION);
  const double *eo = VAR(R, I_ELEC_OLD), *po = VAR(R, I_PION_OLD);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    e[k] = 0.5 * (e[k] + eo[k]);
    p[k] = 0.5 * (p[k] + po[k]);
  }
}

// ---------------------------------------------------------------------------
// fluxes_koren (src/streamer_3d.f90:396-554) on one leaf box per block: the
// box's n_e and |E| slots staged in shared memory (coalesced), the second
// ghost layer (a3_gc2_box with sides2_from_nb / a3_gc2_neumann,
// afivo/src/m_aX_gc.f90:407-483, 588-622) read from the neighbour's slot or
// the box's own, then every x, y and z face of the box (3 (nc+1) nc^2).
template <class T>
__global__ void __launch_bounds__(NTH3) k3_fluxes(Run3 R, const int *ids) {
  __shared__ T se[SLOT3], sf[SLOT3];
  const int id = ids[blockIdx.x];
  constexpr int nc = NC3, g = nc + 2, gs = g * g * g;  // the leaves are boxes of levels >= 1
  const T ds = dscale<T>();
  {
    const double *e = CC(R, I_ELEC, id), *f = CC(R, I_FLD, id);
    for (int k = threadIdx.x; k < gs; k += NTH3) {
      se[k] = T(e[k]) * ds;
      sf[k] = T(f[k]);
    }
  }
  __syncthreads();
  const double dt = R.scal[S_DT];
  const T inv_dr = T(1 / R.geo[4 * id + 3]);
  const T fac = T(-0.8 * UC_EPS0 / (UC_ELEM_CHARGE * dt)) * ds;
  const int *nb = R.nbr + 6 * id;
  const int F = (nc + 1) * nc * nc;
  for (int q = threadIdx.x; q < 3 * F; q += NTH3) {
    const int d = q / F, r = q - d * F;
    int i, j, k;
    if (d == 0) {
      i = r % (nc + 1) + 1;
      j = (r / (nc + 1)) % nc + 1;
      k = r / ((nc + 1) * nc) + 1;
    } else if (d == 1) {
      i = r % nc + 1;
      j = (r / nc) % (nc + 1) + 1;
      k = r / (nc * (nc + 1)) + 1;
    } else {
      i = r % nc + 1;
      j = (r / nc) % nc + 1;
      k = r / (nc * nc) + 1;
    }
    // position along the face normal and the cell strides
    const int a = d == 0 ? i : d == 1 ? j : k;
    const int st = d == 0 ? 1 : d == 1 ? g : g * g;
    const int c0 = ix3(g, i, j, k), cm1 = c0 - st;
    const T e0 = se[c0], em1 = se[cm1];
    T em2, ep1;
    // second ghost layer where the stencil leaves the box (a == 1 / nc + 1)
    if (a == 1) {
      const int n = nb[2 * d];
      // c0 is cell 1: the neighbour's cell nc - 1, or own cell 2
      em2 = n > 0 ? T(CC(R, I_ELEC, n)[c0 + (nc - 2) * st]) * ds : se[c0 + st];
    } else {
      em2 = se[c0 - 2 * st];
    }
    if (a == nc + 1) {
      const int n = nb[2 * d + 1];
      // c0 is the ghost cell nc + 1: the neighbour's cell 2, or own cell nc - 1
      ep1 = n > 0 ? T(CC(R, I_ELEC, n)[c0 - (nc - 1) * st]) * ds : se[c0 - 2 * st];
    } else {
      ep1 = se[c0 + st];
    }
    const T fld_avg = T(0.5) * (sf[c0] + sf[cm1]);
    const LocT<T> loc = lt_locT<T>(R, fld_avg);
    const T mobility = lt_colT<T>(R, C_MOB, loc);
    const T diff_coeff = lt_colT<T>(R, C_DIF, loc);
    double *fe = FC(R, d, F_ELEC, id);
    const T fld = T(FC(R, d, F_FLD, id)[r]);
    const T v_drift = -mobility * fld;
    const T gradc = e0 - em1;
    T out;
    if (v_drift < T(0)) {
      const T gradn = ep1 - e0;
      out = v_drift * (e0 - koren_mlimT<T>(gradc, gradn));
      if (out < fac * fld) out = fac * fld;
    } else {
      const T gradp = em1 - em2;
      out = v_drift * (em1 + koren_mlimT<T>(gradc, gradp));
      if (out > fac * fld) out = fac * fld;
    }
    fe[r] = (double)(out - diff_coeff * gradc * inv_dr) / (double)ds;
  }
}

// Side ghosts pushed by the box that owns their value: a cell on face side
// (2d low, 2d+1 high) of box id is the value of the facing side ghost of the
// same-level neighbour there (sides_from_nb, afivo/src/m_aX_gc.f90:368-402),
// or, on a physical side, of the box's own ghost (a3_gc_neumann, :298-330).
// On a uniform octree every side ghost of a level has exactly one such
// writer, so a kernel that computes every box of a level can fill that
// level's side ghosts in the same pass, with the values a3_gc_box reads
// afterwards. (i, j, k) is the cell, v its new value; bc 1: the physical
// sides of the potential (sides_bc_pot, src/streamer_3d.f90:693-715: -phi at
// low z, 2 V - phi at high z, Neumann on x and y), as k3_gc.
__device__ __forceinline__ void push_side_ghosts(const Run3 &R, int iv, int id, int nc, int i, int j, int k,
                                                 double v, int bc = 0) {
  const int g = nc + 2;
  const int c[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (c[d] != 1 && c[d] != nc) continue;
#pragma unroll
    for (int hi = 0; hi < 2; hi++) {
      if (c[d] != (hi ? nc : 1)) continue;
      const int n = R.nbr[6 * id + 2 * d + hi];
      int q[3] = {i, j, k};
      // the neighbour's ghost on its facing side, or the own ghost
      q[d] = n > 0 ? (hi ? 0 : nc + 1) : (hi ? nc + 1 : 0);
      double w = v;
      if (n <= 0 && bc == 1 && d == 2) w = hi ? 2 * R.voltage - v : -v;
      CC(R, iv, n > 0 ? n : id)[ix3(g, q[0], q[1], q[2])] = w;
    }
  }
}

// update_solution (src/streamer_3d.f90:566-615) on one leaf box per block,
// one interior cell per thread and round; then the dielectric conversion
// (eps > 1: n_e moves into n_i). PUSH: also the side ghosts of n_e and n_i
// on the leaves' level (push_side_ghosts; the update reads no ghost cell),
// so that the ghost fill after the restriction covers the coarser levels
// only.
template <class T, bool PUSH>
__global__ void __launch_bounds__(NTH3) k3_update(Run3 R, const int *ids) {
  const int id = ids[blockIdx.x];
  constexpr int nc = NC3, g = nc + 2, n = nc * nc * nc;  // the leaves are boxes of levels >= 1
  const double dt = R.scal[S_DT];
  const T tdt = T(dt);
  const T inv_dr = T(1 / R.geo[4 * id + 3]);
  const double *fx = FC(R, 0, F_ELEC, id), *fy = FC(R, 1, F_ELEC, id), *fz = FC(R, 2, F_ELEC, id);
  double *e = CC(R, I_ELEC, id), *p = CC(R, I_PION, id);
  const double *fld = CC(R, I_FLD, id), *eps = CC(R, I_EPS, id);
  for (int t = threadIdx.x; t < n; t += NTH3) {
    const int i = t % nc + 1, j = (t / nc) % nc + 1, k = t / (nc * nc) + 1;
    const int c = ix3(g, i, j, k);
    const LocT<T> loc = lt_locT<T>(R, T(fld[c]));
    const T alpha = lt_colT<T>(R, C_ALPHA, loc), eta = lt_colT<T>(R, C_ETA, loc);
    const int xl = (i - 1) + (nc + 1) * ((j - 1) + nc * (k - 1));
    const int yl = (i - 1) + nc * ((j - 1) + (nc + 1) * (k - 1));
    const int zl = (i - 1) + nc * ((j - 1) + nc * (k - 1));
    const T x0 = T(fx[xl]), x1 = T(fx[xl + 1]), y0 = T(fy[yl]), y1 = T(fy[yl + nc]), z0 = T(fz[zl]),
            z1 = T(fz[zl + nc * nc]);
    T dflux[3];
    dflux[0] = x0 + x1;
    dflux[1] = y0 + y1;
    dflux[2] = z0 + z1;
    const T src = T(0.5) * norm2_3T<T>(dflux) * (alpha - eta);
    T sflux = x0 - x1;
    sflux = sflux + y0;
    sflux = sflux - y1;
    sflux = sflux + z0;
    sflux = sflux - z1;
    sflux = sflux * inv_dr;
    double ev = e[c] + (double)((src + sflux) * tdt);
    double pv = p[c] + (double)(src * tdt);
    if (eps[c] > 1.0) {
      pv = pv - ev;
      ev = 0;
    }
    e[c] = ev;
    p[c] = pv;
    if (PUSH) {
      push_side_ghosts(R, I_ELEC, id, nc, i, j, k, ev);
      push_side_ghosts(R, I_PION, id, nc, i, j, k, pv);
    }
  }
}

// a3_restrict_box (afivo/src/m_aX_restrict.f90:67-142, 3D) from every box of
// a level to its parent, for up to two variables: each parent cell is 0.125
// times the sum of its eight child cells in column-major order. One block per
// child box; the child's cells land in its octant of the parent (child
// offset), so the blocks write disjoint parent cells.
__global__ void __launch_bounds__(NTH3) k3_restrict(Run3 R, const int *ids, int iv0, int iv1) {
  const int id = ids[blockIdx.x];
  const int nc = R.nc[id], g = nc + 2, hnc = nc >> 1, nh = hnc * hnc * hnc;
  const int p = R.par[id];
  const int pg = R.nc[p] + 2;
  const int *o = R.off + 3 * id;
  for (int t = threadIdx.x; t < 2 * nh; t += NTH3) {
    const int iv = t < nh ? iv0 : iv1;
    if (iv < 0) continue;
    const int u = t < nh ? t : t - nh;
    const int i = u % hnc + 1, j = (u / hnc) % hnc + 1, k = u / (hnc * hnc) + 1;
    const double *c = CC(R, iv, id);
    const int f = ix3(g, 2 * i - 1, 2 * j - 1, 2 * k - 1);
    double s = c[f];
    s = s + c[f + 1];
    s = s + c[f + g];
    s = s + c[f + g + 1];
    s = s + c[f + g * g];
    s = s + c[f + g * g + 1];
    s = s + c[f + g * g + g];
    s = s + c[f + g * g + g + 1];
    CC(R, iv, p)[ix3(pg, o[0] + i, o[1] + j, o[2] + k)] = 0.125 * s;
  }
}

// Ghost cells of the boxes in ids for up to two variables (a3_gc_box,
// afivo/src/m_aX_gc.f90:50-68): the facing layer of a same-level neighbour
// (sides_from_nb, :368-402), or on a physical side the box's own first
// layer: Neumann (a3_gc_neumann, :298-330), or for the potential with
// bc = 1 sides_bc_pot (src/streamer_3d.f90:693-715): Neumann on x and y,
// -phi at low z, 2 V - phi at high z.
// Item t of box id: variable (t < 6 nc^2 ? iv0 : iv1), side, cell.
template <int NCT>
__device__ __forceinline__ void it_gc(const Run3 &R, int id, int t, int iv0, int iv1, int bc) {
  const int nc = NCT ? NCT : R.nc[id], g = nc + 2, per = nc * nc;
  const int iv = t < 6 * per ? iv0 : iv1;
  if (iv < 0) return;
  const int u = t < 6 * per ? t : t - 6 * per;
  const int side = u / per, w = u - side * per;
  const int a = w % nc + 1, b = w / nc + 1;
  const int d = side >> 1;
  const bool low = (side & 1) == 0;
  const int st = d == 0 ? 1 : d == 1 ? g : g * g;
  // the ghost cell and the box's own first cell on that side
  int gcell;
  if (d == 0) gcell = ix3(g, low ? 0 : nc + 1, a, b);
  else if (d == 1) gcell = ix3(g, a, low ? 0 : nc + 1, b);
  else gcell = ix3(g, a, b, low ? 0 : nc + 1);
  const int own = low ? gcell + st : gcell - st;
  double *x = CC(R, iv, id);
  const int n = R.nbr[6 * id + side];
  double v;
  if (n > 0) {
    // the neighbour's cell nc (low side) or 1 (high side)
    v = CC(R, iv, n)[low ? gcell + nc * st : gcell - nc * st];
  } else if (bc == 1 && side == 4) {
    v = -x[own];
  } else if (bc == 1 && side == 5) {
    v = 2 * R.voltage - x[own];
  } else {
    v = x[own];
  }
  x[gcell] = v;
}
__global__ void __launch_bounds__(NTH3) k3_gc(Run3 R, const int *ids, int iv0, int iv1, int bc) {
  const int id = ids[blockIdx.x];
  const int nc = R.nc[id], per = nc * nc;
  // boxes of levels >= 1 with the box size at compile time
  if (nc == NC3)
    for (int t = threadIdx.x; t < 12 * NC3 * NC3; t += NTH3) it_gc<NC3>(R, id, t, iv0, iv1, bc);
  else
    for (int t = threadIdx.x; t < 12 * per; t += NTH3) it_gc<0>(R, id, t, iv0, iv1, bc);
}

// set_init_cond and set_box_eps (src/streamer_3d.f90:217-270) on every cell
// of every box (ghost cells included): background plus seeds
// (GM_dens_line, src/m_geom.f90:29-111), n_i = n_e, phi = 0, eps = 1.
struct Seeds3 {
  int n;
  double bg;
  double r0[8][3], r1[8][3], dens[8], width[8];
  int falloff[8];
};
__device__ double dist_line3(const double r[3], const double *r0, const double *r1) {
  double line_len2 = 0, temp = 0;
  for (int d = 0; d < 3; d++) line_len2 += (r1[d] - r0[d]) * (r1[d] - r0[d]);
  for (int d = 0; d < 3; d++) temp += (r[d] - r0[d]) * (r1[d] - r0[d]);
  double v[3];
  if (temp <= 0.0) {
    for (int d = 0; d < 3; d++) v[d] = r[d] - r0[d];
  } else if (temp >= line_len2) {
    for (int d = 0; d < 3; d++) v[d] = r[d] - r1[d];
  } else {
    for (int d = 0; d < 3; d++) v[d] = r[d] - (r0[d] + temp / line_len2 * (r1[d] - r0[d]));
  }
  return norm2_3(v);
}
__device__ double dens_line3(const double r[3], const double *r0, const double *r1, double width, int falloff) {
  const double dist = dist_line3(r, r0, r1);
  switch (falloff) {
    case 1: {
      const double tmp = dist / width;
      if (tmp > log(0.5 * 1.7976931348623157e308)) return 0;
      return 2 / (1 + exp(tmp));
    }
    case 2: {
      const double x = dist / width;
      return exp(-(x * x));
    }
    case 3: {
      if (dist < width) return 1;
      if (dist < 2 * width) {
        const double temp = dist / width - 1;
        return (1 - (3 * (temp * temp) - 2 * (temp * temp * temp)));
      }
      return 0.0;
    }
    case 4: return dist < width ? 1.0 : 0.0;
    default: return 0;
  }
}
__global__ void __launch_bounds__(NTH3) k3_init(Run3 R, const int *ids, Seeds3 S) {
  const int id = ids[blockIdx.x];
  const int nc = R.nc[id], g = nc + 2, gs = g * g * g;
  const double *geo = R.geo + 4 * id;
  double *e = CC(R, I_ELEC, id), *p = CC(R, I_PION, id), *phi = CC(R, I_PHI, id), *eps = CC(R, I_EPS, id);
  for (int t = threadIdx.x; t < gs; t += NTH3) {
    const int i = t % g, j = (t / g) % g, k = t / (g * g);
    const double xyz[3] = {geo[0] + (i - 0.5) * geo[3], geo[1] + (j - 0.5) * geo[3], geo[2] + (k - 0.5) * geo[3]};
    double v = S.bg;
    for (int s = 0; s < S.n; s++) v = v + S.dens[s] * dens_line3(xyz, S.r0[s], S.r1[s], S.width[s], S.falloff[s]);
    e[t] = v;
    p[t] = v;
    phi[t] = 0;
    eps[t] = 1.0;
  }
}

// ---------------------------------------------------------------------------
// Multigrid (afivo/src/m_aX_mg.f90, 3D Laplacian operators lpl). Each phase
// is a flat loop over the items of one level (cells or slot elements of all
// its boxes, box-major); phase() runs a share of them, so that the same
// code serves a grid of many blocks on the fine levels (k3_phase) and one
// block running a whole sequence of small coarse-level phases behind block
// barriers (k3_coarse).
enum {
  PH_SWEEP = 0,         // a0 = half-sweep number, a1 = read ghosts from memory
  PH_FILL,              // fill_gc_phi: ghost cells of phi (sides_bc_pot)
  PH_RESID_RESTRICT,    // residual and phi restricted to the parents
  PH_COARSE_RHS,        // a0 = copy tmp = phi
  PH_CORR_DIFF,         // tmp = phi - tmp
  PH_CORRECT,           // phi += prolonged correction of the parent
  PH_COPY,              // a0 -> a1, whole slots
  PH_INIT_PHI_RHS,      // phi = 0, rhs restricted to the parents
  PH_RESIDUAL           // tmp = rhs - lpl(phi)
};

struct Lv {
  int first, n, nc;
};
__device__ __forceinline__ Lv lv_of(const Run3 &R, int l) {
  const int q = l - R.lo;
  return Lv{R.lv_first[q], R.lv_n[q], R.lv_nc[q]};
}

// The arrays a multigrid solve works on: the potential, its right-hand side
// and the scratch variable tmp (per-box slots of SLOT3 entries), and the
// potential of the high-z wall. The FP64 solve works on the run's own
// variables with the applied voltage; the mixed form's correction solve on
// FP32 arrays with wall value 0 (its correction equation is homogeneous).
template <class T>
struct MG3 {
  T *phi, *rhs, *tmp;
  double voltage;
};
template <class T>
__device__ __forceinline__ T *SL(T *a, int id) { return a + (size_t)id * SLOT3; }
template <class T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

// mg3_box_lpl (:814-848) at interior cell c of a box's phi slot
template <class T>
__device__ __forceinline__ T lpl3(const T *phi, int c, int g, T inv_dr_sq) {
  T s = phi[c - 1] + phi[c + 1];
  s = s + phi[c - g];
  s = s + phi[c + g];
  s = s + phi[c - g * g];
  s = s + phi[c + g * g];
  return inv_dr_sq * (s - 6 * phi[c]);
}

// The value phi has, after a ghost fill (fill_gc_phi, :358-371), at the
// neighbour of cell c (position a along direction s >> 1, cell stride st)
// across side s: the cell itself inside the box, else the facing cell of
// the same-level neighbour or sides_bc_pot of cell c (src/streamer_3d.f90:
// 693-715). Equal to the ghost cell in memory whenever that was filled after
// the sources last changed.
template <class T>
__device__ __forceinline__ T phi_side(const Run3 &R, const MG3<T> &M, int id, int nc, const T *phi, int c, int s,
                                      int a, int st) {
  const bool hi = s & 1;
  const int cn = hi ? c + st : c - st;
  const int an = hi ? a + 1 : a - 1;
  if (an >= 1 && an <= nc) return phi[cn];
  const int n = R.nbr[6 * id + s];
  if (n > 0) return SL(M.phi, n)[hi ? cn - nc * st : cn + nc * st];
  if (s == 4) return -phi[c];
  if (s == 5) return T(2 * M.voltage) - phi[c];
  return phi[c];
}

// mg3_box_lpl (:814-848) at interior cell (i, j, k) = c of box id, the ghost
// neighbours from their sources (phi_side)
template <class T>
__device__ __forceinline__ T lpl3_src(const Run3 &R, const MG3<T> &M, int id, int nc, const T *phi, int c, int i,
                                      int j, int k, T inv_dr_sq) {
  const int g = nc + 2;
  T s = phi_side(R, M, id, nc, phi, c, 0, i, 1) + phi_side(R, M, id, nc, phi, c, 1, i, 1);
  s = s + phi_side(R, M, id, nc, phi, c, 2, j, g);
  s = s + phi_side(R, M, id, nc, phi, c, 3, j, g);
  s = s + phi_side(R, M, id, nc, phi, c, 4, k, g * g);
  s = s + phi_side(R, M, id, nc, phi, c, 5, k, g * g);
  return inv_dr_sq * (s - 6 * phi[c]);
}

// One cell of a red-black Gauss-Seidel half-sweep `it` of mg3_box_gsrb_lpl
// (:769-811): the cells with (i + j + k + it) even, phi = sixth (sum of the
// six neighbours - dx^2 rhs). A neighbour outside the box is evaluated from
// its source, which equals the ghost fill gsrb_boxes performs after every
// half-sweep (:403-426): the facing cell of the same-level neighbour (of
// the colour not updated here) or, on a physical side, sides_bc_pot of the
// cell itself (read before it is written). mem: read the ghost cells in
// memory instead (the first half-sweep on the base level of a first FMG
// call, whose ghosts the reference leaves as they were).
template <class T>
__device__ __forceinline__ void it_sweep(const Run3 &R, const MG3<T> &M, int id, int nc, int t, int it, int mem) {
  const int g = nc + 2, hn = nc >> 1;
  const int k = t / (nc * hn) + 1, rem = t - (k - 1) * nc * hn;
  const int j = rem / hn + 1, m = rem - (j - 1) * hn;
  const int i = 2 - ((it + j + k) & 1) + 2 * m;
  const int c = ix3(g, i, j, k);
  const double dr = R.geo[4 * id + 3];
  const T dx2 = T(dr * dr);
  const T sixth = T(1 / 6.0);
  T *phi = SL(M.phi, id);
  const int pos[3] = {i, j, k}, st[3] = {1, g, g * g};
  T v[6];
#pragma unroll
  for (int s = 0; s < 6; s++) {
    const int d = s >> 1;
    v[s] = mem ? phi[(s & 1) ? c + st[d] : c - st[d]] : phi_side(R, M, id, nc, phi, c, s, pos[d], st[d]);
  }
  T sum = v[1] + v[0];
  sum = sum + v[3];
  sum = sum + v[2];
  sum = sum + v[5];
  sum = sum + v[4];
  phi[c] = sixth * (sum - dx2 * SL(M.rhs, id)[c]);
}

// update_coarse / set_coarse_phi_rhs, fine part (:430-523), for one parent
// cell u of box id: the residual rhs - lpl(phi) of its eight child cells
// (residual_box, :551-565) and their phi, each summed in column-major order,
// times 0.125 into the parent's tmp and phi (mg3_box_rstr_lpl, :851-893).
// The box's own tmp is left as it was (update_coarse restores it;
// set_coarse_phi_rhs's copy there is overwritten before any read). Ghost
// neighbours come from their sources, so no fill of this level is needed
// before it.
template <class T>
__device__ __forceinline__ void it_resid_restrict(const Run3 &R, const MG3<T> &M, int id, int nc, int u) {
  const int g = nc + 2, hnc = nc >> 1;
  const int i = u % hnc + 1, j = (u / hnc) % hnc + 1, k = u / (hnc * hnc) + 1;
  const double dr = R.geo[4 * id + 3];
  const T inv_dr_sq = T(1 / (dr * dr));
  const T *phi = SL(M.phi, id), *rhs = SL(M.rhs, id);
  const int f = ix3(g, 2 * i - 1, 2 * j - 1, 2 * k - 1);
  const int o8[8] = {0, 1, g, g + 1, g * g, g * g + 1, g * g + g, g * g + g + 1};
  T sr = 0, sp = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int c = f + o8[q];
    const T r = rhs[c] - lpl3_src(R, M, id, nc, phi, c, 2 * i - 1 + (q & 1), 2 * j - 1 + ((q >> 1) & 1),
                                  2 * k - 1 + (q >> 2), inv_dr_sq);
    sr = q == 0 ? r : sr + r;
    sp = q == 0 ? phi[c] : sp + phi[c];
  }
  const int p = R.par[id], pg = R.nc[p] + 2;
  const int *o = R.off + 3 * id;
  const int pc = ix3(pg, o[0] + i, o[1] + j, o[2] + k);
  SL(M.tmp, p)[pc] = T(0.125) * sr;
  SL(M.phi, p)[pc] = T(0.125) * sp;
}

// Coarse part of update_coarse / set_coarse_phi_rhs (:471-485, :514-521) at
// slot element c of parent box id: rhs = lpl(phi) on interior cells, then
// rhs = rhs + tmp on the whole slot (a3_box_add_cc), then with copy tmp =
// phi (a3_box_copy_cc).
template <class T>
__device__ __forceinline__ void it_coarse_rhs(const Run3 &R, const MG3<T> &M, int id, int nc, int c, int copy) {
  const int g = nc + 2;
  const int i = c % g, j = (c / g) % g, k = c / (g * g);
  const bool in = i >= 1 && i <= nc && j >= 1 && j <= nc && k >= 1 && k <= nc;
  const double dr = R.geo[4 * id + 3];
  const T inv_dr_sq = T(1 / (dr * dr));
  const T *phi = SL(M.phi, id);
  T *rhs = SL(M.rhs, id), *tmp = SL(M.tmp, id);
  const T a = in ? lpl3(phi, c, g, inv_dr_sq) : rhs[c];
  rhs[c] = a + tmp[c];
  if (copy) tmp[c] = phi[c];
}

// correct_children (:374-401): on the parent, tmp = phi - tmp (whole slot),
// then mg3_box_corr_lpl (:714-766) on each child cell: phi += 0.25 (c1 + c2x
// + c2y + c2z) of the parent's correction, c1 the closest coarse cell.
template <class T>
__device__ __forceinline__ void it_correct(const Run3 &R, const MG3<T> &M, int id, int nc, int t) {
  const int g = nc + 2;
  const int p = R.par[id], pg = R.nc[p] + 2;
  const int *o = R.off + 3 * id;
  const T *corr = SL(M.tmp, p);
  T *phi = SL(M.phi, id);
  const int i = t % nc + 1, j = (t / nc) % nc + 1, k = t / (nc * nc) + 1;
  const int i1 = o[0] + ((i + 1) >> 1), i2 = i1 + 1 - 2 * (i & 1);
  const int j1 = o[1] + ((j + 1) >> 1), j2 = j1 + 1 - 2 * (j & 1);
  const int k1 = o[2] + ((k + 1) >> 1), k2 = k1 + 1 - 2 * (k & 1);
  T s = corr[ix3(pg, i1, j1, k1)] + corr[ix3(pg, i2, j1, k1)];
  s = s + corr[ix3(pg, i1, j2, k1)];
  s = s + corr[ix3(pg, i1, j1, k2)];
  const int c = ix3(g, i, j, k);
  phi[c] = phi[c] + T(0.25) * s;
}

// init_phi_rhs (:526-549), the restriction of one parent cell's rhs
template <class T>
__device__ __forceinline__ void it_restrict_rhs(const Run3 &R, const MG3<T> &M, int id, int nc, int u) {
  const int g = nc + 2, hnc = nc >> 1;
  const int i = u % hnc + 1, j = (u / hnc) % hnc + 1, k = u / (hnc * hnc) + 1;
  const T *rhs = SL(M.rhs, id);
  const int f = ix3(g, 2 * i - 1, 2 * j - 1, 2 * k - 1);
  T s = rhs[f];
  s = s + rhs[f + 1];
  s = s + rhs[f + g];
  s = s + rhs[f + g + 1];
  s = s + rhs[f + g * g];
  s = s + rhs[f + g * g + 1];
  s = s + rhs[f + g * g + g];
  s = s + rhs[f + g * g + g + 1];
  const int p = R.par[id], pg = R.nc[p] + 2;
  const int *o = R.off + 3 * id;
  SL(M.rhs, p)[ix3(pg, o[0] + i, o[1] + j, o[2] + k)] = T(0.125) * s;
}

// fill_gc_phi (:358-371) for item t of box id: a ghost cell of phi from the
// facing cell of the same-level neighbour or sides_bc_pot
// (src/streamer_3d.f90:693-715: Neumann on x and y, -phi at low z, 2 V - phi
// at high z).
template <class T>
__device__ __forceinline__ void it_fill(const Run3 &R, const MG3<T> &M, int id, int nc, int t) {
  const int g = nc + 2, per = nc * nc;
  const int side = t / per, w = t - side * per;
  const int a = w % nc + 1, b = w / nc + 1;
  const int d = side >> 1;
  const bool low = (side & 1) == 0;
  const int st = d == 0 ? 1 : d == 1 ? g : g * g;
  int gcell;
  if (d == 0) gcell = ix3(g, low ? 0 : nc + 1, a, b);
  else if (d == 1) gcell = ix3(g, a, low ? 0 : nc + 1, b);
  else gcell = ix3(g, a, b, low ? 0 : nc + 1);
  const int own = low ? gcell + st : gcell - st;
  T *x = SL(M.phi, id);
  const int n = R.nbr[6 * id + side];
  T v;
  if (n > 0) v = SL(M.phi, n)[low ? gcell + nc * st : gcell - nc * st];
  else if (side == 4) v = -x[own];
  else if (side == 5) v = T(2 * M.voltage) - x[own];
  else v = x[own];
  x[gcell] = v;
}

// Items k0, k0 + stride, ... of phase op on level l (fewer than 2^31 items
// per level; a5g3_create checks the tree).
// NCT: the level's box size at compile time (8 on levels >= 1), 0: read it.
template <int NCT, class T>
__device__ __forceinline__ void phase(const Run3 &R, const MG3<T> &M, int op, int l, int a0, int a1, int k0,
                                      int stride) {
  const Lv L = lv_of(R, l);
  const int nc = NCT ? NCT : L.nc, g = nc + 2, gs = g * g * g, n3 = nc * nc * nc, hnc = nc >> 1, nh = hnc * hnc * hnc;
  using P2 = typename Pair<T>::type;
  switch (op) {
    case PH_SWEEP: {
      const int per = n3 / 2;
      for (int k = k0; k < L.n * per; k += stride)
        it_sweep(R, M, L.first + k / per, nc, k % per, a0, a1);
      break;
    }
    case PH_FILL: {
      const int per = 6 * nc * nc;
      for (int k = k0; k < L.n * per; k += stride) it_fill(R, M, L.first + k / per, nc, k % per);
      break;
    }
    case PH_RESID_RESTRICT:
      for (int k = k0; k < L.n * nh; k += stride) it_resid_restrict(R, M, L.first + k / nh, nc, k % nh);
      break;
    case PH_COARSE_RHS:
      for (int k = k0; k < L.n * gs; k += stride) it_coarse_rhs(R, M, L.first + k / gs, nc, k % gs, a0);
      break;
    case PH_CORR_DIFF: {
      // whole slots, two values per item (slots start on 8 SLOT3-byte boundaries)
      const int h = gs / 2;
      for (int k = k0; k < L.n * h; k += stride) {
        const int id = L.first + k / h, c = k % h;
        P2 *tmp = reinterpret_cast<P2 *>(SL(M.tmp, id)) + c;
        const P2 ph = reinterpret_cast<const P2 *>(SL(M.phi, id))[c], t = *tmp;
        P2 o;
        o.x = ph.x - t.x;
        o.y = ph.y - t.y;
        *tmp = o;
      }
      break;
    }
    case PH_CORRECT:
      for (int k = k0; k < L.n * n3; k += stride) it_correct(R, M, L.first + k / n3, nc, k % n3);
      break;
    case PH_COPY: {
      // tmp = phi, whole slots
      const int h = gs / 2;
      for (int k = k0; k < L.n * h; k += stride) {
        const int id = L.first + k / h, c = k % h;
        reinterpret_cast<P2 *>(SL(M.tmp, id))[c] = reinterpret_cast<const P2 *>(SL(M.phi, id))[c];
      }
      break;
    }
    case PH_INIT_PHI_RHS:
      for (int k = k0; k < L.n * (gs + nh); k += stride) {
        const int q = k / (gs + nh);
        const int r = k % (gs + nh), id = L.first + q;
        if (r < gs) SL(M.phi, id)[r] = T(0);
        else it_restrict_rhs(R, M, id, nc, r - gs);
      }
      break;
    case PH_RESIDUAL: {
      for (int k = k0; k < L.n * n3; k += stride) {
        const int id = L.first + k / n3, t = k % n3;
        const double h = R.geo[4 * id + 3];
        const T inv_dr_sq = T(1 / (h * h));
        const int c = ix3(g, t % nc + 1, (t / nc) % nc + 1, t / (nc * nc) + 1);
        SL(M.tmp, id)[c] = SL(M.rhs, id)[c] - lpl3(SL(M.phi, id), c, g, inv_dr_sq);
      }
      break;
    }
  }
  (void)a1;
}

__host__ __device__ __forceinline__ long long phase_items(int op, int n, int nc) {
  const long long g = nc + 2, gs = g * g * g, n3 = (long long)nc * nc * nc, nh = n3 / 8;
  switch (op) {
    case PH_SWEEP: return n * (n3 / 2);
    case PH_FILL: return n * 6LL * nc * nc;
    case PH_RESID_RESTRICT: return n * nh;
    case PH_CORRECT:
    case PH_RESIDUAL: return n * n3;
    case PH_INIT_PHI_RHS: return n * (gs + nh);
    case PH_COPY:
    case PH_CORR_DIFF: return n * (gs / 2);
    default: return n * gs;
  }
}

// One phase on the grid (grid-stride over its items).
// One kernel per phase, box size and storage type, so that each has its own
// registers.
template <int NCT, int OP, class T>
__global__ void __launch_bounds__(NTH3) k3_phase(Run3 R, MG3<T> M, int l, int a0, int a1) {
  phase<NCT>(R, M, OP, l, a0, a1, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Multigrid work per level visit: Gauss-Seidel cycles on the way down, on the
// way up and on the base level (the reference: 2, 2, n_cycle_base).
struct Sweeps3 {
  int down, up, base;
};

// ---------------------------------------------------------------------------
// The coarse levels lo..top in one block: the sequences of the multigrid
// cycle that stay on those levels run as one launch, each phase spread over
// the block's threads and ended by a block barrier.
constexpr int NTHC = 1024;
template <class T>
__device__ __forceinline__ void c_phase(const Run3 &R, const MG3<T> &M, int op, int l, int a0 = 0, int a1 = 0) {
  // levels >= 1 with the box size at compile time (the levels below hold a
  // single box each)
  if (lv_of(R, l).nc == NC3) phase<NC3>(R, M, op, l, a0, a1, threadIdx.x, NTHC);
  else phase<0>(R, M, op, l, a0, a1, threadIdx.x, NTHC);
  __syncthreads();
}
template <class T>
__device__ void c_gsrb(const Run3 &R, const MG3<T> &M, int l, int n_cycle, bool stale) {
  for (int it = 1; it <= 2 * n_cycle; it++) c_phase(R, M, PH_SWEEP, l, it, stale && it == 1 ? 1 : 0);
  c_phase(R, M, PH_FILL, l);
}
template <class T>
__device__ void c_coarse(const Run3 &R, const MG3<T> &M, int l, int copy) {
  c_phase(R, M, PH_RESID_RESTRICT, l);
  c_phase(R, M, PH_FILL, l - 1);
  c_phase(R, M, PH_COARSE_RHS, l - 1, copy);
}
template <class T>
__device__ void c_correct(const Run3 &R, const MG3<T> &M, int l) {
  c_phase(R, M, PH_CORR_DIFF, l - 1);
  c_phase(R, M, PH_CORRECT, l);
  c_phase(R, M, PH_FILL, l);
}
// mg3_fas_vcycle (:208-255) on levels lo..top
template <class T>
__device__ void c_vcycle(const Run3 &R, const MG3<T> &M, const Sweeps3 &S, int top, bool stale) {
  for (int l = top; l >= R.lo + 1; l--) {
    c_gsrb(R, M, l, S.down, false);
    c_coarse(R, M, l, 1);
  }
  c_gsrb(R, M, R.lo, S.base, stale);
  for (int l = R.lo + 1; l <= top; l++) {
    c_correct(R, M, l);
    c_gsrb(R, M, l, S.up, false);
  }
}
enum { CM_VCYCLE = 0, CM_FMG, CM_SETC, CM_INIT };
template <class T>
__global__ void __launch_bounds__(NTHC) k3_coarse(Run3 R, MG3<T> M, Sweeps3 S, int mode, int top, int flag) {
  switch (mode) {
    case CM_VCYCLE:  // the middle of a V-cycle: down from top, base, up to top
      c_vcycle(R, M, S, top, flag != 0);
      break;
    case CM_FMG:  // the FMG's levels lo..top (mg3_fas_fmg, :186-202); flag: first call
      for (int l = R.lo; l <= top; l++) {
        c_phase(R, M, PH_COPY, l);
        if (l > R.lo) c_correct(R, M, l);
        c_vcycle(R, M, S, l, flag != 0 && l == R.lo);
      }
      break;
    case CM_SETC:  // set_coarse_phi_rhs for levels top..lo+1 (:176-180)
      for (int l = top; l >= R.lo + 1; l--) c_coarse(R, M, l, 0);
      break;
    case CM_INIT:  // init_phi_rhs on levels top..lo+1 (:526-549)
      for (int l = top; l >= R.lo + 1; l--) c_phase(R, M, PH_INIT_PHI_RHS, l);
      break;
  }
}

// The mixed form's field solve (defect correction): the FP64 residual of the
// finest level (the leaves of a uniform octree) rhs - lpl(phi), ghost
// neighbours from their sources with the applied voltage, into the FP32
// correction solve's rhs (0 on ghost cells), and the correction 0 on the
// whole slot.
__global__ void __launch_bounds__(NTH3) k3_mx_resid(Run3 R, MG3<float> C, const int *ids) {
  const int id = ids[blockIdx.x];
  const int nc = R.nc[id], g = nc + 2, gs = g * g * g;
  const MG3<double> F{VAR(R, I_PHI), VAR(R, I_RHS), VAR(R, I_FLD), R.voltage};
  const double dr = R.geo[4 * id + 3], inv_dr_sq = 1 / (dr * dr);
  const double *phi = SL(F.phi, id), *rhs = SL(F.rhs, id);
  float *cr = SL(C.rhs, id), *cp = SL(C.phi, id);
  for (int c = threadIdx.x; c < gs; c += NTH3) {
    const int i = c % g, j = (c / g) % g, k = c / (g * g);
    const bool in = i >= 1 && i <= nc && j >= 1 && j <= nc && k >= 1 && k <= nc;
    cr[c] = in ? (float)(rhs[c] - lpl3_src(R, F, id, nc, phi, c, i, j, k, inv_dr_sq)) : 0.0f;
    cp[c] = 0.0f;
  }
}
// phi += c on the interior cells of every box (FP64 accumulation of the FP32
// correction), with the FP64 ghost fill of phi (sides_bc_pot on physical
// sides) pushed in the same pass.
__global__ void __launch_bounds__(NTH3) k3_mx_acc(Run3 R, MG3<float> C, const int *ids) {
  const int id = ids[blockIdx.x];
  const int nc = R.nc[id], g = nc + 2, n = nc * nc * nc;
  double *phi = CC(R, I_PHI, id);
  const float *cp = SL(C.phi, id);
  for (int t = threadIdx.x; t < n; t += NTH3) {
    const int i = t % nc + 1, j = (t / nc) % nc + 1, k = t / (nc * nc) + 1;
    const int c = ix3(g, i, j, k);
    const double v = phi[c] + (double)cp[c];
    phi[c] = v;
    push_side_ghosts(R, I_PHI, id, nc, i, j, k, v, 1);
  }
}

// compute_fld's space charge (src/streamer_3d.f90:317-329): rhs = e/eps0
// (n_e - n_i) on whole slots of the leaves of levels >= 1
__global__ void __launch_bounds__(NTH3) k3_set_rhs(Run3 R, const int *ids) {
  const int id = ids[blockIdx.x];
  const int g = R.nc[id] + 2, gs = g * g * g;
  const double fac = UC_ELEM_CHARGE / UC_EPS0;
  const double *e = CC(R, I_ELEC, id), *p = CC(R, I_PION, id);
  double *rhs = CC(R, I_RHS, id);
  for (int c = threadIdx.x; c < gs; c += NTH3) rhs[c] = fac * (e[c] - p[c]);
}

// fld_from_pot (src/streamer_3d.f90:348-393) on every box: the face fields
// (eps-weighted on the box-edge faces) into the F_FLD slots and shared
// memory, then |E| = 0.5 sqrt(sx^2 + sy^2 + sz^2) per interior cell.
template <int NCT>
__device__ __forceinline__ void fld_box(const Run3 &R, int id, double *sfc) {
  const int nc = NCT ? NCT : R.nc[id], g = nc + 2, F = (nc + 1) * nc * nc;
  const double inv_dr = 1 / R.geo[4 * id + 3];
  const double *phi = CC(R, I_PHI, id), *eps = CC(R, I_EPS, id);
  for (int q = threadIdx.x; q < 3 * F; q += NTH3) {
    const int d = q / F, r = q - d * F;
    int i, j, k, a;
    if (d == 0) {
      i = r % (nc + 1) + 1;
      j = (r / (nc + 1)) % nc + 1;
      k = r / ((nc + 1) * nc) + 1;
      a = i;
    } else if (d == 1) {
      i = r % nc + 1;
      j = (r / nc) % (nc + 1) + 1;
      k = r / (nc * (nc + 1)) + 1;
      a = j;
    } else {
      i = r % nc + 1;
      j = (r / nc) % nc + 1;
      k = r / (nc * nc) + 1;
      a = k;
    }
    const int st = d == 0 ? 1 : d == 1 ? g : g * g;
    const int c0 = ix3(g, i, j, k), cm = c0 - st;
    double v;
    if (a == 1) {
      v = 2 * inv_dr * (phi[cm] - phi[c0]) * eps[cm] / (eps[c0] + eps[cm]);
    } else if (a == nc + 1) {
      v = 2 * inv_dr * (phi[cm] - phi[c0]) * eps[c0] / (eps[c0] + eps[cm]);
    } else {
      v = inv_dr * (phi[cm] - phi[c0]);
    }
    sfc[d * FSLOT3 + r] = v;
    FC(R, d, F_FLD, id)[r] = v;
  }
  __syncthreads();
  double *fld = CC(R, I_FLD, id);
  const int n = nc * nc * nc;
  for (int t = threadIdx.x; t < n; t += NTH3) {
    const int i = t % nc + 1, j = (t / nc) % nc + 1, k = t / (nc * nc) + 1;
    const int xl = (i - 1) + (nc + 1) * ((j - 1) + nc * (k - 1));
    const int yl = (i - 1) + nc * ((j - 1) + (nc + 1) * (k - 1));
    const int zl = (i - 1) + nc * ((j - 1) + nc * (k - 1));
    const double sx = sfc[xl] + sfc[xl + 1];
    const double sy = sfc[FSLOT3 + yl] + sfc[FSLOT3 + yl + nc];
    const double sz = sfc[2 * FSLOT3 + zl] + sfc[2 * FSLOT3 + zl + nc * nc];
    const double v = 0.5 * sqrt(sx * sx + sy * sy + sz * sz);
    fld[ix3(g, i, j, k)] = v;
    push_side_ghosts(R, I_FLD, id, nc, i, j, k, v);
  }
}
__global__ void __launch_bounds__(NTH3) k3_fld(Run3 R, const int *ids) {
  __shared__ double sfc[3 * FSLOT3];
  const int id = ids[blockIdx.x];
  // boxes of levels >= 1 with the box size at compile time
  if (R.nc[id] == NC3) fld_box<NC3>(R, id, sfc);
  else fld_box<0>(R, id, sfc);
}

// ---------------------------------------------------------------------------
// Reductions over the interior cells of the leaves (a3_tree_max_cc /
// a3_tree_min_cc, afivo/src/m_aX_utils.f90:559-619; exact, so in any order).
// kind 0: the three of get_max_dt (max |E|, min |E|, max n_e) per block into
// part[3 b ..]; kind 1 / 2: max / min of variable iv into part[b].
__device__ __forceinline__ double red_op(double a, double b, bool mx) { return mx ? fmax(a, b) : fmin(a, b); }
__global__ void __launch_bounds__(NTH3) k3_reduce_boxes(Run3 R, const int *ids, int kind, int iv) {
  __shared__ double red[3][NTH3 / 32];
  const int id = ids[blockIdx.x];
  const int nc = R.nc[id], g = nc + 2, n = nc * nc * nc;
  const double HUGE_D = 1.7976931348623157e308;
  const double *a = CC(R, kind == 0 ? I_FLD : iv, id), *e = CC(R, I_ELEC, id);
  double v0 = kind == 2 ? HUGE_D : -HUGE_D, v1 = HUGE_D, v2 = -HUGE_D;
  for (int t = threadIdx.x; t < n; t += NTH3) {
    const int c = ix3(g, t % nc + 1, (t / nc) % nc + 1, t / (nc * nc) + 1);
    v0 = red_op(v0, a[c], kind != 2);
    if (kind == 0) {
      v1 = fmin(v1, a[c]);
      v2 = fmax(v2, e[c]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    v0 = red_op(v0, __shfl_xor_sync(0xffffffffu, v0, o), kind != 2);
    v1 = fmin(v1, __shfl_xor_sync(0xffffffffu, v1, o));
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = v0;
    red[1][threadIdx.x >> 5] = v1;
    red[2][threadIdx.x >> 5] = v2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NTH3 / 32; w++) {
      v0 = red_op(v0, red[0][w], kind != 2);
      v1 = fmin(v1, red[1][w]);
      v2 = fmax(v2, red[2][w]);
    }
    if (kind == 0) {
      R.part[3 * blockIdx.x] = v0;
      R.part[3 * blockIdx.x + 1] = v1;
      R.part[3 * blockIdx.x + 2] = v2;
    } else {
      R.part[blockIdx.x] = v0;
    }
  }
}
// The blocks' partial results into scal[S_RED ..] (one block).
__global__ void __launch_bounds__(NTH3) k3_reduce_final(Run3 R, int nb, int kind) {
  __shared__ double red[3][NTH3 / 32];
  const double HUGE_D = 1.7976931348623157e308;
  const int w = kind == 0 ? 3 : 1;
  double v0 = kind == 2 ? HUGE_D : -HUGE_D, v1 = HUGE_D, v2 = -HUGE_D;
  for (int b = threadIdx.x; b < nb; b += NTH3) {
    v0 = red_op(v0, R.part[w * b], kind != 2);
    if (kind == 0) {
      v1 = fmin(v1, R.part[3 * b + 1]);
      v2 = fmax(v2, R.part[3 * b + 2]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    v0 = red_op(v0, __shfl_xor_sync(0xffffffffu, v0, o), kind != 2);
    v1 = fmin(v1, __shfl_xor_sync(0xffffffffu, v1, o));
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = v0;
    red[1][threadIdx.x >> 5] = v1;
    red[2][threadIdx.x >> 5] = v2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < NTH3 / 32; q++) {
      v0 = red_op(v0, red[0][q], kind != 2);
      v1 = fmin(v1, red[1][q]);
      v2 = fmax(v2, red[2][q]);
    }
    R.scal[S_RED] = v0;
    R.scal[S_RED + 1] = v1;
    R.scal[S_RED + 2] = v2;
  }
}

// The step size of the next launches (device scalar, so that one captured
// graph serves every step).
__global__ void k3_set_dt(double *scal, double dt) { scal[S_DT] = dt; }

}  // namespace

// ===========================================================================
// Host side.

static thread_local std::string g_err3;
static int fail3(int code, const std::string &msg) {
  g_err3 = msg;
  return code;
}
#define CK3(x)                                                                   \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) return fail3(A5G_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
static T *SL_host(T *a, int id) { return a + (size_t)id * SLOT3; }

struct a5g3_ctx {
  a5g3_params p{};
  int max_id = 0, min_lvl = 1, max_lvl = 1;
  long long cap = 0;
  // host copy of the tree (per id)
  std::vector<int> lvl, ix, nc, nbr, chl, par, off;
  std::vector<double> geo;
  std::vector<int> lv_off, lv_n;  // per level index: offset into lv_ids, count
  std::vector<int> lv_ids;        // ids level by level, min_lvl..max_lvl
  // device
  double *d_cc = nullptr, *d_fc = nullptr, *d_lt = nullptr, *d_scal = nullptr, *d_part = nullptr;
  int *d_nc = nullptr, *d_nbr = nullptr, *d_chl = nullptr, *d_par = nullptr, *d_off = nullptr;
  int *d_ids = nullptr;
  double *d_geo = nullptr;
  int lt_rows = 0;
  double lt_xmin = 0, lt_inv_dx = 0;
  std::vector<double> h_lt;
  double voltage = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double *h_red = nullptr;  // pinned, 4 doubles

  // mixed precision (a5g3_set_precision): schedule of the FP32 correction
  // solve, its three FP32 arrays (phi, rhs, tmp; cap slots each) and the
  // FP32 copy of the table
  int precision = A5G_FP64;
  a5g_mg_schedule sched{1, 2, 2, 4, 1};
  float *d_c32 = nullptr, *d_lt32 = nullptr;

  int coarse_top = 0;  // levels min_lvl..coarse_top run in one block (k3_coarse)
  MG3<double> mg64() const {
    const size_t n = (size_t)cap * SLOT3;
    return MG3<double>{d_cc + I_PHI * n, d_cc + I_RHS * n, d_cc + I_FLD * n, voltage};
  }
  MG3<float> mg32() const {
    const size_t n = (size_t)cap * SLOT3;
    return MG3<float>{d_c32, d_c32 + n, d_c32 + 2 * n, 0.0};
  }
  Sweeps3 sweeps64() const { return Sweeps3{2, 2, p.n_cycle_base}; }
  int li(int l) const { return l - min_lvl; }
  int nc_of(int l) const { return l >= 1 ? p.box_size : p.box_size >> (1 - l); }
  const int *ids(int l) const { return d_ids + lv_off[li(l)]; }
  int count(int l) const { return lv_n[li(l)]; }
  const int *all_ids() const { return d_ids; }
  int n_all() const { return (int)lv_ids.size(); }
  Run3 run() const {
    Run3 R;
    R.cc = d_cc;
    R.fc = d_fc;
    R.nc = d_nc;
    R.nbr = d_nbr;
    R.chl = d_chl;
    R.par = d_par;
    R.off = d_off;
    R.geo = d_geo;
    R.lt = d_lt;
    R.lt32 = d_lt32;
    R.scal = d_scal;
    R.part = d_part;
    R.cap = cap;
    R.lt_rows = lt_rows;
    R.lt_xmin = lt_xmin;
    R.lt_inv_dx = lt_inv_dx;
    R.voltage = voltage;
    R.ids = d_ids;
    R.lo = min_lvl;
    R.nlev = max_lvl - min_lvl + 1;
    R.n_cycle_base = p.n_cycle_base;
    for (int q = 0; q < 16; q++) {
      const bool in = q < R.nlev;
      R.lv_first[q] = in ? lv_ids[lv_off[q]] : 0;
      R.lv_off[q] = in ? lv_off[q] : 0;
      R.lv_n[q] = in ? lv_n[q] : 0;
      R.lv_nc[q] = in ? nc_of(min_lvl + q) : 0;
    }
    return R;
  }
};

// The uniform octree with the reference's ids: a3_set_base
// (afivo/src/m_aX_core.f90:134-217: the base boxes on level 1 in ix order
// (x fastest), one box per base box on each coarse level min_lvl..0, ids
// level by level from min_lvl), then a3_adjust_refinement with every box of
// the finest level flagged (:456-520, add_children :753-788): each parent's
// eight children take consecutive ids in child order (x fastest), parents in
// level order. Neighbours are the same-level boxes across each face, or -1
// at the domain walls (the physical boundary of nb_list).
static void build_tree(a5g3_ctx *c) {
  const a5g3_params &p = c->p;
  const int nc8 = p.box_size;
  const int nx = p.n_base[0], ny = p.n_base[1], nz = p.n_base[2], nbase = nx * ny * nz;
  c->min_lvl = 1 - (int)std::lround(std::log((double)nc8 / 2) / std::log(2.0));
  c->max_lvl = p.uniform_lvl;
  const int nlev = c->max_lvl - c->min_lvl + 1;
  long long total = 1;  // id 0 unused
  std::vector<long long> per(nlev);
  for (int l = c->min_lvl; l <= c->max_lvl; l++) {
    per[l - c->min_lvl] = l <= 1 ? nbase : per[l - 1 - c->min_lvl] * 8;
    total += per[l - c->min_lvl];
  }
  c->cap = total;
  c->max_id = (int)(total - 1);
  const size_t n = (size_t)total;
  c->lvl.assign(n, 0);
  c->ix.assign(3 * n, 0);
  c->nc.assign(n, 0);
  c->nbr.assign(6 * n, 0);
  c->chl.assign(8 * n, 0);
  c->par.assign(n, 0);
  c->off.assign(3 * n, 0);
  c->geo.assign(4 * n, 0.0);
  c->lv_off.assign(nlev, 0);
  c->lv_n.assign(nlev, 0);
  c->lv_ids.clear();
  int next = 1;
  // base and coarse levels
  for (int l = c->min_lvl; l <= 1; l++) {
    c->lv_off[l - c->min_lvl] = (int)c->lv_ids.size();
    c->lv_n[l - c->min_lvl] = nbase;
    const int first = next;
    for (int kk = 0; kk < nz; kk++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const int id = next++;
          const int q = i + nx * (j + ny * kk);
          c->lv_ids.push_back(id);
          c->lvl[id] = l;
          const int bix[3] = {i + 1, j + 1, kk + 1};
          for (int d = 0; d < 3; d++) {
            c->ix[3 * id + d] = bix[d];
            c->geo[4 * id + d] = 0.0 + (bix[d] - 1) * p.dr_base * nc8;
          }
          c->geo[4 * id + 3] = p.dr_base * std::pow(0.5, l - 1);
          c->nc[id] = nc8 / (1 << (1 - l));
          const int nbq[6] = {i > 0 ? q - 1 : -1, i < nx - 1 ? q + 1 : -1, j > 0 ? q - nx : -1,
                              j < ny - 1 ? q + nx : -1, kk > 0 ? q - nx * ny : -1, kk < nz - 1 ? q + nx * ny : -1};
          for (int s = 0; s < 6; s++) c->nbr[6 * id + s] = nbq[s] >= 0 ? first + nbq[s] : -1;
          if (l > c->min_lvl) {
            const int pid = id - nbase;
            c->par[id] = pid;
            c->chl[8 * pid] = id;
          }
        }
  }
  // finer levels: children of each parent in order
  for (int l = 2; l <= c->max_lvl; l++) {
    const int L0 = c->lv_off[l - 1 - c->min_lvl], Ln = c->lv_n[l - 1 - c->min_lvl];
    c->lv_off[l - c->min_lvl] = (int)c->lv_ids.size();
    c->lv_n[l - c->min_lvl] = 8 * Ln;
    for (int q = 0; q < Ln; q++) {
      const int pid = c->lv_ids[L0 + q];
      for (int ch = 0; ch < 8; ch++) {
        const int id = next++;
        c->lv_ids.push_back(id);
        c->chl[8 * pid + ch] = id;
        c->par[id] = pid;
        c->lvl[id] = l;
        c->nc[id] = nc8;
        const int dix[3] = {ch & 1, (ch >> 1) & 1, (ch >> 2) & 1};
        for (int d = 0; d < 3; d++) {
          c->ix[3 * id + d] = 2 * c->ix[3 * pid + d] - 1 + dix[d];
          c->geo[4 * id + d] = c->geo[4 * pid + d] + 0.5 * c->geo[4 * pid + 3] * dix[d] * nc8;
          c->off[3 * id + d] = l > 1 ? ((c->ix[3 * id + d] - 1) & 1) * (nc8 >> 1) : 0;
        }
        c->geo[4 * id + 3] = 0.5 * c->geo[4 * pid + 3];
      }
    }
    // same-level neighbours through a (ix) -> id map of the level
    const long long ext[3] = {(long long)nx << (l - 1), (long long)ny << (l - 1), (long long)nz << (l - 1)};
    std::vector<int> at((size_t)(ext[0] * ext[1] * ext[2]), 0);
    const int F0 = c->lv_off[l - c->min_lvl], Fn = c->lv_n[l - c->min_lvl];
    auto key = [&](long long a, long long b, long long d) { return (size_t)(a - 1 + ext[0] * ((b - 1) + ext[1] * (d - 1))); };
    for (int q = 0; q < Fn; q++) {
      const int id = c->lv_ids[F0 + q];
      at[key(c->ix[3 * id], c->ix[3 * id + 1], c->ix[3 * id + 2])] = id;
    }
    for (int q = 0; q < Fn; q++) {
      const int id = c->lv_ids[F0 + q];
      for (int s = 0; s < 6; s++) {
        long long v[3] = {c->ix[3 * id], c->ix[3 * id + 1], c->ix[3 * id + 2]};
        const int d = s >> 1;
        v[d] += (s & 1) ? 1 : -1;
        c->nbr[6 * id + s] = (v[d] < 1 || v[d] > ext[d]) ? -1 : at[key(v[0], v[1], v[2])];
      }
    }
  }
}

constexpr int COARSE_BOXES = 8;
static int grid_for(long long n) { return (int)std::min<long long>((n + NTH3 - 1) / NTH3, 148LL * 16); }

template <class T>
static int upload(T *&dst, const std::vector<T> &src, cudaStream_t s) {
  CK3(cudaMallocAsync((void **)&dst, std::max<size_t>(1, src.size()) * sizeof(T), s));
  if (!src.empty()) CK3(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return A5G_OK;
}

// ---------------------------------------------------------------------------
// Launch sequences (all on the context's stream).

// a3_gc_tree for up to two variables on every box (bc 0: Neumann sides;
// bc 1: sides_bc_pot)
static void enq_gc_all(a5g3_ctx *c, int iv0, int iv1, int bc) {
  k3_gc<<<c->n_all(), NTH3, 0, c->stream>>>(c->run(), c->all_ids(), iv0, iv1, bc);
}
template <int NCT, class T>
static void launch_phase(a5g3_ctx *c, const MG3<T> &M, int op, int grid, int l, int a0, int a1) {
  const Run3 R = c->run();
  cudaStream_t s = c->stream;
  switch (op) {
    case PH_SWEEP: k3_phase<NCT, PH_SWEEP, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_FILL: k3_phase<NCT, PH_FILL, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_RESID_RESTRICT: k3_phase<NCT, PH_RESID_RESTRICT, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_COARSE_RHS: k3_phase<NCT, PH_COARSE_RHS, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_CORR_DIFF: k3_phase<NCT, PH_CORR_DIFF, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_CORRECT: k3_phase<NCT, PH_CORRECT, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_COPY: k3_phase<NCT, PH_COPY, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_INIT_PHI_RHS: k3_phase<NCT, PH_INIT_PHI_RHS, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
    case PH_RESIDUAL: k3_phase<NCT, PH_RESIDUAL, T><<<grid, NTH3, 0, s>>>(R, M, l, a0, a1); break;
  }
}

// One multigrid phase of level l on the grid, about one item per thread.
template <class T>
static void enq_phase(a5g3_ctx *c, const MG3<T> &M, int op, int l, int a0 = 0, int a1 = 0) {
  const long long n = phase_items(op, c->count(l), c->nc_of(l));
  const int grid = (int)std::min<long long>((n + NTH3 - 1) / NTH3, 1LL << 20);
  if (c->nc_of(l) == NC3) launch_phase<NC3>(c, M, op, grid, l, a0, a1);
  else launch_phase<0>(c, M, op, grid, l, a0, a1);
}
template <class T>
static void enq_fill(a5g3_ctx *c, const MG3<T> &M, int l) { enq_phase(c, M, PH_FILL, l); }

// gsrb_boxes (afivo/src/m_aX_mg.f90:403-426): 2 n_cycle half-sweeps with the
// ghost sources evaluated inside the sweeps, then (fill) the ghost fill the
// last half-sweep is followed by. stale: the first half-sweep reads the
// ghost cells in memory. Ghost fills whose values no later phase reads from
// memory are left out (fill = false): the phases that follow evaluate those
// ghost cells from their sources, and every level's ghost cells are filled
// after its last change in a cycle.
template <class T>
static void enq_gsrb(a5g3_ctx *c, const MG3<T> &M, int l, int n_cycle, bool stale, bool fill = true) {
  for (int it = 1; it <= 2 * n_cycle; it++) enq_phase(c, M, PH_SWEEP, l, it, stale && it == 1 ? 1 : 0);
  if (fill) enq_fill(c, M, l);
}

// update_coarse (:430-486) / set_coarse_phi_rhs (:490-523) for level l
template <class T>
static void enq_coarse(a5g3_ctx *c, const MG3<T> &M, int l, bool copy) {
  enq_phase(c, M, PH_RESID_RESTRICT, l);
  enq_fill(c, M, l - 1);
  enq_phase(c, M, PH_COARSE_RHS, l - 1, copy ? 1 : 0);
}

// correct_children (:374-401) of level l - 1's parents; its fill_gc_phi of
// l is left out, as every caller smooths level l next (sweeps evaluate their
// ghost neighbours from the sources) and fills it after that.
template <class T>
static void enq_correct(a5g3_ctx *c, const MG3<T> &M, int l) {
  enq_phase(c, M, PH_CORR_DIFF, l - 1);
  enq_phase(c, M, PH_CORRECT, l);
}

template <class T>
static void enq_coarse_kernel(a5g3_ctx *c, const MG3<T> &M, const Sweeps3 &S, int mode, int top, int flag) {
  k3_coarse<T><<<1, NTHC, 0, c->stream>>>(c->run(), M, S, mode, top, flag);
}

// mg3_fas_vcycle (afivo/src/m_aX_mg.f90:208-255). The levels lo..top (top =
// the coarse section, at most max_lvl) run in one k3_coarse launch.
template <class T>
static void enq_vcycle(a5g3_ctx *c, const MG3<T> &M, const Sweeps3 &S, int max_lvl, bool set_residual,
                       bool stale_base) {
  const int lo = c->min_lvl, top = std::min(max_lvl, c->coarse_top);
  for (int l = max_lvl; l >= std::max(lo, top) + 1; l--) {
    enq_gsrb(c, M, l, S.down, false, false);  // the residual evaluates the ghosts itself
    enq_coarse(c, M, l, true);
  }
  if (top >= lo) {
    enq_coarse_kernel(c, M, S, CM_VCYCLE, top, stale_base ? 1 : 0);
  } else {
    enq_gsrb(c, M, lo, S.base, stale_base);
  }
  for (int l = std::max(lo, top) + 1; l <= max_lvl; l++) {
    enq_correct(c, M, l);
    enq_gsrb(c, M, l, S.up, false);
  }
  if (set_residual)
    for (int l = lo; l <= max_lvl; l++) enq_phase(c, M, PH_RESIDUAL, l);
}

// The FMG's stages (mg3_fas_fmg, :186-202) after its coarse set-up: on each
// level from the coarsest, tmp = phi, the correction from the coarser level,
// a V-cycle; the coarse section's part in one k3_coarse launch.
template <class T>
static void enq_fmg_stages(a5g3_ctx *c, const MG3<T> &M, const Sweeps3 &S, bool set_residual, bool first_call) {
  const int lo = c->min_lvl, hi = c->max_lvl, top = c->coarse_top;
  if (top >= lo) enq_coarse_kernel(c, M, S, CM_FMG, top, first_call ? 1 : 0);
  for (int l = std::max(lo, top + 1); l <= hi; l++) {
    enq_phase(c, M, PH_COPY, l);
    if (l > lo) enq_correct(c, M, l);
    enq_vcycle(c, M, S, l, set_residual && l == hi, first_call && l == lo);
  }
}

// mg3_fas_fmg (afivo/src/m_aX_mg.f90:164-203) in FP64 on the run's variables
static void enq_fmg(a5g3_ctx *c, bool set_residual, bool first_call) {
  const MG3<double> M = c->mg64();
  const Sweeps3 S = c->sweeps64();
  const int lo = c->min_lvl, hi = c->max_lvl, top = c->coarse_top;
  if (first_call) {
    for (int l = hi; l >= std::max(lo, top) + 1; l--) enq_phase(c, M, PH_INIT_PHI_RHS, l);
    if (top >= lo + 1) enq_coarse_kernel(c, M, S, CM_INIT, top, 0);
  } else {
    // (the residual evaluates the finest level's ghost cells itself, so its
    // fill_gc_phi, :497-498, is left out)
    for (int l = hi; l >= std::max(lo, top) + 1; l--) enq_coarse(c, M, l, false);
    if (top >= lo + 1) enq_coarse_kernel(c, M, S, CM_SETC, top, 0);
  }
  enq_fmg_stages(c, M, S, set_residual, first_call);
}

// The mixed form's field solve: per correction pass, the FP64 residual of
// the leaves into the FP32 correction equation (homogeneous wall values),
// restricted to the coarser levels with the correction 0 everywhere
// (init_phi_rhs's phases on the FP32 arrays), the FP32 solve with the run's
// schedule (FMG stages or one V-cycle), then phi += c in FP64 and the FP64
// ghost fill of phi.
static void enq_solve_mixed(a5g3_ctx *c) {
  const MG3<float> C = c->mg32();
  const Sweeps3 S{c->sched.n_cycle_down, c->sched.n_cycle_up, c->sched.n_cycle_base};
  const int lo = c->min_lvl, hi = c->max_lvl, top = c->coarse_top;
  for (int pass = 0; pass < c->sched.n_corr; pass++) {
    k3_mx_resid<<<c->count(hi), NTH3, 0, c->stream>>>(c->run(), C, c->ids(hi));
    for (int l = hi; l >= std::max(lo, top) + 1; l--) enq_phase(c, C, PH_INIT_PHI_RHS, l);
    if (top >= lo + 1) enq_coarse_kernel(c, C, S, CM_INIT, top, 0);
    // the coarsest level's correction: 0 (its ids are the first of the tree)
    cudaMemsetAsync(SL_host(C.phi, c->lv_ids[c->lv_off[0]]), 0, (size_t)c->count(lo) * SLOT3 * sizeof(float),
                    c->stream);
    if (c->sched.fmg) enq_fmg_stages(c, C, S, false, false);
    else enq_vcycle(c, C, S, hi, false, false);
    k3_mx_acc<<<c->n_all(), NTH3, 0, c->stream>>>(c->run(), C, c->all_ids());
  }
}

// compute_fld (src/streamer_3d.f90:309-345) with one FMG cycle; in the mixed
// form (not on a first call) the defect-correction solve
static void enq_compute_fld(a5g3_ctx *c, bool no_guess) {
  k3_set_rhs<<<c->count(c->max_lvl), NTH3, 0, c->stream>>>(c->run(), c->ids(c->max_lvl));
  if (c->precision == A5G_MIXED && !no_guess) enq_solve_mixed(c);
  else enq_fmg(c, false, no_guess);
  // the |E| side ghosts of every level are filled by k3_fld itself
  k3_fld<<<c->n_all(), NTH3, 0, c->stream>>>(c->run(), c->all_ids());
}

// a3_restrict_tree (afivo/src/m_aX_restrict.f90:23-64) for up to two variables
static void enq_restrict(a5g3_ctx *c, int iv0, int iv1) {
  for (int l = c->max_lvl; l >= c->min_lvl + 1; l--)
    k3_restrict<<<c->count(l), NTH3, 0, c->stream>>>(c->run(), c->ids(l), iv0, iv1);
}

// One time step (src/streamer_3d.f90:96-128): the leaves are the boxes of the
// finest level; consistent fluxes change nothing on a uniform octree. The
// mixed form runs the fluxes and the update in FP32 and the field solves by
// defect correction.
static void enq_step(a5g3_ctx *c) {
  const long long ncell = c->cap * SLOT3;
  k3_copy2<<<grid_for(ncell / 2), NTH3, 0, c->stream>>>(c->run(), I_ELEC, I_ELEC_OLD, I_PION, I_PION_OLD);
  const int hi = c->max_lvl;
  const bool mx = c->precision == A5G_MIXED;
  for (int stage = 1; stage <= 2; stage++) {
    if (mx) {
      k3_fluxes<float><<<c->count(hi), NTH3, 0, c->stream>>>(c->run(), c->ids(hi));
      k3_update<float, true><<<c->count(hi), NTH3, 0, c->stream>>>(c->run(), c->ids(hi));
    } else {
      k3_fluxes<double><<<c->count(hi), NTH3, 0, c->stream>>>(c->run(), c->ids(hi));
      k3_update<double, true><<<c->count(hi), NTH3, 0, c->stream>>>(c->run(), c->ids(hi));
    }
    enq_restrict(c, I_ELEC, I_PION);
    // the leaves' side ghosts were pushed by the update: the coarser levels
    // (the first ids of the level-ordered list)
    if (c->n_all() > c->count(hi))
      k3_gc<<<c->n_all() - c->count(hi), NTH3, 0, c->stream>>>(c->run(), c->all_ids(), I_ELEC, I_PION, 0);
    if (stage == 1) enq_compute_fld(c, false);
  }
  k3_average<<<grid_for(ncell), NTH3, 0, c->stream>>>(c->run());
  enq_compute_fld(c, false);
}

// The captured step holds the launch arguments (table pointers, precision):
// settings that change them drop it, and the next step captures anew.
static void drop_graph(a5g3_ctx *c) {
  if (c->exec) {
    cudaGraphExecDestroy(c->exec);
    cudaGraphDestroy(c->graph);
    c->exec = nullptr;
    c->graph = nullptr;
  }
}

static int launched(a5g3_ctx *c) {
  CK3(cudaGetLastError());
  (void)c;
  return A5G_OK;
}
static int ready(a5g3_ctx *c) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  if (!c->d_lt) return fail3(A5G_ESTATE, "no transport table set");
  return A5G_OK;
}

extern "C" {

const char *a5g3_last_error(void) { return g_err3.c_str(); }

int a5g3_create(const a5g3_params *p, a5g3_ctx **out) {
  if (!p || !out) return fail3(A5G_EINVAL, "null argument");
  *out = nullptr;
  if (p->box_size != NC3) return fail3(A5G_EINVAL, "box_size must be 8");
  if (p->uniform_lvl < 1 || p->uniform_lvl > 12) return fail3(A5G_EINVAL, "uniform_lvl must be 1..12");
  {
    // every phase of the finest level must have fewer than 2^31 items
    const double boxes = (double)p->n_base[0] * p->n_base[1] * p->n_base[2] * std::pow(8.0, p->uniform_lvl - 1);
    if (boxes * (SLOT3 + 64) >= 2147483647.0) return fail3(A5G_EINVAL, "tree too large (uniform_lvl)");
  }
  for (int d = 0; d < 3; d++)
    if (p->n_base[d] < 1 || p->n_base[d] > 64) return fail3(A5G_EINVAL, "n_base must be 1..64");
  if (!(p->dr_base > 0) || p->n_cycle_base < 1) return fail3(A5G_EINVAL, "dr_base > 0 and n_cycle_base >= 1 required");
  a5g3_ctx *c = new a5g3_ctx();
  c->p = *p;
  build_tree(c);
  const size_t ncc = (size_t)NV3 * c->cap * SLOT3, nfc = (size_t)3 * NF3 * c->cap * FSLOT3;
  auto bail = [&](int code) {
    a5g3_destroy(c);
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail3(A5G_ECUDA, "stream creation failed"));
  if (cudaMalloc((void **)&c->d_cc, ncc * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void **)&c->d_fc, nfc * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail3(A5G_ENOMEM, "device allocation of the cell/face storage failed"));
  }
  if (cudaMemsetAsync(c->d_cc, 0, ncc * sizeof(double), c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_fc, 0, nfc * sizeof(double), c->stream) != cudaSuccess)
    return bail(fail3(A5G_ECUDA, "memset failed"));
  int r;
  if ((r = upload(c->d_nc, c->nc, c->stream)) || (r = upload(c->d_nbr, c->nbr, c->stream)) ||
      (r = upload(c->d_chl, c->chl, c->stream)) || (r = upload(c->d_par, c->par, c->stream)) ||
      (r = upload(c->d_off, c->off, c->stream)) || (r = upload(c->d_geo, c->geo, c->stream)) ||
      (r = upload(c->d_ids, c->lv_ids, c->stream)))
    return bail(r);
  if (cudaMalloc((void **)&c->d_scal, 16 * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void **)&c->d_part, (size_t)3 * c->cap * sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_red, 4 * sizeof(double)) != cudaSuccess)
    return bail(fail3(A5G_ENOMEM, "device allocation failed"));
  c->voltage = -p->domain_len_z * p->applied_fld;
  // the coarse section: the levels from min_lvl up with at most
  // COARSE_BOXES boxes each (4,096 cells), never the finest level
  c->coarse_top = c->min_lvl - 1;
  for (int l = c->min_lvl; l < c->max_lvl && c->count(l) <= COARSE_BOXES; l++) c->coarse_top = l;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail3(A5G_ECUDA, "setup failed"));
  *out = c;
  return A5G_OK;
}

int a5g3_destroy(a5g3_ctx *c) {
  if (!c) return A5G_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  for (void *ptr : {(void *)c->d_cc, (void *)c->d_fc, (void *)c->d_lt, (void *)c->d_lt32, (void *)c->d_c32,
                    (void *)c->d_scal, (void *)c->d_part,
                    (void *)c->d_nc, (void *)c->d_nbr, (void *)c->d_chl, (void *)c->d_par, (void *)c->d_off,
                    (void *)c->d_ids, (void *)c->d_geo})
    if (ptr) cudaFree(ptr);
  if (c->h_red) cudaFreeHost(c->h_red);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return A5G_OK;
}

int a5g3_info(a5g3_ctx *c, int *max_id, int *min_lvl, int *max_lvl, long long *n_leaf_cells) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  if (max_id) *max_id = c->max_id;
  if (min_lvl) *min_lvl = c->min_lvl;
  if (max_lvl) *max_lvl = c->max_lvl;
  if (n_leaf_cells) *n_leaf_cells = (long long)c->count(c->max_lvl) * NC3 * NC3 * NC3;
  return A5G_OK;
}

int a5g3_export_meta(a5g3_ctx *c, int *m24) {
  if (!c || !m24) return fail3(A5G_EINVAL, "null argument");
  for (int id = 0; id <= c->max_id; id++) {
    int *m = m24 + 24 * id;
    std::memset(m, 0, 24 * sizeof(int));
    if (id == 0) continue;
    m[0] = 1;
    m[1] = c->lvl[id];
    for (int d = 0; d < 3; d++) m[2 + d] = c->ix[3 * id + d];
    m[5] = c->par[id];
    for (int k = 0; k < 8; k++) m[6 + k] = c->chl[8 * id + k];
    for (int k = 0; k < 6; k++) m[14 + k] = c->nbr[6 * id + k];
    m[20] = c->nc[id];
  }
  return A5G_OK;
}

int a5g3_export_levels(a5g3_ctx *c, int *counts, int *ids, int cap, int *n_out) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  int k = 0;
  for (int l = c->min_lvl; l <= c->max_lvl; l++) {
    const int q = c->li(l), n = c->lv_n[q];
    const bool leaf = l == c->max_lvl;
    if (counts) {
      counts[3 * q] = n;
      counts[3 * q + 1] = leaf ? n : 0;
      counts[3 * q + 2] = leaf ? 0 : n;
    }
    for (int pass = 0; pass < 2; pass++)  // ids, then leaves or parents
      for (int t = 0; t < n; t++) {
        if (ids && k < cap) ids[k] = c->lv_ids[c->lv_off[q] + t];
        k++;
      }
  }
  if (n_out) *n_out = k;
  return A5G_OK;
}

int a5g3_set_table(a5g3_ctx *c, int n_rows, int n_cols, double x_min, double inv_dx, const double *rc) {
  if (!c || !rc || n_rows < 2 || n_cols != 4) return fail3(A5G_EINVAL, "bad table (n_rows >= 2, 4 columns)");
  if (c->d_lt) cudaFree(c->d_lt);
  c->d_lt = nullptr;
  c->h_lt.assign(rc, rc + (size_t)n_rows * n_cols);
  CK3(cudaMalloc((void **)&c->d_lt, c->h_lt.size() * sizeof(double)));
  CK3(cudaMemcpy(c->d_lt, rc, c->h_lt.size() * sizeof(double), cudaMemcpyHostToDevice));
  {
    // FP32 copy for the lookups of the mixed form
    std::vector<float> t32(c->h_lt.size());
    for (size_t k = 0; k < t32.size(); k++) t32[k] = (float)c->h_lt[k];
    if (c->d_lt32) cudaFree(c->d_lt32);
    c->d_lt32 = nullptr;
    CK3(cudaMalloc((void **)&c->d_lt32, t32.size() * sizeof(float)));
    CK3(cudaMemcpy(c->d_lt32, t32.data(), t32.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  c->lt_rows = n_rows;
  c->lt_xmin = x_min;
  c->lt_inv_dx = inv_dx;
  drop_graph(c);
  return A5G_OK;
}

int a5g3_set_precision(a5g3_ctx *c, int precision, const a5g_mg_schedule *sched) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  if (precision != A5G_FP64 && precision != A5G_MIXED) return fail3(A5G_EINVAL, "precision must be A5G_FP64 or A5G_MIXED");
  a5g_mg_schedule s{1, 2, 2, c->p.n_cycle_base, 1};
  if (sched) s = *sched;
  if (s.fmg < 0 || s.fmg > 1 || s.n_cycle_down < 1 || s.n_cycle_up < 1 || s.n_cycle_base < 1 || s.n_corr < 1 ||
      s.n_cycle_down > 8 || s.n_cycle_up > 8 || s.n_cycle_base > 64 || s.n_corr > 8)
    return fail3(A5G_EINVAL, "bad schedule (fmg 0/1, cycles 1..8, base 1..64, corrections 1..8)");
  if (precision == A5G_MIXED && !c->d_c32) {
    const size_t n = (size_t)3 * c->cap * SLOT3;
    if (cudaMalloc((void **)&c->d_c32, n * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail3(A5G_ENOMEM, "device allocation of the FP32 multigrid storage failed");
    }
    // defined contents everywhere (ghost cells of coarse rhs are carried along)
    CK3(cudaMemsetAsync(c->d_c32, 0, n * sizeof(float), c->stream));
  }
  c->precision = precision;
  c->sched = s;
  drop_graph(c);
  return A5G_OK;
}

int a5g3_get_precision(a5g3_ctx *c, int *precision, a5g_mg_schedule *sched) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  if (precision) *precision = c->precision;
  if (sched) *sched = c->sched;
  return A5G_OK;
}

int a5g3_set_init_cond(a5g3_ctx *c, double bg, int n_seeds, const double *r0, const double *r1, const double *dens,
                       const double *width, const int *falloff) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  if (n_seeds < 0 || n_seeds > 8 || (n_seeds > 0 && (!r0 || !r1 || !dens || !width || !falloff)))
    return fail3(A5G_EINVAL, "0..8 seeds with all arrays");
  Seeds3 S{};
  S.n = n_seeds;
  S.bg = bg;
  for (int s = 0; s < n_seeds; s++) {
    for (int d = 0; d < 3; d++) {
      S.r0[s][d] = r0[3 * s + d];
      S.r1[s][d] = r1[3 * s + d];
    }
    S.dens[s] = dens[s];
    S.width[s] = width[s];
    S.falloff[s] = falloff[s];
  }
  k3_init<<<c->n_all(), NTH3, 0, c->stream>>>(c->run(), c->all_ids(), S);
  return launched(c);
}

int a5g3_upload_cc(a5g3_ctx *c, int iv, const double *h) {
  if (!c || !h || iv < 0 || iv >= NV3) return fail3(A5G_EINVAL, "bad argument");
  CK3(cudaMemcpyAsync(c->d_cc + (size_t)iv * c->cap * SLOT3, h, (size_t)c->cap * SLOT3 * sizeof(double),
                      cudaMemcpyHostToDevice, c->stream));
  CK3(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}
int a5g3_download_cc(a5g3_ctx *c, int iv, double *h) {
  if (!c || !h || iv < 0 || iv >= NV3) return fail3(A5G_EINVAL, "bad argument");
  CK3(cudaMemcpyAsync(h, c->d_cc + (size_t)iv * c->cap * SLOT3, (size_t)c->cap * SLOT3 * sizeof(double),
                      cudaMemcpyDeviceToHost, c->stream));
  CK3(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}
int a5g3_upload_fc(a5g3_ctx *c, int d, int f, const double *h) {
  if (!c || !h || d < 0 || d > 2 || f < 0 || f >= NF3) return fail3(A5G_EINVAL, "bad argument");
  CK3(cudaMemcpyAsync(c->d_fc + ((size_t)d * NF3 + f) * c->cap * FSLOT3, h, (size_t)c->cap * FSLOT3 * sizeof(double),
                      cudaMemcpyHostToDevice, c->stream));
  CK3(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}
int a5g3_download_fc(a5g3_ctx *c, int d, int f, double *h) {
  if (!c || !h || d < 0 || d > 2 || f < 0 || f >= NF3) return fail3(A5G_EINVAL, "bad argument");
  CK3(cudaMemcpyAsync(h, c->d_fc + ((size_t)d * NF3 + f) * c->cap * FSLOT3, (size_t)c->cap * FSLOT3 * sizeof(double),
                      cudaMemcpyDeviceToHost, c->stream));
  CK3(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}

int a5g3_tree_copy_cc(a5g3_ctx *c, int a, int b) {
  if (!c || a < 0 || a >= NV3 || b < 0 || b >= NV3) return fail3(A5G_EINVAL, "bad argument");
  k3_copy2<<<grid_for(c->cap * SLOT3 / 2), NTH3, 0, c->stream>>>(c->run(), a, b, -1, -1);
  return launched(c);
}
static int with_dt(a5g3_ctx *c, double dt) {
  if (!(dt > 0)) return fail3(A5G_EINVAL, "dt must be > 0");
  k3_set_dt<<<1, 1, 0, c->stream>>>(c->d_scal, dt);
  return launched(c);
}
int a5g3_fluxes_koren(a5g3_ctx *c, double dt) {
  int r = ready(c);
  if (r || (r = with_dt(c, dt))) return r;
  k3_fluxes<double><<<c->count(c->max_lvl), NTH3, 0, c->stream>>>(c->run(), c->ids(c->max_lvl));
  return launched(c);
}
int a5g3_update_solution(a5g3_ctx *c, double dt) {
  int r = ready(c);
  if (r || (r = with_dt(c, dt))) return r;
  k3_update<double, false><<<c->count(c->max_lvl), NTH3, 0, c->stream>>>(c->run(), c->ids(c->max_lvl));
  return launched(c);
}
int a5g3_restrict_tree(a5g3_ctx *c, int iv) {
  if (!c || iv < 0 || iv >= NV3) return fail3(A5G_EINVAL, "bad argument");
  enq_restrict(c, iv, -1);
  return launched(c);
}
int a5g3_gc_tree(a5g3_ctx *c, int iv) {
  if (!c || iv < 0 || iv >= NV3) return fail3(A5G_EINVAL, "bad argument");
  enq_gc_all(c, iv, -1, 0);
  return launched(c);
}
int a5g3_average_dens(a5g3_ctx *c) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  k3_average<<<grid_for(c->cap * SLOT3), NTH3, 0, c->stream>>>(c->run());
  return launched(c);
}
int a5g3_compute_fld(a5g3_ctx *c, int no_guess) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  enq_compute_fld(c, no_guess != 0);
  return launched(c);
}
int a5g3_fmg(a5g3_ctx *c, int set_residual, int first_call) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  enq_fmg(c, set_residual != 0, first_call != 0);
  return launched(c);
}
int a5g3_vcycle(a5g3_ctx *c, int max_lvl, int set_residual) {
  if (!c || max_lvl < c->min_lvl || max_lvl > c->max_lvl) return fail3(A5G_EINVAL, "bad argument");
  enq_vcycle(c, c->mg64(), c->sweeps64(), max_lvl, set_residual != 0, false);
  return launched(c);
}
int a5g3_set_rhs(a5g3_ctx *c) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  k3_set_rhs<<<c->count(c->max_lvl), NTH3, 0, c->stream>>>(c->run(), c->ids(c->max_lvl));
  return launched(c);
}
int a5g3_fld_from_pot(a5g3_ctx *c) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  k3_fld<<<c->n_all(), NTH3, 0, c->stream>>>(c->run(), c->all_ids());
  return launched(c);
}

static int reduce(a5g3_ctx *c, int kind, int iv, double *out, int n_out) {
  const int hi = c->max_lvl, nb = c->count(hi);
  k3_reduce_boxes<<<nb, NTH3, 0, c->stream>>>(c->run(), c->ids(hi), kind, iv);
  k3_reduce_final<<<1, NTH3, 0, c->stream>>>(c->run(), nb, kind);
  CK3(cudaGetLastError());
  CK3(cudaMemcpyAsync(c->h_red, c->d_scal + S_RED, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK3(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < n_out; q++) out[q] = c->h_red[q];
  return A5G_OK;
}
int a5g3_tree_max_cc(a5g3_ctx *c, int iv, double *out) {
  if (!c || !out || iv < 0 || iv >= NV3) return fail3(A5G_EINVAL, "bad argument");
  return reduce(c, 1, iv, out, 1);
}
int a5g3_tree_min_cc(a5g3_ctx *c, int iv, double *out) {
  if (!c || !out || iv < 0 || iv >= NV3) return fail3(A5G_EINVAL, "bad argument");
  return reduce(c, 2, iv, out, 1);
}
int a5g3_dt_reductions(a5g3_ctx *c, double *out3) {
  if (!c || !out3) return fail3(A5G_EINVAL, "bad argument");
  return reduce(c, 0, 0, out3, 3);
}

// LT_get_col (fosito/m_lookup_table.f90:107-125, 154-161) on the host copy
static double host_col(const a5g3_ctx *c, int col, double x) {
  const double frac = (x - c->lt_xmin) * c->lt_inv_dx;
  int ix;
  double fr;
  if (frac < 2.0e9 && frac > -2.0e9) {
    ix = (int)std::ceil(frac);
    fr = ix - frac;
  } else {
    ix = frac > 0 ? c->lt_rows : 0;
    fr = 0;
  }
  if (ix < 1) {
    ix = 1;
    fr = 1;
  } else if (ix >= c->lt_rows) {
    ix = c->lt_rows - 1;
    fr = 0;
  }
  const double *v = c->h_lt.data() + (size_t)c->lt_rows * col;
  return fr * v[ix - 1] + (1 - fr) * v[ix];
}

// get_max_dt (src/streamer_3d.f90:274-305)
int a5g3_get_max_dt(a5g3_ctx *c, double *dt) {
  int r = ready(c);
  if (r) return r;
  if (!dt) return fail3(A5G_EINVAL, "null argument");
  double red[3];
  if ((r = a5g3_dt_reductions(c, red))) return r;
  const double max_fld = red[0], min_fld = red[1], max_dns = red[2];
  const double dr_min = std::ldexp(c->p.dr_base, -(c->max_lvl - 1));
  const double mobility = host_col(c, C_MOB, max_fld), max_mobility = host_col(c, C_MOB, min_fld);
  const double diff_coeff = host_col(c, C_DIF, max_fld), alpha = host_col(c, C_ALPHA, max_fld);
  const double dt_cfl = dr_min / (mobility * max_fld);
  const double dt_dif = 0.25 * (dr_min * dr_min) / diff_coeff;
  const double dt_drt = UC_EPS0 / (UC_ELEM_CHARGE * max_mobility * max_dns);
  const double dt_alpha = 1 / std::max(mobility * max_fld * alpha, 2.220446049250313e-16);
  double m = std::min(std::min(1 / (1 / dt_cfl + 1 / dt_dif), dt_alpha), c->p.dt_max);
  if (c->p.use_drt) m = std::min(m, dt_drt);
  *dt = 0.5 * m;
  return A5G_OK;
}

int a5g3_step(a5g3_ctx *c, double dt) {
  int r = ready(c);
  if (r || (r = with_dt(c, dt))) return r;
  if (!c->exec) {
    CK3(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    enq_step(c);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) return fail3(A5G_ECUDA, std::string("step capture: ") + cudaGetErrorString(e));
    c->graph = g;
    CK3(cudaGraphInstantiate(&c->exec, c->graph, 0));
  }
  CK3(cudaGraphLaunch(c->exec, c->stream));
  return A5G_OK;
}

int a5g3_sync(a5g3_ctx *c) {
  if (!c) return fail3(A5G_EINVAL, "null context");
  CK3(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}

int a5g3_stream(a5g3_ctx *c, void **s) {
  if (!c || !s) return fail3(A5G_EINVAL, "null argument");
  *s = (void *)c->stream;
  return A5G_OK;
}

}  // extern "C"
