// a5g — sm_100a device path for a5_streamer's per-timestep work (2D).
//
// Execution model. The trees of the streamer workloads are small (a few
// thousand to a few hundred thousand cells) and every multigrid half-sweep,
// ghost fill or restriction is a dependency point across the boxes of a
// level: one step holds about a thousand of them. Launching a kernel (or
// crossing a grid-wide barrier) per phase would make the step launch-bound.
// Instead one persistent thread block runs a whole operation -- up to a full
// time step -- for one run, with __syncthreads() between phases; independent
// runs are batched as one block each in the same launch. All box data stay
// resident in device memory (L2-resident for these sizes) between calls.
//
// Thread mapping: a block of NTHR threads is split into groups of GT = 64
// threads; a group owns one box at a time (one thread per interior cell of
// an 8x8 box, one per ghost cell, or one per face), and the groups stride
// over the box list of the current phase.
//
// Arithmetic is IEEE double with --fmad=false, so every expression rounds as
// in the reference's Fortran (compiled for x86-64 without FMA) and as in the
// CPU oracle; each device routine cites the reference routine it follows.
#include "../../include/a5g.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

namespace {

constexpr int NC = 8;                 // box_size on levels >= 1
constexpr int SLOT = (NC + 2) * (NC + 2);
constexpr int FSLOT = (NC + 1) * NC;
constexpr int GT = 64;                // threads per box group
constexpr int NTHR = 512;             // threads per block
constexpr int NGRP = NTHR / GT;
constexpr int MAXLEV = 40;            // levels min_lvl..max_lvl+1

// Variable indices, src/m_streamer.f90:17-43 (0-based).
enum { I_ELEC = 0, I_PION, I_ELEC_OLD, I_PION_OLD, I_PHI, I_FLD, I_RHS, I_PHO, I_EPS };
enum { F_ELEC = 0, F_FLD = 1 };
enum { C_MOB = 0, C_DIF = 1, C_ALPHA = 2, C_ETA = 3 };
// Ghost-cell kinds: refinement-boundary / physical-boundary routine pairs.
enum { GC_LIM = 0, GC_INTERP = 1, GC_PHI = 2 };

// fosito/m_units_constants.f90:201-202
constexpr double UC_EPS0 = 8.8541878176e-12;
constexpr double UC_ELEM_CHARGE = 1.6022e-19;

struct BoxMeta {
  int lvl, nc, ix0, ix1;
  int parent, ch[4], nb[4], p0, p1, p2;
  double dr, r0, r1, p3;
};
static_assert(sizeof(BoxMeta) == 96, "BoxMeta layout");

// Plan record of one box, built on the host once per topology (build_plans):
// slot bases (id * SLOT) of the box, its parent (-1: none), its neighbours per
// side (NBR_RB at a refinement boundary, NBR_PHYS at a physical one), the
// parent's neighbours where the box is at a refinement boundary, and its
// children (0: none); its offset in the parent (cells), its first global i
// index, list membership flags, r_min(1) and dr. A second set of records
// addresses the compact shared-memory copy of the multigrid variables
// (bases into that copy; gbase keeps the device-memory slot base).
struct __align__(16) BoxRec {
  int base, pbase;
  int nb[4];
  int pnb[4];
  int ch[4];
  int o0, o1, gi0, flags;
  double r0, dr;
  int gbase, pad;  // slot base in device memory (= base for the device-memory records)
};
static_assert(sizeof(BoxRec) == 96, "plan layout");
constexpr int NBR_RB = -1, NBR_PHYS = -2;
constexpr int CF_LEAF = 1, CF_PARENT = 2;

struct RunDev {
  int capacity, min_lvl, max_lvl, lvls_max;
  int coord, n_cycle_base, nlev, pad0;
  int lv_off[3][MAXLEV + 1];   // [ids|leaves|parents][level index] -> start in lists
  int new_off[MAXLEV + 1];     // new-box lists for prolong_new
  int *lists;
  int *new_lists;
  BoxMeta *meta;
  double *cc, *fx, *fy;
  const double *tbl;
  int tbl_rows, pad1;
  double tbl_xmin, tbl_inv_dx;
  double applied_voltage, domain_len_z, epsilon_diel;
  double ref_init_time, crv_refine;
  int n_seeds, pad2;
  double seed_r0[8][2], seed_r1[8][2], seed_width[8];
  // plans, per level index
  int bx_off[MAXLEV + 1], pb_off[MAXLEV + 1];
  int lv_nc[MAXLEV], pad3;
  double lv_dr[MAXLEV];
  const BoxRec *boxes;
  const BoxRec *sboxes;        // records addressing the shared-memory copy
  // cell plans and cylindrical weights of the shared-memory solve, built on
  // the host per topology: level index li uses block cplan_blk[li] (2 NTHR
  // entries), -1 where the level's colours do not fit one cell per thread
  const int4 *cplan;
  const double2 *cwts;
  int cplan_blk[MAXLEV];
  const int *pbx;
  int smem_doubles;            // per multigrid variable; 0: tree does not fit
  int pad4;
  double *scal;                // dt reductions out
  int *flags;                  // refinement flags out
  int *status;
  // photoionization (see "Photoionization" below)
  int n_ids;                   // max_id + 1
  int ph_enabled, ph_team, ph_lvl, ph_rows, ph_cap;
  double ph_coeff, ph_num_photons, ph_xmin, ph_inv_dx, ph_frac;
  const double *ph_tbl;        // absorption distance per table row
  int *ph_rng;                 // master generator state (4 int32)
  int *ph_ncr;                 // photons created per cell (capacity * SLOT)
  int *ph_cnt;                 // photons absorbed per cell (capacity * SLOT)
  int *ph_ipart;               // photon counts, then first numbers (boxes | team)
  double *ph_part;             // sums of the production (boxes | team)
  double *ph_u;                // uniform number drawn per leaf cell
  struct PhScal *ph_scal;
  const struct MzJump *ph_jump;
  const struct PhBox *ph_boxes;
  // mixed precision (a5g_set_precision): schedule of the FP32 correction
  // solve, FP32 storage when the tree does not fit in shared memory, FP32
  // copy of the transport table
  int mx_enabled, mx_fmg, mx_sw_down, mx_sw_up, mx_sw_base, mx_n_corr;
  int mx_smem;                 // floats per variable of the shared-memory copy; 0: cc32
  int mx_pad;
  float *cc32;
  const float *tbl32;
  // block state of the device-driven loop (a5g_batch): [0] dt of the block,
  // [1] simulated time, [2] end time, [3] 1 while the run is active
  double *blk;
  double dr_min, dt_max;       // finest cell size of the tree; ST_dt_max
  int use_drt;
  // dielectric runs (eps not identically 1): the multigrid tags each box
  // (tags[id]: TAG_NORMAL / TAG_DIEL) and uses the eps operators on
  // dielectric boxes; such runs take the device-memory multigrid path
  int diel;
  int *tags;
  // partial sums of a5g_tree_sum_cc, one per team thread (capacity doubles)
  double *sumbuf;
  // level-set boundaries of the multigrid (a5g_set_level_set): level-set
  // function and boundary value per cell, slot layout; has_lsf: set
  const double *lsf, *bval;
  int has_lsf, pad6;
  int uniform_lvl;             // > 0: uniform refinement to this level
  int local_cells;             // grid mode: levels of at most this many cells on one block
  // grid mode (a5g_set_ctas): barrier words of the run's block group
  // ([0] arrivals, [1] generation, [2] abort), the cycle bound of a barrier
  // wait, and per-block partial reductions (4 doubles per block)
  unsigned *gbar;
  long long gbudget;
  double *gred;
};
constexpr int TAG_NORMAL = 1, TAG_DIEL = 2, TAG_LSF = 3;

// Scalars of one photoionization call: photons created, the factor fac
// of PH_set_src_2d and the master generator state at the start of the call.
struct PhScal {
  long long n_used;
  double fac;
  int st0[4];
  int n_boxes;   // leaf boxes on levels >= 1, ranked in photon-number order
  int pad;
};
// Jump of 2^b draws of the master generator (see mz_advance).
struct MzJump {
  unsigned int m[9];
  unsigned int a, c;
};
constexpr int MZ_NJUMP = 40;
constexpr int PH_THREADS = 256;  // threads per block of the absorption kernel
// Resident absorption blocks per SM the register allocation is bounded for
// (8 x 256 threads: 32 registers a thread, a few spilled). The loop is
// latency-bound (L1/L2 loads, atomics); with twice the warps of the
// unbounded allocation (58 registers, 4 blocks) the 148-run batched step
// took 1.44 ms instead of 1.58 ms (6 blocks: 1.47 ms).
constexpr int PH_BLOCKS_PER_SM = 8;
// Layout of a run's jump table: MZ_NJUMP jumps of 2^b draws; the jumps of
// 4t draws, t < PH_THREADS (a thread of an absorption block from its block's
// generator); the jump of 8W draws (the master's advance per step, W the
// team); the jumps of 4W + 4 PH_THREADS b draws, b < ceil(W / PH_THREADS)
// (absorption block b from the master).
constexpr int MZ_JTHR = MZ_NJUMP, MZ_JSTEP = MZ_JTHR + PH_THREADS, MZ_JBLK = MZ_JSTEP + 1;
// Per box geometry for the absorption-location descent (a$D_get_loc).
struct PhBox {
  double r0, r1, dr;
  int ch[4];
  int lvl, nc;
};
static_assert(sizeof(PhBox) == 48, "PhBox layout");

enum OpCode {
  OP_COPY = 1, OP_FLUXES, OP_CONSISTENT, OP_UPDATE, OP_RESTRICT, OP_GC, OP_AVERAGE,
  OP_COMPUTE_FLD, OP_FMG, OP_FLD_FROM_POT, OP_DT_RED, OP_REF_FLAGS, OP_PROLONG_NEW,
  OP_STEP, OP_NOP, OP_PH_SOURCE, OP_PH_DEPOSIT, OP_STEP_MIXED, OP_COMPUTE_FLD_MIXED, OP_BLOCK_DT,
  OP_VCYCLE, OP_TREE_RED
};
struct Op {
  int code, i0, i1, i2;
  double d0, d1;
};

__constant__ int c_nb_dix[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
__constant__ int c_ch_dix[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
__constant__ int c_ch_adj_nb[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};

// ---------------------------------------------------------------------------
// Accessors. Box `id` of variable v: slot (v * capacity + id); the box's own
// (nc+2)^2 values are stored i-fastest with row length nc+2.
__device__ __forceinline__ double *CC(const RunDev &R, int v, int id) {
  return R.cc + ((size_t)v * R.capacity + id) * SLOT;
}
__device__ __forceinline__ double *FX(const RunDev &R, int f, int id) {
  return R.fx + ((size_t)f * R.capacity + id) * FSLOT;
}
__device__ __forceinline__ double *FY(const RunDev &R, int f, int id) {
  return R.fy + ((size_t)f * R.capacity + id) * FSLOT;
}
// max / min with the operand order of Fortran's max / min (NaN handling)
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

// fx(i, j): i in 1..nc+1, j in 1..nc;  fy(i, j): i in 1..nc, j in 1..nc+1
__device__ __forceinline__ int fxi(int i, int j, int nc) { return (i - 1) + (nc + 1) * (j - 1); }
__device__ __forceinline__ int fyi(int i, int j, int nc) { return (i - 1) + nc * (j - 1); }

__device__ __forceinline__ int list_n(const RunDev &R, int kind, int lvl) {
  int li = lvl - R.min_lvl;
  if (li < 0 || li >= R.nlev) return 0;
  return R.lv_off[kind][li + 1] - R.lv_off[kind][li];
}
__device__ __forceinline__ const int *list_p(const RunDev &R, int kind, int lvl) {
  return R.lists + R.lv_off[kind][lvl - R.min_lvl];
}
// Contiguous list of a kind over levels [lo, hi]
__device__ __forceinline__ void list_range(const RunDev &R, int kind, int lo, int hi,
                                           const int *&p, int &n) {
  lo = max(lo, R.min_lvl);
  hi = min(hi, R.max_lvl);
  if (hi < lo) { p = R.lists; n = 0; return; }
  int a = R.lv_off[kind][lo - R.min_lvl], b = R.lv_off[kind][hi - R.min_lvl + 1];
  p = R.lists + a;
  n = b - a;
}

// ---------------------------------------------------------------------------
// Execution group of a run. A run executes on one thread block, or in grid
// mode (a5g_set_ctas, for trees too large for one SM) on `size` co-resident
// blocks of one cooperative launch. Every phase is a flat loop of the group's
// threads over its items -- thread TID() of NTH() starts at item TID() and
// strides by NTH() -- and phases are separated by PSYNC(): a block barrier,
// or in grid mode a grid barrier whose wait is bounded (A5G_TIMEOUT). The
// state is per block, in shared memory, set at kernel entry (stage_run).
struct GroupCtl {
  int size;          // blocks of the run's group
  int rank;          // this block's rank in the group
  int tid0;          // rank * NTHR
  int nth;           // size * NTHR
  unsigned *bar;     // [0] arrivals, [1] generation, [2] abort
  long long budget;  // SM clock cycles one barrier wait may take
  int *status;
  double *red;       // per-block partial reductions (4 doubles per block)
};
__shared__ GroupCtl s_grp;

__device__ __forceinline__ int TID() { return s_grp.tid0 + (int)threadIdx.x; }
__device__ __forceinline__ int NTH() { return s_grp.nth; }
// the one thread of the group that writes a run's scalars
__device__ __forceinline__ bool LEAD() { return s_grp.tid0 == 0 && threadIdx.x == 0; }

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
  if (s_grp.size > 1) grid_sync();
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
// A box the multigrid treats with the level-set operators (its tag).
__device__ __forceinline__ bool lsf_box(const RunDev &R, const BoxRec &B) {
  return R.has_lsf && R.tags[B.gbase / SLOT] == TAG_LSF;
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

// Kinds of a ghost neighbour: copy of s0 (same-level neighbour or Neumann
// wall), refinement boundary (mg$D_sides_rb after a$D_gc_prolong0:
// 0.5 s0 + own - 0.25 (a + b), s0 the parent cell), grounded wall (-own),
// applied potential (2 V - own); sides_bc_pot (src/streamer_2d.f90:620-638).
enum { GK_COPY = 0, GK_RB = 1, GK_NEG = 2, GK_TOP = 3 };

// A cell plan as an int4: x = cell address (-1: none), y / z = first source
// of the x / y ghost neighbour, w = i | j << 8 | x kind << 16 | y kind << 18.

// First source and kind of side ghost (side, k) of box B (as phi_ghost).
__host__ __device__ __forceinline__ void ghost_src(const BoxRec &B, int nc, int ncg, int side, int k, int &s0,
                                          int &kind) {
  const int dim = side >> 1;
  const bool low = (side & 1) == 0;
  const int nbb = B.nb[side];
  const int ix = low ? 1 : nc;
  if (nbb > 0) {
    s0 = nbb + (dim == 0 ? (low ? nc : 1) + ncg * k : k + ncg * (low ? nc : 1));
    kind = GK_COPY;
  } else if (nbb == NBR_RB) {
    const int ig = ix - (low ? 1 : -1);
    const int h1 = (ig + 1) >> 1, h2 = (k + 1) >> 1;
    s0 = B.pbase + (dim == 0 ? (B.o0 + h1) + ncg * (B.o1 + h2) : (B.o0 + h2) + ncg * (B.o1 + h1));
    kind = GK_RB;
  } else {
    s0 = B.base + (dim == 0 ? ix + ncg * k : k + ncg * ix);
    kind = side == 2 ? GK_NEG : (side == 3 ? GK_TOP : GK_COPY);
  }
}

__host__ __device__ __forceinline__ int4 make_plan(const BoxRec &B, int nc, int ncg, int i, int j) {
  int4 c;
  c.x = B.base + i + ncg * j;
  int xk, yk;
  ghost_src(B, nc, ncg, i == 1 ? 0 : 1, j, c.y, xk);
  ghost_src(B, nc, ncg, j == 1 ? 2 : 3, i, c.z, yk);
  c.w = i | (j << 8) | (xk << 16) | (yk << 18);
  return c;
}

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

// box_gsrb_clpl weights (i+ioff-1)/(i+ioff-1/2) and (i+ioff)/(i+ioff-1/2)
__host__ __device__ __forceinline__ void cyl_weights(int gi, double &rf1, double &rf2) {
  const double den = gi - 0.5;
  rf1 = (gi - 1) / den;
  rf2 = gi / den;
}

extern __shared__ double g_dsmem[];

// The plan slots lead the dynamic shared memory of a shared-memory solve:
// 2 NTHR int4 cell plans, then (cylindrical runs) 2 NTHR double2 weights.
constexpr int PLAN_DOUBLES = 2 * NTHR * 2;     // doubles taken by the cell plans
constexpr int WTS_DOUBLES = 2 * NTHR * 2;      // doubles taken by the weights
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
  if (s_grp.size == 1) return lc;
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
// the leaves where it is first needed (compute_fld).
template <class T>
__device__ void p_fmg_in(const RunDev &R, const MGV<T> &M, bool set_residual, bool first_call,
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
__device__ __forceinline__ void mg_staged(const RunDev &R, F &&body);

__device__ void p_fmg(const RunDev &R, bool set_residual, bool first_call, bool leaf_rhs) {
  mg_staged(R, [&](const MGV<double> &M) { p_fmg_in(R, M, set_residual, first_call, leaf_rhs); });
}

// mg$D_fas_vcycle(tree, mg, max_lvl, set_residual) on its own
// (afivo/src/m_aX_mg.f90:208-254): valid potential ghost cells on input and
// output; with set_residual the residual of levels min..max_lvl in tmp.
__device__ void p_vcycle_alone(const RunDev &R, int max_lvl, bool set_residual) {
  mg_staged(R, [&](const MGV<double> &M) {
    PlanFetch pf;
    p_vcycle(R, M, max_lvl, false, pf, R.max_lvl + 1);
    if (set_residual) p_residual_all(R, M, max_lvl);
    if (pf.li >= 0) cp_async_wait_all();
  });
}

// Runs body(M) on the multigrid variables: staged in shared memory when the
// tree fits, else in device memory (dielectric runs always in device memory).
template <class F>
__device__ __forceinline__ void mg_staged(const RunDev &R, F &&body) {
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
    body(M);
    stage_mg(R, M, VAR(R, MP), VAR(R, MR), VAR(R, MT), false);
  } else {
    MGV<double> M{VAR(R, MP), VAR(R, MR), VAR(R, MT), R.boxes, R.pbx, false, R.applied_voltage,
                  4, 4, 2 * R.n_cycle_base};
    body(M);
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
      if (B.flags & CF_LEAF) {
        rh = fac * (e[g] - pi[g]);
        res = rh - lap_at(R, R.applied_voltage, (const double *)phi, B, L.nc, L.ncg, i, j, inv_dr_sq);
        rhs[g] = rh;
        cr[sc] = (float)res;
      } else {
        rh = rhs[g];
        res = (double)cr[sc];
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
  const MGV<double> G{phi, VAR(R, MR), VAR(R, MT), R.boxes, R.pbx, false, R.applied_voltage, 0, 0, 0};
  for (int lvl = R.min_lvl; lvl <= R.max_lvl; lvl++) p_fill(R, G, lvl);
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
    if (s_grp.size > 1) {
      // grid mode: each block's values, combined by the lead after a barrier
      // (max and min are exact: any order gives the same result)
      double *g = s_grp.red + 4 * s_grp.rank;
      g[0] = mx;
      g[1] = mn;
      g[2] = me;
    }
  }
  if (s_grp.size > 1) {
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
constexpr unsigned int MZ_M = 2147483579u;
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

// Descriptor of one member of a launch of a5g_step_batch_static.
struct BatchSlot {
  const RunDev *run;
  Op op;
};

// Same work as a5g_run_kernel, with each block's run and operation read from
// a descriptor table (the fixed array below).
__global__ void __launch_bounds__(NTHR, 1) a5g_run_kernel_slots(const BatchSlot *slots) {
  __shared__ RunDev sR;
  stage_run(slots[blockIdx.x].run, sR, 1, 0);
  Op op = slots[blockIdx.x].op;
  run_op(sR, op);
}

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

// Descriptors of one launch of a5g_step_batch_static passed by value (as
// kernel parameters, at most SLOT_FILL per launch; 96 x 40 bytes stays under
// the classic 4 KiB parameter limit) and written to the fixed table, so that
// no host staging buffer or copy is involved.
constexpr int SLOT_FILL = 96;
struct SlotChunk {
  BatchSlot s[SLOT_FILL];
};
__global__ void a5g_fill_slots_kernel(BatchSlot *dst, SlotChunk chunk, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = chunk.s[k];
}

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

// Block state of every member of a device-driven batch gathered into one
// array (5 doubles per run: dt, time, end time, active, device status), so
// that the host reads a whole batch with a single copy.
__global__ void a5g_batch_gather_kernel(const RunDev *const *runs, int n, double *out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const RunDev *r = runs[k];
#pragma unroll
    for (int q = 0; q < 4; q++) out[5 * k + q] = r->blk[q];
    out[5 * k + 4] = (double)*r->status;
  }
}

}  // namespace

// Descriptor table of a5g_step_batch_static: a fixed device array, so that
// entry point needs no allocation. Host code must not pass this name to a
// kernel (on the host it only stands in for the symbol); its device address
// comes from cudaGetSymbolAddress.
static __device__ __align__(256) BatchSlot g_batch_scratch[A5G_STATIC_BATCH_MAX];

// ===========================================================================
// Host side: contexts and the C ABI.

static thread_local std::string g_err;

static int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}
#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return fail(e_ == cudaErrorMemoryAllocation ? A5G_ENOMEM : A5G_ECUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));              \
  } while (0)

struct a5g_ctx {
  a5g_params p{};
  cudaStream_t stream = nullptr;
  RunDev h{};
  RunDev *d_run = nullptr;
  int capacity = 0;
  int max_id = 0;
  bool has_tree = false, has_table = false;
  double *cc = nullptr, *fx = nullptr, *fy = nullptr;
  BoxMeta *meta = nullptr;
  int *lists = nullptr;
  size_t lists_cap = 0;
  int *new_lists = nullptr;
  size_t new_cap = 0;
  double *tbl = nullptr;
  double *scal = nullptr;
  int *flags = nullptr;
  int *status = nullptr;
  std::vector<double> h_tbl;
  int tbl_rows = 0, tbl_cols = 0;
  double tbl_xmin = 0, tbl_inv_dx = 0;
  long long n_leaf_cells = 0;
  int min_lvl = 0, max_lvl = 0;
  // plan storage
  BoxRec *p_sboxes = nullptr;
  size_t cap_sboxes = 0;
  size_t dyn_smem = 0;  // dynamic shared memory per launch (bytes)
  BoxRec *p_boxes = nullptr;
  int *p_pbx = nullptr;
  size_t cap_boxes = 0, cap_pbx = 0;
  int4 *p_cplan = nullptr;
  double2 *p_cwts = nullptr;
  size_t cap_cplan = 0, cap_cwts = 0;
  // photoionization storage
  bool has_ph_table = false;
  double *ph_tbl = nullptr;
  std::vector<double> h_ph_tbl;
  int *ph_rng = nullptr, *ph_ncr = nullptr, *ph_cnt = nullptr, *ph_ipart = nullptr;
  double *ph_part = nullptr, *ph_u = nullptr;
  PhScal *ph_scal = nullptr;
  MzJump *ph_jump = nullptr;
  PhBox *ph_boxes = nullptr;
  int ph_capacity = 0;   // capacity the per-box photon buffers are sized for
  size_t ph_boxes_cap = 0;
  // mixed precision
  int precision = 0;     // A5G_FP64 or A5G_MIXED
  a5g_mg_schedule sched{};
  float *tbl32 = nullptr;
  float *cc32 = nullptr;
  int cc32_cap = 0;      // box capacity cc32 is sized for
  int mx_smem_fit = 0;   // floats per variable of the shared-memory copy (0: does not fit)
  size_t dyn_smem32 = 0; // dynamic shared memory of a mixed-precision launch
  // dielectric runs: box tags (device), box sizes of the uploaded tree
  // (host, 0 for ids not in use) to check uploaded eps values
  int *tags = nullptr;
  std::vector<int> h_nc;
  // shared-memory staging of the multigrid (a5g_debug_set_staging can turn it off)
  bool allow_smem = true;
  int fit64 = 0, fit32 = 0;       // per-variable sizes when the tree fits, else 0
  size_t need64 = 0, need32 = 0;  // dynamic shared memory the staged solves take
  // partial sums of a5g_tree_sum_cc (one per box of the capacity)
  double *sumbuf = nullptr;
  // ordering of the batched steps with this context's own stream: recorded
  // on this stream before a batch that includes the context (the batch's
  // stream waits on it), and on the batch's stream after it (this stream
  // waits on it). Created with the context, so no batch call allocates.
  cudaEvent_t ev_order = nullptr;
  // grid mode (a5g_set_ctas): thread blocks per launch of the run's phases,
  // barrier words and per-block reduction slots
  int n_cta = 1;
  unsigned *gbar = nullptr;
  double *gred = nullptr;
  // level-set boundaries (a5g_set_level_set): two cell arrays of the box
  // capacity, grown with the box storage
  double *lsf = nullptr, *bval = nullptr;
};

// Shared-memory staging of the multigrid variables as allowed and as fits
// (never in grid mode: a block holds only part of the tree's work).
static void apply_staging(a5g_ctx *c) {
  const bool on = c->allow_smem && c->n_cta == 1 && !c->h.has_lsf;
  c->h.smem_doubles = on ? c->fit64 : 0;
  c->dyn_smem = on && c->fit64 ? c->need64 : 0;
  c->mx_smem_fit = on ? c->fit32 : 0;
  c->dyn_smem32 = on && c->fit32 ? c->need32 : 0;
  c->h.mx_smem = c->mx_smem_fit;
}

// Dynamic shared memory a step of this context's precision needs.
static size_t step_smem(const a5g_ctx *c) { return c->precision == A5G_MIXED ? c->dyn_smem32 : c->dyn_smem; }

// ---------------------------------------------------------------------------
// Plan builder: one BoxRec per box, level by level in list order, and the
// indices of the parent boxes per level (see "Plan-based operations").
// Leaf / parent status is list membership, as in every box loop of the
// reference (lvl_t%leaves / %parents), not "has children": the two differ on
// level lvls_max, whose lists a$D_adjust_refinement never rebuilds
// (afivo/src/m_aX_core.f90:478-515 calls set_leaves_parents for levels below
// lvls_max and for max_lvl+1 only).
struct HostPlans {
  std::vector<BoxRec> boxes, sboxes;
  std::vector<int4> cplan;      // per fitting level: 2 NTHR cell plans
  std::vector<double2> cwts;    // and their cylindrical weights
  int cplan_blk[MAXLEV];
  int smem_doubles = 0;  // doubles per variable of the compact shared-memory copy
  std::vector<int> pbx;
  int bx_off[MAXLEV + 1], pb_off[MAXLEV + 1];
  int lv_nc[MAXLEV];
  double lv_dr[MAXLEV];
};

static void host_child_offset(const BoxMeta &m, int &o0, int &o1) {
  if (m.lvl > 1) {
    o0 = ((m.ix0 - 1) & 1) * (m.nc >> 1);
    o1 = ((m.ix1 - 1) & 1) * (m.nc >> 1);
  } else {
    o0 = o1 = 0;
  }
}

static void build_plans(const std::vector<BoxMeta> &hm, const std::vector<std::vector<int>> &ids,
                        const std::vector<std::vector<int>> &leaves,
                        const std::vector<std::vector<int>> &parents, int min_lvl, int nlev,
                        double dr_base, HostPlans &P) {
  std::vector<char> is_leaf(hm.size(), 0), is_parent(hm.size(), 0);
  for (const auto &v : leaves)
    for (int id : v) is_leaf[id] = 1;
  for (const auto &v : parents)
    for (int id : v) is_parent[id] = 1;
  P.boxes.clear();
  P.pbx.clear();
  for (int li = 0; li < nlev; li++) {
    const int lvl = min_lvl + li;
    const int nc = lvl >= 1 ? NC : (NC >> (1 - lvl));
    P.lv_nc[li] = nc;
    P.lv_dr[li] = ids[li].empty() ? dr_base * std::pow(0.5, lvl - 1) : hm[ids[li][0]].dr;
    P.bx_off[li] = (int)P.boxes.size();
    P.pb_off[li] = (int)P.pbx.size();
    for (int id : ids[li]) {
      const BoxMeta &m = hm[id];
      BoxRec b{};
      b.base = id * SLOT;
      b.pbase = m.parent > 0 ? m.parent * SLOT : -1;
      for (int s = 0; s < 4; s++) {
        const int nid = m.nb[s];
        b.nb[s] = nid > 0 ? nid * SLOT : (nid == 0 ? NBR_RB : NBR_PHYS);
        const int pn = (nid == 0 && m.parent > 0) ? hm[m.parent].nb[s] : 0;
        b.pnb[s] = pn > 0 ? pn * SLOT : 0;
      }
      for (int q = 0; q < 4; q++) b.ch[q] = m.ch[q] > 0 ? m.ch[q] * SLOT : 0;
      host_child_offset(m, b.o0, b.o1);
      b.gi0 = (m.ix0 - 1) * nc;
      b.flags = (is_leaf[id] ? CF_LEAF : 0) | (is_parent[id] ? CF_PARENT : 0);
      b.r0 = m.r0;
      b.dr = m.dr;
      b.gbase = b.base;
      if (is_parent[id]) P.pbx.push_back((int)P.boxes.size());
      P.boxes.push_back(b);
    }
  }
  P.bx_off[nlev] = (int)P.boxes.size();
  P.pb_off[nlev] = (int)P.pbx.size();
  // compact shared-memory layout: boxes one after another, (nc+2)^2 values
  // each, starting at offset 2 so that no base is 0 (nb[] > 0 means a box)
  std::vector<int> sbase(hm.size(), 0);
  int off = 2;
  for (const BoxRec &b : P.boxes) {
    const int id = b.base / SLOT, ncg = hm[id].nc + 2;
    sbase[id] = off;
    off += ncg * ncg;
  }
  P.smem_doubles = (off + 1) & ~1;
  P.sboxes = P.boxes;
  auto sb = [&](int gb) { return gb > 0 ? sbase[gb / SLOT] : gb; };
  for (BoxRec &b : P.sboxes) {
    b.base = sbase[b.gbase / SLOT];
    b.pbase = b.pbase > 0 ? sbase[b.pbase / SLOT] : b.pbase;
    for (int q = 0; q < 4; q++) {
      b.nb[q] = sb(b.nb[q]);
      b.pnb[q] = sb(b.pnb[q]);
      b.ch[q] = sb(b.ch[q]);
    }
  }
  // Cell plans of every level whose colours have at most one cell per thread
  // (the per-thread slots make_level_plan fills), on the shared-memory
  // records: thread k takes cell item k & (half-1) of box k >> log2(half),
  // its colour-0 and colour-1 cells in plan slots 2k and 2k+1.
  P.cplan.clear();
  P.cwts.clear();
  for (int li = 0; li < MAXLEV; li++) P.cplan_blk[li] = -1;
  for (int li = 0; li < nlev; li++) {
    const int nc = P.lv_nc[li], ncg = nc + 2, half = (nc * nc) >> 1, hn = nc >> 1;
    const int sh = __builtin_ctz(nc), hsh = 2 * sh - 1;
    const int b0 = P.bx_off[li], nb = P.bx_off[li + 1] - b0;
    if (nb * half > NTHR) continue;
    P.cplan_blk[li] = (int)(P.cplan.size() / (2 * NTHR));
    for (int k = 0; k < NTHR; k++) {
      int4 c[2];
      c[0] = c[1] = make_int4(-1, 0, 0, 0);
      double2 w[2] = {make_double2(0, 0), make_double2(0, 0)};
      if (k < nb * half) {
        const BoxRec &B = P.sboxes[b0 + (k >> hsh)];
        const int item = k & (half - 1);
        const int j = (item >> (sh - 1)) + 1, m = item & (hn - 1);
        for (int p = 0; p < 2; p++) {
          c[p] = make_plan(B, nc, ncg, 2 * m + 2 - ((p + j) & 1), j);
          cyl_weights(B.gi0 + (c[p].w & 255), w[p].x, w[p].y);
        }
      }
      P.cplan.push_back(c[0]);
      P.cplan.push_back(c[1]);
      P.cwts.push_back(w[0]);
      P.cwts.push_back(w[1]);
    }
  }
}

template <class T>
static int upload_vec(a5g_ctx *c, T *&dev, size_t &cap, const std::vector<T> &v) {
  if (v.size() + 1 > cap) {
    cudaFree(dev);
    dev = nullptr;
    cap = std::max(v.size() + 1, 2 * cap);
    CK(cudaMalloc(&dev, cap * sizeof(T)));
  }
  if (!v.empty())
    CK(cudaMemcpyAsync(dev, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return A5G_OK;
}

// Host-only export of the plans of a topology (tests and diagnostics; no
// device needed). Level lists in the a5g_upload_tree format. Output arrays
// may be NULL. sizes[2] = boxes, parent boxes; boxes are written as raw
// 96-byte records; offs = bx_off[MAXLEV+1] then pb_off[MAXLEV+1].
extern "C" int a5g_debug_plans(int max_id, int min_lvl, int max_lvl, const int *meta16,
                               const double *geom4, const int *lvl_counts, const int *lvl_ids,
                               double dr_base, int *sizes, int *offs, void *boxes, int *pbx,
                               double *lv_dr, int *lv_nc) {
  const int nlev = max_lvl - min_lvl + 1;
  if (nlev < 1 || nlev + 1 > MAXLEV || max_id < 1) return fail(A5G_EINVAL, "bad tree");
  std::vector<BoxMeta> hm(max_id + 1);
  std::memset(hm.data(), 0, hm.size() * sizeof(BoxMeta));
  for (int id = 1; id <= max_id; id++) {
    const int *m = meta16 + 16 * id;
    if (!m[0]) continue;
    BoxMeta &b = hm[id];
    b.lvl = m[1]; b.ix0 = m[2]; b.ix1 = m[3]; b.parent = m[5];
    for (int k = 0; k < 4; k++) { b.ch[k] = m[6 + k]; b.nb[k] = m[10 + k]; }
    b.nc = m[14];
    b.dr = geom4[4 * id + 3]; b.r0 = geom4[4 * id]; b.r1 = geom4[4 * id + 1];
  }
  std::vector<std::vector<int>> lv_ids(nlev), lv_leaves(nlev), lv_parents(nlev);
  size_t k = 0;
  for (int li = 0; li < nlev; li++)
    for (int kind = 0; kind < 3; kind++)
      for (int q = 0; q < lvl_counts[3 * li + kind]; q++) {
        int id = lvl_ids[k++];
        if (kind == 0) lv_ids[li].push_back(id);
        if (kind == 1) lv_leaves[li].push_back(id);
        if (kind == 2) lv_parents[li].push_back(id);
      }
  HostPlans P;
  build_plans(hm, lv_ids, lv_leaves, lv_parents, min_lvl, nlev, dr_base, P);
  if (sizes) {
    sizes[0] = (int)P.boxes.size();
    sizes[1] = (int)P.pbx.size();
  }
  if (offs)
    for (int li = 0; li <= nlev; li++) {
      offs[li] = P.bx_off[li];
      offs[MAXLEV + 1 + li] = P.pb_off[li];
    }
  if (boxes) std::memcpy(boxes, P.boxes.data(), P.boxes.size() * sizeof(BoxRec));
  if (pbx) std::memcpy(pbx, P.pbx.data(), P.pbx.size() * sizeof(int));
  if (lv_dr) std::memcpy(lv_dr, P.lv_dr, nlev * sizeof(double));
  if (lv_nc) std::memcpy(lv_nc, P.lv_nc, nlev * sizeof(int));
  return A5G_OK;
}

// Largest dynamic shared memory a launch of the run kernels may use on the
// current device; raises the kernels' limit to it on first use.
static size_t dyn_smem_limit() {
  static std::mutex mu;
  static size_t lim[256] = {};
  static bool done[256] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return 0;
  std::lock_guard<std::mutex> lock(mu);
  if (!done[dev]) {
    done[dev] = true;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t stat = 0;
    constexpr int NF = 6;
    cudaFuncAttributes fa[NF];
    const void *fns[NF] = {(const void *)a5g_run_kernel, (const void *)a5g_step_kernel,
                           (const void *)a5g_run_kernel_slots, (const void *)a5g_photon_kernel,
                           (const void *)a5g_step_mixed_kernel, (const void *)a5g_batch_map_kernel};
    for (int k = 0; k < NF; k++)
      if (cudaFuncGetAttributes(&fa[k], fns[k]) == cudaSuccess)
        stat = std::max(stat, fa[k].sharedSizeBytes);
    size_t avail = optin > (int)stat ? (size_t)optin - stat : 0;
    bool ok = true;
    for (int k = 0; k < NF; k++)
      ok = ok && cudaFuncSetAttribute(fns[k], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)avail) == cudaSuccess;
    lim[dev] = ok ? avail : 0;
    cudaGetLastError();
  }
  return lim[dev];
}

static int push_run(a5g_ctx *c) {
  CK(cudaMemcpyAsync(c->d_run, &c->h, sizeof(RunDev), cudaMemcpyHostToDevice, c->stream));
  return A5G_OK;
}

static int check_status(a5g_ctx *c) {
  int st = 0;
  CK(cudaMemcpyAsync(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st != 0) {
    int z = 0;
    CK(cudaMemcpy(c->status, &z, sizeof(int), cudaMemcpyHostToDevice));
    // a barrier that gave up leaves its words mid-count: start clean
    if (st == A5G_TIMEOUT) CK(cudaMemset(c->gbar, 0, 4 * sizeof(unsigned)));
    return fail(st, st == A5G_TIMEOUT ? "a grid barrier wait ran out (A5G_TIMEOUT)"
                                      : "device reported status " + std::to_string(st));
  }
  return A5G_OK;
}

static Op mkop(int code, int i0 = 0, int i1 = 0, double d0 = 0) {
  Op o{};
  o.code = code;
  o.i0 = i0;
  o.i1 = i1;
  o.d0 = d0;
  return o;
}

// Operations whose phases run on the run's whole block group in grid mode;
// the others (photon sources, tree reductions) always take one block.
static bool grid_op(int code) { return code != OP_PH_SOURCE && code != OP_TREE_RED; }

static int launch_smem(a5g_ctx *c, const Op &op, size_t smem) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (!c->has_table) return fail(A5G_ESTATE, "no transport table set");
  if (c->n_cta > 1 && grid_op(op.code)) {
    // co-resident blocks of one cooperative launch (no staging: smem = 0)
    const RunDev *run = c->d_run;
    Op o = op;
    const RunDev *const *runs = nullptr;
    const Op *ops = nullptr;
    void *args[] = {(void *)&run, (void *)&o, (void *)&runs, (void *)&ops};
    CK(cudaLaunchCooperativeKernel((const void *)a5g_run_kernel, dim3(c->n_cta), dim3(NTHR), args, 0,
                                   c->stream));
    return A5G_OK;
  }
  a5g_run_kernel<<<1, NTHR, smem, c->stream>>>(c->d_run, op, nullptr, nullptr);
  CK(cudaGetLastError());
  return A5G_OK;
}
static int launch(a5g_ctx *c, const Op &op) { return launch_smem(c, op, c ? c->dyn_smem : 0); }

// Jumps of 2^b draws of the master generator (see mz_advance): the 3x3
// matrix of (s1, s2, s3) -> (s2, s3, s1 - s3) mod m and the affine map
// s4 -> 69069 s4 + 1013904243 mod 2^32, squared b times.
static void mz_jump_table(MzJump *J) {
  const unsigned long long m = MZ_M;
  unsigned long long M[9] = {0, 1, 0, 0, 0, 1, 1, 0, m - 1};
  unsigned int a = 69069u, cc = 1013904243u;
  for (int b = 0; b < MZ_NJUMP; b++) {
    for (int k = 0; k < 9; k++) J[b].m[k] = (unsigned int)M[k];
    J[b].a = a;
    J[b].c = cc;
    unsigned long long N[9];
    for (int r = 0; r < 3; r++)
      for (int q = 0; q < 3; q++)
        N[3 * r + q] = (M[3 * r] * M[q] % m + M[3 * r + 1] * M[3 + q] % m +
                        M[3 * r + 2] * M[6 + q] % m) % m;
    std::memcpy(M, N, sizeof(M));
    cc = a * cc + cc;
    a = a * a;
  }
}

// a followed by b (jumps are powers of one map, so the order does not matter)
static MzJump mz_compose(const MzJump &a, const MzJump &b) {
  const unsigned long long m = MZ_M;
  MzJump r;
  for (int i = 0; i < 3; i++)
    for (int q = 0; q < 3; q++)
      r.m[3 * i + q] = (unsigned int)(((unsigned long long)b.m[3 * i] * a.m[q] % m +
                                       (unsigned long long)b.m[3 * i + 1] * a.m[3 + q] % m +
                                       (unsigned long long)b.m[3 * i + 2] * a.m[6 + q] % m) % m);
  r.a = b.a * a.a;
  r.c = b.a * a.c + b.c;
  return r;
}
// The jump of k draws from the 2^b jumps.
static MzJump mz_power(const MzJump *J, unsigned long long k) {
  MzJump r{{1, 0, 0, 0, 1, 0, 0, 0, 1}, 1u, 0u};
  for (int b = 0; k != 0 && b < MZ_NJUMP; b++, k >>= 1)
    if (k & 1) r = mz_compose(r, J[b]);
  return r;
}
// A run's whole jump table (layout at MZ_JTHR), for a team of W threads.
static std::vector<MzJump> mz_run_table(long long W) {
  const int nblk = (int)((W + PH_THREADS - 1) / PH_THREADS);
  std::vector<MzJump> T(MZ_JBLK + nblk);
  mz_jump_table(T.data());
  for (int t = 0; t < PH_THREADS; t++) T[MZ_JTHR + t] = mz_power(T.data(), 4ull * t);
  T[MZ_JSTEP] = mz_power(T.data(), 8ull * (unsigned long long)W);
  for (int b = 0; b < nblk; b++)
    T[MZ_JBLK + b] = mz_power(T.data(), 4ull * (unsigned long long)W + 4ull * PH_THREADS * b);
  return T;
}

// Photon buffers sized for the current box capacity: per cell a draw, a
// first photon number and an absorption count; per box and per team thread
// scratch. At most num_photons + one per leaf cell are created (the expected
// total is at most num_photons and stochastic rounding adds at most one per
// cell); photon numbers must stay below 2^31.
static int ph_resize(a5g_ctx *c) {
  if (!c->p.photoi_enabled || c->capacity == c->ph_capacity) return A5G_OK;
  const size_t cells = (size_t)c->capacity * SLOT;
  const size_t src = (size_t)c->p.photoi_num_photons + (size_t)c->capacity * NC * NC + 1024;
  if (src > (size_t)INT_MAX) return fail(A5G_EINVAL, "photon numbers above 2^31");
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->ph_ncr);
  cudaFree(c->ph_cnt);
  cudaFree(c->ph_ipart);
  cudaFree(c->ph_part);
  cudaFree(c->ph_u);
  c->ph_ncr = c->ph_cnt = c->ph_ipart = nullptr;
  c->ph_part = c->ph_u = nullptr;
  if (cudaMalloc(&c->ph_ncr, cells * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->ph_cnt, cells * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->ph_ipart, 5 * (size_t)c->capacity * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->ph_part, 2 * (size_t)c->capacity * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->ph_u, cells * sizeof(double)) != cudaSuccess)
    return fail(A5G_ENOMEM, "cannot allocate photon buffers");
  CK(cudaMemsetAsync(c->ph_ncr, 0, cells * sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->ph_cnt, 0, cells * sizeof(int), c->stream));
  c->ph_capacity = c->capacity;
  RunDev &h = c->h;
  h.ph_ncr = c->ph_ncr;
  h.ph_cnt = c->ph_cnt;
  h.ph_ipart = c->ph_ipart;
  h.ph_part = c->ph_part;
  h.ph_u = c->ph_u;
  h.ph_cap = (int)src;
  return A5G_OK;
}

static int ph_ready(a5g_ctx *c) {
  if (!c->has_ph_table) return fail(A5G_ESTATE, "photoionization enabled but no photon table set");
  return A5G_OK;
}

// Dynamic shared memory of a5g_photon_kernel for a run: its box geometry
// table when that fits, else 0.
static size_t ph_smem_bytes(const a5g_ctx *c) {
  // box geometry and, per leaf box, its rank's first photon number and id
  const size_t need = (size_t)(c->max_id + 1) * (sizeof(PhBox) + 2 * sizeof(int));
  return need <= dyn_smem_limit() ? need : 0;
}

// Photon sources and absorption of one call (the deposit follows, either as
// its own launch or at the start of the step kernel).
static int ph_launch_source_absorb(a5g_ctx *c, double dt, int has_dt) {
  int r = launch(c, mkop(OP_PH_SOURCE, has_dt ? 1 : 0, 0, dt));
  if (r) return r;
  const size_t smem = ph_smem_bytes(c);
  dim3 grid((unsigned)((c->p.photoi_team + PH_THREADS - 1) / PH_THREADS), 1);
  a5g_photon_kernel<<<grid, PH_THREADS, smem, c->stream>>>(c->d_run, nullptr, nullptr, (int)smem);
  CK(cudaGetLastError());
  return A5G_OK;
}

extern "C" {

int a5g_internal_fail(int code, const char *msg) { return fail(code, msg ? msg : ""); }
const char *a5g_last_error(void) { return g_err.c_str(); }
int a5g_version(void) { return 1; }

int a5g_create(const a5g_params *p, a5g_ctx **out) {
  if (!p || !out) return fail(A5G_EINVAL, "null argument");
  *out = nullptr;
  if (p->box_size != NC) return fail(A5G_EINVAL, "box_size must be 8");
  if (p->coord != 0 && p->coord != 1) return fail(A5G_EINVAL, "coord must be 0 or 1");
  if (!(p->epsilon_diel > 0)) return fail(A5G_EINVAL, "epsilon_diel must be > 0");
  if (p->n_seeds < 0 || p->n_seeds > 8) return fail(A5G_EINVAL, "n_seeds must be 0..8");
  if (p->lvls_max < 1 || p->lvls_max > 30) return fail(A5G_EINVAL, "lvls_max must be 1..30");
  if (p->uniform_lvl < 0 || p->uniform_lvl > p->lvls_max)
    return fail(A5G_EINVAL, "uniform_lvl must be 0..lvls_max");
  if (!(p->dr_base > 0)) return fail(A5G_EINVAL, "dr_base must be > 0");
  if (p->photoi_enabled) {
    if (p->coord != 1)
      return fail(A5G_EINVAL, "photoionization is built for the cylindrical form only");
    if (p->photoi_team < 1 || p->photoi_num_photons < 0)
      return fail(A5G_EINVAL, "photoi_team must be >= 1 and photoi_num_photons >= 0");
  }
  a5g_ctx *c = new a5g_ctx();
  c->p = *p;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(A5G_ECUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  if (cudaMalloc(&c->d_run, sizeof(RunDev)) != cudaSuccess ||
      cudaMalloc(&c->scal, 16 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->status, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->gbar, 4 * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&c->gred, 4 * (size_t)A5G_MAX_CTAS * sizeof(double)) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_order, cudaEventDisableTiming) != cudaSuccess) {
    a5g_destroy(c);
    return fail(A5G_ENOMEM, "cudaMalloc failed");
  }
  cudaMemset(c->status, 0, sizeof(int));
  cudaMemset(c->gbar, 0, 4 * sizeof(unsigned));
  {
    // scalars: [0..2] reductions, [8..11] block state (dt, time, end time, active)
    double z[16] = {0};
    z[10] = HUGE_VAL;
    z[11] = 1.0;
    cudaMemcpy(c->scal, z, sizeof(z), cudaMemcpyHostToDevice);
  }
  RunDev &h = c->h;
  std::memset(&h, 0, sizeof(RunDev));
  h.coord = p->coord;
  h.n_cycle_base = p->n_cycle_base;
  h.lvls_max = p->lvls_max;
  h.applied_voltage = -p->domain_len_z * p->applied_fld;
  h.domain_len_z = p->domain_len_z;
  h.epsilon_diel = p->epsilon_diel;
  h.ref_init_time = p->ref_init_time;
  h.crv_refine = p->crv_refine;
  h.n_seeds = p->n_seeds;
  for (int s = 0; s < p->n_seeds; s++) {
    for (int d = 0; d < 2; d++) {
      h.seed_r0[s][d] = p->seed_r0[s][d];
      h.seed_r1[s][d] = p->seed_r1[s][d];
    }
    h.seed_width[s] = p->seed_width[s];
  }
  h.scal = c->scal;
  h.blk = c->scal + 8;
  h.dt_max = p->dt_max;
  h.use_drt = p->use_drt ? 1 : 0;
  h.uniform_lvl = p->uniform_lvl;
  h.diel = p->epsilon_diel != 1.0 ? 1 : 0;
  h.status = c->status;
  h.gbar = c->gbar;
  h.gred = c->gred;
  h.gbudget = A5G_DEFAULT_WAIT_CYCLES;
  h.local_cells = A5G_DEFAULT_LOCAL_CELLS;
  h.mx_fmg = 1;
  h.mx_sw_down = h.mx_sw_up = 4;
  h.mx_sw_base = 2 * p->n_cycle_base;
  h.mx_n_corr = 1;
  if (p->photoi_enabled) {
    const std::vector<MzJump> J = mz_run_table(p->photoi_team);
    const size_t jbytes = J.size() * sizeof(MzJump);
    if (cudaMalloc(&c->ph_rng, 4 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->ph_scal, sizeof(PhScal)) != cudaSuccess ||
        cudaMalloc(&c->ph_jump, jbytes) != cudaSuccess) {
      a5g_destroy(c);
      return fail(A5G_ENOMEM, "cudaMalloc failed");
    }
    cudaMemcpy(c->ph_rng, p->rng_seed, 4 * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->ph_jump, J.data(), jbytes, cudaMemcpyHostToDevice);
    cudaMemset(c->ph_scal, 0, sizeof(PhScal));
    h.ph_enabled = 1;
    h.ph_team = p->photoi_team;
    h.ph_coeff = p->photoi_coeff;
    h.ph_num_photons = (double)p->photoi_num_photons;
    h.ph_rng = c->ph_rng;
    h.ph_scal = c->ph_scal;
    h.ph_jump = c->ph_jump;
  }
  *out = c;
  return A5G_OK;
}

int a5g_destroy(a5g_ctx *c) {
  if (!c) return A5G_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_run);
  cudaFree(c->cc);
  cudaFree(c->fx);
  cudaFree(c->fy);
  cudaFree(c->meta);
  cudaFree(c->lists);
  cudaFree(c->new_lists);
  cudaFree(c->tbl);
  cudaFree(c->scal);
  cudaFree(c->flags);
  cudaFree(c->status);
  cudaFree(c->p_boxes);
  cudaFree(c->p_sboxes);
  cudaFree(c->p_pbx);
  cudaFree(c->p_cplan);
  cudaFree(c->p_cwts);
  cudaFree(c->ph_tbl);
  cudaFree(c->ph_rng);
  cudaFree(c->ph_ncr);
  cudaFree(c->ph_cnt);
  cudaFree(c->ph_ipart);
  cudaFree(c->ph_part);
  cudaFree(c->ph_u);
  cudaFree(c->ph_scal);
  cudaFree(c->ph_jump);
  cudaFree(c->ph_boxes);
  cudaFree(c->tbl32);
  cudaFree(c->cc32);
  cudaFree(c->tags);
  cudaFree(c->sumbuf);
  cudaFree(c->gbar);
  cudaFree(c->gred);
  cudaFree(c->lsf);
  cudaFree(c->bval);
  if (c->ev_order) cudaEventDestroy(c->ev_order);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return A5G_OK;
}

int a5g_set_table(a5g_ctx *c, int n_rows, int n_cols, double x_min, double inv_dx,
                  const double *rows_cols) {
  if (!c || !rows_cols) return fail(A5G_EINVAL, "null argument");
  if (n_rows < 2 || n_cols != 4) return fail(A5G_EINVAL, "table needs >= 2 rows and 4 columns");
  if (!(inv_dx > 0) || !std::isfinite(x_min)) return fail(A5G_EINVAL, "bad table grid");
  cudaFree(c->tbl);
  c->tbl = nullptr;
  CK(cudaMalloc(&c->tbl, sizeof(double) * n_rows * n_cols));
  CK(cudaMemcpyAsync(c->tbl, rows_cols, sizeof(double) * n_rows * n_cols,
                     cudaMemcpyHostToDevice, c->stream));
  c->h_tbl.assign(rows_cols, rows_cols + (size_t)n_rows * n_cols);
  c->tbl_rows = n_rows;
  c->tbl_cols = n_cols;
  c->tbl_xmin = x_min;
  c->tbl_inv_dx = inv_dx;
  {
    // FP32 copy for the lookups of the mixed form
    std::vector<float> t32((size_t)n_rows * n_cols);
    for (size_t k = 0; k < t32.size(); k++) t32[k] = (float)rows_cols[k];
    cudaFree(c->tbl32);
    c->tbl32 = nullptr;
    CK(cudaMalloc(&c->tbl32, sizeof(float) * t32.size()));
    CK(cudaMemcpyAsync(c->tbl32, t32.data(), sizeof(float) * t32.size(), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->h.tbl = c->tbl;
  c->h.tbl32 = c->tbl32;
  c->h.tbl_rows = n_rows;
  c->h.tbl_xmin = x_min;
  c->h.tbl_inv_dx = inv_dx;
  c->has_table = true;
  return push_run(c);
}

// FP32 storage of the correction solve when the tree does not fit in shared
// memory (sized to the box capacity; its contents are scratch).
static int mx_ready(a5g_ctx *c) {
  if (c->precision == A5G_MIXED && c->h.diel)
    return fail(A5G_EINVAL, "the mixed form does not support dielectric runs (eps != 1)");
  if (c->precision == A5G_MIXED && c->h.has_lsf)
    return fail(A5G_EINVAL, "the mixed form does not support level-set boundaries");
  if (c->precision != A5G_MIXED || c->mx_smem_fit > 0 || c->cc32_cap >= c->capacity) return A5G_OK;
  cudaFree(c->cc32);
  c->cc32 = nullptr;
  c->cc32_cap = 0;
  CK(cudaMalloc(&c->cc32, (size_t)3 * c->capacity * SLOT * sizeof(float)));
  c->cc32_cap = c->capacity;
  c->h.cc32 = c->cc32;
  return push_run(c);
}

int a5g_set_precision(a5g_ctx *c, int precision, const a5g_mg_schedule *sched) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (precision != A5G_FP64 && precision != A5G_MIXED)
    return fail(A5G_EINVAL, "precision must be A5G_FP64 or A5G_MIXED");
  a5g_mg_schedule s{1, 2, 2, c->p.n_cycle_base, 1};
  if (sched) s = *sched;
  if (s.fmg != 0 && s.fmg != 1) return fail(A5G_EINVAL, "schedule: fmg must be 0 or 1");
  if (precision == A5G_MIXED && c->h.diel)
    return fail(A5G_EINVAL, "the mixed form does not support dielectric runs (eps != 1)");
  if (s.n_cycle_down < 1 || s.n_cycle_down > 8 || s.n_cycle_up < 1 || s.n_cycle_up > 8 ||
      s.n_cycle_base < 1 || s.n_cycle_base > 64 || s.n_corr < 1 || s.n_corr > 8)
    return fail(A5G_EINVAL, "schedule: cycles down/up 1..8, base 1..64, corrections 1..8");
  c->precision = precision;
  c->sched = s;
  RunDev &h = c->h;
  h.mx_enabled = precision == A5G_MIXED;
  h.mx_fmg = s.fmg;
  h.mx_sw_down = 2 * s.n_cycle_down;
  h.mx_sw_up = 2 * s.n_cycle_up;
  h.mx_sw_base = 2 * s.n_cycle_base;
  h.mx_n_corr = s.n_corr;
  int r = push_run(c);
  if (r) return r;
  return mx_ready(c);
}

int a5g_get_precision(a5g_ctx *c, int *precision, a5g_mg_schedule *sched) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (precision) *precision = c->precision;
  if (sched) *sched = c->precision == A5G_MIXED ? c->sched : a5g_mg_schedule{1, 2, 2, c->p.n_cycle_base, 1};
  return A5G_OK;
}

int a5g_set_photon_table(a5g_ctx *c, int n_rows, double x_min, double inv_dx, const double *dist,
                         double frac_in_tbl) {
  if (!c || !dist) return fail(A5G_EINVAL, "null argument");
  if (!c->p.photoi_enabled) return fail(A5G_ESTATE, "photoionization is not enabled");
  if (n_rows < 2 || !(inv_dx > 0) || !std::isfinite(x_min) || !(frac_in_tbl > 0))
    return fail(A5G_EINVAL, "bad photon table");
  cudaFree(c->ph_tbl);
  c->ph_tbl = nullptr;
  CK(cudaMalloc(&c->ph_tbl, sizeof(double) * n_rows));
  CK(cudaMemcpy(c->ph_tbl, dist, sizeof(double) * n_rows, cudaMemcpyHostToDevice));
  c->h_ph_tbl.assign(dist, dist + n_rows);
  // pi_lengthscale = LT_get_col(tbl, 1, fac_dx) and get_lvl_length
  // (src/m_photons.f90:142-155, 331-336)
  double frac = (c->p.photoi_fac_dx - x_min) * inv_dx;
  int ix = (int)std::ceil(frac);
  double w = ix - frac;
  if (ix < 1) {
    ix = 1;
    w = 1;
  } else if (ix >= n_rows) {
    ix = n_rows - 1;
    w = 0;
  }
  const double length = w * dist[ix - 1] + (1 - w) * dist[ix];
  const double invlog2 = 1 / std::log(2.0);
  const double ratio = c->p.dr_base / length;
  const int lvl = ratio <= 1 ? 1 : 1 + (int)std::ceil(std::log(ratio) * invlog2);
  RunDev &h = c->h;
  h.ph_tbl = c->ph_tbl;
  h.ph_rows = n_rows;
  h.ph_xmin = x_min;
  h.ph_inv_dx = inv_dx;
  h.ph_frac = frac_in_tbl;
  h.ph_lvl = lvl;
  c->has_ph_table = true;
  return push_run(c);
}

int a5g_photon_stats(a5g_ctx *c, long long *n_created, double *fac) {
  if (!c || !n_created || !fac) return fail(A5G_EINVAL, "null argument");
  if (!c->p.photoi_enabled) return fail(A5G_ESTATE, "photoionization is not enabled");
  PhScal h{};
  CK(cudaMemcpyAsync(&h, c->ph_scal, sizeof(PhScal), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *n_created = h.n_used;
  *fac = h.fac;
  return check_status(c);
}

int a5g_get_rng(a5g_ctx *c, int *st) {
  if (!c || !st) return fail(A5G_EINVAL, "null argument");
  if (!c->p.photoi_enabled) return fail(A5G_ESTATE, "photoionization is not enabled");
  CK(cudaMemcpyAsync(st, c->ph_rng, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int a5g_set_rng(a5g_ctx *c, const int *st) {
  if (!c || !st) return fail(A5G_EINVAL, "null argument");
  if (!c->p.photoi_enabled) return fail(A5G_ESTATE, "photoionization is not enabled");
  CK(cudaMemcpyAsync(c->ph_rng, st, 4 * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}

static int grow(a5g_ctx *c, int need) {
  if (need <= c->capacity) return A5G_OK;
  const int old_cap = c->capacity;
  int cap = std::max(need, c->capacity + c->capacity / 2);
  cap = std::max(cap, 64);
  double *ncc = nullptr, *nfx = nullptr, *nfy = nullptr;
  BoxMeta *nmeta = nullptr;
  int *nflags = nullptr;
  size_t scc = (size_t)cap * SLOT * A5G_N_VAR_CELL, sfc = (size_t)cap * FSLOT * A5G_N_VAR_FACE;
  if (cudaMalloc(&ncc, scc * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&nfx, sfc * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&nfy, sfc * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&nmeta, (size_t)cap * sizeof(BoxMeta)) != cudaSuccess ||
      cudaMalloc(&nflags, (size_t)cap * sizeof(int)) != cudaSuccess) {
    cudaFree(ncc); cudaFree(nfx); cudaFree(nfy); cudaFree(nmeta); cudaFree(nflags);
    return fail(A5G_ENOMEM, "cannot grow box storage to " + std::to_string(cap) + " boxes");
  }
  CK(cudaMemsetAsync(ncc, 0, scc * sizeof(double), c->stream));
  CK(cudaMemsetAsync(nfx, 0, sfc * sizeof(double), c->stream));
  CK(cudaMemsetAsync(nfy, 0, sfc * sizeof(double), c->stream));
  CK(cudaMemsetAsync(nmeta, 0, (size_t)cap * sizeof(BoxMeta), c->stream));
  if (c->capacity > 0) {
    for (int v = 0; v < A5G_N_VAR_CELL; v++)
      CK(cudaMemcpyAsync(ncc + (size_t)v * cap * SLOT, c->cc + (size_t)v * c->capacity * SLOT,
                         (size_t)c->capacity * SLOT * sizeof(double), cudaMemcpyDeviceToDevice,
                         c->stream));
    for (int f = 0; f < A5G_N_VAR_FACE; f++) {
      CK(cudaMemcpyAsync(nfx + (size_t)f * cap * FSLOT, c->fx + (size_t)f * c->capacity * FSLOT,
                         (size_t)c->capacity * FSLOT * sizeof(double), cudaMemcpyDeviceToDevice,
                         c->stream));
      CK(cudaMemcpyAsync(nfy + (size_t)f * cap * FSLOT, c->fy + (size_t)f * c->capacity * FSLOT,
                         (size_t)c->capacity * FSLOT * sizeof(double), cudaMemcpyDeviceToDevice,
                         c->stream));
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->cc); cudaFree(c->fx); cudaFree(c->fy); cudaFree(c->meta); cudaFree(c->flags);
  c->cc = ncc; c->fx = nfx; c->fy = nfy; c->meta = nmeta; c->flags = nflags;
  c->capacity = cap;
  c->h.capacity = cap;
  c->h.cc = ncc; c->h.fx = nfx; c->h.fy = nfy; c->h.meta = nmeta; c->h.flags = nflags;
  {
    // box tags of the dielectric multigrid: recomputed at every solve
    int *nt = nullptr;
    if (cudaMalloc(&nt, (size_t)cap * sizeof(int)) != cudaSuccess)
      return fail(A5G_ENOMEM, "cannot grow the box tags to " + std::to_string(cap) + " boxes");
    CK(cudaMemsetAsync(nt, 0, (size_t)cap * sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(c->tags);
    c->tags = nt;
    c->h.tags = nt;
  }
  {
    double *ns = nullptr;
    if (cudaMalloc(&ns, (size_t)cap * sizeof(double)) != cudaSuccess)
      return fail(A5G_ENOMEM, "cannot grow the reduction buffer to " + std::to_string(cap) + " boxes");
    cudaFree(c->sumbuf);
    c->sumbuf = ns;
    c->h.sumbuf = ns;
  }
  if (c->lsf) {
    // level-set arrays follow the box storage (new boxes hold 0 until set)
    double *nl = nullptr, *nb = nullptr;
    const size_t old = (size_t)old_cap * SLOT, sz = (size_t)cap * SLOT;
    if (cudaMalloc(&nl, sz * sizeof(double)) != cudaSuccess || cudaMalloc(&nb, sz * sizeof(double)) != cudaSuccess) {
      cudaFree(nl);
      cudaFree(nb);
      return fail(A5G_ENOMEM, "cannot grow the level-set arrays");
    }
    CK(cudaMemsetAsync(nl, 0, sz * sizeof(double), c->stream));
    CK(cudaMemsetAsync(nb, 0, sz * sizeof(double), c->stream));
    CK(cudaMemcpyAsync(nl, c->lsf, old * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(nb, c->bval, old * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(c->lsf);
    cudaFree(c->bval);
    c->lsf = nl;
    c->bval = nb;
    c->h.lsf = nl;
    c->h.bval = nb;
  }
  if (c->cc32) {  // scratch of the mixed form: reallocated at the next mixed launch
    cudaFree(c->cc32);
    c->cc32 = nullptr;
    c->cc32_cap = 0;
    c->h.cc32 = nullptr;
  }
  return ph_resize(c);
}

int a5g_upload_tree(a5g_ctx *c, int max_id, int min_lvl, int max_lvl, const int *meta16,
                    const double *geom4, const int *lvl_counts, const int *lvl_ids) {
  if (!c || !meta16 || !geom4 || !lvl_counts || !lvl_ids) return fail(A5G_EINVAL, "null argument");
  if (max_id < 1) return fail(A5G_EINVAL, "max_id must be >= 1");
  int nlev = max_lvl - min_lvl + 1;
  if (nlev < 1 || nlev + 1 > MAXLEV) return fail(A5G_EINVAL, "bad level range");
  if (max_lvl > c->p.lvls_max) return fail(A5G_EINVAL, "max_lvl above lvls_max");
  // validate topology
  std::vector<BoxMeta> hm(max_id + 1);
  std::memset(hm.data(), 0, hm.size() * sizeof(BoxMeta));
  for (int id = 1; id <= max_id; id++) {
    const int *m = meta16 + 16 * id;
    if (!m[0]) continue;
    BoxMeta &b = hm[id];
    b.lvl = m[1];
    b.ix0 = m[2];
    b.ix1 = m[3];
    b.parent = m[5];
    for (int k = 0; k < 4; k++) b.ch[k] = m[6 + k];
    for (int k = 0; k < 4; k++) b.nb[k] = m[10 + k];
    b.nc = m[14];
    b.dr = geom4[4 * id + 3];
    b.r0 = geom4[4 * id + 0];
    b.r1 = geom4[4 * id + 1];
    int expect = b.lvl >= 1 ? NC : (NC >> (1 - b.lvl));
    if (b.nc != expect || b.nc < 2) return fail(A5G_EINVAL, "box " + std::to_string(id) + ": bad n_cell");
    if (b.parent < 0 || b.parent > max_id) return fail(A5G_EINVAL, "bad parent id");
    for (int k = 0; k < 4; k++)
      if (b.ch[k] < 0 || b.ch[k] > max_id || b.nb[k] > max_id)
        return fail(A5G_EINVAL, "bad child/neighbour id at box " + std::to_string(id));
    if (!(b.dr > 0)) return fail(A5G_EINVAL, "bad dr");
  }
  std::vector<int> lists;
  int off[3][MAXLEV + 1];
  std::vector<std::vector<int>> lv_ids(nlev), lv_leaves(nlev), lv_parents(nlev);
  {
    // regroup per-level (ids, leaves, parents) into three contiguous blocks
    std::vector<std::vector<int>> by(3);
    size_t k = 0;
    std::vector<int> starts[3];
    for (int li = 0; li < nlev; li++) {
      for (int kind = 0; kind < 3; kind++) {
        int n = lvl_counts[3 * li + kind];
        if (n < 0) return fail(A5G_EINVAL, "negative level count");
        off[kind][li] = (int)by[kind].size();
        for (int q = 0; q < n; q++) {
          int id = lvl_ids[k++];
          if (id < 1 || id > max_id || !meta16[16 * id])
            return fail(A5G_EINVAL, "level list names an unused id");
          if (hm[id].lvl != min_lvl + li) return fail(A5G_EINVAL, "level list / box level mismatch");
          by[kind].push_back(id);
          if (kind == 0) lv_ids[li].push_back(id);
          if (kind == 1) lv_leaves[li].push_back(id);
          if (kind == 2) lv_parents[li].push_back(id);
        }
      }
    }
    for (int kind = 0; kind < 3; kind++) off[kind][nlev] = (int)by[kind].size();
    int base[3] = {0, (int)by[0].size(), (int)(by[0].size() + by[1].size())};
    for (int kind = 0; kind < 3; kind++) {
      for (int li = 0; li <= nlev; li++) off[kind][li] += base[kind];
      lists.insert(lists.end(), by[kind].begin(), by[kind].end());
    }
  }
  // every referenced box must exist and be in use
  for (int id = 1; id <= max_id; id++) {
    if (!meta16[16 * id]) continue;
    const BoxMeta &b = hm[id];
    if (b.parent > 0 && !meta16[16 * b.parent]) return fail(A5G_EINVAL, "parent not in use");
    for (int k = 0; k < 4; k++) {
      if (b.ch[k] > 0 && !meta16[16 * b.ch[k]]) return fail(A5G_EINVAL, "child not in use");
      if (b.nb[k] > 0 && !meta16[16 * b.nb[k]]) return fail(A5G_EINVAL, "neighbour not in use");
    }
    if (b.lvl > min_lvl && b.parent <= 0) return fail(A5G_EINVAL, "box without parent");
  }
  int r = grow(c, max_id + 1);
  if (r) return r;
  CK(cudaMemcpyAsync(c->meta, hm.data(), hm.size() * sizeof(BoxMeta), cudaMemcpyHostToDevice,
                     c->stream));
  if (lists.size() + 1 > c->lists_cap) {
    cudaFree(c->lists);
    c->lists = nullptr;
    c->lists_cap = std::max(lists.size() + 1, 2 * c->lists_cap);
    CK(cudaMalloc(&c->lists, c->lists_cap * sizeof(int)));
  }
  if (!lists.empty())
    CK(cudaMemcpyAsync(c->lists, lists.data(), lists.size() * sizeof(int), cudaMemcpyHostToDevice,
                       c->stream));
  HostPlans P;
  build_plans(hm, lv_ids, lv_leaves, lv_parents, min_lvl, nlev, c->p.dr_base, P);
  if ((r = upload_vec(c, c->p_boxes, c->cap_boxes, P.boxes)) ||
      (r = upload_vec(c, c->p_sboxes, c->cap_sboxes, P.sboxes)) ||
      (r = upload_vec(c, c->p_pbx, c->cap_pbx, P.pbx)) ||
      (r = upload_vec(c, c->p_cplan, c->cap_cplan, P.cplan)) ||
      (r = upload_vec(c, c->p_cwts, c->cap_cwts, P.cwts)))
    return r;
  RunDev &h = c->h;
  {
    // keep the multigrid variables in shared memory when the tree fits
    const size_t need = (PLAN_DOUBLES + (c->p.coord == 1 ? WTS_DOUBLES : 0)) * sizeof(double) +
                        3 * (size_t)P.smem_doubles * sizeof(double) +
                        P.boxes.size() * sizeof(BoxRec) + P.pbx.size() * sizeof(int);
    const size_t limit = dyn_smem_limit();
    c->fit64 = need <= limit ? P.smem_doubles : 0;
    c->need64 = need;
    // the FP32 correction solve of the mixed form: three float arrays
    const int s32 = (P.smem_doubles + 3) & ~3;
    const size_t need32 = (PLAN_DOUBLES + (c->p.coord == 1 ? WTS_DOUBLES : 0)) * sizeof(double) +
                          3 * (size_t)s32 * sizeof(float) + P.boxes.size() * sizeof(BoxRec) +
                          P.pbx.size() * sizeof(int);
    c->fit32 = need32 <= limit ? s32 : 0;
    c->need32 = need32;
    apply_staging(c);
  }
  h.sboxes = c->p_sboxes;
  std::memcpy(h.bx_off, P.bx_off, sizeof(P.bx_off));
  std::memcpy(h.pb_off, P.pb_off, sizeof(P.pb_off));
  std::memcpy(h.lv_nc, P.lv_nc, sizeof(P.lv_nc));
  std::memcpy(h.lv_dr, P.lv_dr, sizeof(P.lv_dr));
  h.boxes = c->p_boxes;
  h.pbx = c->p_pbx;
  h.cplan = c->p_cplan;
  h.cwts = c->p_cwts;
  std::memcpy(h.cplan_blk, P.cplan_blk, sizeof(P.cplan_blk));
  h.min_lvl = min_lvl;
  h.max_lvl = max_lvl;
  h.nlev = nlev;
  h.dr_min = c->p.dr_base * std::pow(0.5, max_lvl - 1);  // as a5g_get_max_dt
  for (int kind = 0; kind < 3; kind++)
    for (int li = 0; li <= nlev; li++) h.lv_off[kind][li] = off[kind][li];
  h.lists = c->lists;
  c->max_id = max_id;
  c->min_lvl = min_lvl;
  c->max_lvl = max_lvl;
  c->h_nc.assign(max_id + 1, 0);
  for (int id = 1; id <= max_id; id++)
    if (meta16[16 * id]) c->h_nc[id] = hm[id].nc;
  long long nl = 0;
  for (int li = 0; li < nlev; li++)
    for (int q = off[1][li]; q < off[1][li + 1]; q++) nl += (long long)hm[lists[q]].nc * hm[lists[q]].nc;
  c->n_leaf_cells = nl;
  h.n_ids = max_id + 1;
  if (c->p.photoi_enabled) {
    std::vector<PhBox> pb(max_id + 1);
    std::memset(pb.data(), 0, pb.size() * sizeof(PhBox));
    for (int id = 1; id <= max_id; id++) {
      if (!meta16[16 * id]) continue;
      const BoxMeta &m = hm[id];
      pb[id].r0 = m.r0;
      pb[id].r1 = m.r1;
      pb[id].dr = m.dr;
      for (int q = 0; q < 4; q++) pb[id].ch[q] = m.ch[q];
      pb[id].lvl = m.lvl;
      pb[id].nc = m.nc;
    }
    if ((r = upload_vec(c, c->ph_boxes, c->ph_boxes_cap, pb))) return r;
    h.ph_boxes = c->ph_boxes;
  }
  c->has_tree = true;
  CK(cudaStreamSynchronize(c->stream));
  return push_run(c);
}

int a5g_upload_cc(a5g_ctx *c, int iv, const double *host) {
  if (!c || !host) return fail(A5G_EINVAL, "null argument");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (iv < 0 || iv >= A5G_N_VAR_CELL) return fail(A5G_EINVAL, "bad variable index");
  CK(cudaMemcpyAsync(c->cc + (size_t)iv * c->capacity * SLOT, host,
                     (size_t)(c->max_id + 1) * SLOT * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (iv == I_EPS) {
    // the run is dielectric when eps differs from 1 anywhere in a box in use
    int diel = c->p.epsilon_diel != 1.0 ? 1 : 0;
    for (int id = 1; id <= c->max_id && !diel; id++) {
      const int g = c->h_nc[id] + 2;
      if (c->h_nc[id] == 0) continue;
      for (int k = 0; k < g * g && !diel; k++)
        if (host[(size_t)id * SLOT + k] != 1.0) diel = 1;
    }
    if (diel != c->h.diel) {
      c->h.diel = diel;
      return push_run(c);
    }
  }
  return A5G_OK;
}

int a5g_download_cc(a5g_ctx *c, int iv, double *host) {
  if (!c || !host) return fail(A5G_EINVAL, "null argument");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (iv < 0 || iv >= A5G_N_VAR_CELL) return fail(A5G_EINVAL, "bad variable index");
  CK(cudaMemcpyAsync(host, c->cc + (size_t)iv * c->capacity * SLOT,
                     (size_t)(c->max_id + 1) * SLOT * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int a5g_upload_fc(a5g_ctx *c, int dimf, int f, const double *host) {
  if (!c || !host) return fail(A5G_EINVAL, "null argument");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (dimf < 0 || dimf > 1 || f < 0 || f >= A5G_N_VAR_FACE) return fail(A5G_EINVAL, "bad face index");
  double *base = dimf == 0 ? c->fx : c->fy;
  CK(cudaMemcpyAsync(base + (size_t)f * c->capacity * FSLOT, host,
                     (size_t)(c->max_id + 1) * FSLOT * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}

int a5g_download_fc(a5g_ctx *c, int dimf, int f, double *host) {
  if (!c || !host) return fail(A5G_EINVAL, "null argument");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (dimf < 0 || dimf > 1 || f < 0 || f >= A5G_N_VAR_FACE) return fail(A5G_EINVAL, "bad face index");
  double *base = dimf == 0 ? c->fx : c->fy;
  CK(cudaMemcpyAsync(host, base + (size_t)f * c->capacity * FSLOT,
                     (size_t)(c->max_id + 1) * FSLOT * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int a5g_tree_copy_cc(a5g_ctx *c, int a, int b) {
  if (a < 0 || a >= A5G_N_VAR_CELL || b < 0 || b >= A5G_N_VAR_CELL)
    return fail(A5G_EINVAL, "bad variable index");
  return launch(c, mkop(OP_COPY, a, b));
}
int a5g_fluxes_koren(a5g_ctx *c, double dt) {
  if (!(dt > 0)) return fail(A5G_EINVAL, "dt must be > 0");
  return launch(c, mkop(OP_FLUXES, 0, 0, dt));
}
int a5g_consistent_fluxes(a5g_ctx *c) { return launch(c, mkop(OP_CONSISTENT)); }
int a5g_update_solution(a5g_ctx *c, double dt) { return launch(c, mkop(OP_UPDATE, 0, 0, dt)); }
int a5g_restrict_tree(a5g_ctx *c, int iv) {
  if (iv < 0 || iv >= A5G_N_VAR_CELL) return fail(A5G_EINVAL, "bad variable index");
  return launch(c, mkop(OP_RESTRICT, iv));
}
int a5g_gc_tree(a5g_ctx *c, int iv, int rb_kind) {
  if (iv < 0 || iv >= A5G_N_VAR_CELL) return fail(A5G_EINVAL, "bad variable index");
  if (rb_kind != 0 && rb_kind != 1) return fail(A5G_EINVAL, "rb_kind must be 0 or 1");
  return launch(c, mkop(OP_GC, iv, rb_kind == 0 ? GC_LIM : GC_INTERP));
}
int a5g_average_dens(a5g_ctx *c) { return launch(c, mkop(OP_AVERAGE)); }
int a5g_compute_fld(a5g_ctx *c, int no_guess) {
  if (c && c->precision == A5G_MIXED && !no_guess) {
    int r = mx_ready(c);
    if (r) return r;
    return launch_smem(c, mkop(OP_COMPUTE_FLD_MIXED), c->dyn_smem32);
  }
  return launch(c, mkop(OP_COMPUTE_FLD, no_guess ? 1 : 0));
}
int a5g_fas_fmg(a5g_ctx *c, int set_residual, int first_call) {
  return launch(c, mkop(OP_FMG, set_residual ? 1 : 0, first_call ? 1 : 0));
}
int a5g_fld_from_pot(a5g_ctx *c) { return launch(c, mkop(OP_FLD_FROM_POT)); }
int a5g_mg_fas_vcycle(a5g_ctx *c, int max_lvl, int set_residual) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (c->has_tree && (max_lvl < c->min_lvl || max_lvl > c->max_lvl))
    return fail(A5G_EINVAL, "max_lvl outside the levels of the tree");
  return launch(c, mkop(OP_VCYCLE, max_lvl, set_residual ? 1 : 0));
}

// a$D_tree_max_cc / _min_cc / _sum_cc: one launch, the value read back.
static int tree_red(a5g_ctx *c, int iv, int kind, int team, double *out) {
  if (!c || !out) return fail(A5G_EINVAL, "null argument");
  if (iv < 0 || iv >= A5G_N_VAR_CELL) return fail(A5G_EINVAL, "bad variable index");
  if (team < 1) return fail(A5G_EINVAL, "team must be >= 1");
  Op o = mkop(OP_TREE_RED, iv, kind);
  o.i2 = team;
  int r = launch(c, o);
  if (r) return r;
  CK(cudaMemcpyAsync(out, c->scal + 4, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}
int a5g_tree_max_cc(a5g_ctx *c, int iv, double *out) { return tree_red(c, iv, 0, 1, out); }
int a5g_tree_min_cc(a5g_ctx *c, int iv, double *out) { return tree_red(c, iv, 1, 1, out); }
int a5g_tree_sum_cc(a5g_ctx *c, int iv, int team, double *out) { return tree_red(c, iv, 2, team, out); }

int a5g_dt_reductions(a5g_ctx *c, double *out3) {
  if (!out3) return fail(A5G_EINVAL, "null argument");
  int r = launch(c, mkop(OP_DT_RED));
  if (r) return r;
  CK(cudaMemcpyAsync(out3, c->scal, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}

static double lt_col(const a5g_ctx *c, int col, double x) {
  double frac = (x - c->tbl_xmin) * c->tbl_inv_dx;
  int ix;
  double fr;
  if (frac < 2.0e9 && frac > -2.0e9) {
    ix = (int)std::ceil(frac);
    fr = ix - frac;
  } else {
    ix = frac > 0 ? c->tbl_rows : 0;
    fr = 0;
  }
  if (ix < 1) { ix = 1; fr = 1; }
  else if (ix >= c->tbl_rows) { ix = c->tbl_rows - 1; fr = 0; }
  const double *T = c->h_tbl.data() + (size_t)c->tbl_rows * col;
  return fr * T[ix - 1] + (1 - fr) * T[ix];
}

int a5g_get_max_dt(a5g_ctx *c, double *dt) {
  if (!dt) return fail(A5G_EINVAL, "null argument");
  double r3[3];
  int r = a5g_dt_reductions(c, r3);
  if (r) return r;
  // get_max_dt, src/streamer_2d.f90:284-302 (cyl :294-313)
  const double max_fld = r3[0], min_fld = r3[1], max_dns = r3[2];
  const double eps_mach = 2.220446049250313e-16;
  double dr_min = c->p.dr_base * std::pow(0.5, c->max_lvl - 1);
  double mobility = lt_col(c, 0, max_fld);
  double max_mobility = lt_col(c, 0, min_fld);
  double diff_coeff = lt_col(c, 1, max_fld);
  double alpha = lt_col(c, 2, max_fld);
  double dt_cfl = dr_min / (mobility * max_fld);
  double dt_dif = 0.25 * (dr_min * dr_min) / diff_coeff;
  double dns = c->p.coord == 1 ? std::max(eps_mach, max_dns) : max_dns;
  double dt_drt = UC_EPS0 / (UC_ELEM_CHARGE * max_mobility * dns);
  double dt_alpha = 1 / std::max(mobility * max_fld * alpha, eps_mach);
  double m = std::min(std::min(1 / (1 / dt_cfl + 1 / dt_dif), dt_alpha), c->p.dt_max);
  if (c->p.use_drt) m = std::min(m, dt_drt);
  *dt = 0.5 * m;
  return A5G_OK;
}

int a5g_ref_flags(a5g_ctx *c, double time, int *flags) {
  if (!flags) return fail(A5G_EINVAL, "null argument");
  int r = launch(c, mkop(OP_REF_FLAGS, 0, 0, time));
  if (r) return r;
  CK(cudaMemcpyAsync(flags, c->flags, (size_t)(c->max_id + 1) * sizeof(int),
                     cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}

int a5g_prolong_new(a5g_ctx *c, const int *n_new, const int *new_ids) {
  if (!c || !n_new || !new_ids) return fail(A5G_EINVAL, "null argument");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  int nlev = c->h.nlev;
  size_t tot = 0;
  for (int li = 0; li < nlev; li++) {
    if (n_new[li] < 0) return fail(A5G_EINVAL, "negative count");
    tot += n_new[li];
  }
  for (size_t k = 0; k < tot; k++)
    if (new_ids[k] < 1 || new_ids[k] > c->max_id) return fail(A5G_EINVAL, "bad new id");
  if (tot + 1 > c->new_cap) {
    cudaFree(c->new_lists);
    c->new_lists = nullptr;
    c->new_cap = std::max(tot + 1, 2 * c->new_cap);
    CK(cudaMalloc(&c->new_lists, c->new_cap * sizeof(int)));
  }
  if (tot) CK(cudaMemcpyAsync(c->new_lists, new_ids, tot * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  int acc = 0;
  for (int li = 0; li < nlev; li++) {
    c->h.new_off[li] = acc;
    acc += n_new[li];
  }
  c->h.new_off[nlev] = acc;
  c->h.new_lists = c->new_lists;
  int r = push_run(c);
  if (r) return r;
  r = launch(c, mkop(OP_PROLONG_NEW));
  if (r) return r;
  CK(cudaStreamSynchronize(c->stream));
  return A5G_OK;
}

int a5g_photoionization(a5g_ctx *c, double dt, int has_dt) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (!c->p.photoi_enabled) return fail(A5G_ESTATE, "photoionization is not enabled");
  if (has_dt && !(dt > 0)) return fail(A5G_EINVAL, "dt must be > 0");
  int r = ph_ready(c);
  if (r) return r;
  if ((r = ph_launch_source_absorb(c, dt, has_dt))) return r;
  return launch(c, mkop(OP_PH_DEPOSIT));
}

int a5g_step(a5g_ctx *c, double dt) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (!(dt > 0)) return fail(A5G_EINVAL, "dt must be > 0");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (!c->has_table) return fail(A5G_ESTATE, "no transport table set");
  int deposit = 0;
  if (c->p.photoi_enabled) {
    int r = ph_ready(c);
    if (r) return r;
    if ((r = ph_launch_source_absorb(c, dt, 1))) return r;
    deposit = 1;
  }
  if (c->precision == A5G_MIXED) {
    int r = mx_ready(c);
    if (r) return r;
  }
  const void *fn = c->precision == A5G_MIXED ? (const void *)a5g_step_mixed_kernel
                                             : (const void *)a5g_step_kernel;
  if (c->n_cta > 1) {
    const RunDev *run = c->d_run;
    void *args[] = {(void *)&run, (void *)&dt, (void *)&deposit};
    CK(cudaLaunchCooperativeKernel(fn, dim3(c->n_cta), dim3(NTHR), args, 0, c->stream));
    return A5G_OK;
  }
  if (c->precision == A5G_MIXED)
    a5g_step_mixed_kernel<<<1, NTHR, c->dyn_smem32, c->stream>>>(c->d_run, dt, deposit);
  else
    a5g_step_kernel<<<1, NTHR, c->dyn_smem, c->stream>>>(c->d_run, dt, deposit);
  CK(cudaGetLastError());
  return A5G_OK;
}

// Largest grid of co-resident blocks a cooperative launch of the run kernels
// may have on the current device (blocks per SM at no dynamic shared memory
// times the SMs, over the kernels a grid-mode run launches).
static int max_coresident_ctas() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  int best = INT_MAX;
  const void *fns[4] = {(const void *)a5g_run_kernel, (const void *)a5g_step_kernel,
                        (const void *)a5g_step_mixed_kernel, (const void *)a5g_batch_map_kernel};
  for (const void *fn : fns) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, NTHR, 0) != cudaSuccess) return 0;
    best = std::min(best, nb * sms);
  }
  return std::min(best, A5G_MAX_CTAS);
}

int a5g_set_ctas(a5g_ctx *c, int n_cta, long long wait_cycles) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (n_cta < 1 || n_cta > A5G_MAX_CTAS) return fail(A5G_EINVAL, "n_cta must be 1..A5G_MAX_CTAS");
  if (n_cta > 1) {
    const int lim = max_coresident_ctas();
    if (n_cta > lim)
      return fail(A5G_EINVAL, "n_cta = " + std::to_string(n_cta) + " exceeds the " + std::to_string(lim) +
                                  " blocks that can be co-resident on this device");
  }
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemset(c->gbar, 0, 4 * sizeof(unsigned)));
  c->n_cta = n_cta;
  c->h.gbudget = wait_cycles < 0 ? A5G_DEFAULT_WAIT_CYCLES : wait_cycles;
  apply_staging(c);
  int r = push_run(c);
  if (r) return r;
  return mx_ready(c);
}

int a5g_set_level_set(a5g_ctx *c, const double *lsf, const double *bval) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if ((lsf == nullptr) != (bval == nullptr)) return fail(A5G_EINVAL, "set both lsf and bval, or neither");
  if (!lsf) {
    CK(cudaStreamSynchronize(c->stream));
    c->h.has_lsf = 0;
    return push_run(c);
  }
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (c->precision == A5G_MIXED)
    return fail(A5G_EINVAL, "the mixed form does not support level-set boundaries");
  const size_t sz = (size_t)c->capacity * SLOT, n = (size_t)(c->max_id + 1) * SLOT;
  if (!c->lsf) {
    if (cudaMalloc(&c->lsf, sz * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->bval, sz * sizeof(double)) != cudaSuccess) {
      cudaFree(c->lsf);
      cudaFree(c->bval);
      c->lsf = c->bval = nullptr;
      return fail(A5G_ENOMEM, "cannot allocate the level-set arrays");
    }
    CK(cudaMemsetAsync(c->lsf, 0, sz * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->bval, 0, sz * sizeof(double), c->stream));
  }
  CK(cudaMemcpyAsync(c->lsf, lsf, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->bval, bval, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->h.lsf = c->lsf;
  c->h.bval = c->bval;
  c->h.has_lsf = 1;
  apply_staging(c);
  return push_run(c);
}

int a5g_set_grid_local(a5g_ctx *c, int cells) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (cells < 0) return fail(A5G_EINVAL, "cells must be >= 0");
  c->h.local_cells = cells;
  return push_run(c);
}

int a5g_get_ctas(a5g_ctx *c, int *n_cta, int *max_cta) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (n_cta) *n_cta = c->n_cta;
  if (max_cta) *max_cta = max_coresident_ctas();
  return A5G_OK;
}

// Orders a batched launch on stream s after the work already queued on each
// member's own stream (in), and each member's later work after it (out):
// events recorded and waited on the device, no host synchronisation.
static int batch_order_in(a5g_ctx *const *ctxs, int n, cudaStream_t s) {
  for (int k = 0; k < n; k++) {
    if (ctxs[k]->stream == s) continue;
    CK(cudaEventRecord(ctxs[k]->ev_order, ctxs[k]->stream));
    CK(cudaStreamWaitEvent(s, ctxs[k]->ev_order, 0));
  }
  return A5G_OK;
}
static int batch_order_out(a5g_ctx *const *ctxs, int n, cudaStream_t s, cudaEvent_t done) {
  CK(cudaEventRecord(done, s));
  for (int k = 0; k < n; k++)
    if (ctxs[k]->stream != s) CK(cudaStreamWaitEvent(ctxs[k]->stream, done, 0));
  return A5G_OK;
}

int a5g_step_batch(a5g_ctx **ctxs, int n, const double *dts) {
  if (!ctxs || !dts || n < 1) return fail(A5G_EINVAL, "bad batch");
  for (int k = 0; k < n; k++) {
    if (!ctxs[k] || !ctxs[k]->has_tree || !ctxs[k]->has_table)
      return fail(A5G_ESTATE, "batch member without tree or table");
    if (!(dts[k] > 0)) return fail(A5G_EINVAL, "dt must be > 0");
  }
  a5g_ctx *c0 = ctxs[0];
  std::vector<const RunDev *> rp(n);
  std::vector<Op> ops(2 * n);
  bool any_ph = false;
  int max_team = 0;
  size_t ph_smem = 0;
  for (int k = 0; k < n; k++) {
    rp[k] = ctxs[k]->d_run;
    const bool ph = ctxs[k]->p.photoi_enabled != 0;
    if (ph) {
      int r = ph_ready(ctxs[k]);
      if (r) return r;
      any_ph = true;
      max_team = std::max(max_team, ctxs[k]->p.photoi_team);
      ph_smem = std::max(ph_smem, ph_smem_bytes(ctxs[k]));
    }
    if (ctxs[k]->precision == A5G_MIXED) {
      int r = mx_ready(ctxs[k]);
      if (r) return r;
    }
    ops[k] = mkop(ctxs[k]->precision == A5G_MIXED ? OP_STEP_MIXED : OP_STEP, ph ? 1 : 0, 0, dts[k]);
    ops[n + k] = ph ? mkop(OP_PH_SOURCE, 1, 0, dts[k]) : mkop(OP_NOP);
  }
  // the batch runs on c0's stream after the other members' queued work
  int ro = batch_order_in(ctxs, n, c0->stream);
  if (ro) return ro;
  const RunDev **d_rp = nullptr;
  Op *d_ops = nullptr;
  CK(cudaMallocAsync((void **)&d_rp, n * sizeof(void *), c0->stream));
  CK(cudaMallocAsync((void **)&d_ops, 2 * n * sizeof(Op), c0->stream));
  CK(cudaMemcpyAsync(d_rp, rp.data(), n * sizeof(void *), cudaMemcpyHostToDevice, c0->stream));
  CK(cudaMemcpyAsync(d_ops, ops.data(), 2 * n * sizeof(Op), cudaMemcpyHostToDevice, c0->stream));
  size_t dyn = 0;
  for (int k = 0; k < n; k++) dyn = std::max(dyn, std::max(ctxs[k]->dyn_smem, step_smem(ctxs[k])));
  if (any_ph) {
    // photon sources of every member with photoionization (the others run
    // an operation that does nothing here), then the absorption
    a5g_run_kernel<<<n, NTHR, dyn, c0->stream>>>(nullptr, Op{}, d_rp, d_ops + n);
    CK(cudaGetLastError());
    dim3 grid((unsigned)((max_team + PH_THREADS - 1) / PH_THREADS), (unsigned)n);
    a5g_photon_kernel<<<grid, PH_THREADS, ph_smem, c0->stream>>>(nullptr, d_rp, nullptr, (int)ph_smem);
    CK(cudaGetLastError());
  }
  a5g_run_kernel<<<n, NTHR, dyn, c0->stream>>>(nullptr, Op{}, d_rp, d_ops);
  CK(cudaGetLastError());
  CK(cudaFreeAsync(d_rp, c0->stream));
  CK(cudaFreeAsync(d_ops, c0->stream));
  // the members' own streams continue after the batch
  return batch_order_out(ctxs, n, c0->stream, c0->ev_order);
}

// Per-device address of g_batch_scratch, looked up on first use with the
// device current.
static std::mutex g_static_mu;
static BatchSlot *g_static_dev[256] = {};

// Writes the n descriptors of one launch into the fixed table on stream s,
// as kernel parameters of fill launches (ordered with the launch that reads
// them like any other work of the stream).
static int static_fill(BatchSlot *table, const BatchSlot *slots, int n, cudaStream_t s) {
  for (int k0 = 0; k0 < n; k0 += SLOT_FILL) {
    const int m = std::min(SLOT_FILL, n - k0);
    SlotChunk chunk;
    std::memset(&chunk, 0, sizeof(chunk));
    std::memcpy(chunk.s, slots + k0, (size_t)m * sizeof(BatchSlot));
    a5g_fill_slots_kernel<<<1, 128, 0, s>>>(table + k0, chunk, m);
    CK(cudaGetLastError());
  }
  return A5G_OK;
}

int a5g_step_batch_static(a5g_ctx **ctxs, int n, const double *dts) {
  if (!ctxs || !dts || n < 1) return fail(A5G_EINVAL, "bad batch");
  if (n > A5G_STATIC_BATCH_MAX)
    return fail(A5G_EINVAL, "a5g_step_batch_static: n = " + std::to_string(n) +
                                " exceeds A5G_STATIC_BATCH_MAX (" +
                                std::to_string(A5G_STATIC_BATCH_MAX) + ")");
  int dev = -1;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return fail(A5G_EINVAL, "device ordinal out of range");
  for (int k = 0; k < n; k++) {
    if (!ctxs[k] || !ctxs[k]->has_tree || !ctxs[k]->has_table)
      return fail(A5G_ESTATE, "batch member without tree or table");
    if (!(dts[k] > 0)) return fail(A5G_EINVAL, "dt must be > 0");
    cudaPointerAttributes at{};
    CK(cudaPointerGetAttributes(&at, ctxs[k]->d_run));
    if (at.device != dev)
      return fail(A5G_EINVAL, "a5g_step_batch_static: context on another device than the current one");
  }
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_dev[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_batch_scratch);
    if (e != cudaSuccess || !p)
      return fail(A5G_ECUDA, std::string("cudaGetSymbolAddress(g_batch_scratch): ") +
                                 cudaGetErrorString(e));
    g_static_dev[dev] = static_cast<BatchSlot *>(p);
  }
  a5g_ctx *c0 = ctxs[0];
  int ro = batch_order_in(ctxs, n, c0->stream);
  if (ro) return ro;
  size_t dyn = 0, ph_smem = 0;
  bool any_ph = false;
  int max_team = 0;
  for (int k = 0; k < n; k++) {
    dyn = std::max(dyn, std::max(ctxs[k]->dyn_smem, step_smem(ctxs[k])));
    if (ctxs[k]->precision == A5G_MIXED) {
      int r = mx_ready(ctxs[k]);
      if (r) return r;
    }
    if (ctxs[k]->p.photoi_enabled) {
      int r = ph_ready(ctxs[k]);
      if (r) return r;
      any_ph = true;
      max_team = std::max(max_team, ctxs[k]->p.photoi_team);
      ph_smem = std::max(ph_smem, ph_smem_bytes(ctxs[k]));
    }
  }
  // descriptors of this call on the host stack (A5G_STATIC_BATCH_MAX x 40 bytes)
  BatchSlot slots[A5G_STATIC_BATCH_MAX];
  if (any_ph) {
    // photon sources and absorption first; the table is then rewritten with
    // the step descriptors (fills and launches are ordered on the stream)
    for (int k = 0; k < n; k++) {
      slots[k].run = ctxs[k]->d_run;
      slots[k].op = ctxs[k]->p.photoi_enabled ? mkop(OP_PH_SOURCE, 1, 0, dts[k]) : mkop(OP_NOP);
    }
    int rf = static_fill(g_static_dev[dev], slots, n, c0->stream);
    if (rf) return rf;
    a5g_run_kernel_slots<<<n, NTHR, dyn, c0->stream>>>(g_static_dev[dev]);
    CK(cudaGetLastError());
    dim3 grid((unsigned)((max_team + PH_THREADS - 1) / PH_THREADS), (unsigned)n);
    a5g_photon_kernel<<<grid, PH_THREADS, ph_smem, c0->stream>>>(nullptr, nullptr, g_static_dev[dev],
                                                                 (int)ph_smem);
    CK(cudaGetLastError());
  }
  for (int k = 0; k < n; k++) {
    slots[k].run = ctxs[k]->d_run;
    slots[k].op = mkop(ctxs[k]->precision == A5G_MIXED ? OP_STEP_MIXED : OP_STEP,
                       ctxs[k]->p.photoi_enabled ? 1 : 0, 0, dts[k]);
  }
  int rf = static_fill(g_static_dev[dev], slots, n, c0->stream);
  if (rf) return rf;
  a5g_run_kernel_slots<<<n, NTHR, dyn, c0->stream>>>(g_static_dev[dev]);
  CK(cudaGetLastError());
  // the members' own streams continue after the batch
  return batch_order_out(ctxs, n, c0->stream, c0->ev_order);
}

// ---------------------------------------------------------------------------
// Device-driven batch of runs (a5g_batch_*): one block of the main loop --
// get_max_dt and num_steps_amr steps -- for every run in one launch per
// kernel, with each run's dt, time and active flag kept on the device, so
// that the block is a fixed sequence of launches that a CUDA graph replays.
struct a5g_batch {
  std::vector<a5g_ctx *> ctxs;
  cudaStream_t stream = nullptr;
  const RunDev **d_rp = nullptr;
  Op *d_ops = nullptr;  // [block dt | photon sources | steps], n each
  bool any_ph = false;
  int max_team = 0;
  size_t ph_smem = 0, dyn = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_steps = -1;
  double *h_state = nullptr;  // pinned, 5 per run (a5g_batch_gather_kernel)
  double *d_state = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // block-to-run map when some member takes several blocks (3 ints per
  // block, A5G_MAX_CTAS blocks at most): the block-dt and step launches are
  // then one cooperative launch of n_blocks blocks
  int *d_gmap = nullptr;
  int n_blocks = 0;
  bool mapped = false;
};

static void batch_drop_graph(a5g_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_steps = -1;
}

// Operation table of the batch from the members' current precision and
// photoionization settings.
static int batch_build_ops(a5g_batch *b) {
  const int n = (int)b->ctxs.size();
  std::vector<const RunDev *> rp(n);
  std::vector<Op> ops(3 * n);
  b->any_ph = false;
  b->max_team = 0;
  size_t ph = 48 << 10;
  for (int k = 0; k < n; k++) {
    a5g_ctx *c = b->ctxs[k];
    rp[k] = c->d_run;
    const bool phk = c->p.photoi_enabled != 0;
    if (phk) {
      b->any_ph = true;
      b->max_team = std::max(b->max_team, c->p.photoi_team);
      ph = std::max(ph, ph_smem_bytes(c));
    }
    ops[k] = mkop(OP_BLOCK_DT);
    ops[n + k] = phk ? mkop(OP_PH_SOURCE, 1, 1) : mkop(OP_NOP);
    ops[2 * n + k] = mkop(c->precision == A5G_MIXED ? OP_STEP_MIXED : OP_STEP, phk ? 1 : 0, 1);
  }
  b->ph_smem = std::min(ph, dyn_smem_limit());
  b->dyn = dyn_smem_limit();
  CK(cudaMemcpy(b->d_rp, rp.data(), n * sizeof(void *), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_ops, ops.data(), 3 * n * sizeof(Op), cudaMemcpyHostToDevice));
  // box-to-block mapping: each member's group of c->n_cta blocks
  b->mapped = false;
  int total = 0;
  for (int k = 0; k < n; k++) {
    total += b->ctxs[k]->n_cta;
    if (b->ctxs[k]->n_cta > 1) b->mapped = true;
  }
  if (b->mapped) {
    const int lim = max_coresident_ctas();
    if (total > lim)
      return fail(A5G_EINVAL, "batch members take " + std::to_string(total) + " blocks; at most " +
                                  std::to_string(lim) + " can be co-resident");
    std::vector<int> gmap(3 * (size_t)total);
    int blk = 0;
    for (int k = 0; k < n; k++)
      for (int r = 0; r < b->ctxs[k]->n_cta; r++, blk++) {
        gmap[3 * blk] = k;
        gmap[3 * blk + 1] = r;
        gmap[3 * blk + 2] = b->ctxs[k]->n_cta;
      }
    CK(cudaMemcpy(b->d_gmap, gmap.data(), gmap.size() * sizeof(int), cudaMemcpyHostToDevice));
    b->n_blocks = total;
  }
  batch_drop_graph(b);
  return A5G_OK;
}

// One launch of the batch's block-dt or step operations (ops: n entries).
static int batch_launch_ops(a5g_batch *b, const Op *ops) {
  const int n = (int)b->ctxs.size();
  if (b->mapped) {
    const RunDev *const *runs = b->d_rp;
    const int *gmap = b->d_gmap;
    void *args[] = {(void *)&runs, (void *)&ops, (void *)&gmap};
    CK(cudaLaunchCooperativeKernel((const void *)a5g_batch_map_kernel, dim3(b->n_blocks), dim3(NTHR), args,
                                   b->dyn, b->stream));
    return A5G_OK;
  }
  a5g_run_kernel<<<n, NTHR, b->dyn, b->stream>>>(nullptr, Op{}, b->d_rp, ops);
  CK(cudaGetLastError());
  return A5G_OK;
}

// The launches of one block on the batch stream. Every launch takes the
// largest dynamic shared memory a run may use, so that a captured graph stays
// valid while the members' trees change between blocks.
static int batch_enqueue(a5g_batch *b, int num_steps) {
  const int n = (int)b->ctxs.size();
  int r = batch_launch_ops(b, b->d_ops);
  if (r) return r;
  for (int s = 0; s < num_steps; s++) {
    if (b->any_ph) {
      a5g_run_kernel<<<n, NTHR, b->dyn, b->stream>>>(nullptr, Op{}, b->d_rp, b->d_ops + n);
      CK(cudaGetLastError());
      dim3 grid((unsigned)((b->max_team + PH_THREADS - 1) / PH_THREADS), (unsigned)n);
      a5g_photon_kernel<<<grid, PH_THREADS, b->ph_smem, b->stream>>>(nullptr, b->d_rp, nullptr,
                                                                     (int)b->ph_smem);
      CK(cudaGetLastError());
    }
    if ((r = batch_launch_ops(b, b->d_ops + 2 * n))) return r;
  }
  return A5G_OK;
}

int a5g_batch_create(a5g_ctx **ctxs, int n, a5g_batch **out) {
  if (!ctxs || !out || n < 1) return fail(A5G_EINVAL, "bad batch");
  *out = nullptr;
  int dev = -1;
  CK(cudaGetDevice(&dev));
  for (int k = 0; k < n; k++) {
    if (!ctxs[k] || !ctxs[k]->has_tree || !ctxs[k]->has_table)
      return fail(A5G_ESTATE, "batch member without tree or table");
    cudaPointerAttributes at{};
    CK(cudaPointerGetAttributes(&at, ctxs[k]->d_run));
    if (at.device != dev) return fail(A5G_EINVAL, "batch member on another device than the current one");
    for (int q = 0; q < k; q++)
      if (ctxs[q] == ctxs[k]) return fail(A5G_EINVAL, "a context appears twice in the batch");
  }
  a5g_batch *b = new a5g_batch();
  b->ctxs.assign(ctxs, ctxs + n);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&b->d_rp, n * sizeof(void *)) != cudaSuccess ||
      cudaMalloc(&b->d_ops, 3 * n * sizeof(Op)) != cudaSuccess ||
      cudaMallocHost(&b->h_state, 5 * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_state, 5 * n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_gmap, 3 * (size_t)A5G_MAX_CTAS * sizeof(int)) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
    a5g_batch_destroy(b);
    return fail(A5G_ENOMEM, "cannot allocate the batch");
  }
  int r = batch_build_ops(b);
  if (r) {
    a5g_batch_destroy(b);
    return r;
  }
  *out = b;
  return A5G_OK;
}

int a5g_batch_destroy(a5g_batch *b) {
  if (!b) return A5G_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  cudaFree(b->d_rp);
  cudaFree(b->d_ops);
  if (b->h_state) cudaFreeHost(b->h_state);
  cudaFree(b->d_state);
  cudaFree(b->d_gmap);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return A5G_OK;
}

int a5g_batch_begin(a5g_batch *b, const double *time, const double *t_end) {
  if (!b || !time || !t_end) return fail(A5G_EINVAL, "null argument");
  for (size_t k = 0; k < b->ctxs.size(); k++) {
    a5g_ctx *c = b->ctxs[k];
    CK(cudaStreamSynchronize(c->stream));
    const double st[4] = {0.0, time[k], t_end[k], 1.0};
    CK(cudaMemcpy(c->scal + 8, st, sizeof(st), cudaMemcpyHostToDevice));
  }
  return batch_build_ops(b);
}

int a5g_batch_launch(a5g_batch *b, int num_steps, int use_graph) {
  if (!b || num_steps < 1) return fail(A5G_EINVAL, "bad argument");
  const int n = (int)b->ctxs.size();
  for (int k = 0; k < n; k++) {
    a5g_ctx *c = b->ctxs[k];
    int r;
    if (c->p.photoi_enabled && (r = ph_ready(c))) return r;
    if ((r = mx_ready(c))) return r;
  }
  // the members' own queued work (uploads, regrids) precedes the block
  {
    int r = batch_order_in(b->ctxs.data(), n, b->stream);
    if (r) return r;
  }
  CK(cudaEventRecord(b->ev0, b->stream));
  if (use_graph) {
    if (!b->exec || b->graph_steps != num_steps) {
      batch_drop_graph(b);
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      int r = batch_enqueue(b, num_steps);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
      }
      if (e != cudaSuccess) return fail(A5G_ECUDA, std::string("stream capture: ") + cudaGetErrorString(e));
      b->graph = g;
      CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
      b->graph_steps = num_steps;
    }
    CK(cudaGraphLaunch(b->exec, b->stream));
  } else {
    int r = batch_enqueue(b, num_steps);
    if (r) return r;
  }
  // ev1 ends the timed block; the members' own streams continue after it
  {
    int r = batch_order_out(b->ctxs.data(), n, b->stream, b->ev1);
    if (r) return r;
  }
  a5g_batch_gather_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_rp, n, b->d_state);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(b->h_state, b->d_state, 5 * n * sizeof(double), cudaMemcpyDeviceToHost,
                     b->stream));
  return A5G_OK;
}

int a5g_batch_finish(a5g_batch *b, double *dt, double *time, int *active, float *gpu_ms) {
  if (!b) return fail(A5G_EINVAL, "null batch");
  const int n = (int)b->ctxs.size();
  CK(cudaStreamSynchronize(b->stream));
  for (int k = 0; k < n; k++) {
    if (b->h_state[5 * k + 4] != 0.0) {
      int r = check_status(b->ctxs[k]);  // reports and clears the status word
      if (r) return r;
    }
    if (dt) dt[k] = b->h_state[5 * k];
    if (time) time[k] = b->h_state[5 * k + 1];
    if (active) active[k] = b->h_state[5 * k + 3] != 0.0;
  }
  if (gpu_ms) CK(cudaEventElapsedTime(gpu_ms, b->ev0, b->ev1));
  return A5G_OK;
}

int a5g_batch_block(a5g_batch *b, int num_steps, int use_graph, double *dt, double *time,
                    int *active, float *gpu_ms) {
  int r = a5g_batch_launch(b, num_steps, use_graph);
  if (r) return r;
  return a5g_batch_finish(b, dt, time, active, gpu_ms);
}

// Diagnostics: allow (1) or forbid (0) the shared-memory staging of the
// multigrid, so that tests can run the device-memory path of the solves on
// trees that fit. Not part of the public interface.
extern "C" int a5g_debug_set_staging(a5g_ctx *c, int allow_smem) {
  if (!c) return fail(A5G_EINVAL, "null context");
  CK(cudaStreamSynchronize(c->stream));
  c->allow_smem = allow_smem != 0;
  apply_staging(c);
  int r = push_run(c);
  if (r) return r;
  return mx_ready(c);
}

int a5g_sync(a5g_ctx *c) {
  if (!c) return fail(A5G_EINVAL, "null context");
  CK(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

// Internal diagnostics (not part of the ABI headers): shared-memory use and
// sizes of the uploaded tree.
int a5g_debug_info(a5g_ctx *c, long long *out8) {
  if (!c || !out8) return fail(A5G_EINVAL, "null argument");
  out8[0] = c->h.smem_doubles;
  out8[1] = (long long)c->dyn_smem;
  out8[2] = c->capacity;
  out8[3] = c->h.nlev;
  out8[4] = (long long)dyn_smem_limit();
  out8[5] = c->h.bx_off[c->h.nlev];
  out8[6] = c->h.mx_smem;
  out8[7] = (long long)c->dyn_smem32;
  return A5G_OK;
}

// Internal diagnostics: the layout of a5g_params as this library was
// compiled, so that tests can hold the documented bindings to it. out[0] is
// sizeof(a5g_params), out[1..] the offsets of its fields in declaration
// order; returns the number of values written (at most n).
int a5g_debug_params_layout(int *out, int n) {
  if (!out) return 0;
  const int v[] = {(int)sizeof(a5g_params),
                   (int)offsetof(a5g_params, box_size), (int)offsetof(a5g_params, coord),
                   (int)offsetof(a5g_params, lvls_max), (int)offsetof(a5g_params, dr_base),
                   (int)offsetof(a5g_params, domain_len_z), (int)offsetof(a5g_params, applied_fld),
                   (int)offsetof(a5g_params, epsilon_diel), (int)offsetof(a5g_params, dt_max),
                   (int)offsetof(a5g_params, use_drt), (int)offsetof(a5g_params, n_cycle_base),
                   (int)offsetof(a5g_params, ref_init_time), (int)offsetof(a5g_params, crv_refine),
                   (int)offsetof(a5g_params, n_seeds), (int)offsetof(a5g_params, seed_r0),
                   (int)offsetof(a5g_params, seed_r1), (int)offsetof(a5g_params, seed_width),
                   (int)offsetof(a5g_params, photoi_enabled),
                   (int)offsetof(a5g_params, photoi_num_photons),
                   (int)offsetof(a5g_params, photoi_team), (int)offsetof(a5g_params, photoi_pad),
                   (int)offsetof(a5g_params, photoi_coeff), (int)offsetof(a5g_params, photoi_fac_dx),
                   (int)offsetof(a5g_params, rng_seed), (int)offsetof(a5g_params, uniform_lvl),
                   (int)offsetof(a5g_params, uniform_pad)};
  const int m = std::min(n, (int)(sizeof(v) / sizeof(v[0])));
  for (int k = 0; k < m; k++) out[k] = v[k];
  return m;
}

int a5g_get_stream(a5g_ctx *c, void **stream) {
  if (!c || !stream) return fail(A5G_EINVAL, "null argument");
  *stream = (void *)c->stream;
  return A5G_OK;
}

int a5g_n_leaf_cells(a5g_ctx *c, long long *n) {
  if (!c || !n) return fail(A5G_EINVAL, "null argument");
  *n = c->n_leaf_cells;
  return A5G_OK;
}

}  // extern "C"
