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
#include "a5_internal.h"

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


extern __shared__ double g_dsmem[];

// The plan slots lead the dynamic shared memory of a shared-memory solve:
// 2 NTHR int4 cell plans, then (cylindrical runs) 2 NTHR double2 weights.
constexpr int PLAN_DOUBLES = 2 * NTHR * 2;     // doubles taken by the cell plans
constexpr int WTS_DOUBLES = 2 * NTHR * 2;      // doubles taken by the weights

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

// box_gsrb_clpl weights (i+ioff-1)/(i+ioff-1/2) and (i+ioff)/(i+ioff-1/2)
__host__ __device__ __forceinline__ void cyl_weights(int gi, double &rf1, double &rf2) {
  const double den = gi - 0.5;
  rf1 = (gi - 1) / den;
  rf2 = gi / den;
}

// Modulus of the mzran generator (fosito/m_random.f90:58-66).
constexpr unsigned int MZ_M = 2147483579u;

// Descriptor of one member of a launch of a5g_step_batch_static.
struct BatchSlot {
  const RunDev *run;
  Op op;
};

// The phases, operations and kernels, compiled twice: `blk` for a run on one
// thread block (the group is the block; thread index, stride and barrier are
// compile-time; no level-set branches), `grd` for a run on a group of
// blocks or with level-set boxes (group state in s_grp, grid barriers, the
// one-block sections of coarse levels, the level-set operators). The host
// launches the blk kernels unless a run needs grd.
namespace blk {
#define A5G_GRID 0
#include "a5g_phases.cuh"
#undef A5G_GRID
}  // namespace blk
namespace grd {
#define A5G_GRID 1
#include "a5g_phases.cuh"
#undef A5G_GRID
}  // namespace grd

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

// The kernels of one execution form (blk or grd).
struct Form {
  void (*run)(const RunDev *, Op, const RunDev *const *, const Op *);
  void (*step)(const RunDev *, double, int);
  void (*step_mixed)(const RunDev *, double, int);
  void (*slots)(const BatchSlot *);
};
constexpr Form kBlockForm = {blk::a5g_run_kernel, blk::a5g_step_kernel, blk::a5g_step_mixed_kernel,
                             blk::a5g_run_kernel_slots};
constexpr Form kGroupForm = {grd::a5g_run_kernel, grd::a5g_step_kernel, grd::a5g_step_mixed_kernel,
                             grd::a5g_run_kernel_slots};
// Photon absorption does not depend on the form.
constexpr auto a5g_photon_kernel = blk::a5g_photon_kernel;
constexpr auto a5g_batch_map_kernel = grd::a5g_batch_map_kernel;

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
  // host copy of the last uploaded topology (a5g_internal_view)
  A5Topo topo;
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
    constexpr int NF = 10;
    cudaFuncAttributes fa[NF];
    const void *fns[NF] = {(const void *)kBlockForm.run,        (const void *)kBlockForm.step,
                           (const void *)kBlockForm.step_mixed, (const void *)kBlockForm.slots,
                           (const void *)kGroupForm.run,        (const void *)kGroupForm.step,
                           (const void *)kGroupForm.step_mixed, (const void *)kGroupForm.slots,
                           (const void *)a5g_photon_kernel,     (const void *)a5g_batch_map_kernel};
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

// The group form for a run on several blocks or with level-set boxes, the
// block form otherwise.
static const Form &form(const a5g_ctx *c) { return c->n_cta > 1 || c->h.has_lsf ? kGroupForm : kBlockForm; }
// A batch of one block per member: the group form if any member has
// level-set boxes.
static const Form &batch_form(a5g_ctx *const *ctxs, int n) {
  for (int k = 0; k < n; k++)
    if (ctxs[k]->h.has_lsf) return kGroupForm;
  return kBlockForm;
}

static int launch_smem(a5g_ctx *c, const Op &op, size_t smem) {
  if (!c) return fail(A5G_EINVAL, "null context");
  if (!c->has_tree) return fail(A5G_ESTATE, "no tree uploaded");
  if (!c->has_table) return fail(A5G_ESTATE, "no transport table set");
  const Form &F = form(c);
  if (c->n_cta > 1 && grid_op(op.code)) {
    // co-resident blocks of one cooperative launch (no staging: smem = 0)
    const RunDev *run = c->d_run;
    Op o = op;
    const RunDev *const *runs = nullptr;
    const Op *ops = nullptr;
    void *args[] = {(void *)&run, (void *)&o, (void *)&runs, (void *)&ops};
    CK(cudaLaunchCooperativeKernel((const void *)F.run, dim3(c->n_cta), dim3(NTHR), args, 0, c->stream));
    return A5G_OK;
  }
  F.run<<<1, NTHR, smem, c->stream>>>(c->d_run, op, nullptr, nullptr);
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
  // defined contents: no phase reads an entry it has not written, and zeros
  // keep it so if one did
  CK(cudaMemsetAsync(c->cc32, 0, (size_t)3 * c->capacity * SLOT * sizeof(float), c->stream));
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
  c->topo.max_id = max_id;
  c->topo.min_lvl = min_lvl;
  c->topo.max_lvl = max_lvl;
  c->topo.meta16.assign(meta16, meta16 + 16 * (size_t)(max_id + 1));
  c->topo.geom4.assign(geom4, geom4 + 4 * (size_t)(max_id + 1));
  c->topo.ids = lv_ids;
  c->topo.leaves = lv_leaves;
  c->topo.parents = lv_parents;
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
int a5g_compute_fld_fp64(a5g_ctx *c, int no_guess) {
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
  const Form &F = form(c);
  const void *fn = c->precision == A5G_MIXED ? (const void *)F.step_mixed : (const void *)F.step;
  if (c->n_cta > 1) {
    const RunDev *run = c->d_run;
    void *args[] = {(void *)&run, (void *)&dt, (void *)&deposit};
    CK(cudaLaunchCooperativeKernel(fn, dim3(c->n_cta), dim3(NTHR), args, 0, c->stream));
    return A5G_OK;
  }
  if (c->precision == A5G_MIXED)
    F.step_mixed<<<1, NTHR, c->dyn_smem32, c->stream>>>(c->d_run, dt, deposit);
  else
    F.step<<<1, NTHR, c->dyn_smem, c->stream>>>(c->d_run, dt, deposit);
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
  const void *fns[4] = {(const void *)kGroupForm.run, (const void *)kGroupForm.step,
                        (const void *)kGroupForm.step_mixed, (const void *)a5g_batch_map_kernel};
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
  const Form &F = batch_form(ctxs, n);
  if (any_ph) {
    // photon sources of every member with photoionization (the others run
    // an operation that does nothing here), then the absorption
    F.run<<<n, NTHR, dyn, c0->stream>>>(nullptr, Op{}, d_rp, d_ops + n);
    CK(cudaGetLastError());
    dim3 grid((unsigned)((max_team + PH_THREADS - 1) / PH_THREADS), (unsigned)n);
    a5g_photon_kernel<<<grid, PH_THREADS, ph_smem, c0->stream>>>(nullptr, d_rp, nullptr, (int)ph_smem);
    CK(cudaGetLastError());
  }
  F.run<<<n, NTHR, dyn, c0->stream>>>(nullptr, Op{}, d_rp, d_ops);
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
      // the checks of mx_ready without its allocation: a mixed member whose
      // FP32 storage is not sized to its tree is refused here
      const a5g_ctx *m = ctxs[k];
      if (m->h.diel || m->h.has_lsf)
        return fail(A5G_EINVAL, "the mixed form does not support dielectric or level-set runs");
      if (m->mx_smem_fit == 0 && m->cc32_cap < m->capacity)
        return fail(A5G_ESTATE, "a5g_step_batch_static: a mixed-precision member's FP32 storage "
                                "is not sized to its tree (call a5g_step_batch or a5g_step once "
                                "after each tree upload)");
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
  const Form &F = batch_form(ctxs, n);
  if (any_ph) {
    // photon sources and absorption first; the table is then rewritten with
    // the step descriptors (fills and launches are ordered on the stream)
    for (int k = 0; k < n; k++) {
      slots[k].run = ctxs[k]->d_run;
      slots[k].op = ctxs[k]->p.photoi_enabled ? mkop(OP_PH_SOURCE, 1, 0, dts[k]) : mkop(OP_NOP);
    }
    int rf = static_fill(g_static_dev[dev], slots, n, c0->stream);
    if (rf) return rf;
    F.slots<<<n, NTHR, dyn, c0->stream>>>(g_static_dev[dev]);
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
  F.slots<<<n, NTHR, dyn, c0->stream>>>(g_static_dev[dev]);
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
  // some member has level-set boxes: the group form (a captured graph holds
  // the form it was captured with)
  bool general = false;
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
  (b->general ? kGroupForm : kBlockForm).run<<<n, NTHR, b->dyn, b->stream>>>(nullptr, Op{}, b->d_rp, ops);
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
      (b->general ? kGroupForm : kBlockForm).run<<<n, NTHR, b->dyn, b->stream>>>(nullptr, Op{}, b->d_rp,
                                                                                 b->d_ops + n);
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
  {
    const bool gen = &batch_form(b->ctxs.data(), n) == &kGroupForm;
    if (gen != b->general) {
      b->general = gen;
      batch_drop_graph(b);
    }
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

int a5g_set_applied_field(a5g_ctx *c, double applied_fld) {
  if (!c) return fail(A5G_EINVAL, "null argument");
  if (!std::isfinite(applied_fld)) return fail(A5G_EINVAL, "applied field must be finite");
  c->p.applied_fld = applied_fld;
  c->h.applied_voltage = -c->p.domain_len_z * applied_fld;
  return push_run(c);
}

int a5g_internal_view(a5g_ctx *c, A5View *v) {
  if (!c || !v) return fail(A5G_EINVAL, "null argument");
  v->stream = (void *)c->stream;
  v->cc = c->cc;
  v->fx = c->fx;
  v->fy = c->fy;
  v->capacity = c->capacity;
  v->coord = c->p.coord;
  v->n_cycle_base = c->p.n_cycle_base;
  v->precision = c->precision;
  v->photoi_enabled = c->p.photoi_enabled;
  v->n_cta = c->n_cta;
  v->has_lsf = c->h.has_lsf;
  v->has_table = c->has_table;
  v->applied_fld = c->p.applied_fld;
  v->domain_len_z = c->p.domain_len_z;
  v->epsilon_diel = c->p.epsilon_diel;
  v->tbl_rows = c->tbl_rows;
  v->tbl_cols = c->tbl_cols;
  v->tbl_xmin = c->tbl_xmin;
  v->tbl_inv_dx = c->tbl_inv_dx;
  v->tbl_host = c->h_tbl.data();
  v->topo = c->has_tree ? &c->topo : nullptr;
  return A5G_OK;
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
