// Internal declarations shared by the host (C++) and device (CUDA) sources of
// libtamm_b200.so.  Nothing here is part of the public C ABI (include/tamm_b200.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/tamm_b200.h"

namespace tb {

constexpr int kMaxModes = 8; // modes per tensor
constexpr int kMaxClass = 4; // labels per label class in a contraction

// Status-carrying exception used inside the library; converted to a status code
// and tb_last_error() message at the C-ABI boundary.
struct Error: std::runtime_error {
  int code;
  Error(int c, const std::string& m): std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg);
void              set_last_error(const std::string& msg);

#define TB_EXPECTS(cond, msg)                                                          \
  do {                                                                                 \
    if(!(cond)) ::tb::fail(TB_ERR_INVALID, std::string("EXPECTS failed: ") + (msg));   \
  } while(0)

#define TB_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if(e_ != cudaSuccess)                                                              \
      ::tb::fail(e_ == cudaErrorMemoryAllocation ? TB_ERR_NO_MEMORY : TB_ERR_CUDA,      \
                 std::string(#call) + ": " + cudaGetErrorString(e_));                  \
  } while(0)

// Label classes of one contraction C(cl) += A(al) * B(bl), following
// kernels::block_multiply (src/tamm/kernels/multiply.hpp:237-330):
//   batch  : in C, A and B          (mode positions in C, A, B)
//   m      : in C and A only        (A-outer; C order)
//   n      : in C and B only        (B-outer; C order)
//   k      : in A and B only        (inner; A order)
//   ar, br : only in A / only in B  (reduced by beta-chained GEMM steps)
struct LabelClasses {
  int    nc = 0, na = 0, nb = 0;
  int    nbatch = 0, nm = 0, nn = 0, nk = 0, nar = 0, nbr = 0;
  int8_t batch_c[kMaxClass], batch_a[kMaxClass], batch_b[kMaxClass];
  int8_t m_c[kMaxClass], m_a[kMaxClass];
  int8_t n_c[kMaxClass], n_b[kMaxClass];
  int8_t k_a[kMaxClass], k_b[kMaxClass];
  int8_t ar_a[kMaxClass], br_b[kMaxClass];
  // which class holds the stride-1 (last) mode of A and of B: 0 m/n, 1 k, 2 other
  int8_t a_contig = 0, b_contig = 0;
};

LabelClasses classify(const int* cl, int nc, const int* al, int na, const int* bl, int nb);

// Device work-list records.
struct DevGroup {
  int64_t c_off;
  int32_t task_begin, task_end;
  int32_t cdims[kMaxModes];
};
struct DevTask {
  int64_t a_off, b_off;
  int32_t adims[kMaxModes];
  int32_t bdims[kMaxModes];
};
// One CTA's output tile: group, batch index, first row / column of the tile.
struct DevItem {
  int32_t group, batch, m0, n0;
};

// Host mirror of a work list plus its device copies.
struct WorkList {
  std::vector<DevGroup> groups;
  std::vector<DevTask>  tasks;
  double                flops = 0;         // admitted FP64 FLOPs (tasks that run + skipped tasks)
  double                flops_run = 0;     // FP64 FLOPs of the tasks in the list
  double                flops_skipped = 0; // admitted tasks left out: an exactly-zero block of a read-only operand
  int64_t               ntasks_skipped = 0;
  DevGroup*             d_groups = nullptr;
  DevTask*              d_tasks  = nullptr;
  int                   device   = -1;
  // tile items of the FP64 kernel, built (and uploaded) on its first launch over this
  // work list: contractions that run split-INT8 or BF16x3 never need them
  mutable std::vector<DevItem> items_fp64;
  mutable DevItem*             d_items     = nullptr;
  mutable bool                 items_built = false;
  mutable int                  items_bn    = 64; // output tile width of those items
  ~WorkList();
};

class Arena;
struct Tensor;

// Energy epilogue of a contraction (tb_sched_mult_energy): instead of C (+)= alpha * A * B
// the kernels add sum (C + alpha * A * B)^2 / D over the elements of the output groups
// with tasks and leave C unchanged; D = sum_m sg[m] * eps[estart[group * nc + m] + x_m]
// is the orbital-energy denominator of element (x_0, ..., x_(nc-1)) of the group's
// block.  Each warp of a tile writes one partial sum into `part` (tile index x warps).
struct EnergyArgs {
  const double*  eps    = nullptr;
  const int32_t* estart = nullptr;
  double*        part   = nullptr;
  double         sg[kMaxModes] = {0, 0, 0, 0, 0, 0, 0, 0};
};

#ifdef __CUDACC__
// 1 / D for a normal, nonzero double: two Newton-Raphson steps x' = x + x (1 - D x)
// from the hardware's approximate reciprocal (rcp.approx.ftz.f64); the denominator
// kernels and the energy epilogues share it, so their sums see the same 1 / D.
__device__ __forceinline__ double recip_nr(double D) {
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(D));
  double e = fma(-D, x, 1.0);
  x        = fma(x, e, x);
  e        = fma(-D, x, 1.0);
  return fma(x, e, x);
}

// The part of D over `n` modes of a C block: x decomposed over dims[0..n) (last
// fastest), sum_j sg[cm[j]] * eps[start[cm[j]] + x_j].
__device__ __forceinline__ double energy_part(int32_t x, int n, const int32_t* dims, const int8_t* cm,
                                              const EnergyArgs& en, const int32_t* start) {
  double d = 0.0;
  for(int j = n - 1; j >= 0; j--) {
    const int32_t q = x / dims[j];
    const int     c = cm[j];
    d += en.sg[c] * __ldg(en.eps + start[c] + (x - q * dims[j]));
    x = q;
  }
  return d;
}
#endif

// Scratch of a captured CUDA graph: buffers stay allocated for the graph's lifetime;
// ops of the graph run in stream order, so a buffer returned by one op can serve the
// next.  The graph holds the largest scratch of one op, not the sum.
struct CapturePool {
  Arena*                                    arena = nullptr;
  std::vector<std::tuple<void*, int64_t, bool>> bufs; // pointer, bytes, in use
  void*                                     get(int64_t bytes);
  void                                      put(void* p);
  void                                      release(); // back to the arena
};

struct Plan {
  LabelClasses lc;
  int          mode       = TB_MODE_FP64;
  double       err_target = 1e-11;
  int          nslices    = 0;
  tb_stats     last{};
  Arena*       arena        = nullptr; // scratch source (null: cudaMallocAsync)
  int          tile_n       = 0;       // split-INT8 output tile width (0: default for S)
  bool         check_errors = true;    // read the device error word after a launch
  // while a CUDA graph is being captured: scratch comes from (and returns to) this
  // pool, which keeps it allocated for the graph's replays
  struct CapturePool* pinned = nullptr;
  bool         profile      = false;   // time the phases with CUDA events (synchronises)
  // C = alpha * A * B instead of C += alpha * A * B on the output blocks of groups with
  // tasks: the FP64 kernel stores its result without reading C (each element of C
  // belongs to exactly one output tile); blocks of groups without tasks are left
  // untouched
  bool         store        = false;
  // energy epilogue (EnergyArgs): *energy_out += energy_scale * the kernels' partial
  // sums; null for a plain contraction
  const EnergyArgs* energy       = nullptr;
  double*           energy_out   = nullptr;
  double            energy_scale = 1.0;
  // read-only operands whose split digits may be kept (tb_ctx_set_digit_cache), and the
  // context's cache account
  const Tensor* cache_a = nullptr;
  const Tensor* cache_b = nullptr;
  int64_t       cache_limit = 0;
  int64_t*      cache_used  = nullptr;
};

void forget_int8_layout(const WorkList* wl);
// FP64 FLOPs of one task of a group (2 * |C block| * K, times the one-sided steps).
double task_flops(const LabelClasses& lc, const DevGroup& g, const DevTask& t);
// Largest split-INT8 slice count the error target needs (3..8).
int int8_slices_for(double err_target);

// ---- launchers (device code in *.cu) ----
void launch_contract_fp64(const Plan& plan, const WorkList& wl, double alpha, double beta,
                          int is_assign, const double* A, const double* B, double* C,
                          cudaStream_t stream);
void contract_int8(Plan& plan, const WorkList& wl, double alpha, const double* A,
                   const double* B, double* C, cudaStream_t stream);
void contract_bf16x3(Plan& plan, const WorkList& wl, double alpha, const double* A,
                     const double* B, double* C, cudaStream_t stream);

struct AssignLoop {
  int     nd = 0;
  int64_t dims[4];
  int64_t dld[4];
  int64_t sld[4];
};
AssignLoop plan_assign(const int64_t* ddims, const int* dlabels, int nd, const int64_t* sdims,
                       const int* slabels, int ns);
void launch_assign(const AssignLoop& lp, double* dst, double scale, const double* src,
                   int is_assign, cudaStream_t stream);
// One block pair of a permuted AddOp: offsets and the loop of plan_assign, with the
// position of the source's stride-1 loop mode when the pair goes through the
// shared-memory transpose (-1: streamed by rows of the destination's last mode).  The
// pair's work is cut into `units` work units of at most 2048 elements, numbered from
// `first` across the launch: `per_unit` sub-tiles of tq x tp (q: the destination's
// last mode, tq <= 64; p: the source's stride-1 mode, tp <= 32) of the transposed
// plane, or `per_unit` rows of tq elements when streamed (`upr` > 1: a row longer
// than a unit, cut into upr units).
// Counts, strides and offsets within one pair are below 2^31; `mag` holds the 64-bit
// multipliers of the divisions the kernel makes (x / d = umul64hi(x, mag) for d >= 2).
struct BlockAssign {
  int64_t  dst_off, src_off;
  int64_t  first;
  int32_t  nd, p;
  int32_t  dims[4], dld[4], sld[4];
  int32_t  units, per_unit;
  int32_t  tq, tp, upr;
  int32_t  nsub;     // sub-tiles (transposed) or rows (streamed) of the pair
  int32_t  nbq, nbp; // sub-tiles along q and p
  uint64_t mag[6];   // multipliers for dims[0..3], nbq, nbp (0: divisor 1)
};
// `first` is the number of work units of the pairs before this one in the launch.
BlockAssign make_block_assign(const AssignLoop& lp, int64_t dst_off, int64_t src_off, int64_t first);
// All block pairs of an AddOp in one launch (device array of nblocks BlockAssign
// holding nunits work units in all).
void launch_assign_blocks(double* dst, double scale, const double* src, const BlockAssign* blocks, int nblocks,
                          int64_t nunits, int is_assign, cudaStream_t stream);
void launch_fill(double* x, int64_t n, double value, int is_assign, cudaStream_t stream);
// Segment lists of the block-wise fill and map: per run of blocks (dst offset, src
// offset or -1, n, first), `first` the sum of n over the runs before it.
// seg_list merges blocks that are adjacent on both sides into one run.
std::vector<int64_t> seg_list(const std::vector<int64_t>& triples);
// x[off .. off + n) (=|+=) value for each run of a device segment list holding
// `total` elements
void launch_fill_blocks(double* x, const int64_t* segs, int nseg, int64_t total, double value, int is_assign,
                        cudaStream_t stream);
void launch_axpby(double alpha, const double* x, double beta, double* y, int64_t n,
                  cudaStream_t stream);
// For each run (dst offset, src offset or -1, n, first) of a device segment list
// holding `total` elements: dst[0:n) = f(src[0:n)) with f = TB_MAP_* and parameter p
// (src -1: zeros).
void launch_map_blocks(double* dst, const double* src, const int64_t* segs, int nseg, int64_t total, int fn,
                       double p, cudaStream_t stream);
double reduce_dot(const double* x, const double* y, int64_t n, cudaStream_t stream);
// *out = scale * x.y (root: scale * sqrt(x.x)), staying on the device; part holds
// 1024 doubles of scratch.  y == nullptr means x.x.
void launch_dot_to(const double* x, const double* y, int64_t n, double scale, int root, double* out, double* part,
                   cudaStream_t stream);
// One admitted block of a denominator update: packed offset, dims, and the root
// orbital index of each mode's first element.
struct DenomBlock {
  int64_t off;
  int64_t dims[kMaxModes];
  int64_t first[kMaxModes];
};
struct DenomSigns {
  double s[kMaxModes];
};
// A unit of denominator work: `rows` consecutive rows (all modes but the last) of one
// block, from row r0.
struct DenomUnit {
  int32_t block, rows;
  int64_t r0;
};
constexpr int kDenomUnitRows  = 2048;  // at most, so that the row parts fit in shared memory
constexpr int kDenomUnitElems = 16384; // about, per unit
void launch_denom(double* t, const double* r, double scale, const DenomBlock* blocks, const DenomUnit* units,
                  int nunits, int nmodes, const double* eps, DenomSigns signs, cudaStream_t stream);
// *out += scale * sum w^2 / D over the blocks (part: nunits doubles of scratch).
void launch_denom_energy(const double* w, double scale, const DenomBlock* blocks, const DenomUnit* units,
                         int nunits, int nmodes, const double* eps, DenomSigns signs, double* part, double* out,
                         cudaStream_t stream);
void launch_set_scalar(double* out, double v, cudaStream_t stream);
// *out += scale * sum part[0 .. np), summed in a fixed order (deterministic).
void launch_energy_final(const double* part, int64_t np, double scale, double* out, cudaStream_t stream);
// nonzero[b] = 1 if x[off_b, off_b + n_b) holds an element other than +0.0 / -0.0, else
// 0, for the (off, n) pairs of a device array (the launcher clears nonzero first).
void launch_block_nonzero(const double* x, const int64_t* pairs, int nblocks, uint32_t* nonzero,
                          cudaStream_t stream);
// Reads and clears the device error word of the split-INT8 launches of a work list;
// throws TB_ERR_TIMEOUT if a device-side wait gave up.
void check_int8_errors(const WorkList& wl, cudaStream_t stream);
void   launch_fill_random(double* x, int64_t n, uint64_t seed, uint64_t first, int dist, double p0,
                          double p1, cudaStream_t stream);

// Build the work list for one block triple (the single-block entry point).
WorkList* single_block_worklist(const LabelClasses& lc, const int64_t* adims, const int64_t* bdims,
                                const int64_t* cdims);
void finalize_worklist(const LabelClasses& lc, WorkList& wl, bool upload = true); // items + device copy

} // namespace tb
