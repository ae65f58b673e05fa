// Runtime tier: execution context with a stream-ordered device arena, index spaces,
// tiled index spaces, block-sparse tensors in a device-resident block store, and the
// Scheduler.  Exposed through the runtime half of include/tamm_b200.h.
#pragma once

#include "tb_internal.hpp"

#include <functional>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <utility>
#include <vector>

struct tb_tensor_s;
struct tb_sched_s;

namespace tb {

// Stream-ordered arena: one cudaMalloc carved by a coalescing best-fit free list
// (the role of TAMM's RMM pool_memory_resource, src/tamm/mr/pool_memory_resource.hpp,
// with TAMM_GPU_POOL semantics).  Every user of an arena works on the context's
// single stream, so a block freed on the host is reusable by any later stream work.
class Arena {
public:
  Arena(int device, int64_t bytes);
  ~Arena();
  Arena(const Arena&)            = delete;
  Arena& operator=(const Arena&) = delete;
  void*   allocate(int64_t bytes);
  void    deallocate(void* p);
  int64_t used() const { return used_; }
  int64_t peak() const { return peak_; }
  int64_t capacity() const { return capacity_; }

private:
  int                        device_;
  char*                      base_     = nullptr;
  int64_t                    capacity_ = 0;
  int64_t                    used_     = 0;
  int64_t                    peak_     = 0;
  std::map<int64_t, int64_t> free_;  // offset -> size
  std::map<int64_t, int64_t> inuse_; // offset -> size
  // the free blocks again, ordered by (size, offset): best fit in O(log n), ties to the
  // lowest offset
  std::set<std::pair<int64_t, int64_t>> by_size_;
  void                                  add_free(int64_t off, int64_t size);
  void                                  drop_free(std::map<int64_t, int64_t>::iterator it);
};

struct Ctx {
  int                    device = 0;
  cudaStream_t           stream = nullptr;          // compute
  cudaStream_t           h2d = nullptr, d2h = nullptr; // asynchronous host transfers (created on first use)
  std::unique_ptr<Arena> arena;
  int                    mode       = TB_MODE_FP64;
  double                 err_target = 1e-11;
  int                    nslices    = 0;
  int64_t                digit_cache_bytes = 0; // split digits of read-only operands kept, at most
  int64_t                digit_cache_used  = 0;
  ~Ctx();
};

using Range = std::pair<int64_t, int64_t>; // [lo, hi)

struct IndexSpace {
  int64_t                                                 n = 0;
  std::vector<std::pair<std::string, std::vector<Range>>> named;
  std::vector<std::pair<int, std::vector<Range>>>         spin;
  bool                                                    has_spin() const { return !spin.empty(); }
  int                                                     spin_of(int64_t idx) const;
  std::vector<int64_t>                                    boundaries(bool with_named) const;
};

// The root tiling of an IndexSpace (TiledIndexSpaceInfo): tile start offsets and
// the spin of each tile (spin of its first index, tiled_index_space.hpp:1327).
struct RootTiling {
  std::shared_ptr<IndexSpace> is;
  std::vector<int64_t>        offsets; // ntiles + 1
  std::vector<int>            spins;
};

// A tiled index space: a list of root tiles (all of them for the root space,
// a subset for named subspaces and tile sub-ranges).
// Identity of a runtime object for the scheduler's caches: a number no other object
// of this process has had, so that an object created at the address of a destroyed
// one never matches the cache entries of its predecessor.  A copy is a new object.
uint64_t next_serial();
struct Serial {
  uint64_t v;
  Serial() : v(next_serial()) {}
  Serial(const Serial&) : v(next_serial()) {}
  Serial& operator=(const Serial&) { return *this; }
};

// Dependency of a tiled index space on the tiles of other spaces (TAMM's dependent
// TiledIndexSpace, tiled_index_space.hpp:60-72, as DLPNO's PNO space depends on an LMO
// pair): for each tuple of tiles of the `on` spaces, which tiles of the dependent space
// exist; tuples not listed have none.
struct Dependency {
  std::vector<std::shared_ptr<struct TIS>>             on;
  std::map<std::vector<int64_t>, std::vector<uint8_t>> valid; // on-space tiles -> per tile, 1 if it exists
};

struct TIS {
  Serial                      serial;
  std::shared_ptr<RootTiling> root;
  std::vector<int64_t>        tiles;
  std::shared_ptr<Dependency> dep; // set for a dependent space
  int64_t                     ntiles() const { return (int64_t) tiles.size(); }
  int64_t size(int64_t t) const { return root->offsets[tiles[t] + 1] - root->offsets[tiles[t]]; }
  int     spin(int64_t t) const { return root->spins[tiles[t]]; }
  // index of root tile r in this space, -1 if absent (TiledIndexSpace::info_translate)
  int64_t find_root(int64_t r) const;
};

// Kept split digits of a read-only tensor under one operand view (defined by the
// split-INT8 contraction).  retire() returns the entry's device memory and its share
// of the context's cache budget at once, also while a cached contraction layout still
// refers to the entry (that layout is rebuilt before its next launch); the arena's
// frees are stream ordered, so work already enqueued still reads valid memory.
struct DigitCacheEntry {
  virtual ~DigitCacheEntry() = default;
  virtual void retire()      = 0;
};

struct Tensor {
  Serial                            serial;
  int                               nmodes = 0;
  std::vector<std::shared_ptr<TIS>> tis;
  bool                              has_spin = false;
  int                               mask[kMaxModes] = {0};
  std::vector<int64_t>              key_stride;
  std::vector<int64_t>              keys, offsets; // admitted blocks, key order
  int64_t                           nelems = 0;
  std::shared_ptr<Ctx>              ctx;
  double*                           data   = nullptr;
  bool                              owns   = true; // false: storage attached by the caller
  cudaEvent_t                       used   = nullptr; // end of the last compute op that touched it
  cudaEvent_t                       filled = nullptr; // end of the last asynchronous host write
  // Read-only mark (tb_tensor_set_read_only): the contents stay constant while it is
  // set, so contractions may rely on zero_block, one byte per stored block (key order),
  // 1 where every element of the block is zero; ro_serial identifies the marking in
  // the scheduler's cache keys.
  bool                              read_only = false;
  uint64_t                          ro_serial = 0;
  std::vector<uint8_t>              zero_block;
  // split digits of this (read-only) tensor per operand view, kept by the split-INT8
  // contraction (retired whenever the read-only mark changes or the storage goes)
  mutable std::map<std::string, std::shared_ptr<DigitCacheEntry>> digit_cache;
  // lambda tensor (tb_tensor_create_lambda / _built): no storage, blocks on demand
  tb_block_fn                       lambda_block = nullptr;
  tb_batch_fn                       lambda_batch = nullptr;
  void*                             lambda_user  = nullptr;
  int64_t                           batch_bytes  = 0; // per materialised batch (0: default)
  // modes a dependent mode's tiles depend on (empty for an ordinary mode)
  std::vector<std::vector<int>>     dep_modes;
  bool                              is_lambda() const { return lambda_block || lambda_batch; }
  ~Tensor();

  void    build_table(); // Distribution_NW (distribution.hpp:201-243)
  bool    is_non_zero(const int64_t* blockid) const;
  int64_t key(const int64_t* blockid) const;
  int64_t locate(const int64_t* blockid) const; // -1 if not stored
  int64_t block_size(const int64_t* blockid) const;
  void    block_dims(const int64_t* blockid, int32_t* dims) const;
  void    check_blockid(const int64_t* blockid) const;
  void    require_allocated() const;
  void    require_writable() const; // TB_ERR_STATE while the read-only mark is set
  // true if the tensor is marked read-only and the stored block is all zeros
  bool    block_is_zero(const int64_t* blockid) const;
  int64_t block_index(const int64_t* blockid) const; // position in keys, -1 if not stored
};

struct Labeled {
  Tensor*                           t = nullptr;
  std::vector<int>                  labels;
  std::vector<std::shared_ptr<TIS>> ltis; // label space per mode
};

struct DenomSpec;
struct EnergySpec;

// tb_labeled (C ABI) -> Labeled; NULL label spaces mean the tensor's own.
Labeled labeled_from_c(const tb_labeled& x);

struct Op {
  // Dot: scalar slot `slot` = alpha * sum a * b (root: alpha * sqrt(sum a * a)), kept on
  // the device; Denom: lhs += alpha * a / D with the orbital-energy denominator D.
  // DenomEnergy: slot += alpha * sum lhs^2 / D; SetScalar: slot = value.
  // Map: lhs = f(a) element by element (f = TB_MAP_* in `fn`, parameter `value`).
  enum Kind { Set, Add, Mult, Dot, Denom, DenomEnergy, SetScalar, Map } kind;
  Labeled lhs, a, b;
  double  alpha = 1.0, value = 0.0;
  int     is_assign = 0;
  int     slot = 0, root = 0;
  std::shared_ptr<DenomSpec> denom;
  // Mult with the energy epilogue (tb_sched_mult_energy): slot += value * sum
  // (lhs + alpha * a * b)^2 / D over the output blocks the op addresses, lhs unchanged
  // (D from `denom`)
  bool                        energy = false;
  std::shared_ptr<EnergySpec> espec;
  std::string                tune_key; // set when the autotuner chose this op's kernel
  // cached execution state
  std::shared_ptr<Plan>     plan;
  std::shared_ptr<WorkList> wl;
  struct AddBlock {
    int64_t dst_off, src_off;
    int64_t ddims[kMaxModes], sdims[kMaxModes];
  };
  std::shared_ptr<std::vector<AddBlock>> add_blocks;
  std::shared_ptr<int64_t>               add_dev;   // device BlockAssign list (scheduler's cache)
  int                                    add_n = 0;
  int64_t                                add_units = 0; // work units of the list
  int                                    fn = 0;     // Map: element function
  std::shared_ptr<int64_t>               map_dev;    // Map: device segment list (seg_list)
  int                                    map_n = 0;  // runs in the list
  int64_t                                map_total = 0; // elements in the list
  bool                                   flat = false;
  std::shared_ptr<std::vector<int64_t>>  set_blocks; // (offset, size) pairs; empty = whole store
  std::shared_ptr<int64_t>               set_dev;    // set_blocks as a device segment list (scheduler's cache)
  int                                    set_nseg = 0;
  int64_t                                set_total = 0;
  std::string                            fill_key;   // its key in that cache
  // an assignment C = alpha * A * B queued as Set(0) + Mult runs fused on one rank in
  // FP64: the Mult stores its result (store), the Set zeroes only the output blocks the
  // Mult's work list leaves without tasks (fill_none: there are none)
  bool                                   store = false, fill_none = false;
  double                                 flops = 0;
  // blocks of the operands known to be zero by construction at this op's place in its
  // execute (one byte per stored block; null: nothing known): an earlier assignment of
  // the same op list left them without any contribution
  std::shared_ptr<const std::vector<uint8_t>> za, zb;
};

// Orbital energies over a root index space (device copy) and per-mode signs of a
// denominator update, with the block table built on first use.
struct DenomSpec {
  std::vector<double>     eps;   // host copy, indexed by root orbital index
  double                  signs[kMaxModes] = {0};
  double*                 d_eps    = nullptr;
  DenomBlock*             d_blocks = nullptr;
  DenomUnit*              d_units  = nullptr; // row work units (kDenomUnitRows / kDenomUnitElems)
  double*                 d_part   = nullptr; // per-CTA partial sums of the energy reduction
                                              // (nunits entries: the grid is never larger)
  int                     nblocks  = 0, nunits = 0;
  // over the stored blocks of t (only those at the sorted element offsets `only`, if given)
  void                    build(const Tensor& t, const std::shared_ptr<Ctx>& ctx,
                                const std::vector<int64_t>* only = nullptr);
  std::shared_ptr<Ctx>    ctx;
  ~DenomSpec();
};

// Device state of a Mult's energy epilogue, built on its first execution: the
// denominators' first orbital index of each output mode per work-list group (groups
// with tasks: the kernels' epilogue), the kernels' partial sums, and a denominator-
// energy pass over the blocks of groups without tasks.
struct EnergySpec {
  EnergyArgs                 args;
  std::shared_ptr<DenomSpec> rest;
  int64_t                    npart = 0;
  std::shared_ptr<Ctx>       ctx;
  ~EnergySpec();
};

// Choice of the autotuner for one contraction signature and precision request.
struct TuneChoice {
  int                 mode   = TB_MODE_FP64;
  int                 tile_n = 0;
  std::vector<double> ms;     // timed candidates, in candidate order
  std::vector<int>    modes, tiles;
};

struct Sched {
  std::shared_ptr<Ctx>                              ctx;
  std::vector<Op>                                   ops;
  size_t                                            start = 0, last_first = 0; // ops[last_first, start): last execute
  std::vector<double>                               prof_ms, prof_flops;
  std::vector<tb_stats>                             prof_stats;
  bool                                              profiling = false;
  std::map<std::string, std::shared_ptr<Plan>>     plan_cache;
  std::map<std::string, std::shared_ptr<WorkList>> wl_cache;
  // device block lists of SetOps over some of a tensor's blocks, by the op's signature
  // (or, for the fill of a fused assignment, its contraction's), uploaded once
  std::map<std::string, std::shared_ptr<int64_t>>  fill_cache;
  std::map<std::string, int>                        map_count; // triples of each cached map list
  std::map<std::string, int64_t>                    add_units; // work units of each cached add list
  std::map<std::string, int64_t>                    seg_total; // elements of each cached segment list
  // intermediates of multi-factor products (tb_sched_mult_n), by signature; freed with
  // the scheduler
  std::map<std::string, std::unique_ptr<Tensor>>    temps;
  // batch tensors of lambda operands (storage only while a batch runs) and the
  // scheduler that batch builders queue their ops on
  std::map<std::string, std::unique_ptr<tb_tensor_s>> lambda_batches;
  std::unique_ptr<tb_sched_s>                         builder;
  // work lists of lambda batches run while capturing a graph (their error words are
  // checked by the graph's sync)
  std::vector<std::shared_ptr<WorkList>>              batch_lists;
  // blocks known to be zero by construction at the end of the last execute
  std::map<const Tensor*, std::shared_ptr<std::vector<uint8_t>>> last_zeros;
  void                                                run_lambda_mult(Op& op);
  static constexpr int                              kSlots = 64;
  double*                                           d_scalars = nullptr; // kSlots + 1024 partials
  bool                                              autotune  = false;
  int                                               rank = 0, nranks = 1; // owner-computes share of Mult ops
  std::map<std::string, TuneChoice>                 tune_cache;
  CapturePool*                                      pinned = nullptr; // set while capturing a graph
  bool                                              deferred_checks = false; // execute_async
  std::vector<std::shared_ptr<WorkList>>            pending;         // INT8 lists to check at wait()
  void                                              execute(bool profile);
  void                                              run(Op& op);
  void                                              prepare_mult(Op& op);
  void note_zeros(const Op& op, std::map<const Tensor*, std::shared_ptr<std::vector<uint8_t>>>& szero);
  void                                              fuse_assign(Op& set, Op& mult);
  void                                              tune(Op& op, const std::string& key);
  double*                                           scalars();
  ~Sched();
};

// Multi-factor products (tb_opmin.cpp): queue as binary contractions; the chosen tree.
void queue_mult_n(Sched& s, const Labeled& lhs, double alpha, const std::vector<Labeled>& f, int is_assign,
                  const std::function<void(Op&&)>& push);
void mult_n_order(const Labeled& lhs, const std::vector<Labeled>& f, std::vector<int64_t>& pairs, double& cost);

// A captured sequence of scheduler ops: replayed with one graph launch.  Holds the
// scratch the capture used and the work lists whose error words are checked.
struct Graph {
  std::shared_ptr<Ctx>                   ctx;
  cudaGraph_t                            graph = nullptr;
  cudaGraphExec_t                        exec  = nullptr;
  CapturePool                            pool;
  std::vector<std::shared_ptr<WorkList>> int8_lists;
  std::vector<std::shared_ptr<Plan>>     plans;
  ~Graph();
};

// scratch memory source for split operands
struct Scratch {
  Arena*       arena  = nullptr; // null: cudaMallocAsync on the stream
  cudaStream_t stream = nullptr;
  void*        get(int64_t bytes);
  void         put(void* p);
};

} // namespace tb

struct tb_ctx_s {
  std::shared_ptr<tb::Ctx> p;
};
struct tb_is_s {
  std::shared_ptr<tb::IndexSpace> p;
};
struct tb_tis_s {
  std::shared_ptr<tb::TIS> p;
};
struct tb_tensor_s {
  std::unique_ptr<tb::Tensor> p;
};
struct tb_sched_s {
  std::unique_ptr<tb::Sched> p;
};
struct tb_graph_s {
  std::unique_ptr<tb::Graph> p;
};
struct tb_plan_s {
  tb::Plan p;
};
struct tb_worklist_s {
  std::unique_ptr<tb::WorkList> p;
};
