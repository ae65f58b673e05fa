/*
 * tamm_b200 — C ABI of the B200-native block-sparse tensor-contraction path.
 *
 * Drop-in boundary for TAMM's block-contraction hot path.  Two tiers:
 *
 *  1. Kernel tier: replaces the block kernels TAMM's operations call
 *     (tamm::kernels::block_multiply, tamm::kernels::assign, the GEMM wrappers) and
 *     adds the grouped, device-built work-list form of MultOp::execute_bufacc.
 *     Device pointers in, device pointers out, explicit CUDA stream.
 *
 *  2. Runtime tier: index spaces, tiled index spaces, block-sparse tensors in a
 *     device-resident block store, and a Scheduler that queues Set/Add/Mult ops and
 *     executes them on the GPU.  This is what TAMM's LabeledTensor/Scheduler API
 *     lowers to; the C++ header tamm_b200/include/tamm_b200/tamm.hpp and the Python
 *     package tamm_b200 are thin front-ends over it.
 *
 * Conventions: every function returns an int status (TB_OK == 0).  No C++
 * exception crosses the boundary; tb_last_error() returns the message of the last
 * failure on the calling thread.  Labels are plain ints: equal ints name the same
 * index label (TAMM's per-op int labels, multop.hpp:955-970).  Block dims are tile
 * extents, row-major, last mode fastest (TAMM's block layout).  All floating-point
 * data is double (FP64), the element type of every configuration in scope.
 * Citations are relative to the TAMM source tree.
 */
#ifndef TAMM_B200_H
#define TAMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define TB_OK 0
#define TB_ERR_INVALID 1         /* malformed arguments: TAMM's EXPECTS (errors.hpp:49-57) */
#define TB_ERR_NOT_IMPLEMENTED 2 /* TAMM's NOT_IMPLEMENTED() */
#define TB_ERR_NO_MEMORY 3       /* device arena / host allocation failed */
#define TB_ERR_CUDA 4            /* a CUDA runtime call failed (TAMM's CUDA_CHECK) */
#define TB_ERR_TIMEOUT 5         /* a bounded device-side wait gave up */
#define TB_ERR_DEVICE 6          /* a kernel raised its device error flag */
#define TB_ERR_STATE 7           /* object used in the wrong state (e.g. not allocated) */

/* Human-readable name of a status code. */
const char* tb_status_string(int status);
/* Copies the last failure message of the calling thread into buf (NUL-terminated). */
int tb_last_error(char* buf, size_t len);
/* Library version (major, minor). */
int tb_version(int* major, int* minor);

/* --------------------------------------------------------------- precision modes */
#define TB_MODE_FP64 0   /* plain FP64 (DMMA tensor-core) contraction */
#define TB_MODE_INT8 1   /* Ozaki-style split-INT8: INT8 slices, INT32 tcgen05 MMA, FP64 recombination */
#define TB_MODE_BF16X3 2 /* three-term BF16 split, FP32 accumulate (FP32-class accuracy) */

/* ================================================================ KERNEL TIER === */

/* C (=|+=) alpha * A * B for ONE block triple, device buffers.
 * Replaces tamm::kernels::block_multiply<T,T1,T2,T3>(th_a, th_b, thandle, alpha,
 * abuf, adims, alabels, bbuf, bdims, blabels, beta, cbuf, cdims, clabels, hw,
 * is_assign, cinter_buf_dev, cinter_tmp_buf_dev) (src/tamm/kernels/multiply.hpp:212-220)
 * for T = double.  Labels are classified as batch / A-outer / B-outer / inner /
 * A-only / B-only exactly as multiply.hpp:237-302; beta chains the A-only x B-only
 * reduction steps as gemm_wrapper does (multiply.hpp:42-74); the result is assigned
 * (is_assign) or accumulated into C in C's own label order (transpose_output,
 * multiply.hpp:196-210).  No intermediate transposed copy is made.  mode: TB_MODE_*.
 * Scratch memory is taken from cudaMallocAsync on `stream` when mode needs it. */
int tb_block_multiply(double alpha, const double* a, const int64_t* adims, const int* alabels,
                      int na, const double* b, const int64_t* bdims, const int* blabels, int nb,
                      double beta, double* c, const int64_t* cdims, const int* clabels, int nc,
                      int is_assign, int mode, void* stream);

/* dst (=|+=) scale * src with labels mapping modes, device buffers.
 * Replaces tamm::kernels::assign<T>(dst, ddims, dlabels, scale, src, sdims, slabels,
 * is_assign) (src/tamm/kernels/assign.hpp:467-485): label permutations (the HPTT
 * branch, assign.hpp:375-401) and the general strided loop (ip_gen_loop,
 * assign.hpp:312-373, up to 4 dst modes) share one device kernel.  Also serves
 * internal::block_add (assign.hpp:418-460) and BlockAssignPlan::apply
 * (block_assign_plan.hpp:111-157). */
int tb_block_assign(double* dst, const int64_t* ddims, const int* dlabels, int nd, double scale,
                    const double* src, const int64_t* sdims, const int* slabels, int ns,
                    int is_assign, void* stream);

/* x[0:n] = value (is_assign) or x[0:n] += value.  Device-side SetOp body
 * (src/tamm/setop.hpp:130-274). */
int tb_fill(double* x, int64_t n, double value, int is_assign, void* stream);

/* y[0:n] = alpha * x[0:n] + beta * y[0:n] on the device (the axpy of multop.hpp:830
 * and the flat AddOp plan, addop.hpp:426-454). */
int tb_axpby(double alpha, const double* x, double beta, double* y, int64_t n, void* stream);

/* Split-INT8 C += alpha * A * B for ONE block triple without allocating anything.
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory — applications whose device memory is already owned by other
 * allocators (TAMM's RMM pool takes 80% of the free memory at start-up, a caching
 * allocator the rest), or code that must not trigger the device-wide
 * synchronisation cudaMalloc / cudaFree can cause.  It makes no cudaMalloc,
 * cudaMallocAsync or cudaFree call and, when it succeeds, allocates no host memory
 * either (a failure builds its tb_last_error message string): its scratch (digit
 * slices, exponents, the one-task work list) is a file-scope device array of 64 MiB
 * that every GPU loading the library holds until exit.  A triple needing more scratch
 * (about 6 * K * (M + N) bytes at the default 6 digits) is rejected with
 * TB_ERR_INVALID and a message giving the size.  Labels as in tb_block_multiply
 * (plain contractions only: no Hadamard or one-sided reduction labels); nslices 0
 * picks the digit count for a 1e-11 target, 3..8 forces it.  The first call on a
 * device looks up the array's device address for that device, once.  Every call
 * reuses the same array and leaves its contents behind; each call resets what it
 * needs to start from a known value, and calls that overlap on the GPU (other
 * streams, other threads) race on the array.  The call reads its status back and
 * returns after the stream has drained, so it cannot be captured into a CUDA graph
 * (a call on a capturing stream returns TB_ERR_INVALID before enqueuing anything). */
int tb_block_multiply_int8_noalloc(double alpha, const double* a, const int64_t* adims,
                                   const int* alabels, int na, const double* b,
                                   const int64_t* bdims, const int* blabels, int nb, double* c,
                                   const int64_t* cdims, const int* clabels, int nc, int nslices,
                                   void* stream);

/* sqrt(sum x^2) over x[0:n], written to *host_out after the stream drains
 * (tamm::norm, src/tamm/tamm_utils.hpp:1180-1200).  Deterministic two-pass reduction. */
int tb_norm2(const double* x, int64_t n, double* host_out, void* stream);

/* sum x*y over [0:n] into *host_out (deterministic). */
int tb_dot(const double* x, const double* y, int64_t n, double* host_out, void* stream);

/* Seeded counter-based fill (same stream as the test oracle's generator up to the
 * last ulp of log/cos): dist 0 = uniform [p0, p1), 1 = normal(mean p0, sd p1). */
int tb_fill_random(double* x, int64_t n, uint64_t seed, uint64_t first, int dist, double p0,
                   double p1, void* stream);

/* ---- grouped contraction: the whole MultOp::execute_bufacc loop in one launch ---- */

/* A contraction plan: label classes of C(clabels) += A(alabels) * B(blabels) as in
 * multiply.hpp:237-330, plus the precision mode.  err_target is the max relative
 * error allowed for TB_MODE_INT8 (slice count chosen per block from it; <= 0 picks
 * the default 1e-11); nslices > 0 forces the slice count (6..8). */
typedef struct tb_plan_s* tb_plan;
int tb_plan_contraction(const int* clabels, int nc, const int* alabels, int na, const int* blabels,
                        int nb, int mode, double err_target, int nslices, tb_plan* out);
int tb_plan_destroy(tb_plan plan);

/* A device work list for a plan: output-block groups, each with the (A block,
 * B block) tasks of its admitted reduction tiles (multop.hpp:645-851).  Offsets are
 * element offsets into the A/B/C arenas; dims are the blocks' tile extents in each
 * tensor's own mode order.  group_task_begin has ngroups+1 entries. */
typedef struct tb_worklist_s* tb_worklist;
int tb_worklist_build(tb_plan plan, int64_t ngroups, const int64_t* group_c_off,
                      const int32_t* group_cdims, const int64_t* group_task_begin,
                      const int64_t* task_a_off, const int64_t* task_b_off,
                      const int32_t* task_adims, const int32_t* task_bdims, tb_worklist* out);
int tb_worklist_destroy(tb_worklist wl);
/* Number of tasks and admitted FP64 FLOPs (2 * |C block| * K per task). */
int tb_worklist_info(tb_worklist wl, int64_t* ntasks, double* flops);

/* Per-launch statistics of the last tb_contract on a plan. */
typedef struct tb_stats {
  double flops;           /* admitted FP64 FLOPs */
  double int8_ops;        /* INT8 tensor-core ops issued (TB_MODE_INT8) */
  int    slices_min;      /* slice counts chosen (TB_MODE_INT8) */
  int    slices_max;
  int64_t scratch_bytes;  /* scratch used by the split operands */
  double split_ms;        /* device time of the operand splitting (profiled runs) */
  double gemm_ms;         /* device time of the tensor-core contraction kernel (profiled runs) */
  int    mode;            /* kernel that ran: TB_MODE_FP64 or TB_MODE_INT8 (autotuner's choice) */
  int    tile_n;          /* split-INT8 output tile width (0: the default for the slice count) */
  double flops_run;       /* FP64 FLOPs of the tasks that ran: admitted minus the tasks skipped
                             over exactly-zero blocks of read-only operands */
  double int8_ops_alg;    /* the INT8 ops of int8_ops without tile padding (profiled runs) */
} tb_stats;

/* C += alpha * sum over tasks of A * B, all groups, one stream-ordered pass.
 * Scratch (INT8 slices) comes from cudaMallocAsync on the stream. */
int tb_contract(tb_plan plan, tb_worklist wl, double alpha, const double* a, const double* b,
                double* c, void* stream);
int tb_plan_stats(tb_plan plan, tb_stats* out);

/* =============================================================== RUNTIME TIER === */

/* ExecutionContext (src/tamm/execution_context.hpp:120): one GPU, one stream, a
 * stream-ordered device arena of pool_bytes (0 = 80% of free memory, TAMM's
 * TAMM_GPU_POOL default, rmm_memory_pool.hpp:30-46), and the precision options. */
typedef struct tb_ctx_s* tb_ctx;
int tb_ctx_create(int device, int64_t pool_bytes, tb_ctx* out);
int tb_ctx_destroy(tb_ctx ctx);
int tb_ctx_set_precision(tb_ctx ctx, int mode, double err_target, int nslices);
int tb_ctx_stream(tb_ctx ctx, void** stream);
int tb_ctx_synchronize(tb_ctx ctx); /* compute and copy streams */
/* Makes later work on the compute stream wait for everything enqueued so far on the
 * context's copy streams (e.g. to time transfers with events on the compute stream). */
int tb_ctx_join(tb_ctx ctx);
/* Digit cache (no counterpart in TAMM): up to `bytes` of the context's arena keep the
 * split-INT8 digits of read-only tensors (tb_tensor_set_read_only) per operand view,
 * so that a constant operand, such as the integrals of a coupled-cluster run, is split
 * once instead of in every contraction that reads it.  0 (the default) turns it off
 * and frees nothing already kept (entries go when their tensor's mark changes).
 * *used receives the bytes kept now. */
int tb_ctx_set_digit_cache(tb_ctx ctx, int64_t bytes);
int tb_ctx_digit_cache_info(tb_ctx ctx, int64_t* used, int64_t* limit);
/* Sub-allocation from the context's stream-ordered arena (TAMM's RMM pool,
 * rmm_memory_pool.hpp:50-263): 256-byte aligned device memory, reusable by any
 * later work on the context's stream as soon as it is freed. */
int tb_ctx_alloc(tb_ctx ctx, int64_t bytes, void** out);
int tb_ctx_free(tb_ctx ctx, void* p);
/* Arena occupancy: bytes in use, high-water mark, capacity. */
int tb_ctx_arena_info(tb_ctx ctx, int64_t* used, int64_t* peak, int64_t* capacity);

/* IndexSpace{range(n), {{name, {ranges}}...}, {{Spin{s}, {ranges}}...}}
 * (src/tamm/index_space.hpp:64).  name_ranges / spin_ranges hold [lo, hi) pairs,
 * name_nranges[i] / spin_nranges[i] of them per name / spin value. */
typedef struct tb_is_s* tb_is;
int tb_is_create(int64_t n, int nnamed, const char* const* names, const int* name_nranges,
                 const int64_t* name_ranges, int nspin, const int* spin_values,
                 const int* spin_nranges, const int64_t* spin_ranges, tb_is* out);
int tb_is_destroy(tb_is is);

/* TiledIndexSpace{is, tile} (tiles == NULL) or TiledIndexSpace{is, tile_list}
 * (src/tamm/tiled_index_space.hpp:31,49; tiling rules :1135-1262). */
typedef struct tb_tis_s* tb_tis;
int tb_tis_create(tb_is is, int64_t tile, const int64_t* tiles, int64_t ntiles, tb_tis* out);
/* tis("name"): the tiles of a named subspace (e.g. MO("occ")). */
int tb_tis_named(tb_tis tis, const char* name, tb_tis* out);
/* TiledIndexSpace{tis, range(first, last)}: tiles [first, last) of tis
 * (tiled_index_space.hpp:84-110). */
int tb_tis_subrange(tb_tis tis, int64_t first_tile, int64_t last_tile, tb_tis* out);
int tb_tis_num_tiles(tb_tis tis, int64_t* ntiles);
/* Per tile: size, spin (of its first index, tiled_index_space.hpp:342-345,1327)
 * and index in the root tiled space.  Arrays hold num_tiles entries. */
int tb_tis_tiles(tb_tis tis, int64_t* sizes, int* spins, int64_t* root_tiles);
int tb_tis_destroy(tb_tis tis);
/* Dependent tiled index space (TiledIndexSpace{reference, {on...}, dep_map},
 * src/tamm/tiled_index_space.hpp:60-72; DLPNO's PNO space over LMO pairs): for key n,
 * the tile tuple keys[n * ndep .. n * ndep + ndep) of the spaces `on` (1..4 of them,
 * ordinary spaces) maps to the sub-space values[n] of `reference`, whose tiles are the
 * dependent space's tiles for that tuple; tuples not listed have no tiles.  The
 * dependent space has the reference's tiles; a tensor mode over it exists only where
 * its tile is listed for the tiles of the modes it depends on. */
int tb_tis_create_dependent(tb_tis reference, int ndep, const tb_tis* on, int64_t nkeys, const int64_t* keys,
                            const tb_tis* values, tb_tis* out);

/* Tensor<T>{tis...} or Tensor<T>{{tis...}, SpinMask} (src/tamm/tensor.hpp:87-136,
 * spin rule tensor_base.hpp:243-263).  spin_mask NULL: no spin symmetry; else per
 * mode 0 upper, 1 lower, 2 ignore.  Blocks are stored in Distribution_NW order
 * (distribution.hpp:197-285): admitted blocks sorted by row-major tile key,
 * packed contiguously in one device arena allocation. */
typedef struct tb_tensor_s* tb_tensor;
int tb_tensor_create(int nmodes, const tb_tis* tis, const int* spin_mask, tb_tensor* out);
/* Tensor with dependent modes (Tensor<T>{i, j, a(i, j), e(i, j)}): dep_modes holds 4
 * ints per mode, the modes a mode over a dependent space depends on (in the order of
 * that space's `on` list; -1 unused); admitted blocks also satisfy the dependency
 * (translate_blockid_if_possible, src/tamm/utils.hpp:369). */
int tb_tensor_create_dependent(int nmodes, const tb_tis* tis, const int* spin_mask, const int* dep_modes,
                               tb_tensor* out);
/* Tensor{{tis...}, {nupper, nlower}} form (tensor_impl.hpp:153-209). */
int tb_tensor_create_spin_sizes(int nmodes, const tb_tis* tis, int nupper, int nlower,
                                tb_tensor* out);
int tb_tensor_allocate(tb_tensor t, tb_ctx ctx);
int tb_tensor_deallocate(tb_tensor t);
int tb_tensor_destroy(tb_tensor t);
int tb_tensor_info(tb_tensor t, int* nmodes, int64_t* nblocks, int64_t* nelems);
/* Packed block table in storage order: keys and element offsets (nblocks each). */
int tb_tensor_block_table(tb_tensor t, int64_t* keys, int64_t* offsets);
int tb_tensor_data(tb_tensor t, double** device_ptr);
/* Read-only mark (no counterpart in TAMM): on != 0 declares the tensor's contents
 * constant until the mark is cleared, e.g. the two-electron integrals of a
 * coupled-cluster iteration.  While it is set, every library call that would write
 * the tensor fails with TB_ERR_STATE (tb_tensor_put / add / write / write_async /
 * load, and Set / Add / Mult / denominator ops with it on the left-hand side, at
 * execute time); writes through the pointer of tb_tensor_data are the caller's to
 * avoid.  Setting the mark scans the stored blocks once on the device (after the work
 * already enqueued on the context's stream) for blocks whose elements are all zero
 * (+0.0 or -0.0).  Contractions then skip every admitted task over such a block: its
 * product is exactly zero, so the result is the same up to the sign of zero entries
 * of C (non-finite values in the other operand's block are not propagated through a
 * skipped task, as with BLAS implementations that skip zero operands).  The skipped
 * tasks still count in the admitted FLOPs (tb_stats.flops) and not in
 * tb_stats.flops_run.  Deallocating the tensor clears the mark; on == 0 clears it. */
int tb_tensor_set_read_only(tb_tensor t, int on);
/* Whether the mark is set, and how many stored blocks / elements the scan found zero. */
int tb_tensor_read_only_info(tb_tensor t, int* on, int64_t* zero_blocks, int64_t* zero_elems);
int tb_tensor_is_non_zero(tb_tensor t, const int64_t* blockid, int* out);
int tb_tensor_block_size(tb_tensor t, const int64_t* blockid, int64_t* out);
int tb_tensor_block_dims(tb_tensor t, const int64_t* blockid, int64_t* dims);
/* Element offset of a stored block, -1 if the block is not admitted. */
int tb_tensor_locate(tb_tensor t, const int64_t* blockid, int64_t* offset);
/* Gives an unallocated tensor caller-owned device storage of >= 8 * nelems bytes,
 * 16-byte aligned (no counterpart in TAMM): several tensors used one after another
 * in stream order can share one buffer, e.g. the batches of an integral tensor
 * built on demand.  tb_tensor_deallocate detaches it without freeing. */
int tb_tensor_attach(tb_tensor t, tb_ctx ctx, void* device_ptr, int64_t bytes);
/* Lambda tensors (Tensor<T>(tis, Func), src/tamm/tensor.hpp:166-190, whose
 * LambdaTensorImpl computes a block on request, src/tamm/tensor_impl.hpp:566-693): a
 * tensor without storage whose blocks are produced on demand.  A contraction that
 * reads it (either operand) is run in batches along the lambda tensor's first mode:
 * the tiles of that mode's label space are cut into consecutive ranges whose admitted
 * blocks fit the batch budget (tb_tensor_set_batch_bytes; default a quarter of the
 * context arena's free bytes), each range is materialised into scratch on the context's
 * stream and contracted with the label restricted to those tiles, then released.
 *  - tb_tensor_create_lambda: fn fills ONE block (TAMM's lambda): blockid in the
 *    tensor's own tile numbering, its dims, and a device buffer of n doubles that fn
 *    must fill with work enqueued on `stream` (or before returning); nonzero return
 *    aborts the op with TB_ERR_INVALID.
 *  - tb_tensor_create_built: fn fills a whole batch at once (no counterpart in TAMM):
 *    `batch` is an allocated tensor over tiles [first_tile, last_tile) of the first
 *    mode's label space and the full other modes, and fn queues ops writing it on
 *    `sch` (a scheduler on the same context, executed right after fn returns), e.g.
 *    batch(a',b,c,d) = L(Q,a',c) * L(Q,b,d) for integrals built from Cholesky vectors.
 * Only contractions read lambda tensors (other ops fail with TB_ERR_NOT_IMPLEMENTED);
 * a graph capture records the callbacks' device work, so they must only enqueue work
 * on the stream they are given. */
typedef struct tb_sched_s* tb_sched; /* Scheduler handle (declared with its calls below) */
typedef int (*tb_block_fn)(const int64_t* blockid, int nmodes, const int64_t* dims, double* block, int64_t n,
                           void* stream, void* user);
typedef int (*tb_batch_fn)(tb_tensor batch, int64_t first_tile, int64_t last_tile, tb_sched sch, void* user);
int tb_tensor_create_lambda(int nmodes, const tb_tis* tis, const int* spin_mask, tb_block_fn fn, void* user,
                            tb_tensor* out);
int tb_tensor_create_built(int nmodes, const tb_tis* tis, const int* spin_mask, tb_batch_fn fn, void* user,
                           tb_tensor* out);
/* Device bytes one batch of a lambda tensor may take (0: a quarter of the free arena). */
int tb_tensor_set_batch_bytes(tb_tensor t, int64_t bytes);
/* A new handle to the tiled space of mode `mode` of t (destroy with tb_tis_destroy),
 * e.g. the first-mode tile range of a lambda tensor's batch. */
int tb_tensor_space(tb_tensor t, int mode, tb_tis* out);

/* Tensor::get / put / add of one block with a HOST buffer of n >= block size
 * (tensor_impl.hpp:321-455; get of a non-admitted block returns zeros). */
int tb_tensor_get(tb_tensor t, const int64_t* blockid, double* host, int64_t n);
int tb_tensor_put(tb_tensor t, const int64_t* blockid, const double* host, int64_t n);
int tb_tensor_add(tb_tensor t, const int64_t* blockid, const double* host, int64_t n);
/* Asynchronous whole-store transfers with pinned host memory (no counterpart in
 * TAMM): they run on the context's copy streams, a write after the compute work
 * already enqueued on the tensor and before any compute enqueued later, a read after
 * the compute work enqueued on the tensor.  With two sets of tensors used in turn,
 * the transfers of one step overlap the contraction of the next.  The host buffer
 * must stay untouched until tb_ctx_synchronize / tb_sched_wait returns. */
int tb_tensor_write_async(tb_tensor t, const double* host, int64_t n);
int tb_tensor_read_async(tb_tensor t, double* host, int64_t n);
/* Marks the end of the work enqueued so far on the context's compute stream as the
 * tensor's last use (no counterpart in TAMM): a caller that enqueues its own work on
 * the tensor there, e.g. an NCCL all-reduce assembling the shares of an owner-computes
 * contraction, calls it so that a later asynchronous read or write waits for that
 * work too. */
int tb_tensor_record_use(tb_tensor t);
/* Whole packed store <-> host (n == nelems). */
int tb_tensor_write(tb_tensor t, const double* host, int64_t n);
int tb_tensor_read(tb_tensor t, double* host, int64_t n);
int tb_tensor_norm(tb_tensor t, double* out);
/* Checkpoint / restart (TAMM's write_to_disk / read_from_disk, tamm_io.hpp:230-465,
 * in its tammio element order: admitted blocks in row-major tile order, each block
 * row-major — a raw file instead of an HDF5 dataset).  The file records the spaces'
 * tiles, spins and the spin mask; load checks them against the tensor. */
int tb_tensor_save(tb_tensor t, const char* path);
int tb_tensor_load(tb_tensor t, const char* path);

/* A labelled operand: tensor, per-mode int label, per-mode label space (NULL array
 * or NULL entry: the tensor's own tiled space; else a sub-space of it, as for
 * TiledIndexLabels of MO("occ") on a tensor over MO). */
typedef struct tb_labeled {
  tb_tensor     tensor;
  const int*    labels;
  const tb_tis* label_tis;
} tb_labeled;

/* Scheduler (src/tamm/scheduler.hpp:40-51,160-438): ops are queued with
 * operator() and run by execute() in dependence levels on the context's stream. */
int tb_sched_create(tb_ctx ctx, tb_sched* out);
int tb_sched_destroy(tb_sched s);
/* SetOp: lhs = value (is_assign) or lhs += value. */
int tb_sched_set(tb_sched s, tb_labeled lhs, double value, int is_assign);
/* AddOp: lhs (=|+=) alpha * rhs (addop.hpp:242-271). */
int tb_sched_add(tb_sched s, tb_labeled lhs, double alpha, tb_labeled rhs, int is_assign);
/* MultOp: lhs (=|+=) alpha * a * b; "=" is canonicalised to SetOp(0) then "+="
 * (multop.hpp:255-269). */
int tb_sched_mult(tb_sched s, tb_labeled lhs, double alpha, tb_labeled a, tb_labeled b,
                  int is_assign);
/* Work of lhs += a * b without running it: admitted output blocks, admitted
 * (C, A, B) block triples and their FP64 FLOPs, from the same enumeration the
 * MultOp uses (multop.hpp:645-893).  Needs no GPU and no allocation.  Triples over
 * zero blocks of read-only operands are counted (they are admitted). */
int tb_mult_info(tb_labeled lhs, tb_labeled a, tb_labeled b, int64_t* ngroups, int64_t* ntasks,
                 double* flops);
/* Owner-computes share for one of nranks processes (TAMM's rule, multop.hpp:880-891,
 * with a FLOP-balanced assignment): Mult ops of this scheduler compute only the
 * output blocks this rank owns; Set and Add ops still cover the whole local tensor.
 * Every rank derives the same assignment from the same operands, without exchange;
 * assembling the result (e.g. an all-reduce of a zero-initialised output) is the
 * caller's. */
int tb_sched_set_owner(tb_sched s, int rank, int nranks);
/* Output blocks of lhs += a * b owned by `rank` of nranks: their number, FP64 FLOPs
 * and packed offsets in lhs (up to cap).  Host-only, like tb_mult_info. */
int tb_mult_owned(tb_labeled lhs, tb_labeled a, tb_labeled b, int rank, int nranks, int64_t* ngroups,
                  double* flops, int64_t* c_offsets, int64_t cap);
/* Scheduler::execute(ExecutionHW, profile).  hw: 0 DEFAULT, 1 CPU, 2 GPU — every op
 * runs on the GPU (there is no host execution path); profile records per-op device
 * times readable with tb_sched_profile. */
int tb_sched_execute(tb_sched s, int hw, int profile);
/* Scheduler::execute without waiting: the ops are enqueued on the context's stream
 * and the call returns; split-INT8 device error words are checked by tb_sched_wait,
 * which waits for the compute and copy streams. */
int tb_sched_execute_async(tb_sched s);
int tb_sched_wait(tb_sched s);
/* Number of ops in the last execute; per op: device milliseconds and FP64 FLOPs. */
int tb_sched_profile(tb_sched s, int64_t* nops, double* ms, double* flops, int64_t cap);
/* Kernel statistics of op `index` of the last profiled execute (zeros for Set/Add ops). */
int tb_sched_op_stats(tb_sched s, int64_t index, tb_stats* out);
/* Drops queued ops without running them. */
int tb_sched_clear(tb_sched s);
/* Waits for the stream, then frees the plans and work lists (with their device
 * arrays) cached for executed ops; queued ops stay.  For long streams of
 * contractions that never repeat (e.g. a triples energy streamed over occupied
 * indices), call it between steps.  Graphs keep what they use. */
int tb_sched_release(tb_sched s);

/* Scalar results kept on the device, in 64 slots per Scheduler (read with
 * tb_sched_scalars after execute or a graph launch): slot = alpha * sum a * b over
 * the stored elements (a and b with the same labels and block layout), or
 * slot = alpha * sqrt(sum a * a) (tamm::norm, tamm_utils.hpp:1180-1200). */
int tb_sched_dot(tb_sched s, int slot, double alpha, tb_labeled a, tb_labeled b);
int tb_sched_norm(tb_sched s, int slot, double alpha, tb_labeled a);
int tb_sched_scalars(tb_sched s, double* host, int n);
/* Multi-factor product lhs (=|+=) alpha * F_0 * ... * F_(n-1) (TAMM's OpMin /
 * OpExecutor, src/tamm/opmin.hpp:395-660, src/tamm/op_executor.hpp): the binary
 * contraction tree of least cost under opmin::Optimizer's model (dynamic programming
 * over factor subsets; a pair costs the product of the dense extents of the labels the
 * two parts still need) is queued as Set(0) + Mult ops into intermediates over the
 * needed labels (no spin symmetry; owned by the scheduler and reused when the same
 * product is queued again), the root updating lhs.  n = 1 is an AddOp, n = 2 a MultOp. */
int tb_sched_mult_n(tb_sched s, tb_labeled lhs, double alpha, const tb_labeled* factors, int n, int is_assign);
/* The tree tb_sched_mult_n would run, host only: pairs[2k], pairs[2k+1] are the factor
 * bit masks joined by the k-th binary contraction (execution order, n - 1 steps), and
 * *cost the model's total. */
int tb_opmin_order(tb_labeled lhs, const tb_labeled* factors, int n, int64_t* pairs, double* cost);

/* MapOp family (src/tamm/mapop.hpp:28-120; Scheduler::exact_copy, scheduler.hpp:461-474;
 * apply_ewise_ip / apply_ewise and their wrappers, tamm_utils.hpp:866-1100) on the
 * device: lhs(labels) = f(rhs(labels)) element by element, over the blocks of lhs
 * admitted in its label spaces; rhs carries the same labels in the same order (the
 * same block ids, translated to its own tiled spaces as TAMM's translate_blockid) and
 * may be lhs itself (in place).  A block of rhs that is not stored reads as zeros, as
 * TAMM's get of a non-admitted block.  Device code cannot run a host lambda, so f is
 * one of the element functions below (those of TAMM's apply_ewise wrappers), with
 * parameter p where noted. */
#define TB_MAP_COPY 0    /* x            (exact_copy) */
#define TB_MAP_SCALE 1   /* p * x        (scale, scale_ip) */
#define TB_MAP_SET 2     /* p            (set_val_ip) */
#define TB_MAP_SQUARE 3  /* x * x        (square) */
#define TB_MAP_SQRT 4    /* sqrt(x)      (sqrt) */
#define TB_MAP_LOG 5     /* log(x)       (log) */
#define TB_MAP_LOG10 6   /* log10(x)     (log10) */
#define TB_MAP_INVERSE 7 /* 1 / x        (einverse) */
#define TB_MAP_POW 8     /* pow(x, p)    (pow) */
#define TB_MAP_ABS 9     /* |x| */
int tb_sched_map(tb_sched s, tb_labeled lhs, tb_labeled rhs, int fn, double p);

/* Orbital-energy denominator update of CC amplitudes (TAMM's jacobi_cc via
 * apply_ewise, tamm_utils.hpp:866-936): t += alpha * r / D element by element, with
 * D = sum over modes of signs[m] * eps[orbital index of mode m] (eps over the root
 * index space shared by t's modes, neps entries; r with t's labels and layout). */
int tb_sched_denom(tb_sched s, tb_labeled t, double alpha, tb_labeled r, const double* eps, int64_t neps,
                   const double* signs);
/* slot += alpha * sum w^2 / D over w's stored elements, D as in tb_sched_denom: the
 * energy reduction of a perturbative-triples-style term, without storing w / D
 * (no counterpart in TAMM's ops).  tb_sched_set_scalar queues slot = value. */
int tb_sched_denom_energy(tb_sched s, int slot, double alpha, tb_labeled w, const double* eps, int64_t neps,
                          const double* signs);
/* slot += scale * sum (lhs + alpha * a * b)^2 / D over the elements of the output
 * blocks the contraction addresses, D as in tb_sched_denom, lhs left unchanged: the
 * MultOp lhs += alpha * a * b (multop.hpp:576-893) with tb_sched_denom_energy fused
 * into the contraction's epilogue, so the summed tensor is read once and never
 * written (no counterpart in TAMM's ops).  Blocks without contributions enter with
 * their stored values.  Lambda operands are not supported (TB_ERR_NOT_IMPLEMENTED). */
int tb_sched_mult_energy(tb_sched s, int slot, double scale, tb_labeled lhs, double alpha, tb_labeled a,
                         tb_labeled b, const double* eps, int64_t neps, const double* signs);
int tb_sched_set_scalar(tb_sched s, int slot, double value);
/* Autotuner (no counterpart in TAMM): with enable != 0, the first execution of each
 * contraction under a split-INT8 request times the candidate kernels (FP64; split-
 * INT8 with output tiles 80 / 64 / 48 wide where the slice count allows) on a saved
 * copy of the output and keeps the fastest for that contraction and request. */
int tb_sched_autotune(tb_sched s, int enable);
/* The choice for op `index` of the last execute (ncand = 0: not tuned) and the
 * timed candidates (up to cap). */
int tb_sched_tune_info(tb_sched s, int64_t index, int* mode, int* tile_n, int* ncand, int* cand_modes,
                       int* cand_tiles, double* cand_ms, int cap);

/* CUDA graph of the queued ops (no counterpart in TAMM): runs them once eagerly
 * (building plans, work lists and autotuner choices), then captures the same ops on
 * the context's stream.  tb_graph_launch enqueues one replay; tb_graph_sync waits
 * for it and checks the device error words of its split-INT8 contractions.  The
 * tensors the ops use must stay allocated while the graph exists; the graph keeps
 * the scratch its capture used. */
typedef struct tb_graph_s* tb_graph;
int tb_sched_graph_create(tb_sched s, tb_graph* out);
int tb_graph_launch(tb_graph g);
int tb_graph_sync(tb_graph g);
int tb_graph_destroy(tb_graph g);

/* ========================================================== DIFFERENTIATION === */

/* No counterpart in TAMM (it has no automatic differentiation).  A tape records
 * Functions that run eagerly on its own Scheduler, in the context's precision mode:
 *   Contract  y(Ly) = alpha * a(La) * b(Lb)
 *             backward: da(La) += alpha * dy(Ly) * b(Lb),  db(Lb) += alpha * a(La) * dy(Ly)
 *             (the dy-weighted contractions over the labels free in the other operand:
 *             TAMM's MultOp with swapped operands, multop.hpp:576-893);
 *   Dot       s = alpha * sum p(Lp) * q(Lq)  (same label set, any order)
 *             backward: dp += alpha * q,  dq += alpha * p  (AddOp, addop.hpp:242-271).
 * The objective is the sum of the Dot values.  tb_tape_backward accumulates its
 * gradient into the gradient tensors given for the leaves (zero them first; reset
 * the tape before recording the next evaluation).  Tensors that are neither leaves
 * nor Contract outputs are constants.  At the start of the backward sweep, Contract
 * outputs are kept in recording order while their total size fits budget_bytes;
 * the rest are freed and recomputed from their producer when the sweep needs their
 * values.  The tape holds plain references: destroy it before its tensors. */
typedef struct tb_tape_s* tb_tape;
int tb_tape_create(tb_ctx ctx, int64_t budget_bytes, tb_tape* out);
int tb_tape_destroy(tb_tape t);
/* Declares x a leaf whose gradient accumulates into grad (same spaces and spin mask;
 * NULL: x is a constant). */
int tb_tape_leaf(tb_tape t, tb_tensor x, tb_tensor grad);
/* Contract Function; y is an allocated tensor written once on this tape, labelled
 * over its full spaces.  An operand label summed inside that operand alone (whose
 * gradient would need a broadcast output) is TB_ERR_NOT_IMPLEMENTED. */
int tb_tape_contract(tb_tape t, tb_labeled y, double alpha, tb_labeled a, tb_labeled b);
/* Dot Function; *value (may be NULL) receives alpha * sum p * q. */
int tb_tape_dot(tb_tape t, double alpha, tb_labeled p, tb_labeled q, double* value);
int tb_tape_backward(tb_tape t);
/* Recorded Functions, objective (sum of the Dot values), bytes of Contract outputs
 * kept by the last backward sweep, and how many outputs it recomputed. */
int tb_tape_info(tb_tape t, int64_t* nnodes, double* objective, int64_t* kept_bytes,
                 int64_t* recomputed);
/* Forgets the recorded Functions and intermediate gradients (leaves stay declared);
 * outputs freed by the budget get their storage back. */
int tb_tape_reset(tb_tape t);

#ifdef __cplusplus
}
#endif
#endif
