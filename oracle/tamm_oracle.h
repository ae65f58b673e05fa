/*
 * TEST INFRASTRUCTURE ONLY — the oracle.
 *
 * A plain-C restatement of TAMM's block-sparse contraction path on the CPU, used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * Nothing in the tamm_b200 product links, loads or calls this code.
 *
 * Every function names the reference file:line it restates (paths relative to the
 * TAMM source tree).  Parity of this restatement is pinned against the reference's
 * own kernels::block_multiply / kernels::assign compiled from the TAMM sources
 * (oracle/Makefile -> oracle/_ref/) and against the reference tests' known answers.
 */
#ifndef TAMM_ORACLE_H
#define TAMM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAXR 8

/* Return codes. */
#define OR_OK 0
#define OR_EINVAL 1 /* malformed arguments (the reference's EXPECTS) */
#define OR_ENOTIMPL 2 /* the reference's NOT_IMPLEMENTED() */

/* kernels::assign (src/tamm/kernels/assign.hpp:467-485):
 * dst (=|+=) scale * src with labels mapping modes; permutations go through the
 * HPTT semantics (assign.hpp:375-401), everything else through ip_gen_loop
 * (assign.hpp:312-373). */
int or_assign(double* dst, const int64_t* ddims, const int* dlabels, int nd, double scale,
              const double* src, const int64_t* sdims, const int* slabels, int ns, int is_assign);

/* kernels::block_multiply, CPU branch, real x real -> real
 * (src/tamm/kernels/multiply.hpp:212-381). */
int or_block_multiply(double alpha, const double* abuf, const int64_t* adims, const int* alabels,
                      int na, const double* bbuf, const int64_t* bdims, const int* blabels, int nb,
                      double beta, double* cbuf, const int64_t* cdims, const int* clabels, int nc,
                      int is_assign);

/* TiledIndexSpaceInfo::construct_tiled_indices, uniform tile size
 * (src/tamm/tiled_index_space.hpp:1135-1194).  bounds = every lo/hi of the named
 * and spin ranges, in any order.  Writes tile start offsets followed by n into
 * out (capacity cap); returns the number written (ntiles + 1) or -1. */
int64_t or_tile_offsets_uniform(int64_t n, const int64_t* bounds, int nbounds, int64_t tile,
                                int64_t* out, int64_t cap);

/* TiledIndexSpaceInfo::construct_tiled_indices, explicit tile list
 * (src/tamm/tiled_index_space.hpp:1205-1262).  Returns ntiles + 1, or -1 when the
 * sizes do not add up to n or a boundary is not a tile start (the EXPECTS). */
int64_t or_tile_offsets_list(int64_t n, const int64_t* bounds, int nbounds, const int64_t* tiles,
                             int64_t ntiles, int64_t* out);

/* TensorBase::is_non_zero (src/tamm/tensor_base.hpp:243-263).
 * spins[i] = spin of the block's tile in mode i; mask[i] 0 upper, 1 lower, 2 ignore. */
int or_is_non_zero(int nmodes, const int* spins, const int* mask, int has_spin);

/* A block-sparse tensor stored as in Distribution_NW (src/tamm/distribution.hpp:197-285):
 * admitted blocks sorted by key = sum blockid[i] * prod_{j>i} ntiles[j], packed
 * contiguously, each block row-major in mode order. */
typedef struct or_tensor {
  int            nmodes;
  int            has_spin;
  int            spin_mask[OR_MAXR];
  int64_t        ntiles[OR_MAXR];
  const int64_t* tile_size[OR_MAXR];
  const int*     tile_spin[OR_MAXR];
  int64_t        nblocks;
  const int64_t* keys;    /* sorted ascending */
  const int64_t* offsets; /* element offset of each block */
  double*        data;
} or_tensor;

/* Distribution_NW constructor (distribution.hpp:201-243): enumerate admitted
 * blocks row-major, key them, sort by key and assign packed offsets.
 * keys/offsets need room for prod(ntiles) entries; returns the number of
 * admitted blocks and writes the total element count. */
int64_t or_nw_pack(or_tensor* t, int64_t* keys_out, int64_t* offsets_out, int64_t* total_out);

/* Distribution_NW::locate (distribution.hpp:270-285) on one process: element
 * offset of an admitted block, -1 when the block is not stored. */
int64_t or_nw_locate(const or_tensor* t, const int64_t* blockid);

/* One operand of a labelled expression: its tensor, the int label of each mode
 * (equal ints = same index label) and, per mode, the map from the label's tile
 * index to the tensor's tile index (internal::translate_blockid, utils.hpp:264-286;
 * NULL = identity) plus the number of tiles in the label's space. */
typedef struct or_operand {
  const or_tensor* t;
  int              labels[OR_MAXR];
  const int64_t*   tmap[OR_MAXR];
  int64_t          lntiles[OR_MAXR];
} or_operand;

/* MultOp::execute_bufacc on one process, CPU hardware
 * (src/tamm/multop.hpp:576-893): C += alpha * A * B over admitted output blocks x
 * admitted reduction tiles, each pair through or_block_multiply(beta=1,
 * is_assign=0) into a zeroed per-block buffer, then added into C. */
int or_mult_bufacc(or_operand* c, double alpha, const or_operand* a, const or_operand* b);

/* Same loop with a caller-chosen block kernel of or_block_multiply's signature (the
 * tests pass the reference's own kernels::block_multiply compiled in oracle/_ref). */
typedef int (*or_block_fn)(double, const double*, const int64_t*, const int*, int, const double*,
                           const int64_t*, const int*, int, double, double*, const int64_t*,
                           const int*, int, int);
int or_mult_bufacc_fn(or_operand* c, double alpha, const or_operand* a, const or_operand* b,
                      or_block_fn fn);

/* Counts the admitted (C, A, B) block triples and their FLOPs (2*|C|*K per triple,
 * with K the product of the reduction tile sizes), without computing. */
int or_mult_count(const or_operand* c, const or_operand* a, const or_operand* b,
                  int64_t* ntriples, double* flops);

/* SetOp over every stored element (src/tamm/setop.hpp:130-274): C = value, or
 * C += value when is_assign == 0. */
void or_set(or_tensor* t, double value, int is_assign);

/* tamm::norm (src/tamm/tamm_utils.hpp:1180-1200): sqrt of the sum of squares over
 * every stored element, in storage order. */
double or_norm(const or_tensor* t);

/* Seeded input generator shared by the tests: counter-based splitmix64 stream.
 * Uniform in [lo, hi) and normal(mean, sd) (Box-Muller) at element index i. */
double or_uniform(uint64_t seed, uint64_t i, double lo, double hi);
double or_normal(uint64_t seed, uint64_t i, double mean, double sd);
void   or_fill_uniform(double* x, int64_t n, uint64_t seed, uint64_t first, double lo, double hi);
void   or_fill_normal(double* x, int64_t n, uint64_t seed, uint64_t first, double mean, double sd);

#ifdef __cplusplus
}
#endif
#endif
